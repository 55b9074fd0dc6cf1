"""Polarized Monte-Carlo transport (host mirror of ``kp_transport_forward``).

One call replaces one cycle of the reference's particle module: the
generator launch and the integrator launch that walks every packet
(modules/particle/driver.h:59-79, evolve/generate_par.h:51-62,
evolve/integrator.h:47-63), extended with the physics that the reference
leaves to its ``proc_phys``/``proc_step`` hooks (radiation/photon.h:73-102).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr

c_int, c_ll, c_float, c_double, c_void_p, c_u32 = (ctypes.c_int, ctypes.c_longlong,
                                                   ctypes.c_float, ctypes.c_double,
                                                   ctypes.c_void_p, ctypes.c_uint32)

PHASE_RAYLEIGH, PHASE_HG_POL = 0, 1
SOURCE_POINT, SOURCE_PLANE_BASE = 0, 1
EMIT_ISOTROPIC, EMIT_UP_UNIFORM = 0, 1
TALLY_FIXED, TALLY_FLOAT = 0, 1
MAX_SOURCES, MAX_BATCHES = 64, 64
COUNTERS = ("steps", "peel_steps", "scatter", "escaped", "absorbed", "capped", "lost",
            "emitted", "hops", "deposits")


class CSource(ctypes.Structure):
    _fields_ = [("kind", c_int), ("emit", c_int), ("pos", c_double * 3)]


class CTransportCfg(ctypes.Structure):
    _fields_ = [("n_packets", c_ll), ("packet_offset", c_ll), ("seed", c_u32),
                ("stream_id", c_u32), ("phase", c_int), ("hg_g", c_float),
                ("pol_max", c_float), ("n_sources", c_int), ("sources", ctypes.POINTER(CSource)),
                ("n_mu_bins", c_int), ("mu_lo", c_float), ("mu_hi", c_float),
                ("image_n", c_int), ("inclination_deg", c_double), ("azimuth_deg", c_double),
                ("image_center", c_double * 3), ("image_half_width", c_double),
                ("tau_peel_max", c_float), ("tally_mode", c_int), ("fx_shift", c_int),
                ("n_batches", c_int), ("image_batch_n", c_int), ("w_min", c_float),
                ("rr_survive", c_float),
                ("max_scatter", c_int), ("max_steps", c_ll), ("n_record", c_ll),
                ("lane_batch", c_int), ("flux_fx_shift", c_int)]


class CTallies(ctypes.Structure):
    _fields_ = [("mu", c_void_p), ("image", c_void_p), ("image_batch", c_void_p),
                ("counters", c_void_p), ("records", c_void_p), ("flux", c_void_p)]


# numpy view of kp_packet_record_t (88 bytes)
RECORD_DTYPE = np.dtype([("x", "<f8", 3), ("d", "<f4", 3), ("stokes", "<f4", 3), ("w", "<f4"),
                         ("ib", "<i4"), ("cell", "<i4", 3), ("n_scatter", "<i4"),
                         ("status", "<i4"), ("rng_draws", "<u4"), ("n_steps", "<i8")])
assert RECORD_DTYPE.itemsize == 88

_lib.register("kp_transport_forward", [c_void_p, ctypes.POINTER(CTransportCfg),
                                       ctypes.POINTER(CTallies), c_void_p])


@dataclass
class Source:
    kind: int = SOURCE_POINT
    emit: int = EMIT_ISOTROPIC
    pos: tuple = (0.0, 0.0, 0.0)


@dataclass
class TransportConfig:
    """Python form of ``kp_transport_cfg_t`` (see include/kp_transport.h)."""
    n_packets: int
    sources: list
    seed: int = 1
    stream_id: int = 0
    packet_offset: int = 0
    phase: int = PHASE_RAYLEIGH
    hg_g: float = 0.0
    pol_max: float = 1.0
    n_mu_bins: int = 0
    mu_lo: float = 0.0
    mu_hi: float = 1.0
    image_n: int = 0
    inclination_deg: float = 90.0
    azimuth_deg: float = 0.0
    image_center: tuple = (0.0, 0.0, 0.0)
    image_half_width: float = 1.0
    tau_peel_max: float = 40.0
    tally_mode: int = TALLY_FIXED
    fx_shift: int = 32
    n_batches: int = 32
    image_batch_n: int = 1
    w_min: float = 0.0
    rr_survive: float = 0.1
    max_scatter: int = 100000
    max_steps: int = 1 << 24
    n_record: int = 0
    lane_batch: int = 0
    flux_fx_shift: int = 24
    # Python side only: keep the per-cell path-length flux tally (rad_t::flx)
    flux: bool = False

    def to_c(self):
        src = (CSource * max(1, len(self.sources)))()
        for k, s in enumerate(self.sources):
            src[k].kind, src[k].emit = int(s.kind), int(s.emit)
            for a in range(3):
                src[k].pos[a] = float(s.pos[a])
        c = CTransportCfg()
        for name, _ in CTransportCfg._fields_:
            if name in ("sources", "n_sources", "image_center"):
                continue
            setattr(c, name, getattr(self, name))
        c.n_sources = len(self.sources)
        c.sources = ctypes.cast(src, ctypes.POINTER(CSource))
        for a in range(3):
            c.image_center[a] = float(self.image_center[a])
        c._keep = src
        return c


class Tallies:
    """Device output buffers of a transport run (accumulated across calls).

    ``n_cells`` sizes the path-length flux tally when ``cfg.flux`` is set
    (the mesh's cell count; a decomposed rank's own cells).
    """

    def __init__(self, cfg: TransportConfig, device="cuda", n_cells: int = 0):
        dt = torch.int64 if cfg.tally_mode == TALLY_FIXED else torch.float32
        self.cfg = cfg
        self.mu = torch.zeros((cfg.n_batches, max(cfg.n_mu_bins, 1), 4), dtype=dt, device=device)
        n = max(cfg.image_n, 1)
        self.image = torch.zeros((n, n, 4), dtype=dt, device=device)
        bn = max(cfg.image_batch_n, 1)
        self.image_batch = torch.zeros((cfg.n_batches, bn, bn, 4), dtype=dt, device=device)
        self.counters = torch.zeros(len(COUNTERS), dtype=torch.int64, device=device)
        self.records = (torch.zeros((max(cfg.n_record, 1), 88), dtype=torch.uint8, device=device)
                        if cfg.n_record else None)
        if cfg.flux and n_cells <= 0:
            raise ValueError("the flux tally needs the mesh's cell count (n_cells)")
        self.flux = torch.zeros(n_cells, dtype=dt, device=device) if cfg.flux else None

    def zero_(self):
        for t in (self.mu, self.image, self.image_batch, self.counters):
            t.zero_()
        if self.flux is not None:
            self.flux.zero_()
        if self.records is not None:
            self.records.zero_()
        return self

    def to_c(self):
        t = CTallies()
        t.mu = ptr(self.mu) if self.cfg.n_mu_bins else None
        t.image = ptr(self.image) if self.cfg.image_n else None
        t.image_batch = ptr(self.image_batch) if self.cfg.image_n else None
        t.counters = ptr(self.counters)
        t.records = ptr(self.records) if self.records is not None else None
        t.flux = ptr(self.flux) if self.flux is not None else None
        return t

    def scale(self) -> float:
        return 2.0 ** -self.cfg.fx_shift if self.cfg.tally_mode == TALLY_FIXED else 1.0

    def flux_scale(self) -> float:
        """Factor that turns the flux tally into w * dl / volume sums."""
        if self.cfg.tally_mode != TALLY_FIXED:
            return 1.0
        return 2.0 ** -(self.cfg.flux_fx_shift or self.cfg.fx_shift)

    def flux_values(self) -> np.ndarray:
        """Flux tally as float64 sums of w * dl / volume per cell."""
        return self.flux.cpu().numpy().astype(np.float64) * self.flux_scale()

    def counts(self) -> dict:
        c = self.counters.cpu().numpy()
        return {k: int(v) for k, v in zip(COUNTERS, c)}

    def record_array(self) -> np.ndarray:
        return self.records.cpu().numpy().view(RECORD_DTYPE).reshape(-1)


def forward(mesh, cfg: TransportConfig, tallies: Tallies | None = None,
            stream: int | None = None, tape: bool = False) -> Tallies:
    """Runs ``cfg.n_packets`` packets through ``mesh``; returns the tallies.

    With ``tape`` the mesh also keeps the solve's peel-off rays for a later
    ``adjoint(..., tape_id=tallies.tape_id)``; ``tallies.tape_id`` is 0 when
    the solve was too large to tape (more packets than one queue chunk).
    """
    if tallies is None:
        tallies = Tallies(cfg, n_cells=mesh.n_cells if cfg.flux else 0)
    c, t = cfg.to_c(), tallies.to_c()
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    tallies.tape_id = 0
    if tape:
        tid = ctypes.c_longlong(0)
        call("kp_transport_forward_tape", mesh.handle, ctypes.byref(c), ctypes.byref(t), s,
             ctypes.byref(tid))
        tallies.tape_id = tid.value
    else:
        call("kp_transport_forward", mesh.handle, ctypes.byref(c), ctypes.byref(t), s)
    return tallies


def polarization(I, Q, U):
    """Linear polarization fraction sqrt(Q^2+U^2)/I."""
    I = np.asarray(I, np.float64)
    return np.sqrt(np.asarray(Q, np.float64) ** 2 + np.asarray(U, np.float64) ** 2) / np.where(I == 0, 1, I)


def batch_std_error(batch_iqu: np.ndarray) -> tuple[float, float]:
    """Polarization fraction and its relative std-error from batch sums.

    ``batch_iqu``: [n_batches, >=3] per-batch (I, Q, U) sums; each batch is an
    independent packet subset, so the spread of per-batch fractions gives the
    error of their mean (batch means).
    """
    b = np.asarray(batch_iqu, np.float64)
    p_b = polarization(b[:, 0], b[:, 1], b[:, 2])
    tot = b.sum(0)
    p = float(polarization(tot[0], tot[1], tot[2]))
    err = float(np.std(p_b, ddof=1) / math.sqrt(len(p_b)))
    return p, (err / p if p > 0 else float("inf"))
