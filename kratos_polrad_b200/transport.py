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

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .config import (COUNTERS, EMIT_ISOTROPIC, EMIT_UP_UNIFORM, MAX_BATCHES,  # noqa: F401
                     MAX_SOURCES, PACKET_INIT_DTYPE, PACKET_STATE_DTYPE, PHASE_HG_POL,
                     PHASE_RAYLEIGH, RECORD_DTYPE, SOURCE_PLANE_BASE, SOURCE_POINT, TALLY_FIXED,
                     TALLY_FLOAT, CSource, CTallies, CTransportCfg, Source, TransportConfig)

_lib.register("kp_transport_forward", [ctypes.c_void_p, ctypes.POINTER(CTransportCfg),
                                       ctypes.POINTER(CTallies), ctypes.c_void_p])


class CResume(ctypes.Structure):
    """ctypes mirror of kp_resume_t."""
    _fields_ = [("in_", ctypes.c_void_p), ("n_in", ctypes.c_longlong),
                ("out", ctypes.c_void_p), ("cap_out", ctypes.c_longlong),
                ("out_count", ctypes.c_void_p), ("step_budget", ctypes.c_int)]


_lib.register("kp_transport_forward_resume", [ctypes.c_void_p, ctypes.POINTER(CTransportCfg),
                                              ctypes.POINTER(CResume), ctypes.POINTER(CTallies),
                                              ctypes.c_void_p])


class Tallies:
    """Device output buffers of a transport run (accumulated across calls).

    ``n_cells`` sizes the path-length flux tally when ``cfg.flux`` is set
    (the mesh's cell count; a decomposed rank's own cells).  In float mode
    the tallies come with their rounding-error carry (kp_tallies_t::carry),
    which each solve folds into them at its end; ``carry=False`` leaves plain
    float atomics.
    """

    def __init__(self, cfg: TransportConfig, device="cuda", n_cells: int = 0, carry: bool = True):
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
        n_carry = 0
        if cfg.image_n:
            n_carry += self.image.numel() + self.image_batch.numel()
        if cfg.n_mu_bins:
            n_carry += self.mu.numel()
        if self.flux is not None:
            n_carry += self.flux.numel()
        self.carry = (torch.zeros(max(n_carry, 1), dtype=torch.float32, device=device)
                      if carry and cfg.tally_mode == TALLY_FLOAT else None)

    def zero_(self):
        for t in (self.mu, self.image, self.image_batch, self.counters):
            t.zero_()
        for t in (self.flux, self.carry):
            if t is not None:
                t.zero_()
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
        t.flux_n = self.flux.numel() if self.flux is not None else 0
        t.carry = ptr(self.carry) if self.carry is not None else None
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


def forward_resume(mesh, cfg: TransportConfig, step_budget: int, resumed=None,
                   tallies: Tallies | None = None, capacity: int | None = None,
                   stream: int | None = None):
    """One call with a per-call step budget (``kp_transport_forward_resume``).

    Resumes the packets in ``resumed`` (a device uint8 tensor [n, 128] of
    kp_packet_state_t, as returned by an earlier call), then emits
    ``cfg.n_packets`` new ones; every packet walks at most ``step_budget``
    segments in this call.  Returns ``(tallies, suspended)``: the packets
    that used up their budget, for the next call (``PACKET_STATE_DTYPE``
    views them).  ``capacity`` bounds the suspended queue (default: every
    packet of the call); an overflow raises.
    """
    if tallies is None:
        tallies = Tallies(cfg, n_cells=mesh.n_cells if cfg.flux else 0)
    dev = tallies.counters.device
    if resumed is not None and not (resumed.dtype == torch.uint8 and resumed.dim() == 2
                                    and resumed.shape[1] == PACKET_STATE_DTYPE.itemsize
                                    and resumed.is_contiguous() and resumed.device == dev):
        raise ValueError("resumed must be a contiguous uint8 [n, 128] tensor of packet states "
                         "on the tallies' device")
    n_in = 0 if resumed is None else int(resumed.shape[0])
    cap = n_in + cfg.n_packets if capacity is None else int(capacity)
    out = torch.empty((max(cap, 1), PACKET_STATE_DTYPE.itemsize), dtype=torch.uint8, device=dev)
    count = torch.zeros(1, dtype=torch.int64, device=dev)
    r = CResume()
    r.in_ = ptr(resumed) if n_in else None
    r.n_in = n_in
    r.out = ptr(out)
    r.cap_out = cap
    r.out_count = ptr(count)
    r.step_budget = int(step_budget)
    c, t = cfg.to_c(), tallies.to_c()
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    call("kp_transport_forward_resume", mesh.handle, ctypes.byref(c), ctypes.byref(r),
         ctypes.byref(t), s)
    n_out = int(count.item())
    if n_out > cap:
        raise RuntimeError(f"{n_out} packets suspended, the queue holds {cap}")
    return tallies, out[:n_out]


def packet_states(suspended: torch.Tensor) -> np.ndarray:
    """Host view (PACKET_STATE_DTYPE) of a queue of suspended packets."""
    return suspended.cpu().numpy().view(PACKET_STATE_DTYPE).reshape(-1)


def packet_array(x, d, w=1.0, stokes=None, ib=-1, peel_I=0.0) -> np.ndarray:
    """Host array of kp_packet_init_t records (PACKET_INIT_DTYPE): positions
    x [n, 3], unit directions d [n, 3], weights w, Stokes (q, u, v) relative
    to the packet's frame (default unpolarized), block ids (-1: located on the
    device) and the emission's intensity per steradian toward the observer
    per unit weight (0: no peel-off ray at emission)."""
    x = np.asarray(x, np.float64).reshape(-1, 3)
    a = np.zeros(len(x), PACKET_INIT_DTYPE)
    a["x"] = x
    a["d"] = np.asarray(d, np.float32).reshape(-1, 3)
    a["w"] = w
    if stokes is not None:
        a["stokes"] = np.asarray(stokes, np.float32).reshape(-1, 3)
    a["ib"] = ib
    a["peel_I"] = peel_I
    return a


def packet_table(records: np.ndarray, device="cuda") -> torch.Tensor:
    """Device copy ([n, 64] uint8) of packet_array records, for cfg.packets."""
    return torch.from_numpy(np.ascontiguousarray(records).view(np.uint8).reshape(-1, 64)).to(device)


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
