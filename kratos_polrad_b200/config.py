"""Plain configuration types of the C ABI (include/kp_transport.h).

Dataclasses for the mesh description (the reference's [mesh], [boundary]
and [refine_region*] keys) and the transport configuration, with the
ctypes mirrors of kp_transport_cfg_t, kp_source_t and kp_tallies_t.  This
module loads no library and needs no GPU, so that set-ups can be described
(and handed to other implementations of the path, such as the oracle's)
without the product library.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

c_int, c_ll, c_float, c_double, c_void_p, c_u32 = (ctypes.c_int, ctypes.c_longlong,
                                                   ctypes.c_float, ctypes.c_double,
                                                   ctypes.c_void_p, ctypes.c_uint32)


@dataclass
class RefineRegion:
    """One ``[refine_region*]`` section (meshgen.cpp:111-142)."""
    level: int
    x_min: tuple
    x_max: tuple


@dataclass
class MeshConfig:
    """The ``[mesh]`` / ``[boundary]`` / ``[refine_region*]`` keys."""
    x_min: tuple
    x_max: tuple
    n_cell_global: tuple
    n_cell_block: tuple = (16, 16, 16)
    periodic: tuple = (False, False, False)
    refine: list = field(default_factory=list)

    def to_ini(self) -> str:
        """INI text with the reference's section and key names."""
        f = lambda v: " ".join(repr(float(t)) for t in v)
        kinds = []
        for a in range(3):
            kinds += ["periodic", "periodic"] if self.periodic[a] else ["outflow", "outflow"]
        lines = ["[mesh]", f"x_min = {f(self.x_min)}", f"x_max = {f(self.x_max)}",
                 "n_cell_global = " + " ".join(str(int(v)) for v in self.n_cell_global),
                 "n_cell_block = " + " ".join(str(int(v)) for v in self.n_cell_block),
                 "", "[boundary]", "kinds = " + " ".join(kinds)]
        for k, r in enumerate(self.refine):
            lines += ["", f"[refine_region_{k:05d}]", f"level = {int(r.level)}",
                      f"x_min = {f(r.x_min)}", f"x_max = {f(r.x_max)}"]
        return "\n".join(lines) + "\n"



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
                ("lane_batch", c_int), ("flux_fx_shift", c_int), ("packets", c_void_p)]


class CTallies(ctypes.Structure):
    _fields_ = [("mu", c_void_p), ("image", c_void_p), ("image_batch", c_void_p),
                ("counters", c_void_p), ("records", c_void_p), ("flux", c_void_p),
                ("carry", c_void_p), ("flux_n", c_ll)]


# numpy view of kp_packet_record_t (88 bytes)
RECORD_DTYPE = np.dtype([("x", "<f8", 3), ("d", "<f4", 3), ("stokes", "<f4", 3), ("w", "<f4"),
                         ("ib", "<i4"), ("cell", "<i4", 3), ("n_scatter", "<i4"),
                         ("status", "<i4"), ("rng_draws", "<u4"), ("n_steps", "<i8")])
assert RECORD_DTYPE.itemsize == 88

# numpy view of kp_packet_init_t (64 bytes): a packet made by a user generator
PACKET_INIT_DTYPE = np.dtype([("x", "<f8", 3), ("d", "<f4", 3), ("w", "<f4"),
                              ("stokes", "<f4", 3), ("ib", "<i4"), ("peel_I", "<f4"),
                              ("pad", "<i4")])
assert PACKET_INIT_DTYPE.itemsize == 64

# numpy view of kp_packet_state_t (128 bytes): a packet carried between calls
# (suspended by a step budget, or a decomposed round's migrating walk)
PACKET_STATE_DTYPE = np.dtype([("x", "<f8", 3), ("d", "<f4", 3), ("e1", "<f4", 3),
                               ("stokes", "<f4", 3), ("w", "<f4"), ("tau", "<f4"),
                               ("ib", "<i4"), ("cell", "<i4", 3), ("n_scatter", "<i4"),
                               ("n_steps", "<i4"), ("stream_id", "<u4"), ("pid_lo", "<u4"),
                               ("pid_hi", "<u4"), ("rng_draws", "<u4"), ("batch", "<i4"),
                               ("pad", "<i4", 4)])
assert PACKET_STATE_DTYPE.itemsize == 128


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
    # the caller's packets (kp_packet_init_t records, [n_packets] of
    # PACKET_INIT_DTYPE): a device uint8 tensor [n_packets, 64] for the GPU,
    # or a host array of PACKET_INIT_DTYPE for the oracle; None: the sources
    packets: object = None

    def to_c(self):
        src = (CSource * max(1, len(self.sources)))()
        for k, s in enumerate(self.sources):
            src[k].kind, src[k].emit = int(s.kind), int(s.emit)
            for a in range(3):
                src[k].pos[a] = float(s.pos[a])
        c = CTransportCfg()
        for name, _ in CTransportCfg._fields_:
            if name in ("sources", "n_sources", "image_center", "packets"):
                continue
            setattr(c, name, getattr(self, name))
        if self.packets is not None:
            # the kernels read the table: it must be device memory
            if not getattr(self.packets, "is_cuda", False):
                raise ValueError("cfg.packets must be a CUDA tensor (transport.packet_table)")
            n = self.packets.numel() // 64
            if n < self.n_packets:
                raise ValueError(f"packet table holds {n} packets, the call {self.n_packets}")
            c.packets = self.packets.data_ptr()
        c.n_sources = len(self.sources)
        c.sources = ctypes.cast(src, ctypes.POINTER(CSource))
        for a in range(3):
            c.image_center[a] = float(self.image_center[a])
        c._keep = src
        return c
