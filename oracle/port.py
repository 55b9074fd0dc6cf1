"""ctypes driver of the C restatement (oracle/_ref/libkporacle.so).

Test infrastructure only.  The walk consumes flat block tables, either the
reference harness's (refharness.RefMesh) or the product's (kp_mesh_*).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libkporacle.so")
LIB64 = os.path.join(_HERE, "_ref", "libkporacle64.so")   # every float in double


class _Mesh(ctypes.Structure):
    _fields_ = [("n_blocks", ctypes.c_int), ("nc", ctypes.c_int * 3),
                ("xf0", ctypes.c_void_p), ("dx0", ctypes.c_void_p), ("vol0", ctypes.c_void_p),
                ("phybnd", ctypes.c_void_p), ("nb_id", ctypes.c_void_p),
                ("nb_shift", ctypes.c_void_p), ("d_lvl", ctypes.c_void_p),
                ("periodic", ctypes.c_int * 3), ("xlim", ctypes.c_double * 6),
                ("lbox", ctypes.c_double * 3)]


_lib = None
_lib64 = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise FileNotFoundError(f"{LIB} missing: run `make -C oracle`")
        _lib = ctypes.CDLL(LIB)
    return _lib


def lib64():
    """The FP64 build of the restatement (exports with a _f64 suffix)."""
    global _lib64
    if _lib64 is None:
        if not os.path.exists(LIB64):
            raise FileNotFoundError(f"{LIB64} missing: run `make -C oracle`")
        _lib64 = ctypes.CDLL(LIB64)
    return _lib64


def available() -> bool:
    return os.path.exists(LIB)


class Tables:
    """Flat tables (block-id order) of a mesh for one float_t precision."""

    def __init__(self, nc, xf0, dx0, vol0, phybnd, nb_id, nb_shift, d_lvl, periodic, xlim, lbox):
        c = lambda a, t: np.ascontiguousarray(a, t)
        self.nc = tuple(int(v) for v in nc)
        self.xf0, self.dx0, self.vol0 = c(xf0, np.float64), c(dx0, np.float64), c(vol0, np.float64)
        self.phybnd, self.nb_id = c(phybnd, np.int32), c(nb_id, np.int32)
        self.nb_shift, self.d_lvl = c(nb_shift, np.int32), c(d_lvl, np.int32)
        self.periodic = [int(v) for v in periodic]
        self.xlim = np.asarray(xlim, np.float64).reshape(2, 3)
        self.lbox = np.asarray(lbox, np.float64)
        self.n_blocks = len(self.vol0)
        self.cells_per_block = int(np.prod(self.nc))

    @classmethod
    def from_ref(cls, ref):
        xf0, dx0, vol0, pb = ref.geometry()
        ids, sh, dl = ref.neighbors()
        xlim, lbox, per = ref.box()
        return cls(ref.nc, xf0, dx0, vol0, pb, ids, sh, dl, per, xlim, lbox)

    @classmethod
    def from_mesh(cls, mesh, precision):
        xf0, dx0, vol0, pb = mesh.geometry(precision)
        ids, sh, dl = mesh.neighbors()
        xlim = np.array([mesh.x_min, mesh.x_max])
        lbox = xlim[1] - xlim[0]
        if precision == 4:
            xlim = xlim.astype(np.float32).astype(np.float64)
            lbox = lbox.astype(np.float32).astype(np.float64)
        return cls(mesh.nc, xf0, dx0, vol0, pb, ids, sh, dl, mesh.periodic, xlim, lbox)

    def _struct(self):
        s = _Mesh()
        s.n_blocks = self.n_blocks
        for a in range(3):
            s.nc[a] = self.nc[a]
            s.periodic[a] = self.periodic[a]
            s.lbox[a] = self.lbox[a]
        for k, v in enumerate(self.xlim.reshape(-1)):
            s.xlim[k] = v
        for f in ("xf0", "dx0", "vol0", "phybnd", "nb_id", "nb_shift", "d_lvl"):
            setattr(s, f, getattr(self, f).ctypes.data)
        return s


def trace(tab: Tables, precision: int, x, dir, cell, ib, proper, steps, fx_shift=32, todo=None):
    """Restated cart_t::proc walk; returns final state, both flux sums and,
    per packet, the number of cached-face shifts of geo_loc_t::fix that left
    the cell index behind (``fix``)."""
    n = len(ib)
    x = np.array(x, np.float64).reshape(n, 3)
    dir = np.ascontiguousarray(dir, np.float64).reshape(n, 3)
    cell = np.array(cell, np.int32).reshape(n, 3)
    ib = np.array(ib, np.int32)
    proper = np.ascontiguousarray(proper, np.float64)
    steps = np.array(steps, np.int32)
    todo = np.full(n, -2, np.int32) if todo is None else np.array(todo, np.int32)
    ncell = tab.n_blocks * tab.cells_per_block
    flux_f, flux_fx = np.zeros(ncell), np.zeros(ncell, np.int64)
    fix = np.zeros(n, np.int32)
    s = tab._struct()
    L = lib()
    L.kpo_trace_ex.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_long] + \
        [ctypes.c_void_p] * 7 + [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    p = lambda a: a.ctypes.data
    st = L.kpo_trace_ex(ctypes.byref(s), precision, n, p(x), p(dir), p(cell), p(ib), p(proper),
                        p(steps), p(todo), fx_shift, p(flux_f), p(flux_fx), p(fix))
    if st != 0:
        raise RuntimeError("kpo_trace: bad block id")
    return dict(x=x, cell=cell, ib=ib, step=steps, todo=todo, flux=flux_f, flux_fx=flux_fx,
                fix=fix)


# ---------------------------------------------------------------------------
# Polarized transport restatement (kpo_transport)

class _Source(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("emit", ctypes.c_int), ("pos", ctypes.c_double * 3),
                ("ib", ctypes.c_int), ("cell", ctypes.c_int * 3)]


class _Cfg(ctypes.Structure):
    _fields_ = [("n_packets", ctypes.c_longlong), ("packet_offset", ctypes.c_longlong),
                ("seed", ctypes.c_uint32), ("stream_id", ctypes.c_uint32), ("phase", ctypes.c_int),
                ("hg_g", ctypes.c_float), ("pol_max", ctypes.c_float), ("n_sources", ctypes.c_int),
                ("sources", ctypes.POINTER(_Source)), ("n_mu_bins", ctypes.c_int),
                ("mu_lo", ctypes.c_float), ("mu_hi", ctypes.c_float), ("image_n", ctypes.c_int),
                ("inclination_deg", ctypes.c_double), ("azimuth_deg", ctypes.c_double),
                ("image_center", ctypes.c_double * 3), ("image_half_width", ctypes.c_double),
                ("tau_peel_max", ctypes.c_float), ("fx_shift", ctypes.c_int),
                ("n_batches", ctypes.c_int), ("image_batch_n", ctypes.c_int),
                ("w_min", ctypes.c_float), ("rr_survive", ctypes.c_float),
                ("max_scatter", ctypes.c_int), ("max_steps", ctypes.c_longlong),
                ("n_record", ctypes.c_longlong), ("flux_fx_shift", ctypes.c_int),
                ("packets", ctypes.c_void_p)]


def _cfg_struct(cfg, src):
    """kpo_cfg_t of a TransportConfig-like cfg; a packet table (cfg.packets,
    records of kp_packet_init_t's layout, host or device) is copied to the
    host and kept alive by the struct."""
    c = _Cfg()
    for name, _ in _Cfg._fields_:
        if name in ("sources", "n_sources", "image_center", "packets"):
            continue
        setattr(c, name, getattr(cfg, name, 0))
    c.n_sources = len(cfg.sources)
    c.sources = ctypes.cast(src, ctypes.POINTER(_Source))
    for a in range(3):
        c.image_center[a] = float(cfg.image_center[a])
    pk = getattr(cfg, "packets", None)
    if pk is not None:
        if hasattr(pk, "cpu"):
            pk = pk.cpu().numpy()
        pk = np.ascontiguousarray(pk).view(np.uint8).reshape(-1)
        if pk.size < 64 * cfg.n_packets:
            raise ValueError("packet table shorter than n_packets")
        c.packets = pk.ctypes.data
        c._keep = pk
    return c


def lookup_grid(levels, regs, nc_root_blocks):
    """Finest-level leaf lookup built from the blocks' region keys."""
    L = int(levels.max())
    n = [int(v) << L for v in nc_root_blocks]
    g = np.full((n[2], n[1], n[0]), -1, np.int32)
    for b, (lev, r) in enumerate(zip(levels, regs)):
        f = 1 << (L - int(lev))
        g[r[2] * f:(r[2] + 1) * f, r[1] * f:(r[1] + 1) * f, r[0] * f:(r[0] + 1) * f] = b
    return g, n


def transport(tab: Tables, sigma2, lookup, lookup_n, cfg, source_cells, flux=False,
              deposits=0):
    """Runs the restated transport for a TransportConfig-like ``cfg``.

    ``source_cells``: (ib, cell[3]) per source (point sources), located by
    the caller.  Returns dict of int64 tallies, counters and records; with
    ``flux`` also the int64 path-length flux tally ([n_cells]); with
    ``deposits`` = cap > 0 also "deposits": (pixel [k] int32, (I, Q, U, V)
    [k, 4] float32) of the first cap image deposits in deposit order, and
    "n_deposits", the count of all of them.
    """
    src = (_Source * max(1, len(cfg.sources)))()
    for k, s in enumerate(cfg.sources):
        src[k].kind, src[k].emit = int(s.kind), int(s.emit)
        for a in range(3):
            src[k].pos[a] = float(s.pos[a])
        ib, cell = source_cells[k]
        src[k].ib = int(ib)
        for a in range(3):
            src[k].cell[a] = int(cell[a])
    c = _cfg_struct(cfg, src)
    nm = max(cfg.n_mu_bins, 1)
    ni = max(cfg.image_n, 1)
    out = dict(mu=np.zeros((cfg.n_batches, nm, 4), np.int64),
               image=np.zeros((ni, ni, 4), np.int64),
               image_batch=np.zeros((cfg.n_batches, max(cfg.image_batch_n, 1),
                                     max(cfg.image_batch_n, 1), 4), np.int64),
               counters=np.zeros(10, np.uint64))
    from kratos_polrad_b200.transport import RECORD_DTYPE
    rec = np.zeros(max(cfg.n_record, 1), RECORD_DTYPE)
    sigma2 = np.ascontiguousarray(sigma2, np.float32)
    lookup = np.ascontiguousarray(lookup, np.int32)
    lk_n = np.ascontiguousarray(lookup_n, np.int32)
    s = tab._struct()
    L = lib()
    if flux:
        out["flux"] = np.zeros(tab.n_blocks * tab.cells_per_block, np.int64)
    L.kpo_transport.argtypes = [ctypes.c_void_p] * 11
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    if deposits:
        d_pix, d_val = np.zeros(deposits, np.int32), np.zeros((deposits, 4), np.float32)
        d_n = np.zeros(1, np.int64)
        L.kpo_set_pixel_sink.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong,
                                         ctypes.c_void_p]
        L.kpo_set_pixel_sink(p(d_pix), p(d_val), deposits, p(d_n))
    try:
        st = L.kpo_transport(ctypes.byref(s), p(sigma2), p(lookup), p(lk_n), ctypes.byref(c),
                             p(out["mu"]), p(out["image"]), p(out["image_batch"]),
                             p(out["counters"]), p(rec), p(out["flux"]) if flux else None)
    finally:
        if deposits:
            L.kpo_set_pixel_sink(None, None, 0, None)
    if st != 0:
        raise RuntimeError(f"kpo_transport failed ({st})")
    if deposits:
        k = int(min(d_n[0], deposits))
        out["deposits"] = (d_pix[:k], d_val[:k])
        out["n_deposits"] = int(d_n[0])
    out["records"] = rec[:cfg.n_record]
    return out


def adjoint(tab: Tables, sigma2, lookup, lookup_n, cfg, source_cells, adj_img, grad_shift=24,
            abs_sum=False, fp64=False):
    """Restated path-replay adjoint; returns int64 (g_len, g_int), counters,
    and with ``abs_sum`` also the per-cell sum of |deposit| over both
    tallies and the per-cell deposit count ([n_cells, 2] float64).  With
    ``fp64`` the FP64 build runs it (every float quantity in double)."""
    src = (_Source * max(1, len(cfg.sources)))()
    for k, s in enumerate(cfg.sources):
        src[k].kind, src[k].emit = int(s.kind), int(s.emit)
        for a in range(3):
            src[k].pos[a] = float(s.pos[a])
        ib, cell = source_cells[k]
        src[k].ib = int(ib)
        for a in range(3):
            src[k].cell[a] = int(cell[a])
    c = _cfg_struct(cfg, src)
    n_cells = tab.n_blocks * tab.cells_per_block
    g_len, g_int = np.zeros(n_cells, np.int64), np.zeros(n_cells, np.int64)
    cnt = np.zeros(10, np.uint64)
    ftype = np.float64 if fp64 else np.float32
    sigma2 = np.ascontiguousarray(sigma2, np.float32).astype(ftype)
    lookup = np.ascontiguousarray(lookup, np.int32)
    lk_n = np.ascontiguousarray(lookup_n, np.int32)
    adj = np.ascontiguousarray(adj_img, np.float32).astype(ftype)
    s = tab._struct()
    L = lib64() if fp64 else lib()
    sfx = "_f64" if fp64 else ""
    f_adj, f_sink = getattr(L, "kpo_adjoint" + sfx), getattr(L, "kpo_set_abs_sink" + sfx)
    f_adj.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_int] + [ctypes.c_void_p] * 3
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    sink = np.zeros((n_cells, 2), np.float64) if abs_sum else None
    f_sink.argtypes = [ctypes.c_void_p]
    f_sink(p(sink) if abs_sum else None)
    try:
        st = f_adj(ctypes.byref(s), p(sigma2), p(lookup), p(lk_n), ctypes.byref(c),
                   p(adj), grad_shift, p(g_len), p(g_int), p(cnt))
    finally:
        f_sink(None)
    if st != 0:
        raise RuntimeError(f"kpo_adjoint failed ({st})")
    return (g_len, g_int, cnt, sink) if abs_sum else (g_len, g_int, cnt)
