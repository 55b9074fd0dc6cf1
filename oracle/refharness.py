"""ctypes driver of oracle/_ref/libkpref_p{1,2}.so (reference code on the host).

Test infrastructure only.  See ref_harness.cpp for what is the reference's
code and what the harness restates.
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")


def available(precision: int = 1) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libkpref_p{precision}.so"))


def _p(a):
    return ctypes.c_void_p(0 if a is None else a.ctypes.data)


class RefMesh:
    """Mesh built by the reference's tree/meshgen/proxy code from INI text."""

    _libs: dict = {}

    @classmethod
    def _lib_for(cls, precision):
        if precision not in cls._libs:
            path = os.path.join(REF_DIR, f"libkpref_p{precision}.so")
            if not os.path.exists(path):
                raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
            cls._libs[precision] = ctypes.CDLL(path)
        return cls._libs[precision]

    _loader = "kpref_mesh_load"

    def __init__(self, ini_text: str, precision: int = 1):
        self.lib = L = self._lib_for(precision)
        self.precision = precision
        self.ftype = np.float32 if precision == 1 else np.float64
        with tempfile.NamedTemporaryFile("w", suffix=".ini", delete=False) as f:
            f.write(ini_text)
            path = f.name
        try:
            n = getattr(L, self._loader)(path.encode())
        finally:
            os.unlink(path)
        if n < 0:
            raise RuntimeError("reference harness rejected the mesh")
        self.n_blocks = n
        nc = np.zeros(3, np.int32)
        self.cells_per_block = L.kpref_block_cells(_p(nc))
        self.nc = tuple(int(v) for v in nc)
        self.n_cells = n * self.cells_per_block

    def blocks(self):
        lev = np.zeros(self.n_blocks, np.int32)
        reg = np.zeros((self.n_blocks, 3), np.int32)
        self.lib.kpref_blocks(_p(lev), _p(reg))
        return lev, reg

    def geometry(self):
        nb = self.n_blocks
        xf0, dx0, vol0 = np.zeros((nb, 3)), np.zeros((nb, 3)), np.zeros(nb)
        pb = np.zeros((nb, 6), np.int32)
        self.lib.kpref_geo(_p(xf0), _p(dx0), _p(vol0), _p(pb))
        return xf0, dx0, vol0, pb

    def neighbors(self):
        nb = self.n_blocks
        ids = np.zeros((nb, 24), np.int32)
        sh = np.zeros((nb, 48), np.int32)
        dl = np.zeros((nb, 6), np.int32)
        self.lib.kpref_nb(_p(ids), _p(sh), _p(dl))
        return ids, sh, dl

    def box(self):
        xlim, lbox, per = np.zeros(6), np.zeros(3), np.zeros(3, np.int32)
        self.lib.kpref_box(_p(xlim), _p(lbox), _p(per))
        return xlim.reshape(2, 3), lbox, per

    def trace(self, x, dir, cell, ib, proper, steps, fx_shift=32, n_threads=1):
        """Runs cart_t<>::proc for every packet; returns final state + flux."""
        n = len(ib)
        x = np.ascontiguousarray(x, np.float64).reshape(n, 3)
        dir = np.ascontiguousarray(dir, np.float64).reshape(n, 3)
        cell = np.ascontiguousarray(cell, np.int32).reshape(n, 3)
        ib = np.ascontiguousarray(ib, np.int32)
        proper = np.ascontiguousarray(proper, np.float64)
        steps = np.ascontiguousarray(steps, np.int32)
        out = dict(x=np.zeros((n, 3)), cell=np.zeros((n, 3), np.int32),
                   ib=np.zeros(n, np.int32), step=np.zeros(n, np.int32),
                   todo=np.zeros(n, np.int32), flux=np.zeros(self.n_cells),
                   flux_fx=np.zeros(self.n_cells, np.int64))
        self.lib.kpref_trace.argtypes = [ctypes.c_long] + [ctypes.c_void_p] * 6 + \
            [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 7
        st = self.lib.kpref_trace(n, _p(x), _p(dir), _p(cell), _p(ib), _p(proper), _p(steps),
                                  fx_shift, n_threads, _p(out["x"]), _p(out["cell"]),
                                  _p(out["ib"]), _p(out["step"]), _p(out["todo"]),
                                  _p(out["flux"]), _p(out["flux_fx"]))
        if st != 0:
            raise RuntimeError("kpref_trace failed")
        return out


def deposits_outside(precision: int) -> int:
    """Reference deposits skipped since the last call because their cell lay
    beyond the flux pool (the spherical walk after some corner crossings)."""
    L = RefMesh._lib_for(precision)
    L.kpref_deposits_outside.restype = ctypes.c_longlong
    return int(L.kpref_deposits_outside())


class RefMeshSph(RefMesh):
    """Spherical-polar mesh built by the reference's meshgen::sph_t; axes
    (r, theta, phi); [mesh] r_ratio sets the radial spacing."""

    _loader = "kpref_mesh_load_sph"

    def geometry_sph(self):
        """(radial faces [nb, nc0 + 1], cell volumes [n_cells]) as float_t."""
        rf = np.zeros((self.n_blocks, self.nc[0] + 1))
        vol = np.zeros(self.n_cells)
        if self.lib.kpref_geo_sph(_p(rf), _p(vol)) != 0:
            raise RuntimeError("kpref_geo_sph failed")
        return rf, vol

    def trace(self, x, x_car, dir, cell, ib, proper, steps, fx_shift=32, n_threads=1):
        """photon::sph_t::proc for every packet; final state + flux."""
        n = len(ib)
        c = lambda a, dt=np.float64, k=3: np.ascontiguousarray(a, dt).reshape(n, k) if k > 1 \
            else np.ascontiguousarray(a, dt)
        x, x_car, dir = c(x), c(x_car), c(dir)
        cell, ib = c(cell, np.int32), c(ib, np.int32, 1)
        proper, steps = c(proper, np.float64, 1), c(steps, np.int32, 1)
        out = dict(x=np.zeros((n, 3)), x_car=np.zeros((n, 3)), cell=np.zeros((n, 3), np.int32),
                   ib=np.zeros(n, np.int32), step=np.zeros(n, np.int32),
                   todo=np.zeros(n, np.int32), flux=np.zeros(self.n_cells),
                   flux_fx=np.zeros(self.n_cells, np.int64))
        self.lib.kpref_trace_sph.argtypes = [ctypes.c_long] + [ctypes.c_void_p] * 7 + \
            [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 8
        st = self.lib.kpref_trace_sph(n, _p(x), _p(x_car), _p(dir), _p(cell), _p(ib), _p(proper),
                                      _p(steps), fx_shift, n_threads, _p(out["x"]),
                                      _p(out["x_car"]), _p(out["cell"]), _p(out["ib"]),
                                      _p(out["step"]), _p(out["todo"]), _p(out["flux"]),
                                      _p(out["flux_fx"]))
        if st != 0:
            raise RuntimeError("kpref_trace_sph failed")
        return out


def bio_write(path: str, entries, precision: int = 2) -> None:
    """Writes (tag, numpy array) pairs with the reference's own
    binary_io::base_t (write with copy, then save)."""
    L = RefMesh._lib_for(precision)
    n = len(entries)
    arrs = [np.ascontiguousarray(a).reshape(-1) for _, a in entries]
    tags = (ctypes.c_char_p * n)(*[t.encode("ascii") for t, _ in entries])
    data = (ctypes.c_void_p * n)(*[a.ctypes.data for a in arrs])
    counts = (ctypes.c_ulonglong * n)(*[a.size for a in arrs])
    units = (ctypes.c_int * n)(*[a.dtype.itemsize for a in arrs])
    L.kpref_bio_write.argtypes = [ctypes.c_char_p, ctypes.c_int] + [ctypes.c_void_p] * 4
    if L.kpref_bio_write(path.encode(), n, tags, data, counts, units) != 0:
        raise RuntimeError("reference binary_io rejected the entries")


def bio_read(path: str, tag: str, precision: int = 2):
    """(bytes, unit size) of one entry, read by the reference's
    binary_io::base_t (load, then read)."""
    L = RefMesh._lib_for(precision)
    L.kpref_bio_read.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.c_void_p]
    L.kpref_bio_read.restype = ctypes.c_longlong
    size, unit = ctypes.c_ulonglong(), ctypes.c_int()
    if L.kpref_bio_read(path.encode(), tag.encode(), None, ctypes.byref(size),
                        ctypes.byref(unit)) < 0:
        raise KeyError(tag)
    buf = np.zeros(max(1, size.value), np.uint8)
    if L.kpref_bio_read(path.encode(), tag.encode(), buf.ctypes.data, None, None) < 0:
        raise KeyError(tag)
    return buf[:size.value].tobytes(), unit.value
