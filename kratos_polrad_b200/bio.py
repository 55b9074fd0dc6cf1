"""The reference's binary container (io/binary/binary_io.h:6-32) for the
transport's fields and tallies, through ``kp_bio_*`` of the C ABI.

``write`` produces the file binary_io::base_t::save would for the same
entries (tags sorted, data packed in tag order); ``BinaryFile`` reads it or a
file of the reference's Python writer, with the reference reader's
``as_array(key, dtype)`` convention (visual/binary_io.py:96-99: dtype letter
plus the stored unit size, little-endian).

``save_solution`` / ``load_solution`` keep a solve restartable, as
mesh_t::save and the restart load do (mesh/mesh.cpp:63-69, 99-112):

* per block, the reference's own tags: ``block_<id>|i_logic`` (3 int32) and
  ``block_<id>|level`` (int32) as block_t::write stores them
  (mesh/block/block.cpp:31-38), and the rad_t flux field
  ``block_<id>|rad_flx_flux_{n_int,n_step,n_cell,n_gh,field}`` as
  dat_3d_t::write lays it out (mesh/types/dat_3d.h:117-125,
  modules/particle/radiation/rad_data.cpp:45-49): the ``flux`` argument (a
  geometric walk's deposits), or else the transport's path-length flux tally
  (``tallies.flux``, as float32 sums of w * dl / volume);
* the transport's arrays under ``kp|<name>`` (flat, with their shape under
  ``kp|shape|<name>``): ``sigma`` [n_cells, 2], the tallies ``mu``,
  ``image``, ``image_batch``, ``counters``, ``flux`` (raw, int64 when fixed
  point, so that a restart keeps accumulating exactly), gradients ``grad_sca``,
  ``grad_abs``, and ``kp|config`` (JSON of the TransportConfig) with
  ``kp|packets_done``.  A restart reloads sigma and the int64 tallies and
  continues with ``packet_offset = packets_done``: fixed-point tallies of the
  two runs add up to those of one run over all packets, bit for bit.
"""
from __future__ import annotations

import ctypes
import dataclasses
import json
import os

import numpy as np

from . import _lib
from ._lib import call


class BioEntry(ctypes.Structure):
    _fields_ = [("tag", ctypes.c_char_p), ("data", ctypes.c_void_p),
                ("count", ctypes.c_ulonglong), ("unit_size", ctypes.c_int)]


_ull = ctypes.c_ulonglong
_lib.register("kp_bio_write", [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(BioEntry)])
_lib.register("kp_bio_open", [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)])
_lib.register("kp_bio_close", [ctypes.c_void_p])
_lib.register("kp_bio_n_entries", [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)])
_lib.register("kp_bio_entry", [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t,
                               ctypes.POINTER(_ull), ctypes.POINTER(ctypes.c_int)])
_lib.register("kp_bio_read", [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, _ull,
                              ctypes.POINTER(_ull)])


def _as_bytes_array(v):
    """(contiguous numpy array, unit size) of an entry value."""
    if isinstance(v, str):
        v = v.encode()
    if isinstance(v, (bytes, bytearray)):
        return np.frombuffer(bytes(v), np.uint8), 1
    a = np.ascontiguousarray(v)
    if a.dtype.byteorder == ">":
        a = a.astype(a.dtype.newbyteorder("<"))
    return a.reshape(-1), a.dtype.itemsize


def write(path: str, entries) -> None:
    """Writes ``entries`` (dict or (tag, value) pairs; value: numpy array,
    bytes or str) as one container; a repeated tag keeps its last value."""
    items = list(entries.items()) if isinstance(entries, dict) else list(entries)
    keep, arr = [], (BioEntry * max(1, len(items)))()
    for k, (tag, v) in enumerate(items):
        a, u = _as_bytes_array(v)
        keep.append(a)
        arr[k].tag = tag.encode("ascii")
        arr[k].data = a.ctypes.data if a.size else None
        arr[k].count = a.size
        arr[k].unit_size = u
    call("kp_bio_write", os.fsencode(path), len(items), arr)


class BinaryFile:
    """Reader of a container (either writer's); ``tags`` in file order."""

    def __init__(self, path: str):
        self.path = path
        h = ctypes.c_void_p()
        call("kp_bio_open", os.fsencode(path), ctypes.byref(h))
        self._h = h
        n = ctypes.c_int()
        call("kp_bio_n_entries", h, ctypes.byref(n))
        self.hmap = {}
        buf = ctypes.create_string_buffer(4096)
        for i in range(n.value):
            size, u = _ull(), ctypes.c_int()
            call("kp_bio_entry", h, i, buf, len(buf), ctypes.byref(size), ctypes.byref(u))
            self.hmap[buf.value.decode("ascii")] = (int(size.value), int(u.value))
        self.tags = list(self.hmap)

    def close(self):
        if self._h:
            call("kp_bio_close", self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __contains__(self, tag):
        return tag in self.hmap

    def __getitem__(self, tag: str) -> bytes:
        size = self.hmap.get(tag, (0, 0))[0]       # a missing tag fails in kp_bio_read
        out = np.empty(size, np.uint8)
        got = _ull()
        call("kp_bio_read", self._h, tag.encode("ascii"), out.ctypes.data if size else None,
             size, ctypes.byref(got))
        return out.tobytes()

    def as_array(self, tag: str, dtype: str = "f") -> np.ndarray:
        """Entry as a little-endian array of kind ``dtype`` ('f', 'i', 'u')
        and the stored unit size, as the reference's reader returns it."""
        return np.frombuffer(self[tag], dtype="<%s%d" % (dtype, self.hmap[tag][1]))

    def read(self, tag: str, dtype) -> np.ndarray:
        return np.frombuffer(self[tag], dtype=np.dtype(dtype).newbyteorder("<"))


def _np(t):
    if t is None:
        return None
    if hasattr(t, "detach"):
        t = t.detach().cpu().numpy()
    return np.asarray(t)


def save_solution(path: str, mesh, sigma2=None, tallies=None, cfg=None, grads=None,
                  flux=None, packets_done: int | None = None) -> None:
    """Writes the mesh's block keys and the given arrays (numpy or torch,
    any device) into one container; see the module docstring for the tags."""
    ent = []
    lev, reg = mesh.blocks()
    cpb = mesh.cells_per_block
    fl = _np(flux)
    if fl is None and getattr(tallies, "flux", None) is not None:
        fl = _np(tallies.flux).astype(np.float64)
        if fl.dtype != np.float32 and np.issubdtype(_np(tallies.flux).dtype, np.integer):
            c = cfg if cfg is not None else tallies.cfg
            fl *= 2.0 ** -(c.flux_fx_shift or c.fx_shift)
        fl = fl.astype(np.float32)
    for b in range(mesh.n_blocks):
        p = f"block_{b}|"
        ent.append((p + "i_logic", reg[b].astype(np.int32)))
        ent.append((p + "level", np.int32([lev[b]])))
        if fl is not None:
            q = p + "rad_flx_flux_"
            ent += [(q + "n_int", np.int32([1])), (q + "n_step", np.int32([1])),
                    (q + "n_cell", np.int32(mesh.nc)), (q + "n_gh", np.int32([0, 0, 0])),
                    (q + "field", fl[b * cpb:(b + 1) * cpb])]

    def put(name, a):
        a = _np(a)
        if a is not None:
            ent.append((f"kp|{name}", a))
            ent.append((f"kp|shape|{name}", np.int64(a.shape if a.ndim else [1])))

    put("sigma", sigma2)
    if tallies is not None:
        for name in ("mu", "image", "image_batch", "counters", "flux"):
            put(name, getattr(tallies, name, None))
    if grads is not None:
        put("grad_sca", grads[0])
        put("grad_abs", grads[1])
    if cfg is not None:
        d = dataclasses.asdict(cfg)
        ent.append(("kp|config", json.dumps(d, default=list)))
        done = packets_done if packets_done is not None else cfg.packet_offset + cfg.n_packets
        ent.append(("kp|packets_done", np.int64([done])))
    write(path, ent)


_DT = {"sigma": np.float32, "counters": np.uint64}


def load_solution(path: str) -> dict:
    """Arrays saved by save_solution (shaped), ``config`` (dict) and
    ``packets_done``; tallies come back as int64 (fixed-point runs) unless
    their unit size says float32."""
    out = {}
    with BinaryFile(path) as f:
        for tag in f.tags:
            if not tag.startswith("kp|") or tag.startswith("kp|shape|") or tag in (
                    "kp|config", "kp|packets_done"):
                continue
            name = tag[3:]
            u = f.hmap[tag][1]
            dt = _DT.get(name, {8: np.int64, 4: np.float32}.get(u, np.uint8))
            if name.startswith("grad_"):
                dt = np.float64 if u == 8 else np.float32
            a = f.read(tag, dt)
            shp = tuple(int(v) for v in f.read(f"kp|shape|{name}", np.int64))
            out[name] = a.reshape(shp).copy()
        if "kp|config" in f:
            out["config"] = json.loads(f["kp|config"].decode())
        if "kp|packets_done" in f:
            out["packets_done"] = int(f.read("kp|packets_done", np.int64)[0])
    return out
