"""ctypes binding of the C ABI declared in include/kp_transport.h.

The shared library ``libkp_b200.so`` is built in-tree (``build()`` in
``__graft_entry__.py`` or ``make -C kratos_polrad_b200/csrc``).  There is no
fallback: if the library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkp_b200.so")
HEADER_DIR = os.path.join(os.path.dirname(_HERE), "include")

c_int, c_ll, c_double, c_float, c_void_p = (ctypes.c_int, ctypes.c_longlong,
                                            ctypes.c_double, ctypes.c_float,
                                            ctypes.c_void_p)
P = ctypes.POINTER

KP_OK, KP_ERR_ARG, KP_ERR_CUDA, KP_ERR_CONFIG, KP_ERR_CAPACITY, KP_ERR_DEVICE, \
    KP_ERR_ALLOC = range(7)
KP_FLUX_FLOAT, KP_FLUX_FIXED = 0, 1


class KPError(RuntimeError):
    """Raised for a non-zero status; ``code`` holds the kp_status value."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[kp status {code}] {msg}")
        self.code = code


class RefineBox(ctypes.Structure):
    _fields_ = [("level", c_int), ("x_min", c_double * 3), ("x_max", c_double * 3)]


class MeshDesc(ctypes.Structure):
    _fields_ = [("x_min", c_double * 3), ("x_max", c_double * 3),
                ("n_cell_global", c_int * 3), ("n_cell_block", c_int * 3),
                ("periodic", c_int * 3), ("n_refine", c_int),
                ("refine", P(RefineBox))]


class MeshInfo(ctypes.Structure):
    _fields_ = [("n_blocks", c_int), ("n_cell_block", c_int * 3),
                ("cells_per_block", c_int), ("max_level", c_int),
                ("n_cells", c_ll), ("periodic", c_int * 3),
                ("x_min", c_double * 3), ("x_max", c_double * 3)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C kratos_polrad_b200/csrc` "
            "(there is no CPU fallback for the transport path)")
    return ctypes.CDLL(LIB_PATH)


lib = _load()

# Signatures (argtypes) of every entry point; status-returning functions
# are wrapped by `call`.
_SIGS = {
    "kp_abi_version": [],
    "kp_device_init": [c_int],
    "kp_device_count": [P(c_int)],
    "kp_malloc": [P(c_void_p), ctypes.c_size_t],
    "kp_malloc_host": [P(c_void_p), ctypes.c_size_t],
    "kp_free": [c_void_p],
    "kp_free_host": [c_void_p],
    "kp_memset_async": [c_void_p, c_int, ctypes.c_size_t, c_void_p],
    "kp_memcpy": [c_void_p, c_void_p, ctypes.c_size_t],
    "kp_memcpy_async": [c_void_p, c_void_p, ctypes.c_size_t, c_void_p],
    "kp_stream_create": [P(c_void_p)],
    "kp_stream_destroy": [c_void_p],
    "kp_stream_sync": [c_void_p],
    "kp_event_create": [P(c_void_p)],
    "kp_event_destroy": [c_void_p],
    "kp_event_record": [c_void_p, c_void_p],
    "kp_event_wait": [c_void_p, c_void_p],
    "kp_event_sync": [c_void_p],
    "kp_event_elapsed": [P(c_float), c_void_p, c_void_p],
    "kp_launch_host": [c_void_p, c_void_p, c_void_p],
    "kp_transport_split_event": [c_void_p],
    "kp_mesh_peel_queue_limit": [c_void_p, c_ll],
    "kp_mesh_peel_order": [c_void_p, c_int],
    "kp_transport_forward_tape": [c_void_p, c_void_p, c_void_p, c_void_p, P(c_ll)],
    "kp_transport_adjoint_tape": [c_void_p, c_ll, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                  c_void_p, c_void_p],
    "kp_mesh_tape_id": [c_void_p, P(c_ll)],
    "kp_mesh_create": [P(MeshDesc), P(c_void_p)],
    "kp_mesh_create_ini": [ctypes.c_char_p, P(c_void_p)],
    "kp_mesh_destroy": [c_void_p],
    "kp_mesh_info": [c_void_p, P(MeshInfo)],
    "kp_mesh_blocks": [c_void_p, c_void_p, c_void_p],
    "kp_mesh_geometry": [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p],
    "kp_mesh_neighbors": [c_void_p, c_void_p, c_void_p, c_void_p],
    "kp_mesh_locate": [c_void_p, c_ll, c_void_p, c_void_p, c_void_p],
    "kp_mesh_upload": [c_void_p],
    "kp_mesh_set_sigma": [c_void_p, c_void_p, c_ll, c_int, c_void_p],
    "kp_mesh_sigma_ptr": [c_void_p, P(c_void_p)],
    "kp_mesh_status": [c_void_p, c_void_p, P(ctypes.c_uint)],
    "kp_mesh_flag_tau": [c_void_p, c_float, c_float, c_void_p, c_void_p],
    "kp_mesh_create_sph": [c_void_p, c_double, P(c_void_p)],
    "kp_mesh_create_sph_ini": [ctypes.c_char_p, P(c_void_p)],
    "kp_mesh_geometry_sph": [c_void_p, c_int, c_void_p, c_void_p],
    "kp_trace_sph": [c_void_p, c_int, c_ll] + [c_void_p] * 8 + [c_int, c_int, c_void_p,
                                                                 c_void_p],
    "kp_mesh_adapt": [c_void_p, c_void_p, P(c_void_p)],
    "kp_mesh_remap": [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p],
    "kp_trace": [c_void_p, c_int, c_ll, c_void_p, c_void_p, c_void_p, c_void_p,
                 c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p],
}

lib.kp_last_error.restype = ctypes.c_char_p
lib.kp_last_error.argtypes = []

# Layout of the structs mirrored below (kp_transport_cfg_t, kp_tallies_t):
# a library built from another header would read them wrongly.
ABI_VERSION = 2
if lib.kp_abi_version() != ABI_VERSION:
    raise ImportError(f"{LIB_PATH} has ABI version {lib.kp_abi_version()}, this package "
                      f"expects {ABI_VERSION}: rebuild it with `make -C kratos_polrad_b200/csrc`")
for _name, _args in _SIGS.items():
    _f = getattr(lib, _name, None)
    if _f is not None:
        _f.argtypes = _args
        _f.restype = c_int


def register(name: str, argtypes):
    """Declare the argtypes of an entry point added after this module."""
    f = getattr(lib, name)
    f.argtypes = argtypes
    f.restype = c_int
    _SIGS[name] = argtypes


def call(name: str, *args) -> None:
    """Calls a status-returning entry point; raises KPError on failure."""
    st = getattr(lib, name)(*args)
    if st != KP_OK:
        raise KPError(st, lib.kp_last_error().decode(errors="replace"))


def header_symbols() -> list[str]:
    """Every kp_* function declared in include/*.h."""
    names = []
    for fn in sorted(os.listdir(HEADER_DIR)):
        if fn.endswith(".h"):
            text = open(os.path.join(HEADER_DIR, fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"\b(kp_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def ptr(a) -> int:
    """Address of a numpy array or torch tensor (0 for None)."""
    if a is None:
        return 0
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data
