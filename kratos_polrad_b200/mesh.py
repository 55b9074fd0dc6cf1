"""Block-structured AMR mesh handle (host mirror of the reference's mesh set-up).

Mirrors what the reference's ``mesh_t::init`` + ``meshgen::base_t`` +
``particle::block_map_t::update`` produce for the transport path
(mesh/meshgen/meshgen.cpp:44-106, modules/particle/types/block_map.h:53-103):
a static 2:1-balanced block tree, per-block geometry and the face-neighbour
table, built by the C++ host code behind ``kp_mesh_create``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import call, ptr
from .config import MeshConfig, RefineRegion  # noqa: F401  (re-exported)


# kp_mesh_peel_order's orders
PEEL_ORDER_AUTO, PEEL_ORDER_QUEUE, PEEL_ORDER_CELL = -1, 0, 1


class Mesh:
    """Owns a ``kp_mesh_t``; building needs no GPU."""

    def __init__(self, cfg: MeshConfig | None = None, ini_path: str | None = None,
                 _handle: ctypes.c_void_p | None = None, spherical: bool = False,
                 r_ratio: float = 1.0):
        """Cartesian mesh from a MeshConfig or INI file; ``spherical``: axes
        (r, theta, phi) of meshgen::sph_t with cyl_t's radial spacing
        (``r_ratio`` for a MeshConfig; an INI file gives [mesh] r_ratio)."""
        h = ctypes.c_void_p()
        self.spherical = bool(spherical)
        if _handle is not None:
            h = _handle
        elif ini_path is not None and spherical:
            call("kp_mesh_create_sph_ini", ini_path.encode(), ctypes.byref(h))
        elif ini_path is not None:
            call("kp_mesh_create_ini", ini_path.encode(), ctypes.byref(h))
        else:
            d = _lib.MeshDesc()
            for a in range(3):
                d.x_min[a], d.x_max[a] = cfg.x_min[a], cfg.x_max[a]
                d.n_cell_global[a] = int(cfg.n_cell_global[a])
                d.n_cell_block[a] = int(cfg.n_cell_block[a])
                d.periodic[a] = int(bool(cfg.periodic[a]))
            boxes = (_lib.RefineBox * max(1, len(cfg.refine)))()
            for k, r in enumerate(cfg.refine):
                boxes[k].level = int(r.level)
                for a in range(3):
                    boxes[k].x_min[a], boxes[k].x_max[a] = r.x_min[a], r.x_max[a]
            d.n_refine = len(cfg.refine)
            d.refine = ctypes.cast(boxes, ctypes.POINTER(_lib.RefineBox))
            if spherical:
                call("kp_mesh_create_sph", ctypes.byref(d), float(r_ratio), ctypes.byref(h))
            else:
                call("kp_mesh_create", ctypes.byref(d), ctypes.byref(h))
        self.handle = h
        info = _lib.MeshInfo()
        call("kp_mesh_info", h, ctypes.byref(info))
        self.n_blocks = info.n_blocks
        self.nc = tuple(info.n_cell_block)
        self.cells_per_block = info.cells_per_block
        self.n_cells = info.n_cells
        self.max_level = info.max_level
        self.periodic = tuple(bool(v) for v in info.periodic)
        self.x_min = tuple(info.x_min)
        self.x_max = tuple(info.x_max)

    def close(self):
        if self.handle:
            call("kp_mesh_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- tables (host) ----
    def blocks(self):
        lev = np.zeros(self.n_blocks, np.int32)
        reg = np.zeros((self.n_blocks, 3), np.int32)
        call("kp_mesh_blocks", self.handle, ptr(lev), ptr(reg))
        return lev, reg

    def geometry(self, precision: int = 8):
        nb = self.n_blocks
        xf0, dx0 = np.zeros((nb, 3)), np.zeros((nb, 3))
        vol0, pb = np.zeros(nb), np.zeros((nb, 6), np.int32)
        call("kp_mesh_geometry", self.handle, precision, ptr(xf0), ptr(dx0), ptr(vol0), ptr(pb))
        return xf0, dx0, vol0, pb

    def neighbors(self):
        nb = self.n_blocks
        ids = np.zeros((nb, 24), np.int32)
        sh = np.zeros((nb, 48), np.int32)
        dl = np.zeros((nb, 6), np.int32)
        call("kp_mesh_neighbors", self.handle, ptr(ids), ptr(sh), ptr(dl))
        return ids, sh, dl

    def locate(self, x):
        x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        ib = np.zeros(len(x), np.int32)
        cell = np.zeros((len(x), 3), np.int32)
        call("kp_mesh_locate", self.handle, len(x), ptr(x), ptr(ib), ptr(cell))
        return ib, cell

    # ---- device ----
    def upload(self):
        call("kp_mesh_upload", self.handle)

    def set_sigma(self, sigma2):
        """Per-cell (sigma_sca, sigma_abs), shape (n_cells, 2), host or torch CUDA."""
        on_dev = int(hasattr(sigma2, "is_cuda") and sigma2.is_cuda)
        if not on_dev:
            sigma2 = np.ascontiguousarray(sigma2, np.float32)
        n = int(np.prod(sigma2.shape))
        call("kp_mesh_set_sigma", self.handle, ptr(sigma2), n, on_dev, None)

    def geometry_sph(self, precision: int = 8):
        """Spherical meshes: radial faces [n_blocks, nc0 + 1] and cell volumes
        [n_cells] as float_t of ``precision`` bytes holds them."""
        rf = np.zeros((self.n_blocks, self.nc[0] + 1))
        vol = np.zeros(self.n_cells)
        call("kp_mesh_geometry_sph", self.handle, precision, ptr(rf), ptr(vol))
        return rf, vol

    # ---- runtime refinement ----
    def flag_tau(self, tau_refine: float, tau_coarsen: float = 0.0, stream=None):
        """Per-block flags on the device (int32 tensor): +1 where a cell's
        extinction depth across the widest cell side exceeds ``tau_refine``,
        -1 where all stay below ``tau_coarsen``, else 0."""
        import torch
        flags = torch.empty(self.n_blocks, dtype=torch.int32, device="cuda")
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        call("kp_mesh_flag_tau", self.handle, float(tau_refine), float(tau_coarsen), ptr(flags), s)
        return flags

    def adapt(self, flags) -> "Mesh":
        """New mesh: blocks flagged > 0 refined, families of eight leaves all
        flagged < 0 coarsened, 2:1 balance restored (host; needs no GPU)."""
        f = np.ascontiguousarray(_host(flags), np.int32).reshape(-1)
        if f.size != self.n_blocks:
            raise ValueError(f"need {self.n_blocks} flags, got {f.size}")
        h = ctypes.c_void_p()
        call("kp_mesh_adapt", self.handle, ptr(f), ctypes.byref(h))
        return Mesh(_handle=h, spherical=self.spherical)

    def remap_to(self, other: "Mesh", field, stream=None):
        """Per-cell field [n_cells, n_comp] (CUDA tensor, float32) of this mesh
        carried onto ``other`` (same domain): copy where a cell of ``other``
        lies in one cell here, mean of eight octant samples where it covers
        several."""
        import torch
        src = field.to(torch.float32).contiguous()
        n_comp = 1 if src.dim() == 1 else src.shape[1]
        if src.shape[0] != self.n_cells:
            raise ValueError("field must have n_cells rows")
        dst = torch.empty((other.n_cells, n_comp), dtype=torch.float32, device=src.device)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        call("kp_mesh_remap", self.handle, other.handle, n_comp, ptr(src), ptr(dst), s)
        return dst if src.dim() > 1 else dst[:, 0]

    def tape_id(self) -> int:
        """Id of the taped forward solve the mesh holds (0: none)."""
        tid = ctypes.c_longlong(0)
        call("kp_mesh_tape_id", self.handle, ctypes.byref(tid))
        return tid.value

    def set_peel_order(self, order: int) -> None:
        """The order the forward solve marches its queued peel-off rays in:
        PEEL_ORDER_AUTO (default), PEEL_ORDER_QUEUE or PEEL_ORDER_CELL (sorted
        by starting cell).  The fixed-point tallies do not depend on it."""
        call("kp_mesh_peel_order", self.handle, int(order))

    def status(self, stream=None) -> int:
        flags = ctypes.c_uint()
        call("kp_mesh_status", self.handle, stream, ctypes.byref(flags))
        return flags.value


def _host(a):
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)
