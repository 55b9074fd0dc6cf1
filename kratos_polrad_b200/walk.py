"""Geometric walk with the path-length flux estimator (reference semantics).

Host mirror of ``particle::integrate::base_t::intg`` running
``photon::cart_t::proc`` over the packet pool
(modules/particle/evolve/integrator.h:47-63,80-106;
modules/particle/radiation/photon.h:20-125): every packet walks cell by cell
until its step budget is spent or it leaves the domain, depositing
``proper * path_length / cell_volume`` into the per-cell flux field.
"""
from __future__ import annotations

import torch

from ._lib import KP_FLUX_FIXED, KP_FLUX_FLOAT, call, ptr

TO_KEEP, TO_RM = -2, -3


class PacketPool:
    """Structure-of-arrays packet pool on the device (particle_pool.h:18-249).

    Fields follow ``particle::par_base_t`` (types/particle_base.h:17-81):
    position ``x`` and direction ``dir`` in float_t, cell index ``cell``,
    block id ``ib``, weight ``proper``, step budget ``step`` and ``todo``.
    """

    def __init__(self, x, dir, cell, ib, proper, step, todo=None):
        dev = x.device
        self.x = x.contiguous()
        self.dir = dir.to(x.dtype).contiguous()
        self.cell = cell.to(torch.int32).contiguous()
        self.ib = ib.to(torch.int32).contiguous()
        self.proper = proper.to(x.dtype).contiguous()
        self.step = step.to(torch.int32).contiguous()
        if todo is None:
            todo = torch.full((len(self.ib),), TO_KEEP, dtype=torch.int8, device=dev)
        self.todo = todo.to(torch.int8).contiguous()

    def __len__(self):
        return self.ib.numel()


def trace(mesh, pool: PacketPool, flux_mode: str = "fixed", fx_shift: int = 32,
          flux: torch.Tensor | None = None, stream: int | None = None) -> torch.Tensor:
    """Walks every ``to_keep`` packet of ``pool`` in place; returns the flux.

    ``flux_mode`` "float": float_t atomics as the reference (photon.h:81);
    "fixed": int64 sums of ``round(deposit * 2**fx_shift)`` (order independent).
    """
    prec = pool.x.element_size()
    if flux is None:
        dt = torch.int64 if flux_mode == "fixed" else pool.x.dtype
        flux = torch.zeros(mesh.n_cells, dtype=dt, device=pool.x.device)
    mode = KP_FLUX_FIXED if flux_mode == "fixed" else KP_FLUX_FLOAT
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    call("kp_trace", mesh.handle, prec, len(pool), ptr(pool.x), ptr(pool.dir),
         ptr(pool.cell), ptr(pool.ib), ptr(pool.proper), ptr(pool.step),
         ptr(pool.todo), mode, fx_shift, ptr(flux), s)
    return flux


def trace_sph(mesh, pool: PacketPool, x_car: torch.Tensor, flux_mode: str = "fixed",
              fx_shift: int = 32, flux: torch.Tensor | None = None,
              stream: int | None = None) -> torch.Tensor:
    """``photon::sph_t::proc`` (modules/particle/radiation/photon_sph.h) over a
    spherical mesh: ``pool.x`` holds (r, theta, phi) and ``x_car`` [n, 3] its
    Cartesian copy (both updated in place); otherwise as ``trace``."""
    prec = pool.x.element_size()
    xc = x_car.to(pool.x.dtype)
    if not xc.is_contiguous() or xc.data_ptr() != x_car.data_ptr():
        raise ValueError("x_car must be a contiguous tensor of the pool's float type")
    if flux is None:
        dt = torch.int64 if flux_mode == "fixed" else pool.x.dtype
        flux = torch.zeros(mesh.n_cells, dtype=dt, device=pool.x.device)
    mode = KP_FLUX_FIXED if flux_mode == "fixed" else KP_FLUX_FLOAT
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    call("kp_trace_sph", mesh.handle, prec, len(pool), ptr(pool.x), ptr(x_car), ptr(pool.dir),
         ptr(pool.cell), ptr(pool.ib), ptr(pool.proper), ptr(pool.step),
         ptr(pool.todo), mode, fx_shift, ptr(flux), s)
    return flux
