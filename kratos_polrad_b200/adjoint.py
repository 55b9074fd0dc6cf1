"""Differentiable transport: the path-replay adjoint behind torch.autograd.

``TransportImage.apply(sigma_sca, sigma_abs, mesh, cfg)`` returns the peel-off
image (expected Stokes per packet, float64 [n, n, 4]) of the forward solve;
its backward runs the adjoint with the same packets (same seed, ids and
sources: common random numbers), so the gradient is that of the same
estimator.  Every packet is replayed from its RNG counter; the forward is
taped (``kp_transport_forward_tape``: the packets' peel-off rays and their
attenuation stay in the mesh), so that the backward skips the first replay
and its march when nothing has replaced the tape in between.
"""
from __future__ import annotations

import ctypes
import dataclasses

import torch

from . import _lib
from ._lib import call, ptr
from .transport import CTransportCfg, TALLY_FIXED, Tallies, TransportConfig, forward

_lib.register("kp_transport_adjoint", [ctypes.c_void_p, ctypes.POINTER(CTransportCfg),
                                       ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p])


def adjoint(mesh, cfg: TransportConfig, adj_image: torch.Tensor, grad_fx_shift: int = 24,
            counters: torch.Tensor | None = None, stream: int | None = None, tape_id: int = 0):
    """Raw adjoint tallies for dL/d(image tally) = ``adj_image`` [n, n, 4].

    Returns (grad_len, grad_int) as int64 (fixed mode) or float32 tensors
    of n_cells; dL/dsigma_sca = len + int, dL/dsigma_abs = len (times
    2^-grad_fx_shift in fixed mode).  With ``tape_id`` (from
    ``forward(..., tape=True)``) it differentiates that taped solve from its
    tape; KPError (KP_ERR_CONFIG) if the tape is gone.
    """
    dt = torch.int64 if cfg.tally_mode == TALLY_FIXED else torch.float32
    dev = adj_image.device
    g_len = torch.zeros(mesh.n_cells, dtype=dt, device=dev)
    g_int = torch.zeros(mesh.n_cells, dtype=dt, device=dev)
    a = adj_image.to(torch.float32).contiguous()
    c = cfg.to_c()
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    if tape_id:
        call("kp_transport_adjoint_tape", mesh.handle, tape_id, ctypes.byref(c), ptr(a),
             grad_fx_shift, ptr(g_len), ptr(g_int), ptr(counters), s)
    else:
        call("kp_transport_adjoint", mesh.handle, ctypes.byref(c), ptr(a), grad_fx_shift,
             ptr(g_len), ptr(g_int), ptr(counters), s)
    return g_len, g_int


def gradients(mesh, cfg, adj_image, grad_fx_shift=24, counters=None, tape_id=0):
    """(dL/dsigma_sca, dL/dsigma_abs) as float64 tensors for dL/dimage_tally."""
    g_len, g_int = adjoint(mesh, cfg, adj_image, grad_fx_shift, counters, tape_id=tape_id)
    sc = 2.0 ** -grad_fx_shift if cfg.tally_mode == TALLY_FIXED else 1.0
    gl = g_len.double() * sc
    gi = g_int.double() * sc
    return gl + gi, gl


class TransportImage(torch.autograd.Function):
    """sigma (per cell) -> expected peel-off image per packet."""

    @staticmethod
    def forward(ctx, sigma_sca, sigma_abs, mesh, cfg: TransportConfig, grad_fx_shift: int = 24):
        sig2 = torch.stack([sigma_sca, sigma_abs], 1).to(torch.float32).contiguous()
        mesh.set_sigma(sig2)
        cfg = dataclasses.replace(cfg, n_record=0)
        tal = forward(mesh, cfg, Tallies(cfg, device=sigma_sca.device), tape=True)
        img = tal.image.double() * (tal.scale() / cfg.n_packets)
        ctx.save_for_backward(sig2)
        ctx.mesh, ctx.cfg, ctx.shift, ctx.tape_id = mesh, cfg, grad_fx_shift, tal.tape_id
        return img

    @staticmethod
    def backward(ctx, g_img):
        (sig2,) = ctx.saved_tensors
        mesh, cfg = ctx.mesh, ctx.cfg
        # the tape is ours only if no solve or coefficient change came since
        # (both drop it); then the mesh still holds sig2
        tape_id = ctx.tape_id if ctx.tape_id and mesh.tape_id() == ctx.tape_id else 0
        if not tape_id:
            mesh.set_sigma(sig2)
        # image = (sum of per-packet contributions C) / N.  The kernel returns
        # d/dsigma of sum_k <a, C_k> for an adjoint image a; it is called with
        # a = g / max|g| (order one, so the fixed-point deposits keep their
        # precision) and the result is scaled back by max|g| / N.
        gmax = g_img.abs().max()
        if not torch.isfinite(gmax) or gmax == 0:
            z = torch.zeros(mesh.n_cells, dtype=torch.float64, device=g_img.device)
            return z, z.clone(), None, None, None
        g_sca, g_abs = gradients(mesh, cfg, (g_img / gmax).to(torch.float32), ctx.shift,
                                 tape_id=tape_id)
        f = gmax / cfg.n_packets
        return g_sca * f, g_abs * f, None, None, None
