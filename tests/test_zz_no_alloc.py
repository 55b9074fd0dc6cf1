"""The no-allocation forward entry point (kp_transport_forward_noalloc).

Some callers cannot allocate device memory while they run a solve: code that
owns every device byte itself (an arena sized at start-up), or a step that
runs where cudaMalloc is not allowed.  For them the library offers a forward
solve whose only scratch, the packet counter, lives in a static device array.
These tests call it through the C ABI and check that two calls in a row give
exactly what the ordinary entry point gives (int64 tallies: no tolerance),
and that a mesh that was never put on the device is refused.

The file name makes pytest collect it last; it also passes on its own in a
fresh process (it builds its own mesh and uploads it first).
"""
import ctypes

import numpy as np
import pytest

from kratos_polrad_b200 import _lib
from kratos_polrad_b200._lib import KP_ERR_CONFIG, KPError, call
from kratos_polrad_b200.transport import CTallies, CTransportCfg, Tallies, forward
from transport_cases import case

_lib.register("kp_transport_forward_noalloc", [ctypes.c_void_p, ctypes.POINTER(CTransportCfg),
                                               ctypes.POINTER(CTallies), ctypes.c_void_p])


def _noalloc(mesh, cfg, tallies, stream):
    c, t = cfg.to_c(), tallies.to_c()
    call("kp_transport_forward_noalloc", mesh.handle, ctypes.byref(c), ctypes.byref(t), stream)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["amr_point", "slab"])
def test_noalloc_matches_forward_on_two_calls(name):
    """With an image (amr_point: the walk marches its peel-off rays inline,
    the ordinary entry point queues them) and without (slab: both run the
    same kernel); the flux tally too.  int64 tallies: no tolerance."""
    import dataclasses
    import torch
    mesh, sig, cfg = case(name)
    cfg = dataclasses.replace(cfg, flux=True, flux_fx_shift=24)
    mesh.set_sigma(sig)                      # set-up: puts the mesh on the device
    ref = forward(mesh, cfg)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        tal = Tallies(cfg, n_cells=mesh.n_cells)
        _noalloc(mesh, cfg, tal, stream)
        torch.cuda.synchronize()
        assert mesh.status() == 0
        for name in ("mu", "image", "image_batch", "counters", "flux"):
            assert torch.equal(getattr(tal, name), getattr(ref, name)), name
        a, b = tal.record_array(), ref.record_array()
        for f in a.dtype.names:
            np.testing.assert_array_equal(a[f], b[f], err_msg=f)


@pytest.mark.gpu
def test_noalloc_float_tallies_within_rounding():
    """Float tallies: the inline peel-off rays add into the image in another
    order than the queued ones.  Both carry their rounding errors
    (kp_tallies_t::carry, the caller's memory: the fold after the walk is
    the only other launch), so each pixel agrees within 1e-6 of its I."""
    import dataclasses
    import torch
    from kratos_polrad_b200.transport import TALLY_FLOAT
    mesh, sig, cfg = case("amr_point")
    cfg = dataclasses.replace(cfg, tally_mode=TALLY_FLOAT, n_record=0)
    mesh.set_sigma(sig)
    ref = forward(mesh, cfg)
    tal = Tallies(cfg)
    _noalloc(mesh, cfg, tal, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert mesh.status() == 0
    a, b = tal.image.cpu().numpy().astype(np.float64), ref.image.cpu().numpy().astype(np.float64)
    lit = b[..., 0] > 0
    assert (a[~lit] == 0).all()
    assert (np.abs(a - b)[lit] / b[..., 0][lit][:, None]).max() <= 1e-6
    assert abs(a[..., 0].sum() - b[..., 0].sum()) <= 1e-7 * abs(b[..., 0].sum())
    assert torch.equal(tal.counters, ref.counters)


def test_noalloc_refuses_mesh_not_on_device():
    mesh, _, cfg = case("slab")              # built on the host only
    cfg.n_record = 0
    tal = CTallies()                         # never reached: the mesh check comes first
    with pytest.raises(KPError) as e:
        call("kp_transport_forward_noalloc", mesh.handle, ctypes.byref(cfg.to_c()),
             ctypes.byref(tal), None)
    assert e.value.code == KP_ERR_CONFIG
    assert "kp_mesh_upload" in str(e.value)
