"""Path-replay adjoint on the GPU vs the C restatement, bit for bit, and the
torch.autograd wrapper."""
import dataclasses

import numpy as np
import pytest
import torch

from kratos_polrad_b200.adjoint import TransportImage, adjoint, gradients
from kratos_polrad_b200.transport import TALLY_FLOAT
from oracle import port
from transport_cases import case, run_oracle_adjoint, to_device

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not port.available(), reason="oracle not built")]


@pytest.mark.parametrize("name", ["amr_point", "hg_multi", "table"])
def test_adjoint_bit_exact(name):
    mesh, sig, t = case(name)
    t = dataclasses.replace(t, n_record=0)
    mesh.set_sigma(sig)
    rng = np.random.default_rng(1)
    adj = rng.normal(size=(t.image_n, t.image_n, 4)).astype(np.float32)
    cnt = torch.zeros(10, dtype=torch.int64, device="cuda")
    gl, gi = adjoint(mesh, to_device(t), torch.tensor(adj, device="cuda"), 24, counters=cnt)
    torch.cuda.synchronize()
    assert mesh.status() == 0
    rl, ri, rc = run_oracle_adjoint(mesh, sig, t, adj, 24)
    np.testing.assert_array_equal(gl.cpu().numpy(), rl)
    np.testing.assert_array_equal(gi.cpu().numpy(), ri)
    c = cnt.cpu().numpy()
    assert c[0] == rc[0] and c[2] == rc[2]          # walk segments, interactions


@pytest.mark.parametrize("name", ["amr_point", "hg_multi"])
def test_adjoint_cell_ordered_bit_exact(name):
    """Both adjoint marches read the queue sorted by starting cell: the
    int64 gradients equal the oracle's."""
    from kratos_polrad_b200.mesh import PEEL_ORDER_AUTO, PEEL_ORDER_CELL
    mesh, sig, t = case(name)
    t = dataclasses.replace(t, n_record=0)
    mesh.set_sigma(sig)
    adj = np.random.default_rng(1).normal(size=(t.image_n, t.image_n, 4)).astype(np.float32)
    mesh.set_peel_order(PEEL_ORDER_CELL)
    try:
        gl, gi = adjoint(mesh, to_device(t), torch.tensor(adj, device="cuda"), 24)
        torch.cuda.synchronize()
        assert mesh.status() == 0
    finally:
        mesh.set_peel_order(PEEL_ORDER_AUTO)
    rl, ri, _ = run_oracle_adjoint(mesh, sig, t, adj, 24)
    np.testing.assert_array_equal(gl.cpu().numpy(), rl)
    np.testing.assert_array_equal(gi.cpu().numpy(), ri)


def test_adjoint_float_mode_close():
    mesh, sig, t = case("amr_point")
    t = dataclasses.replace(t, n_record=0)
    mesh.set_sigma(sig)
    adj = torch.tensor(np.random.default_rng(2).normal(size=(t.image_n, t.image_n, 4)),
                       dtype=torch.float32, device="cuda")
    a_s, a_a = gradients(mesh, t, adj, 24)
    b_s, b_a = gradients(mesh, dataclasses.replace(t, tally_mode=TALLY_FLOAT), adj, 24)
    # Per cell, the float32 atomic sum of n deposits v_k (each first rounded to
    # float) differs from the exact sum by at most (gamma_n + u) * sum|v_k|,
    # gamma_n = n u / (1 - n u), u = 2^-24, in any order; the int64 sum of
    # round(v_k 2^24) differs by at most n 2^-25.  Cells crossed by every
    # packet (around the source) sum thousands of terms that nearly cancel,
    # so the bound is taken per cell from the oracle's |v| sums and counts.
    rl, ri, _, S = run_oracle_adjoint(mesh, sig, t, adj.cpu().numpy(), 24, abs_sum=True)
    np.testing.assert_array_equal(a_a.cpu().numpy(), rl * 2.0 ** -24)
    A, n = S[:, 0], S[:, 1]
    u = 2.0 ** -24
    tol = (n * u / (1 - n * u) + u) * A + n * 2.0 ** -25
    for x, y in ((a_s, b_s), (a_a, b_a)):
        x, y = x.cpu().numpy(), y.cpu().numpy()
        err = np.abs(y - x)
        assert np.all(err <= tol), (err - tol).max()
        # and in all but a few heavy cells, far inside the peak's 1e-3
        assert np.mean(err > 1e-3 * np.abs(x).max()) < 1e-3


def test_autograd_backward_is_the_adjoint():
    mesh, sig, t = case("amr_point")
    t = dataclasses.replace(t, n_record=0)
    s = torch.tensor(sig, device="cuda", dtype=torch.float64)
    sca = s[:, 0].clone().requires_grad_(True)
    ab = s[:, 1].clone().requires_grad_(True)
    img = TransportImage.apply(sca, ab, mesh, t)
    target = torch.zeros_like(img)
    loss = ((img - target)[..., 1:3] ** 2).sum()          # Q/U L2 loss
    loss.backward()
    g_img = torch.zeros_like(img)
    g_img[..., 1:3] = 2 * img[..., 1:3]
    gmax = g_img.abs().max()
    e_sca, e_abs = gradients(mesh, t, (g_img / gmax).float(), 24)
    f = gmax / t.n_packets
    torch.testing.assert_close(sca.grad, e_sca * f, rtol=0, atol=0)
    torch.testing.assert_close(ab.grad, e_abs * f, rtol=0, atol=0)
    assert torch.isfinite(sca.grad).all() and sca.grad.abs().sum() > 0


@pytest.mark.parametrize("name", ["amr_point", "hg_multi", "table"])
def test_adjoint_small_queue_bit_exact(name):
    """A queue of 1024 vertex rays: the adjoint runs in chunks of 85 packets,
    and the packets whose rays find the queue full are replayed inline by
    k_adjoint.  Gradients and walk counters still equal the oracle's."""
    from kratos_polrad_b200._lib import call
    mesh, sig, t = case(name)
    t = dataclasses.replace(t, n_record=0)
    mesh.set_sigma(sig)
    adj = np.random.default_rng(3).normal(size=(t.image_n, t.image_n, 4)).astype(np.float32)
    cnt = torch.zeros(10, dtype=torch.int64, device="cuda")
    call("kp_mesh_peel_queue_limit", mesh.handle, 1024)
    try:
        gl, gi = adjoint(mesh, to_device(t), torch.tensor(adj, device="cuda"), 24, counters=cnt)
        torch.cuda.synchronize()
        assert mesh.status() == 0
    finally:
        call("kp_mesh_peel_queue_limit", mesh.handle, 1 << 27)
    rl, ri, rc = run_oracle_adjoint(mesh, sig, t, adj, 24)
    np.testing.assert_array_equal(gl.cpu().numpy(), rl)
    np.testing.assert_array_equal(gi.cpu().numpy(), ri)
    c = cnt.cpu().numpy()
    assert c[0] == rc[0] and c[2] == rc[2]
