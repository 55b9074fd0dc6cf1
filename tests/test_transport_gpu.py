"""Polarized transport on the GPU vs the C restatement, bit for bit.

Per-packet final states (position, direction, Stokes, weight, cell, block,
interaction and step counts, RNG draws), int64 escape tallies, peel-off
images, batch sums and counters must be identical.
"""
import dataclasses

import numpy as np
import pytest
import torch

from kratos_polrad_b200.transport import TALLY_FLOAT, Tallies, forward
from oracle import port
from transport_cases import case, run_oracle, to_device

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not port.available(), reason="oracle not built")]


@pytest.mark.parametrize("name", ["slab", "amr_point", "hg_multi", "table"])
def test_transport_bit_exact(name):
    """"table": packets made by a user generator (kp_packet_init_t) instead
    of a source."""
    mesh, sig, t = case(name)
    mesh.set_sigma(sig)
    tal = forward(mesh, to_device(t))
    torch.cuda.synchronize()
    assert mesh.status() == 0
    ref = run_oracle(mesh, sig, t)
    rec, rref = tal.record_array(), ref["records"]
    for f in rec.dtype.names:
        np.testing.assert_array_equal(rec[f], rref[f], err_msg=f)
    np.testing.assert_array_equal(tal.counters.cpu().numpy(), ref["counters"].astype(np.int64))
    if t.n_mu_bins:
        np.testing.assert_array_equal(tal.mu.cpu().numpy(), ref["mu"])
    if t.image_n:
        np.testing.assert_array_equal(tal.image.cpu().numpy(), ref["image"])
        np.testing.assert_array_equal(tal.image_batch.cpu().numpy(), ref["image_batch"])


def test_transport_repeatable_and_split():
    """Same packets in two launches (offsets) give the same int64 tallies."""
    mesh, sig, t = case("amr_point")
    mesh.set_sigma(sig)
    a = forward(mesh, t)
    t1 = case("amr_point")[2]
    t1.n_packets, t1.n_record = 1200, 0
    b = forward(mesh, t1)
    t1.packet_offset, t1.n_packets = 1200, 800
    forward(mesh, t1, b)
    torch.cuda.synchronize()
    assert torch.equal(a.image, b.image)
    assert torch.equal(a.mu, b.mu)
    assert torch.equal(a.counters, b.counters)


def test_float_tally_mode_close_to_fixed():
    mesh, sig, t = case("amr_point")
    mesh.set_sigma(sig)
    fx = forward(mesh, t)
    tf = dataclasses.replace(t, tally_mode=TALLY_FLOAT, n_record=0)
    fl = forward(mesh, tf)
    torch.cuda.synchronize()
    img_fx = fx.image.cpu().numpy() * 2.0 ** -t.fx_shift
    img_fl = fl.image.cpu().numpy().astype(np.float64)
    # Float atomics sum the same deposits in another order.  On every pixel
    # whose intensity is above a noise floor of 1e-3 of the peak, each Stokes
    # component agrees within 1e-6 of the pixel's I: a deposit's |Q|, |U|,
    # |V| never exceed its I, so the summation error of every component is
    # bounded relative to I, while Q, U and V themselves may cancel to near
    # zero.  Below the floor the bar is 1e-9 of the peak (the int64 rounding
    # is 2^-32 per deposit).
    I_fx = img_fx[..., 0]
    peak = I_fx.max()
    big = I_fx > 1e-3 * peak
    assert big.sum() > 100
    rel = (np.abs(img_fl - img_fx)[big] / I_fx[big][:, None]).max(1)
    assert rel.max() <= 1e-6, (rel.max(), np.percentile(rel, 99))
    np.testing.assert_allclose(img_fl[~big], img_fx[~big], rtol=1e-6, atol=1e-9 * peak)
    np.testing.assert_allclose(img_fl[..., 0].sum(), img_fx[..., 0].sum(), rtol=1e-7)


@pytest.mark.parametrize("name", ["amr_point", "hg_multi", "table"])
def test_chunked_solve_with_small_peel_queue(name):
    """A peel-off queue of 1024 rays: the solve runs in chunks of 85 packets,
    and chunks whose packets queue more rays than that march the rest where
    they start.  Records, tallies and counters equal the oracle's."""
    from kratos_polrad_b200._lib import call
    mesh, sig, t = case(name)
    mesh.set_sigma(sig)
    call("kp_mesh_peel_queue_limit", mesh.handle, 1024)
    try:
        tal = forward(mesh, to_device(t))
        torch.cuda.synchronize()
        assert mesh.status() == 0
    finally:
        call("kp_mesh_peel_queue_limit", mesh.handle, 1 << 27)
    ref = run_oracle(mesh, sig, t)
    rec, rref = tal.record_array(), ref["records"]
    for f in rec.dtype.names:
        np.testing.assert_array_equal(rec[f], rref[f], err_msg=f)
    np.testing.assert_array_equal(tal.counters.cpu().numpy(), ref["counters"].astype(np.int64))
    np.testing.assert_array_equal(tal.image.cpu().numpy(), ref["image"])
    np.testing.assert_array_equal(tal.image_batch.cpu().numpy(), ref["image_batch"])


def test_peel_queue_limit_refuses_tiny_queue():
    from kratos_polrad_b200._lib import KP_ERR_CONFIG, KPError, call
    mesh, _, _ = case("slab")
    with pytest.raises(KPError) as e:
        call("kp_mesh_peel_queue_limit", mesh.handle, 100)
    assert e.value.code == KP_ERR_CONFIG
