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


def _exact_image(t, deposits):
    """Per-pixel float64 sums of the oracle's float deposits (the GPU's,
    bit for bit) and their counts."""
    pix, val = deposits
    n = t.image_n * t.image_n
    ex = np.zeros((n, 4))
    np.add.at(ex, pix, val.astype(np.float64))
    return ex.reshape(t.image_n, t.image_n, 4), np.bincount(pix, minlength=n).reshape(t.image_n, t.image_n)


def test_float_tally_mode_within_1e6_of_exact():
    """Both tally modes against the exact sums of the same float deposits.

    Fixed point: each deposit rounds to 2^-fx_shift, so every entry is within
    n_deposits * 2^-(fx_shift + 1) of its exact sum.  Float mode (with the
    tallies' carry, the default): on EVERY pixel each Stokes component is
    within 1e-6 of the pixel's exact I (a deposit's |Q|, |U|, |V| never
    exceed its I, so I bounds every component's summation error), and the
    total within 1e-7; plain float atomics (no carry) miss that bar by the
    summation error of thousands of deposits per pixel (up to 8e-6 here), so
    they are held only to the worst-case bound n * 2^-24 * sum |deposit|."""
    mesh, sig, t = case("amr_point")
    mesh.set_sigma(sig)
    fx = forward(mesh, t)
    tf = dataclasses.replace(t, tally_mode=TALLY_FLOAT, n_record=0)
    fl = forward(mesh, tf)
    plain = forward(mesh, tf, Tallies(tf, carry=False))
    torch.cuda.synchronize()
    assert mesh.status() == 0
    ref = run_oracle(mesh, sig, t, deposits=1 << 20)
    assert ref["n_deposits"] == len(ref["deposits"][0]) > 10000
    ex, cnt = _exact_image(t, ref["deposits"])
    I = ex[..., 0]
    assert (I > 0).sum() > 200 and cnt.max() > 1000

    img_fx = fx.image.cpu().numpy() * 2.0 ** -t.fx_shift
    assert (np.abs(img_fx - ex) <= cnt[..., None] * 2.0 ** -(t.fx_shift + 1) + 1e-15).all()

    img_fl = fl.image.cpu().numpy().astype(np.float64)
    lit = I > 0
    assert (img_fl[~lit] == 0).all()
    rel = (np.abs(img_fl - ex)[lit] / I[lit][:, None]).max(1)
    assert rel.max() <= 1e-6, (rel.max(), np.percentile(rel, 99))
    assert abs(img_fl[..., 0].sum() - I.sum()) <= 1e-7 * I.sum()

    pix, val = ref["deposits"]
    abs_sum = np.zeros((t.image_n * t.image_n, 4))
    np.add.at(abs_sum, pix, np.abs(val.astype(np.float64)))
    bound = cnt[..., None] * 2.0 ** -24 * abs_sum.reshape(ex.shape)
    img_pl = plain.image.cpu().numpy().astype(np.float64)
    assert (np.abs(img_pl - ex) <= bound + 1e-30).all()
    print("float vs exact / I: carry", rel.max(), "plain",
          (np.abs(img_pl - ex)[lit] / I[lit][:, None]).max())

    # escape tallies (at most one deposit per packet) and the per-batch image
    # (at most every deposit in one entry): float (carry) against fixed,
    # within the fixed point's rounding plus 1e-6 of the entry's I
    for name, n_dep in (("mu", t.n_packets), ("image_batch", ref["n_deposits"])):
        a = getattr(fl, name).cpu().numpy().astype(np.float64)
        b = getattr(fx, name).cpu().numpy() * 2.0 ** -t.fx_shift
        tol = 1e-6 * np.abs(b[..., :1]) + n_dep * 2.0 ** -(t.fx_shift + 1)
        assert (np.abs(a - b) <= tol).all(), name


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


@pytest.mark.parametrize("name,limit", [("amr_point", None), ("hg_multi", None), ("table", None),
                                        ("amr_point", 1024)])
def test_cell_ordered_march_bit_exact(name, limit):
    """The queue marched sorted by starting cell (in scrambled groups of 32,
    the last group partly empty), also with a 1024-ray queue in chunks:
    records, int64 tallies and counters equal the oracle's."""
    from kratos_polrad_b200._lib import call
    from kratos_polrad_b200.mesh import PEEL_ORDER_AUTO, PEEL_ORDER_CELL
    mesh, sig, t = case(name)
    mesh.set_sigma(sig)
    mesh.set_peel_order(PEEL_ORDER_CELL)
    if limit:
        call("kp_mesh_peel_queue_limit", mesh.handle, limit)
    try:
        tal = forward(mesh, to_device(t))
        torch.cuda.synchronize()
        assert mesh.status() == 0
    finally:
        mesh.set_peel_order(PEEL_ORDER_AUTO)
        call("kp_mesh_peel_queue_limit", mesh.handle, 1 << 27)
    ref = run_oracle(mesh, sig, t)
    rec, rref = tal.record_array(), ref["records"]
    for f in rec.dtype.names:
        np.testing.assert_array_equal(rec[f], rref[f], err_msg=f)
    np.testing.assert_array_equal(tal.counters.cpu().numpy(), ref["counters"].astype(np.int64))
    np.testing.assert_array_equal(tal.image.cpu().numpy(), ref["image"])
    np.testing.assert_array_equal(tal.image_batch.cpu().numpy(), ref["image_batch"])


def test_cell_ordered_march_float_tallies_within_rounding():
    """Float tallies sum in another order when sorted: within 1e-6 of each
    pixel's I of the queue-ordered solve."""
    from kratos_polrad_b200.mesh import PEEL_ORDER_CELL, PEEL_ORDER_QUEUE
    mesh, sig, t = case("amr_point")
    mesh.set_sigma(sig)
    tf = dataclasses.replace(t, tally_mode=TALLY_FLOAT, n_record=0)
    out = []
    for order in (PEEL_ORDER_QUEUE, PEEL_ORDER_CELL):
        mesh.set_peel_order(order)
        out.append(forward(mesh, tf).image.cpu().numpy().astype(np.float64))
    torch.cuda.synchronize()
    a, b = out
    I = np.abs(a[..., :1])
    assert (a[..., 0] > 0).sum() > 200
    assert (np.abs(a - b) <= 1e-6 * I + 1e-30).all()


def test_peel_queue_limit_refuses_tiny_queue():
    from kratos_polrad_b200._lib import KP_ERR_CONFIG, KPError, call
    mesh, _, _ = case("slab")
    with pytest.raises(KPError) as e:
        call("kp_mesh_peel_queue_limit", mesh.handle, 100)
    assert e.value.code == KP_ERR_CONFIG
