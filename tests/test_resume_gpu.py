"""Resumable packets: a per-call step budget (kp_transport_forward_resume).

The reference walks a packet for at most `step` segments per cycle
(photon::cart_t::proc, modules/particle/radiation/photon.h:104-125) and keeps
the pool's unfinished particles between cycles (types/particle_pool.h:
191-248).  Here a packet that uses up its budget is written out whole and a
later call continues it; the calls that carry every packet to its end must
give the tallies, counters, flux and final-state records of one uninterrupted
solve, bit for bit in fixed point.
"""
import dataclasses

import numpy as np
import pytest
import torch

from kratos_polrad_b200._lib import call
from kratos_polrad_b200.transport import (TALLY_FLOAT, Tallies, forward, forward_resume,
                                          packet_states)
from transport_cases import case, to_device

pytestmark = pytest.mark.gpu


def _setup(name, **over):
    mesh, sig, t = case(name)
    mesh.set_sigma(sig)
    t = to_device(dataclasses.replace(t, flux=True, max_steps=300, **over))
    return mesh, t


def _resumed_solve(mesh, t, budget, max_calls=200):
    """Calls with `budget` steps each until no packet is left; the first one
    emits t's packets, the later ones only resume.  Returns the tallies, the
    number of calls and the suspended-queue sizes."""
    tal = Tallies(t, n_cells=mesh.n_cells)
    tal, out = forward_resume(mesh, t, budget, tallies=tal)
    sizes = [int(out.shape[0])]
    rest = dataclasses.replace(t, n_packets=0)
    calls = 1
    while out.shape[0] > 0:
        assert calls < max_calls
        tal, out = forward_resume(mesh, rest, budget, resumed=out.clone(), tallies=tal)
        sizes.append(int(out.shape[0]))
        calls += 1
    torch.cuda.synchronize()
    assert mesh.status() == 0
    return tal, calls, sizes


def _assert_same(a, b, t):
    for name in ("counters", "flux", "mu", "image", "image_batch"):
        if name in ("mu",) and not t.n_mu_bins:
            continue
        if name in ("image", "image_batch") and not t.image_n:
            continue
        assert torch.equal(getattr(a, name), getattr(b, name)), name
    ra, rb = a.record_array(), b.record_array()
    for f in ra.dtype.names:
        np.testing.assert_array_equal(ra[f], rb[f], err_msg=f)


@pytest.mark.parametrize("name,budget", [("amr_point", 9), ("slab", 5), ("hg_multi", 13),
                                         ("table", 7)])
def test_budgeted_calls_equal_one_solve(name, budget):
    """amr_point, hg_multi and table have an image (walk + k_peel per call),
    slab has none (single-kernel walk); table's packets come from a caller's
    table; max_steps = 300 caps some packets in the same step as a budget."""
    mesh, t = _setup(name)
    full = forward(mesh, t, Tallies(t, n_cells=mesh.n_cells))
    torch.cuda.synchronize()
    assert mesh.status() == 0
    tal, calls, sizes = _resumed_solve(mesh, t, budget)
    assert calls > 3 and sizes[0] > 0
    _assert_same(tal, full, t)


@pytest.mark.parametrize("name,budget", [("amr_point", 9), ("hg_multi", 13)])
def test_budgeted_calls_in_cell_order(name, budget):
    """Every call's queue marched sorted by starting cell: same as one
    solve in queue order."""
    from kratos_polrad_b200.mesh import PEEL_ORDER_AUTO, PEEL_ORDER_CELL
    mesh, t = _setup(name)
    full = forward(mesh, t, Tallies(t, n_cells=mesh.n_cells))
    torch.cuda.synchronize()
    mesh.set_peel_order(PEEL_ORDER_CELL)
    try:
        tal, calls, _ = _resumed_solve(mesh, t, budget)
    finally:
        mesh.set_peel_order(PEEL_ORDER_AUTO)
    assert calls > 3
    _assert_same(tal, full, t)


def test_two_half_budget_calls():
    """The first call suspends every packet still walking after 150 of its
    300 segments; the second finishes them: same as one solve."""
    mesh, t = _setup("amr_point")
    full = forward(mesh, t, Tallies(t, n_cells=mesh.n_cells))
    tal, out = forward_resume(mesh, t, 150, tallies=Tallies(t, n_cells=mesh.n_cells))
    st = packet_states(out)
    assert len(st) > 0 and np.all(st["n_steps"] == 150)
    tal, out2 = forward_resume(mesh, dataclasses.replace(t, n_packets=0), 150, resumed=out,
                               tallies=tal)
    torch.cuda.synchronize()
    assert out2.shape[0] == 0 and mesh.status() == 0
    _assert_same(tal, full, t)


def test_resume_mixed_with_new_packets_and_chunks():
    """Each call resumes the previous call's packets and emits a new range of
    ids; a 1024-ray peel-off queue splits every call into chunks that cut
    across resumed and new packets."""
    mesh, t = _setup("amr_point")
    full = forward(mesh, t, Tallies(t, n_cells=mesh.n_cells))
    call("kp_mesh_peel_queue_limit", mesh.handle, 1024)
    tal = Tallies(t, n_cells=mesh.n_cells)
    out = None
    done = 0
    for k in range(200):
        n = (700, 500, 800)[k] if k < 3 else 0
        if n == 0 and out.shape[0] == 0:
            break
        c = dataclasses.replace(t, n_packets=n, packet_offset=done, n_record=0)
        tal, out = forward_resume(mesh, c, 11, resumed=out, tallies=tal)
        done += n
    torch.cuda.synchronize()
    assert out.shape[0] == 0 and done == t.n_packets and mesh.status() == 0
    # records: the calls' packet_offset differ; compare the tallies alone
    for name in ("counters", "flux", "mu", "image", "image_batch"):
        assert torch.equal(getattr(tal, name), getattr(full, name)), name


def test_budget_beyond_every_walk():
    mesh, t = _setup("slab")
    full = forward(mesh, t, Tallies(t, n_cells=mesh.n_cells))
    tal, out = forward_resume(mesh, t, 1 << 30, tallies=Tallies(t, n_cells=mesh.n_cells))
    torch.cuda.synchronize()
    assert out.shape[0] == 0
    _assert_same(tal, full, t)


def test_float_tallies_within_rounding():
    """Float atomics sum in another order across calls: within float rounding
    of the uninterrupted solve (the tallies carry their rounding error)."""
    mesh, t = _setup("amr_point", tally_mode=TALLY_FLOAT)
    full = forward(mesh, t, Tallies(t, n_cells=mesh.n_cells))
    tal, _, _ = _resumed_solve(mesh, t, 9)
    assert torch.equal(tal.counters, full.counters)
    for name in ("flux", "image", "mu"):
        a, b = getattr(tal, name).double(), getattr(full, name).double()
        tol = 1e-6 * b.abs().max().item()
        assert (a - b).abs().max().item() <= tol, name


def test_queue_overflow_is_reported():
    mesh, t = _setup("amr_point")
    with pytest.raises(RuntimeError, match="suspended"):
        forward_resume(mesh, t, 5, capacity=10)
    torch.cuda.synchronize()
    assert mesh.status() != 0          # queue overflow, read and cleared
    assert mesh.status() == 0
