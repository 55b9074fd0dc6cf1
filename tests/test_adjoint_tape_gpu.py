"""Taped forward solves and their gradients (kp_transport_forward_tape,
kp_transport_adjoint_tape) against the untaped entry points, bit for bit.

A taped solve is an ordinary forward solve that leaves each packet's
peel-off rays and their attenuation in the mesh, so that the gradient of
that solve skips the adjoint's first replay.  Its tallies must equal the
plain solve's and its gradients the full adjoint's (int64 tallies: no
tolerance), for several adjoint images per tape; the tape must be refused
once anything replaced it.
"""
import dataclasses

import numpy as np
import pytest
import torch

from kratos_polrad_b200._lib import KP_ERR_CONFIG, KPError
from kratos_polrad_b200.adjoint import adjoint
from kratos_polrad_b200.transport import Tallies, forward
from transport_cases import case

pytestmark = pytest.mark.gpu


def _adj(t, seed):
    a = np.random.default_rng(seed).normal(size=(t.image_n, t.image_n, 4)).astype(np.float32)
    return torch.tensor(a, device="cuda")


@pytest.mark.parametrize("name", ["amr_point", "hg_multi"])
def test_tape_matches_plain_solve_and_full_adjoint(name):
    mesh, sig, t = case(name)
    mesh.set_sigma(sig)
    plain = forward(mesh, t)
    taped = forward(mesh, t, Tallies(t), tape=True)
    torch.cuda.synchronize()
    assert taped.tape_id > 0 and mesh.tape_id() == taped.tape_id
    for k in ("mu", "image", "image_batch", "counters", "records"):
        assert torch.equal(getattr(taped, k), getattr(plain, k)), k
    t0 = dataclasses.replace(t, n_record=0)
    a1, a2 = _adj(t, 1), _adj(t, 2)
    tape1 = adjoint(mesh, t0, a1, 24, tape_id=taped.tape_id)
    tape2 = adjoint(mesh, t0, a2, 24, tape_id=taped.tape_id)      # same tape again
    torch.cuda.synchronize()
    assert mesh.status() == 0
    full1 = adjoint(mesh, t0, a1, 24)                               # replaces the tape
    full2 = adjoint(mesh, t0, a2, 24)
    torch.cuda.synchronize()
    assert mesh.tape_id() == 0
    for x, y in zip(tape1 + tape2, full1 + full2):
        assert torch.equal(x, y)


@pytest.mark.parametrize("name", ["amr_point", "hg_multi"])
def test_tape_in_cell_order(name):
    """A taped solve marched sorted by starting cell keeps that order for its
    gradient, even after the mesh's order changed: tallies equal the plain
    solve's and gradients the full adjoint's (queue order)."""
    from kratos_polrad_b200.mesh import PEEL_ORDER_AUTO, PEEL_ORDER_CELL, PEEL_ORDER_QUEUE
    mesh, sig, t = case(name)
    mesh.set_sigma(sig)
    plain = forward(mesh, t)
    try:
        mesh.set_peel_order(PEEL_ORDER_CELL)
        taped = forward(mesh, t, Tallies(t), tape=True)
        mesh.set_peel_order(PEEL_ORDER_QUEUE)
        t0 = dataclasses.replace(t, n_record=0)
        a1 = _adj(t, 1)
        tape1 = adjoint(mesh, t0, a1, 24, tape_id=taped.tape_id)
        torch.cuda.synchronize()
        assert mesh.status() == 0
        full1 = adjoint(mesh, t0, a1, 24)
        torch.cuda.synchronize()
    finally:
        mesh.set_peel_order(PEEL_ORDER_AUTO)
    for k in ("mu", "image", "image_batch", "counters", "records"):
        assert torch.equal(getattr(taped, k), getattr(plain, k)), k
    for x, y in zip(tape1, full1):
        assert torch.equal(x, y)


def test_tape_is_dropped_by_new_coefficients_and_later_solves():
    mesh, sig, t = case("amr_point")
    t = dataclasses.replace(t, n_record=0)
    mesh.set_sigma(sig)
    tid = forward(mesh, t, tape=True).tape_id
    assert tid > 0
    mesh.set_sigma(sig)                                             # same values, new upload
    assert mesh.tape_id() == 0
    with pytest.raises(KPError) as e:
        adjoint(mesh, t, _adj(t, 3), 24, tape_id=tid)
    assert e.value.code == KP_ERR_CONFIG
    tid2 = forward(mesh, t, tape=True).tape_id
    assert tid2 > tid
    forward(mesh, t)                                                # an untaped solve
    assert mesh.tape_id() == 0
    # a cfg that is not the taped solve's
    tid3 = forward(mesh, t, tape=True).tape_id
    with pytest.raises(KPError) as e:
        adjoint(mesh, dataclasses.replace(t, seed=t.seed + 1), _adj(t, 3), 24, tape_id=tid3)
    assert e.value.code == KP_ERR_CONFIG


def test_tape_with_overflowing_queue_matches_full_adjoint():
    """A 1024-ray queue and a thick slab (vertical tau 20, albedo 1: far more
    than 12 rays per packet): the taped solve flags the packets whose rays
    found the queue full, and their gradients come from k_adjoint.  Taped
    tallies equal the plain solve's, tape gradients the full adjoint's."""
    from kratos_polrad_b200._lib import call
    mesh, sig, t = case("slab")
    sig = sig * 10.0
    t = dataclasses.replace(t, n_packets=85, n_record=0, image_n=16, inclination_deg=60.0,
                            image_center=(16.0, 16.0, 8.0), image_half_width=24.0)
    mesh.set_sigma(sig)
    call("kp_mesh_peel_queue_limit", mesh.handle, 1024)
    try:
        plain = forward(mesh, t)
        taped = forward(mesh, t, Tallies(t), tape=True)
        torch.cuda.synchronize()
        assert taped.tape_id > 0
        for k in ("mu", "image", "image_batch", "counters"):
            assert torch.equal(getattr(taped, k), getattr(plain, k)), k
        # every interaction projects into the image (it covers the slab), so
        # more rays than the queue holds: some packets were flagged
        assert int(plain.counters[2]) > 1024
        a = _adj(t, 5)
        tape = adjoint(mesh, t, a, 24, tape_id=taped.tape_id)
        full = adjoint(mesh, t, a, 24)
        torch.cuda.synchronize()
        assert mesh.status() == 0
    finally:
        call("kp_mesh_peel_queue_limit", mesh.handle, 1 << 27)
    for x, y in zip(tape, full):
        assert torch.equal(x, y)


def test_tape_in_float_mode_close_to_full_adjoint():
    """Float tallies accumulate with float atomics in any order, so the taped
    solve and its gradients agree with the untaped ones to float rounding:
    within 1e-5 of the largest value (the int64 comparison above is exact)."""
    from kratos_polrad_b200.transport import TALLY_FLOAT
    mesh, sig, t = case("amr_point")
    t = dataclasses.replace(t, n_record=0, tally_mode=TALLY_FLOAT)
    mesh.set_sigma(sig)
    plain = forward(mesh, t)
    taped = forward(mesh, t, Tallies(t), tape=True)
    a = _adj(t, 6)
    tape = adjoint(mesh, t, a, 24, tape_id=taped.tape_id)
    full = adjoint(mesh, t, a, 24)
    torch.cuda.synchronize()
    assert taped.tape_id > 0 and mesh.status() == 0
    assert torch.equal(taped.counters, plain.counters)
    for x, y in [(taped.image, plain.image)] + list(zip(tape, full)):
        x, y = x.double(), y.double()
        assert (x - y).abs().max() <= 1e-5 * y.abs().max()
