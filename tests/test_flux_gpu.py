"""The path-length flux tally of k_forward (rad_t::flx) on the GPU.

With scattering, absorption and peel-off on, the GPU's int64 flux equals the
C restatement's bit for bit on every launch path: the single-kernel walk
(no image), the deferred walk with its peel-off queue, a queue too small for
the chunk (rays marched inline), and the taped solve.  With zero
coefficients the GPU walk is held packet by packet against the reference's
own cart_t::proc (straight_walks.py): every packet that the reference's
geo_loc_t::fix leaves alone takes the same cells, and the flux of those
packets, run on the GPU, matches the reference's within the stated bar.
"""
import dataclasses

import numpy as np
import pytest
import torch

import straight_walks as sw
from kratos_polrad_b200._lib import call
from kratos_polrad_b200.transport import TALLY_FLOAT, Tallies, forward
from oracle import port, refharness
from transport_cases import case, oracle_inputs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not port.available(), reason="oracle not built")]


def _flux_case(name):
    mesh, sig, t = case(name)
    return mesh, sig, dataclasses.replace(t, flux=True, flux_fx_shift=24)


def _oracle(mesh, sig, t):
    tab, grid, gn, cells = oracle_inputs(mesh, t)
    return port.transport(tab, sig, grid, gn, t, cells, flux=True)


def _assert_same(tal, ref, t):
    rec, rref = tal.record_array(), ref["records"]
    for f in rec.dtype.names:
        np.testing.assert_array_equal(rec[f], rref[f], err_msg=f)
    np.testing.assert_array_equal(tal.counters.cpu().numpy(), ref["counters"].astype(np.int64))
    if t.n_mu_bins:
        np.testing.assert_array_equal(tal.mu.cpu().numpy(), ref["mu"])
    if t.image_n:
        np.testing.assert_array_equal(tal.image.cpu().numpy(), ref["image"])
        np.testing.assert_array_equal(tal.image_batch.cpu().numpy(), ref["image_batch"])
    np.testing.assert_array_equal(tal.flux.cpu().numpy(), ref["flux"])


@pytest.mark.parametrize("name", ["slab", "amr_point", "hg_multi"])
def test_flux_bit_exact_with_scattering(name):
    mesh, sig, t = _flux_case(name)
    mesh.set_sigma(sig)
    tal = forward(mesh, t)
    torch.cuda.synchronize()
    assert mesh.status() == 0
    ref = _oracle(mesh, sig, t)
    assert ref["flux"].sum() > 0
    _assert_same(tal, ref, t)


@pytest.mark.parametrize("name", ["amr_point", "hg_multi"])
def test_flux_with_small_peel_queue(name):
    mesh, sig, t = _flux_case(name)
    mesh.set_sigma(sig)
    call("kp_mesh_peel_queue_limit", mesh.handle, 1024)
    try:
        tal = forward(mesh, t)
        torch.cuda.synchronize()
        assert mesh.status() == 0
    finally:
        call("kp_mesh_peel_queue_limit", mesh.handle, 1 << 27)
    _assert_same(tal, _oracle(mesh, sig, t), t)


def test_flux_of_taped_solve():
    mesh, sig, t = _flux_case("amr_point")
    mesh.set_sigma(sig)
    tal = forward(mesh, t, tape=True)
    torch.cuda.synchronize()
    assert tal.tape_id > 0
    _assert_same(tal, _oracle(mesh, sig, t), t)


def test_flux_float_mode_close_to_fixed():
    """Float atomics sum the same deposits in another order: per cell within
    the float summation bound (2e-6 relative for the few hundred deposits a
    cell of this case receives), the total within 1e-6."""
    mesh, sig, t = _flux_case("amr_point")
    mesh.set_sigma(sig)
    fx = forward(mesh, dataclasses.replace(t, n_record=0))
    fl = forward(mesh, dataclasses.replace(t, n_record=0, tally_mode=TALLY_FLOAT))
    torch.cuda.synchronize()
    a = fx.flux_values()
    b = fl.flux_values()
    assert a.sum() > 0
    np.testing.assert_allclose(b, a, rtol=2e-6, atol=1e-6 * np.abs(a).max())
    assert abs(b.sum() - a.sum()) <= 1e-6 * a.sum()


@pytest.mark.skipif(not refharness.available(2), reason="reference walk not built")
@pytest.mark.parametrize("name", sorted(sw.STRAIGHT))
def test_gpu_flux_matches_reference_walk(name):
    mesh, sig, t = sw.setup(name)
    mesh.set_sigma(sig)
    tal = forward(mesh, t)
    torch.cuda.synchronize()
    assert mesh.status() == 0
    _assert_same(tal, _oracle(mesh, sig, t), t)          # the GPU is the restatement
    rec = tal.record_array()
    ref, perm, r, fix, start = sw.reference_walks(name, mesh, rec)
    clean, summary = sw.compare_walks(name, mesh, rec, r, fix)
    # the GPU's flux over exactly the packets the reference walks alike
    part = Tallies(t, n_cells=mesh.n_cells)
    for a, b in sw.clean_runs(clean):
        forward(mesh, dataclasses.replace(t, packet_offset=a, n_packets=b - a, n_record=0), part)
    torch.cuda.synchronize()
    summary.update(sw.compare_flux(mesh, perm, part.flux.cpu().numpy(),
                                   sw.reference_clean_flux(ref, start, clean)))
    print(name, summary)
