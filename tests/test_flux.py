"""The path-length flux tally of the polarized transport (rad_t::flx), on CPU.

The C restatement of the transport walk, run with zero coefficients, is held
against the reference's own cart_t::proc (compiled from the reference
sources, PRECISION=2) packet by packet; see straight_walks.py.  A second
check needs no reference: in the periodic slab a straight packet's path to
the top or bottom face has the length |z_face - z0| / |d_z|, so the tally's
volume-weighted sum is known in closed form.
"""
import dataclasses

import numpy as np
import pytest

import straight_walks as sw
from oracle import port, refharness
from transport_cases import case, oracle_inputs

pytestmark = pytest.mark.skipif(not (refharness.available(2) and port.available()),
                                reason="oracle libraries not built")


@pytest.mark.parametrize("name", sorted(sw.STRAIGHT))
def test_restated_flux_matches_reference_walk(name):
    mesh, sig, cfg = sw.setup(name)
    tab, grid, gn, cells = oracle_inputs(mesh, cfg)
    o = port.transport(tab, sig, grid, gn, cfg, cells, flux=True)
    rec = o["records"]
    assert (rec["n_scatter"] == 0).all()
    ref, perm, r, fix, start = sw.reference_walks(name, mesh, rec)
    clean, summary = sw.compare_walks(name, mesh, rec, r, fix)
    ours = sw.oracle_clean_flux(mesh, sig, cfg, clean)
    theirs = sw.reference_clean_flux(ref, start, clean)
    summary.update(sw.compare_flux(mesh, perm, ours, theirs))
    print(name, summary)
    # the clean and the shifted packets together are the whole solve
    rest = sw.oracle_clean_flux(mesh, sig, cfg, ~clean)
    np.testing.assert_array_equal(ours + rest, o["flux"])


def test_flux_path_length_closed_form():
    mesh, sig, cfg = sw.setup("slab")
    cfg = dataclasses.replace(cfg, n_packets=2000, n_record=2000)
    tab, grid, gn, cells = oracle_inputs(mesh, cfg)
    o = port.transport(tab, sig, grid, gn, cfg, cells, flux=True)
    rec = o["records"]
    esc = rec["status"] == 1
    z0 = cfg.sources[0].pos[2]
    dz = rec["d"][:, 2].astype(np.float64)
    length = np.where(dz > 0, (64.0 - z0) / np.where(dz > 0, dz, 1), z0 / np.where(dz < 0, -dz, 1))
    vol = np.repeat(tab.vol0, tab.cells_per_block)
    got = (o["flux"] * 2.0 ** -sw.FLUX_SHIFT * vol).sum()
    # capped packets walked max_steps segments of unknown total length: few
    assert (~esc).sum() < 0.05 * len(rec)
    capped = sw.oracle_clean_flux(mesh, sig, cfg, ~esc)
    got -= (capped * 2.0 ** -sw.FLUX_SHIFT * vol).sum()
    want = length[esc].sum()
    assert abs(got - want) <= 1e-9 * want, (got, want)


def test_flux_weights_follow_interactions():
    """With scattering and absorption the tally sums w * dl / volume with the
    weight along each segment: zero coefficients give zero weight loss, and
    halving sigma_abs's share leaves the unit-albedo path lengths alone."""
    mesh, sig, cfg = case("amr_point")
    cfg = dataclasses.replace(cfg, n_packets=300, n_record=300, flux=True, flux_fx_shift=24,
                              w_min=0.0)
    tab, grid, gn, cells = oracle_inputs(mesh, cfg)
    a = port.transport(tab, sig, grid, gn, cfg, cells, flux=True)
    # same packets with unit albedo: same walks (the albedo only weighs), so
    # the weighted tally is below the unit-weight one cell by cell
    sig1 = np.stack([sig.sum(1), np.zeros(len(sig), np.float32)], 1).astype(np.float32)
    ext_same = np.array_equal(sig1.sum(1), sig.sum(1))
    b = port.transport(tab, sig1, grid, gn, cfg, cells, flux=True)
    if ext_same:
        assert (a["flux"] <= b["flux"] + 1).all()
        assert a["flux"].sum() < b["flux"].sum()
    assert (a["flux"] >= 0).all() and a["flux"].sum() > 0
