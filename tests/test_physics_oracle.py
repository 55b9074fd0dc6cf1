"""Physics primitives of the oracle against published values and analytics.

The device code reproduces these primitives bit for bit (checked through
the full transport on the GPU), so these CPU checks cover both.
"""
import ctypes

import numpy as np
import pytest

from oracle import port

pytestmark = pytest.mark.skipif(not port.available(), reason="oracle not built")


def _lib():
    L = port.lib()
    L.kpo_philox.argtypes = [ctypes.c_void_p] * 3
    L.kpo_log_exp.argtypes = [ctypes.c_long] + [ctypes.c_void_p] * 3
    L.kpo_scatter_sample.argtypes = [ctypes.c_long, ctypes.c_uint32, ctypes.c_int, ctypes.c_float,
                                     ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                     ctypes.c_void_p]
    return L


# Known-answer vectors of Philox4x32-10 published with Random123
# (Salmon et al., SC'11): (counter, key) -> output.
KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(ctr, key, want):
    L = _lib()
    c = np.array(ctr, np.uint32)
    k = np.array(key, np.uint32)
    out = np.zeros(4, np.uint32)
    L.kpo_philox(c.ctypes.data, k.ctypes.data, out.ctypes.data)
    assert tuple(int(v) for v in out) == want


def test_log_exp_accuracy():
    L = _lib()
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.random(20000), 2.0 ** -np.arange(1, 25),
                        rng.random(5000) * 60, [1e-30, 0.5, 1.0, 2.0]])
    ln, ex = np.zeros_like(x), np.zeros_like(x)
    L.kpo_log_exp(len(x), x.ctypes.data, ln.ctypes.data, ex.ctypes.data)
    np.testing.assert_allclose(ln, np.log(x), rtol=4e-16, atol=4e-16)
    np.testing.assert_allclose(ex, np.exp(-x), rtol=4e-15, atol=0)


def _scatter(n, kind, g=0.0, pmax=1.0, q=0.0, u=0.0, v=0.0, seed=3):
    L = _lib()
    out = np.zeros((n, 9), np.float32)
    L.kpo_scatter_sample(n, seed, kind, g, pmax, q, u, v, out.ctypes.data)
    return out.astype(np.float64)


def test_rayleigh_unpolarized_angles_and_polarization():
    n = 200000
    o = _scatter(n, 0)
    d, e1, S = o[:, :3], o[:, 3:6], o[:, 6:]
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1, atol=1e-6)
    np.testing.assert_allclose(np.einsum("ij,ij->i", d, e1), 0, atol=1e-6)
    mu = d[:, 2]
    # p(mu) = 3/8 (1 + mu^2): moments <mu^2> = 2/5, <mu> = 0
    assert abs(mu.mean()) < 0.01
    assert abs((mu ** 2).mean() - 0.4) < 0.005
    # scattered polarization in the scattering-plane frame: q = (mu^2-1)/(1+mu^2)
    np.testing.assert_allclose(S[:, 0], (mu ** 2 - 1) / (1 + mu ** 2), atol=2e-6)
    np.testing.assert_allclose(S[:, 1:], 0, atol=1e-6)


def test_rayleigh_polarized_azimuth():
    # Incoming light fully polarized along e1 (= +x): scattering into the
    # plane perpendicular to the polarization is favoured: the intensity is
    # (1+mu^2) - (1-mu^2) cos 2phi, so <cos 2phi> < 0 and <d_x^2> < <d_y^2>.
    o = _scatter(200000, 0, q=1.0)
    d = o[:, :3]
    # exact: <dx^2> = 1/5, <dy^2> = 2/5 for dipole scattering of x-polarized light
    assert abs((d[:, 0] ** 2).mean() - 0.2) < 0.005
    assert abs((d[:, 1] ** 2).mean() - 0.4) < 0.005


@pytest.mark.parametrize("g", [0.3, 0.6, -0.4])
def test_hg_mean_cosine(g):
    o = _scatter(200000, 1, g=g, pmax=0.5)
    mu = o[:, 2]
    assert abs(mu.mean() - g) < 0.006
    # polarization at 90 degrees: -pmax (1-mu^2)/(1+mu^2) for unpolarized light
    m = np.abs(mu) < 0.05
    np.testing.assert_allclose(o[m, 6], -0.5 * (1 - mu[m] ** 2) / (1 + mu[m] ** 2), atol=3e-6)


def test_packet_table_emission_restatement():
    """Packets from a caller's table start where the table says: with zero
    coefficients each walks straight from its entry, its record keeps the
    entry's direction, weight and Stokes vector, and located and given
    blocks agree."""
    import dataclasses
    import sys, os
    sys.path.insert(0, os.path.dirname(__file__))
    from transport_cases import case, run_oracle
    mesh, sig, t = case("table")
    t = dataclasses.replace(t, image_n=0, n_mu_bins=0)
    o = run_oracle(mesh, np.zeros_like(sig), t)
    rec, tab = o["records"], t.packets
    np.testing.assert_array_equal(rec["d"], tab["d"])
    np.testing.assert_array_equal(rec["w"], tab["w"])
    np.testing.assert_array_equal(rec["stokes"], tab["stokes"])
    assert (rec["status"] == 1).all() and (rec["n_scatter"] == 0).all()
    # every packet left along its straight line from the entry's position,
    # through the boundary
    lo, hi = np.array(mesh.x_min), np.array(mesh.x_max)
    assert (np.isclose(rec["x"], lo, atol=1e-12) | np.isclose(rec["x"], hi, atol=1e-12)).any(1).all()
    r = rec["x"] - tab["x"]
    cr = np.cross(r, tab["d"].astype(np.float64))
    assert np.abs(cr).max() < 1e-6
    # the same packets with every block left to the device: same walks
    t2 = dataclasses.replace(t, packets=tab.copy())
    t2.packets["ib"] = -1
    o2 = run_oracle(mesh, np.zeros_like(sig), t2)
    np.testing.assert_array_equal(o2["records"], rec)
