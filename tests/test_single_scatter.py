"""The single-scattering quadrature (oracle/single_scatter.py) checked on its
own: its image totals against a plain Monte-Carlo estimate of the same
integral (random directions about the source and random distances along
them), and the unscattered emission against its closed form."""
import numpy as np

from oracle import single_scatter as ss

LO, HI = np.zeros(3), np.array([1.0, 1.0, 2.0])
SRC = np.array([0.43, 0.55, 0.8])


def _mc_totals(sigma_s, sigma_a, inc, az, kind, g, pmax, n=2_000_000, seed=3):
    rng = np.random.default_rng(seed)
    o, ev, eh = ss.observer_frame(inc, az)
    e2 = np.cross(o, ev)
    z = rng.uniform(-1, 1, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    st = np.sqrt(1 - z * z)
    k = np.stack([st * np.cos(ph), st * np.sin(ph), z], 1)
    R = ss.wall_distance(SRC, k, LO, HI)
    r = rng.uniform(0, 1, n) * R
    x = SRC + r[:, None] * k
    l_out = ss.exit_length(x, o, LO, HI)
    f11, p = ss.phase(kind, k @ o, g, pmax)
    nvec = np.cross(k, o)
    nn = np.linalg.norm(nvec, axis=1)
    c, s = (nvec @ ev) / nn, (nvec @ e2) / nn
    # density of (direction, distance): 1 / (4 pi R); integrand sigma_s e^-.. f11 / (4 pi)
    val = sigma_s * np.exp(-(sigma_s + sigma_a) * (r + l_out)) * f11 * R
    return np.array([val.mean(), (val * p * (c * c - s * s)).mean(),
                     (val * p * 2 * c * s).mean()]), val.std() / np.sqrt(n)


def test_quadrature_totals_match_a_monte_carlo_estimate():
    for kind, inc, az, sig_s, sig_a, g, pmax in [("rayleigh", 90.0, 0.0, 0.6, 0.4, 0.0, 1.0),
                                                  ("hg", 60.0, 30.0, 0.9, 0.6, 0.6, 0.5)]:
        img = ss.single_scatter_image(LO, HI, SRC, sig_s, sig_a, inc, az, (0.5, 0.5, 1.0), 3.0, 32,
                                      kind=kind, g=g, p_max=pmax)
        o, _, _ = ss.observer_frame(inc, az)
        direct = np.exp(-(sig_s + sig_a) * ss.exit_length(SRC[None], o, LO, HI)[0]) / (4 * np.pi)
        quad = img.sum((0, 1))[:3] - np.array([direct, 0.0, 0.0])
        mc, se = _mc_totals(sig_s, sig_a, inc, az, kind, g, pmax)
        assert np.all(np.abs(quad - mc) <= 5 * se + 1e-4 * quad[0]), (kind, quad, mc, se)
        if kind == "rayleigh":             # the check sees the polarization
            assert abs(quad[1]) > 0.02 * quad[0]


def test_unscattered_emission_in_the_source_pixel():
    img = ss.single_scatter_image(LO, HI, SRC, 0.0, 0.7, 90.0, 0.0, (0.5, 0.5, 1.0), 1.3, 32)
    # no scattering: only the emission, attenuated over the 0.57 to the x = 1 wall
    assert np.count_nonzero(img[..., 0]) == 1
    assert np.isclose(img[..., 0].sum(), np.exp(-0.7 * 0.57) / (4 * np.pi), rtol=1e-12)
