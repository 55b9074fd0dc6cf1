"""The single-scattering quadrature (oracle/single_scatter.py) checked on its
own: its coarse image against a plain Monte-Carlo estimate of the same
integral (random directions about the source and random distances along
them, binned into the pixels), and the unscattered emission against its
closed form."""
import numpy as np

from oracle import single_scatter as ss

LO, HI = np.zeros(3), np.array([1.0, 1.0, 2.0])
SRC = np.array([0.43, 0.55, 0.8])


CENTER, HALF, N_PIX, BN = (0.5, 0.5, 1.0), 1.6, 32, 8


def _mc_image(sigma_s, sigma_a, inc, az, kind, g, pmax, n=4_000_000, seed=3):
    """Plain Monte-Carlo estimate of the first-scattering image (coarse,
    [BN, BN, 4]): random directions about the source, random distances along
    them, each sample binned into its pixel; and the standard error of I."""
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
    val = sigma_s * np.exp(-(sigma_s + sigma_a) * (r + l_out)) * f11 * R / n
    pix = 2 * HALF / N_PIX
    fx = np.floor((x - CENTER) @ eh / pix + N_PIX / 2).astype(int) * BN // N_PIX
    fy = np.floor((x - CENTER) @ ev / pix + N_PIX / 2).astype(int) * BN // N_PIX
    idx = fy * BN + fx
    img = np.stack([np.bincount(idx, weights=val * w, minlength=BN * BN)
                    for w in (1.0, p * (c * c - s * s), p * 2 * c * s)], 1)
    se = np.sqrt(np.bincount(idx, weights=(val * n) ** 2, minlength=BN * BN) / n) / np.sqrt(n)
    return img.reshape(BN, BN, 3), se.reshape(BN, BN)


def test_quadrature_matches_a_monte_carlo_estimate():
    """Coarse pixels (but the source's, where the 1 / r^2 peak sits) and their
    totals, I, Q and U, within 5 standard errors of the plain estimate."""
    for kind, inc, az, sig_s, sig_a, g, pmax in [("rayleigh", 90.0, 0.0, 0.6, 0.4, 0.0, 1.0),
                                                  ("hg", 60.0, 30.0, 0.9, 0.6, 0.6, 0.5)]:
        img = ss.single_scatter_image(LO, HI, SRC, sig_s, sig_a, inc, az, CENTER, HALF, N_PIX,
                                      kind=kind, g=g, p_max=pmax, n_sub=32, n_theta=40)
        quad = img.reshape(BN, N_PIX // BN, BN, N_PIX // BN, 4).sum((1, 3))[..., :3]
        mc, se = _mc_image(sig_s, sig_a, inc, az, kind, g, pmax)
        o, ev, eh = ss.observer_frame(inc, az)
        pix = 2 * HALF / N_PIX
        sp = tuple(int(np.floor((SRC - CENTER) @ e / pix + N_PIX / 2)) * BN // N_PIX
                   for e in (ev, eh))
        keep = quad[..., 0] > 2e-3 * quad[..., 0].max()
        keep[sp] = False
        err = np.abs(quad - mc)[keep]
        assert np.all(err <= 5 * se[keep][:, None] + 2e-3 * quad[..., 0][keep][:, None]), \
            (kind, err.max(0))
        tot_se = np.sqrt((se[keep] ** 2).sum())
        assert np.all(np.abs(quad[keep].sum(0) - mc[keep].sum(0)) <= 5 * tot_se
                      + 1e-3 * quad[keep][:, 0].sum()), (kind, quad[keep].sum(0), mc[keep].sum(0))
        if kind == "rayleigh":             # the check sees the polarization
            assert abs(quad[keep][:, 1].sum()) > 0.02 * quad[keep][:, 0].sum()


def test_unscattered_emission_in_the_source_pixel():
    img = ss.single_scatter_image(LO, HI, SRC, 0.0, 0.7, 90.0, 0.0, CENTER, HALF, N_PIX)
    # no scattering: only the emission, attenuated over the 0.57 to the x = 1 wall
    assert np.count_nonzero(img[..., 0]) == 1
    assert np.isclose(img[..., 0].sum(), np.exp(-0.7 * 0.57) / (4 * np.pi), rtol=1e-12)
