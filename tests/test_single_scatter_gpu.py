"""The polarized transport against an independent calculation: the single-
scattering image of a point source in a uniform absorbing box.

With max_scatter = 1 every packet ends at its first interaction, after the
interaction's peel-off, so the expected image is exactly the first-scattering
integral that oracle/single_scatter.py evaluates by quadrature from the
physics (isotropic emission, exponential free paths, survival weighting by
the albedo, attenuation toward the observer, the Rayleigh or HG+polarization
phase matrix, the image frame), plus the unscattered emission.  None of it
shares code or arithmetic with the kernels or the C restatement.  Each coarse
pixel's I, Q and U (but the source's) must agree within 4 batch-means
standard errors plus 0.5 % of the pixel's intensity, and so must the image's
totals.

Russian roulette is checked the same way, as an invariance: with up to three
interactions, roulette below a weight of 0.5 changes no expectation, so the
images with and without it agree within their standard errors.
"""
import dataclasses

import numpy as np
import pytest
import torch

from kratos_polrad_b200 import Mesh, MeshConfig
from kratos_polrad_b200.transport import (EMIT_ISOTROPIC, PHASE_HG_POL, PHASE_RAYLEIGH,
                                          SOURCE_POINT, Source, Tallies, TransportConfig,
                                          forward)
from oracle import single_scatter as ss

pytestmark = pytest.mark.gpu

LO, HI = (0.0, 0.0, 0.0), (1.0, 1.0, 2.0)
SRC = (0.43, 0.55, 0.8)
# pixels of 0.1: the box's edges fall on pixel edges in the face-on view, so
# that no pixel is cut by the box's outline
CENTER, HALF, N_PIX, BN = (0.5, 0.5, 1.0), 1.6, 32, 8


def _box(sigma_s, sigma_a):
    mesh = Mesh(MeshConfig(LO, HI, (32, 32, 64), (16, 16, 16), (False, False, False)))
    sig = np.empty((mesh.n_cells, 2), np.float32)
    sig[:, 0], sig[:, 1] = sigma_s, sigma_a
    mesh.set_sigma(sig)
    return mesh


def _cfg(n, phase, inc, az, **kw):
    base = dict(n_packets=n, sources=[Source(SOURCE_POINT, EMIT_ISOTROPIC, SRC)], seed=11,
                phase=phase, image_n=N_PIX, inclination_deg=inc, azimuth_deg=az,
                image_center=CENTER, image_half_width=HALF, n_batches=32, image_batch_n=BN,
                w_min=0.0, max_scatter=1, fx_shift=32)
    base.update(kw)
    return TransportConfig(**base)


def _coarse_batches(tal):
    """Per-batch coarse images [batches, BN, BN, 4] in packet weight units."""
    return tal.image_batch.cpu().numpy().astype(np.float64) * tal.scale()


def _coarse(img):
    return img.reshape(BN, N_PIX // BN, BN, N_PIX // BN, 4).sum((1, 3))


@pytest.mark.parametrize("kind,inc,az,sigma_s,sigma_a", [
    ("rayleigh", 90.0, 0.0, 0.6, 0.4),
    ("hg", 60.0, 30.0, 0.9, 0.6),
])
def test_first_scattering_image_matches_quadrature(kind, inc, az, sigma_s, sigma_a):
    n = 8_000_000
    g, pmax = (0.6, 0.5) if kind == "hg" else (0.0, 1.0)
    mesh = _box(sigma_s, sigma_a)
    cfg = _cfg(n, PHASE_HG_POL if kind == "hg" else PHASE_RAYLEIGH, inc, az, hg_g=g, pol_max=pmax)
    tal = forward(mesh, cfg, Tallies(cfg))
    torch.cuda.synchronize()
    assert mesh.status() == 0
    c = tal.counts()
    assert c["emitted"] == n and c["capped"] > 0.3 * n       # ended at the first interaction
    b = _coarse_batches(tal)
    mc = b.sum(0)
    se = np.sqrt(b.shape[0]) * b.std(0, ddof=1)
    want = n * _coarse(ss.single_scatter_image(LO, HI, SRC, sigma_s, sigma_a, inc, az, CENTER, HALF,
                                               N_PIX, kind=kind, g=g, p_max=pmax, n_sub=32,
                                               n_theta=40))
    # the fine image sums to the coarse one
    np.testing.assert_allclose(_coarse(tal.image.cpu().numpy().astype(np.float64) * tal.scale()),
                               mc, rtol=1e-12, atol=1e-6)
    # pixels lit above 0.2 % of the brightest, the source's, which is left out:
    # it holds the unscattered emission, and the light scattered next to the
    # source, whose polarization the quadrature's pixel sampling resolves
    # worst, is part of it
    src_pix = np.unravel_index(np.argmax(want[..., 0]), want.shape[:2])
    lit = want[..., 0] > 2e-3 * want[..., 0].max()
    lit[src_pix] = False
    assert lit.sum() >= 8
    for q, name in enumerate("IQU"):
        err = np.abs(mc[..., q] - want[..., q])[lit]
        bar = (4 * se[..., q] + 5e-3 * np.abs(want[..., 0]))[lit]
        worst = np.argmax(err / bar)
        assert np.all(err <= bar), (name, err[worst], bar[worst], want[..., q][lit][worst])
    # the image-integrated polarization (but the source's pixel), a sharper
    # check of the frame
    keep = np.ones(want.shape[:2], bool)
    keep[src_pix] = False
    tot, tot_w = mc[keep].sum(0), want[keep].sum(0)
    tot_se = np.sqrt(b.shape[0]) * b[:, keep].sum(1).std(0, ddof=1)
    for q in range(3):
        assert abs(tot[q] - tot_w[q]) <= 4 * tot_se[q] + 2e-3 * tot_w[0], (q, tot, tot_w, tot_se)


def test_roulette_changes_no_expectation():
    n = 8_000_000
    mesh = _box(0.9, 0.6)
    base = _cfg(n, PHASE_HG_POL, 60.0, 30.0, hg_g=0.6, pol_max=0.5, max_scatter=3)
    runs = []
    for w_min in (0.0, 0.5):
        cfg = dataclasses.replace(base, w_min=w_min, rr_survive=0.1)
        tal = forward(mesh, cfg, Tallies(cfg))
        torch.cuda.synchronize()
        runs.append((tal.counts(), _coarse_batches(tal)))
    assert runs[0][0]["absorbed"] == 0 and runs[1][0]["absorbed"] > 0.1 * n
    (_, a), (_, b) = runs
    ta, tb = a.sum((1, 2)), b.sum((1, 2))                     # per-batch image totals
    diff = ta.sum(0) - tb.sum(0)
    se = np.sqrt(a.shape[0] * (ta.var(0, ddof=1) + tb.var(0, ddof=1)))
    assert np.all(np.abs(diff[:3]) <= 4 * se[:3]), (diff, se)
    lit = a.sum(0)[..., 0] > 0.02 * a.sum(0)[..., 0].max()
    da = a.sum(0)[..., 0] - b.sum(0)[..., 0]
    sa = np.sqrt(a.shape[0] * (a[..., 0].var(0, ddof=1) + b[..., 0].var(0, ddof=1)))
    assert np.mean(np.abs(da[lit]) <= 4 * sa[lit]) >= 0.98
