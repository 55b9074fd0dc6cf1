"""Multiple scattering against an independent Monte Carlo.

oracle/box_mc.py is a polarized Monte Carlo of a point source in a uniform
box written from the physics in vectorised numpy: its own RNG, analytic wall
distances instead of cells, explicit rotation angles for the Stokes frames,
the scattering matrix applied as a matrix.  Up to ten interactions per packet
at albedo 0.9, its peel-off image and the GPU's agree statistically: every
coarse pixel and the image totals, I, Q and U, within 4 combined
batch-means standard errors.  This holds the GPU's polarization transfer
between interactions (frame rotations, r12 and r33, the rejection sampling of
the scattering direction against the Stokes vector) to an implementation
that shares none of its code.
"""
import numpy as np
import pytest
import torch

from kratos_polrad_b200 import Mesh, MeshConfig
from kratos_polrad_b200.transport import (EMIT_ISOTROPIC, PHASE_HG_POL, PHASE_RAYLEIGH,
                                          SOURCE_POINT, Source, Tallies, TransportConfig,
                                          forward)
from oracle import box_mc

pytestmark = pytest.mark.gpu

LO, HI = (0.0, 0.0, 0.0), (1.0, 1.0, 2.0)
SRC = (0.43, 0.55, 0.8)
CENTER, HALF, N_PIX, BN = (0.5, 0.5, 1.0), 1.6, 32, 8


def _coarse(img):
    """[..., N_PIX, N_PIX, c] -> [..., BN, BN, c]"""
    s = img.shape
    return img.reshape(*s[:-3], BN, N_PIX // BN, BN, N_PIX // BN, s[-1]).sum((-4, -2))


@pytest.mark.parametrize("kind,inc,az", [("rayleigh", 90.0, 0.0), ("hg", 60.0, 30.0)])
def test_multiple_scattering_matches_an_independent_monte_carlo(kind, inc, az):
    sig_s, sig_a, n_max = 1.35, 0.15, 10
    g, pmax = (0.6, 0.5) if kind == "hg" else (0.0, 1.0)
    n_gpu, n_np = 8_000_000, 1_600_000
    mesh = Mesh(MeshConfig(LO, HI, (32, 32, 64), (16, 16, 16), (False, False, False)))
    sig = np.empty((mesh.n_cells, 2), np.float32)
    sig[:, 0], sig[:, 1] = sig_s, sig_a
    mesh.set_sigma(sig)
    cfg = TransportConfig(n_packets=n_gpu, sources=[Source(SOURCE_POINT, EMIT_ISOTROPIC, SRC)],
                          seed=21, phase=PHASE_HG_POL if kind == "hg" else PHASE_RAYLEIGH,
                          hg_g=g, pol_max=pmax, image_n=N_PIX, inclination_deg=inc,
                          azimuth_deg=az, image_center=CENTER, image_half_width=HALF,
                          n_batches=32, image_batch_n=BN, w_min=0.0, max_scatter=n_max,
                          fx_shift=30)
    tal = forward(mesh, cfg, Tallies(cfg))
    torch.cuda.synchronize()
    assert mesh.status() == 0 and tal.counts()["scatter"] > n_gpu
    gb = tal.image_batch.cpu().numpy().astype(np.float64)[..., :3] * tal.scale() / n_gpu
    nb = _coarse(box_mc.box_mc_image(LO, HI, SRC, sig_s, sig_a, inc, az, CENTER, HALF, N_PIX, n_np,
                                     n_max, kind=kind, g=g, p_max=pmax, n_batches=16,
                                     seed=5)) / n_np
    # per packet: means over the batches' packets, and their standard errors
    g_mean, n_mean = gb.sum(0), nb.sum(0)
    g_se = gb.std(0, ddof=1) * np.sqrt(gb.shape[0])
    n_se = nb.std(0, ddof=1) * np.sqrt(nb.shape[0])
    se = np.sqrt(g_se ** 2 + n_se ** 2)
    lit = n_mean[..., 0] > 2e-3 * n_mean[..., 0].max()
    assert lit.sum() >= 8
    for q, name in enumerate("IQU"):
        err = np.abs(g_mean[..., q] - n_mean[..., q])[lit]
        bar = 4 * se[..., q][lit] + 1e-9
        worst = np.argmax(err / bar)
        assert np.all(err <= bar), (name, err[worst], bar[worst], n_mean[..., q][lit][worst])
    tg, tn = gb.sum((1, 2)), nb.sum((1, 2))
    tse = np.sqrt(tg.std(0, ddof=1) ** 2 * tg.shape[0] + tn.std(0, ddof=1) ** 2 * tn.shape[0])
    assert np.all(np.abs(tg.sum(0) - tn.sum(0)) <= 4 * tse), (tg.sum(0), tn.sum(0), tse)
    # the polarization is seen, not lost in the noise
    assert np.abs(n_mean[..., 1][lit]).max() > 10 * n_se[..., 1][lit].mean()
