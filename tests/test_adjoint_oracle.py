"""Path-replay adjoint (oracle restatement) vs common-random-number finite
differences.

With tau-threshold sampling the interaction points move with sigma, so a
CRN finite difference of the Monte-Carlo estimator jumps whenever a point
crosses a cell face into a cell of another albedo, a pixel boundary or a
roulette threshold; such jumps make its variance grow like 1/h.  The check
therefore uses perturbations that keep the estimator continuous (scaling the
extinction uniformly keeps every albedo fixed; one image pixel; no
roulette) and compares the two estimates of the same derivative of the
expectation with their batch-means error bars: 32 independent packet
batches, |FD - adjoint| < 4 combined standard errors, and the adjoint's
relative error below 2%.
"""
import concurrent.futures as cf
import dataclasses

import numpy as np
import pytest

from kratos_polrad_b200 import Mesh, MeshConfig
from kratos_polrad_b200.transport import EMIT_ISOTROPIC, SOURCE_POINT, Source, TransportConfig
from oracle import port
from transport_cases import oracle_inputs

pytestmark = pytest.mark.skipif(not port.available(), reason="oracle not built")


def _scene(image_n=1, w_min=0.0):
    mesh = Mesh(MeshConfig((0, 0, 0), (1, 1, 1), (16, 16, 16), (8, 8, 8), (False,) * 3))
    rng = np.random.default_rng(4)
    rho = np.exp(0.5 * rng.normal(size=mesh.n_cells))
    ext = 2.0 * rho / rho.mean()
    sig = np.stack([0.9 * ext, 0.1 * ext], 1).astype(np.float32)
    t = TransportConfig(n_packets=3000, sources=[Source(SOURCE_POINT, EMIT_ISOTROPIC, (0.5, 0.5, 0.5))],
                        seed=4, image_n=image_n, inclination_deg=60.0, image_center=(0.5, 0.5, 0.5),
                        image_half_width=0.8, w_min=w_min)
    adj = rng.normal(size=(image_n, image_n, 4)).astype(np.float32)
    if image_n == 1:                     # loss weighted toward the image intensity
        adj[...] = (1.0, 0.3, 0.3, 0.0)
    return mesh, sig, t, adj


def _batches(mesh, sig, t, adj, direction, h, n_batches=32):
    tab, grid, n, cells = oracle_inputs(mesh, t)

    def one(k):
        tk = dataclasses.replace(t, packet_offset=k * t.n_packets)

        def loss(s):
            img = port.transport(tab, s, grid, n, tk, cells)["image"] * 2.0 ** -32
            return float((img * adj).sum())
        fd = (loss((sig * (1 + h * direction)).astype(np.float32))
              - loss((sig * (1 - h * direction)).astype(np.float32))) / (2 * h)
        gl, gi, _ = port.adjoint(tab, sig, grid, n, tk, cells, adj, 24)
        g_sca, g_abs = (gl + gi) * 2.0 ** -24, gl * 2.0 ** -24
        ad = float((g_sca * sig[:, 0] * direction[:, 0]).sum()
                   + (g_abs * sig[:, 1] * direction[:, 1]).sum())
        return fd, ad
    with cf.ThreadPoolExecutor(8) as ex:
        return np.array(list(ex.map(one, range(n_batches))))


@pytest.mark.parametrize("which", ["extinction", "absorption_share"])
def test_adjoint_matches_crn_finite_differences(which):
    mesh, sig, t, adj = _scene()
    if which == "extinction":            # scale both coefficients: albedo unchanged
        d = np.ones(sig.shape)
    else:                                # shift extinction between the two, uniformly
        d = np.stack([-np.ones(len(sig)), 9 * np.ones(len(sig))], 1)
    r = _batches(mesh, sig, t, adj, d, h=1e-2)
    fd, ad = r[:, 0], r[:, 1]
    se = lambda v: v.std(ddof=1) / np.sqrt(len(v))
    assert se(ad) < 0.02 * abs(ad.mean())
    assert abs(fd.mean() - ad.mean()) < 4 * np.hypot(se(fd), se(ad)), (fd.mean(), ad.mean())


def test_adjoint_single_cells_with_image_and_roulette():
    """Cells next to the source, 16x16 image, roulette on: a 5% single-cell
    perturbation, batch-means comparison as above."""
    mesh, sig, t, adj = _scene(image_n=16, w_min=0.01)
    tab, grid, n, cells = oracle_inputs(mesh, t)
    gl, gi, _ = port.adjoint(tab, sig, grid, n, dataclasses.replace(t, n_packets=20000), cells, adj, 24)
    top = np.argsort(-np.abs((gl + gi).astype(np.float64)))[:3]
    for ci in top:
        d = np.zeros(sig.shape)
        d[ci, 0] = 1.0
        r = _batches(mesh, sig, t, adj, d, h=5e-2, n_batches=24)
        fd, ad = r[:, 0], r[:, 1]
        se = lambda v: v.std(ddof=1) / np.sqrt(len(v))
        assert abs(fd.mean() - ad.mean()) < 4 * np.hypot(se(fd), se(ad)) + 0.05 * abs(ad.mean())
