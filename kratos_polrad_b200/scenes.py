"""Synthetic problem set-ups (the counterpart of the reference's user problem
generator, src/user/probgen.cpp:8-22, whose default ``prob::run`` is empty).

Each builder returns ``(mesh, sigma2, TransportConfig)`` where ``sigma2`` is
the per-cell (sigma_sca, sigma_abs) array in block-id, x-fastest order.
All inputs are seeded synthetic fields; no external dataset is involved.
"""
from __future__ import annotations

import math

import numpy as np

from . import problems
from .mesh import Mesh, MeshConfig, RefineRegion
from .problems import clump_mesh_config, root_refine_boxes  # noqa: F401  (re-exported)
from .transport import (EMIT_ISOTROPIC, EMIT_UP_UNIFORM, PHASE_HG_POL, PHASE_RAYLEIGH,
                        SOURCE_PLANE_BASE, SOURCE_POINT, Source, TransportConfig)


def cell_centers(mesh: Mesh) -> np.ndarray:
    """Cell-centre coordinates [n_cells, 3] in the mesh's cell order."""
    xf0, dx0, _, _ = mesh.geometry(8)
    nc = mesh.nc
    k, j, i = np.meshgrid(np.arange(nc[2]), np.arange(nc[1]), np.arange(nc[0]), indexing="ij")
    idx = np.stack([i.ravel(), j.ravel(), k.ravel()], 1) + 0.5
    return (xf0[:, None, :] + idx[None] * dx0[:, None, :]).reshape(-1, 3)


def clump_amr(n_packets=10_000_000, n_root=128, block=16, peak=100.0, fwhm=0.1, tau_edge=5.0,
              albedo=(0.5, 0.99), seed=2, image_n=128, inclination=90.0):
    """Static 2-level AMR clump (see problems.clump_spec): the mesh, its
    per-cell coefficients and the transport configuration."""
    mcfg, sigma_of, cfg = problems.clump_spec(n_packets, n_root, block, peak, fwhm, tau_edge,
                                              albedo, seed, image_n, inclination)
    mesh = Mesh(mcfg)
    return mesh, sigma_of(cell_centers(mesh)), cfg


def slab(n_packets=1_000_000, nx=128, ny=128, nz=64, block=16, tau=10.0, seed=1, n_mu=20):
    """Plane-parallel electron-scattering slab: periodic in x, y; albedo 1;
    Thomson (Rayleigh) phase matrix; vertical optical depth tau; unpolarized
    packets from the base with mu uniform in (0, 1]; escaping I,Q,U,V in
    n_mu bins of mu in [0, 1]."""
    mesh = Mesh(MeshConfig((0, 0, 0), (nx, ny, nz), (nx, ny, nz), (block,) * 3,
                           (True, True, False)))
    sigma2 = np.zeros((mesh.n_cells, 2), np.float32)
    sigma2[:, 0] = tau / nz
    cfg = TransportConfig(n_packets=n_packets, seed=seed,
                          sources=[Source(SOURCE_PLANE_BASE, EMIT_UP_UNIFORM)],
                          phase=PHASE_RAYLEIGH, n_mu_bins=n_mu, mu_lo=0.0, mu_hi=1.0,
                          n_batches=32, fx_shift=24)
    return mesh, sigma2, cfg


def tangential_polarization(img_iquv: np.ndarray, centres=None) -> float:
    """Intensity-weighted tangential polarization of an image about its centre:
    sum(-Q cos 2phi + U sin 2phi) / sum(I), phi the pixel's position angle
    from the vertical toward the horizontal image axis (positive for the
    centrosymmetric pattern of scattered light).  The image's Stokes frame is
    e1 = vertical, e2 = -horizontal, hence the sign of the U term.  With
    ``centres`` ([k, 2] (vertical, horizontal) offsets from the image centre
    in pixels, source_pixels) phi is taken about the nearest of them: the
    pattern around several sources."""
    n = img_iquv.shape[0]
    c = (np.arange(n) + 0.5) - n / 2
    Y, X = np.meshgrid(c, c, indexing="ij")
    if centres is not None:
        cen = np.asarray(centres, np.float64)
        d2 = (Y[..., None] - cen[:, 0]) ** 2 + (X[..., None] - cen[:, 1]) ** 2
        near = cen[d2.argmin(-1)]
        Y, X = Y - near[..., 0], X - near[..., 1]
    phi = np.arctan2(X, Y)
    I, Q, U = (img_iquv[..., k].astype(np.float64) for k in range(3))
    return float((-Q * np.cos(2 * phi) + U * np.sin(2 * phi)).sum() / max(I.sum(), 1e-300))


def source_pixels(cfg, n: int) -> np.ndarray:
    """Image positions of cfg's point sources on an n x n image of the
    observer cfg names: [k, 2] (vertical, horizontal) offsets from the image
    centre in pixels, the projection the peel-off uses (image vertical = the
    projection of +z, horizontal = vertical x observer direction)."""
    inc, az = math.radians(cfg.inclination_deg), math.radians(cfg.azimuth_deg)
    o = np.array([math.sin(inc) * math.cos(az), math.sin(inc) * math.sin(az), math.cos(inc)])
    ev = np.array([-math.cos(inc) * math.cos(az), -math.cos(inc) * math.sin(az), math.sin(inc)])
    eh = np.cross(ev, o)
    r = np.array([s.pos for s in cfg.sources], np.float64) - np.asarray(cfg.image_center)
    inv_pix = n / (2.0 * cfg.image_half_width)
    return np.stack([r @ ev * inv_pix, r @ eh * inv_pix], 1)


def batch_rel_error(batch_images: np.ndarray, centres=None) -> tuple[float, float]:
    """Tangential polarization (about ``centres``, else the image centre) and
    its batch-means relative std-error from per-batch coarse images
    [n_batches, bn, bn, 4]."""
    p = np.array([tangential_polarization(b, centres) for b in batch_images])
    tot = tangential_polarization(batch_images.sum(0), centres)
    err = p.std(ddof=1) / math.sqrt(len(p))
    return tot, (err / abs(tot) if tot != 0 else float("inf"))


def batched_cubes(n_scenes=256, sides=(16, 32, 48, 64, 96), tau=(0.1, 20.0), albedo=(0.3, 1.0),
                  packets=(100_000, 1_000_000), seed=3, n_mu=32, block=16):
    """Independent uniform cubes for a batched solve: side drawn uniformly from
    ``sides`` (cells), centre-to-face extinction depth log-uniform in ``tau``,
    albedo uniform in ``albedo`` (seed ``seed``), a central isotropic point
    source, and packets in proportion to tau, clipped to ``packets``.
    Returns (scenes, cfg): scenes is a list of (mesh, sigma2, n_packets,
    stream_id, Source); cfg the common TransportConfig (32-bin mu tallies)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        side = int(rng.choice(sides))
        t = float(np.exp(rng.uniform(np.log(tau[0]), np.log(tau[1]))))
        alb = float(rng.uniform(*albedo))
        n = int(np.clip(round(packets[1] * t / tau[1]), packets[0], packets[1]))
        mesh = Mesh(MeshConfig((0, 0, 0), (1, 1, 1), (side,) * 3, (block,) * 3, (False,) * 3))
        ext = 2.0 * t                      # unit box: centre-to-face depth t
        sigma2 = np.empty((mesh.n_cells, 2), np.float32)
        sigma2[:, 0] = ext * alb
        sigma2[:, 1] = ext * (1.0 - alb)
        out.append((mesh, sigma2, n, k, Source(SOURCE_POINT, EMIT_ISOTROPIC, (0.5, 0.5, 0.5))))
    cfg = TransportConfig(n_packets=0, sources=[Source()], seed=seed, phase=PHASE_RAYLEIGH,
                          n_mu_bins=n_mu, mu_lo=-1.0, mu_hi=1.0, n_batches=32, w_min=0.01,
                          fx_shift=32)
    return out, cfg


def lognormal_field(n, sigma_ln, slope=-11.0 / 3.0, seed=4):
    """Periodic lognormal density on an n^3 grid: exp of a Gaussian random
    field with power spectrum P(k) ~ k^slope (FFT-filtered white noise,
    seed), scaled to std(ln rho) = sigma_ln and mean(rho) = 1.  Axis order
    [z, y, x]."""
    rng = np.random.default_rng(seed)
    w = rng.normal(size=(n, n, n))
    k = np.fft.fftfreq(n) * n
    kr = np.fft.rfftfreq(n) * n
    K = np.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + kr[None, None, :] ** 2)
    amp = np.where(K > 0, K, 1.0) ** (slope / 2.0)
    amp[0, 0, 0] = 0.0
    g = np.fft.irfftn(np.fft.rfftn(w) * amp, s=(n, n, n))
    g = (g - g.mean()) / g.std()
    rho = np.exp(sigma_ln * g)
    return rho / rho.mean()


def _sample(grid, x):
    """Nearest-cell sample of a periodic [z, y, x] grid on the unit box at points x [..., 3]."""
    n = grid.shape[0]
    i = np.clip((np.asarray(x) * n).astype(np.int64), 0, n - 1)
    return grid[i[..., 2], i[..., 1], i[..., 0]]


def lognormal_cube(n_packets=1_000_000, n=96, sigma_ln=1.0, albedo=0.9, tau_mean=2.0, seed=4,
                   image_n=64, inclination=60.0):
    """Uniform n^3 grid (16^3 blocks) holding a lognormal density (std of
    ln rho sigma_ln, k^-11/3 spectrum, seed); sigma_sca proportional to rho with
    the given albedo; mean centre-to-face extinction depth tau_mean; Rayleigh
    matrix; central isotropic point source; n x n peel-off image at the given
    inclination.  Returns (mesh, sigma2, cfg, rho_grid)."""
    rho = lognormal_field(n, sigma_ln, seed=seed)
    mesh = Mesh(MeshConfig((0, 0, 0), (1, 1, 1), (n,) * 3, (16,) * 3, (False,) * 3))
    r = _sample(rho, cell_centers(mesh))
    ext = 2.0 * tau_mean * r
    sigma2 = np.stack([albedo * ext, (1.0 - albedo) * ext], 1).astype(np.float32)
    cfg = TransportConfig(n_packets=n_packets, seed=seed,
                          sources=[Source(SOURCE_POINT, EMIT_ISOTROPIC, (0.5, 0.5, 0.5))],
                          phase=PHASE_RAYLEIGH, image_n=image_n, inclination_deg=inclination,
                          image_center=(0.5, 0.5, 0.5), image_half_width=0.75, image_batch_n=8,
                          n_batches=32, w_min=0.01, fx_shift=32)
    return mesh, sigma2, cfg, rho


def large_amr(n_packets=1_000_000_000, n_root=256, block=16, sigma_ln=1.5, levels=3, seed=5,
              target_cells=20_000_000, n_sources=64, image_n=256, tau_mean=2.0):
    """Large AMR scene: root n_root^3 in block^3, refined up to `levels`
    levels on a lognormal density (std of ln rho sigma_ln, k^-11/3, seed)
    with thresholds chosen so that the mesh holds about target_cells cells;
    HG (g = 0.6) with a Rayleigh-like polarization (peak 0.5 at 90 deg); albedo
    0.9; n_sources isotropic point sources placed uniformly at random;
    image_n^2 IQUV peel-off.  Returns (mesh, sigma2, cfg)."""
    rho = lognormal_field(n_root, sigma_ln, seed=seed)
    nb = n_root // block
    bmax = rho.reshape(nb, block, nb, block, nb, block).max(axis=(1, 3, 5))
    order = np.sort(bmax.ravel())[::-1]
    # choose the level-1 and level-2 block counts so that cells ~ target:
    # each refined block adds 7 blocks per level
    extra = max(0, target_cells // (block ** 3) - nb ** 3)
    n1 = min(len(order) // 4, max(1, int(extra / 7 * 0.7)))
    n2 = max(1, int(extra / 49 * 0.3 / 1.0)) if levels >= 3 else 0
    n2 = min(n2, n1 // 2)
    t1 = order[n1 - 1]
    t2 = order[n2 - 1] if n2 else np.inf
    boxes = []
    h = 1.0 / nb
    for lvl, thr in ((1, t1), (2, t2)):
        if lvl >= levels or not np.isfinite(thr):
            continue
        for kz, ky, kx in zip(*np.nonzero(bmax >= thr)):
            lo = tuple((np.array([kx, ky, kz]) + 0.25) * h)
            hi = tuple((np.array([kx, ky, kz]) + 0.75) * h)
            boxes.append(RefineRegion(lvl, lo, hi))
    mesh = Mesh(MeshConfig((0, 0, 0), (1, 1, 1), (n_root,) * 3, (block,) * 3, (False,) * 3, boxes))
    r = _sample(rho, cell_centers(mesh))
    ext = 2.0 * tau_mean * r
    sigma2 = np.stack([0.9 * ext, 0.1 * ext], 1).astype(np.float32)
    rng = np.random.default_rng(seed)
    srcs = [Source(SOURCE_POINT, EMIT_ISOTROPIC, tuple(p)) for p in rng.uniform(0.05, 0.95, (n_sources, 3))]
    cfg = TransportConfig(n_packets=n_packets, seed=seed, sources=srcs, phase=PHASE_HG_POL,
                          hg_g=0.6, pol_max=0.5, image_n=image_n, inclination_deg=60.0,
                          image_center=(0.5, 0.5, 0.5), image_half_width=0.75, image_batch_n=64,
                          n_batches=32, w_min=0.01, fx_shift=30)
    return mesh, sigma2, cfg
