"""Synthetic problem set-ups as plain data: mesh description, per-cell
coefficients as a function of the cell centres, transport configuration.

The counterpart of the reference's user problem generator
(src/user/probgen.cpp:8-22, whose default ``prob::run`` is empty).  Nothing
here loads the product library: ``scenes`` builds these set-ups on the
product's mesh, and the oracle builds the same ones on the reference's own
meshgen.  All inputs are seeded synthetic fields; no external dataset is
involved.
"""
from __future__ import annotations

import math

import numpy as np

from .config import (EMIT_ISOTROPIC, PHASE_RAYLEIGH, SOURCE_POINT, MeshConfig, RefineRegion,
                     Source, TransportConfig)


def root_refine_boxes(field_fn, n_root, block, box_lo, box_hi, threshold, level=1):
    """One refine region per root block whose field exceeds ``threshold`` at
    any root-cell centre (static, data-driven refinement expressed as the
    reference's [refine_region*] boxes)."""
    nb = [n_root[a] // block[a] for a in range(3)]
    h = [(box_hi[a] - box_lo[a]) / n_root[a] for a in range(3)]
    axes = [box_lo[a] + (np.arange(n_root[a]) + 0.5) * h[a] for a in range(3)]
    Z, Y, X = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    f = field_fn(np.stack([X, Y, Z], -1)).reshape(nb[2], block[2], nb[1], block[1], nb[0], block[0])
    fmax = f.max(axis=(1, 3, 5))
    boxes = []
    for kz, ky, kx in zip(*np.nonzero(fmax > threshold)):
        lo = [box_lo[a] + (k + 0.25) * block[a] * h[a] for a, k in enumerate((kx, ky, kz))]
        hi = [box_lo[a] + (k + 0.75) * block[a] * h[a] for a, k in enumerate((kx, ky, kz))]
        boxes.append(RefineRegion(level, tuple(lo), tuple(hi)))
    return boxes


def clump_mesh_config(n_root=128, block=16, peak=100.0, fwhm=0.1) -> MeshConfig:
    """Mesh of the 2-level AMR clump: root n_root^3 in block^3, refined x2
    where the Gaussian clump's density (peak, FWHM in box units, on a unit
    background) exceeds 3x its mean."""
    s = fwhm / (2.0 * math.sqrt(2.0 * math.log(2.0)))

    def rho(x):
        r2 = ((np.asarray(x) - 0.5) ** 2).sum(-1)
        return 1.0 + (peak - 1.0) * np.exp(-r2 / (2 * s * s))

    n3 = (n_root,) * 3
    g = (np.arange(n_root) + 0.5) / n_root
    mean = (1.0 + (peak - 1.0) * np.exp(-((g - 0.5) ** 2) / (2 * s * s)).mean() ** 3)
    boxes = root_refine_boxes(rho, n3, (block,) * 3, (0, 0, 0), (1, 1, 1), 3.0 * mean)
    return MeshConfig((0, 0, 0), (1, 1, 1), n3, (block,) * 3, (False,) * 3, boxes)


def clump_spec(n_packets=10_000_000, n_root=128, block=16, peak=100.0, fwhm=0.1, tau_edge=5.0,
               albedo=(0.5, 0.99), seed=2, image_n=128, inclination=90.0):
    """Static 2-level AMR clump: root n_root^3 in block^3, refined x2 where the
    density exceeds 3x its mean; Gaussian clump (peak, FWHM in box units) on a
    unit background with centre-to-edge extinction depth tau_edge; per-cell
    albedo log-uniform in [albedo]; isotropic point source at the centre;
    peel-off image and int64 tallies.  Returns (MeshConfig, sigma_of, cfg):
    sigma_of(cell centres [n_cells, 3]) gives the coefficients."""
    s = fwhm / (2.0 * math.sqrt(2.0 * math.log(2.0)))

    def rho(x):
        r2 = ((np.asarray(x) - 0.5) ** 2).sum(-1)
        return 1.0 + (peak - 1.0) * np.exp(-r2 / (2 * s * s))

    mcfg = clump_mesh_config(n_root, block, peak, fwhm)
    # extinction coefficient: integral of kappa*rho from the centre to a face = tau_edge
    col = 0.5 + (peak - 1.0) * s * math.sqrt(math.pi / 2) * math.erf(0.5 / (s * math.sqrt(2)))

    def sigma_of(centres):
        """(sigma_sca, sigma_abs) [n_cells, 2] float32 at the cell centres
        (block-id order, x fastest); the albedos are drawn in that order."""
        ext = (tau_edge / col) * rho(centres)
        rng = np.random.default_rng(seed)
        alb = np.exp(rng.uniform(math.log(albedo[0]), math.log(albedo[1]), len(centres)))
        return np.stack([ext * alb, ext * (1.0 - alb)], 1).astype(np.float32)

    cfg = TransportConfig(n_packets=n_packets, seed=seed,
                          sources=[Source(SOURCE_POINT, EMIT_ISOTROPIC, (0.5, 0.5, 0.5))],
                          phase=PHASE_RAYLEIGH, n_mu_bins=20, mu_lo=-1.0, mu_hi=1.0,
                          image_n=image_n, inclination_deg=inclination,
                          image_center=(0.5, 0.5, 0.5), image_half_width=0.5,
                          image_batch_n=8, n_batches=32, w_min=0.01, fx_shift=32)
    return mcfg, sigma_of, cfg
