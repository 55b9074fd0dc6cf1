"""Single-scattering image of a point source in a uniform box, by quadrature
(test infrastructure: an independent check of the polarized transport).

Nothing here follows the kernels' code.  In a box of uniform extinction
sigma_e = sigma_s + sigma_a, an isotropic point source of unit power at s
makes first interactions at x with density sigma_e exp(-sigma_e r) / (4 pi r^2)
(r = |x - s|).  With survival weighting the packet carries the albedo
sigma_s / sigma_e after the interaction, and its peel-off toward the observer
direction o adds f11(mu) exp(-sigma_e l(x)) per steradian, l(x) the path from
x to the box boundary along o and mu = k.o the cosine of the scattering angle
(k = (x - s) / r).  So the first-scattering image is

    I(pixel) = integral over the pixel's column of
               sigma_s exp(-sigma_e (r + l(x))) f11(mu) / (4 pi r^2) dV,

which in spherical coordinates about the source is a smooth integral over
directions k and distances r (the 1 / r^2 cancels the volume element).  The
scattered light of unpolarized incident light is linearly polarized
perpendicular to the scattering plane (the plane of k and o) with fraction
p(mu): Rayleigh (Chandrasekhar 1960): f11 = 3 (1 + mu^2) / (16 pi),
p = (1 - mu^2) / (1 + mu^2); Henyey-Greenstein with a Rayleigh-like term
(White 1979): f11 = (1 - g^2) / (4 pi (1 + g^2 - 2 g mu)^1.5),
p = p_max (1 - mu^2) / (1 + mu^2).  Q and U are given in the image frame:
Q > 0 along ev (the projection of +z on the sky), U > 0 along ev + e2 with
e2 = o x ev.  The unscattered light of the emission, (1 / 4 pi)
exp(-sigma_e l(s)), lands in the source's pixel.  Higher orders of
scattering add a relative O(albedo).
"""
from __future__ import annotations

import numpy as np


def observer_frame(inclination_deg: float, azimuth_deg: float):
    """Observer direction o, image vertical ev (projection of +z) and
    horizontal eh = ev x o, for inclination from +z and azimuth about +z."""
    i, a = np.radians(inclination_deg), np.radians(azimuth_deg)
    o = np.array([np.sin(i) * np.cos(a), np.sin(i) * np.sin(a), np.cos(i)])
    ev = np.array([-np.cos(i) * np.cos(a), -np.cos(i) * np.sin(a), np.sin(i)])
    eh = np.cross(ev, o)
    return o, ev, eh


def phase(kind: str, mu, g=0.0, p_max=1.0):
    """(f11 per steradian, linear polarization fraction) at scattering cosine mu."""
    mu = np.asarray(mu, float)
    shape = (1 - mu ** 2) / (1 + mu ** 2)
    if kind == "rayleigh":
        return 3 * (1 + mu ** 2) / (16 * np.pi), shape
    f = (1 - g * g) / (4 * np.pi * (1 + g * g - 2 * g * mu) ** 1.5)
    return f, p_max * shape


def exit_length(x, o, lo, hi):
    """Distance from points x [..., 3] (inside the box) to its boundary along o."""
    t = np.full(x.shape[:-1], np.inf)
    for a in range(3):
        if o[a] > 0:
            t = np.minimum(t, (hi[a] - x[..., a]) / o[a])
        elif o[a] < 0:
            t = np.minimum(t, (lo[a] - x[..., a]) / o[a])
    return t


def wall_distance(s, k, lo, hi):
    """Distance from the point s inside the box to its boundary along each
    direction k [..., 3]."""
    t = np.full(k.shape[:-1], np.inf)
    for a in range(3):
        ka = k[..., a]
        with np.errstate(divide="ignore", invalid="ignore"):
            ta = np.where(ka > 0, (hi[a] - s[a]) / ka, np.where(ka < 0, (lo[a] - s[a]) / ka, np.inf))
        t = np.minimum(t, ta)
    return t


def single_scatter_image(lo, hi, src, sigma_s, sigma_a, inclination_deg, azimuth_deg,
                         center, half_width, n_pix, kind="rayleigh", g=0.0, p_max=1.0,
                         n_mu=160, n_phi=320, n_r=48):
    """Expected image [n_pix, n_pix, 4] (I, Q, U, V; row = vertical pixel) per
    emitted packet of unit weight: first scatterings by quadrature, plus the
    unscattered emission in the source's pixel."""
    lo, hi, src, center = (np.asarray(v, float) for v in (lo, hi, src, center))
    sig_e = sigma_s + sigma_a
    o, ev, eh = observer_frame(inclination_deg, azimuth_deg)
    e2 = np.cross(o, ev)
    mu_n, mu_w = np.polynomial.legendre.leggauss(n_mu)            # cos(theta) of k
    phi = (np.arange(n_phi) + 0.5) * 2 * np.pi / n_phi
    st = np.sqrt(1 - mu_n ** 2)
    k = np.stack([st[:, None] * np.cos(phi)[None, :], st[:, None] * np.sin(phi)[None, :],
                  np.broadcast_to(mu_n[:, None], (n_mu, n_phi))], -1)       # [mu, phi, 3]
    w_dir = mu_w[:, None] * (2 * np.pi / n_phi) * np.ones((1, n_phi))    # dOmega
    R = wall_distance(src, k, lo, hi)                               # [mu, phi]
    r_n, r_w = np.polynomial.legendre.leggauss(n_r)
    img = np.zeros((n_pix * n_pix, 4))
    inv_pix = n_pix / (2 * half_width)
    for j in range(n_mu):                                           # one cone at a time
        kk = k[j]                                                   # [phi, 3]
        Rj = R[j]
        r = 0.5 * Rj[:, None] * (r_n[None, :] + 1)                  # [phi, r]
        wr = 0.5 * Rj[:, None] * r_w[None, :]
        x = src + r[..., None] * kk[:, None, :]                     # [phi, r, 3]
        l_out = exit_length(x, o, lo, hi)
        mu_s = kk @ o                                               # [phi]
        f11, p = phase(kind, mu_s, g, p_max)
        n = np.cross(kk, o)                                         # E-vector direction
        nn = np.linalg.norm(n, axis=-1)
        nn = np.where(nn > 0, nn, 1.0)
        c, s = (n @ ev) / nn, (n @ e2) / nn
        cos2, sin2 = c * c - s * s, 2 * c * s
        val = sigma_s * np.exp(-sig_e * (r + l_out)) * wr * (w_dir[j][:, None] / (4 * np.pi))
        I = val * f11[:, None]
        Q = I * (p * cos2)[:, None]
        U = I * (p * sin2)[:, None]
        d = x - center
        fx = np.floor(d @ eh * inv_pix + 0.5 * n_pix).astype(np.int64)
        fy = np.floor(d @ ev * inv_pix + 0.5 * n_pix).astype(np.int64)
        ok = (fx >= 0) & (fy >= 0) & (fx < n_pix) & (fy < n_pix)
        pix = (fy * n_pix + fx)[ok]
        for q, v in enumerate((I, Q, U)):
            img[:, q] += np.bincount(pix, weights=v[ok], minlength=n_pix * n_pix)
    # the unscattered emission toward the observer
    d = src - center
    fx = int(np.floor(d @ eh * inv_pix + 0.5 * n_pix))
    fy = int(np.floor(d @ ev * inv_pix + 0.5 * n_pix))
    if 0 <= fx < n_pix and 0 <= fy < n_pix:
        img[fy * n_pix + fx, 0] += np.exp(-sig_e * exit_length(src[None], o, lo, hi)[0]) / (4 * np.pi)
    return img.reshape(n_pix, n_pix, 4)
