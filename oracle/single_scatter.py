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

which is integrated along the pixel's lines of sight (a change of variable
removes the 1 / r^2 peak near the source).  The
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


def _box_span(P, o, lo, hi):
    """Entry and exit parameters (l_in, l_out) of the lines P + l o through the
    box (l_in >= l_out where a line misses it)."""
    l_in = np.full(P.shape[:-1], -np.inf)
    l_out = np.full(P.shape[:-1], np.inf)
    for a in range(3):
        if o[a] != 0:
            t1, t2 = (lo[a] - P[..., a]) / o[a], (hi[a] - P[..., a]) / o[a]
            l_in = np.maximum(l_in, np.minimum(t1, t2))
            l_out = np.minimum(l_out, np.maximum(t1, t2))
        else:
            inside = (P[..., a] >= lo[a]) & (P[..., a] <= hi[a])
            l_out = np.where(inside, l_out, -np.inf)
    return l_in, l_out


def single_scatter_image(lo, hi, src, sigma_s, sigma_a, inclination_deg, azimuth_deg,
                         center, half_width, n_pix, kind="rayleigh", g=0.0, p_max=1.0,
                         n_sub=24, n_theta=48):
    """Expected image [n_pix, n_pix, 4] (I, Q, U, V; row = vertical pixel) per
    emitted packet of unit weight: first scatterings integrated pixel by
    pixel along the lines of sight (n_sub x n_sub lines per pixel, midpoint
    rule), plus the unscattered emission in the source's pixel.

    Along a line x = P + l o with closest approach b to the source at l0,
    r^2 = b^2 + (l - l0)^2 and l - l0 = b tan(theta) turns dl / r^2 into
    dtheta / b; the path to the wall, l_exit - l, is linear in l, so the
    integrand is smooth in theta (Gauss-Legendre, n_theta nodes)."""
    lo, hi, src, center = (np.asarray(v, float) for v in (lo, hi, src, center))
    sig_e = sigma_s + sigma_a
    o, ev, eh = observer_frame(inclination_deg, azimuth_deg)
    e2 = np.cross(o, ev)
    pix = 2 * half_width / n_pix
    th_n, th_w = np.polynomial.legendre.leggauss(n_theta)
    sub = (np.arange(n_sub) + 0.5) / n_sub
    dA = (pix / n_sub) ** 2
    img = np.zeros((n_pix, n_pix, 4))
    for fy in range(n_pix):
        # the sub-lines of one row of pixels: [n_pix * n_sub, n_sub] lines
        hs = (np.arange(n_pix)[:, None] + sub[None, :]).reshape(-1) * pix - half_width
        vs = (fy + sub) * pix - half_width
        P = center + hs[:, None, None] * eh + vs[None, :, None] * ev     # [H, V, 3]
        l_in, l_out = _box_span(P, o, lo, hi)
        hit = l_out > l_in                          # lines that miss add nothing
        l_in, l_out = np.where(hit, l_in, 0.0), np.where(hit, l_out, 0.0)
        l0 = np.einsum("hvk,k->hv", src - P, o)
        b = np.maximum(np.linalg.norm(P + l0[..., None] * o - src, axis=-1), 1e-12)
        t1, t2 = np.arctan((l_in - l0) / b), np.arctan((l_out - l0) / b)
        th = 0.5 * (t2 - t1)[..., None] * (th_n + 1) + t1[..., None]      # [H, V, n]
        wth = 0.5 * (t2 - t1)[..., None] * th_w
        r = b[..., None] / np.cos(th)
        along = l0[..., None] + b[..., None] * np.tan(th)                 # l of each node
        k = (P[..., None, :] + along[..., None] * o - src) / r[..., None]
        f11, p = phase(kind, np.sin(th), g, p_max)                         # k . o = sin(th)
        n = np.cross(k, o)
        nn = np.linalg.norm(n, axis=-1)
        nn = np.where(nn > 0, nn, 1.0)
        c, s = (n @ ev) / nn, (n @ e2) / nn
        val = sigma_s * np.exp(-sig_e * (r + l_out[..., None] - along)) * f11 * wth
        val = np.where(hit[..., None], val / (4 * np.pi * b[..., None]), 0.0) * dA
        for q, w in enumerate((1.0, p * (c * c - s * s), p * 2 * c * s)):
            img[fy, :, q] = (val * w).sum(-1).reshape(n_pix, n_sub, n_sub).sum((1, 2))
    # the unscattered emission toward the observer
    d = src - center
    fx = int(np.floor(d @ eh / pix + 0.5 * n_pix))
    fy = int(np.floor(d @ ev / pix + 0.5 * n_pix))
    if 0 <= fx < n_pix and 0 <= fy < n_pix:
        img[fy, fx, 0] += np.exp(-sig_e * exit_length(src[None], o, lo, hi)[0]) / (4 * np.pi)
    return img
