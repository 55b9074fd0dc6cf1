"""Polarized Monte Carlo with multiple scattering in a uniform box, written
from the physics in vectorised numpy (test infrastructure: an independent
check of the transport's multiple scattering).

It shares nothing with the kernels or the C restatement but the physical
model: isotropic unpolarized emission from a point source; exponential free
paths in the uniform extinction sigma_e = sigma_s + sigma_a, the distance to
the walls found analytically (no cells); survival weighting by the albedo at
every interaction; the scattering matrix of Rayleigh or Henyey-Greenstein with
a Rayleigh-like polarization term,

    I' = f11 (1 + r12 Q),  Q' = f11 (r12 + Q),  U' = f11 r33 U,  V' = f11 r33 V

in the frame of the scattering plane (r12 = (mu^2 - 1) / (1 + mu^2) for
Rayleigh, -p_max (1 - mu^2) / (1 + mu^2) for HG; r33 = 2 mu / (1 + mu^2));
scattering directions drawn from I' by rejection; and a peel-off image at
every interaction and at the emission.  Polarization frames are handled with
explicit rotation angles: the Stokes parameters of a photon refer to a
vector e1 perpendicular to its direction d (e2 = d x e1); turning the frame by
psi (e1 -> cos psi e1 + sin psi e2) maps (Q, U) to (Q cos 2psi + U sin 2psi,
U cos 2psi - Q sin 2psi).  Image Stokes refer to ev (Q > 0 along the
projection of +z) and e2 = o x ev, as in oracle/single_scatter.py.
"""
from __future__ import annotations

import numpy as np

from oracle.single_scatter import exit_length, observer_frame, phase, wall_distance


def _r12_r33(kind, mu, p_max):
    s = (1 - mu * mu) / (1 + mu * mu)
    r12 = -s if kind == "rayleigh" else -p_max * s
    return r12, 2 * mu / (1 + mu * mu)


def _rotate(q, u, c, s):
    """Stokes (q, u) in the frame turned by the angle with cosine/sine (c, s)."""
    n2 = c * c + s * s
    n2 = np.where(n2 > 0, n2, 1.0)
    c2, s2 = (c * c - s * s) / n2, 2 * c * s / n2
    return q * c2 + u * s2, u * c2 - q * s2


def _unit(v):
    n = np.linalg.norm(v, axis=-1, keepdims=True)
    return v / np.where(n > 0, n, 1.0)


def _perp(d):
    """A unit vector perpendicular to each direction d."""
    a = np.where(np.abs(d[:, 2:3]) < 0.9, np.array([[0.0, 0.0, 1.0]]), np.array([[1.0, 0.0, 0.0]]))
    return _unit(np.cross(a, d))


def box_mc_image(lo, hi, src, sigma_s, sigma_a, inclination_deg, azimuth_deg, center,
                 half_width, n_pix, n_packets, max_scatter, kind="rayleigh", g=0.0, p_max=1.0,
                 n_batches=16, seed=1):
    """Per-batch peel-off images [n_batches, n_pix, n_pix, 3] (I, Q, U) of
    n_packets packets (n_packets / n_batches each), each ending at its
    max_scatter-th interaction or at the wall."""
    lo, hi, src, center = (np.asarray(v, float) for v in (lo, hi, src, center))
    sig_e = sigma_s + sigma_a
    alb = sigma_s / sig_e
    o, ev, eh = observer_frame(inclination_deg, azimuth_deg)
    e2_img = np.cross(o, ev)
    pix = 2 * half_width / n_pix
    rng = np.random.default_rng(seed)
    out = np.zeros((n_batches, n_pix * n_pix, 3))

    def deposit(batch, x, vals):
        fx = np.floor((x - center) @ eh / pix + 0.5 * n_pix).astype(np.int64)
        fy = np.floor((x - center) @ ev / pix + 0.5 * n_pix).astype(np.int64)
        ok = (fx >= 0) & (fy >= 0) & (fx < n_pix) & (fy < n_pix)
        idx = (batch * n_pix * n_pix + fy * n_pix + fx)[ok]
        flat = out.reshape(-1, 3)
        for q in range(3):
            flat[:, q] += np.bincount(idx, weights=vals[q][ok], minlength=flat.shape[0])

    per = n_packets // n_batches
    n = per * n_batches
    batch = np.repeat(np.arange(n_batches), per)
    # emission: its unscattered light, then isotropic directions, unpolarized
    direct = np.exp(-sig_e * exit_length(src[None], o, lo, hi)[0]) / (4 * np.pi)
    deposit(np.arange(n_batches), np.repeat(src[None], n_batches, 0),
            (np.full(n_batches, direct * per), np.zeros(n_batches), np.zeros(n_batches)))
    z = rng.uniform(-1, 1, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    st = np.sqrt(1 - z * z)
    d = np.stack([st * np.cos(ph), st * np.sin(ph), z], 1)
    x = np.repeat(src[None], n, 0)
    e1 = _perp(d)
    Q = np.zeros(n); U = np.zeros(n); V = np.zeros(n)
    w = np.ones(n)
    for _ in range(max_scatter):
        # free path: interaction inside the box, or escape
        s = rng.exponential(1.0, len(w)) / sig_e
        inside = s < wall_distance_each(x, d, lo, hi)
        x, d, e1, Q, U, V, w, batch, s = (a[inside] for a in (x, d, e1, Q, U, V, w, batch, s))
        if len(w) == 0:
            break
        x = x + s[:, None] * d
        w = w * alb
        e2 = np.cross(d, e1)
        # peel-off toward the observer
        mu = d @ o
        nrm = _unit(np.cross(d, o))
        a_in = np.cross(nrm, d)
        qa, ua = _rotate(Q, U, np.einsum("ij,ij->i", e1, a_in), np.einsum("ij,ij->i", e2, a_in))
        f11, _ = phase(kind, mu, g, p_max)
        r12, r33 = _r12_r33(kind, mu, p_max)
        Io, Qo, Uo = f11 * (1 + r12 * qa), f11 * (r12 + qa), f11 * r33 * ua
        a_out = np.cross(nrm, o)
        qi, ui = _rotate(Qo, Uo, a_out @ ev, np.cross(o, a_out) @ ev)
        att = w * np.exp(-sig_e * exit_length(x, o, lo, hi))
        deposit(batch, x, (att * Io, att * qi, att * ui))
        # the new direction, by rejection from the scattering matrix
        m = len(w)
        mu_n = np.empty(m); phi = np.empty(m)
        todo = np.arange(m)
        while len(todo):
            k = len(todo)
            if kind == "rayleigh":
                mu_p = rng.uniform(-1, 1, k)
            else:
                xi = rng.uniform(0, 1, k)
                t = (1 - g * g) / (1 - g + 2 * g * xi)
                mu_p = (1 + g * g - t * t) / (2 * g)
            ph_p = rng.uniform(0, 2 * np.pi, k)
            q_phi = Q[todo] * np.cos(2 * ph_p) + U[todo] * np.sin(2 * ph_p)
            r12p, _ = _r12_r33(kind, mu_p, p_max)
            if kind == "rayleigh":
                acc = (1 + mu_p ** 2) * (1 + r12p * q_phi) / 2
            else:
                acc = (1 + r12p * q_phi) / (1 + p_max)
            ok = rng.uniform(0, 1, k) < acc
            mu_n[todo[ok]] = mu_p[ok]
            phi[todo[ok]] = ph_p[ok]
            todo = todo[~ok]
        sn = np.sqrt(np.maximum(0.0, 1 - mu_n ** 2))
        dn = mu_n[:, None] * d + sn[:, None] * (np.cos(phi)[:, None] * e1 + np.sin(phi)[:, None] * e2)
        # the frame of the scattering plane: in-plane vectors a_in (incoming)
        # and a_out (outgoing); the incoming frame turned by phi is a_in
        nrm = np.cos(phi)[:, None] * e2 - np.sin(phi)[:, None] * e1
        qa, ua = _rotate(Q, U, np.cos(phi), np.sin(phi))
        r12, r33 = _r12_r33(kind, mu_n, p_max)
        I1 = 1 + r12 * qa
        Q, U, V = (r12 + qa) / I1, r33 * ua / I1, r33 * V / I1
        d = _unit(dn)
        e1 = _unit(np.cross(nrm, d))
    return out.reshape(n_batches, n_pix, n_pix, 3)


def wall_distance_each(x, d, lo, hi):
    """Distance from each point x[i] to the box boundary along d[i]."""
    t = np.full(len(x), np.inf)
    for a in range(3):
        with np.errstate(divide="ignore", invalid="ignore"):
            ta = np.where(d[:, a] > 0, (hi[a] - x[:, a]) / d[:, a],
                          np.where(d[:, a] < 0, (lo[a] - x[:, a]) / d[:, a], np.inf))
        t = np.minimum(t, ta)
    return t
