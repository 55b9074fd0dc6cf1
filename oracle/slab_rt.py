"""Deterministic polarized radiative transfer in a plane-parallel slab
(test infrastructure: the analytic check of the slab configuration).

Conservative Rayleigh (Thomson) scattering in the (I_l, I_r) representation
(l in the meridian plane, r perpendicular to it), azimuth-independent field.
The azimuth-averaged phase matrix is computed numerically from dipole
scattering geometry: the field scattered from polarization e into
polarization e' has amplitude e'.e, so M_pq = 3/(8 pi) <|e'_p . e_q|^2>_phi,
which integrates to the Rayleigh phase function 3/(16 pi)(1 + cos^2 Theta) for
unpolarized light.  The transfer equation mu dI/dtau = I - S (tau from the top,
mu > 0 upward) is solved in the second-order form of Feautrier,
mu^2 u'' = u - S(u) with u = (I(mu) + I(-mu))/2 (Gauss-Legendre directions,
graded depth grid, second-order boundary conditions: vacuum at the top, a
given upward intensity at the base), then the emergent intensity at any mu is
the formal solution of the converged source function.  For a thick slab the
emergent polarization approaches that of Chandrasekhar's electron-scattering
atmosphere (about 11.7% at the limb).
"""
from __future__ import annotations

import numpy as np


def rayleigh_matrix(mu_out, mu_in, n_phi=64):
    """Azimuth-averaged Rayleigh matrix <M>[o, i, p, q] per steradian, p/q = (l, r)."""
    mo = np.asarray(mu_out, float)[:, None, None]
    mi = np.asarray(mu_in, float)[None, :, None]
    phi = (np.arange(n_phi) + 0.5) * 2 * np.pi / n_phi          # midpoint rule: exact for trig polys
    st_o, st_i = np.sqrt(1 - mo ** 2), np.sqrt(1 - mi ** 2)
    # outgoing direction at azimuth 0, incoming at azimuth phi
    lo = (mo, 0.0, -st_o)
    ro = (0.0, 1.0, 0.0)
    cp, sp = np.cos(phi)[None, None, :], np.sin(phi)[None, None, :]
    li = (mi * cp, mi * sp, -st_i + 0 * cp)
    ri = (-sp + 0 * mi, cp + 0 * mi, 0 * cp)
    dot = lambda a, b: a[0] * b[0] + a[1] * b[1] + a[2] * b[2]
    out = np.empty((mo.shape[0], mi.shape[1], 2, 2))
    for p, ep in enumerate((lo, ro)):
        for q, eq in enumerate((li, ri)):
            out[:, :, p, q] = (dot(ep, eq) ** 2).mean(-1)
    return out * 3.0 / (8.0 * np.pi)


def _grid(tau_max, n):
    """Depth grid: logarithmic near the top, then uniform."""
    top = np.logspace(-5, 0, n // 3)
    deep = np.linspace(1.0, tau_max, n - n // 3 + 1)[1:]
    return np.concatenate([[0.0], top[top < 1.0], deep])


class SlabSolution:
    def __init__(self, tau, mu, w, u, A_fn):
        self.tau, self.mu, self.w, self.u, self._A = tau, mu, w, u, A_fn

    def source(self, mu_q):
        """Source function S[k, m, p] for arbitrary directions mu_q (> 0)."""
        A = self._A(np.asarray(mu_q, float))            # [m, (j, q), p]
        return np.einsum("mjqp,kjq->kmp", A, self.u)

    def emergent(self, mu_q, i_inc=None):
        """Emergent (I_l, I_r) at the top for directions mu_q: formal solution
        with S linear between grid points (exact exponential weights), plus the
        attenuated base intensity."""
        mu_q = np.asarray(mu_q, float)
        S = self.source(mu_q)                             # [k, m, 2]
        t = self.tau
        out = np.zeros((len(mu_q), 2))
        for m, mq in enumerate(mu_q):
            e = np.exp(-t / mq)
            dt = np.diff(t)
            # integral of (a + b (tau - t0)) e^{-tau/mu} dtau/mu over each interval
            e0, e1 = e[:-1], e[1:]
            x = dt / mq
            # exact weights for linear interpolation on each interval
            em = -np.expm1(-x)                            # 1 - e^{-x}
            g0 = em - (1 - (1 + x) * np.exp(-x)) / np.where(x > 0, x, 1)   # weight of S at left
            g1 = (1 - (1 + x) * np.exp(-x)) / np.where(x > 0, x, 1)        # weight of S at right
            for p in range(2):
                s = S[:, m, p]
                out[m, p] = np.sum(e0 * (g0 * s[:-1] + g1 * s[1:]))
            if i_inc is not None:
                out[m] += np.asarray(i_inc(np.array([mq])))[0] * e[-1]
        return out


def solve_slab(tau_max=10.0, n_mu=24, n_tau=360, i_inc=None):
    """Solves the slab with upward intensity i_inc(mu) -> (I_l, I_r) at the base
    (default: unpolarized 1/mu, i.e. emission uniform in mu, as the Monte-Carlo
    slab source) and vacuum at the top.  Returns a SlabSolution."""
    if i_inc is None:
        i_inc = lambda m: np.stack([0.5 / m, 0.5 / m], -1)
    x, wx = np.polynomial.legendre.leggauss(2 * n_mu)
    mu, w = x[n_mu:], wx[n_mu:]                          # (0, 1), weights of int_0^1
    tau = _grid(tau_max, n_tau)
    K, M = len(tau), len(mu)
    # S_p(mu) = 2 pi sum_j 2 w_j sum_q <M>(mu, mu_j)_pq u_q(mu_j)
    def A_fn(mu_q):
        R = rayleigh_matrix(mu_q, mu)                     # [m, j, p, q]
        return (4 * np.pi * w[None, :, None, None] * R).transpose(0, 1, 3, 2)  # [m, j, q, p]
    A = A_fn(mu)                                          # [m, j, q, p]
    N = 2 * M
    Amat = A.transpose(0, 3, 1, 2).reshape(N, N)          # rows (m, p), cols (j, q)
    I_N = np.eye(N)
    mu2 = np.repeat(mu ** 2, 2)
    muv = np.repeat(mu, 2)
    dt = np.diff(tau)
    # block tridiagonal: -a_k u_{k-1} + B_k u_k - c_k u_{k+1} = d_k
    Bs, as_, cs, ds = [], [], [], []
    inc = np.asarray(i_inc(mu)).reshape(N)
    for k in range(K):
        if k == 0:
            h = dt[0]
            # mu (u1 - u0)/h = u0 + h/(2 mu) (u0 - S0)
            B = np.diag(muv / h + 1.0 + h / (2 * muv)) - np.diag(h / (2 * muv)) @ Amat
            c = np.diag(muv / h)
            a = np.zeros((N, N))
            d = np.zeros(N)
        elif k == K - 1:
            h = dt[-1]
            # mu (uK - uK-1)/h = I_inc - uK - h/(2 mu) (uK - SK)
            B = np.diag(muv / h + 1.0 + h / (2 * muv)) - np.diag(h / (2 * muv)) @ Amat
            a = np.diag(muv / h)
            c = np.zeros((N, N))
            d = inc.copy()
        else:
            hm, hp = dt[k - 1], dt[k]
            hc = 0.5 * (hm + hp)
            a = np.diag(mu2 / (hm * hc))
            c = np.diag(mu2 / (hp * hc))
            B = np.diag(mu2 / (hm * hc) + mu2 / (hp * hc) + 1.0) - Amat
            d = np.zeros(N)
        Bs.append(B); as_.append(a); cs.append(c); ds.append(d)
    # block Thomas algorithm
    Cp, Dp = [None] * K, [None] * K
    inv = np.linalg.inv(Bs[0])
    Cp[0], Dp[0] = inv @ cs[0], inv @ ds[0]
    for k in range(1, K):
        den = Bs[k] - as_[k] @ Cp[k - 1]
        inv = np.linalg.inv(den)
        Cp[k] = inv @ cs[k]
        Dp[k] = inv @ (ds[k] + as_[k] @ Dp[k - 1])
    U = np.zeros((K, N))
    U[-1] = Dp[-1]
    for k in range(K - 2, -1, -1):
        U[k] = Dp[k] + Cp[k] @ U[k + 1]
    u = U.reshape(K, M, 2)
    sol = SlabSolution(tau, mu, w, u, A_fn)
    sol.i_inc = i_inc
    return sol


def binned_polarization(sol, edges, n_sub=64):
    """Flux-weighted bin averages over mu bins: returns (I, Q) per bin with
    Q = I_l - I_r (l in the meridian plane), as escaping packets tally them."""
    res = []
    for lo, hi in zip(edges[:-1], edges[1:]):
        x, wx = np.polynomial.legendre.leggauss(n_sub)
        m = 0.5 * (hi - lo) * x + 0.5 * (hi + lo)
        wm = 0.5 * (hi - lo) * wx
        I = sol.emergent(m, sol.i_inc)
        res.append((np.sum(wm * m * (I[:, 0] + I[:, 1])), np.sum(wm * m * (I[:, 0] - I[:, 1]))))
    return np.array(res)
