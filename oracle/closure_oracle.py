"""CPU oracle for the closure's features, ballistic base and gate (TEST
INFRASTRUCTURE ONLY: used by tests/ and bench.py's checks, never by the
product).

A float64 numpy restatement of include/ce_closure.h for mixed rows of 10 atoms:

* ballistic base: p + sum_j k q_i q_j (r_ij I0 + w_ij I1) with
  I0 = 1/(|r|(|r||w| + r.w)), I1 = 1/(|w|(|r||w| + r.w)), rescaled to
  KE = E_0 (the reference's rescale, src/driver.cpp:38-42, applied to the
  ballistic state);
* features: per atom (x - x_com)/L, p/P, (p_base - p)/P, q/3, ln(m/amu)/3.5,
  1, then PE_stop/E_0 * 20 and n/10 (BF16-rounded like the device); the
  network output is in units of Q, the RMS per-atom size of p_base - p;
* training targets and the relative loss weights;
* gate: |KE/E_0 - 1|, |sum p|/sum|p|, |correction|/|base|, then projection
  to zero net momentum (mass weighted) and rescale to E_0.
"""
from __future__ import annotations

import numpy as np

from mlp_oracle import to_bf16

MASS_UNIT = 1822.888486209
A = 10


def pair_impulse(r, w):
    """int_0^inf (r + w t) / |r + w t|^3 dt = r I0 + w I1 in closed form; for an
    approaching pair (r.w < 0) |r|^2|w|^2 - (r.w)^2 = |r x w|^2 replaces the
    cancelling sum."""
    a, b, c = w @ w, r @ w, r @ r
    g = np.sqrt(a * c) + b if b >= 0 else np.sum(np.cross(r, w) ** 2) / (np.sqrt(a * c) - b)
    return r / (np.sqrt(c) * g) + w / (np.sqrt(a) * g)


def ballistic_base(n, mass, charge, x, p, e0, k=1.0):
    """(p_base [S,10,3], P [S], L [S], com [S,3], Q [S]) in float64; Q is the
    RMS per-atom size of the analytic step |p_base - p|."""
    S = n.shape[0]
    pb = np.zeros((S, A, 3))
    P = np.zeros(S)
    L = np.zeros(S)
    com = np.zeros((S, 3))
    Q = np.zeros(S)
    for s in range(S):
        k_ = int(n[s])
        m = mass[s, :k_].astype(np.float64)
        q = charge[s, :k_].astype(np.float64)
        xs = x[s, :k_].astype(np.float64)
        ps = p[s, :k_].astype(np.float64)
        v = ps / m[:, None]
        dp = np.zeros_like(ps)
        for i in range(k_):
            for j in range(i + 1, k_):
                t = k * q[i] * q[j] * pair_impulse(xs[i] - xs[j], v[i] - v[j])
                dp[i] += t
                dp[j] -= t
        b2 = ps + dp
        ke = 0.5 * np.sum(np.sum(b2 * b2, 1) / m)
        b2 = b2 * np.sqrt(e0[s] / ke)
        pb[s, :k_] = b2
        P[s] = np.sqrt(np.sum(b2 * b2) / k_)
        Q[s] = np.sqrt(np.sum((b2 - ps) ** 2) / k_)
        c0 = (m[:, None] * xs).sum(0) / m.sum()
        com[s] = c0
        L[s] = np.sqrt(np.sum((xs - c0) ** 2) / k_)
    return pb, P, L, com, Q


def features(n, mass, charge, x, p, e0, pe_final, k=1.0):
    """(feats [S,128] float64 of BF16 values, p_base, Q)."""
    pb, P, L, com, Q = ballistic_base(n, mass, charge, x, p, e0, k)
    S = n.shape[0]
    f = np.zeros((S, 128), np.float32)
    for s in range(S):
        k_ = int(n[s])
        for i in range(k_):
            o = 12 * i
            f[s, o:o + 3] = (x[s, i] - com[s]) / L[s]
            f[s, o + 3:o + 6] = p[s, i] / P[s]
            f[s, o + 6:o + 9] = (pb[s, i] - p[s, i]) / P[s]
            f[s, o + 9] = charge[s, i] / 3.0
            f[s, o + 10] = np.log(mass[s, i] / MASS_UNIT) / 3.5
            f[s, o + 11] = 1.0
        f[s, 120] = pe_final[s] / e0[s] * 20.0
        f[s, 121] = k_ * 0.1
    return to_bf16(f), pb, Q


def targets(n, p_base, Q, p_true, weight_scale=1.0):
    """(target [S,32], weight [S,32]): (p_true - p_base)/Q and the relative
    loss weight weight_scale/(3n) * 1e-2 / sqrt(rms^2 + (1e-4)^2)."""
    S = n.shape[0]
    t = np.zeros((S, 32))
    w = np.zeros((S, 32))
    for s in range(S):
        k_ = int(n[s])
        v = ((p_true[s, :k_] - p_base[s, :k_]) / Q[s]).reshape(-1)
        t[s, :3 * k_] = v
        rms2 = np.sum(v * v) / (3 * k_)
        w[s, :3 * k_] = weight_scale / (3 * k_) * 1e-2 / np.sqrt(rms2 + 1e-4 ** 2)
    return t, w


def apply_gate(n, mass, e0, p_base, Q, out, tol_e, tol_p, tol_c):
    """(accepted [S] bool, momenta [S,10,3] for accepted sims, rho, mu, corr)."""
    S = n.shape[0]
    acc = np.zeros(S, bool)
    mom = np.zeros((S, A, 3))
    rho = np.zeros(S)
    mu = np.zeros(S)
    corr = np.zeros(S)
    for s in range(S):
        k_ = int(n[s])
        m = mass[s, :k_]
        d = Q[s] * out[s, :3 * k_].reshape(k_, 3)
        pp = p_base[s, :k_] + d
        ke = 0.5 * np.sum(np.sum(pp * pp, 1) / m)
        rho[s] = abs(ke / e0[s] - 1.0)
        mu[s] = np.linalg.norm(pp.sum(0)) / np.sum(np.linalg.norm(pp, axis=1))
        corr[s] = np.linalg.norm(d) / np.linalg.norm(p_base[s, :k_])
        acc[s] = rho[s] <= tol_e and mu[s] <= tol_p and corr[s] <= tol_c
        if acc[s]:
            pp = pp - (m / m.sum())[:, None] * pp.sum(0)[None, :]
            ke2 = 0.5 * np.sum(np.sum(pp * pp, 1) / m)
            mom[s, :k_] = pp * np.sqrt(e0[s] / ke2)
    return acc, mom, rho, mu, corr
