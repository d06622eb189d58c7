"""FP64 scipy oracle: the reference's Python oracle restated.

TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's
accuracy and CPU-baseline legs use this module; nothing in the engine imports it.

The reference's ground truth (python/reference/coulomb.py:23-109) integrates each
explosion with scipy's ``solve_ivp`` (method RK45, the Dormand-Prince 5(4) pair)
from rest to t = 1e10 at rtol 1e-8 / atol 1e-16 and reads the velocities there;
at t = 1e10 the residual potential energy of a 2..10-atom explosion is far below
the tolerances, so m v is the asymptotic momentum. The integrator is the
third-party dependency scipy (the reference pins 1.16.3,
python/reference/requirements.txt:2; the image has 1.18.1), called here exactly
as the reference calls it (coulomb.py:101: same t_span, t_eval, rtol, atol).
The right-hand side is restated: pair forces k q_i q_j (x_i - x_j)/|x_i - x_j|^3
(coulomb.py:23-55, k = 1), accelerations F/m (coulomb.py:58-77), state
[x (3N), v (3N)].

Pinned against outputs of the reference's own module in
tests/golden/reference_cases.json and tests/golden/scipy_ref.npz (generated by
tests/golden/make_golden.py); tests/test_scipy_oracle.py holds the check.
``run_many`` spreads sims over a ``spawn`` process pool (a pool forked after a
CUDA context exists can hang); a worker that dies ends the call with an error
(concurrent.futures' broken-pool rule) instead of being replaced.
"""
from __future__ import annotations

import multiprocessing as mp
import os
from concurrent.futures import ProcessPoolExecutor

import numpy as np
from scipy.integrate import solve_ivp

RTOL = 1e-8   # coulomb.py:9 (RKRTOL)
ATOL = 1e-16  # coulomb.py:10 (RKATOL)
T_END = 1e10  # coulomb.py:101

try:  # JIT the right-hand side when numba is importable; plain numpy otherwise
    import numba

    _jit = numba.njit(cache=False)
except Exception:  # pragma: no cover - numba absent
    def _jit(f):
        return f


@_jit
def _rhs(t, y, inv_mass, qq):
    n = inv_mass.shape[0]
    dy = np.empty(6 * n)
    for c in range(3 * n):
        dy[c] = y[3 * n + c]
    acc = np.zeros((n, 3))
    for i in range(n - 1):
        for j in range(i + 1, n):
            rx = y[3 * i] - y[3 * j]
            ry = y[3 * i + 1] - y[3 * j + 1]
            rz = y[3 * i + 2] - y[3 * j + 2]
            r = np.sqrt(rx * rx + ry * ry + rz * rz)
            s = qq[i, j] / (r * r * r)
            acc[i, 0] += s * rx
            acc[i, 1] += s * ry
            acc[i, 2] += s * rz
            acc[j, 0] -= s * rx
            acc[j, 1] -= s * ry
            acc[j, 2] -= s * rz
    for i in range(n):
        for c in range(3):
            dy[3 * n + 3 * i + c] = acc[i, c] * inv_mass[i]
    return dy


def asymptotic_momenta(pos, masses, charges, k: float = 1.0) -> np.ndarray:
    """One explosion from rest at positions pos [n, 3]: m v at t = 1e10, [n, 3] float64."""
    pos = np.asarray(pos, dtype=np.float64)
    masses = np.asarray(masses, dtype=np.float64)
    charges = np.asarray(charges, dtype=np.float64)
    n = len(masses)
    y0 = np.concatenate([pos.reshape(-1), np.zeros(3 * n)])
    qq = k * np.outer(charges, charges)
    sol = solve_ivp(_rhs, (0.0, T_END), y0, t_eval=(T_END,), rtol=RTOL, atol=ATOL, args=(1.0 / masses, qq))
    if sol.status != 0:
        raise RuntimeError(f"solve_ivp failed: {sol.message}")
    v = sol.y[3 * n:, 0].reshape(n, 3)
    return masses[:, None] * v


def _chunk(args):
    pos, masses, charges, n_per = args
    out = np.zeros(pos.shape)
    for s in range(pos.shape[0]):
        n = int(n_per[s]) if n_per is not None else pos.shape[1]
        m = masses[s] if masses.ndim == 2 else masses
        q = charges[s] if charges.ndim == 2 else charges
        out[s, :n] = asymptotic_momenta(pos[s, :n], m[:n], q[:n])
    return out


def run_many(pos, masses, charges, n_per=None, processes: int | None = None) -> np.ndarray:
    """Asymptotic momenta of S explosions, [S, n, 3] float64.

    pos [S, n, 3]; masses / charges [n] (one molecule) or [S, n] (per sim, with
    n_per [S] live atoms, rows zero past n). processes: worker processes of a
    spawn pool (None: all usable cores; 1: this process)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    masses = np.asarray(masses, dtype=np.float64)
    charges = np.asarray(charges, dtype=np.float64)
    S = pos.shape[0]
    if processes is None:
        processes = len(os.sched_getaffinity(0))
    processes = max(1, min(processes, S))
    if processes == 1:
        return _chunk((pos, masses, charges, n_per))
    bounds = np.linspace(0, S, processes + 1).astype(int)
    jobs = []
    for a, b in zip(bounds[:-1], bounds[1:]):
        jobs.append((pos[a:b], masses[a:b] if masses.ndim == 2 else masses,
                     charges[a:b] if charges.ndim == 2 else charges,
                     None if n_per is None else np.asarray(n_per)[a:b]))
    with ProcessPoolExecutor(max_workers=processes, mp_context=mp.get_context("spawn")) as pool:
        parts = list(pool.map(_chunk, jobs))
    return np.concatenate(parts)
