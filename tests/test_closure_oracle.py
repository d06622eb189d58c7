"""The closure oracle (oracle/closure_oracle.py) on the CPU.

* the closed-form straight-line impulse integrals against numerical quadrature
  (receding and approaching pairs);
* the ballistic base conserves momentum, has KE = E_0, and converges to the
  converged momenta as the loose stop tightens (loose states from the oracle
  engine in f32, converged momenta from the oracle in f64);
* the gate's projection removes the net momentum and restores KE = E_0.
"""
from __future__ import annotations

import sys

import numpy as np
import pytest
from scipy.integrate import quad

from conftest import ROOT

sys.path.insert(0, str(ROOT / "oracle"))
import closure_oracle as co  # noqa: E402
import oracle_lib as ol  # noqa: E402


def _impulse_quad(r, w):
    f = [quad(lambda t, c=c: (r[c] + w[c] * t) / np.linalg.norm(r + w * t) ** 3, 0, np.inf, limit=200)[0]
         for c in range(3)]
    return np.array(f)


@pytest.mark.parametrize("sign", [1.0, -1.0])
def test_pair_impulse_matches_quadrature(sign):
    rng = np.random.default_rng(4 if sign > 0 else 5)
    for _ in range(6):
        r = rng.normal(size=3) * 3
        w = rng.normal(size=3) * 0.05
        if np.sign(r @ w) != sign:
            w = -w
        np.testing.assert_allclose(co.pair_impulse(r, w), _impulse_quad(r, w), rtol=1e-7, atol=1e-12)


def test_ballistic_base_conserves_and_converges(wl):
    n, m, q, pos = wl.sample_mixed(40, seed=17)
    tight = ol.run_batch_mixed(n, m, q, pos, bits=64, rtol=1e-10, atol=1e-16, pe_stop=1e-11)
    errs = {}
    for pes in (0.05, 0.01):
        xs = np.zeros((40, 10, 3))
        ps = np.zeros((40, 10, 3))
        e0 = np.zeros(40)
        for s in range(40):
            k = int(n[s])
            x, p, st = ol.run_state(k, m[s, :k], q[s, :k], pos[s, :k], rtol=1e-10, atol=1e-16, pe_stop=pes)
            xs[s, :k], ps[s, :k], e0[s] = x, p, st.e0
        pb, P, L, _, Q = co.ballistic_base(n, m, q, xs, ps, e0)
        for s in range(40):
            k = int(n[s])
            assert np.linalg.norm(pb[s, :k].sum(0)) < 2e-5 * np.abs(pb[s, :k]).max()  # f32 loose state
            ke = 0.5 * np.sum(np.sum(pb[s, :k] ** 2, 1) / m[s, :k])
            assert abs(ke / e0[s] - 1) < 1e-12
        errs[pes] = np.median([np.linalg.norm(pb[s, :n[s]] - tight["momenta"][s, :n[s]]) /
                               np.linalg.norm(tight["momenta"][s, :n[s]]) for s in range(40)])
    assert errs[0.05] < 2e-3 and errs[0.01] < errs[0.05] / 4


def test_gate_projection():
    rng = np.random.default_rng(1)
    n = np.array([4], np.uint8)
    mass = np.zeros((1, 10))
    mass[0, :4] = [2.0, 3.0, 5.0, 7.0]
    pb = np.zeros((1, 10, 3))
    pb[0, :4] = rng.normal(size=(4, 3))
    pb[0, :4] -= pb[0, :4].mean(0)
    e0 = np.array([0.5 * np.sum(np.sum(pb[0, :4] ** 2, 1) / mass[0, :4])])
    out = np.zeros((1, 32))
    out[0, :12] = rng.normal(size=12) * 1e-3
    acc, mom, rho, mu, corr = co.apply_gate(n, mass, e0, pb, np.array([1.0]), out, 1.0, 1.0, 1.0)
    assert acc[0] and rho[0] > 0 and mu[0] > 0
    assert np.linalg.norm(mom[0, :4].sum(0)) < 1e-12
    assert abs(0.5 * np.sum(np.sum(mom[0, :4] ** 2, 1) / mass[0, :4]) / e0[0] - 1) < 1e-12
    acc2, *_ = co.apply_gate(n, mass, e0, pb, np.array([1.0]), out, 0.0, 1.0, 1.0)
    assert not acc2[0]
