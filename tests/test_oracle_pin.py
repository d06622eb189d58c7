"""Pin the CPU oracle before trusting it (CPU only).

1. Against the reference's golden vectors (tests/golden/reference_cases.json,
   recomputed from the reference's Python oracle): the tolerances of the
   reference's own tests/test_reference.cpp:83-167.
2. Against the reference's known-answer unit tests (tests/test_system.cpp:28-50,
   tests/test_integrator.cpp:34-82).
3. Bit-for-bit against the reference scalar engine's outputs committed in
   tests/golden/*.npz (engine built from the reference's own sources), and,
   where oracle/_ref is present, live on fresh random molecules.
"""
from __future__ import annotations

import json

import numpy as np
import pytest

import oracle_lib as ol
from conftest import GOLDEN


def cases():
    return json.loads((GOLDEN / "reference_cases.json").read_text())


@pytest.mark.parametrize("case", [c["name"] for c in cases()["cases"]])
def test_forces_match_reference_oracle(case):
    doc = cases()
    c = next(c for c in doc["cases"] if c["name"] == case)
    m, q, x = np.array(c["masses"]), np.array(c["charges"]), np.array(c["positions_init"])
    a = ol.accel(x, m, q, bits=64)
    # test_reference.cpp:95-100: F = m a within abs 1e-9
    np.testing.assert_allclose(a * m[:, None], np.array(c["forces_init"]), rtol=0, atol=1e-9)


@pytest.mark.parametrize("case", [c["name"] for c in cases()["cases"]])
def test_potential_matches_reference_oracle(case):
    c = next(c for c in cases()["cases"] if c["name"] == case)
    pe = ol.potential(np.array(c["positions_init"]), np.array(c["charges"]), bits=64)
    assert pe == pytest.approx(c["potential_energy_init"], rel=1e-12)  # test_reference.cpp:163-164


@pytest.mark.parametrize("case", [c["name"] for c in cases()["cases"]])
def test_asymptotic_momenta_match_reference_oracle(case):
    doc = cases()
    c = next(c for c in doc["cases"] if c["name"] == case)
    m, q, x = np.array(c["masses"]), np.array(c["charges"]), np.array(c["positions_init"])
    # test_reference.cpp:123-126: RK45 at the fixture tolerances, pe_stop 1e-10.
    r = ol.run_batch(x[None], m, q, bits=64, rtol=doc["rk_rtol"], atol=doc["rk_atol"], pe_stop=1e-10)
    assert r["status"][0] == 0
    ref = np.array(c["momenta_final"])
    scale = np.abs(ref).max()
    p = r["momenta"][0]
    ok = np.isclose(p, ref, rtol=1e-6, atol=0) | (np.abs(p - ref) <= scale * 1e-6)
    assert ok.all(), (p, ref)


def test_two_unit_charges_known_answer():
    # tests/test_system.cpp:28-50: PE = 1, a = -1 / +1 along x.
    x = np.array([[0.0, 0, 0], [1.0, 0, 0]])
    m = np.ones(2)
    q = np.ones(2)
    assert ol.potential(x, q) == pytest.approx(1.0, rel=1e-12)
    a = ol.accel(x, m, q)
    np.testing.assert_allclose(a, [[-1, 0, 0], [1, 0, 0]], rtol=1e-12, atol=1e-12)


def test_dp45_two_body_energy_conservation():
    # tests/test_integrator.cpp:34-56 (rtol 1e-10): energy kept to ~1e-7.
    x = np.array([[[0.0, 0, 0], [1.0, 0, 0]]])
    r = ol.run_batch(x, np.array([1.0, 2.0]), np.ones(2), bits=64, rtol=1e-10, atol=1e-16, pe_stop=1e-6,
                     redistribute=False)
    e0 = 1.0
    assert abs(r["ke_before"][0] + r["pe_final"][0] - e0) < 1e-7


def test_dp45_symmetric_explosion_momentum():
    # tests/test_integrator.cpp:58-82: equal masses from rest keep total momentum 0.
    x = np.array([[[-0.5, 0, 0], [0.5, 0, 0]]])
    r = ol.run_batch(x, np.ones(2), np.ones(2), bits=64)
    p = r["momenta"][0]
    assert abs(p[:, 0].sum()) <= 1e-10 * abs(p[0, 0])


def _golden_sets():
    out = []
    for fname in ("ch4_ref.npz", "h2o_ref.npz"):
        for tag in ("prod", "tight"):
            for bits in (32, 64):
                out.append((fname, tag, bits))
    return out


@pytest.mark.parametrize("fname,tag,bits", _golden_sets())
def test_oracle_bitexact_vs_reference_engine_golden(fname, tag, bits, wl):
    g = dict(np.load(GOLDEN / fname))
    rtol, atol, pes = {"prod": wl.PRODUCTION, "tight": wl.TIGHT}[tag]
    r = ol.run_batch(g["pos"], g["masses"], g["charges"], bits=bits, rtol=rtol, atol=atol, pe_stop=pes)
    np.testing.assert_array_equal(r["momenta"], g[f"p_{tag}_f{bits}"])
    np.testing.assert_array_equal(r["steps"], g[f"steps_{tag}_f{bits}"])
    np.testing.assert_array_equal(r["status"], g[f"status_{tag}_f{bits}"])


@pytest.mark.parametrize("bits", [32, 64])
def test_oracle_bitexact_vs_reference_engine_mixed_golden(golden_mixed, wl, bits):
    g = golden_mixed
    r = ol.run_batch_mixed(g["n_per"], g["masses"], g["charges"], g["pos"], bits=bits, rtol=wl.TIGHT[0],
                           atol=wl.TIGHT[1], pe_stop=wl.TIGHT[2])
    np.testing.assert_array_equal(r["momenta"], g[f"p_tight_f{bits}"])
    np.testing.assert_array_equal(r["steps"], g[f"steps_tight_f{bits}"])


def test_oracle_vs_scipy_oracle(golden_ch4, wl):
    g = golden_ch4
    n = len(g["p_scipy"])
    r = ol.run_batch(g["pos"][:n], g["masses"], g["charges"], bits=64, rtol=1e-10, atol=1e-16, pe_stop=1e-11)
    err = ol.config_norm_error(r["momenta"], g["p_scipy"])
    assert err.max() < 1e-7, err.max()


@pytest.mark.skipif(not ol.ref_available(), reason="reference engine (oracle/_ref) not built")
@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("n", [2, 3, 5, 7, 10])
def test_oracle_bitexact_vs_reference_engine_live(bits, n, wl):
    rng = np.random.default_rng(1000 + n)
    pos = wl.sample_ball(rng, 64, n, 2.0 * n ** (1 / 3), 0.4)
    mass = rng.choice([1.008, 12.011, 15.999, 32.06], n) * wl.AMU_TO_ME
    q = rng.integers(1, 4, n).astype(float)
    for rtol, atol, pes in (wl.PRODUCTION, wl.TIGHT):
        a = ol.run_batch(pos, mass, q, bits=bits, rtol=rtol, atol=atol, pe_stop=pes)
        b = ol.ref_run_batch(pos, mass, q, bits=bits, rtol=rtol, atol=atol, pe_stop=pes)
        np.testing.assert_array_equal(a["momenta"], b["momenta"])
        np.testing.assert_array_equal(a["steps"], b["steps"])
        np.testing.assert_array_equal(a["status"], b["status"])


@pytest.mark.skipif(not ol.ref_available(), reason="reference engine (oracle/_ref) not built")
def test_oracle_failure_codes_match_reference_engine(wl):
    mol = wl.CH4
    pos = wl.sample_molecule(mol, 8, seed=5)
    # Rejection limit: in f32 with rtol 0 / atol 1e-30 no attempt is ever
    # accepted and the reference throws after 100 rejections
    # (src/integrators.cpp:78-82); the oracle reports status 1 with the state kept.
    a = ol.run_batch(pos, mol.masses_me, mol.charge_array, bits=32, rtol=0.0, atol=1e-30, pe_stop=1e-7)
    b = ol.ref_run_batch(pos, mol.masses_me, mol.charge_array, bits=32, rtol=0.0, atol=1e-30, pe_stop=1e-7)
    assert (a["status"] == 1).all() and (b["status"] == 1).all()
    np.testing.assert_array_equal(a["momenta"], b["momenta"])
    # Coincident atoms: PE_0 = inf, so pe_stop = inf and the reference driver's
    # loop never runs (src/driver.cpp:19): zero steps, zero momenta, no error.
    # The oracle (like the GPU engine) returns the same zero momenta but flags
    # the sim as non-finite (status 3) instead of silently converged.
    pos = np.array([[[0.0, 0, 0], [0.0, 0, 0], [1.0, 0, 0]]])
    m, q = np.ones(3) * 1836.0, np.ones(3)
    a = ol.run_batch(pos, m, q, bits=32, rtol=1e-6, atol=1e-7, pe_stop=1e-7)
    b = ol.ref_run_batch(pos, m, q, bits=32, rtol=1e-6, atol=1e-7, pe_stop=1e-7)
    assert b["steps"][0] == 0 and not b["momenta"].any()
    assert a["status"][0] == 3 and a["steps"][0] == 0 and not a["momenta"].any()
    # max_steps reached first.
    pos = wl.sample_molecule(wl.CH4, 4, seed=5)
    a = ol.run_batch(pos, wl.CH4.masses_me, wl.CH4.charge_array, bits=32, rtol=1e-6, atol=1e-7,
                     pe_stop=1e-7, max_steps=3)
    b = ol.ref_run_batch(pos, wl.CH4.masses_me, wl.CH4.charge_array, bits=32, rtol=1e-6, atol=1e-7,
                         pe_stop=1e-7, max_steps=3)
    assert (a["status"] == 2).all() and (b["status"] == 2).all()
    np.testing.assert_array_equal(a["momenta"], b["momenta"])
