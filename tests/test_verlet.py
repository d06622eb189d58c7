"""Velocity Verlet (IntegratorKind::VelocityVerlet, src/integrators.cpp:14-47)
under the convergence driver (src/driver.cpp:7-46).

CPU: the oracle's Velocity Verlet equals the reference engine's, built from its
own sources, bit for bit (f32 and f64), including max_steps truncation.
GPU: ce_run_verlet_device equals the oracle's f32 run bit for bit (momenta,
steps, status, t_final, pe_final), and rejects a non-positive step and precision
modes.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle_lib as ol

CASES = [(5.0, 0.05), (2.0, 0.01)]


def _geoms(wl, mol, S, seed):
    return wl.sample_molecule(mol, S, seed=seed).astype(np.float32).astype(np.float64)


@pytest.mark.skipif(not ol.ref_available(), reason="reference engine not built")
@pytest.mark.parametrize("bits", [32, 64])
@pytest.mark.parametrize("dt,pes", CASES)
def test_oracle_verlet_matches_reference(wl, bits, dt, pes):
    for mol in (wl.CH4, wl.C2H6_LIKE):
        pos = _geoms(wl, mol, 48, seed=7)
        o = ol.run_batch(pos, mol.masses_me, mol.charge_array, bits=bits, pe_stop=pes, max_dt=dt, integrator=1)
        r = ol.ref_run_batch(pos, mol.masses_me, mol.charge_array, bits=bits, pe_stop=pes, max_dt=dt, integrator=1)
        assert np.array_equal(o["momenta"], r["momenta"])
        assert np.array_equal(o["steps"], r["steps"])
        assert np.array_equal(o["t_final"], r["t_final"])
        assert np.all(o["status"] == 0) and np.all(r["status"] == 0)
        assert o["steps"].min() > 50


@pytest.mark.skipif(not ol.ref_available(), reason="reference engine not built")
def test_oracle_verlet_max_steps_matches_reference(wl):
    mol = wl.CH4
    pos = _geoms(wl, mol, 16, seed=8)
    o = ol.run_batch(pos, mol.masses_me, mol.charge_array, bits=32, pe_stop=1e-3, max_dt=5.0, max_steps=40,
                     integrator=1)
    r = ol.ref_run_batch(pos, mol.masses_me, mol.charge_array, bits=32, pe_stop=1e-3, max_dt=5.0, max_steps=40,
                         integrator=1)
    assert np.all(o["status"] == 2) and np.all(r["status"] == 2)  # max_steps
    assert np.array_equal(o["momenta"], r["momenta"]) and np.all(o["steps"] == 40)


def _run_gpu(ce, engine, mol, pos32, dt, pes, max_steps=1_000_000):
    torch = pytest.importorskip("torch")
    S = pos32.shape[0]
    engine.set_molecule(mol.masses_me, mol.charge_array)
    x = torch.from_numpy(np.ascontiguousarray(pos32)).cuda()
    d = {"m": torch.zeros((S, mol.n, 3), device="cuda"), "k": torch.zeros(S, dtype=torch.float64, device="cuda"),
         "s": torch.zeros(S, dtype=torch.int32, device="cuda"), "st": torch.zeros(S, dtype=torch.uint8, device="cuda"),
         "t": torch.zeros(S, dtype=torch.float64, device="cuda"), "pe": torch.zeros(S, dtype=torch.float64, device="cuda")}
    out = ce.CeOutputs(d["m"].data_ptr(), d["k"].data_ptr(), d["s"].data_ptr(), d["st"].data_ptr(), None,
                       d["t"].data_ptr(), d["pe"].data_ptr())
    cfg = ce.RunConfig(pe_stop_fraction=pes, max_dt=dt, max_steps=max_steps)
    engine.run_verlet_device(S, x.data_ptr(), cfg, out)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in d.items()}


@pytest.mark.gpu
@pytest.mark.parametrize("dt,pes", CASES)
def test_gpu_verlet_matches_oracle_bit_for_bit(ce, engine, wl, dt, pes):
    for mol in (wl.CH4, wl.C2H6_LIKE):
        pos = _geoms(wl, mol, 256, seed=9)
        g = _run_gpu(ce, engine, mol, pos.astype(np.float32), dt, pes)
        o = ol.run_batch(pos, mol.masses_me, mol.charge_array, bits=32, pe_stop=pes, max_dt=dt, integrator=1)
        assert np.array_equal(g["m"].astype(np.float64), o["momenta"])
        assert np.array_equal(g["s"].astype(np.uint32), o["steps"])
        assert np.array_equal(g["st"], o["status"])
        assert np.array_equal(g["t"], o["t_final"]) and np.array_equal(g["pe"], o["pe_final"])
        np.testing.assert_allclose(g["k"], o["ker"], rtol=1e-12)


@pytest.mark.gpu
def test_gpu_verlet_max_steps_and_errors(ce, engine, wl):
    mol = wl.CH4
    pos = _geoms(wl, mol, 64, seed=10)
    g = _run_gpu(ce, engine, mol, pos.astype(np.float32), 5.0, 1e-3, max_steps=40)
    assert np.all(g["st"] == ce.CE_SIM_MAX_STEPS) and np.all(g["s"] == 40)
    torch = pytest.importorskip("torch")
    x = torch.zeros((4, 5, 3), device="cuda")
    m = torch.zeros((4, 5, 3), device="cuda")
    out = ce.CeOutputs(m.data_ptr())
    with pytest.raises(ce.EngineError):
        engine.run_verlet_device(4, x.data_ptr(), ce.RunConfig(max_dt=0.0), out)
    with pytest.raises(ce.EngineError):
        engine.run_verlet_device(4, x.data_ptr(), ce.RunConfig(max_dt=1.0, precision_mode=1), out)
