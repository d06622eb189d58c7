"""The C++ host API (coulomb-explosion_b200/host) and the dataset pipeline.

CPU: the host mirror of the reference sampler reproduces the reference's own
draws bit for bit (golden vectors from its UniformSphereSampler), and the
argument / exception contract. GPU: coulomb::gpu::BatchedRK45 and
run_to_convergence_batch against the oracle, and bin/ce_generate_dataset end to
end, checked the way the reference's verify_subset.py (oracle on a subset,
config-norm error) and sanity_check.py (energy, momentum, species partition)
check its datasets.
"""
from __future__ import annotations

import json
import subprocess

import numpy as np
import pytest

import oracle_lib as ol
from conftest import GOLDEN, ROOT
from pkg_loader import load_submodule

BIN = ROOT / "coulomb-explosion_b200" / "bin"
TEST = BIN / "ce_test_host"
GEN = BIN / "ce_generate_dataset"


def run(*args, timeout=600):
    return subprocess.run([str(a) for a in args], capture_output=True, text=True, timeout=timeout)


@pytest.mark.parametrize("seed,n,r,d", [(49188291, 5, 4.0, 0.25), (7, 10, 4.0, 0.5), (123, 3, 2.0, 0.3)])
def test_uniform_sphere_sampler_reproduces_reference_draws(tmp_path, seed, n, r, d):
    g = np.load(GOLDEN / "sampler_ref.npz")[f"pos_{seed}_{n}"]
    out = tmp_path / "s.bin"
    p = run(TEST, "sampler", seed, n, r, d, len(g), out)
    assert p.returncode == 0, p.stderr
    got = np.fromfile(out, dtype=np.float64).reshape(g.shape)
    np.testing.assert_array_equal(got, g)


def test_argument_and_exception_contract():
    p = run(TEST, "errors")
    assert p.returncode == 0, p.stdout + p.stderr


@pytest.mark.gpu
def test_batched_rk45_dropin_and_batched_driver(tmp_path, wl):
    S, n = 2000, 5
    out = tmp_path / "g.bin"
    p = run(TEST, "gpu", S, out)
    assert p.returncode == 0, p.stdout + p.stderr
    raw = out.read_bytes()
    off = 0

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off)
        off += a.nbytes
        return a

    pos = take(np.float64, S * n * 3).reshape(S, n, 3)
    mom = take(np.float64, S * n * 3).reshape(S, n, 3)
    mom_drv = take(np.float64, S * n * 3).reshape(S, n, 3)
    e0 = take(np.float64, S)
    ker = take(np.float64, S)
    steps = take(np.uint32, S)
    status = take(np.uint8, S)
    assert (status == 0).all() and steps.min() > 0
    mol = wl.CH4
    ref = ol.run_batch(pos.astype(np.float32).astype(np.float64), mol.masses_me, mol.charge_array, bits=64,
                       rtol=1e-10, atol=1e-16, pe_stop=1e-11)
    assert ol.config_norm_error(mom, ref["momenta"]).max() <= 1e-5
    np.testing.assert_allclose(mom_drv, mom, rtol=1e-12, atol=1e-9)
    pe0 = np.array([ol.potential(x, mol.charge_array) for x in pos])
    np.testing.assert_allclose(e0, pe0, rtol=1e-12)
    np.testing.assert_allclose(ker, e0, rtol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("sampler", ["philox", "uniform-sphere"])
def test_generate_dataset_end_to_end(tmp_path, wl, sampler):
    ds = load_submodule("dataset")
    out = tmp_path / "ch4.bin"
    S = 150_000
    p = run(GEN, "--out", out, "--sims", S, "--chunk", 65536, "--sampler", sampler, "--rtol", "1e-6",
            "--pe-stop", "1e-7", "--seed", 49188291)
    assert p.returncode == 0, p.stdout + p.stderr
    meta, rec = ds.read_dataset(out)
    assert len(rec) == S == meta["n_sims"] and meta["n_failed_convergence"] == 0
    assert meta["symbols"] == ["C", "H", "H", "H", "H"] and meta["lanes"] == 65536
    s = ds.sanity(meta, rec, 50_000)
    assert s["ker_vs_pe_max_rel"] < 1e-4 and s["momentum_ratio_mean"] < 1e-4 and s["converged_frac"] == 1.0
    for measured, predicted in s["partition"].values():
        assert abs(measured - predicted) < 0.01
    # verify_subset: the first 200 records against the FP64 oracle
    k = 200
    x = rec["init_pos"][:k].reshape(k, 5, 3).astype(np.float64)
    pf = rec["final_p"][:k].reshape(k, 5, 3).astype(np.float64)
    mol = wl.CH4
    ref = ol.run_batch(x, mol.masses_me, mol.charge_array, bits=64, rtol=1e-10, atol=1e-16, pe_stop=1e-11)
    assert ol.config_norm_error(pf, ref["momenta"]).max() <= 1e-5
    if sampler == "uniform-sphere" and ol.ref_available():
        # the geometries are the reference sampler's own, seed for seed
        g = np.zeros((k, 5, 3))
        assert ol.ref(64).ref_sample(4.0, 0.25, 10000, 49188291, 5, k, ol._p(g)) == 0
        np.testing.assert_array_equal(rec["init_pos"][:k].reshape(k, 5, 3), g.astype(np.float32))
