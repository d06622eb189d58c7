"""The C++ drop-in (coulomb::gpu, coulomb-explosion_b200/host) and the dataset pipeline.

The drop-in is built against the reference's own include/coulomb headers and
linked beside the reference's engine library (bin/libcoulomb_engine.so, compiled
from the reference's src/ by build.py).
CPU: one translation unit uses the reference's scalar driver, sampler and
BatchedRK45<float> next to coulomb::gpu, with Real = double and Real = float;
the reference sampler the test binaries link reproduces the golden draws; the
argument / exception contract. GPU: coulomb::gpu::BatchedRK45 and
run_to_convergence_batch against the oracle, the reference generator's call
shape against the reference's f32 engines, and bin/ce_generate_dataset end to
end, checked the way the reference's verify_subset.py (oracle on a subset,
config-norm error) and sanity_check.py (energy, momentum, species partition)
check its datasets.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
from pathlib import Path

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


def _reference_include():
    ref = os.environ.get("COULOMB_REFERENCE_DIR") or "/root/reference"
    inc = Path(ref) / "include"
    return inc if (inc / "coulomb" / "driver.hpp").exists() else None


@pytest.mark.skipif(_reference_include() is None or shutil.which("g++") is None,
                    reason="needs the reference's headers and g++")
def test_dropin_builds_and_links_beside_reference_engine(tmp_path):
    """coulomb::gpu uses the reference's coulomb:: types (no redeclaration), so
    one program can hold the reference's engine and the drop-in together."""
    inc = _reference_include()
    pkg = ROOT / "coulomb-explosion_b200"
    incs = ["-I", str(pkg / "host" / "include"), "-I", str(inc), "-I", str(ROOT / "include"),
            "-I", str(ROOT / "oracle" / "hwy_shim"), "-DWITH_REFERENCE_BATCHED"]
    src = ROOT / "tests" / "cpp" / "dropin_beside_engine.cpp"
    exe = tmp_path / "dropin"
    p = run("g++", "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror", *incs, src, "-L", pkg, "-lce_host", "-lce_gpu",
            "-L", BIN, "-lcoulomb_engine", f"-Wl,-rpath,{pkg}:{BIN}", "-o", exe)
    assert p.returncode == 0, p.stderr
    p = run(exe)
    assert p.returncode == 0 and "converged 1" in p.stdout, p.stdout + p.stderr
    # Real = float (COULOMB_SINGLE_PRECISION): the headers and the library sources compile too.
    for f in [src, *sorted((pkg / "host" / "src").glob("*.cpp"))]:
        p = run("g++", "-std=c++20", "-fsyntax-only", "-Wall", "-Wextra", "-Werror", "-DCOULOMB_SINGLE_PRECISION",
                *incs, "-I", "/usr/local/cuda/include", f)
        assert p.returncode == 0, f"{f.name}: {p.stderr}"
    # The drop-in's headers declare nothing in namespace coulomb itself, only coulomb::gpu.
    for h in (pkg / "host" / "include").rglob("*.hpp"):
        assert "namespace coulomb {" not in h.read_text(), h


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
    # E0 is the potential the device integrated: the float geometry, its pair terms
    # k q_i q_j / r formed in FP32 (as BatchedRK45<float> forms PE0 in T) and
    # summed in FP64, so it agrees with the FP64 potential to FP32 rounding.
    pe0 = np.array([ol.potential(x, mol.charge_array) for x in pos.astype(np.float32).astype(np.float64)])
    np.testing.assert_allclose(e0, pe0, rtol=1e-6)
    np.testing.assert_allclose(ker, e0, rtol=1e-6)


@pytest.mark.gpu
def test_generator_call_shape_matches_reference_engines(tmp_path, wl):
    """examples/generate_dataset.cpp:173-227 with coulomb::gpu::BatchedRK45 in
    place of BatchedRK45<float>: the reference's UniformSphereSampler fills the
    lanes, one run per batch. Geometries are the reference sampler's seed for
    seed; momenta within 1e-5 of the FP64 oracle and of the reference's f32
    engines (scalar and SIMD batched) at the tight point."""
    sims, lanes, seed = 5000, 1024, 49188291
    out = tmp_path / "gen.bin"
    p = run(TEST, "generate", sims, lanes, seed, "1e-6", "1e-7", out)
    assert p.returncode == 0, p.stdout + p.stderr
    rec = np.fromfile(out, dtype=np.dtype([("pos", "<f4", 15), ("p", "<f4", 15), ("steps", "<u4"), ("conv", "u1")]))
    assert len(rec) == sims and (rec["conv"] == 1).all()
    mol = wl.CH4
    pos = rec["pos"].reshape(sims, 5, 3).astype(np.float64)
    mom = rec["p"].reshape(sims, 5, 3).astype(np.float64)
    k = 1000
    if ol.ref_available():
        g = np.zeros((sims, 5, 3))
        assert ol.ref(64).ref_sample(4.0, 0.25, 10000, seed, 5, sims, ol._p(g)) == 0
        np.testing.assert_array_equal(rec["pos"].reshape(sims, 5, 3), g.astype(np.float32))
        f32 = ol.ref_run_batch(pos[:k], mol.masses_me, mol.charge_array, bits=32, rtol=1e-6, atol=1e-7, pe_stop=1e-7)
        assert ol.config_norm_error(mom[:k], f32["momenta"]).max() <= 1e-5
    ref = ol.run_batch(pos[:k], mol.masses_me, mol.charge_array, bits=64, rtol=1e-10, atol=1e-16, pe_stop=1e-11)
    assert ol.config_norm_error(mom[:k], ref["momenta"]).max() <= 1e-5
    if ol.batched_available():
        b32 = ol.batched_run(pos[:k], mol.masses_me, mol.charge_array, bits=32, rtol=1e-6, atol=1e-7, pe_stop=1e-7,
                             threads=4)
        assert ol.config_norm_error(mom[:k], b32["momenta"]).max() <= 1e-5


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
