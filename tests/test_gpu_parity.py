"""Parity of the CUDA engine (through the C ABI) with the oracle and the
reference engine's golden outputs.

Error statistic: per-sim config-norm ||p - p_ref|| / ||p_ref|| over all 3N
momentum components (python/analysis/plot_precision.py:52-56).

Tolerances, stated once:
  TIGHT point (rtol 1e-6, atol 1e-7, pe_stop 1e-7): every sim within 1e-5 of the
      reference f32 engine, of the reference f64 engine and of the scipy oracle
      (<= 1e-5 relative momentum error, max over the set).
  PRODUCTION point (rtol 1e-4, atol 1e-7, pe_stop 1e-5): the reference's own f32
      and f64 engines already differ by up to ~5e-5 there (accept/reject flips),
      so parity is statistical: median <= 1e-6, p99 <= 2e-5, max <= 5e-4.
"""
from __future__ import annotations

import json

import numpy as np
import pytest

import oracle_lib as ol
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TIGHT_MAX = 1e-5
PROD_MEDIAN, PROD_P99, PROD_MAX = 1e-6, 2e-5, 5e-4


def cfg_for(ce, point, mode=0, **kw):
    rtol, atol, pes = point
    return ce.RunConfig(rtol=rtol, atol=atol, pe_stop_fraction=pes, precision_mode=mode, **kw)


def run(engine, ce, mol_m, mol_q, pos, point, mode=0, diagnostics=False, **kw):
    engine.set_molecule(mol_m, mol_q)
    return engine.run(np.asarray(pos, np.float32), cfg_for(ce, point, mode, **kw), diagnostics=diagnostics)


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_ch4_tight_matches_reference_engine(engine, ce, wl, golden_ch4, mode):
    g = golden_ch4
    r = run(engine, ce, g["masses"], g["charges"], g["pos"], wl.TIGHT, mode)
    assert (r.status == 0).all()
    for bits in (32, 64):
        err = ol.config_norm_error(r.momenta, g[f"p_tight_f{bits}"])
        assert err.max() <= TIGHT_MAX, (bits, err.max())
    steps_ref = g["steps_tight_f32"].astype(float)
    assert abs(r.steps.mean() - steps_ref.mean()) <= 0.03 * steps_ref.mean()


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("point", ["prod", "tight"])
def test_ch4_thread_per_sim_layout_matches_reference_engine(engine, ce, wl, golden_ch4, mode, point):
    """The thread-per-sim kernel (rolled stage loop, stages in shared memory) on
    the CH4 golden set, every precision mode, both tolerance points."""
    g = golden_ch4
    engine.set_tuning(lanes_per_sim=1)
    try:
        r = run(engine, ce, g["masses"], g["charges"], g["pos"], wl.TIGHT if point == "tight" else wl.PRODUCTION,
                mode)
    finally:
        engine.set_tuning()
    assert (r.status == 0).all()
    if point == "tight":
        for bits in (32, 64):
            err = ol.config_norm_error(r.momenta, g[f"p_tight_f{bits}"])
            assert err.max() <= TIGHT_MAX, (bits, err.max())
        steps_ref = g["steps_tight_f32"].astype(float)
    else:
        err = ol.config_norm_error(r.momenta, g["p_prod_f32"])
        assert np.median(err) <= PROD_MEDIAN and np.percentile(err, 99) <= PROD_P99 and err.max() <= PROD_MAX, (
            np.median(err), np.percentile(err, 99), err.max())
        steps_ref = g["steps_prod_f32"].astype(float)
    assert abs(r.steps.mean() - steps_ref.mean()) <= 0.03 * steps_ref.mean()


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("point", ["prod", "tight"])
def test_ch4_two_thread_layout_matches_reference_engine(engine, ce, wl, golden_ch4, mode, point):
    """The two-thread layout on the CH4 golden set (5 atoms: 3 + 2, the second
    thread's last slot a phantom), every precision mode, both tolerance points."""
    g = golden_ch4
    engine.set_tuning(lanes_per_sim=2)
    try:
        r = run(engine, ce, g["masses"], g["charges"], g["pos"], wl.TIGHT if point == "tight" else wl.PRODUCTION,
                mode, diagnostics=True)
    finally:
        engine.set_tuning()
    assert (r.status == 0).all()
    if point == "tight":
        for bits in (32, 64):
            err = ol.config_norm_error(r.momenta, g[f"p_tight_f{bits}"])
            assert err.max() <= TIGHT_MAX, (bits, err.max())
        steps_ref = g["steps_tight_f32"].astype(float)
    else:
        err = ol.config_norm_error(r.momenta, g["p_prod_f32"])
        assert np.median(err) <= PROD_MEDIAN and np.percentile(err, 99) <= PROD_P99 and err.max() <= PROD_MAX, (
            np.median(err), np.percentile(err, 99), err.max())
        steps_ref = g["steps_prod_f32"].astype(float)
    assert abs(r.steps.mean() - steps_ref.mean()) <= 0.03 * steps_ref.mean()
    # KER = E_0, and the FP64 sums over both threads' atoms
    np.testing.assert_allclose(r.ker, r.e0, rtol=1e-9)
    assert np.isfinite(r.positions).all() and (np.abs(r.positions) < 1e12).all()  # no phantom written out


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("n", [7, 8, 9, 10])
def test_two_thread_layout_every_mode_matches_oracle(engine, ce, wl, n, mode):
    """Seven to ten atoms, where the two-thread layout is meant to run (odd
    counts carry a phantom), every precision mode, against the FP64 oracle at
    the tight point, plus the potential / energy bookkeeping."""
    rng = np.random.default_rng(700 + n)
    pos = wl.sample_ball(rng, 160, n, 2.0 * n ** (1 / 3), 0.5).astype(np.float32)
    mass = rng.choice([1.008, 12.011, 14.007, 15.999, 32.06], n) * wl.AMU_TO_ME
    q = rng.integers(1, 4, n).astype(float)
    engine.set_tuning(lanes_per_sim=2)
    try:
        r = run(engine, ce, mass, q, pos, wl.TIGHT, mode, diagnostics=True)
    finally:
        engine.set_tuning()
    ref = ol.run_batch(pos.astype(np.float64), mass, q, bits=64, rtol=wl.TIGHT[0], atol=wl.TIGHT[1],
                       pe_stop=wl.TIGHT[2])
    assert (r.status == ce.CE_SIM_OK).all()
    err = ol.config_norm_error(r.momenta, ref["momenta"])
    assert err.max() <= TIGHT_MAX, err.max()
    np.testing.assert_allclose(r.e0, ref["ker"], rtol=1e-6)  # the oracle's KER is its E_0 = PE_0
    np.testing.assert_allclose(r.ker, r.e0, rtol=1e-9)
    assert (r.pe_final <= wl.TIGHT[2] * r.e0 * (1 + 1e-6)).all()


def test_ch4_tight_matches_scipy_oracle(engine, ce, wl, golden_ch4):
    g = golden_ch4
    n = len(g["p_scipy"])
    r = run(engine, ce, g["masses"], g["charges"], g["pos"][:n], wl.TIGHT, 3)
    err = ol.config_norm_error(r.momenta, g["p_scipy"])
    assert err.max() <= TIGHT_MAX, err.max()


def test_ch4_production_point_statistics(engine, ce, wl, golden_ch4):
    g = golden_ch4
    r = run(engine, ce, g["masses"], g["charges"], g["pos"], wl.PRODUCTION, 0)
    assert (r.status == 0).all()
    err = ol.config_norm_error(r.momenta, g["p_prod_f32"])
    assert np.median(err) <= PROD_MEDIAN and np.percentile(err, 99) <= PROD_P99 and err.max() <= PROD_MAX, (
        np.median(err), np.percentile(err, 99), err.max())
    steps_ref = g["steps_prod_f32"].astype(float)
    assert abs(r.steps.mean() - steps_ref.mean()) <= 0.03 * steps_ref.mean()


@pytest.mark.parametrize("point", ["prod", "tight"])
def test_stiff_h2o_matches_reference_engine(engine, ce, wl, golden_h2o, point):
    g = golden_h2o
    pt = wl.PRODUCTION if point == "prod" else wl.TIGHT
    r = run(engine, ce, g["masses"], g["charges"], g["pos"], pt, 3)
    assert (r.status == 0).all()
    err = ol.config_norm_error(r.momenta, g[f"p_{point}_f64"])
    if point == "tight":
        assert err.max() <= TIGHT_MAX, err.max()
    else:
        assert np.median(err) <= 10 * PROD_MEDIAN and err.max() <= 10 * PROD_MAX, (np.median(err), err.max())


def test_reference_golden_cases(engine, ce, wl):
    doc = json.loads((GOLDEN / "reference_cases.json").read_text())
    for c in doc["cases"]:
        m, q = np.array(c["masses"]), np.array(c["charges"])
        r = run(engine, ce, m, q, np.array(c["positions_init"])[None], wl.TIGHT, 3)
        assert r.status[0] == 0
        err = ol.config_norm_error(r.momenta, np.array(c["momenta_final"])[None])
        assert err[0] <= TIGHT_MAX, (c["name"], err[0])
        # KER = E_0 = PE_0 after redistribution (demo/sanity_check.py:89-96)
        assert r.ker[0] == pytest.approx(c["potential_energy_init"], rel=1e-6)


LAYOUT_LANES = {"sim": lambda n: 1, "pair": lambda n: 2, "atom": lambda n: n}


@pytest.mark.parametrize("layout", ["sim", "pair", "atom"])
@pytest.mark.parametrize("n", list(range(1, 11)))
def test_every_atom_count_matches_oracle(engine, ce, wl, n, layout):
    if layout == "atom" and n == 1:
        pytest.skip("the lane-per-atom layout needs at least two atoms")
    if layout == "pair" and n < 3:
        pytest.skip("the two-thread layout starts at three atoms")
    rng = np.random.default_rng(50 + n)
    pos = wl.sample_ball(rng, 200, n, 2.0 * n ** (1 / 3), 0.5).astype(np.float32)
    mass = rng.choice([1.008, 12.011, 14.007, 15.999, 32.06], n) * wl.AMU_TO_ME
    q = rng.integers(1, 4, n).astype(float)
    engine.set_tuning(lanes_per_sim=LAYOUT_LANES[layout](n))
    try:
        r = run(engine, ce, mass, q, pos, wl.TIGHT, 3)
    finally:
        engine.set_tuning()
    ref = ol.run_batch(pos.astype(np.float64), mass, q, bits=64, rtol=wl.TIGHT[0], atol=wl.TIGHT[1],
                       pe_stop=wl.TIGHT[2])
    if n == 1:  # a lone ion: PE_0 = 0 = pe_stop, zero steps, zero momenta
        assert (r.status == 0).all() and (r.steps == 0).all() and not r.momenta.any()
        return
    assert (r.status == 0).all()
    err = ol.config_norm_error(r.momenta, ref["momenta"])
    assert err.max() <= TIGHT_MAX, err.max()
    np.testing.assert_allclose(r.ker, ref["ker"], rtol=1e-6)


def test_diagnostics_and_energy_bookkeeping(engine, ce, wl, golden_ch4):
    g = golden_ch4
    r = run(engine, ce, g["masses"], g["charges"], g["pos"], wl.TIGHT, 3, diagnostics=True)
    o = ol.run_batch(g["pos"], g["masses"], g["charges"], bits=32, mode=3, rtol=wl.TIGHT[0], atol=wl.TIGHT[1],
                     pe_stop=wl.TIGHT[2])
    pe0 = np.array([ol.potential(x, g["charges"]) for x in g["pos"]])
    # stop criterion met: PE_final <= pe_stop * PE_0
    assert (r.pe_final <= wl.TIGHT[2] * pe0 * (1 + 1e-5)).all()
    # energy drift before redistribution |KE + PE_final - E_0| / E_0 is small
    drift = np.abs(r.ke_before + r.pe_final - pe0) / pe0
    assert drift.max() < 1e-5, drift.max()
    # t_final is dominated by the last (largest) accepted step, whose size
    # depends on the whole step-size history, so it is not a parity quantity:
    # only its magnitude is checked (same decade as the oracle's).
    assert np.isfinite(r.t_final).all() and (r.t_final > 0).all()
    assert (np.abs(np.log10(r.t_final / o["t_final"])) < 1.0).all()
    assert abs(int(r.rejects.sum()) - int(o["rejects"].sum())) <= 0.1 * len(r.rejects) + 10


def test_ragged_sizes_and_empty(engine, ce, wl):
    mol = wl.CH4
    engine.set_molecule(mol.masses_me, mol.charge_array)
    cfg = cfg_for(ce, wl.TIGHT, 0)
    r0 = engine.run(np.zeros((0, 5, 3), np.float32), cfg)
    assert r0.momenta.shape == (0, 5, 3)
    pos = wl.sample_molecule(mol, 1000, seed=11).astype(np.float32)
    full = engine.run(pos, cfg)
    for S in (1, 31, 33, 257, 999):
        part = engine.run(pos[:S], cfg)
        np.testing.assert_array_equal(part.momenta, full.momenta[:S])
        np.testing.assert_array_equal(part.steps, full.steps[:S])


@pytest.mark.parametrize("case", ["ch4_thread_streamed", "c2h6_pair_streamed", "nine_atoms_pair_streamed",
                                  "ch4_lane_chunked"])
def test_host_buffer_paths_match_device_path(engine, ce, wl, case):
    # ce_run, host buffers (pageable here), must give bit for bit what one
    # ce_run_device launch gives, in every output. The thread-per-sim and
    # two-thread layouts stream their I/O around one launch (positions up in
    # chunks the kernel waits for, results down chunk by chunk as the kernel
    # completes them: 29 chunks here, the last one short); the lane-per-atom
    # layout cuts the batch into chunks that alternate between two device slots,
    # each integrated on its own stream with its own work queue (7 chunks here,
    # the two at each end tapered).
    torch = pytest.importorskip("torch")
    S = 7 * 65536 + 777
    if case == "nine_atoms_pair_streamed":  # an odd count: the second thread carries a phantom slot
        rng = np.random.default_rng(909)
        mass = rng.choice([1.008, 12.011, 14.007, 15.999, 32.06], 9) * wl.AMU_TO_ME
        q = rng.integers(1, 4, 9).astype(float)
        engine.set_molecule(mass, q)
        pos = wl.sample_ball(rng, S, 9, 2.0 * 9 ** (1 / 3), 0.5).astype(np.float32)
        lanes, mode = 0, 0
    else:
        mol, lanes, mode = {"ch4_thread_streamed": (wl.CH4, 0, 3), "c2h6_pair_streamed": (wl.C2H6_LIKE, 0, 0),
                            "ch4_lane_chunked": (wl.CH4, 5, 3)}[case]
        engine.set_molecule(mol.masses_me, mol.charge_array)
        pos = wl.sample_molecule(mol, S, seed=41).astype(np.float32)
    cfg = cfg_for(ce, wl.TIGHT, mode)
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(pos).to(dev)
    names = ("momenta", "ker", "steps", "status", "rejects", "t_final", "pe_final", "ke_before", "positions", "e0")
    engine.set_tuning(lanes_per_sim=lanes)
    try:
        host = engine.run(pos, cfg, diagnostics=True)
        assert engine.last_launch_count() == (1 if lanes == 0 else 7)
        # raw byte buffers on the device, read back with each output's dtype and shape
        d = {k: torch.zeros(getattr(host, k).nbytes, dtype=torch.uint8, device=dev) for k in names}
        out = ce.CeOutputs(*(d[k].data_ptr() for k in names))
        stream = torch.cuda.Stream(device=dev)
        engine.run_device(S, x.data_ptr(), cfg, out, stream.cuda_stream)
        stream.synchronize()
    finally:
        engine.set_tuning()
    assert (host.status == 0).all()
    for k in names:
        h = getattr(host, k)
        np.testing.assert_array_equal(h, d[k].cpu().numpy().view(h.dtype).reshape(h.shape), err_msg=k)


def test_host_buffer_path_with_blocking_launches(ce, wl, tmp_path):
    # With blocking launches (or a tool injected into the CUDA runtime, which
    # serialises kernels and copies) the streamed ce_run could not overlap its
    # copies with its kernel; ce_run then takes the chunked pipeline. A child
    # process with CUDA_LAUNCH_BLOCKING=1 must finish promptly with the same bits
    # as this process's streamed run.
    import os
    import subprocess
    import sys

    from conftest import ROOT

    mol = wl.CH4
    S = 1 << 19  # three chunks in the chunked pipeline
    pos = wl.sample_molecule(mol, S, seed=43).astype(np.float32)
    np.save(tmp_path / "pos.npy", pos)
    eng = ce.Engine(0)
    try:
        eng.set_molecule(mol.masses_me, mol.charge_array)
        here = eng.run(pos, cfg_for(ce, wl.TIGHT, 0))
        assert eng.last_launch_count() == 1  # streamed: one launch
    finally:
        eng.close()
    script = (
        "import sys, numpy as np\n"
        f"sys.path.insert(0, {str(ROOT)!r})\n"
        "import __graft_entry__ as g\n"
        "ce = g.load_package()\n"
        "from coulomb_explosion_b200 import workloads as wl\n"
        f"pos = np.load({str(tmp_path / 'pos.npy')!r})\n"
        "e = ce.Engine(0)\n"
        "e.set_molecule(wl.CH4.masses_me, wl.CH4.charge_array)\n"
        "r = e.run(pos, ce.RunConfig(rtol=1e-6, atol=1e-7, pe_stop_fraction=1e-7, precision_mode=0))\n"
        "assert e.last_launch_count() > 1, e.last_launch_count()\n"
        f"np.save({str(tmp_path / 'mom.npy')!r}, r.momenta)\n"
        "e.close()\n")
    env = dict(os.environ, CUDA_LAUNCH_BLOCKING="1")
    subprocess.run([sys.executable, "-c", script], env=env, check=True, timeout=300)
    np.testing.assert_array_equal(np.load(tmp_path / "mom.npy"), here.momenta)


def test_full_size_invariants(engine, ce, wl):
    # The benchmark's full size (1e6 CH4 explosions, tight point, plain FP32),
    # checked per sim through properties that hold at any size: every sim
    # converges, KER equals E_0 after redistribution, the momenta sum to zero
    # (the reference's check, demo/sanity_check.py:102-106: mean over sims of
    # |sum p| / the typical per-atom |p| below 1e-4; here also every sim's
    # |sum p| / sum |p|), and a second run reproduces every bit.
    torch = pytest.importorskip("torch")
    import importlib

    sp = importlib.import_module("coulomb_explosion_b200.sampling")
    mol = wl.CH4
    S = 1_000_000
    pos, _, flags = sp.sample_ball_host(mol, S, seed=20261203)
    assert not flags.any()
    engine.set_molecule(mol.masses_me, mol.charge_array)
    cfg = cfg_for(ce, wl.TIGHT, 0)
    x = torch.from_numpy(pos).cuda()
    runs = []
    for _ in range(2):
        mom = torch.zeros((S, mol.n, 3), dtype=torch.float32, device="cuda")
        ker = torch.zeros(S, dtype=torch.float64, device="cuda")
        steps = torch.zeros(S, dtype=torch.int32, device="cuda")
        status = torch.full((S,), 255, dtype=torch.uint8, device="cuda")
        e0 = torch.zeros(S, dtype=torch.float64, device="cuda")
        out = ce.CeOutputs(mom.data_ptr(), ker.data_ptr(), steps.data_ptr(), status.data_ptr(), None, None, None,
                           None, None, e0.data_ptr())
        stream = torch.cuda.Stream()
        engine.run_device(S, x.data_ptr(), cfg, out, stream.cuda_stream)
        stream.synchronize()
        runs.append([t.cpu().numpy() for t in (mom, ker, steps, status, e0)])
    mom, ker, steps, status, e0 = runs[0]
    assert (status == ce.CE_SIM_OK).all()
    assert np.abs(ker / e0 - 1.0).max() < 1e-9
    p = mom.astype(np.float64)
    tot = np.linalg.norm(p.sum(axis=1), axis=1)
    assert (tot / np.linalg.norm(p, axis=2).mean()).mean() < 1e-4
    assert (tot / np.linalg.norm(p, axis=2).sum(axis=1)).max() < 1e-4
    assert 30 < steps.mean() < 60
    for a, b in zip(runs[0], runs[1]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("lanes", [1, 2, 5])
def test_results_independent_of_launch_shape(engine, ce, wl, lanes):
    # Each sim's arithmetic is private to its thread (or its lane group), so
    # block size, grid size and refill granularity cannot change a single bit.
    mol = wl.CH4
    engine.set_molecule(mol.masses_me, mol.charge_array)
    pos = wl.sample_molecule(mol, 3000, seed=12).astype(np.float32)
    cfg = cfg_for(ce, wl.TIGHT, 3)
    engine.set_tuning(lanes_per_sim=lanes)
    base = engine.run(pos, cfg)
    try:
        for bt, bps, thr in ((32, 0, 1), (64, 1, 8), (256, 0, 32), (96, 2, 4)):
            engine.set_tuning(block_threads=bt, blocks_per_sm=bps, refill_threshold=thr, lanes_per_sim=lanes)
            r = engine.run(pos, cfg)
            np.testing.assert_array_equal(r.momenta, base.momenta)
            np.testing.assert_array_equal(r.steps, base.steps)
            np.testing.assert_array_equal(r.ker, base.ker)
    finally:
        engine.set_tuning()


def test_failure_status_codes(engine, ce, wl):
    mol = wl.CH4
    engine.set_molecule(mol.masses_me, mol.charge_array)
    pos = wl.sample_molecule(mol, 64, seed=13).astype(np.float32)
    # max_steps reached first -> status 2, steps == max_steps (src/driver.cpp:20-23)
    r = engine.run(pos, ce.RunConfig(rtol=1e-6, atol=1e-7, pe_stop_fraction=1e-7, max_steps=3), diagnostics=True)
    assert (r.status == ce.CE_SIM_MAX_STEPS).all() and (r.steps == 3).all()
    o = ol.run_batch(pos.astype(np.float64), mol.masses_me, mol.charge_array, bits=32, rtol=1e-6, atol=1e-7,
                     pe_stop=1e-7, max_steps=3)
    # A run cut at 3 steps is path dependent: the f32 embedded-error estimate is
    # a small difference of large stage terms, so two correct f32 formulations
    # pick step sizes that differ at ~1e-4 relative; after only three steps
    # that shows directly in t_final and in the (not yet asymptotic) momenta.
    # A flipped accept/reject in those three steps changes t_final by up to tens
    # of percent; sims that took the same path (t_final within 1e-3) must agree.
    assert np.isfinite(r.momenta).all()
    np.testing.assert_allclose(r.ker, o["ker"], rtol=1e-5)  # KER = E_0 either way
    same = np.abs(r.t_final - o["t_final"]) <= 1e-3 * o["t_final"]
    assert same.sum() >= 8, same.sum()
    assert ol.config_norm_error(r.momenta[same], o["momenta"][same]).max() < 1e-3
    # rejection limit -> status 1 (the reference throws, src/integrators.cpp:78-82)
    r = engine.run(pos, ce.RunConfig(rtol=0.0, atol=1e-30, pe_stop_fraction=1e-7))
    assert (r.status == ce.CE_SIM_REJECT_LIMIT).all()
    # already below the stop (pe_stop_fraction >= 1): zero steps, at rest
    r = engine.run(pos, ce.RunConfig(rtol=1e-6, atol=1e-7, pe_stop_fraction=1.0))
    assert (r.status == 0).all() and (r.steps == 0).all() and not r.momenta.any()
    # NaN coordinates and coincident atoms -> non-finite initial energy -> status 3
    bad = pos[:4].copy()
    bad[0, 2, 1] = np.nan
    bad[1, 3] = bad[1, 0]
    r = engine.run(bad, ce.RunConfig(rtol=1e-6, atol=1e-7, pe_stop_fraction=1e-7))
    assert r.status[0] == ce.CE_SIM_NONFINITE and r.status[1] == ce.CE_SIM_NONFINITE
    assert (r.status[2:] == 0).all()
    # redistribution off: KER is the raw kinetic energy, below E_0
    r = engine.run(pos, ce.RunConfig(rtol=1e-6, atol=1e-7, pe_stop_fraction=1e-7, redistribute_energy=False),
                   diagnostics=True)
    np.testing.assert_allclose(r.ker, r.ke_before, rtol=1e-6)


def test_invalid_arguments_are_rejected(engine, ce):
    with pytest.raises(ce.EngineError):
        engine.set_molecule(np.ones(11), np.ones(11))
    with pytest.raises(ce.EngineError):
        engine.set_molecule(np.array([1.0, -1.0]), np.ones(2))
    engine.set_molecule(np.ones(2) * 1836.0, np.ones(2))
    with pytest.raises(ce.EngineError):
        engine.run(np.zeros((4, 2, 3), np.float32), ce.RunConfig(rtol=0.0, atol=0.0))
    with pytest.raises(ce.EngineError):
        engine.run(np.zeros((4, 2, 3), np.float32), ce.RunConfig(max_dt=0.0))
    with pytest.raises(ce.EngineError):
        engine.set_tuning(block_threads=48)
