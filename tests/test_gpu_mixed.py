"""Mixed 2..10-atom batches (one persistent launch over size buckets, or one
launch per size), CUDA-graph capture and the autotuner, through the C ABI.

Parity bar as in test_gpu_parity.py: at the tight point every sim within 1e-5
config-norm relative momentum error of the reference engine (golden mixed set:
the reference's scalar engine run per molecule) and of the oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu

TIGHT_MAX = 1e-5


def tight(ce, wl, mode=3, **kw):
    r, a, p = wl.TIGHT
    return ce.RunConfig(rtol=r, atol=a, pe_stop_fraction=p, precision_mode=mode, **kw)


def per_sim_err(r, ref, n_per):
    return per_sim_err_arrays(r.momenta, ref, n_per)


def per_sim_err_arrays(p, ref, n_per):
    errs = []
    for s, n in enumerate(n_per):
        errs.append(ol.config_norm_error(p[s:s + 1, :n], ref[s:s + 1, :n])[0])
    return np.array(errs)


@pytest.mark.parametrize("lanes", [0, 2])
@pytest.mark.parametrize("bits", [32, 64])
def test_mixed_golden_matches_reference_engine(engine, ce, wl, golden_mixed, bits, lanes):
    # lanes 0: one lane per atom (the default); 2: two threads per sim from 3 atoms
    g = golden_mixed
    engine.set_tuning(lanes_per_sim=lanes)
    try:
        r = engine.run_mixed(g["n_per"], g["masses"], g["charges"], g["pos"], tight(ce, wl))
    finally:
        engine.set_tuning()
    assert (r.status == 0).all()
    err = per_sim_err(r, g[f"p_tight_f{bits}"], g["n_per"])
    assert err.max() <= TIGHT_MAX, err.max()


def test_mixed_matches_oracle_and_padding(engine, ce, wl):
    n_per, m, q, pos = wl.sample_mixed(3000, seed=31)
    r = engine.run_mixed(n_per, m, q, pos, tight(ce, wl))
    o = ol.run_batch_mixed(n_per, m, q, pos.astype(np.float32).astype(np.float64), bits=64, rtol=wl.TIGHT[0],
                           atol=wl.TIGHT[1], pe_stop=wl.TIGHT[2])
    assert (r.status == 0).all()
    assert per_sim_err(r, o["momenta"], n_per).max() <= TIGHT_MAX
    np.testing.assert_allclose(r.ker, o["ker"], rtol=1e-6)
    # rows past each sim's atom count are untouched (zero here)
    for n in range(2, 10):
        assert not r.momenta[n_per == n][:, n:].any()


def test_mixed_equals_fixed_molecule_path(engine, ce, wl):
    # A mixed batch of one molecule is bit-identical to the fixed-molecule
    # lane-per-atom path (same pair constants, same arithmetic).
    mol = wl.CH4
    S = 2000
    pos5 = wl.sample_molecule(mol, S, seed=32).astype(np.float32)
    n_per = np.full(S, 5, np.uint8)
    m = np.ones((S, 10))
    q = np.zeros((S, 10))
    m[:, :5] = mol.masses_me
    q[:, :5] = mol.charge_array
    pos = np.zeros((S, 10, 3), np.float32)
    pos[:, :5] = pos5
    rm = engine.run_mixed(n_per, m, q, pos, tight(ce, wl))
    engine.set_molecule(mol.masses_me, mol.charge_array)
    engine.set_tuning(lanes_per_sim=5)
    try:
        rf = engine.run(pos5, tight(ce, wl))
    finally:
        engine.set_tuning()
    np.testing.assert_array_equal(rm.momenta[:, :5], rf.momenta)
    np.testing.assert_array_equal(rm.steps, rf.steps)
    np.testing.assert_array_equal(rm.ker, rf.ker)


@pytest.mark.parametrize("molecule", ["CH4", "C2H6_LIKE"])
def test_mixed_pair_layout_equals_fixed_pair_path(engine, ce, wl, molecule):
    # With two threads per sim in both, a mixed batch of one molecule equals the
    # fixed-molecule path bit for bit (same pair constants, same arithmetic;
    # CH4's 5 atoms put a phantom in the second thread).
    mol = getattr(wl, molecule)
    S, n = 3000, mol.n
    posn = wl.sample_molecule(mol, S, seed=37).astype(np.float32)
    n_per = np.full(S, n, np.uint8)
    m = np.ones((S, 10))
    q = np.zeros((S, 10))
    m[:, :n] = mol.masses_me
    q[:, :n] = mol.charge_array
    pos = np.zeros((S, 10, 3), np.float32)
    pos[:, :n] = posn
    engine.set_tuning(lanes_per_sim=2)
    try:
        rm = engine.run_mixed(n_per, m, q, pos, tight(ce, wl, 0))
        engine.set_molecule(mol.masses_me, mol.charge_array)
        rf = engine.run(posn, tight(ce, wl, 0))
    finally:
        engine.set_tuning()
    assert (rm.status == 0).all()
    np.testing.assert_array_equal(rm.momenta[:, :n], rf.momenta)
    np.testing.assert_array_equal(rm.steps, rf.steps)
    np.testing.assert_array_equal(rm.ker, rf.ker)


def test_one_atom_and_invalid_counts(engine, ce, wl):
    n_per, m, q, pos = wl.sample_mixed(64, seed=33)
    n_per = n_per.copy()
    n_per[3] = 1
    n_per[5] = 0
    n_per[7] = 11
    r = engine.run_mixed(n_per, m, q, pos, tight(ce, wl))
    assert r.status[3] == ce.CE_SIM_OK and r.steps[3] == 0 and not r.momenta[3].any() and r.ker[3] == 0.0
    assert r.status[5] == ce.CE_SIM_BAD_INPUT and r.status[7] == ce.CE_SIM_BAD_INPUT
    ok = np.ones(64, bool)
    ok[[3, 5, 7]] = False
    assert (r.status[ok] == 0).all()


def _device_batch(torch, ce, n_per, m, q, pos):
    d = dict(n=torch.from_numpy(np.ascontiguousarray(n_per, np.uint8)).cuda(),
             m=torch.from_numpy(np.ascontiguousarray(m, np.float64)).cuda(),
             q=torch.from_numpy(np.ascontiguousarray(q, np.float64)).cuda(),
             x=torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda())
    b = ce.CeMixedBatch(d["n"].data_ptr(), d["m"].data_ptr(), d["q"].data_ptr(), d["x"].data_ptr())
    return d, b


def _device_out(torch, ce, S):
    d = dict(m=torch.zeros((S, 10, 3), dtype=torch.float32, device="cuda"),
             k=torch.zeros(S, dtype=torch.float64, device="cuda"),
             s=torch.zeros(S, dtype=torch.int32, device="cuda"),
             t=torch.zeros(S, dtype=torch.uint8, device="cuda"))
    o = ce.CeOutputs(d["m"].data_ptr(), d["k"].data_ptr(), d["s"].data_ptr(), d["t"].data_ptr(), None, None, None,
                     None)
    return d, o


def test_chunked_host_mixed_path_matches_device_path(engine, ce, wl):
    # ce_run_mixed cuts a batch of 2^18 sims or more into chunks over two device
    # slots with the copies on side streams (3 chunks here); every chunk's result
    # must equal one ce_run_mixed_device launch over the whole batch, bit for bit.
    torch = pytest.importorskip("torch")
    S = 3 * 131072 + 123
    n_per, m, q, pos = wl.sample_mixed(S, seed=51)
    cfg = tight(ce, wl)
    host = engine.run_mixed(n_per, m, q, pos, cfg)
    keep, batch = _device_batch(torch, ce, n_per, m, q, pos)
    d, o = _device_out(torch, ce, S)
    stream = torch.cuda.Stream()
    engine.run_mixed_device(S, batch, cfg, o, ce.CE_SCHEDULE_ONE_LAUNCH, stream.cuda_stream)
    stream.synchronize()
    assert (host.status == 0).all()
    np.testing.assert_array_equal(host.momenta, d["m"].cpu().numpy())
    np.testing.assert_array_equal(host.ker, d["k"].cpu().numpy())
    np.testing.assert_array_equal(host.steps, d["s"].cpu().numpy().astype(np.uint32))
    np.testing.assert_array_equal(host.status, d["t"].cpu().numpy())


def test_full_size_mixed_invariants(engine, ce, wl):
    # The benchmark's full mixed population (1e7 sims of 2..10 atoms from the
    # device sampler, one persistent launch, plain FP32), checked per sim on the
    # device: every sim converges, KER equals E_0 after redistribution, and the
    # momenta sum to zero (|sum p| / sum |p| < 1e-4, demo/sanity_check.py:102-106).
    torch = pytest.importorskip("torch")
    import importlib

    cl = importlib.import_module("coulomb_explosion_b200.closure")
    S = 10_000_000
    b = cl.sample_mixed_device(S, seed=20261203)
    cfg = tight(ce, wl, mode=0)
    mom = torch.zeros((S, 10, 3), dtype=torch.float32, device="cuda")
    ker = torch.zeros(S, dtype=torch.float64, device="cuda")
    steps = torch.zeros(S, dtype=torch.int32, device="cuda")
    status = torch.full((S,), 255, dtype=torch.uint8, device="cuda")
    e0 = torch.zeros(S, dtype=torch.float64, device="cuda")
    out = ce.CeOutputs(mom.data_ptr(), ker.data_ptr(), steps.data_ptr(), status.data_ptr(), None, None, None, None,
                       None, e0.data_ptr())
    engine.reserve_mixed(S)
    stream = torch.cuda.Stream()
    engine.run_mixed_device(S, b.c(), cfg, out, ce.CE_SCHEDULE_ONE_LAUNCH, stream.cuda_stream)
    stream.synchronize()
    assert bool((status == ce.CE_SIM_OK).all())
    assert float((ker / e0 - 1.0).abs().max()) < 1e-9
    tot = mom.double().sum(dim=1).norm(dim=1)
    size = mom.double().norm(dim=2).sum(dim=1)
    assert float((tot / size).max()) < 1e-4
    assert 30.0 < float(steps.double().mean()) < 70.0


@pytest.mark.parametrize("lanes", [0, 2])
def test_schedules_and_graph_replay_are_bit_identical(engine, ce, wl, lanes):
    # lanes 2 (two threads per sim from 3 atoms) runs the one-launch request as
    # the per-size schedule
    torch = pytest.importorskip("torch")
    engine.set_tuning(lanes_per_sim=lanes)
    try:
        _schedules_and_graph_replay(engine, ce, wl, torch)
    finally:
        engine.set_tuning()


def _schedules_and_graph_replay(engine, ce, wl, torch):
    S = 5000
    n_per, m, q, pos = wl.sample_mixed(S, seed=34)
    keep, batch = _device_batch(torch, ce, n_per, m, q, pos)
    cfg = tight(ce, wl)
    stream = torch.cuda.Stream()
    outs = []
    for sched in (ce.CE_SCHEDULE_ONE_LAUNCH, ce.CE_SCHEDULE_PER_SIZE, ce.CE_SCHEDULE_OVERLAP):
        d, o = _device_out(torch, ce, S)
        engine.run_mixed_device(S, batch, cfg, o, sched, stream.cuda_stream)
        stream.synchronize()
        outs.append({k: v.cpu().numpy() for k, v in d.items()})
    for other in outs[1:]:
        for k in outs[0]:
            np.testing.assert_array_equal(outs[0][k], other[k])
    # the overlapped per-size schedule (two streams, fork / join) captured and replayed
    engine.reserve_mixed(S)
    d, o = _device_out(torch, ce, S)
    engine.graph_begin(stream.cuda_stream)
    engine.run_mixed_device(S, batch, cfg, o, ce.CE_SCHEDULE_OVERLAP, stream.cuda_stream)
    g = engine.graph_end(stream.cuda_stream)
    try:
        d["m"].zero_()
        torch.cuda.synchronize()
        g.launch(stream.cuda_stream)
        stream.synchronize()
        np.testing.assert_array_equal(d["m"].cpu().numpy(), outs[0]["m"])
    finally:
        g.close()
    # capture the one-launch call into a graph and replay it twice
    engine.reserve_mixed(S)
    d, o = _device_out(torch, ce, S)
    engine.graph_begin(stream.cuda_stream)
    engine.run_mixed_device(S, batch, cfg, o, ce.CE_SCHEDULE_ONE_LAUNCH, stream.cuda_stream)
    g = engine.graph_end(stream.cuda_stream)
    try:
        for _ in range(2):
            d["m"].zero_()
            torch.cuda.synchronize()
            g.launch(stream.cuda_stream)
            stream.synchronize()
            np.testing.assert_array_equal(d["m"].cpu().numpy(), outs[0]["m"])
            np.testing.assert_array_equal(d["s"].cpu().numpy(), outs[0]["s"])
    finally:
        g.close()


def test_autotuner_picks_a_measured_candidate_and_keeps_results(ce, wl):
    torch = pytest.importorskip("torch")
    engine = ce.Engine(0)  # its own engine: tuned entries stay out of the shared one
    S = 20000
    n_per, m, q, pos = wl.sample_mixed(S, seed=35)
    keep, batch = _device_batch(torch, ce, n_per, m, q, pos)
    cfg = tight(ce, wl)
    stream = torch.cuda.Stream()
    report, best = engine.autotune_mixed(S, batch, cfg)
    # one lane per atom: 3 schedules x 3 block sizes x 4 refill thresholds (0 =
    # each size's default); two threads per sim: the 2 per-size schedules x 4
    assert len(report) == 44 and all(r["sims_per_s"] > 0 for r in report)
    assert {r["lanes_per_sim"] for r in report} == {0, 2}
    assert best in (ce.CE_SCHEDULE_ONE_LAUNCH, ce.CE_SCHEDULE_PER_SIZE, ce.CE_SCHEDULE_OVERLAP)
    d1, o1 = _device_out(torch, ce, S)
    engine.run_mixed_device(S, batch, cfg, o1, best, stream.cuda_stream)
    stream.synchronize()
    # the picked layout's results: bit for bit what that layout gives with any
    # launch shape and schedule (both layouts' parity: the golden tests above)
    best_r = max(report, key=lambda r: r["sims_per_s"])
    engine.set_tuning(lanes_per_sim=best_r["lanes_per_sim"])
    try:
        d2, o2 = _device_out(torch, ce, S)
        engine.run_mixed_device(S, batch, cfg, o2, ce.CE_SCHEDULE_PER_SIZE, stream.cuda_stream)
        stream.synchronize()
    finally:
        engine.set_tuning()
    np.testing.assert_array_equal(d1["m"].cpu().numpy(), d2["m"].cpu().numpy())
    # fixed path
    mol = wl.CH4
    engine.set_molecule(mol.masses_me, mol.charge_array)
    x = torch.from_numpy(wl.sample_molecule(mol, S, seed=36).astype(np.float32)).cuda()
    rep = engine.autotune_fixed(S, x.data_ptr(), cfg)
    # thread per sim and two threads per sim (128 threads each) and lane per atom
    # (3 block sizes), x 5 refill thresholds
    assert len(rep) == 25 and {r["lanes_per_sim"] for r in rep} == {1, 2, 5}
    t = engine.get_tuning()
    best_f = max(rep, key=lambda r: r["sims_per_s"])
    # get_tuning reports the resolved shape: refill 0 is CH4's per-layout default
    default_refill = {1: 4, 2: 2, 5: 1}[best_f["lanes_per_sim"]]
    assert (t["block_threads"], t["refill_threshold"], t["lanes_per_sim"]) == (
        best_f["block_threads"], best_f["refill_threshold"] or default_refill, best_f["lanes_per_sim"])


def _state(torch, ce, S):
    d = dict(x=torch.zeros((S, 10, 3), dtype=torch.float32, device="cuda"),
             v=torch.zeros((S, 10, 3), dtype=torch.float32, device="cuda"),
             h=torch.zeros(S, dtype=torch.float32, device="cuda"),
             t=torch.zeros(S, dtype=torch.float64, device="cuda"),
             s=torch.zeros(S, dtype=torch.int32, device="cuda"),
             r=torch.zeros(S, dtype=torch.int32, device="cuda"),
             e=torch.zeros(S, dtype=torch.float64, device="cuda"),
             c=torch.zeros((S, 10, 6), dtype=torch.float32, device="cuda"))
    st = ce.CeSimState(*(d[k].data_ptr() for k in ("x", "v", "h", "t", "s", "r", "e", "c")))
    return d, st


@pytest.mark.parametrize("lanes", [0, 2])
@pytest.mark.parametrize("schedule", ["one", "per_size", "overlap"])
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_saved_state_resumes_bit_for_bit(engine, ce, wl, mode, schedule, lanes):
    """A run to a loose stop that saves each sim's integrator state, then a run
    that continues from it, equals one uninterrupted run bit for bit (momenta,
    KER, steps, rejects, status); sims whose saved step is 0 restart from rest
    and equal it too. The closure continues the sims its gate sends back this way.
    lanes 2: two threads per sim from 3 atoms (the one-launch request runs per size)."""
    torch = pytest.importorskip("torch")
    engine.set_tuning(lanes_per_sim=lanes)
    try:
        _saved_state_resumes(engine, ce, wl, torch, mode, schedule)
    finally:
        engine.set_tuning()


def _saved_state_resumes(engine, ce, wl, torch, mode, schedule):
    sch = {"one": ce.CE_SCHEDULE_ONE_LAUNCH, "per_size": ce.CE_SCHEDULE_PER_SIZE,
           "overlap": ce.CE_SCHEDULE_OVERLAP}[schedule]
    S = 6000
    n_per, m, q, pos = wl.sample_mixed(S, seed=61)
    keep, batch = _device_batch(torch, ce, n_per, m, q, pos)
    cfg = tight(ce, wl, mode)
    loose = tight(ce, wl, mode, redistribute_energy=False)
    loose.pe_stop_fraction = 0.01

    def outputs():
        d, o = _device_out(torch, ce, S)
        d["r"] = torch.zeros(S, dtype=torch.int32, device="cuda")
        d["tf"] = torch.zeros(S, dtype=torch.float64, device="cuda")
        o.rejects, o.t_final = d["r"].data_ptr(), d["tf"].data_ptr()
        return d, o

    dp, op = outputs()
    engine.run_mixed_device(S, batch, cfg, op, sch)
    dl, ol_ = outputs()
    ds, st = _state(torch, ce, S)
    engine.run_mixed_device_state(S, batch, loose, ol_, save=st, schedule=sch)
    torch.cuda.synchronize()
    assert (dl["t"].cpu().numpy() == 0).all()
    h = ds["h"].cpu().numpy()
    assert (h > 0).all() and (ds["s"].cpu().numpy() > 0).all()
    ds["h"][::7] = 0.0  # these restart from rest
    dr, orr = outputs()
    engine.run_mixed_device_state(S, batch, cfg, orr, resume=st, schedule=sch)
    torch.cuda.synchronize()
    for k in ("m", "k", "s", "t", "r", "tf"):
        np.testing.assert_array_equal(dr[k].cpu().numpy(), dp[k].cpu().numpy(), err_msg=k)
    assert (dp["t"].cpu().numpy() == 0).all()
