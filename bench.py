#!/usr/bin/env python3
"""Benchmark: explosions/s of the B200 engine on the CH4 workload.

Workload (one "step"): integrate S = 1e6 independent CH4 Coulomb explosions
(C + 4 H, all q = +1, positions uniform in a 3.3-bohr ball, pairs >= 0.5 bohr,
at rest) to their asymptotic momenta with adaptive DP5(4) at rtol 1e-6,
atol 1e-7, pe_stop 1e-7 -- the operating point at which every sim is within
1e-5 relative momentum error of FP64 (checked live on a subset below).

  value   explosions/s with inputs resident in HBM, device-timed with CUDA
          events on the launch stream (max over ranks), L2 flushed between steps
  e2e     the same through the C ABI host-buffer call (ce_run): pinned host
          positions in, momenta / KER / steps / status out, every step
  roofline  FP32 CUDA-core bound of the integration kernel (the pair force is
          not a dense contraction): algorithmic FLOPs (flops_per_sim) per
          launch over the event-timed launch, against a measured FP32 FMA peak
  cpu_baseline  the reference's SIMD batched engine BatchedRK45<float> (its
          unmodified header compiled against the project's Highway-API shim,
          oracle/_ref) on every host core, one pinned process per core over
          disjoint slices of the same 1e6 sims; and on one pinned core, median
          of 7 passes (the denominator of the single-core speed-up); the
          reference scalar f32 engine on one core as a secondary figure
  accuracy  a 500-sim subset against the reference's f32 engines (scalar and
          batched), the FP64 reference (scalar f64 engine at rtol 1e-12 /
          atol 1e-20 / pe_stop 1e-13) and the FP64 scipy oracle (solve_ivp to
          t = 1e10, the reference's Python ground truth)

`--impl reference` runs only the reference CPU engine (BatchedRK45<float>, all
host cores) on the same workload.
Multi-GPU: each rank integrates its own S sims (weak scaling, no collective on
the data path); timing is max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "explosions/s on 1 B200 at <=1e-5 rel momentum err vs FP64; closure vs plain RK45"
UNIT = "explosions/s"
S_DEFAULT = 1_000_000
SEED = 20261203
TIGHT = (1e-6, 1e-7, 1e-7)


def flops_per_sim(steps: np.ndarray, n: int) -> np.ndarray:
    """Algorithmic FP32 FLOPs per sim: steps * (137 P + 438 N) + C_init with
    C_init = 2 (21 P + 3 N) + 11 P + 60 N, P = N (N - 1) / 2 pairs. Counting:
    add, sub and mul 1, FMA 2, rsqrt, div and sqrt 1, abs and max 0; zero
    Butcher coefficients skipped; each pair counted once. Per accepted step: 6
    force evaluations of 21 P + 3 N (pair: 3 sub + 5 for r^2 + 3 for r^-3 + 1
    scale + 3 force + 6 accumulate), the potential 11 P, stage combinations
    52 * 6N, error norm 18 * 6N. C_init: k1, the initial-step probe and PE_0."""
    p = n * (n - 1) // 2
    return steps.astype(np.float64) * (137 * p + 438 * n) + (2 * (21 * p + 3 * n) + 11 * p + 60 * n)


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed region
    (NVML, read only; nvidia-smi as the fallback)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        # NVML read-only queries every 10 ms (a timed region can be ~0.1 s);
        # nvidia-smi every 0.2 s where NVML is not available.
        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            bits = [pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap]
        except Exception:
            h = None
        while not self._stop.is_set():
            try:
                if h is not None:
                    sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
                    pw = pynvml.nvmlDeviceGetPowerUsage(h) / 1000.0
                    rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.rows.append([str(self.index), str(sm), str(mx), f"{pw:.1f}", hex(rs)] +
                                     ["Active" if rs & b else "Not Active" for b in bits])
                else:
                    out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.rows.append([c.strip() for c in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.01 if h is not None else 0.2)
        if h is not None:
            try:
                pynvml.nvmlShutdown()
            except Exception:
                pass

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _oracle_lib():
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as ol  # the checker and the CPU baseline only

    return ol


def _scipy_oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import scipy_oracle as so  # the checker only

    return so


def cpu_batched_baseline(pos64, mol, point, *, all_steps=3, single_reps=7, single_sample=65536,
                         scalar_sample=8192):
    """The reference's CPU engines on this host, on the step's own inputs.

    all cores: BatchedRK45<float> (K lanes per batch as the host ISA gives),
    one pinned process per usable core over disjoint contiguous slices of all
    of pos64; median of `all_steps` passes. single core: one pinned process,
    median of `single_reps` passes over the first `single_sample` sims.
    Secondary: the reference scalar f32 engine on one pinned core."""
    ol = _oracle_lib()
    if not ol.batched_available():
        return None
    rtol, atol, pes = point
    kw = dict(bits=32, rtol=rtol, atol=atol, pe_stop=pes)
    cores = ol.usable_cores()
    with ol.CorePool(pos64, mol.masses_me, mol.charge_array, cores, engine="batched", **kw) as pool:
        walls = [pool.step()[0] for _ in range(all_steps)]
    all_rate = len(pos64) / float(np.median(walls))
    one, one_secs = ol.single_core_rate(pos64[:single_sample], mol.masses_me, mol.charge_array,
                                        reps=single_reps, engine="batched", **kw)
    sc, _ = ol.single_core_rate(pos64[:scalar_sample], mol.masses_me, mol.charge_array, reps=3,
                                engine="scalar", **kw)
    k = ol.ref_batched().refb_lanes(32)
    return {
        "value": all_rate, "unit": UNIT, "cores": len(cores), "kind": "reference",
        "engine": f"BatchedRK45<float> (reference SIMD lockstep engine, K={k} lanes, {ol.host_isa()}, "
                  "unmodified header + project Highway-API shim, -O2)",
        "sample": f"all {len(pos64)} sims of the step, one pinned process per core on disjoint slices, "
                  f"median of {all_steps} passes",
        "single_core_value": one,
        "single_core_sample": f"{single_sample} sims, 1 pinned core, median of {single_reps} passes",
        "single_core_secs": one_secs,
        "scalar_f32_single_core_value": sc,
        "host_cpu": _host_cpu(),
    }


def _host_cpu():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def accuracy_leg(pos64, p_gpu, mol, point, *, scipy_processes=None):
    """Per-sim config-norm errors of the GPU momenta on a subset of the step:
    against the reference f32 engines (scalar run_to_convergence and the SIMD
    BatchedRK45<float>) at the same tolerance point, the FP64 reference (the
    reference scalar f64 engine at rtol 1e-12 / atol 1e-20 / pe_stop 1e-13) and
    the FP64 scipy oracle (solve_ivp RK45 to t = 1e10 at rtol 1e-8 / atol 1e-16)."""
    ol = _oracle_lib()
    so = _scipy_oracle()
    rtol, atol, pes = point
    m, q = mol.masses_me, mol.charge_array

    def dist(e):
        return {"median": float(np.median(e)), "p99": float(np.percentile(e, 99)), "max": float(e.max())}

    out = {"subset": int(len(pos64))}
    f64 = ol.ref_run_batch(pos64, m, q, bits=64, rtol=1e-12, atol=1e-20, pe_stop=1e-13)
    out["vs_fp64_reference"] = dist(ol.config_norm_error(p_gpu, f64["momenta"]))
    sci = so.run_many(pos64, m, q, processes=scipy_processes)
    out["vs_fp64_scipy"] = dist(ol.config_norm_error(p_gpu, sci))
    out["fp64_reference_vs_scipy"] = dist(ol.config_norm_error(f64["momenta"], sci))
    f32 = ol.ref_run_batch(pos64, m, q, bits=32, rtol=rtol, atol=atol, pe_stop=pes)
    out["vs_reference_f32_scalar"] = dist(ol.config_norm_error(p_gpu, f32["momenta"]))
    if ol.batched_available():
        b32 = ol.batched_run(pos64, m, q, bits=32, rtol=rtol, atol=atol, pe_stop=pes, threads=8)
        out["vs_reference_f32_batched"] = dist(ol.config_norm_error(p_gpu, b32["momenta"]))
        out["reference_f32_batched_vs_fp64"] = dist(ol.config_norm_error(b32["momenta"], f64["momenta"]))
    out["reference_f32_scalar_vs_fp64"] = dist(ol.config_norm_error(f32["momenta"], f64["momenta"]))
    out["fp64_reference"] = "reference scalar f64 engine, rtol 1e-12, atol 1e-20, pe_stop 1e-13"
    out["fp64_scipy"] = "solve_ivp RK45 to t = 1e10, rtol 1e-8, atol 1e-16 (the reference's Python oracle, restated)"
    return out


def run_reference_arm(args):
    """The reference's own CPU engine on this workload: BatchedRK45<float> over
    the full step (S sims, the same Philox geometries as the GPU arm), one pinned
    process per host core on disjoint slices, `--warmup` untimed then `--steps`
    timed passes; plus the single-core rate (one pinned core, median of 7)."""
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return 0
    ol = _oracle_lib()
    from __graft_entry__ import load_package

    load_package()
    import importlib

    wl = importlib.import_module("coulomb_explosion_b200.workloads")
    sp = importlib.import_module("coulomb_explosion_b200.sampling")
    if not ol.batched_available():
        why = ("reference batched engine not built (oracle/_ref)" if ol.host_isa()
               else "host CPU has neither AVX2+FMA nor AVX-512")
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return 0
    mol = wl.CH4
    S = args.sims
    pos32, _, flags = sp.sample_ball_host(mol, S, seed=SEED)
    assert not flags.any()
    pos = pos32.astype(np.float64)
    rtol, atol, pes = TIGHT
    cores = ol.usable_cores()
    kw = dict(bits=32, rtol=rtol, atol=atol, pe_stop=pes)
    with ol.CorePool(pos, mol.masses_me, mol.charge_array, cores, engine="batched", **kw) as pool:
        for _ in range(args.warmup):
            pool.step()
        times = [pool.step()[0] for _ in range(args.steps)]
    one, one_secs = ol.single_core_rate(pos[:65536], mol.masses_me, mol.charge_array, reps=7, engine="batched",
                                        **kw)
    total = sum(times)
    value = S * len(times) / total
    k = ol.ref_batched().refb_lanes(32)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"CH4 (C+4H, q=+1, r 3.3, min pair 0.5) Coulomb explosions, {S} sims per step",
                   "sims_per_step": S, "atoms": 5, "rtol": rtol, "atol": atol, "pe_stop": pes,
                   "inputs": f"Philox4x32-10 uniform-ball geometries (seed {SEED}), the GPU arm's, generated "
                             "before timing"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": len(cores), "kind": "reference",
                         "engine": f"BatchedRK45<float> (reference SIMD lockstep engine, K={k}, {ol.host_isa()}, "
                                   "unmodified header + project Highway-API shim, -O2)",
                         "sample": f"the full {S}-sim step, one pinned process per core on disjoint slices",
                         "single_core_value": one,
                         "single_core_sample": "65536 sims, 1 pinned core, median of 7 passes",
                         "host_cpu": _host_cpu()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_mixed(args):
    """Mixed workload: a population of 2..10-atom molecules (species
    H/C/N/O/S, charges +1..+3, ball radius 2.0 N^(1/3), pairs >= 0.5), generated
    on the device, integrated by one persistent launch (captured in a CUDA graph)
    and, for comparison, by the per-size launch schedule."""
    import ctypes
    import importlib

    import torch

    from __graft_entry__ import load_package

    ce = load_package()
    wl = importlib.import_module("coulomb_explosion_b200.workloads")
    sp = importlib.import_module("coulomb_explosion_b200.sampling")
    lib = ce.load_library()
    S = args.sims if args.sims != S_DEFAULT else 10_000_000
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rtol, atol, pes = TIGHT
    cfg = ce.RunConfig(rtol=rtol, atol=atol, pe_stop_fraction=pes, precision_mode=args.mode)

    n_d = torch.empty(S, dtype=torch.uint8, device=dev)
    m_d = torch.empty((S, 10), dtype=torch.float64, device=dev)
    q_d = torch.empty((S, 10), dtype=torch.float64, device=dev)
    x_d = torch.empty((S, 10, 3), dtype=torch.float32, device=dev)
    f_d = torch.empty(S, dtype=torch.uint8, device=dev)
    scfg = sp.mixed_config(SEED)
    rc = lib.ce_sample_mixed_device(0, S, ctypes.byref(scfg), ctypes.c_void_p(n_d.data_ptr()),
                                    ctypes.c_void_p(m_d.data_ptr()), ctypes.c_void_p(q_d.data_ptr()),
                                    ctypes.c_void_p(x_d.data_ptr()), ctypes.c_void_p(f_d.data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(f_d.sum().item()) == 0
    batch = ce.CeMixedBatch(n_d.data_ptr(), m_d.data_ptr(), q_d.data_ptr(), x_d.data_ptr())
    mom = torch.empty((S, 10, 3), dtype=torch.float32, device=dev)
    ker = torch.empty(S, dtype=torch.float64, device=dev)
    steps = torch.empty(S, dtype=torch.int32, device=dev)
    status = torch.empty(S, dtype=torch.uint8, device=dev)
    out = ce.CeOutputs(mom.data_ptr(), ker.data_ptr(), steps.data_ptr(), status.data_ptr(), None, None, None, None)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    eng = ce.Engine(0)
    t0 = time.perf_counter()
    report, best = ([], 0) if args.no_autotune else eng.autotune_mixed(min(S, 1_000_000), batch, cfg)
    tune_s = time.perf_counter() - t0
    eng.reserve_mixed(S)
    stream = torch.cuda.Stream(device=dev)
    names = {ce.CE_SCHEDULE_ONE_LAUNCH: "one_launch", ce.CE_SCHEDULE_PER_SIZE: "per_size",
             ce.CE_SCHEDULE_OVERLAP: "overlap"}
    graphs, launches = {}, {}
    for sch in names:  # every schedule captured once into a CUDA graph
        eng.graph_begin(stream.cuda_stream)
        eng.run_mixed_device(S, batch, cfg, out, sch, stream.cuda_stream)
        launches[sch] = eng.last_launch_count()
        graphs[sch] = eng.graph_end(stream.cuda_stream)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
                ev[i][0].record(stream)
            fn()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev)

    ms = {}
    with ClockSampler(0) as clk:
        for sch in names:
            ms[sch] = timed(lambda: graphs[sch].launch(stream.cuda_stream))
            if sch == ce.CE_SCHEDULE_ONE_LAUNCH:
                st_np = status.cpu().numpy()
                steps_np = steps.cpu().numpy().astype(np.uint32)
                mom_one = mom.cpu().numpy()
            else:
                assert np.array_equal(mom.cpu().numpy(), mom_one), names[sch]
    for g_ in graphs.values():
        g_.close()
    # headline: the schedule the autotuner picked (the overlapped one when untuned)
    head = best if report else ce.CE_SCHEDULE_OVERLAP
    ms_one = ms[head]
    launches_per_step = launches[head]
    value = S * args.steps / (ms_one / 1e3)

    n_np = n_d.cpu().numpy()
    p = n_np.astype(np.int64) * (n_np.astype(np.int64) - 1) // 2
    nn = n_np.astype(np.int64)
    fl = float((steps_np * (137 * p + 438 * nn) + 2 * (21 * p + 3 * nn) + 11 * p + 60 * nn).sum())
    achieved = fl / (ms_one / args.steps / 1e3) / 1e12
    peak = measure_fp32_peak(torch, dev)

    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as ol

    sub = np.arange(0, S, max(1, S // 400))[:400]
    nn_s = np.zeros(len(sub), np.uint8)
    mm_s = np.zeros((len(sub), 10))
    qq_s = np.zeros((len(sub), 10))
    xx_s = np.zeros((len(sub), 10, 3))
    for k, i in enumerate(sub):
        a, b, c, _, x64, _ = sp.sample_mixed_host(1, SEED, first_sim=int(i))
        nn_s[k], mm_s[k], qq_s[k] = a[0], b[0], c[0]
        xx_s[k] = x64[0].astype(np.float32)
    ref = ol.run_batch_mixed(nn_s, mm_s, qq_s, xx_s, bits=64, rtol=1e-10, atol=1e-16, pe_stop=1e-11)
    err = np.array([ol.config_norm_error(mom_one[i:i + 1, :k], ref["momenta"][j:j + 1, :k])[0]
                    for j, (i, k) in enumerate(zip(sub, nn_s))])
    line = {
        "metric": METRIC + " [mixed 2..10-atom population, 1e7 sims, CUDA-graph replay]", "value": value, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_one / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"mixed population, {S} sims per step, N ~ U{{2..10}}, species U{{H,C,N,O,S}}, "
                               "q ~ U{+1,+2,+3}, radius 2.0 N^(1/3), min pair 0.5 (Philox, generated on device)",
                   "rtol": rtol, "atol": atol, "pe_stop": pes, "precision_mode": args.mode,
                   "schedule": f"{names[head]} (autotuner's pick), replayed as a CUDA graph",
                   "launches_per_step": launches_per_step,
                   "l2": "flushed between timed steps (256 MiB write, outside the events)"},
        "schedules": {names[k]: {"value": S * args.steps / (v / 1e3), "ms_per_step": v / args.steps,
                                 "launches": launches[k]} for k, v in ms.items()},
        "schedules_identical_results": True,
        "autotune": ({"seconds": tune_s, "best_schedule": names[best],
                      "best": max(report, key=lambda r: r["sims_per_s"]), "candidates": len(report)}
                     if report else "off (engine defaults)"),
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak["tflops"], "unit": "TFLOP/s",
                     "frac": achieved / peak["tflops"], "peak_source": peak["source"]},
        "accuracy": {"vs": "fp64 oracle (rtol 1e-10, pe_stop 1e-11)", "subset": int(len(sub)),
                     "max_rel_err": float(err.max()), "median_rel_err": float(np.median(err)),
                     "status_ok_frac": float((st_np == 0).mean())},
        "clocks": clk.summary(),
    }
    print(json.dumps(line))
    eng.close()
    return 0


def run_precision(args):
    """Precision study: CH4 and stiff H2O (O q=+3, 2 H q=+1, 2.0-bohr ball, pairs
    >= 0.3), 1e6 sims each, every precision mode at the production and tight
    points. Errors against the FP64 reference (oracle f64 at rtol 1e-12 /
    atol 1e-20 / pe_stop 1e-13) on a 1e4 subset: per-atom |dp_i| / |p_i| and the
    per-sim config norm; the config norm against the FP64 scipy oracle (the
    reference's simulate_explosion, restated) on the same subset; energy drift
    |KE + PE_final - E0| / E0 before redistribution; accepted steps per sim."""
    import importlib

    import torch

    from __graft_entry__ import load_package

    ce = load_package()
    wl = importlib.import_module("coulomb_explosion_b200.workloads")
    sp = importlib.import_module("coulomb_explosion_b200.sampling")
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as ol

    so = _scipy_oracle()
    S = args.sims
    n_sub = min(10_000, S)
    eng = ce.Engine(0)
    rows = []
    scipy_check = {}
    for name, mol in (("CH4", wl.CH4), ("H2O-stiff", wl.H2O_STIFF)):
        pos, pos64, flags = sp.sample_ball_host(mol, S, seed=SEED)
        assert not flags.any()
        sub = np.linspace(0, S - 1, n_sub).astype(np.int64)
        ref = ol.run_batch(pos[sub].astype(np.float64), mol.masses_me, mol.charge_array, bits=64, rtol=1e-12,
                           atol=1e-20, pe_stop=1e-13)
        pe0 = np.array([ol.potential(x, mol.charge_array) for x in pos[sub].astype(np.float64)])
        t_sci = time.perf_counter()
        sci = so.run_many(pos[sub].astype(np.float64), mol.masses_me, mol.charge_array)
        e_rs = ol.config_norm_error(ref["momenta"], sci)
        scipy_check[name] = {"fp64_reference_vs_scipy": {"median": float(np.median(e_rs)), "max": float(e_rs.max())},
                             "scipy_seconds": time.perf_counter() - t_sci}
        eng.set_molecule(mol.masses_me, mol.charge_array)
        x_d = torch.from_numpy(pos).cuda()
        for point_name, (rtol, atol, pes) in (("production", wl.PRODUCTION), ("tight", wl.TIGHT)):
            for mode in (0, 1, 2, 3):
                cfg = ce.RunConfig(rtol=rtol, atol=atol, pe_stop_fraction=pes, precision_mode=mode)
                mom = torch.empty((S, mol.n, 3), dtype=torch.float32, device="cuda")
                ker = torch.empty(S, dtype=torch.float64, device="cuda")
                stp = torch.empty(S, dtype=torch.int32, device="cuda")
                sts = torch.empty(S, dtype=torch.uint8, device="cuda")
                pef = torch.empty(S, dtype=torch.float64, device="cuda")
                keb = torch.empty(S, dtype=torch.float64, device="cuda")
                out = ce.CeOutputs(mom.data_ptr(), ker.data_ptr(), stp.data_ptr(), sts.data_ptr(), None, None,
                                   pef.data_ptr(), keb.data_ptr())
                stream = torch.cuda.current_stream().cuda_stream
                eng.run_device(S, x_d.data_ptr(), cfg, out, stream)  # warm-up
                torch.cuda.synchronize()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                eng.run_device(S, x_d.data_ptr(), cfg, out, stream)
                b.record()
                torch.cuda.synchronize()
                ms = a.elapsed_time(b)
                p = mom.cpu().numpy()[sub].astype(np.float64)
                atom_err = np.linalg.norm(p - ref["momenta"], axis=2) / np.linalg.norm(ref["momenta"], axis=2)
                cn = ol.config_norm_error(p, ref["momenta"])
                cs_ = ol.config_norm_error(p, sci)
                drift = np.abs(keb.cpu().numpy()[sub] + pef.cpu().numpy()[sub] - pe0) / pe0
                rows.append({
                    "molecule": name, "point": point_name, "rtol": rtol, "atol": atol, "pe_stop": pes,
                    "mode": {0: "fp32", 1: "fp32+kahan", 2: "fp32+fp64 t/E", 3: "fp32+kahan+fp64 t/E"}[mode],
                    "explosions_per_s": S / (ms / 1e3),
                    "atom_rel_err": {"median": float(np.median(atom_err)), "p99": float(np.percentile(atom_err, 99)),
                                     "max": float(atom_err.max())},
                    "config_rel_err": {"median": float(np.median(cn)), "p99": float(np.percentile(cn, 99)),
                                       "max": float(cn.max())},
                    "config_rel_err_vs_scipy": {"median": float(np.median(cs_)), "p99": float(np.percentile(cs_, 99)),
                                                "max": float(cs_.max())},
                    "energy_drift": {"median": float(np.median(drift)), "max": float(drift.max())},
                    "mean_steps": float(stp.cpu().numpy().mean()),
                    "status_ok_frac": float((sts.cpu().numpy() == 0).mean()),
                })
    eng.close()
    print(json.dumps({"metric": "precision study (CH4 and stiff H2O, every precision mode)", "sims_per_case": S, "fp64_subset": n_sub,
                      "fp64_reference": "oracle f64, rtol 1e-12, atol 1e-20, pe_stop 1e-13",
                      "fp64_scipy": "solve_ivp RK45 to t = 1e10, rtol 1e-8, atol 1e-16 (the reference's Python oracle, "
                                    "restated), same subset", "scipy_check": scipy_check, "rows": rows}))
    return 0


def run_closure(args):
    """Closure study: the learned closure on the mixed 2..10-atom population.

    Training pairs: `--train-sims` sims (default 5e6) integrated to the loose
    stop (PE <= 5% PE_0, no rescale) and, for targets, to convergence by plain
    RK45 at the tight point; a seeded 2% of them is held out for validation and
    gate calibration. The network is trained by the library's tensor-core
    kernels (Adam, cosine schedule). Serving: `--sims` (default 1e7) further
    sims from a disjoint Philox counter range, closure (ce_closure_serve) and
    plain RK45 (ce_run_mixed_device) timed back to back with CUDA events, L2
    flushed between steps. Errors: per-sim config norm against plain RK45 on
    every sim and against the FP64 oracle on a subset."""
    import importlib

    import torch

    from __graft_entry__ import load_package

    ce = load_package()
    cl = importlib.import_module("coulomb_explosion_b200.closure")
    sp = importlib.import_module("coulomb_explosion_b200.sampling")
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as ol

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rtol, atol, pes = TIGHT
    cfg = ce.RunConfig(rtol=rtol, atol=atol, pe_stop_fraction=pes, precision_mode=args.mode)
    S_train = args.train_sims
    S = args.sims if args.sims != S_DEFAULT else 10_000_000
    mb = args.minibatch
    eng = ce.Engine(0)
    seed = SEED + 4

    # ---- training pairs
    t0 = time.perf_counter()
    tb = cl.sample_mixed_device(S_train, seed=seed)
    ts, loose_t, base_t, plain_t = cl.make_training_set(eng, tb, cfg, loose_pe_stop=args.loose_pe_stop,
                                                         minibatch=mb)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    perm = torch.randperm(S_train, generator=g, device=dev)
    n_val = max(mb, int(S_train * args.val_frac))
    val_rows, train_rows = perm[:n_val], perm[n_val:]
    train_rows = train_rows[ts.valid[train_rows]]

    # ---- training
    net = cl.Network(max_batch=65536, seed=seed)
    rep = cl.train(net, ts, epochs=args.epochs, minibatch=mb, lr=args.lr, lr_final=args.lr * 1e-2, seed=seed,
                   train_rows=train_rows)
    net.scale_output_layer(1.0 / cl.TARGET_SCALE)
    losses = np.array(rep.losses)

    # ---- validation: errors of the three closures and gate calibration
    out_t = cl.net_forward(net, ts.feats)
    stats = cl.gate_stats(tb, loose_t, base_t, out_t)
    vmask = torch.zeros(S_train, dtype=torch.bool, device=dev)
    vmask[val_rows] = True
    vmask &= ts.valid
    p_net = cl.predict(tb, base_t, out_t)
    if args.gate_target_err:
        gate = cl.calibrate_gate_for_error(stats, cl.rel_err(p_net, plain_t["momenta"]), vmask, args.gate_target_err,
                                           quantile=args.gate_quantile)
    else:
        gate = cl.calibrate_gate(stats, vmask, quantile=args.gate_quantile)
    p_ana = base_t["p_base"]
    pl = loose_t["momenta"].double()
    live = (torch.arange(10, device=dev)[None, :] < tb.n[:, None].long()).double()
    m_ = torch.where(live > 0, tb.mass, torch.ones_like(tb.mass))
    ke = 0.5 * ((pl * pl).sum(-1) / m_ * live).sum(-1)
    p_red = pl * torch.sqrt(loose_t["e0"] / ke)[:, None, None]

    def dist(e):
        e = e.float()
        return {"median": float(e.median()), "p99": float(torch.quantile(e[: 1 << 24], 0.99)),
                "max": float(e.max())}

    ref_v = plain_t["momenta"][vmask]
    val = {"sims": int(vmask.sum()), "network": dist(cl.rel_err(p_net[vmask], ref_v)),
           "analytic_only": dist(cl.rel_err(p_ana[vmask], ref_v)),
           "redistribution_only": dist(cl.rel_err(p_red[vmask], ref_v))}
    keep = {k: stats[k][vmask] for k in stats}
    passed = (keep["rho"] <= gate.tol_energy) & (keep["mu"] <= gate.tol_momentum) & (keep["corr"] <= gate.tol_correction)
    val["gate_pass_frac"] = float(passed.float().mean())
    del ts, loose_t, base_t, plain_t, out_t, stats, p_net, p_ana, p_red, pl, tb
    torch.cuda.empty_cache()

    # ---- serving: held-out sims, closure vs plain
    sb = cl.sample_mixed_device(S, seed=seed, first_sim=S_train)
    eng.reserve_mixed(S)
    # launch shape and schedule picked by the autotuner; plain RK45 and the
    # closure's two integration passes all run with them
    _, sched = eng.autotune_mixed(min(S, 1_000_000), sb.c(), cfg)
    eng.reserve_mixed(S)
    clo = cl.Closure(eng, net, S)

    def outs():
        d = {"momenta": torch.zeros((S, 10, 3), dtype=torch.float32, device=dev),
             "ker": torch.zeros(S, dtype=torch.float64, device=dev),
             "steps": torch.zeros(S, dtype=torch.int32, device=dev),
             "status": torch.zeros(S, dtype=torch.uint8, device=dev)}
        return d, ce.CeOutputs(d["momenta"].data_ptr(), d["ker"].data_ptr(), d["steps"].data_ptr(),
                               d["status"].data_ptr())

    oc, c_oc = outs()
    op, c_op = outs()
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    batch_c = sb.c()

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
                ev[i][0].record(stream)
            fn()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev) / args.steps

    with ClockSampler(0) as clk:
        ms_plain = timed(lambda: eng.run_mixed_device(S, batch_c, cfg, c_op, sched, stream.cuda_stream))
        ms_clo = timed(lambda: clo.serve(sb, cfg, gate, c_oc, loose_pe_stop=args.loose_pe_stop,
                                         stream=stream.cuda_stream, cbatch=batch_c))
    acc, fbk = clo.counts()
    fbf = clo.fallback_flags(S, stream.cuda_stream)
    torch.cuda.synchronize()
    # stage breakdown: the loose run alone, and the plain rerun of the sims the gate sent back
    lcfg = ce.RunConfig(rtol=rtol, atol=atol, pe_stop_fraction=args.loose_pe_stop, redistribute_energy=False,
                        precision_mode=args.mode)
    lo_m = torch.empty((S, 10, 3), dtype=torch.float32, device=dev)
    lo_x = torch.empty((S, 10, 3), dtype=torch.float32, device=dev)
    lo_d = torch.empty((3, S), dtype=torch.float64, device=dev)
    lo_s = torch.empty(S, dtype=torch.int32, device=dev)
    lo_st = torch.empty(S, dtype=torch.uint8, device=dev)
    c_lo = ce.CeOutputs(lo_m.data_ptr(), None, lo_s.data_ptr(), lo_st.data_ptr(), None, None, lo_d[1].data_ptr(),
                        None, lo_x.data_ptr(), lo_d[2].data_ptr())
    ms_loose = timed(lambda: eng.run_mixed_device(S, batch_c, lcfg, c_lo, sched, stream.cuda_stream))
    del lo_m, lo_x, lo_d, lo_s, lo_st

    # network forward alone (tensor-core roofline of the learned part)
    feats = torch.zeros((cl.pad128(S), ce.CLOSURE_FEATURES), dtype=torch.bfloat16, device=dev)
    fl_row = 2 * (ce.CLOSURE_FEATURES * net.hidden + (net.depth - 1) * net.hidden * net.hidden + net.hidden * 32)
    fwd_out = torch.empty((feats.shape[0], ce.CLOSURE_OUTPUTS), dtype=torch.float32, device=dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cur = torch.cuda.current_stream(dev).cuda_stream
    net.forward(feats, fwd_out, feats.shape[0], cur)  # warm (outside the events: no allocation inside)
    torch.cuda.synchronize()
    a.record()
    net.forward(feats, fwd_out, feats.shape[0], cur)
    b.record()
    torch.cuda.synchronize()
    ms_fwd = a.elapsed_time(b)
    fwd_tflops = fl_row * feats.shape[0] / (ms_fwd / 1e3) / 1e12
    del feats, fwd_out
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    bf16_peak = peaks.get("bf16_tflops") or 1590.0

    okc = (oc["status"] == 0) & (op["status"] == 0) & (sb.n >= 2)
    accepted = okc & (fbf == 0)
    e_all = cl.rel_err(oc["momenta"][okc], op["momenta"][okc])
    e_acc = cl.rel_err(oc["momenta"][accepted], op["momenta"][accepted])

    # FP64 oracle on a subset of the served sims
    n_sub = args.fp64_subset
    sub = np.linspace(0, S - 1, n_sub).astype(np.int64)
    nn_s, mm_s, qq_s, xx_s = [], [], [], []
    for i in sub:
        a_, b_, c_, x32, _, _ = sp.sample_mixed_host(1, seed, first_sim=int(S_train + i))
        nn_s.append(a_[0]), mm_s.append(b_[0]), qq_s.append(c_[0]), xx_s.append(x32[0].astype(np.float64))
    nn_s, mm_s, qq_s, xx_s = np.array(nn_s), np.array(mm_s), np.array(qq_s), np.array(xx_s)
    ref = ol.run_batch_mixed(nn_s, mm_s, qq_s, xx_s, bits=64, rtol=1e-10, atol=1e-16, pe_stop=1e-11)
    pc, pp = oc["momenta"].cpu().numpy()[sub], op["momenta"].cpu().numpy()[sub]
    acc_np = accepted.cpu().numpy()[sub]
    e64_c = np.array([ol.config_norm_error(pc[j:j + 1, :k], ref["momenta"][j:j + 1, :k])[0]
                      for j, k in enumerate(nn_s)])
    e64_p = np.array([ol.config_norm_error(pp[j:j + 1, :k], ref["momenta"][j:j + 1, :k])[0]
                      for j, k in enumerate(nn_s)])

    def d_np(e):
        return {"median": float(np.median(e)), "p99": float(np.percentile(e, 99)), "max": float(e.max())} if len(
            e) else None

    steps_c = oc["steps"].double()
    line = {
        "metric": METRIC + " [learned closure vs plain RK45, mixed 2..10-atom population, 1e7 sims]",
        "value": S / (ms_clo / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_clo, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 integration, bf16/f32-accumulate network", "data": "synthetic",
        "config": {"workload": f"closure serving of {S} held-out mixed sims per step (N ~ U{{2..10}}, species "
                               "U{H,C,N,O,S}, q ~ U{+1,+2,+3}, radius 2.0 N^(1/3), min pair 0.5, Philox on device)",
                   "rtol": rtol, "atol": atol, "pe_stop": pes, "loose_pe_stop": args.loose_pe_stop,
                   "network": f"{ce.CLOSURE_FEATURES} -> {net.depth} x {net.hidden} SiLU -> 32, bf16 weights/activations, f32 accumulate",
                   "schedule": "per-size launches" if sched == ce.CE_SCHEDULE_PER_SIZE else "one persistent launch",
                   "l2": "flushed between timed steps (256 MiB write, outside the events)"},
        "plain": {"value": S / (ms_plain / 1e3), "unit": UNIT, "ms_per_step": ms_plain,
                  "mean_steps": float(op["steps"].double().mean())},
        "speedup_vs_plain": ms_plain / ms_clo,
        "breakdown_ms": {"loose_run": ms_loose, "network_forward": None,
                         "rest (features, gate, continuation of the sims sent back, merge)": None},
        "accepted_frac": acc / max(1, acc + fbk), "fallback_sims": fbk,
        "mean_steps_closure_path": float(steps_c[accepted].mean()) if bool(accepted.any()) else None,
        "gate": {"tol_energy": gate.tol_energy, "tol_momentum": gate.tol_momentum,
                 "tol_correction": gate.tol_correction,
                 "calibration": (f"correction bound for max validation error <= {args.gate_target_err}, "
                                 f"energy/momentum at the {args.gate_quantile} quantile") if args.gate_target_err
                 else f"{args.gate_quantile} quantile on validation"},
        "rel_err_vs_plain": {"all": dist(e_all), "accepted": dist(e_acc)},
        "rel_err_vs_fp64": {"subset": int(n_sub), "closure_all": d_np(e64_c), "closure_accepted": d_np(e64_c[acc_np]),
                            "plain": d_np(e64_p), "fp64": "oracle f64, rtol 1e-10, atol 1e-16, pe_stop 1e-11"},
        "training": {"sims": S_train, "generation_s": gen_s, "train_rows": int(train_rows.numel()),
                     "epochs": rep.epochs, "steps": rep.steps, "minibatch": mb, "seconds": rep.seconds,
                     "samples_per_s": rep.samples_per_s, "loss_first": float(losses[:20].mean()),
                     "loss_last": float(losses[-50:].mean())},
        "validation": val,
        "network_forward": {"rows": int(cl.pad128(S)), "ms": ms_fwd, "tflops": fwd_tflops,
                            "frac_of_bf16_peak": fwd_tflops / bf16_peak,
                            "peak_source": "MEASURED_PEAKS.json bf16_tflops" if peaks else "fallback 1590"},
        "clocks": clk.summary(),
    }
    line["breakdown_ms"]["network_forward"] = ms_fwd
    line["breakdown_ms"]["rest (features, gate, continuation of the sims sent back, merge)"] = (
        ms_clo - ms_loose - ms_fwd)
    print(json.dumps(line))
    clo.close()
    net.close()
    eng.close()
    return 0


def run_stream(args):
    """Streamed production generation: `--total` (default 1e8) explosions of the
    10-atom C2H6-like molecule (2 C q=+2, 8 H q=+1, radius 4.0, pairs >= 0.5) in
    1e6-sim chunks. Per chunk, on a compute stream: Philox geometries on the
    device, then the integration replayed from a CUDA graph captured once per
    buffer slot; on a side stream: the chunk's momenta / KER / steps / status
    copied into a pinned host ring (two slots) that the host consumes while the
    next chunk computes. Plain RK45 (the fixed-molecule entry point
    ce_run_device, autotuned layout) and the learned closure (a network trained
    on this molecule, held-out sims; its loose run and continuation go through
    the mixed-batch entry points, which save and resume integrator state) run
    the same pipeline back to back; the timed region is the whole stream, first
    geometry to last host byte."""
    import ctypes
    import importlib

    import torch

    from __graft_entry__ import load_package

    ce = load_package()
    cl = importlib.import_module("coulomb_explosion_b200.closure")
    wl = importlib.import_module("coulomb_explosion_b200.workloads")
    sp = importlib.import_module("coulomb_explosion_b200.sampling")
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_lib as ol

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    mol = wl.C2H6_LIKE
    rtol, atol, pes = TIGHT
    cfg = ce.RunConfig(rtol=rtol, atol=atol, pe_stop_fraction=pes, precision_mode=args.mode)
    C_ = 1_000_000
    total = (args.total // C_) * C_
    seed = SEED + 5
    eng = ce.Engine(0)
    eng.reserve_mixed(C_)

    # ---- network for this molecule, trained on held-out sims (counter range above the stream)
    t0 = time.perf_counter()
    mb = args.minibatch
    tb = cl.sample_molecule_device(mol, args.train_sims, seed, first_sim=1 << 40)
    torch.cuda.synchronize()
    ts, loose_t, base_t, plain_t = cl.make_training_set(eng, tb, cfg, loose_pe_stop=args.loose_pe_stop,
                                                         minibatch=mb)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    perm = torch.randperm(ts.S, generator=g, device=dev)
    n_val = max(mb, ts.S // 50)
    val_rows, train_rows = perm[:n_val], perm[n_val:]
    train_rows = train_rows[ts.valid[train_rows]]
    net = cl.Network(max_batch=65536, seed=seed)
    rep = cl.train(net, ts, epochs=args.epochs, minibatch=mb, lr=args.lr, lr_final=args.lr * 1e-2, seed=seed,
                   train_rows=train_rows)
    net.scale_output_layer(1.0 / cl.TARGET_SCALE)
    out_t = cl.net_forward(net, ts.feats)
    stats = cl.gate_stats(tb, loose_t, base_t, out_t)
    vmask = torch.zeros(ts.S, dtype=torch.bool, device=dev)
    vmask[val_rows] = True
    vmask &= ts.valid
    gate = cl.calibrate_gate(stats, vmask, quantile=args.gate_quantile)
    p_net_t = cl.predict(tb, base_t, out_t)
    if args.gate_target_err:
        gate = cl.calibrate_gate_for_error(stats, cl.rel_err(p_net_t, plain_t["momenta"]), vmask, args.gate_target_err,
                                           quantile=args.gate_quantile)
    val_err = cl.rel_err(p_net_t[vmask], plain_t["momenta"][vmask]).float()
    ana_err = cl.rel_err(base_t["p_base"][vmask], plain_t["momenta"][vmask]).float()
    train_s = time.perf_counter() - t0
    del ts, loose_t, base_t, plain_t, out_t, stats, tb
    torch.cuda.empty_cache()

    # ---- two buffer slots, pinned host ring
    slots = []
    for _ in range(2):
        b = cl.sample_molecule_device(mol, C_, seed, first_sim=0)
        d = {"batch": b, "cb": b.c(),
             "momenta": torch.empty((C_, 10, 3), dtype=torch.float32, device=dev),
             "ker": torch.empty(C_, dtype=torch.float64, device=dev),
             "steps": torch.empty(C_, dtype=torch.int32, device=dev),
             "status": torch.empty(C_, dtype=torch.uint8, device=dev)}
        d["out"] = ce.CeOutputs(d["momenta"].data_ptr(), d["ker"].data_ptr(), d["steps"].data_ptr(),
                                d["status"].data_ptr())
        d["host"] = {k: torch.empty(d[k].shape, dtype=d[k].dtype, pin_memory=True)
                     for k in ("momenta", "ker", "steps", "status")}
        slots.append(d)
    mrep, sched = eng.autotune_mixed(C_, slots[0]["cb"], cfg)
    mixed_pick = max(mrep, key=lambda r: r["sims_per_s"]) if mrep else {"lanes_per_sim": 0}
    eng.reserve_mixed(C_)
    # the plain leg: this molecule through the fixed-molecule entry point (rows of
    # 10 atoms are the same [S][10][3] layout in both), its layout autotuned
    eng.set_molecule(mol.masses_me, mol.charge_array)
    eng.autotune_fixed(C_, slots[0]["batch"].pos.data_ptr(), cfg)
    fixed_tuning = eng.get_tuning()
    clo = cl.Closure(eng, net, C_)
    compute = torch.cuda.Stream(device=dev)
    side = torch.cuda.Stream(device=dev)
    cs, ss = compute.cuda_stream, side.cuda_stream
    bcfg = sp.ball_config(mol, seed)
    lib = ce.load_library()
    d2h_bytes = C_ * (120 + 8 + 4 + 1)

    def capture(mode):
        graphs = []
        for d in slots:
            # one eager call first: sizes engine scratch and packs the network weights outside the capture
            if mode == "closure":
                clo.serve(d["batch"], cfg, gate, d["out"], loose_pe_stop=args.loose_pe_stop, stream=cs, cbatch=d["cb"])
            else:
                eng.run_device(C_, d["batch"].pos.data_ptr(), cfg, d["out"], cs)
            torch.cuda.synchronize()
            eng.graph_begin(cs)
            if mode == "closure":
                clo.serve(d["batch"], cfg, gate, d["out"], loose_pe_stop=args.loose_pe_stop, stream=cs, cbatch=d["cb"])
            else:
                eng.run_device(C_, d["batch"].pos.data_ptr(), cfg, d["out"], cs)
            graphs.append(eng.graph_end(cs))
        return graphs

    def stream_run(graphs, keep_first):
        done_ev = [torch.cuda.Event() for _ in range(2)]
        copied_ev = [torch.cuda.Event() for _ in range(2)]
        first = None
        ok_count = 0
        nchunks = total // C_
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(compute)

        def consume(i):
            nonlocal first, ok_count
            d = slots[i % 2]
            copied_ev[i % 2].synchronize()
            ok_count += int((d["host"]["status"].numpy() == 0).sum())
            if keep_first and i == 0:
                first = {k: v.clone() for k, v in d["host"].items()}

        for i in range(nchunks):
            d = slots[i % 2]
            if i >= 2:
                compute.wait_event(copied_ev[i % 2])
            rc = lib.ce_sample_ball_device(10, i * C_, C_, ctypes.byref(bcfg), ctypes.c_void_p(d["batch"].pos.data_ptr()),
                                           None, ctypes.c_void_p(cs))
            assert rc == 0
            graphs[i % 2].launch(cs)
            done_ev[i % 2].record(compute)
            side.wait_event(done_ev[i % 2])
            with torch.cuda.stream(side):
                for k in ("momenta", "ker", "steps", "status"):
                    d["host"][k].copy_(d[k], non_blocking=True)
            copied_ev[i % 2].record(side)
            if i >= 1:
                consume(i - 1)
        consume(nchunks - 1)
        stop.record(side)
        torch.cuda.synchronize()
        return start.elapsed_time(stop), ok_count, first

    res = {}
    firsts = {}
    with ClockSampler(0) as clk:
        for mode in ("plain", "closure"):
            graphs = capture(mode)
            stream_run(graphs, False)  # warm-up pass over the first chunks is the capture call; one full untimed pass
            ms, okc, first = stream_run(graphs, True)
            res[mode] = {"explosions_per_s": total / (ms / 1e3), "seconds": ms / 1e3, "status_ok_frac": okc / total}
            firsts[mode] = first
            for gph in graphs:
                gph.close()
    acc, fbk = clo.counts()

    # ---- kernel-level rooflines, event-timed outside the stream: the plain
    # integration of chunk 0 (FP32 CUDA cores, algorithmic FLOPs from its own
    # step counts at N = 10, P = 45) and the closure network's fused forward on
    # C_ rows (tensor cores, against the measured bf16 peak)
    d0 = slots[0]
    assert lib.ce_sample_ball_device(10, 0, C_, ctypes.byref(bcfg), ctypes.c_void_p(d0["batch"].pos.data_ptr()),
                                     None, ctypes.c_void_p(cs)) == 0
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(4)]
    for a_, b_ in evs:
        a_.record(compute)
        eng.run_device(C_, d0["batch"].pos.data_ptr(), cfg, d0["out"], cs)
        b_.record(compute)
    torch.cuda.synchronize()
    int_ms = float(np.median([a_.elapsed_time(b_) for a_, b_ in evs[1:]]))
    int_flops = float(flops_per_sim(d0["steps"].cpu().numpy().astype(np.uint32), 10).sum())
    fp32 = measure_fp32_peak(torch, dev)
    int_tf = int_flops / (int_ms / 1e3) / 1e12
    rows = cl.pad128(C_)
    gx = torch.Generator(device=dev)
    gx.manual_seed(seed)
    xf = torch.randn((rows, ce.CLOSURE_FEATURES), generator=gx, device=dev).to(torch.bfloat16)
    of = torch.empty((rows, ce.CLOSURE_OUTPUTS), dtype=torch.float32, device=dev)
    for a_, b_ in evs:
        a_.record(compute)
        net.forward(xf, of, rows, cs)
        b_.record(compute)
    torch.cuda.synchronize()
    net.check(cs)
    fwd_ms = float(np.median([a_.elapsed_time(b_) for a_, b_ in evs[1:]]))
    fl_row = 2 * (ce.CLOSURE_FEATURES * net.hidden + (net.depth - 1) * net.hidden * net.hidden + net.hidden * 32)
    fwd_tf = fl_row * rows / (fwd_ms / 1e3) / 1e12
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    bf16_peak = peaks.get("bf16_tflops") or 1590.0
    del xf, of

    # ---- the reference's SIMD batched engine on this host, same molecule and
    # tolerance point, on a bounded sample of the stream's geometries
    cpu = None
    if not args.no_cpu:
        n_cpu = 1 << 17
        x_cpu, _, fl_cpu = sp.sample_ball_host(mol, n_cpu, seed=seed, first_sim=0)
        assert not fl_cpu.any()
        cpu = cpu_batched_baseline(x_cpu.astype(np.float64), mol, TIGHT, all_steps=3, single_reps=5,
                                   single_sample=4096, scalar_sample=1024)
        if cpu:
            cpu["sample"] = f"{n_cpu} sims of the stream (first chunk's geometries), " + cpu["sample"].split(", ", 1)[1]
            cpu["gpu_e2e_speedup_vs_all_cores"] = res["plain"]["explosions_per_s"] / cpu["value"]
            cpu["gpu_e2e_speedup_vs_single_core"] = res["plain"]["explosions_per_s"] / cpu["single_core_value"]

    # accuracy on the first chunk: closure vs plain, both vs the FP64 oracle on a subset
    pc = firsts["closure"]["momenta"].double()
    pp = firsts["plain"]["momenta"].double()
    okm = (firsts["closure"]["status"] == 0) & (firsts["plain"]["status"] == 0)
    e_cp = cl.rel_err(pc[okm], pp[okm]).float()
    n_sub = args.fp64_subset
    sub = np.linspace(0, C_ - 1, n_sub).astype(np.int64)
    x32 = np.zeros((n_sub, 10, 3), np.float32)
    for j, i in enumerate(sub):
        a_, _, _ = sp.sample_ball_host(mol, 1, seed, first_sim=int(i))
        x32[j] = a_[0]
    ref = ol.run_batch(x32.astype(np.float64), mol.masses_me, mol.charge_array, bits=64, rtol=1e-10, atol=1e-16,
                       pe_stop=1e-11)
    e64_c = ol.config_norm_error(pc.numpy()[sub], ref["momenta"])
    e64_p = ol.config_norm_error(pp.numpy()[sub], ref["momenta"])

    def dist_t(e):
        return {"median": float(e.median()), "p99": float(torch.quantile(e[: 1 << 24], 0.99)), "max": float(e.max())}

    def dist_n(e):
        return {"median": float(np.median(e)), "p99": float(np.percentile(e, 99)), "max": float(e.max())}

    line = {
        "metric": METRIC + " [1e8 C2H6-like N=10 explosions streamed in 1e6 chunks, closure vs plain]",
        "value": res["closure"]["explosions_per_s"], "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": res["closure"]["seconds"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 integration, bf16/f32-accumulate network", "data": "synthetic",
        "config": {"workload": f"{total} C2H6-like (2 C q=+2, 8 H q=+1, r 4.0, min pair 0.5) explosions, "
                               f"{C_}-sim chunks, Philox geometries on device",
                   "rtol": rtol, "atol": atol, "pe_stop": pes, "loose_pe_stop": args.loose_pe_stop,
                   "pipeline": "compute stream: sampler + CUDA-graph replay per chunk; side stream: D2H into a "
                               "2-slot pinned host ring consumed by the host",
                   "plain_path": "ce_run_device (fixed molecule), autotuned lanes_per_sim "
                                 f"{fixed_tuning['lanes_per_sim']}, refill {fixed_tuning['refill_threshold']}",
                   "closure_path": "ce_closure_serve: loose run and continuation through the mixed-batch kernels, "
                                   "autotuned " + ("two threads per sim" if mixed_pick["lanes_per_sim"] == 2
                                                   else "one lane per atom"),
                   "d2h_bytes_per_chunk": d2h_bytes},
        "plain": res["plain"], "closure": res["closure"],
        "speedup_vs_plain": res["closure"]["explosions_per_s"] / res["plain"]["explosions_per_s"],
        "closure_last_chunk": {"accepted": acc, "fallback": fbk},
        "gate": {"tol_energy": gate.tol_energy, "tol_momentum": gate.tol_momentum,
                 "tol_correction": gate.tol_correction},
        "e2e": {"value": res["closure"]["explosions_per_s"], "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": d2h_bytes * (total // C_),
                "path": "whole stream, first geometry to last host byte: geometries drawn on the device (no input "
                        "copy), every chunk's results copied into pinned host memory"},
        "roofline": {"bound": "fp32", "kernel": "plain integration of one 1e6-sim chunk (ce_run_device, "
                                                "N = 10), event-timed outside the stream",
                     "achieved": int_tf, "peak": fp32["tflops"], "unit": "TFLOP/s", "frac": int_tf / fp32["tflops"],
                     "peak_source": fp32["source"], "flops_per_chunk": int_flops, "chunk_ms": int_ms},
        "roofline_network": {"bound": "tensor", "kernel": f"fused closure-network forward, {rows} rows",
                             "achieved": fwd_tf, "peak": bf16_peak, "unit": "TFLOP/s", "frac": fwd_tf / bf16_peak,
                             "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)" if peaks else "fallback 1590",
                             "chunk_ms": fwd_ms},
        "cpu_baseline": cpu,
        "rel_err_vs_plain_first_chunk": dist_t(e_cp),
        "rel_err_vs_fp64": {"subset": n_sub, "closure": dist_n(e64_c), "plain": dist_n(e64_p),
                            "fp64": "oracle f64, rtol 1e-10, atol 1e-16, pe_stop 1e-11"},
        "training": {"sims": args.train_sims, "epochs": rep.epochs, "steps": rep.steps, "seconds_total": train_s,
                     "validation_network": dist_t(val_err), "validation_analytic_only": dist_t(ana_err)},
        "clocks": clk.summary(),
    }
    print(json.dumps(line))
    clo.close()
    net.close()
    eng.close()
    return 0


def run_network(args):
    """The closure network's serving forward alone (fused tcgen05 kernel):
    `--sims` rows (default 1e7) of random BF16 features through 128 -> 4 x 256
    SiLU -> 32 with random weights, event-timed, against the measured bf16
    tensor-core peak."""
    import importlib

    import torch

    from __graft_entry__ import load_package

    ce = load_package()
    cl = importlib.import_module("coulomb_explosion_b200.closure")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rows = cl.pad128(args.sims if args.sims != S_DEFAULT else 10_000_000)
    net = cl.Network(max_batch=65536, seed=SEED)
    g = torch.Generator(device=dev)
    g.manual_seed(SEED)
    x = torch.randn((rows, ce.CLOSURE_FEATURES), generator=g, device=dev).to(torch.bfloat16)
    out = torch.empty((rows, ce.CLOSURE_OUTPUTS), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for _ in range(args.warmup):
        net.forward(x, out, rows, stream)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(0) as clk:
        for a, b in ev:
            a.record()
            net.forward(x, out, rows, stream)
            b.record()
        torch.cuda.synchronize()
    net.check(stream)
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    fl_row = 2 * (ce.CLOSURE_FEATURES * net.hidden + (net.depth - 1) * net.hidden * net.hidden + net.hidden * 32)
    tflops = fl_row * rows / (ms / 1e3) / 1e12
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("bf16_tflops") or 1590.0
    print(json.dumps({
        "metric": "closure network forward (fused tcgen05 kernel)", "value": rows / (ms / 1e3), "unit": "rows/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "dtype": "bf16 in, f32 accumulate", "data": "synthetic",
        "config": {"workload": f"{rows} rows, {ce.CLOSURE_FEATURES} -> {net.depth} x {net.hidden} SiLU -> 32",
                   "flops_per_row": fl_row},
        "roofline": {"bound": "tensor", "achieved": tflops, "peak": peak, "unit": "TFLOP/s", "frac": tflops / peak,
                     "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)" if peaks else "fallback 1590"},
        "clocks": clk.summary()}))
    net.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sims", type=int, default=S_DEFAULT)
    ap.add_argument("--mode", type=int, default=0,
                    help="CE_PREC_* bits: 0 plain FP32 (the f32 the workloads name, like the reference f32 engine); "
                         "1 Kahan x/v, 2 FP64 t/E, 3 both (see --workload precision)")
    ap.add_argument("--lanes", type=int, default=0, help="lanes per sim: 0 auto, 1 thread-per-sim, N lane-per-atom")
    ap.add_argument("--block", type=int, default=0, help="threads per block (0: engine default)")
    ap.add_argument("--refill", type=int, default=0, help="refill threshold in idle sims per warp (0: engine default)")
    ap.add_argument("--molecule", default="ch4", choices=["ch4", "c2h6", "h2o"],
                    help="ch4 (the headline workload), c2h6 (10-atom C2H6-like), h2o (stiff H2O)")
    ap.add_argument("--cpu-budget", type=float, default=8.0)
    ap.add_argument("--no-autotune", action="store_true",
                    help="mixed: skip the autotuner (engine defaults), e.g. to profile a known launch shape")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="fixed",
                    choices=["fixed", "mixed", "precision", "closure", "network", "stream"],
                    help="fixed: one molecule (--molecule); mixed: 2..10-atom population, one launch vs per size; "
                         "closure: learned closure vs plain RK45 on the mixed population; network: the closure "
                         "network's fused forward alone; stream: 1e8 C2H6-like explosions streamed in 1e6 chunks, "
                         "closure vs plain")
    ap.add_argument("--train-sims", type=int, default=5_000_000, help="closure: training pairs")
    ap.add_argument("--epochs", type=int, default=40, help="closure: training epochs")
    ap.add_argument("--minibatch", type=int, default=8192, help="closure: rows per training step")
    ap.add_argument("--lr", type=float, default=1e-3, help="closure: peak Adam learning rate")
    ap.add_argument("--gate-quantile", type=float, default=0.99, help="closure: gate bounds quantile")
    ap.add_argument("--val-frac", type=float, default=0.02,
                    help="closure: fraction of the training sims held out to validate and calibrate the gate")
    ap.add_argument("--fp64-subset", type=int, default=300, help="closure: sims checked against the FP64 oracle")
    ap.add_argument("--total", type=int, default=100_000_000, help="stream: explosions in the whole stream")
    ap.add_argument("--gate-target-err", type=float, default=0.0,
                    help="closure/stream: calibrate the gate so accepted validation sims stay within this relative "
                         "error (0: quantile bounds only)")
    ap.add_argument("--loose-pe-stop", type=float, default=0.05,
                    help="closure/stream: potential-energy fraction at which integration hands over to the closure")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "mixed":
        return run_mixed(args)
    if args.workload == "precision":
        return run_precision(args)
    if args.workload == "closure":
        return run_closure(args)
    if args.workload == "network":
        return run_network(args)
    if args.workload == "stream":
        return run_stream(args)

    import torch

    world, rank, local = dist_setup(args)
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)

    from __graft_entry__ import load_package

    ce = load_package()
    import importlib

    wl = importlib.import_module("coulomb_explosion_b200.workloads")
    mol = {"ch4": wl.CH4, "c2h6": wl.C2H6_LIKE, "h2o": wl.H2O_STIFF}[args.molecule]
    mol_desc = {"ch4": "CH4 (C+4H, q=+1, r 3.3, min pair 0.5)",
                "c2h6": "C2H6-like N=10 (2C q=+2, 8H q=+1, r 4.0, min pair 0.5)",
                "h2o": "stiff H2O (O q=+3, 2H q=+1, r 2.0, min pair 0.3)"}[args.molecule]
    S, n = args.sims, mol.n
    rtol, atol, pes = TIGHT
    cfg = ce.RunConfig(rtol=rtol, atol=atol, pe_stop_fraction=pes, precision_mode=args.mode)

    sp = importlib.import_module("coulomb_explosion_b200.sampling")
    rp = importlib.import_module("coulomb_explosion_b200.replicas")
    # Seeded Philox geometries; rank r integrates sims [r*S, (r+1)*S) of one population.
    first, _ = rp.shard(rank, world, S)
    pos_host, _, flags = sp.sample_ball_host(mol, S, seed=SEED, first_sim=first)
    assert not flags.any()
    eng = ce.Engine(dev.index)
    eng.set_molecule(mol.masses_me, mol.charge_array)
    if args.lanes or args.block or args.refill:
        eng.set_tuning(block_threads=args.block, lanes_per_sim=args.lanes, refill_threshold=args.refill)

    stream = torch.cuda.Stream(device=dev)
    pos_d = torch.from_numpy(pos_host).to(dev)
    mom_d = torch.empty((S, n, 3), dtype=torch.float32, device=dev)
    ker_d = torch.empty(S, dtype=torch.float64, device=dev)
    steps_d = torch.empty(S, dtype=torch.int32, device=dev)
    status_d = torch.empty(S, dtype=torch.uint8, device=dev)
    out = ce.CeOutputs(mom_d.data_ptr(), ker_d.data_ptr(), steps_d.data_ptr(), status_d.data_ptr(), None, None,
                       None, None)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2
    torch.cuda.synchronize(dev)

    def launch():
        eng.run_device(S, pos_d.data_ptr(), cfg, out, stream.cuda_stream)
        return eng.last_launch_count()

    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize(dev)

    # ---- device-timed region ----
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches = 0
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(dev.index) as clk:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
                ev[i][0].record(stream)
            launches += launch()
            ev[i][1].record(stream)
        torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    per = [a.elapsed_time(b) for a, b in ev]  # ms per launch (flush excluded)
    total_ms = rp.max_over_ranks(float(sum(per)), dev)
    value = rp.aggregate_rate(world, S, args.steps, total_ms)

    # ---- results of the last step: accuracy and FLOP accounting ----
    mom = mom_d.cpu().numpy()
    steps = steps_d.cpu().numpy().astype(np.uint32)
    status = status_d.cpu().numpy()
    ker = ker_d.cpu().numpy()

    # ---- end-to-end through the C ABI host-buffer call ----
    pin_pos = torch.from_numpy(pos_host).pin_memory()
    pin_mom = torch.empty((S, n, 3), dtype=torch.float32).pin_memory()
    pin_ker = torch.empty(S, dtype=torch.float64).pin_memory()
    pin_steps = torch.empty(S, dtype=torch.int32).pin_memory()
    pin_status = torch.empty(S, dtype=torch.uint8).pin_memory()
    hout = ce.CeOutputs(pin_mom.data_ptr(), pin_ker.data_ptr(), pin_steps.data_ptr(), pin_status.data_ptr(),
                        None, None, None, None)
    import ctypes

    cc = cfg.to_c()
    e2e_steps = max(3, args.steps // 2)
    eng.lib.ce_run(eng.h, S, ctypes.c_void_p(pin_pos.data_ptr()), ctypes.byref(cc), ctypes.byref(hout))
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        rc = eng.lib.ce_run(eng.h, S, ctypes.c_void_p(pin_pos.data_ptr()), ctypes.byref(cc), ctypes.byref(hout))
        assert rc == 0, eng.lib.ce_last_error(eng.h)
    e2e_s = rp.max_over_ranks(time.perf_counter() - t0, dev)
    e2e_value = rp.aggregate_rate(world, S, e2e_steps, e2e_s * 1e3)
    h2d = S * n * 3 * 4
    d2h = S * (n * 3 * 4 + 8 + 4 + 1)

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0

    sub = np.arange(0, S, max(1, S // 500))[:500]
    acc = accuracy_leg(pos_host[sub].astype(np.float64), mom[sub], mol, TIGHT)
    ol = _oracle_lib()
    pe0 = np.array([ol.potential(x, mol.charge_array) for x in pos_host[sub].astype(np.float64)])

    fl = flops_per_sim(steps, n).sum()
    per_launch_ms = total_ms / args.steps if world == 1 else float(np.mean(per))
    achieved_tflops = fl / (per_launch_ms / 1e3) / 1e12
    peak = measure_fp32_peak(torch, dev)

    cpu = None
    if not args.no_cpu and world == 1:
        cpu = cpu_batched_baseline(pos_host.astype(np.float64), mol, TIGHT)
        if cpu:
            cpu["gpu_speedup_vs_single_core"] = value / cpu["single_core_value"]
            cpu["gpu_e2e_speedup_vs_single_core"] = e2e_value / cpu["single_core_value"]
            cpu["gpu_speedup_vs_all_cores"] = value / cpu["value"]

    # DRAM traffic of one integration launch, from the committed ncu summary of
    # this workload (dram__bytes_read.sum + dram__bytes_write.sum).
    traffic = None
    lanes = eng.get_tuning()["lanes_per_sim"]
    layout = "thread" if lanes == 1 else ("pair" if lanes == 2 and mol.n >= 3 else "atom")
    tp = ROOT / "profiles" / f"rk45_{layout}_{args.molecule}_1e6.md"
    if tp.exists() and S == S_DEFAULT and args.molecule == "ch4" and args.mode == 0:
        import re

        m = re.search(r"traffic_bytes_per_launch:\s*([0-9]+)", tp.read_text())
        traffic = int(m.group(1)) if m else None

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {
            "workload": f"{mol_desc} Coulomb explosions, {S} sims per step per GPU",
            "sims_per_step": S, "atoms": n, "rtol": rtol, "atol": atol, "pe_stop": pes,
            "precision_mode": args.mode, "parallelism": f"replicas x{world} (independent shards)",
            "tuning": eng.get_tuning(),
            "l2": "flushed between timed steps (256 MiB write, outside the events)",
            "inputs": f"Philox4x32-10 uniform-ball geometries (seed {SEED}, whole-geometry min-pair rejection), "
                      "resident in HBM",
        },
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "ce_run (C ABI, pinned host buffers, synchronous)"},
        "gpu_launches": launches,
        "roofline": {"bound": "fp32", "achieved": achieved_tflops, "peak": peak["tflops"], "unit": "TFLOP/s",
                     "frac": achieved_tflops / peak["tflops"], "traffic": traffic,
                     "peak_source": peak["source"], "peak_probes": peak.get("probes"),
                     "frac_of_nominal": achieved_tflops / NOMINAL_FP32_TFLOPS,
                     "flops_per_launch": fl, "mean_steps": float(steps.mean())},
        "accuracy": dict(acc, status_ok_frac=float((status == 0).mean()),
                         ker_vs_pe0_max_rel=float(np.max(np.abs(ker[sub] - pe0) / pe0))),
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    eng.close()
    return 0


NOMINAL_FP32_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 148 SMs x 128 FP32 lanes x 2 x 1.965 GHz


def measure_fp32_peak(torch, dev):
    """FP32 FMA throughput of this GPU, measured live with the engine's probe
    kernels sized to >= 20 ms per launch: scalar FFMA and packed FFMA2 (the
    explosion kernel issues both); the larger is the roofline denominator.
    Falls back to the nominal 148 SMs x 128 lanes x 2 x 1.965 GHz."""
    from __graft_entry__ import load_package

    ce = load_package()
    lib = ce.load_library()
    import ctypes

    got = {}
    if hasattr(lib, "ce_probe_fp32_peak_ex"):
        for packed, name in ((0, "ffma"), (1, "ffma2")):
            v, ms = ctypes.c_double(0.0), ctypes.c_double(0.0)
            rc = lib.ce_probe_fp32_peak_ex(int(dev.index), packed, ctypes.c_double(20.0), ctypes.byref(v),
                                           ctypes.byref(ms))
            if rc == 0 and v.value > 0:
                got[name] = {"tflops": v.value, "launch_ms": ms.value}
    if got:
        best = max(got.values(), key=lambda r: r["tflops"])["tflops"]
        return {"tflops": best, "source": "measured in this run: FFMA / FFMA2 probe kernels, >= 20 ms per launch, "
                                          "best of 5, larger of the two",
                "probes": got, "nominal_tflops": NOMINAL_FP32_TFLOPS}
    return {"tflops": NOMINAL_FP32_TFLOPS, "source": "nominal (148 SMs x 128 FP32 lanes x 1.965 GHz)",
            "nominal_tflops": NOMINAL_FP32_TFLOPS}


if __name__ == "__main__":
    sys.exit(main())
