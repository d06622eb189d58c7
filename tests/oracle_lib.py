"""ctypes bindings to the CPU oracle (test infrastructure only).

  oracle/libce_oracle.so   the C restatement of the reference scalar engine
  oracle/_ref/libref_*.so  the reference scalar engine built from its own sources
  oracle/_ref/libref_batched_<isa>.so  the reference SIMD batched engine
                           (BatchedRK45<T>) built from its unmodified headers
                           against the project's Highway-API shim

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_SO = ROOT / "oracle" / "libce_oracle.so"
REF_F32_SO = ROOT / "oracle" / "_ref" / "libref_f32.so"
REF_F64_SO = ROOT / "oracle" / "_ref" / "libref_f64.so"
REF_BATCHED_SO = {isa: ROOT / "oracle" / "_ref" / f"libref_batched_{isa}.so" for isa in ("avx512", "avx2")}

KAHAN = 1
FP64 = 2


class OracleCfg(C.Structure):
    _fields_ = [
        ("rtol", C.c_double),
        ("atol", C.c_double),
        ("pe_stop_fraction", C.c_double),
        ("max_dt", C.c_double),
        ("max_steps", C.c_uint64),
        ("redistribute_energy", C.c_int),
        ("mode", C.c_int),
        ("integrator", C.c_int),
    ]


class OracleStats(C.Structure):
    _fields_ = [
        ("steps", C.c_uint32),
        ("rejects", C.c_uint32),
        ("status", C.c_uint8),
        ("t_final", C.c_double),
        ("e0", C.c_double),
        ("pe_final", C.c_double),
        ("ke_before", C.c_double),
        ("ke_after", C.c_double),
        ("scale", C.c_double),
    ]


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


_oracle = None
_refs: dict = {}


def oracle() -> C.CDLL:
    global _oracle
    if _oracle is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"oracle not built: {ORACLE_SO} (make -C oracle)")
        lib = C.CDLL(str(ORACLE_SO))
        vp = C.c_void_p
        lib.ce_oracle_run_batch.argtypes = [C.c_int, C.c_int, vp, vp, C.c_double, C.c_uint64, vp,
                                            C.POINTER(OracleCfg)] + [vp] * 8 + [C.c_int]
        lib.ce_oracle_run_batch_mixed.argtypes = [C.c_int, C.c_uint64, vp, vp, vp, C.c_double, vp,
                                                  C.POINTER(OracleCfg), vp, vp, vp, vp, C.c_int]
        for s in ("f32", "f64"):
            f = getattr(lib, f"ce_oracle_accel_{s}")
            f.argtypes = [C.c_int, vp, vp, vp, C.c_double, vp]
            f = getattr(lib, f"ce_oracle_pe_{s}")
            f.argtypes = [C.c_int, vp, vp, C.c_double]
            f.restype = C.c_double
            f = getattr(lib, f"ce_oracle_run_{s}")
            f.argtypes = [C.c_int, vp, vp, C.c_double, vp, C.POINTER(OracleCfg), vp, C.POINTER(OracleStats)]
        lib.ce_oracle_run_state_f32.argtypes = [C.c_int, vp, vp, C.c_double, vp, C.POINTER(OracleCfg), vp, vp,
                                                C.POINTER(OracleStats)]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return REF_F32_SO.exists() and REF_F64_SO.exists()


def ref(bits: int) -> C.CDLL:
    if bits not in _refs:
        path = REF_F32_SO if bits == 32 else REF_F64_SO
        if not path.exists():
            raise RuntimeError(f"reference engine not built: {path}")
        lib = C.CDLL(str(path))
        vp = C.c_void_p
        lib.ref_run_batch.argtypes = [C.c_int, vp, vp, C.c_double, C.c_uint64, vp, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_uint64, C.c_int, vp, vp, vp, vp, C.c_int]
        lib.ref_run_batch_kind.argtypes = [C.c_int] + lib.ref_run_batch.argtypes
        lib.ref_accel.argtypes = [C.c_int, vp, vp, vp, C.c_double, vp]
        lib.ref_pe.argtypes = [C.c_int, vp, vp, C.c_double]
        lib.ref_pe.restype = C.c_double
        lib.ref_sample.argtypes = [C.c_double, C.c_double, C.c_uint64, C.c_uint64, C.c_int, C.c_uint64, vp]
        lib.ref_sample.restype = C.c_int
        lib.ref_real_bytes.restype = C.c_int
        _refs[bits] = lib
    return _refs[bits]


def host_isa() -> str | None:
    """The widest vector ISA of this host the batched engine is built for, as the
    reference's -march=native static dispatch would pick it: "avx512"
    (x86-64-v4: AVX-512 F/BW/CD/DQ/VL), "avx2" (x86-64-v3: AVX2 + FMA) or None."""
    try:
        flags = set()
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("flags"):
                flags = set(line.split(":", 1)[1].split())
                break
    except OSError:
        return None
    if {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags:
        return "avx512"
    if {"avx2", "fma", "bmi2"} <= flags:
        return "avx2"
    return None


def batched_available(isa: str | None = None) -> bool:
    isa = isa or host_isa()
    return isa is not None and REF_BATCHED_SO[isa].exists()


_batched: dict = {}


def ref_batched(isa: str | None = None) -> C.CDLL:
    """The reference's BatchedRK45<T> library for `isa` (default: this host's)."""
    isa = isa or host_isa()
    if isa is None:
        raise RuntimeError("no AVX2/AVX-512 support on this host for the batched engine")
    if isa not in _batched:
        path = REF_BATCHED_SO[isa]
        if not path.exists():
            raise RuntimeError(f"reference batched engine not built: {path}")
        lib = C.CDLL(str(path))
        vp = C.c_void_p
        lib.refb_lanes.argtypes = [C.c_int]
        lib.refb_lanes.restype = C.c_int
        lib.refb_run.argtypes = [C.c_int, C.c_int, vp, vp, C.c_double, C.c_uint64, vp, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_uint64, C.c_int, vp, vp, vp, vp, C.c_int]
        lib.refb_run.restype = C.c_uint64
        _batched[isa] = lib
    return _batched[isa]


def batched_run(pos, mass, charge, *, bits=32, k=1.0, rtol=1e-8, atol=1e-16, pe_stop=1e-9, max_dt=1e12,
                max_steps=1_000_000, redistribute=True, threads=1, isa=None, outputs=True):
    """The reference's SIMD lockstep engine BatchedRK45<float> (bits 32) or
    <double> (bits 64) over pos [S, N, 3], K sims per batch as
    examples/generate_dataset.cpp:184-227 drives it. Returns a dict with
    momenta [S, N, 3] (float64, post-redistribution), steps, converged, status and
    batch_steps (lockstep iterations summed over batches)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    charge = np.ascontiguousarray(charge, dtype=np.float64)
    S, n, _ = pos.shape
    lib = ref_batched(isa)
    out = dict(momenta=np.zeros((S, n, 3)), steps=np.zeros(S, np.uint32), converged=np.zeros(S, np.uint8),
               status=np.zeros(S, np.uint8)) if outputs else {}
    bs = lib.refb_run(int(bits), n, _p(mass), _p(charge), k, S, _p(pos), rtol, atol, pe_stop, max_dt,
                      int(max_steps), 1 if redistribute else 0, _p(out.get("momenta")), _p(out.get("steps")),
                      _p(out.get("converged")), _p(out.get("status")), int(threads))
    out["batch_steps"] = int(bs)
    out["lanes"] = int(lib.refb_lanes(int(bits)))
    return out


def cfg(rtol=1e-8, atol=1e-16, pe_stop=1e-9, max_dt=1e12, max_steps=1_000_000, redistribute=True, mode=0,
        integrator=0):
    return OracleCfg(rtol, atol, pe_stop, max_dt, max_steps, 1 if redistribute else 0, mode, integrator)


def run_batch(pos, mass, charge, *, bits=32, k=1.0, threads=0, **kw):
    """Oracle over pos [S, N, 3] (float64) for one molecule. Returns a dict."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    charge = np.ascontiguousarray(charge, dtype=np.float64)
    S, n, _ = pos.shape
    out = dict(
        momenta=np.zeros((S, n, 3)), steps=np.zeros(S, np.uint32), status=np.zeros(S, np.uint8),
        rejects=np.zeros(S, np.uint32), ker=np.zeros(S), t_final=np.zeros(S), pe_final=np.zeros(S),
        ke_before=np.zeros(S),
    )
    c = cfg(**kw)
    oracle().ce_oracle_run_batch(bits, n, _p(mass), _p(charge), k, S, _p(pos), C.byref(c), _p(out["momenta"]),
                                 _p(out["steps"]), _p(out["status"]), _p(out["rejects"]), _p(out["ker"]),
                                 _p(out["t_final"]), _p(out["pe_final"]), _p(out["ke_before"]), int(threads))
    return out


def run_batch_mixed(n_per, mass, charge, pos, *, bits=32, k=1.0, threads=0, **kw):
    """Oracle over mixed molecules: n_per [S], mass/charge [S,10], pos [S,10,3]."""
    n_per = np.ascontiguousarray(n_per, dtype=np.uint8)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    charge = np.ascontiguousarray(charge, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    S = n_per.size
    out = dict(momenta=np.zeros((S, 10, 3)), steps=np.zeros(S, np.uint32), status=np.zeros(S, np.uint8),
               ker=np.zeros(S))
    c = cfg(**kw)
    oracle().ce_oracle_run_batch_mixed(bits, S, _p(n_per), _p(mass), _p(charge), k, _p(pos), C.byref(c),
                                       _p(out["momenta"]), _p(out["steps"]), _p(out["status"]),
                                       _p(out["ker"]), int(threads))
    return out


def ref_run_batch(pos, mass, charge, *, bits=32, k=1.0, rtol=1e-8, atol=1e-16, pe_stop=1e-9, max_dt=1e12,
                  max_steps=1_000_000, redistribute=True, threads=0, integrator=0):
    """The reference scalar engine (run_to_convergence per sim) over pos [S, N, 3];
    integrator 0 = RK45, 1 = Velocity Verlet with the fixed step max_dt."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    charge = np.ascontiguousarray(charge, dtype=np.float64)
    S, n, _ = pos.shape
    out = dict(momenta=np.zeros((S, n, 3)), steps=np.zeros(S, np.uint32), status=np.zeros(S, np.uint8),
               t_final=np.zeros(S))
    ref(bits).ref_run_batch_kind(int(integrator), n, _p(mass), _p(charge), k, S, _p(pos), rtol, atol, pe_stop,
                                 max_dt, max_steps, 1 if redistribute else 0, _p(out["momenta"]), _p(out["steps"]),
                                 _p(out["status"]), _p(out["t_final"]), int(threads))
    return out


def accel(x, mass, charge, *, bits=64, k=1.0):
    x = np.ascontiguousarray(x, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    charge = np.ascontiguousarray(charge, dtype=np.float64)
    a = np.zeros_like(x)
    getattr(oracle(), f"ce_oracle_accel_f{bits}")(x.shape[0], _p(x), _p(mass), _p(charge), k, _p(a))
    return a


def potential(x, charge, *, bits=64, k=1.0):
    x = np.ascontiguousarray(x, dtype=np.float64)
    charge = np.ascontiguousarray(charge, dtype=np.float64)
    return getattr(oracle(), f"ce_oracle_pe_f{bits}")(x.shape[0], _p(x), _p(charge), k)


def run_state(n, mass, charge, pos, *, k=1.0, **kw):
    """Loose-stop state of one sim (f32 engine arithmetic): (x [n,3], p [n,3], stats)."""
    lib = oracle()
    x = np.zeros((n, 3))
    p = np.zeros((n, 3))
    st = OracleStats()
    c = cfg(**kw)
    lib.ce_oracle_run_state_f32(int(n), _p(np.ascontiguousarray(mass, np.float64)),
                                _p(np.ascontiguousarray(charge, np.float64)), float(k),
                                _p(np.ascontiguousarray(pos, np.float64)), C.byref(c), _p(x), _p(p), C.byref(st))
    return x, p, st


def config_norm_error(p, p_ref):
    """Per-sim ||p - p_ref||_2 / ||p_ref||_2 over all 3N components
    (python/analysis/plot_precision.py:52-56; examples/verify_subset.py:77-79)."""
    p = np.asarray(p, dtype=np.float64).reshape(len(p), -1)
    q = np.asarray(p_ref, dtype=np.float64).reshape(len(p_ref), -1)
    return np.linalg.norm(p - q, axis=1) / np.linalg.norm(q, axis=1)


# ---------------------------------------------------------------------------
# Timed CPU baseline: one pinned process per core (test / bench infrastructure)
# ---------------------------------------------------------------------------

def usable_cores() -> list[int]:
    """The logical CPUs this process may run on, in order."""
    import os

    return sorted(os.sched_getaffinity(0))


def _core_worker(core, pos, mass, charge, params, cmd_q, res_q):
    """Pinned to `core`; runs its slice once per "run" command."""
    import os
    import time

    try:
        os.sched_setaffinity(0, {core})
        engine = params.pop("engine")
        if engine == "batched":
            ref_batched(params.get("isa"))
        else:
            ref(params["bits"])
        res_q.put(("ready", core, 0.0, 0))
        while True:
            cmd = cmd_q.get()
            if cmd is None:
                break
            t0 = time.perf_counter()
            if engine == "batched":
                r = batched_run(pos, mass, charge, threads=1, **params)
                work = r["batch_steps"]
            else:
                p = {k: v for k, v in params.items() if k != "isa"}
                r = ref_run_batch(pos, mass, charge, threads=1, **p)
                work = int(r["steps"].sum())
            res_q.put(("done", core, time.perf_counter() - t0, work))
    except Exception as e:  # report instead of dying silently
        res_q.put(("error", core, repr(e), 0))


class CorePool:
    """One `spawn` process per core, each pinned to its core (sched_setaffinity,
    the `taskset` of the reference's single-core measurements) and owning a
    disjoint contiguous slice of the sims. step() runs every slice once and
    returns the wall time of the whole step (coordinator clock: command out to
    last result in). engine "batched": the reference's BatchedRK45<T> driven
    like examples/generate_dataset.cpp:184-227; "scalar": the reference's
    run_to_convergence per sim. Geometries are generated before the pool starts
    and never timed (bench/bench_batched_integrator.cpp:140-174)."""

    def __init__(self, pos, mass, charge, cores, *, engine="batched", bits=32, rtol=1e-8, atol=1e-16,
                 pe_stop=1e-9, isa=None, timeout=600.0):
        import multiprocessing as mp

        pos = np.ascontiguousarray(pos, dtype=np.float64)
        self.S = pos.shape[0]
        self.cores = list(cores)
        self.timeout = timeout
        ctx = mp.get_context("spawn")
        self.res_q = ctx.Queue()
        self.cmd_qs = []
        self.procs = []
        # slices in whole K = 16 lane batches, so the lockstep batches are the
        # ones a single process would run
        bounds = (np.linspace(0, self.S // 16, len(self.cores) + 1).astype(int) * 16)
        bounds[-1] = self.S
        params = dict(engine=engine, bits=bits, rtol=rtol, atol=atol, pe_stop=pe_stop, isa=isa)
        for c, a, b in zip(self.cores, bounds[:-1], bounds[1:]):
            q = ctx.Queue()
            p = ctx.Process(target=_core_worker, args=(c, pos[a:b], mass, charge, dict(params), q, self.res_q),
                            daemon=True)
            p.start()
            self.cmd_qs.append(q)
            self.procs.append(p)
        self._collect("ready")

    def _collect(self, kind):
        out = []
        for _ in self.procs:
            msg = self.res_q.get(timeout=self.timeout)
            if msg[0] == "error":
                self.close()
                raise RuntimeError(f"CPU baseline worker on core {msg[1]} failed: {msg[2]}")
            assert msg[0] == kind, msg
            out.append(msg)
        return out

    def step(self) -> tuple[float, float, int]:
        """(wall seconds of one pass over all S sims, slowest worker's own
        seconds, work units: lockstep iterations or scalar steps)."""
        import time

        t0 = time.perf_counter()
        for q in self.cmd_qs:
            q.put("run")
        res = self._collect("done")
        wall = time.perf_counter() - t0
        return wall, max(r[2] for r in res), sum(r[3] for r in res)

    def close(self):
        for q in self.cmd_qs:
            try:
                q.put(None)
            except Exception:
                pass
        for p in self.procs:
            p.join(timeout=10)
            if p.is_alive():
                p.kill()
        self.procs = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def single_core_rate(pos, mass, charge, *, core=None, reps=7, **kw):
    """Explosions/s of one pinned core: median of `reps` passes over pos."""
    core = usable_cores()[-1] if core is None else core
    with CorePool(pos, mass, charge, [core], **kw) as pool:
        secs = [pool.step()[0] for _ in range(reps)]
    return len(pos) / float(np.median(secs)), secs
