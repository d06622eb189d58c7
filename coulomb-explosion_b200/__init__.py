"""B200-native Coulomb-explosion engine: Python plumbing over the C ABI.

The product is ``libce_gpu.so`` (CUDA, sm_100a) behind ``include/ce_gpu.h`` and
the C++ host mirror of the reference's ``coulomb::engine`` API under ``host/``.
This module binds the same C ABI with ctypes for tests and the benchmark; it
holds no numerics of its own and fails loudly when the CUDA library is absent.

Reference interfaces this mirrors (paths inside the reference project):
  BatchedRK45<T>(mol, k, lanes, rtol, atol)   include/coulomb/batched_integrator.hpp:71
  set_lane_geometry(lane, pos)                 include/coulomb/batched_integrator.hpp:112
  run(RunConfig) -> Result                     include/coulomb/batched_integrator.hpp:123
  RunConfig / IntegratorOptions                include/coulomb/driver.hpp:141, integrator.hpp:230
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libce_gpu.so"

AMU_TO_ME = 1822.888486209  # include/coulomb/units.hpp:13

CE_OK = 0
CE_ERR_INVALID = -1
CE_ERR_CUDA = -2
CE_ERR_NO_DEVICE = -3
CE_ERR_STATE = -4

CE_SIM_OK = 0
CE_SIM_REJECT_LIMIT = 1
CE_SIM_MAX_STEPS = 2
CE_SIM_NONFINITE = 3

CE_PREC_FP32 = 0
CE_PREC_KAHAN = 1
CE_PREC_FP64 = 2


class CeRunConfig(C.Structure):
    _fields_ = [
        ("rtol", C.c_double),
        ("atol", C.c_double),
        ("pe_stop_fraction", C.c_double),
        ("max_dt", C.c_double),
        ("max_steps", C.c_uint64),
        ("redistribute_energy", C.c_int32),
        ("precision_mode", C.c_int32),
    ]


class CeOutputs(C.Structure):
    _fields_ = [
        ("momenta", C.c_void_p),
        ("ker", C.c_void_p),
        ("steps", C.c_void_p),
        ("status", C.c_void_p),
        ("rejects", C.c_void_p),
        ("t_final", C.c_void_p),
        ("pe_final", C.c_void_p),
        ("ke_before", C.c_void_p),
        ("positions", C.c_void_p),
        ("e0", C.c_void_p),
    ]


class CeTuning(C.Structure):
    _fields_ = [
        ("block_threads", C.c_int32),
        ("blocks_per_sm", C.c_int32),
        ("refill_threshold", C.c_int32),
        ("lanes_per_sim", C.c_int32),
    ]


class CeMixedBatch(C.Structure):
    _fields_ = [("n_atoms", C.c_void_p), ("mass_me", C.c_void_p), ("charge", C.c_void_p), ("pos", C.c_void_p)]


class CeSimState(C.Structure):
    """ce_sim_state: a run's saved integrator state, or the state a resumed run
    continues from (device pointers, mixed layout)."""
    _fields_ = [("positions", C.c_void_p), ("velocities", C.c_void_p), ("h", C.c_void_p), ("t", C.c_void_p),
                ("steps", C.c_void_p), ("rejects", C.c_void_p), ("e0", C.c_void_p), ("comp", C.c_void_p)]


class CeTuneResult(C.Structure):
    _fields_ = [("t", CeTuning), ("sims_per_s", C.c_double), ("schedule", C.c_int32)]


class CeBallSampler(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("radius", C.c_double), ("min_separation", C.c_double),
                ("max_attempts", C.c_uint32)]


class CeMixedSampler(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("n_min", C.c_int32), ("n_max", C.c_int32), ("radius_coeff", C.c_double),
                ("min_separation", C.c_double), ("max_attempts", C.c_uint32), ("q_min", C.c_int32),
                ("q_max", C.c_int32), ("n_species", C.c_int32), ("species_amu", C.c_double * 8)]


class CeClosureState(C.Structure):
    _fields_ = [("positions", C.c_void_p), ("momenta", C.c_void_p), ("e0", C.c_void_p), ("pe_final", C.c_void_p),
                ("status", C.c_void_p)]


class CeClosureGate(C.Structure):
    _fields_ = [("tol_energy", C.c_float), ("tol_momentum", C.c_float), ("tol_correction", C.c_float)]


CLOSURE_FEATURES = 128
CLOSURE_OUTPUTS = 32
CE_SIM_BAD_INPUT = 4
CE_SCHEDULE_ONE_LAUNCH = 0
CE_SCHEDULE_PER_SIZE = 1
CE_SCHEDULE_OVERLAP = 2
MAX_ATOMS = 10


# Every entry point include/ce_gpu.h declares, with its ctypes signature.
_SIGNATURES = {
    "ce_version": ([], C.c_char_p),
    "ce_default_config": ([C.POINTER(CeRunConfig)], None),
    "ce_create": ([C.POINTER(C.c_void_p), C.c_int], C.c_int),
    "ce_destroy": ([C.c_void_p], None),
    "ce_last_error": ([C.c_void_p], C.c_char_p),
    "ce_set_molecule": ([C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double], C.c_int),
    "ce_set_tuning": ([C.c_void_p, C.POINTER(CeTuning)], C.c_int),
    "ce_get_tuning": ([C.c_void_p, C.POINTER(CeTuning)], C.c_int),
    "ce_run": ([C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(CeRunConfig), C.POINTER(CeOutputs)], C.c_int),
    "ce_run_device": (
        [C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(CeRunConfig), C.POINTER(CeOutputs), C.c_void_p],
        C.c_int,
    ),
    "ce_run_verlet_device": (
        [C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(CeRunConfig), C.POINTER(CeOutputs), C.c_void_p],
        C.c_int,
    ),
    "ce_last_launch_count": ([C.c_void_p], C.c_int),
    "ce_probe_fp32_peak": ([C.c_int, C.POINTER(C.c_double)], C.c_int),
    "ce_probe_fp32_peak_ex": ([C.c_int, C.c_int, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)],
                              C.c_int),
    "ce_probe_bounded_wait": ([C.c_int, C.c_uint, C.POINTER(C.c_int)], C.c_int),
    "ce_reserve_mixed": ([C.c_void_p, C.c_uint64], C.c_int),
    "ce_run_mixed_device_state": (
        [C.c_void_p, C.c_uint64, C.POINTER(CeMixedBatch), C.c_double, C.POINTER(CeRunConfig), C.POINTER(CeSimState),
         C.POINTER(CeSimState), C.POINTER(CeOutputs), C.c_int, C.c_void_p],
        C.c_int,
    ),
    "ce_run_mixed_device": (
        [C.c_void_p, C.c_uint64, C.POINTER(CeMixedBatch), C.c_double, C.POINTER(CeRunConfig), C.POINTER(CeOutputs),
         C.c_int, C.c_void_p],
        C.c_int,
    ),
    "ce_run_mixed": (
        [C.c_void_p, C.c_uint64, C.POINTER(CeMixedBatch), C.c_double, C.POINTER(CeRunConfig), C.POINTER(CeOutputs)],
        C.c_int,
    ),
    "ce_graph_begin": ([C.c_void_p, C.c_void_p], C.c_int),
    "ce_graph_end": ([C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
    "ce_graph_launch": ([C.c_void_p, C.c_void_p], C.c_int),
    "ce_graph_destroy": ([C.c_void_p], None),
    "ce_autotune_fixed": (
        [C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(CeRunConfig), C.POINTER(CeTuneResult), C.c_int,
         C.POINTER(C.c_int)],
        C.c_int,
    ),
    "ce_autotune_mixed": (
        [C.c_void_p, C.c_uint64, C.POINTER(CeMixedBatch), C.c_double, C.POINTER(CeRunConfig),
         C.POINTER(CeTuneResult), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)],
        C.c_int,
    ),
    "ce_sample_ball_device": (
        [C.c_int, C.c_uint64, C.c_uint64, C.POINTER(CeBallSampler), C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "ce_sample_ball_host": (
        [C.c_int, C.c_uint64, C.c_uint64, C.POINTER(CeBallSampler), C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "ce_sample_mixed_device": (
        [C.c_uint64, C.c_uint64, C.POINTER(CeMixedSampler), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
         C.c_void_p, C.c_void_p], C.c_int),
    "ce_sample_mixed_host": (
        [C.c_uint64, C.c_uint64, C.POINTER(CeMixedSampler), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
         C.c_void_p, C.c_void_p], C.c_int),
    "ce_philox4x32_10": ([C.c_void_p, C.c_void_p, C.c_void_p], None),
    "ce_mlp_create": ([C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_uint64],
                      C.c_int),
    "ce_mlp_destroy": ([C.c_void_p], None),
    "ce_mlp_last_error": ([C.c_void_p], C.c_char_p),
    "ce_mlp_param_count": ([C.c_void_p], C.c_uint64),
    "ce_mlp_set_params": ([C.c_void_p, C.c_void_p], C.c_int),
    "ce_mlp_get_params": ([C.c_void_p, C.c_void_p], C.c_int),
    "ce_mlp_forward": ([C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p], C.c_int),
    "ce_mlp_forward_layered": ([C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p], C.c_int),
    "ce_mlp_gradients": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                          C.c_void_p], C.c_int),
    "ce_mlp_train_step": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_float, C.c_void_p,
                           C.c_void_p], C.c_int),
    "ce_mlp_check": ([C.c_void_p, C.c_void_p], C.c_int),
    "ce_umma_gemm_f32": ([C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                          C.c_void_p, C.c_void_p], C.c_int),
    "ce_mlp_shape": ([C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                      C.POINTER(C.c_uint64)], C.c_int),
    "ce_closure_default_gate": ([C.POINTER(CeClosureGate)], None),
    "ce_closure_features": ([C.c_uint64, C.POINTER(CeMixedBatch), C.c_double, C.POINTER(CeClosureState), C.c_void_p,
                             C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
                            C.c_int),
    "ce_closure_apply": ([C.c_uint64, C.POINTER(CeMixedBatch), C.POINTER(CeClosureState), C.c_void_p, C.c_void_p,
                          C.c_void_p, C.c_void_p, C.POINTER(CeClosureGate), C.POINTER(CeOutputs), C.c_void_p,
                          C.c_void_p, C.c_void_p], C.c_int),
    "ce_closure_create": ([C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p, C.c_uint64], C.c_int),
    "ce_closure_destroy": ([C.c_void_p], None),
    "ce_closure_last_error": ([C.c_void_p], C.c_char_p),
    "ce_closure_serve": ([C.c_void_p, C.c_uint64, C.POINTER(CeMixedBatch), C.c_double, C.POINTER(CeRunConfig),
                          C.c_double, C.POINTER(CeClosureGate), C.POINTER(CeOutputs), C.c_void_p], C.c_int),
    "ce_closure_counts": ([C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)], C.c_int),
    "ce_closure_fallback_flags": ([C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p], C.c_int),
    "ce_run_device_noalloc": (
        [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_uint64, C.c_void_p, C.POINTER(CeRunConfig),
         C.POINTER(CeOutputs), C.c_void_p, C.c_char_p, C.c_size_t],
        C.c_int,
    ),
}

_lib = None


def load_library(path: os.PathLike | None = None) -> C.CDLL:
    """Load libce_gpu.so (built in-tree by ``build.py``). Raises if missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"CUDA engine library not built: {p} (run __graft_entry__.build())")
    lib = C.CDLL(str(p))
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _lib = lib
    return lib


class EngineError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ce_gpu error {code}: {msg}")
        self.code = code


@dataclass
class RunConfig:
    """RunConfig + IntegratorOptions (driver.hpp:141-163, integrator.hpp:230-233).

    Defaults are the reference's: rtol 1e-8, atol 1e-16, pe_stop 1e-9,
    max_dt 1e12, max_steps 1e6, redistribution on."""

    rtol: float = 1e-8
    atol: float = 1e-16
    pe_stop_fraction: float = 1e-9
    max_dt: float = 1e12
    max_steps: int = 1_000_000
    redistribute_energy: bool = True
    precision_mode: int = CE_PREC_FP32

    def to_c(self) -> CeRunConfig:
        return CeRunConfig(
            float(self.rtol), float(self.atol), float(self.pe_stop_fraction), float(self.max_dt),
            int(self.max_steps), 1 if self.redistribute_energy else 0, int(self.precision_mode),
        )


@dataclass
class Result:
    """Per-sim outputs (BatchedRK45<T>::Result, batched_integrator.hpp:64-69, plus
    KER, status and diagnostics)."""

    momenta: np.ndarray  # [S, N, 3] float32
    ker: np.ndarray  # [S] float64
    steps: np.ndarray  # [S] uint32
    status: np.ndarray  # [S] uint8
    rejects: np.ndarray | None = None
    t_final: np.ndarray | None = None
    pe_final: np.ndarray | None = None
    ke_before: np.ndarray | None = None
    positions: np.ndarray | None = None  # [S, N, 3] float32 positions at termination
    e0: np.ndarray | None = None  # [S] float64 initial energy (= PE_0)
    extra: dict = field(default_factory=dict)

    @property
    def converged(self) -> np.ndarray:
        return self.status == CE_SIM_OK


def _ptr(a: np.ndarray | None):
    return None if a is None else C.c_void_p(a.ctypes.data)


class Engine:
    """One engine per host thread and device (include/ce_gpu.h)."""

    def __init__(self, device: int = 0, lib_path: os.PathLike | None = None):
        self.lib = load_library(lib_path)
        h = C.c_void_p()
        rc = self.lib.ce_create(C.byref(h), int(device))
        if rc != CE_OK:
            raise EngineError(rc, f"ce_create(device={device}) failed")
        self.h = h
        self.n = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.ce_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != CE_OK:
            raise EngineError(rc, self.lib.ce_last_error(self.h).decode())

    def set_molecule(self, masses_me, charges, coulomb_k: float = 1.0):
        m = np.ascontiguousarray(masses_me, dtype=np.float64)
        q = np.ascontiguousarray(charges, dtype=np.float64)
        if m.shape != q.shape or m.ndim != 1:
            raise ValueError("masses and charges must be 1-D of equal length")
        self._check(self.lib.ce_set_molecule(self.h, int(m.size), _ptr(m), _ptr(q), float(coulomb_k)))
        self.n = int(m.size)
        self.masses = m
        self.charges = q

    def set_tuning(self, block_threads=0, blocks_per_sm=0, refill_threshold=0, lanes_per_sim=0):
        t = CeTuning(int(block_threads), int(blocks_per_sm), int(refill_threshold), int(lanes_per_sim))
        self._check(self.lib.ce_set_tuning(self.h, C.byref(t)))

    def get_tuning(self) -> dict:
        t = CeTuning()
        self._check(self.lib.ce_get_tuning(self.h, C.byref(t)))
        return {f: getattr(t, f) for f, _ in CeTuning._fields_}

    def run(self, pos, cfg: RunConfig | None = None, diagnostics: bool = False) -> Result:
        """Host-buffer path (ce_run): positions [S, N, 3] -> Result."""
        if self.n is None:
            raise EngineError(CE_ERR_STATE, "no molecule set")
        cfg = cfg or RunConfig()
        x = np.ascontiguousarray(pos, dtype=np.float32)
        if x.ndim != 3 or x.shape[1] != self.n or x.shape[2] != 3:
            raise ValueError(f"pos must be [S, {self.n}, 3]")
        S = x.shape[0]
        r = Result(
            momenta=np.zeros((S, self.n, 3), np.float32), ker=np.zeros(S, np.float64),
            steps=np.zeros(S, np.uint32), status=np.zeros(S, np.uint8),
        )
        if diagnostics:
            r.rejects = np.zeros(S, np.uint32)
            r.t_final = np.zeros(S, np.float64)
            r.pe_final = np.zeros(S, np.float64)
            r.ke_before = np.zeros(S, np.float64)
            r.positions = np.zeros_like(r.momenta)
            r.e0 = np.zeros(S, np.float64)
        out = CeOutputs(_ptr(r.momenta), _ptr(r.ker), _ptr(r.steps), _ptr(r.status), _ptr(r.rejects),
                        _ptr(r.t_final), _ptr(r.pe_final), _ptr(r.ke_before), _ptr(r.positions), _ptr(r.e0))
        c = cfg.to_c()
        self._check(self.lib.ce_run(self.h, S, _ptr(x), C.byref(c), C.byref(out)))
        return r

    def run_device(self, S: int, pos_ptr: int, cfg: RunConfig, out: CeOutputs, stream: int = 0):
        """Device-buffer path (ce_run_device): raw device pointers, async on `stream`."""
        c = cfg.to_c()
        self._check(self.lib.ce_run_device(self.h, int(S), C.c_void_p(pos_ptr), C.byref(c), C.byref(out),
                                           C.c_void_p(stream)))

    def run_verlet_device(self, S: int, pos_ptr: int, cfg: RunConfig, out: CeOutputs, stream: int = 0):
        """Velocity Verlet with the fixed step cfg.max_dt (ce_run_verlet_device)."""
        c = cfg.to_c()
        self._check(self.lib.ce_run_verlet_device(self.h, int(S), C.c_void_p(pos_ptr), C.byref(c), C.byref(out),
                                                  C.c_void_p(stream)))

    def last_launch_count(self) -> int:
        return int(self.lib.ce_last_launch_count(self.h))

    # ---- mixed molecules ----
    def run_mixed(self, n_atoms, masses_me, charges, pos, cfg: RunConfig | None = None, coulomb_k: float = 1.0,
                  diagnostics: bool = False) -> Result:
        """Host-buffer mixed path (ce_run_mixed): n_atoms [S], masses/charges [S, 10],
        pos [S, 10, 3] -> Result with momenta [S, 10, 3]."""
        cfg = cfg or RunConfig()
        n = np.ascontiguousarray(n_atoms, dtype=np.uint8)
        m = np.ascontiguousarray(masses_me, dtype=np.float64)
        q = np.ascontiguousarray(charges, dtype=np.float64)
        x = np.ascontiguousarray(pos, dtype=np.float32)
        S = n.size
        if m.shape != (S, MAX_ATOMS) or q.shape != (S, MAX_ATOMS) or x.shape != (S, MAX_ATOMS, 3):
            raise ValueError("mixed batch rows must be padded to 10 atoms")
        r = Result(momenta=np.zeros((S, MAX_ATOMS, 3), np.float32), ker=np.zeros(S, np.float64),
                   steps=np.zeros(S, np.uint32), status=np.zeros(S, np.uint8))
        if diagnostics:
            r.rejects = np.zeros(S, np.uint32)
            r.t_final = np.zeros(S, np.float64)
            r.pe_final = np.zeros(S, np.float64)
            r.ke_before = np.zeros(S, np.float64)
            r.positions = np.zeros_like(r.momenta)
            r.e0 = np.zeros(S, np.float64)
        out = CeOutputs(_ptr(r.momenta), _ptr(r.ker), _ptr(r.steps), _ptr(r.status), _ptr(r.rejects),
                        _ptr(r.t_final), _ptr(r.pe_final), _ptr(r.ke_before), _ptr(r.positions), _ptr(r.e0))
        batch = CeMixedBatch(_ptr(n), _ptr(m), _ptr(q), _ptr(x))
        c = cfg.to_c()
        self._check(self.lib.ce_run_mixed(self.h, S, C.byref(batch), float(coulomb_k), C.byref(c), C.byref(out)))
        return r

    def run_mixed_device_state(self, S: int, batch: CeMixedBatch, cfg: RunConfig, out: CeOutputs,
                               resume: "CeSimState | None" = None, save: "CeSimState | None" = None,
                               schedule: int = CE_SCHEDULE_ONE_LAUNCH, stream: int = 0, coulomb_k: float = 1.0):
        """ce_run_mixed_device_state: save the integrator state of every sim it
        finishes and / or continue sims from a saved state."""
        c = cfg.to_c()
        self._check(self.lib.ce_run_mixed_device_state(
            self.h, int(S), C.byref(batch), float(coulomb_k), C.byref(c), C.byref(resume) if resume else None,
            C.byref(save) if save else None, C.byref(out), int(schedule), C.c_void_p(stream)))

    def run_mixed_device(self, S: int, batch: CeMixedBatch, cfg: RunConfig, out: CeOutputs,
                         schedule: int = CE_SCHEDULE_ONE_LAUNCH, stream: int = 0, coulomb_k: float = 1.0):
        c = cfg.to_c()
        self._check(self.lib.ce_run_mixed_device(self.h, int(S), C.byref(batch), float(coulomb_k), C.byref(c),
                                                 C.byref(out), int(schedule), C.c_void_p(stream)))

    def reserve_mixed(self, S: int):
        self._check(self.lib.ce_reserve_mixed(self.h, int(S)))

    # ---- graphs ----
    def graph_begin(self, stream: int):
        self._check(self.lib.ce_graph_begin(self.h, C.c_void_p(stream)))

    def graph_end(self, stream: int) -> "Graph":
        g = C.c_void_p()
        self._check(self.lib.ce_graph_end(self.h, C.c_void_p(stream), C.byref(g)))
        return Graph(self.lib, g)

    # ---- autotuner ----
    def autotune_fixed(self, S: int, pos_ptr: int, cfg: RunConfig, cap: int = 64) -> list[dict]:
        rep = (CeTuneResult * cap)()
        n = C.c_int(0)
        c = cfg.to_c()
        self._check(self.lib.ce_autotune_fixed(self.h, int(S), C.c_void_p(pos_ptr), C.byref(c), rep, cap, C.byref(n)))
        return [_tune_dict(rep[i]) for i in range(n.value)]

    def autotune_mixed(self, S: int, batch: CeMixedBatch, cfg: RunConfig, coulomb_k: float = 1.0, cap: int = 64):
        rep = (CeTuneResult * cap)()
        n = C.c_int(0)
        best = C.c_int(0)
        c = cfg.to_c()
        self._check(self.lib.ce_autotune_mixed(self.h, int(S), C.byref(batch), float(coulomb_k), C.byref(c), rep, cap,
                                               C.byref(n), C.byref(best)))
        return [_tune_dict(rep[i]) for i in range(n.value)], int(best.value)


def _tune_dict(r: CeTuneResult) -> dict:
    return {"block_threads": r.t.block_threads, "blocks_per_sm": r.t.blocks_per_sm,
            "refill_threshold": r.t.refill_threshold, "lanes_per_sim": r.t.lanes_per_sim,
            "sims_per_s": r.sims_per_s, "schedule": r.schedule}


class Graph:
    """An instantiated CUDA graph of engine calls (ce_graph_*)."""

    def __init__(self, lib, handle):
        self.lib = lib
        self.h = handle

    def launch(self, stream: int):
        rc = self.lib.ce_graph_launch(self.h, C.c_void_p(stream))
        if rc != CE_OK:
            raise EngineError(rc, "ce_graph_launch failed")

    def close(self):
        if self.h:
            self.lib.ce_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def methane(charge_c: float = 1.0, charge_h: float = 1.0):
    """CH4 as examples/generate_dataset.cpp:56-66: C then 4 H, singly ionized."""
    amu = np.array([12.011, 1.008, 1.008, 1.008, 1.008])
    q = np.array([charge_c] + [charge_h] * 4, dtype=np.float64)
    return amu * AMU_TO_ME, q
