"""Learned asymptotic closure (include/ce_closure.h): training-pair generation,
training on the GPU with the library's own tensor-core kernels, gate
calibration and serving.

The reference's only closure is the uniform velocity rescale at the stop
(src/driver.cpp:38-42). Here every sim is integrated to a loose stop
(PE <= 5% PE_0), the closed-form straight-line pair impulse to t -> infinity
plus that rescale gives a base, and a BF16 MLP (128 -> 4 x 256 SiLU -> 32)
predicts the remaining correction in units of the analytic step's size.
Training targets are the engine's own fully converged momenta on the same
inputs. Device memory is held in torch tensors; every computation on the
closure path runs in libce_gpu.so.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import (CLOSURE_FEATURES, CLOSURE_OUTPUTS, MAX_ATOMS, CeClosureGate, CeClosureState, CeMixedBatch, CeOutputs,
               Engine, EngineError, RunConfig, load_library)
from .sampling import mixed_config

# The output layer is trained on targets scaled by this power of two and
# divided back before serving (exact in BF16 and FP32).
TARGET_SCALE = 128.0
LOOSE_PE_STOP = 0.05


def _torch():
    import torch

    return torch


def _vp(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def pad128(S: int) -> int:
    return (S + 127) // 128 * 128


class Network:
    """ce_mlp handle: in 128 -> hidden x depth (SiLU) -> 32."""

    def __init__(self, device: int = 0, hidden: int = 256, depth: int = 4, max_batch: int = 65536, seed: int = 1):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.ce_mlp_create(C.byref(h), int(device), CLOSURE_FEATURES, int(hidden), int(depth),
                                    CLOSURE_OUTPUTS, int(max_batch), int(seed))
        if rc != 0:
            raise EngineError(rc, "ce_mlp_create failed")
        self.h = h
        self.device = device
        self.hidden, self.depth, self.max_batch = hidden, depth, max_batch
        self.n_params = int(self.lib.ce_mlp_param_count(h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.ce_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != 0:
            raise EngineError(rc, self.lib.ce_mlp_last_error(self.h).decode())

    def layer_shapes(self):
        dims = [CLOSURE_FEATURES] + [self.hidden] * self.depth + [CLOSURE_OUTPUTS]
        return [(dims[i + 1], dims[i]) for i in range(len(dims) - 1)]

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.n_params, np.float32)
        self._check(self.lib.ce_mlp_get_params(self.h, C.c_void_p(p.ctypes.data)))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.n_params:
            raise ValueError("parameter count mismatch")
        self._check(self.lib.ce_mlp_set_params(self.h, C.c_void_p(p.ctypes.data)))

    def scale_output_layer(self, factor: float):
        """Multiply the last layer's weights and bias by `factor`."""
        p = self.get_params()
        fo, fi = self.layer_shapes()[-1]
        tail = fo * fi + fo
        p[-tail:] *= np.float32(factor)
        self.set_params(p)

    def forward(self, feats, out, B: int, stream: int = 0):
        self._check(self.lib.ce_mlp_forward(self.h, _vp(feats), int(B), _vp(out), C.c_void_p(stream)))

    def train_step(self, feats, target, weight, B: int, lr: float, loss_dev=None, stream: int = 0):
        self._check(self.lib.ce_mlp_train_step(self.h, _vp(feats), _vp(target), _vp(weight), int(B), float(lr),
                                               _vp(loss_dev), C.c_void_p(stream)))

    def check(self, stream: int = 0):
        self._check(self.lib.ce_mlp_check(self.h, C.c_void_p(stream)))

    def save(self, path):
        np.savez(path, params=self.get_params(), hidden=self.hidden, depth=self.depth)

    def load(self, path):
        z = np.load(path)
        if int(z["hidden"]) != self.hidden or int(z["depth"]) != self.depth:
            raise ValueError("network shape mismatch")
        self.set_params(z["params"])


@dataclass
class DeviceBatch:
    """A mixed batch in device memory (rows padded to 10 atoms)."""

    n: object
    mass: object
    charge: object
    pos: object

    @property
    def S(self) -> int:
        return int(self.n.shape[0])

    def c(self) -> CeMixedBatch:
        return CeMixedBatch(self.n.data_ptr(), self.mass.data_ptr(), self.charge.data_ptr(), self.pos.data_ptr())

    def slice(self, a: int, b: int) -> "DeviceBatch":
        return DeviceBatch(self.n[a:b], self.mass[a:b], self.charge[a:b], self.pos[a:b])


def sample_mixed_device(S: int, seed: int, first_sim: int = 0, device: int = 0, **kw) -> DeviceBatch:
    """The mixed population (2..10 atoms, species H/C/N/O/S, charges +1..+3) from
    the device Philox sampler."""
    torch = _torch()
    lib = load_library()
    dev = torch.device("cuda", device)
    n = torch.empty(S, dtype=torch.uint8, device=dev)
    m = torch.empty((S, MAX_ATOMS), dtype=torch.float64, device=dev)
    q = torch.empty((S, MAX_ATOMS), dtype=torch.float64, device=dev)
    x = torch.empty((S, MAX_ATOMS, 3), dtype=torch.float32, device=dev)
    f = torch.empty(S, dtype=torch.uint8, device=dev)
    cfg = mixed_config(seed, **kw)
    rc = lib.ce_sample_mixed_device(int(first_sim), int(S), C.byref(cfg), _vp(n), _vp(m), _vp(q), _vp(x), _vp(f),
                                    None)
    if rc != 0:
        raise EngineError(rc, "ce_sample_mixed_device failed")
    torch.cuda.synchronize(dev)
    if int(f.sum().item()) != 0:
        raise RuntimeError("sampler rejection budget exhausted")
    return DeviceBatch(n, m, q, x)


def sample_molecule_device(mol, S: int, seed: int, first_sim: int = 0, device: int = 0, stream: int = 0,
                           out: DeviceBatch | None = None) -> DeviceBatch:
    """One molecule (n <= 10 atoms) in the padded mixed layout: positions from
    the device Philox ball sampler, masses/charges repeated per row."""
    from .sampling import ball_config

    torch = _torch()
    lib = load_library()
    dev = torch.device("cuda", device)
    n = mol.n
    if out is None:
        m = torch.ones((S, MAX_ATOMS), dtype=torch.float64, device=dev)
        q = torch.zeros((S, MAX_ATOMS), dtype=torch.float64, device=dev)
        m[:, :n] = torch.from_numpy(mol.masses_me).to(dev)
        q[:, :n] = torch.from_numpy(mol.charge_array).to(dev)
        out = DeviceBatch(torch.full((S,), n, dtype=torch.uint8, device=dev), m, q,
                          torch.zeros((S, MAX_ATOMS, 3), dtype=torch.float32, device=dev))
    if n != MAX_ATOMS:
        raise ValueError("sample_molecule_device fills rows in place only for 10-atom molecules")
    cfg = ball_config(mol, seed)
    rc = lib.ce_sample_ball_device(n, int(first_sim), int(S), C.byref(cfg), _vp(out.pos), None, C.c_void_p(stream))
    if rc != 0:
        raise EngineError(rc, "ce_sample_ball_device failed")
    return out


def run_plain(engine: Engine, batch: DeviceBatch, cfg: RunConfig, stream: int = 0, coulomb_k: float = 1.0) -> dict:
    """Plain RK45 to cfg's stop, device outputs."""
    torch = _torch()
    S, dev = batch.S, batch.n.device
    o = {"momenta": torch.zeros((S, MAX_ATOMS, 3), dtype=torch.float32, device=dev),
         "ker": torch.zeros(S, dtype=torch.float64, device=dev),
         "steps": torch.zeros(S, dtype=torch.int32, device=dev),
         "status": torch.zeros(S, dtype=torch.uint8, device=dev)}
    out = CeOutputs(_vp(o["momenta"]), _vp(o["ker"]), _vp(o["steps"]), _vp(o["status"]))
    engine.run_mixed_device(S, batch.c(), cfg, out, stream=stream, coulomb_k=coulomb_k)
    return o


def run_loose(engine: Engine, batch: DeviceBatch, cfg: RunConfig, loose_pe_stop: float = LOOSE_PE_STOP,
              stream: int = 0, coulomb_k: float = 1.0) -> dict:
    """Integrate to PE <= loose_pe_stop * PE_0 without the energy rescale and
    keep the state there (positions, m v, E_0, PE, status, steps)."""
    torch = _torch()
    S, dev = batch.S, batch.n.device
    lcfg = RunConfig(rtol=cfg.rtol, atol=cfg.atol, pe_stop_fraction=loose_pe_stop, max_dt=cfg.max_dt,
                     max_steps=cfg.max_steps, redistribute_energy=False, precision_mode=cfg.precision_mode)
    o = {"momenta": torch.zeros((S, MAX_ATOMS, 3), dtype=torch.float32, device=dev),
         "positions": torch.zeros((S, MAX_ATOMS, 3), dtype=torch.float32, device=dev),
         "e0": torch.zeros(S, dtype=torch.float64, device=dev),
         "pe_final": torch.zeros(S, dtype=torch.float64, device=dev),
         "steps": torch.zeros(S, dtype=torch.int32, device=dev),
         "status": torch.zeros(S, dtype=torch.uint8, device=dev)}
    out = CeOutputs(_vp(o["momenta"]), None, _vp(o["steps"]), _vp(o["status"]), None, None, _vp(o["pe_final"]),
                    None, _vp(o["positions"]), _vp(o["e0"]))
    engine.run_mixed_device(S, batch.c(), lcfg, out, stream=stream, coulomb_k=coulomb_k)
    return o


def closure_state(loose: dict) -> CeClosureState:
    return CeClosureState(_vp(loose["positions"]), _vp(loose["momenta"]), _vp(loose["e0"]), _vp(loose["pe_final"]),
                          _vp(loose["status"]))


def features(batch: DeviceBatch, loose: dict, p_true=None, weight_scale: float = 1.0, stream: int = 0,
             coulomb_k: float = 1.0) -> dict:
    """ce_closure_features: BF16 features [pad128(S), 128], ballistic base
    [S, 10, 3], scale P [S] and, with p_true, targets/weights [pad128(S), 32]."""
    torch = _torch()
    lib = load_library()
    S, dev = batch.S, batch.n.device
    Sp = pad128(S)
    d = {"feats": torch.empty((Sp, CLOSURE_FEATURES), dtype=torch.bfloat16, device=dev),
         "p_base": torch.empty((S, MAX_ATOMS, 3), dtype=torch.float32, device=dev),
         "p_scale": torch.empty(S, dtype=torch.float32, device=dev)}
    if p_true is not None:
        d["target"] = torch.empty((Sp, CLOSURE_OUTPUTS), dtype=torch.float32, device=dev)
        d["weight"] = torch.empty((Sp, CLOSURE_OUTPUTS), dtype=torch.float32, device=dev)
    st = closure_state(loose)
    rc = lib.ce_closure_features(S, C.byref(batch.c()), float(coulomb_k), C.byref(st), _vp(p_true),
                                 float(weight_scale), _vp(d["feats"]), _vp(d["p_base"]), _vp(d["p_scale"]),
                                 _vp(d.get("target")), _vp(d.get("weight")), C.c_void_p(stream))
    if rc != 0:
        raise EngineError(rc, "ce_closure_features failed")
    return d


def net_forward(net: Network, feats, stream: int = 0):
    """Network output [pad128(S), 32] over rows of feats, chunked by max_batch."""
    torch = _torch()
    Sp = feats.shape[0]
    out = torch.empty((Sp, CLOSURE_OUTPUTS), dtype=torch.float32, device=feats.device)
    chunk = Sp if (net.hidden % 32 == 0 and net.depth + 1 <= 8) else net.max_batch  # fused kernel: one launch
    for a in range(0, Sp, chunk):
        b = min(Sp, a + chunk)
        net.forward(feats[a:b], out[a:b], b - a, stream)
    return out


def gate_stats(batch: DeviceBatch, loose: dict, base: dict, out) -> dict:
    """The gate's three quantities per sim, computed with torch for
    calibration only (the serving gate is ce_closure_apply)."""
    torch = _torch()
    S = batch.S
    n = batch.n.long()
    live = (torch.arange(MAX_ATOMS, device=n.device)[None, :] < n[:, None]).float()
    P = base["p_scale"].double()
    d = out[:S, :3 * MAX_ATOMS].double().view(S, MAX_ATOMS, 3) * P[:, None, None] * live[..., None]
    pb = base["p_base"].double() * live[..., None]
    p = pb + d
    m = torch.where(live > 0, batch.mass, torch.ones_like(batch.mass))
    ke = 0.5 * ((p * p).sum(-1) / m * live).sum(-1)
    rho = (ke / loose["e0"] - 1.0).abs()
    mu = p.sum(1).norm(dim=-1) / (p.norm(dim=-1) * live).sum(-1)
    corr = d.flatten(1).norm(dim=-1) / pb.flatten(1).norm(dim=-1)
    return {"rho": rho, "mu": mu, "corr": corr}


def rel_err(p, p_ref):
    """Config-norm relative error per sim, ||p - p_ref|| / ||p_ref|| over all components."""
    d = (p.double() - p_ref.double()).flatten(1).norm(dim=-1)
    return d / p_ref.double().flatten(1).norm(dim=-1)


def predict(batch: DeviceBatch, base: dict, out) -> object:
    """Corrected momenta p_base + Q * out (before the gate's projection); Q is
    p_scale, the size of the analytic step."""
    S = batch.S
    return base["p_base"] + base["p_scale"][:, None, None] * out[:S, :3 * MAX_ATOMS].view(S, MAX_ATOMS, 3) * (
        (_torch().arange(MAX_ATOMS, device=batch.n.device)[None, :] < batch.n[:, None].long())[..., None])


@dataclass
class TrainingSet:
    feats: object
    target: object
    weight: object
    S: int
    valid: object  # bool [S]: sims the network is trained on


def make_training_set(engine: Engine, batch: DeviceBatch, cfg: RunConfig, loose_pe_stop: float = LOOSE_PE_STOP,
                      minibatch: int = 8192) -> tuple[TrainingSet, dict, dict, dict]:
    """(training set, loose state, base, plain result) for every sim of batch;
    targets are the plain run's converged momenta (cfg), scaled by TARGET_SCALE."""
    loose = run_loose(engine, batch, cfg, loose_pe_stop)
    plain = run_plain(engine, batch, cfg)
    base = features(batch, loose, p_true=plain["momenta"], weight_scale=1.0 / minibatch)
    valid = (base["p_scale"] > 0) & (plain["status"] == 0) & (loose["status"] == 0)
    w = base["weight"]
    w[: batch.S] *= valid[:, None].float()
    base["target"] *= TARGET_SCALE
    ts = TrainingSet(base.pop("feats"), base.pop("target"), base.pop("weight"), batch.S, valid)
    return ts, loose, base, plain


@dataclass
class TrainReport:
    steps: int
    epochs: int
    seconds: float
    losses: list = field(default_factory=list)
    samples_per_s: float = 0.0


def train(net: Network, ts: TrainingSet, epochs: int = 20, minibatch: int = 8192, lr: float = 1e-3,
          lr_final: float = 1e-5, seed: int = 7, train_rows=None) -> TrainReport:
    """Adam with cosine decay over `epochs` passes of a seeded shuffle of the
    training rows; one ce_mlp_train_step per minibatch (no host sync inside)."""
    import time

    torch = _torch()
    dev = ts.feats.device
    rows = train_rows if train_rows is not None else torch.arange(ts.S, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    per_epoch = rows.numel() // minibatch
    total = per_epoch * epochs
    loss_buf = torch.zeros(total, dtype=torch.float32, device=dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    step = 0
    for ep in range(epochs):
        perm = rows[torch.randperm(rows.numel(), generator=g, device=dev)]
        for b in range(per_epoch):
            idx = perm[b * minibatch:(b + 1) * minibatch]
            x = ts.feats.index_select(0, idx)
            t = ts.target.index_select(0, idx)
            w = ts.weight.index_select(0, idx)
            frac = step / max(1, total - 1)
            cur = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * frac))
            net.train_step(x, t, w, minibatch, cur, loss_buf[step:step + 1],
                           torch.cuda.current_stream(dev).cuda_stream)
            step += 1
    net.check(torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize(dev)
    dt = time.perf_counter() - t0
    losses = loss_buf.cpu().numpy()
    return TrainReport(steps=step, epochs=epochs, seconds=dt, losses=losses.tolist(),
                       samples_per_s=step * minibatch / dt if dt > 0 else 0.0)


def calibrate_gate(stats: dict, valid, quantile: float = 0.99) -> CeClosureGate:
    """Bounds at the given quantile of each gate quantity over validation sims."""
    torch = _torch()
    q = []
    for k in ("rho", "mu", "corr"):
        v = stats[k][valid].float()
        q.append(float(torch.quantile(v[: 1 << 24], quantile).item()) if v.numel() else 0.0)
    return CeClosureGate(*q)


def calibrate_gate_for_error(stats: dict, err, valid, target: float, quantile: float = 0.99) -> CeClosureGate:
    """Energy and momentum bounds at `quantile` of the validation sims; the
    correction bound is the largest for which every validation sim that passes
    all three bounds has error <= target (err: per-sim error of the network's
    prediction against converged momenta)."""
    torch = _torch()
    g = calibrate_gate(stats, valid, quantile)
    ok = valid & (stats["rho"] <= g.tol_energy) & (stats["mu"] <= g.tol_momentum)
    c = stats["corr"][ok].double()
    e = err[ok].double()
    if c.numel() == 0:
        return CeClosureGate(g.tol_energy, g.tol_momentum, 0.0)
    order = torch.argsort(c)
    bad = torch.cummax(e[order], dim=0).values > target
    first_bad = int(torch.nonzero(bad)[0].item()) if bool(bad.any()) else c.numel()
    tol_c = float(c[order[first_bad - 1]].item()) if first_bad > 0 else 0.0
    return CeClosureGate(g.tol_energy, g.tol_momentum, tol_c)


class Closure:
    """ce_closure handle: serving pipeline bound to an engine and a network."""

    def __init__(self, engine: Engine, net: Network, max_sims: int):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.ce_closure_create(C.byref(h), engine.h, net.h, int(max_sims))
        if rc != 0:
            raise EngineError(rc, "ce_closure_create failed")
        self.h = h
        self.engine, self.net = engine, net

    def close(self):
        if getattr(self, "h", None):
            self.lib.ce_closure_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def serve(self, batch: DeviceBatch, cfg: RunConfig, gate: CeClosureGate, out: CeOutputs,
              loose_pe_stop: float = LOOSE_PE_STOP, stream: int = 0, coulomb_k: float = 1.0, S: int | None = None,
              cbatch: CeMixedBatch | None = None):
        c = cfg.to_c()
        b = cbatch if cbatch is not None else batch.c()
        rc = self.lib.ce_closure_serve(self.h, int(S if S is not None else batch.S), C.byref(b), float(coulomb_k),
                                       C.byref(c), float(loose_pe_stop), C.byref(gate), C.byref(out),
                                       C.c_void_p(stream))
        if rc != 0:
            raise EngineError(rc, self.lib.ce_closure_last_error(self.h).decode())

    def fallback_flags(self, S: int, stream: int = 0):
        """uint8 tensor [S]: n for each sim the last serve sent back, else 0."""
        torch = _torch()
        out = torch.empty(S, dtype=torch.uint8, device="cuda")
        rc = self.lib.ce_closure_fallback_flags(self.h, _vp(out), int(S), C.c_void_p(stream))
        if rc != 0:
            raise EngineError(rc, "ce_closure_fallback_flags failed")
        return out

    def counts(self) -> tuple[int, int]:
        a, f = C.c_uint64(), C.c_uint64()
        rc = self.lib.ce_closure_counts(self.h, C.byref(a), C.byref(f))
        if rc != 0:
            raise EngineError(rc, self.lib.ce_closure_last_error(self.h).decode())
        return int(a.value), int(f.value)
