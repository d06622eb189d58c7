"""Learned closure (include/ce_closure.h) on the GPU.

* features and ballistic base against the float64 oracle
  (oracle/closure_oracle.py): base within 3e-5 relative (FP32 pair sums), the
  output scale Q within 2e-4, features within one BF16 rounding step;
* gate and projection against the oracle on a random network output;
* serving: a gate that accepts nothing reproduces plain RK45 bit for bit, a
  gate that accepts everything leaves no sim behind, one-atom and invalid
  sims pass through;
* training: a network trained on the GPU by the library's own kernels beats
  both the analytic ballistic base and the reference's redistribution-only
  closure (src/driver.cpp:38-42) on held-out sims at the same loose stop.
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np
import pytest

from conftest import ROOT
from pkg_loader import load_submodule

sys.path.insert(0, str(ROOT / "oracle"))
import closure_oracle as co  # noqa: E402

pytestmark = pytest.mark.gpu

TIGHT = (1e-6, 1e-7, 1e-7)


@pytest.fixture(scope="module")
def cl():
    pytest.importorskip("torch")
    return load_submodule("closure")


def _cfg(ce):
    r, a, p = TIGHT
    return ce.RunConfig(rtol=r, atol=a, pe_stop_fraction=p)


def _np(t):
    return t.detach().cpu().numpy()


def test_features_match_oracle(ce, engine, cl):
    torch = pytest.importorskip("torch")
    b = cl.sample_mixed_device(600, seed=11, first_sim=1000)
    loose = cl.run_loose(engine, b, _cfg(ce))
    plain = cl.run_plain(engine, b, _cfg(ce))
    d = cl.features(b, loose, p_true=plain["momenta"], weight_scale=0.5)
    torch.cuda.synchronize()
    ok = (_np(loose["status"]) == 0) & (_np(b.n) >= 2)
    assert ok.mean() > 0.98
    n, m, q = _np(b.n)[ok], _np(b.mass)[ok], _np(b.charge)[ok]
    x, p = _np(loose["positions"])[ok], _np(loose["momenta"])[ok]
    e0, pef = _np(loose["e0"])[ok], _np(loose["pe_final"])[ok]
    f_ref, pb_ref, Q_ref = co.features(n, m, q, x, p, e0, pef)
    Q = _np(d["p_scale"])[ok]
    np.testing.assert_allclose(Q, Q_ref, rtol=2e-4)
    pb = _np(d["p_base"])[ok]
    err = np.linalg.norm((pb - pb_ref).reshape(len(n), -1), axis=1) / np.linalg.norm(pb_ref.reshape(len(n), -1), axis=1)
    assert err.max() < 3e-5
    f = _np(d["feats"].float())[: len(ok)][ok]
    tol = np.abs(f_ref) * 2.0 ** -7 + 1e-6
    assert np.all(np.abs(f - f_ref) <= tol)
    # padded rows of the feature matrix are zero
    assert float(d["feats"][600:].float().abs().sum()) == 0.0
    # training targets and relative weights (targets inherit the FP32 base error)
    t_ref, w_ref = co.targets(n, pb_ref, Q_ref, _np(plain["momenta"])[ok].astype(np.float64), 0.5)
    t = _np(d["target"])[:600][ok]
    w = _np(d["weight"])[:600][ok]
    P_ref = np.sqrt((pb_ref ** 2).sum(axis=(1, 2)) / n)
    assert np.all(np.abs(t - t_ref).max(axis=1) < 3e-5 * P_ref / Q_ref)
    np.testing.assert_allclose(w, w_ref, rtol=0.15, atol=0)
    assert float(d["weight"][600:].abs().sum()) == 0.0
    # loose stop: remaining PE at most 5% (and not far below) of PE_0
    frac = pef / e0
    assert np.all(frac <= 0.05 + 1e-6) and np.median(frac) > 0.03


def test_gate_and_projection_match_oracle(ce, engine, cl):
    torch = pytest.importorskip("torch")
    lib = ce.load_library()
    b = cl.sample_mixed_device(512, seed=12, first_sim=5000)
    loose = cl.run_loose(engine, b, _cfg(ce))
    d = cl.features(b, loose)
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    # corrections of ~2e-3 of the base momenta (the output is in units of Q)
    P = torch.sqrt((d["p_base"].double() ** 2).sum(dim=(1, 2)) / b.n.double().clamp(min=1))
    ratio = torch.nan_to_num(P / d["p_scale"].double(), nan=0.0, posinf=0.0).float()
    out = torch.randn((512, 32), generator=g, device="cuda") * 2e-3 * ratio[:, None]
    out[::2] *= 0.1  # even rows pass the bounds below, odd rows mostly fail them
    gate = ce.CeClosureGate(1e-3, 1e-3, 3e-3)
    mom = torch.full((512, 10, 3), -7.0, device="cuda")
    ker = torch.zeros(512, dtype=torch.float64, device="cuda")
    steps = torch.zeros(512, dtype=torch.int32, device="cuda")
    status = torch.full((512,), 99, dtype=torch.uint8, device="cuda")
    fb = torch.zeros(512, dtype=torch.uint8, device="cuda")
    counts = torch.zeros(2, dtype=torch.int64, device="cuda")
    o = ce.CeOutputs(mom.data_ptr(), ker.data_ptr(), steps.data_ptr(), status.data_ptr())
    st = cl.closure_state(loose)
    rc = lib.ce_closure_apply(512, C.byref(b.c()), C.byref(st), C.c_void_p(loose["steps"].data_ptr()),
                              C.c_void_p(d["p_base"].data_ptr()), C.c_void_p(d["p_scale"].data_ptr()),
                              C.c_void_p(out.data_ptr()), C.byref(gate), C.byref(o), C.c_void_p(fb.data_ptr()),
                              C.c_void_p(counts.data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize()
    n = _np(b.n)
    ok = (_np(loose["status"]) == 0) & (n >= 2)
    acc, mom_ref, rho, mu, corr = co.apply_gate(n, _np(b.mass), _np(loose["e0"]), _np(d["p_base"]).astype(np.float64),
                                                _np(d["p_scale"]).astype(np.float64), _np(out).astype(np.float64),
                                                gate.tol_energy, gate.tol_momentum, gate.tol_correction)
    acc_gpu = _np(status) == 0
    fbn = _np(fb)
    assert np.all(acc_gpu[ok] == (fbn[ok] == 0))
    # decisions agree away from the boundaries
    margin = (np.abs(rho / gate.tol_energy - 1) > 1e-3) & (np.abs(mu / gate.tol_momentum - 1) > 1e-3) & (
        np.abs(corr / gate.tol_correction - 1) > 1e-3)
    sel = ok & margin
    assert np.array_equal(acc_gpu[sel], acc[sel])
    assert 0.05 < acc[ok].mean() < 0.95  # the random output exercises both branches
    both = ok & acc & acc_gpu
    e = np.linalg.norm((_np(mom)[both] - mom_ref[both]).reshape(both.sum(), -1), axis=1) / np.linalg.norm(
        mom_ref[both].reshape(both.sum(), -1), axis=1)
    assert e.max() < 1e-5
    # accepted sims: zero net momentum, KER = E_0
    np.testing.assert_allclose(_np(ker)[both], _np(loose["e0"])[both], rtol=1e-6)
    net = np.abs(_np(mom)[both].sum(1)).max(axis=1) / np.abs(_np(mom)[both]).max(axis=(1, 2))
    assert net.max() < 1e-5
    # rejected sims keep their outputs untouched and carry n
    rej = ok & ~acc_gpu
    assert np.all(_np(mom)[rej] == -7.0) and np.all(fbn[rej] == n[rej])
    c = _np(counts)
    assert c[0] == acc_gpu[ok].sum() and c[1] == rej.sum()


def _serve(ce, cl, engine, net, b, gate):
    torch = pytest.importorskip("torch")
    S = b.S
    clo = cl.Closure(engine, net, S)
    mom = torch.zeros((S, 10, 3), device="cuda")
    ker = torch.zeros(S, dtype=torch.float64, device="cuda")
    steps = torch.zeros(S, dtype=torch.int32, device="cuda")
    status = torch.zeros(S, dtype=torch.uint8, device="cuda")
    o = ce.CeOutputs(mom.data_ptr(), ker.data_ptr(), steps.data_ptr(), status.data_ptr())
    clo.serve(b, _cfg(ce), gate, o)
    acc, fb = clo.counts()
    clo.close()
    return {"momenta": mom, "ker": ker, "steps": steps, "status": status}, acc, fb


def test_serve_reject_all_equals_plain_and_accept_all(ce, engine, cl):
    torch = pytest.importorskip("torch")
    b = cl.sample_mixed_device(4000, seed=13, first_sim=9000)
    # plant one-atom and invalid sims
    b.n[5] = 1
    b.n[6] = 0
    b.n[7] = 11
    plain = cl.run_plain(engine, b, _cfg(ce))
    net = cl.Network(max_batch=2048, seed=5)
    out, acc, fb = _serve(ce, cl, engine, net, b, ce.CeClosureGate(0.0, 0.0, 0.0))
    torch.cuda.synchronize()
    assert acc == 0 and fb == 4000 - 3
    assert torch.equal(out["momenta"], plain["momenta"])
    assert torch.equal(out["ker"], plain["ker"]) and torch.equal(out["status"], plain["status"])
    assert torch.equal(out["steps"], plain["steps"])
    inf = float("inf")
    out2, acc2, fb2 = _serve(ce, cl, engine, net, b, ce.CeClosureGate(inf, inf, inf))
    st = _np(out2["status"])
    assert fb2 == 0 and acc2 == 4000 - 3
    assert st[5] == 0 and st[6] == ce.CE_SIM_BAD_INPUT and st[7] == ce.CE_SIM_BAD_INPUT
    assert float(out2["momenta"][5:8].abs().sum()) == 0.0
    # accepted sims: energy exact, fewer steps than plain
    ok = st == 0
    ok[5] = False
    np.testing.assert_allclose(_np(out2["ker"])[ok], _np(plain["ker"])[ok], rtol=1e-5)
    assert _np(out2["steps"])[ok].mean() < 0.75 * _np(plain["steps"])[ok].mean()
    # the serving pipeline equals the step-by-step public calls bit for bit
    loose = cl.run_loose(engine, b, _cfg(ce))
    d = cl.features(b, loose)
    o_net = cl.net_forward(net, d["feats"])
    mom = torch.zeros((b.S, 10, 3), device="cuda")
    fbf = torch.zeros(b.S, dtype=torch.uint8, device="cuda")
    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    o = ce.CeOutputs(mom.data_ptr())
    lib = ce.load_library()
    gate = ce.CeClosureGate(inf, inf, inf)
    assert lib.ce_closure_apply(b.S, C.byref(b.c()), C.byref(cl.closure_state(loose)),
                                C.c_void_p(loose["steps"].data_ptr()), C.c_void_p(d["p_base"].data_ptr()),
                                C.c_void_p(d["p_scale"].data_ptr()), C.c_void_p(o_net.data_ptr()), C.byref(gate),
                                C.byref(o), C.c_void_p(fbf.data_ptr()), C.c_void_p(cnt.data_ptr()), None) == 0
    torch.cuda.synchronize()
    assert torch.equal(mom[torch.from_numpy(ok).cuda()], out2["momenta"][torch.from_numpy(ok).cuda()])


def test_trained_network_beats_analytic_and_redistribution(ce, engine, cl):
    torch = pytest.importorskip("torch")
    lib = ce.load_library()
    S_train, S_val, mb = 262_144, 16_384, 4096
    train_b = cl.sample_mixed_device(S_train, seed=21)
    ts, _, _, _ = cl.make_training_set(engine, train_b, _cfg(ce), minibatch=mb)
    net = cl.Network(max_batch=mb, seed=9)
    rep = cl.train(net, ts, epochs=20, minibatch=mb, lr=1e-3, lr_final=1e-5, seed=4)
    net.scale_output_layer(1.0 / cl.TARGET_SCALE)
    losses = np.array(rep.losses)
    print(f"training: {rep.steps} steps in {rep.seconds:.2f} s, loss {losses[:20].mean():.3e} -> "
          f"{losses[-50:].mean():.3e}")
    assert np.isfinite(losses).all() and losses[-50:].mean() < 0.7 * losses[:20].mean()

    val_b = cl.sample_mixed_device(S_val, seed=21, first_sim=10_000_000)
    loose = cl.run_loose(engine, val_b, _cfg(ce))
    plain = cl.run_plain(engine, val_b, _cfg(ce))
    d = cl.features(val_b, loose)
    out = cl.net_forward(net, d["feats"])
    zero = torch.zeros_like(out)
    st = cl.closure_state(loose)
    inf = float("inf")
    gate = ce.CeClosureGate(inf, inf, inf)

    def apply(o_net):
        mom = torch.zeros((S_val, 10, 3), device="cuda")
        status = torch.full((S_val,), 99, dtype=torch.uint8, device="cuda")
        fb = torch.zeros(S_val, dtype=torch.uint8, device="cuda")
        counts = torch.zeros(2, dtype=torch.int64, device="cuda")
        o = ce.CeOutputs(mom.data_ptr(), None, None, status.data_ptr())
        rc = lib.ce_closure_apply(S_val, C.byref(val_b.c()), C.byref(st), C.c_void_p(loose["steps"].data_ptr()),
                                  C.c_void_p(d["p_base"].data_ptr()), C.c_void_p(d["p_scale"].data_ptr()),
                                  C.c_void_p(o_net.data_ptr()), C.byref(gate), C.byref(o), C.c_void_p(fb.data_ptr()),
                                  C.c_void_p(counts.data_ptr()), None)
        assert rc == 0
        return mom, status

    mom_net, s1 = apply(out)
    mom_ana, s2 = apply(zero)
    # redistribution only: the loose state's momenta rescaled to KE = E_0
    p = loose["momenta"].double()
    live = (torch.arange(10, device="cuda")[None, :] < val_b.n[:, None].long()).double()
    m = torch.where(live > 0, val_b.mass, torch.ones_like(val_b.mass))
    ke = 0.5 * ((p * p).sum(-1) / m * live).sum(-1)
    mom_red = p * torch.sqrt(loose["e0"] / ke)[:, None, None]
    ok = (s1 == 0) & (s2 == 0) & (plain["status"] == 0) & (val_b.n >= 2)
    e_net = cl.rel_err(mom_net[ok], plain["momenta"][ok])
    e_ana = cl.rel_err(mom_ana[ok], plain["momenta"][ok])
    e_red = cl.rel_err(mom_red[ok], plain["momenta"][ok])
    med = [float(torch.median(e)) for e in (e_net, e_ana, e_red)]
    p99 = [float(torch.quantile(e.float(), 0.99)) for e in (e_net, e_ana, e_red)]
    print(f"median rel err: network {med[0]:.2e}  analytic {med[1]:.2e}  redistribution {med[2]:.2e}; "
          f"p99 {p99[0]:.2e} {p99[1]:.2e} {p99[2]:.2e}")
    assert med[1] < 0.2 * med[2]
    assert med[0] < 0.75 * med[1] and p99[0] < p99[1]
