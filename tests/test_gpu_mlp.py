"""Tensor-core (tcgen05) GEMM and closure-network kernels against the numpy
oracle (oracle/mlp_oracle.py).

GEMM: every operand-major combination, ragged K (zero-padded slices), N from
16 to 256 and split-K, against float64 products of the same bfloat16 inputs:
rel. error <= 1e-5 (FP32 accumulation order only).
Network: loss and gradients against the oracle with bfloat16 rounding at the
kernels' rounding points: rel. error of each parameter tensor's gradient
<= 2e-2 (bfloat16 rounding of activations can flip at ties); forward output
<= 1e-2 relative to its norm; a few Adam steps reduce the loss.
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, str(ROOT / "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu


def bf16_tensor(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).cuda()


@pytest.mark.parametrize("a_mn,b_mn", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (256, 96, 96), (384, 256, 256), (256, 32, 1040), (128, 512, 200)])
def test_umma_gemm_matches_float64(ce, a_mn, b_mn, M, N, K):
    torch = pytest.importorskip("torch")
    lib = ce.load_library()
    rng = np.random.default_rng(M * 7 + N * 3 + K + a_mn * 2 + b_mn)
    A = mo.to_bf16(rng.standard_normal((M, K)))
    B = mo.to_bf16(rng.standard_normal((N, K)))
    a_dev = bf16_tensor(torch, A.T if a_mn else A)
    b_dev = bf16_tensor(torch, B.T if b_mn else B)
    c = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.ce_umma_gemm_f32(a_dev.data_ptr(), a_mn, b_dev.data_ptr(), b_mn, M, N, K, c.data_ptr(), err.data_ptr(),
                              None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A @ B.T
    got = c.cpu().numpy().astype(np.float64)
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max() + 1e-6


def make_net(ce, in_dim=96, hidden=64, depth=2, out_dim=32, batch=256, seed=5):
    lib = ce.load_library()
    h = C.c_void_p()
    assert lib.ce_mlp_create(C.byref(h), 0, in_dim, hidden, depth, out_dim, batch, seed) == 0
    return lib, h


def test_network_gradients_match_oracle(ce):
    torch = pytest.importorskip("torch")
    in_dim, hidden, depth, out_dim, B = 96, 64, 2, 32, 256
    lib, h = make_net(ce, in_dim, hidden, depth, out_dim, B)
    try:
        P = int(lib.ce_mlp_param_count(h))
        params = np.zeros(P, np.float32)
        assert lib.ce_mlp_get_params(h, params.ctypes.data) == 0
        rng = np.random.default_rng(3)
        params += rng.standard_normal(P).astype(np.float32) * 0.01  # non-zero biases too
        assert lib.ce_mlp_set_params(h, params.ctypes.data) == 0
        x = mo.to_bf16(rng.standard_normal((B, in_dim)))
        t = rng.standard_normal((B, out_dim)).astype(np.float32)
        w = (rng.random((B, out_dim)) < 0.9).astype(np.float32)
        w /= w.sum()
        xd = bf16_tensor(torch, x)
        td = torch.from_numpy(t).cuda()
        wd = torch.from_numpy(w).cuda()
        loss = C.c_float(0)
        g = np.zeros(P, np.float32)
        assert lib.ce_mlp_gradients(h, xd.data_ptr(), td.data_ptr(), wd.data_ptr(), B, C.byref(loss), g.ctypes.data,
                                    None) == 0, lib.ce_mlp_last_error(h)
        ref_loss, ref_g = mo.gradients(params, x, t, w, in_dim, hidden, depth, out_dim, bf16=True)
        assert abs(loss.value - ref_loss) <= 1e-2 * ref_loss
        ws, bs = mo.unpack(np.arange(P), in_dim, hidden, depth, out_dim)
        for tensor in list(ws) + list(bs):
            idx = tensor.ravel().astype(np.int64)
            num = np.linalg.norm(g[idx] - ref_g[idx])
            assert num <= 2e-2 * np.linalg.norm(ref_g[idx]) + 1e-9, (idx[:3], num, np.linalg.norm(ref_g[idx]))
        out = torch.zeros((B, out_dim), dtype=torch.float32, device="cuda")
        assert lib.ce_mlp_forward(h, xd.data_ptr(), B, out.data_ptr(), None) == 0
        torch.cuda.synchronize()
        ref_out, _, _ = mo.forward(params, x, in_dim, hidden, depth, out_dim, bf16=True)
        assert np.linalg.norm(out.cpu().numpy() - ref_out) <= 1e-2 * np.linalg.norm(ref_out)
        # Adam steps reduce the loss on a fixed batch
        first = loss.value
        for _ in range(30):
            assert lib.ce_mlp_train_step(h, xd.data_ptr(), td.data_ptr(), wd.data_ptr(), B, 3e-3, None, None) == 0
        assert lib.ce_mlp_check(h, None) == 0
        assert lib.ce_mlp_gradients(h, xd.data_ptr(), td.data_ptr(), wd.data_ptr(), B, C.byref(loss), None,
                                    None) == 0
        assert loss.value < 0.8 * first
    finally:
        lib.ce_mlp_destroy(h)


def test_fused_forward_equals_layered_forward(ce):
    """The serving network (128 -> 4 x 256 -> 32) through the fused persistent
    kernel over 301 row tiles (more than one pass of the grid, and an odd tile
    count, so the last pair holds a single tile) equals the training path's
    per-layer forward bit for bit, and the oracle within 1e-2."""
    torch = pytest.importorskip("torch")
    in_dim, hidden, depth, out_dim, B = 128, 256, 4, 32, 128 * 301
    lib, h = make_net(ce, in_dim, hidden, depth, out_dim, B, seed=11)
    try:
        P = int(lib.ce_mlp_param_count(h))
        params = np.zeros(P, np.float32)
        assert lib.ce_mlp_get_params(h, params.ctypes.data) == 0
        rng = np.random.default_rng(8)
        params += rng.standard_normal(P).astype(np.float32) * 0.02
        assert lib.ce_mlp_set_params(h, params.ctypes.data) == 0
        x = mo.to_bf16(rng.standard_normal((B, in_dim)))
        xd = bf16_tensor(torch, x)
        fused = torch.full((B, out_dim), float("nan"), dtype=torch.float32, device="cuda")
        layered = torch.zeros((B, out_dim), dtype=torch.float32, device="cuda")
        for _ in range(2):  # a second call reuses the same kernel state
            assert lib.ce_mlp_forward(h, xd.data_ptr(), B, fused.data_ptr(), None) == 0, lib.ce_mlp_last_error(h)
        assert lib.ce_mlp_forward_layered(h, xd.data_ptr(), B, layered.data_ptr(), None) == 0
        assert lib.ce_mlp_check(h, None) == 0
        torch.cuda.synchronize()
        assert torch.equal(fused, layered)
        ref, _, _ = mo.forward(params, x[:512], in_dim, hidden, depth, out_dim, bf16=True)
        got = fused[:512].cpu().numpy()
        assert np.linalg.norm(got - ref) <= 1e-2 * np.linalg.norm(ref)
    finally:
        lib.ce_mlp_destroy(h)


def test_forward_limits(ce):
    torch = pytest.importorskip("torch")
    # a width that is not a multiple of 32 takes the per-layer path, bounded by max_batch
    lib, h = make_net(ce, 96, 48, 2, 32, 256)
    try:
        x = torch.zeros((512, 96), dtype=torch.bfloat16, device="cuda")
        out = torch.zeros((512, 32), dtype=torch.float32, device="cuda")
        assert lib.ce_mlp_forward(h, x.data_ptr(), 256, out.data_ptr(), None) == 0
        assert lib.ce_mlp_forward(h, x.data_ptr(), 512, out.data_ptr(), None) == ce.CE_ERR_INVALID
        assert lib.ce_mlp_forward(h, x.data_ptr(), 100, out.data_ptr(), None) == ce.CE_ERR_INVALID
        assert lib.ce_mlp_check(h, None) == 0
    finally:
        lib.ce_mlp_destroy(h)


def test_bounded_wait_gives_up_and_context_survives(ce, engine, wl):
    """Failure detection of the tensor-core kernels: a wait on an mbarrier that
    nothing arrives on gives up after its poll budget, records its code, and the
    context keeps working (a plain integration runs afterwards)."""
    import time

    lib = ce.load_library()
    code = C.c_int(-1)
    timings = {}
    for spins in (1000, 20000):
        t0 = time.perf_counter()
        assert lib.ce_probe_bounded_wait(0, spins, C.byref(code)) == 0
        timings[spins] = time.perf_counter() - t0
        assert code.value == 7
    print(f"bounded wait: 1000 polls {timings[1000] * 1e3:.2f} ms, 20000 polls {timings[20000] * 1e3:.2f} ms")
    assert lib.ce_probe_bounded_wait(0, 0, C.byref(code)) == ce.CE_ERR_INVALID
    mol = wl.CH4
    engine.set_molecule(mol.masses_me, mol.charge_array)
    pos = wl.sample_molecule(mol, 64, seed=4).astype(np.float32)
    r = engine.run(pos, ce.RunConfig(rtol=1e-6, atol=1e-7, pe_stop_fraction=1e-7))
    assert np.all(r.status == 0)
