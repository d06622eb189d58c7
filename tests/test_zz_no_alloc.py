"""ce_run_device_noalloc: the integration entry point for callers that cannot
allocate device memory (a framework that owns every device allocation, a
memory-budgeted serving process, a host with a fixed arena). They pass their own
input and output buffers; the kernel's work-queue cursor lives in a static device
array inside the library.

The test calls it through the C ABI twice in a row and checks both outputs
against the engine's ordinary ce_run_device on the same inputs, with the parity
tolerance the other GPU tests use (1e-5 config-norm relative momentum error; the
kernel is the same, so the results are expected to be identical). This file is
named so that pytest collects it last, and it needs no state from other tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _device_buffers(torch, S, n):
    return dict(
        momenta=torch.zeros((S, n, 3), dtype=torch.float32, device="cuda"),
        ker=torch.zeros(S, dtype=torch.float64, device="cuda"),
        steps=torch.zeros(S, dtype=torch.int32, device="cuda"),
        status=torch.full((S,), 255, dtype=torch.uint8, device="cuda"),
    )


def _outputs(ce, b):
    return ce.CeOutputs(b["momenta"].data_ptr(), b["ker"].data_ptr(), b["steps"].data_ptr(),
                        b["status"].data_ptr(), None, None, None, None)


@pytest.mark.parametrize("case", ["ch4_full_precision", "c2h6_fp32"])
def test_noalloc_entry_point_matches_ce_run_device(ce, wl, case):
    # CH4 in the full precision form runs one thread per sim, the 10-atom
    # C2H6-like molecule in plain FP32 two threads per sim.
    torch = pytest.importorskip("torch")
    lib = ce.load_library()
    mol, mode = {"ch4_full_precision": (wl.CH4, 3), "c2h6_fp32": (wl.C2H6_LIKE, 0)}[case]
    S = 20_000
    pos = torch.from_numpy(wl.sample_molecule(mol, S, seed=99).astype(np.float32)).cuda()
    cfg = ce.RunConfig(rtol=wl.TIGHT[0], atol=wl.TIGHT[1], pe_stop_fraction=wl.TIGHT[2], precision_mode=mode)

    # Ordinary path: engine-owned scratch, default launch shape (the layout the
    # allocation-free entry point launches too).
    eng = ce.Engine(0)
    eng.set_molecule(mol.masses_me, mol.charge_array)
    ref = _device_buffers(torch, S, mol.n)
    stream = torch.cuda.current_stream().cuda_stream
    eng.run_device(S, pos.data_ptr(), cfg, _outputs(ce, ref), stream)
    torch.cuda.synchronize()
    eng.close()

    m = np.ascontiguousarray(mol.masses_me, dtype=np.float64)
    q = np.ascontiguousarray(mol.charge_array, dtype=np.float64)
    c = cfg.to_c()
    err = C.create_string_buffer(256)
    for call in range(2):  # two calls in a row share (and reuse) the static scratch
        got = _device_buffers(torch, S, mol.n)
        rc = lib.ce_run_device_noalloc(mol.n, m.ctypes.data, q.ctypes.data, 1.0, S, pos.data_ptr(), C.byref(c),
                                       C.byref(_outputs(ce, got)), stream, err, len(err))
        assert rc == ce.CE_OK, err.value.decode()
        torch.cuda.synchronize()
        e = ol.config_norm_error(got["momenta"].cpu().numpy(), ref["momenta"].cpu().numpy())
        assert e.max() <= TOL, (call, e.max())
        np.testing.assert_array_equal(got["steps"].cpu().numpy(), ref["steps"].cpu().numpy())
        np.testing.assert_array_equal(got["status"].cpu().numpy(), ref["status"].cpu().numpy())
        np.testing.assert_allclose(got["ker"].cpu().numpy(), ref["ker"].cpu().numpy(), rtol=TOL)

    # The same two calls on a side stream (not torch's current stream), ordered by
    # that stream alone: the cursor is cleared on the caller's stream, so stream
    # order is all a caller needs to serialise calls.
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    outs = []
    with torch.cuda.stream(side):
        for call in range(2):
            got = _device_buffers(torch, S, mol.n)
            rc = lib.ce_run_device_noalloc(mol.n, m.ctypes.data, q.ctypes.data, 1.0, S, pos.data_ptr(), C.byref(c),
                                           C.byref(_outputs(ce, got)), side.cuda_stream, err, len(err))
            assert rc == ce.CE_OK, err.value.decode()
            outs.append(got)
    side.synchronize()
    for call, got in enumerate(outs):
        e = ol.config_norm_error(got["momenta"].cpu().numpy(), ref["momenta"].cpu().numpy())
        assert e.max() <= TOL, ("side stream", call, e.max())
        np.testing.assert_array_equal(got["steps"].cpu().numpy(), ref["steps"].cpu().numpy())
        np.testing.assert_array_equal(got["status"].cpu().numpy(), ref["status"].cpu().numpy())

    # Sizes beyond the supported maximum are rejected before any launch.
    rc = lib.ce_run_device_noalloc(11, m.ctypes.data, q.ctypes.data, 1.0, S, pos.data_ptr(), C.byref(c),
                                   C.byref(_outputs(ce, ref)), stream, err, len(err))
    assert rc == ce.CE_ERR_INVALID and b"1..10" in err.value
    rc = lib.ce_run_device_noalloc(mol.n, m.ctypes.data, q.ctypes.data, 1.0, (1 << 40) + 1, pos.data_ptr(),
                                   C.byref(c), C.byref(_outputs(ce, ref)), stream, err, len(err))
    assert rc == ce.CE_ERR_INVALID and b"2^40" in err.value
