"""Geometry sampler (include/ce_sampler.h): Philox4x32-10 known answers, the
ball / minimum-separation contract (the reference's tests/test_sampler.cpp:40-117
checks the same properties of its own sampler), chunk independence, the mixed
population's ranges, and (GPU) device == host bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from pkg_loader import load_submodule

sp = load_submodule("sampling")


def test_philox_known_answer_vectors():
    # Salmon et al. (SC 2011), Random123 known-answer vectors for Philox4x32-10.
    assert sp.philox((0, 0, 0, 0), (0, 0)) == (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)
    f = 0xFFFFFFFF
    assert sp.philox((f, f, f, f), (f, f)) == (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)
    assert sp.philox((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0)) == (
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)


def test_ball_contract_and_determinism(wl):
    mol = wl.CH4
    pos, pos64, flags = sp.sample_ball_host(mol, 4000, seed=7)
    assert not flags.any()
    r = np.linalg.norm(pos64, axis=2)
    assert (r <= mol.radius).all()
    d = np.linalg.norm(pos64[:, :, None] - pos64[:, None], axis=-1) + np.eye(mol.n) * 1e9
    assert d.min() >= mol.min_sep
    np.testing.assert_array_equal(pos, pos64.astype(np.float32))
    again, _, _ = sp.sample_ball_host(mol, 4000, seed=7)
    np.testing.assert_array_equal(pos, again)
    other, _, _ = sp.sample_ball_host(mol, 4000, seed=8)
    assert not np.array_equal(pos, other)
    # uniform in the ball: mean radius of a uniform ball is 3R/4
    assert abs(r.mean() - 0.75 * mol.radius) < 0.02 * mol.radius


def test_chunks_are_independent(wl):
    mol = wl.C2H6_LIKE
    whole, _, _ = sp.sample_ball_host(mol, 300, seed=11)
    a, _, _ = sp.sample_ball_host(mol, 120, seed=11, first_sim=0)
    b, _, _ = sp.sample_ball_host(mol, 180, seed=11, first_sim=120)
    np.testing.assert_array_equal(whole, np.concatenate([a, b]))


def test_mixed_population_ranges(wl):
    n, m, q, pos, pos64, flags = sp.sample_mixed_host(6000, seed=5)
    assert not flags.any()
    assert n.min() == 2 and n.max() == 10
    counts = np.bincount(n, minlength=11)[2:]
    assert counts.min() > 0.8 * counts.mean()
    amu = m / wl.AMU_TO_ME
    species = {round(v, 3) for v in wl.SPECIES_AMU.values()}
    for s in range(len(n)):
        k = int(n[s])
        assert {round(v, 3) for v in amu[s, :k]} <= species
        assert set(q[s, :k]) <= {1.0, 2.0, 3.0} and not q[s, k:].any() and (m[s, k:] == 1.0).all()
        rad = 2.0 * k ** (1 / 3)
        assert (np.linalg.norm(pos64[s, :k], axis=1) <= rad).all() and not pos64[s, k:].any()
        if k > 1:
            d = np.linalg.norm(pos64[s, :k, None] - pos64[s, None, :k], axis=-1) + np.eye(k) * 1e9
            assert d.min() >= 0.5


def test_invalid_sampler_configs_are_rejected(ce, wl):
    import ctypes as C

    lib = ce.load_library()
    pos = np.zeros((4, 5, 3), np.float32)
    bad = ce.CeBallSampler(1, -1.0, 0.5, 0)
    assert lib.ce_sample_ball_host(5, 0, 4, C.byref(bad), C.c_void_p(pos.ctypes.data), None, None) == ce.CE_ERR_INVALID
    bad = ce.CeBallSampler(1, 3.3, -0.5, 0)
    assert lib.ce_sample_ball_host(5, 0, 4, C.byref(bad), C.c_void_p(pos.ctypes.data), None, None) == ce.CE_ERR_INVALID
    # infeasible packing is flagged, not looped forever (max_attempts bound)
    tight = ce.CeBallSampler(1, 0.5, 0.9, 20)
    flags = np.zeros(4, np.uint8)
    assert lib.ce_sample_ball_host(5, 0, 4, C.byref(tight), C.c_void_p(pos.ctypes.data), None,
                                   C.c_void_p(flags.ctypes.data)) == ce.CE_OK
    assert flags.all()


@pytest.mark.gpu
def test_device_sampler_equals_host_twin(ce, wl):
    torch = pytest.importorskip("torch")
    import ctypes as C

    lib = ce.load_library()
    mol = wl.CH4
    S = 20000
    host, _, _ = sp.sample_ball_host(mol, S, seed=21, first_sim=1000)
    dev = torch.zeros((S, mol.n, 3), dtype=torch.float32, device="cuda")
    cfg = sp.ball_config(mol, 21)
    assert lib.ce_sample_ball_device(mol.n, 1000, S, C.byref(cfg), C.c_void_p(dev.data_ptr()), None, None) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dev.cpu().numpy(), host)

    n, m, q, pos, _, _ = sp.sample_mixed_host(S, seed=22)
    dn = torch.zeros(S, dtype=torch.uint8, device="cuda")
    dm = torch.zeros((S, 10), dtype=torch.float64, device="cuda")
    dq = torch.zeros((S, 10), dtype=torch.float64, device="cuda")
    dx = torch.zeros((S, 10, 3), dtype=torch.float32, device="cuda")
    mc = sp.mixed_config(22)
    assert lib.ce_sample_mixed_device(0, S, C.byref(mc), C.c_void_p(dn.data_ptr()), C.c_void_p(dm.data_ptr()),
                                      C.c_void_p(dq.data_ptr()), C.c_void_p(dx.data_ptr()), None, None) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dn.cpu().numpy(), n)
    np.testing.assert_array_equal(dm.cpu().numpy(), m)
    np.testing.assert_array_equal(dq.cpu().numpy(), q)
    np.testing.assert_array_equal(dx.cpu().numpy(), pos)
