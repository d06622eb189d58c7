"""The reference's SIMD batched engine, built here, checked before it is trusted (CPU only).

`BatchedRK45<T>` (include/coulomb/batched_integrator.hpp, unmodified) is compiled
against the project's Highway-API shim (oracle/hwy_shim/) into
oracle/_ref/libref_batched_<isa>.so. It is the timed CPU baseline and a second
parity oracle, so the shim must reproduce the engine the reference measured:

1. The reference's own correctness gate (bench/bench_batched_integrator.cpp:101-126):
   BatchedRK45<double> vs the scalar run_to_convergence on the same geometries,
   config-norm max |dP|/|P| < max(50 rtol, 1e-6) at rtol 1e-8 / atol 1e-16 with the
   default RunConfig, every lane converged; its molecule (N atoms cycling H, C, N,
   O, q = +1, :48-62) and sampler (r 4.0, min 0.25, :64-69).
2. The same gate for the production path BatchedRK45<float> vs the scalar f32
   engine, at the reference production point and the <= 1e-5 point, for CH4 and
   N = 10.
3. At the <= 1e-5 point the f32 batched engine is within 1e-5 of the FP64
   reference on every sim.
4. Lockstep semantics: a lane's result depends only on the set of lanes in its
   batch (shared dt = the worst active lane), so padding a partial batch with
   copies of its own lanes leaves the real lanes' results bit-identical.
5. Both ISA builds (K = 8 with AVX2, K = 16 with AVX-512) pass, where the host
   runs them.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.skipif(not (ol.batched_available() and ol.ref_available()),
                                reason="reference engines (oracle/_ref) not built, or no AVX2/AVX-512")

AMU = 1822.888486209


def cycle_molecule(n):
    """bench_batched_integrator.cpp:48-62: atoms cycling H, C, N, O, all q = +1."""
    amu = [1.008, 12.011, 14.007, 15.999]
    return np.array([amu[i % 4] * AMU for i in range(n)]), np.ones(n)


def ref_pool(n, count, seed):
    """The reference's UniformSphereSampler (r 4.0, min 0.25), bench_batched_integrator.cpp:64-69."""
    pos = np.zeros((count, n, 3))
    lib = ol.ref(64)
    assert lib.ref_sample(4.0, 0.25, 10000, seed, n, count, ol._p(pos)) == 0
    return pos


def isas():
    host = ol.host_isa()
    return [i for i in ("avx2", "avx512") if ol.REF_BATCHED_SO[i].exists() and
            (i == host or (i == "avx2" and host == "avx512"))]


@pytest.mark.parametrize("isa", isas())
@pytest.mark.parametrize("n", [5, 10])
def test_reference_gate_f64(isa, n):
    mass, q = cycle_molecule(n)
    k = ol.ref_batched(isa).refb_lanes(64)
    pos = ref_pool(n, 4 * k, 0xC0FFEE)
    rtol, atol, pes = 1e-8, 1e-16, 1e-9  # the gate's point: RunConfig defaults
    b = ol.batched_run(pos, mass, q, bits=64, rtol=rtol, atol=atol, pe_stop=pes, isa=isa)
    s = ol.ref_run_batch(pos, mass, q, bits=64, rtol=rtol, atol=atol, pe_stop=pes, threads=4)
    err = ol.config_norm_error(b["momenta"], s["momenta"])
    assert b["lanes"] == k and (b["converged"] == 1).all()
    assert err.max() < max(50 * rtol, 1e-6), err.max()


@pytest.mark.parametrize("isa", isas())
@pytest.mark.parametrize("point", ["production", "tight"])
@pytest.mark.parametrize("mol", ["ch4", "n10"])
def test_f32_gate_vs_scalar(wl, isa, point, mol):
    rtol, atol, pes = wl.PRODUCTION if point == "production" else wl.TIGHT
    if mol == "ch4":
        m = wl.CH4
        mass, q = m.masses_me, m.charge_array
        pos = wl.sample_molecule(m, 512, seed=71)
    else:
        mass, q = cycle_molecule(10)
        pos = ref_pool(10, 256, 0x5EED)
    b = ol.batched_run(pos, mass, q, bits=32, rtol=rtol, atol=atol, pe_stop=pes, isa=isa, threads=4)
    s = ol.ref_run_batch(pos, mass, q, bits=32, rtol=rtol, atol=atol, pe_stop=pes, threads=4)
    err = ol.config_norm_error(b["momenta"], s["momenta"])
    assert (b["status"] == 0).all() and (s["status"] == 0).all()
    assert err.max() < max(50 * rtol, 1e-6), (point, mol, err.max())
    # lockstep costs steps, never accuracy: the lanes' step counts are the
    # batch's, so the mean is at least the scalar engine's
    assert b["steps"].mean() >= 0.95 * s["steps"].mean()


def test_f32_tight_point_within_1e5_of_fp64(wl):
    m = wl.CH4
    pos = wl.sample_molecule(m, 512, seed=72)
    rtol, atol, pes = wl.TIGHT
    b = ol.batched_run(pos, m.masses_me, m.charge_array, bits=32, rtol=rtol, atol=atol, pe_stop=pes, threads=4)
    f = ol.ref_run_batch(pos, m.masses_me, m.charge_array, bits=64, rtol=1e-12, atol=1e-20, pe_stop=1e-13,
                         threads=4)
    err = ol.config_norm_error(b["momenta"], f["momenta"])
    assert err.max() <= 1e-5, err.max()


def test_partial_batch_padding_is_invisible(wl):
    m = wl.CH4
    k = ol.ref_batched().refb_lanes(32)
    base = wl.sample_molecule(m, 3, seed=73)
    tiled = np.concatenate([base] * (k // 3 + 1))[:k]
    rtol, atol, pes = wl.TIGHT
    a = ol.batched_run(base, m.masses_me, m.charge_array, bits=32, rtol=rtol, atol=atol, pe_stop=pes)
    b = ol.batched_run(tiled, m.masses_me, m.charge_array, bits=32, rtol=rtol, atol=atol, pe_stop=pes)
    np.testing.assert_array_equal(a["momenta"], b["momenta"][:3])
    np.testing.assert_array_equal(a["steps"], b["steps"][:3])
    assert a["batch_steps"] == b["batch_steps"]


def test_threads_do_not_change_results(wl):
    m = wl.CH4
    pos = wl.sample_molecule(m, 200, seed=74)
    rtol, atol, pes = wl.PRODUCTION
    one = ol.batched_run(pos, m.masses_me, m.charge_array, bits=32, rtol=rtol, atol=atol, pe_stop=pes, threads=1)
    many = ol.batched_run(pos, m.masses_me, m.charge_array, bits=32, rtol=rtol, atol=atol, pe_stop=pes, threads=4)
    np.testing.assert_array_equal(one["momenta"], many["momenta"])
    assert one["batch_steps"] == many["batch_steps"]


def test_reject_limit_is_a_status_not_a_crash(wl):
    """More than 100 rejections of one step throws in the reference
    (batched_integrator.hpp:268-271); the driver marks that batch status 1.
    Force it with rtol 0 and atol 1e-300 in double precision: every error is
    far above the scale, and 100 rejections shrink h by 0.2^100 without it
    underflowing to zero (in float it would, and h = 0 passes)."""
    m = wl.CH4
    pos = wl.sample_molecule(m, 20, seed=75)
    r = ol.batched_run(pos, m.masses_me, m.charge_array, bits=64, rtol=0.0, atol=1e-300, pe_stop=1e-7)
    assert (r["status"] == 1).all() and not r["momenta"].any()
