// dropin_beside_engine.cpp -- one translation unit that uses the reference's
// coulomb::engine (scalar driver, integrator factory, sampler and, when the
// Highway API is on the include path, BatchedRK45<float>) together with the GPU
// drop-in's coulomb::gpu headers. Built by tests/test_host_api.py with and
// without COULOMB_SINGLE_PRECISION; linked beside the reference's engine
// library and libce_host.so, then run on the CPU path only.
#include <cstdio>
#include <memory>
#include <type_traits>
#include <vector>

#include "coulomb/driver.hpp"
#include "coulomb/gpu/batched_rk45.hpp"
#include "coulomb/gpu/dataset.hpp"
#include "coulomb/gpu/philox_sampler.hpp"
#include "coulomb/integrator.hpp"
#include "coulomb/molecule.hpp"
#include "coulomb/sampler.hpp"
#include "coulomb/system.hpp"
#if defined(WITH_REFERENCE_BATCHED)
#include "coulomb/batched_integrator.hpp"
#endif

using namespace coulomb;

// The drop-in's results are the reference's own types.
static_assert(std::is_same_v<decltype(gpu::run_to_convergence_batch(
                                 std::declval<const Molecule&>(), std::declval<std::vector<State>&>(),
                                 std::declval<const RunConfig&>(), std::declval<const IntegratorOptions&>())),
                             std::vector<RunResult>>);
static_assert(std::is_base_of_v<Sampler, gpu::PhiloxBallSampler>);
static_assert(std::is_same_v<decltype(gpu::BatchedRK45::Result::momenta), std::vector<double>>);
#if defined(WITH_REFERENCE_BATCHED)
// Both batched engines' Result members have the same names and types.
static_assert(std::is_same_v<decltype(gpu::BatchedRK45::Result::momenta), decltype(BatchedRK45<float>::Result::momenta)>);
static_assert(std::is_same_v<decltype(gpu::BatchedRK45::Result::steps), decltype(BatchedRK45<float>::Result::steps)>);
static_assert(std::is_same_v<decltype(gpu::BatchedRK45::Result::converged),
                             decltype(BatchedRK45<float>::Result::converged)>);
static_assert(std::is_same_v<decltype(gpu::BatchedRK45::Result::batch_steps),
                             decltype(BatchedRK45<float>::Result::batch_steps)>);
#endif

int main() {
  // The reference's scalar path, from the reference's engine library.
  Molecule mol;
  mol.atoms.push_back(atom_from_amu("C", static_cast<Real>(12.011), Real{1}));
  for (int i = 0; i < 4; ++i) mol.atoms.push_back(atom_from_amu("H", static_cast<Real>(1.008), Real{1}));
  UniformSphereSampler ref_sampler({Real{4}, static_cast<Real>(0.25)}, 49188291);
  State st;
  ref_sampler.sample(mol, st);
  CoulombForce force(Real{1});
  auto integ = make_integrator(IntegratorKind::RK45, IntegratorOptions{static_cast<Real>(1e-6), static_cast<Real>(1e-7)});
  RunConfig cfg;
  cfg.pe_stop_fraction = static_cast<Real>(1e-7);
  const RunResult r = run_to_convergence(mol, force, *integ, st, cfg);
  // The drop-in's host-side sampler, from libce_host.so (no device needed).
  gpu::PhiloxBallSampler ph({3.3, 0.5, 1000}, 20261203);
  State st2;
  ph.sample(mol, st2);
  std::printf("reference scalar: %zu steps, converged %d; philox sim 0 atom 0 x %.6f; real bytes %zu\n", r.steps,
              r.converged ? 1 : 0, static_cast<double>(st2.positions[0].x), sizeof(Real));
  return r.converged && st2.size() == mol.size() ? 0 : 1;
}
