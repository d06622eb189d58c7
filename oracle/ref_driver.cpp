// ref_driver.cpp -- C entry points around the reference scalar engine.
//
// TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile together with the
// reference's own, unmodified sources (src/system.cpp, src/integrators.cpp,
// src/driver.cpp, src/sampler.cpp, read in place from the reference checkout)
// into oracle/_ref/libref_f32.so (COULOMB_SINGLE_PRECISION) and libref_f64.so.
// It drives the reference exactly as its own callers do:
//   - examples/generate_dataset.cpp / bench/bench_batched_integrator.cpp:183-199
//     (make_integrator(RK45, {rtol, atol}) + run_to_convergence per sim),
//   - bench/bench_precision_sweep.cpp:227-250 (FailureCode classification).
// Used to pin the C oracle bit-for-bit and as bench.py's reference arm
// (all host threads, one integrator instance per sim, as the reference's
// threading rule requires).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <exception>
#include <stdexcept>
#include <thread>
#include <vector>

#include "coulomb/driver.hpp"
#include "coulomb/integrator.hpp"
#include "coulomb/molecule.hpp"
#include "coulomb/sampler.hpp"
#include "coulomb/system.hpp"

using namespace coulomb;

namespace {

Molecule make_mol(int n, const double* mass, const double* charge) {
  Molecule m;
  for (int i = 0; i < n; ++i)
    m.atoms.push_back(Atom{"X", static_cast<Real>(mass[i]), static_cast<Real>(charge[i])});
  return m;
}

State make_state(int n, const double* pos) {
  State s;
  s.positions.resize(static_cast<std::size_t>(n));
  s.velocities.assign(static_cast<std::size_t>(n), Vec3{});
  for (int i = 0; i < n; ++i)
    s.positions[static_cast<std::size_t>(i)] =
        Vec3{static_cast<Real>(pos[i * 3]), static_cast<Real>(pos[i * 3 + 1]),
             static_cast<Real>(pos[i * 3 + 2])};
  return s;
}

}  // namespace

extern "C" {

int ref_real_bytes() { return static_cast<int>(sizeof(Real)); }

void ref_accel(int n, const double* x, const double* mass, const double* charge, double k,
               double* a) {
  const Molecule m = make_mol(n, mass, charge);
  const State s = make_state(n, x);
  std::vector<Vec3> acc;
  CoulombForce(static_cast<Real>(k)).accelerations(m, s, acc);
  for (int i = 0; i < n; ++i) {
    a[i * 3] = static_cast<double>(acc[static_cast<std::size_t>(i)].x);
    a[i * 3 + 1] = static_cast<double>(acc[static_cast<std::size_t>(i)].y);
    a[i * 3 + 2] = static_cast<double>(acc[static_cast<std::size_t>(i)].z);
  }
}

double ref_pe(int n, const double* x, const double* charge, double k) {
  std::vector<double> ones(static_cast<std::size_t>(n), 1.0);
  const Molecule m = make_mol(n, ones.data(), charge);
  const State s = make_state(n, x);
  return static_cast<double>(CoulombForce(static_cast<Real>(k)).potential_energy(m, s));
}

// One run_to_convergence per sim over [0, S), split across `threads` host
// threads (<= 0: hardware_concurrency). status: 0 ok, 1 integrator threw,
// 2 max_steps, 3 non-finite momenta (bench_precision_sweep.cpp:80-85).
// kind: 0 = IntegratorKind::RK45, 1 = IntegratorKind::VelocityVerlet (fixed step max_dt).
void ref_run_batch_kind(int kind, int n, const double* mass, const double* charge, double k, uint64_t S,
                        const double* pos, double rtol, double atol, double pe_stop, double max_dt,
                        uint64_t max_steps, int redistribute, double* p_out, uint32_t* steps,
                        uint8_t* status, double* t_final, int threads) {
  const IntegratorKind ikind = kind == 1 ? IntegratorKind::VelocityVerlet : IntegratorKind::RK45;
  const Molecule mol = make_mol(n, mass, charge);
  const CoulombForce force(static_cast<Real>(k));
  RunConfig cfg;
  cfg.pe_stop_fraction = static_cast<Real>(pe_stop);
  cfg.redistribute_energy = redistribute != 0;
  cfg.max_dt = static_cast<Real>(max_dt);
  cfg.max_steps = static_cast<std::size_t>(max_steps);
  const IntegratorOptions opts{static_cast<Real>(rtol), static_cast<Real>(atol)};

  std::atomic<uint64_t> next{0};
  auto worker = [&]() {
    for (;;) {
      const uint64_t s0 = next.fetch_add(64);
      if (s0 >= S) break;
      const uint64_t s1 = std::min<uint64_t>(S, s0 + 64);
      for (uint64_t s = s0; s < s1; ++s) {
        State st = make_state(n, pos + s * static_cast<uint64_t>(n) * 3);
        auto integ = make_integrator(ikind, opts);
        uint8_t code = 0;
        RunResult rr;
        try {
          rr = run_to_convergence(mol, force, *integ, st, cfg);
          // A zero-step run (PE_0 already at or below the stop) leaves
          // RunResult::converged false in the scalar driver; it is not a
          // max_steps failure, so only a run that stopped at max_steps is.
          if (!rr.converged && rr.steps >= cfg.max_steps) code = 2;
        } catch (const std::exception&) {
          code = 1;
        }
        double* p = p_out + s * static_cast<uint64_t>(n) * 3;
        for (int i = 0; i < n; ++i) {
          const Real m = mol.atoms[static_cast<std::size_t>(i)].mass;
          const Vec3 pv = st.velocities[static_cast<std::size_t>(i)] * m;
          p[i * 3] = static_cast<double>(pv.x);
          p[i * 3 + 1] = static_cast<double>(pv.y);
          p[i * 3 + 2] = static_cast<double>(pv.z);
          if (code == 0 && !(std::isfinite(p[i * 3]) && std::isfinite(p[i * 3 + 1]) &&
                             std::isfinite(p[i * 3 + 2])))
            code = 3;
        }
        if (steps) steps[s] = static_cast<uint32_t>(rr.steps);
        if (status) status[s] = code;
        if (t_final) t_final[s] = static_cast<double>(rr.t_final);
      }
    }
  };
  unsigned nt = threads > 0 ? static_cast<unsigned>(threads) : std::thread::hardware_concurrency();
  if (nt == 0) nt = 1;
  if (nt == 1) {
    worker();
    return;
  }
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nt; ++t) pool.emplace_back(worker);
  for (auto& th : pool) th.join();
}

// UniformSphereSampler::sample `count` times (sampler.cpp:28-57) into
// pos_out[count][n][3]. Returns 0, -1 on std::runtime_error (infeasible),
// -2 on std::invalid_argument (bad options).
void ref_run_batch(int n, const double* mass, const double* charge, double k, uint64_t S,
                   const double* pos, double rtol, double atol, double pe_stop, double max_dt,
                   uint64_t max_steps, int redistribute, double* p_out, uint32_t* steps,
                   uint8_t* status, double* t_final, int threads) {
  ref_run_batch_kind(0, n, mass, charge, k, S, pos, rtol, atol, pe_stop, max_dt, max_steps, redistribute, p_out,
                     steps, status, t_final, threads);
}

int ref_sample(double radius, double min_sep, uint64_t max_attempts, uint64_t seed, int n,
               uint64_t count, double* pos_out) {
  try {
    UniformSphereSampler::Options o;
    o.radius = static_cast<Real>(radius);
    o.min_separation = static_cast<Real>(min_sep);
    o.max_attempts_per_atom = static_cast<std::size_t>(max_attempts);
    UniformSphereSampler sampler(o, seed);
    std::vector<double> ones(static_cast<std::size_t>(n), 1.0);
    const Molecule mol = make_mol(n, ones.data(), ones.data());
    State st;
    for (uint64_t c = 0; c < count; ++c) {
      sampler.sample(mol, st);
      for (int i = 0; i < n; ++i) {
        pos_out[(c * static_cast<uint64_t>(n) + static_cast<uint64_t>(i)) * 3] =
            static_cast<double>(st.positions[static_cast<std::size_t>(i)].x);
        pos_out[(c * static_cast<uint64_t>(n) + static_cast<uint64_t>(i)) * 3 + 1] =
            static_cast<double>(st.positions[static_cast<std::size_t>(i)].y);
        pos_out[(c * static_cast<uint64_t>(n) + static_cast<uint64_t>(i)) * 3 + 2] =
            static_cast<double>(st.positions[static_cast<std::size_t>(i)].z);
      }
    }
  } catch (const std::invalid_argument&) {
    return -2;
  } catch (const std::runtime_error&) {
    return -1;
  }
  return 0;
}

}  // extern "C"
