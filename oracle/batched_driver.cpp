// batched_driver.cpp -- C entry points around the reference's SIMD batched engine.
//
// TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile with the reference's own,
// unmodified include/coulomb/batched_integrator.hpp and batched_force.hpp (read in
// place from the reference checkout) against the project-written Highway shim in
// oracle/hwy_shim/, once per x86 vector ISA:
//   _ref/libref_batched_avx512.so  (-march=x86-64-v4: K = 16 float lanes)
//   _ref/libref_batched_avx2.so    (-march=x86-64-v3: K = 8 float lanes)
// The engine library types (Molecule, RunConfig, Vec3) are in their default
// double precision, as in the reference's generator build (Real = double; the
// batched element type T is the template argument).
//
// refb_run drives BatchedRK45<T> exactly like examples/generate_dataset.cpp:173-227
// (one instance, set_lane_geometry for each of the K lanes, run(cfg), read
// Result::momenta / steps / converged), except that geometries come pre-generated
// from the caller, as in bench/bench_batched_integrator.cpp:140-174. A final
// partial batch is padded with copies of its own first lane: a duplicated lane
// has the same error as its original, so the shared-dt trajectory (max error over
// active lanes) of the real lanes is unchanged by the padding.
//
// Per-sim status (the C ABI's codes, bench/bench_precision_sweep.cpp:80-85):
//   0 converged, 1 the batch threw (more than 100 rejections of one step,
//   batched_integrator.hpp:268-271: every lane of that batch), 2 max_steps
//   reached before the stop, 3 non-finite momenta.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <exception>
#include <thread>
#include <vector>

#include "coulomb/batched_integrator.hpp"

using namespace coulomb;

namespace {

Molecule make_mol(int n, const double* mass, const double* charge) {
  Molecule m;
  for (int i = 0; i < n; ++i)
    m.atoms.push_back(Atom{"X", static_cast<Real>(mass[i]), static_cast<Real>(charge[i])});
  return m;
}

struct RunArgs {
  int n;
  const double* mass;
  const double* charge;
  double k;
  uint64_t S;
  const double* pos;
  double rtol, atol, pe_stop, max_dt;
  uint64_t max_steps;
  int redistribute;
  double* p_out;
  uint32_t* steps;
  uint8_t* converged;
  uint8_t* status;
};

template <class T>
uint64_t run_range(const RunArgs& a, uint64_t b0, uint64_t b1) {
  const Molecule mol = make_mol(a.n, a.mass, a.charge);
  const std::size_t n = static_cast<std::size_t>(a.n);
  const std::size_t K = hwy::HWY_NAMESPACE::Lanes(hwy::HWY_NAMESPACE::ScalableTag<T>());
  BatchedRK45<T> bi(mol, static_cast<Real>(a.k), K, static_cast<T>(a.rtol), static_cast<T>(a.atol));
  RunConfig cfg;
  cfg.pe_stop_fraction = static_cast<Real>(a.pe_stop);
  cfg.redistribute_energy = a.redistribute != 0;
  cfg.max_dt = static_cast<Real>(a.max_dt);
  cfg.max_steps = static_cast<std::size_t>(a.max_steps);

  std::vector<Vec3> geom(n);
  uint64_t batch_steps = 0;
  for (uint64_t b = b0; b < b1; ++b) {
    const uint64_t first = b * K;
    const uint64_t real = std::min<uint64_t>(K, a.S - first);
    for (std::size_t lane = 0; lane < K; ++lane) {
      const uint64_t s = first + (lane < real ? lane : 0);
      const double* p = a.pos + s * n * 3;
      for (std::size_t i = 0; i < n; ++i)
        geom[i] = Vec3{static_cast<Real>(p[i * 3]), static_cast<Real>(p[i * 3 + 1]),
                       static_cast<Real>(p[i * 3 + 2])};
      bi.set_lane_geometry(lane, geom);
    }
    try {
      const auto r = bi.run(cfg);
      batch_steps += r.batch_steps;
      for (uint64_t lane = 0; lane < real; ++lane) {
        const uint64_t s = first + lane;
        uint8_t code = r.converged[lane] ? 0 : 2;
        for (std::size_t c = 0; c < n * 3; ++c) {
          const double v = r.momenta[lane * n * 3 + c];
          if (a.p_out) a.p_out[s * n * 3 + c] = v;
          if (code == 0 && !std::isfinite(v)) code = 3;
        }
        if (a.steps) a.steps[s] = static_cast<uint32_t>(r.steps[lane]);
        if (a.converged) a.converged[s] = static_cast<uint8_t>(r.converged[lane] ? 1 : 0);
        if (a.status) a.status[s] = code;
      }
    } catch (const std::exception&) {
      for (uint64_t lane = 0; lane < real; ++lane) {
        const uint64_t s = first + lane;
        if (a.p_out)
          for (std::size_t c = 0; c < n * 3; ++c) a.p_out[s * n * 3 + c] = 0.0;
        if (a.steps) a.steps[s] = 0;
        if (a.converged) a.converged[s] = 0;
        if (a.status) a.status[s] = 1;
      }
    }
  }
  return batch_steps;
}

template <class T>
uint64_t run_threads(const RunArgs& a, int threads) {
  const std::size_t K = hwy::HWY_NAMESPACE::Lanes(hwy::HWY_NAMESPACE::ScalableTag<T>());
  const uint64_t nb = (a.S + K - 1) / K;
  unsigned nt = threads > 0 ? static_cast<unsigned>(threads) : 1u;
  nt = static_cast<unsigned>(std::min<uint64_t>(nt, std::max<uint64_t>(nb, 1)));
  if (nt <= 1) return run_range<T>(a, 0, nb);
  // Whole batches in chunks of 16, taken dynamically; one engine instance per
  // thread (BatchedRK45 keeps per-instance state).
  std::atomic<uint64_t> next{0}, total{0};
  auto worker = [&]() {
    for (;;) {
      const uint64_t b0 = next.fetch_add(16);
      if (b0 >= nb) break;
      total += run_range<T>(a, b0, std::min<uint64_t>(nb, b0 + 16));
    }
  };
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nt; ++t) pool.emplace_back(worker);
  for (auto& th : pool) th.join();
  return total.load();
}

}  // namespace

extern "C" {

// Lanes K of BatchedRK45<float> (bits 32) or BatchedRK45<double> (bits 64) in
// this build, i.e. the SIMD width the reference's constructor insists on
// (batched_integrator.hpp:73-75).
int refb_lanes(int bits) {
  return bits == 64 ? static_cast<int>(hwy::HWY_NAMESPACE::Lanes(hwy::HWY_NAMESPACE::ScalableTag<double>()))
                    : static_cast<int>(hwy::HWY_NAMESPACE::Lanes(hwy::HWY_NAMESPACE::ScalableTag<float>()));
}

// S sims of one molecule through BatchedRK45<T> (T = float for bits 32, double
// for bits 64) in batches of K lanes; threads <= 1 runs on the calling thread.
// pos [S][n][3] float64; p_out [S][n][3] float64 (Result::momenta order);
// steps / converged / status [S] (any may be NULL). Returns the summed
// Result::batch_steps over all batches (the lockstep iterations run).
uint64_t refb_run(int bits, int n, const double* mass, const double* charge, double k, uint64_t S,
                  const double* pos, double rtol, double atol, double pe_stop, double max_dt,
                  uint64_t max_steps, int redistribute, double* p_out, uint32_t* steps,
                  uint8_t* converged, uint8_t* status, int threads) {
  const RunArgs a{n,      mass,   charge,      k,         S,     pos,       rtol,     atol,
                  pe_stop, max_dt, max_steps, redistribute, p_out, steps, converged, status};
  if (S == 0 || n <= 0) return 0;
  return bits == 64 ? run_threads<double>(a, threads) : run_threads<float>(a, threads);
}

}  // extern "C"
