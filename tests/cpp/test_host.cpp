// test_host.cpp -- C++ checks of the drop-in, driven by tests/test_host_api.py.
//
// Built against the reference's own headers and linked beside its engine
// library (coulomb::engine: Molecule, State, RunConfig, RunResult,
// IntegratorOptions, UniformSphereSampler are the reference's), plus
// coulomb::gpu from libce_host.so.
//
// Modes (argv[1]):
//   sampler <seed> <n> <radius> <min_sep> <count> <out.bin>
//       UniformSphereSampler draws as raw doubles [count][n][3] (compared with
//       the reference sampler's golden draws).
//   errors
//       the reference's sampler / batched-engine argument contract
//       (tests/test_sampler.cpp:40-117 and batched_integrator.hpp:73-75 of the
//       reference): exit 0 when every expected exception is thrown.
//   gpu <S> <out.bin>
//       coulomb::gpu::BatchedRK45 over S Philox CH4 geometries at the tight
//       point, then run_to_convergence_batch on the same geometries; writes
//       positions, both momenta sets, E0, KER, steps and status.
//   generate <sims> <lanes> <seed> <rtol> <pe_stop> <out.bin>
//       the reference generator's call shape (examples/generate_dataset.cpp:173-227):
//       the reference's UniformSphereSampler (r 4.0, min 0.25) fills each lane
//       with set_lane_geometry, run(cfg) per batch of `lanes`, records written
//       as float32 positions and momenta, u32 steps, u8 converged.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "coulomb/driver.hpp"
#include "coulomb/gpu/batched_rk45.hpp"
#include "coulomb/gpu/philox_sampler.hpp"
#include "coulomb/integrator.hpp"
#include "coulomb/molecule.hpp"
#include "coulomb/sampler.hpp"
#include "coulomb/system.hpp"

using namespace coulomb;
using gpu::PhiloxBallSampler;

namespace {

Molecule make_methane() {
  Molecule m;
  m.atoms.push_back(atom_from_amu("C", static_cast<Real>(12.011), Real{1}));
  for (int i = 0; i < 4; ++i) m.atoms.push_back(atom_from_amu("H", static_cast<Real>(1.008), Real{1}));
  return m;
}

template <typename T>
void put(std::ofstream& f, const std::vector<T>& v) {
  f.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
}

int mode_sampler(char** argv) {
  const std::uint64_t seed = std::stoull(argv[2]);
  const int n = std::stoi(argv[3]);
  UniformSphereSampler s({static_cast<Real>(std::stod(argv[4])), static_cast<Real>(std::stod(argv[5])), 10000}, seed);
  const std::size_t count = std::stoull(argv[6]);
  Molecule mol;
  for (int i = 0; i < n; ++i) mol.atoms.push_back(Atom{"X", Real{1}, Real{1}});
  std::vector<double> out;
  State st;
  for (std::size_t c = 0; c < count; ++c) {
    s.sample(mol, st);
    for (const Vec3& p : st.positions) {
      out.push_back(static_cast<double>(p.x));
      out.push_back(static_cast<double>(p.y));
      out.push_back(static_cast<double>(p.z));
    }
  }
  std::ofstream f(argv[7], std::ios::binary);
  put(f, out);
  return 0;
}

template <typename E, typename F>
bool throws(F&& f) {
  try {
    f();
  } catch (const E&) {
    return true;
  } catch (...) {
    return false;
  }
  return false;
}

int mode_errors() {
  int bad = 0;
  Molecule mol;
  for (int i = 0; i < 8; ++i) mol.atoms.push_back(Atom{"X", Real{1}, Real{1}});
  State st;
  bad += !throws<std::invalid_argument>([] { UniformSphereSampler({Real{0}, static_cast<Real>(0.25), 10}, 1); });
  bad += !throws<std::invalid_argument>([] { UniformSphereSampler({Real{1}, static_cast<Real>(-0.1), 10}, 1); });
  bad += !throws<std::runtime_error>([&] {
    UniformSphereSampler s({static_cast<Real>(0.5), static_cast<Real>(0.9), 50}, 1);
    s.sample(mol, st);
  });
  bad += !throws<std::invalid_argument>([] { PhiloxBallSampler({-1.0, 0.5, 10}, 1); });
  // Same seed, same draws; different seeds differ (reference test_sampler.cpp:64-86).
  const UniformSphereSampler::Options o{Real{4}, static_cast<Real>(0.25), 10000};
  UniformSphereSampler a(o, 7), b(o, 7), c(o, 8);
  State sa, sb, sc;
  a.sample(mol, sa);
  b.sample(mol, sb);
  c.sample(mol, sc);
  bad += sa.positions[3].x != sb.positions[3].x;
  bad += sa.positions[3].x == sc.positions[3].x;
  for (const Vec3& v : sa.velocities) bad += (v.x != 0 || v.y != 0 || v.z != 0);
  std::printf("errors: %d\n", bad);
  return bad == 0 ? 0 : 1;
}

int mode_gpu(char** argv) {
  const std::size_t S = std::stoull(argv[2]);
  const Molecule mol = make_methane();
  const std::size_t n = mol.size();
  PhiloxBallSampler sampler({3.3, 0.5, 1000}, 20261203);
  std::vector<State> states(S);
  for (State& st : states) sampler.sample(mol, st);
  gpu::BatchedRK45 bi(mol, Real{1}, S, static_cast<Real>(1e-6), static_cast<Real>(1e-7));
  for (std::size_t l = 0; l < S; ++l) bi.set_lane_geometry(l, states[l].positions);
  RunConfig cfg;
  cfg.pe_stop_fraction = static_cast<Real>(1e-7);
  const auto res = bi.run(cfg);
  int bad = 0;
  bad += !throws<std::invalid_argument>([&] { bi.set_lane_geometry(S, states[0].positions); });
  bad += !throws<std::invalid_argument>(
      [&] { gpu::BatchedRK45(mol, Real{1}, 0, static_cast<Real>(1e-6), static_cast<Real>(1e-7)); });
  auto states2 = states;
  gpu::BatchStatus extra;
  const std::vector<RunResult> rr = gpu::run_to_convergence_batch(
      mol, states2, cfg, IntegratorOptions{static_cast<Real>(1e-6), static_cast<Real>(1e-7)}, Real{1}, 0,
      gpu::kKahanFP64, &extra);
  std::vector<double> pos, mom_driver, e0, ker;
  std::vector<std::uint32_t> steps;
  std::vector<std::uint8_t> status;
  for (std::size_t s = 0; s < S; ++s) {
    for (std::size_t i = 0; i < n; ++i) {
      pos.push_back(static_cast<double>(states[s].positions[i].x));
      pos.push_back(static_cast<double>(states[s].positions[i].y));
      pos.push_back(static_cast<double>(states[s].positions[i].z));
      const double m = static_cast<double>(mol.atoms[i].mass);
      mom_driver.push_back(static_cast<double>(states2[s].velocities[i].x) * m);
      mom_driver.push_back(static_cast<double>(states2[s].velocities[i].y) * m);
      mom_driver.push_back(static_cast<double>(states2[s].velocities[i].z) * m);
    }
    steps.push_back(static_cast<std::uint32_t>(res.steps[s]));
    status.push_back(static_cast<std::uint8_t>(res.status[s]));
    e0.push_back(static_cast<double>(rr[s].energy_initial));
    ker.push_back(static_cast<double>(rr[s].ke_after_redist));
    bad += rr[s].converged != (res.converged[s] != 0);
    bad += extra.status[s] != res.status[s];
    bad += rr[s].steps != res.steps[s];
  }
  std::ofstream f(argv[3], std::ios::binary);
  put(f, pos);
  put(f, res.momenta);
  put(f, mom_driver);
  put(f, e0);
  put(f, ker);
  put(f, steps);
  put(f, status);
  std::printf("gpu: %zu lanes, batch_steps %zu, bad %d\n", S, res.batch_steps, bad);
  return bad == 0 ? 0 : 1;
}

int mode_generate(char** argv) {
  const std::size_t sims = std::stoull(argv[2]), lanes = std::stoull(argv[3]);
  const std::uint64_t seed = std::stoull(argv[4]);
  const Molecule mol = make_methane();
  const std::size_t n = mol.size();
  UniformSphereSampler sampler({Real{4}, static_cast<Real>(0.25)}, seed);
  gpu::BatchedRK45 bi(mol, Real{1}, lanes, static_cast<Real>(std::stod(argv[5])), static_cast<Real>(1e-7));
  RunConfig cfg;
  cfg.pe_stop_fraction = static_cast<Real>(std::stod(argv[6]));
  std::ofstream out(argv[7], std::ios::binary);
  const std::size_t n_batches = (sims + lanes - 1) / lanes;
  std::vector<State> lane_geoms(lanes);
  std::vector<float> pos_buf(n * 3), mom_buf(n * 3);
  std::size_t written = 0, failed = 0;
  for (std::size_t b = 0; b < n_batches; ++b) {
    for (std::size_t lane = 0; lane < lanes; ++lane) {
      sampler.sample(mol, lane_geoms[lane]);
      bi.set_lane_geometry(lane, lane_geoms[lane].positions);
    }
    const auto res = bi.run(cfg);
    for (std::size_t lane = 0; lane < lanes && written < sims; ++lane, ++written) {
      for (std::size_t i = 0; i < n; ++i) {
        pos_buf[i * 3 + 0] = static_cast<float>(lane_geoms[lane].positions[i].x);
        pos_buf[i * 3 + 1] = static_cast<float>(lane_geoms[lane].positions[i].y);
        pos_buf[i * 3 + 2] = static_cast<float>(lane_geoms[lane].positions[i].z);
        for (int c = 0; c < 3; ++c) mom_buf[i * 3 + c] = static_cast<float>(res.momenta[(lane * n + i) * 3 + c]);
      }
      const auto steps = static_cast<std::uint32_t>(res.steps[lane]);
      const auto converged = static_cast<std::uint8_t>(res.converged[lane] ? 1 : 0);
      failed += converged ? 0 : 1;
      out.write(reinterpret_cast<const char*>(pos_buf.data()), static_cast<std::streamsize>(pos_buf.size() * 4));
      out.write(reinterpret_cast<const char*>(mom_buf.data()), static_cast<std::streamsize>(mom_buf.size() * 4));
      out.write(reinterpret_cast<const char*>(&steps), sizeof(steps));
      out.write(reinterpret_cast<const char*>(&converged), sizeof(converged));
    }
  }
  std::printf("generate: %zu sims in %zu batches of %zu lanes, %zu failed\n", written, n_batches, lanes, failed);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    const std::string mode = argc > 1 ? argv[1] : "";
    if (mode == "sampler" && argc == 8) return mode_sampler(argv);
    if (mode == "errors") return mode_errors();
    if (mode == "gpu" && argc == 4) return mode_gpu(argv);
    if (mode == "generate" && argc == 8) return mode_generate(argv);
    std::fprintf(stderr, "usage: test_host sampler|errors|gpu|generate ...\n");
    return 2;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "exception: %s\n", e.what());
    return 3;
  }
}
