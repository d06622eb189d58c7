// test_host.cpp -- C++ checks of the host API, driven by tests/test_host_api.py.
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
//       positions, both momenta sets, steps and status.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "coulomb/driver.hpp"
#include "coulomb/gpu/batched_rk45.hpp"
#include "coulomb/molecule.hpp"
#include "coulomb/sampler.hpp"

using namespace coulomb;

namespace {

template <typename T>
void put(std::ofstream& f, const std::vector<T>& v) {
  f.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(T)));
}

int mode_sampler(char** argv) {
  const std::uint64_t seed = std::stoull(argv[2]);
  const int n = std::stoi(argv[3]);
  UniformSphereSampler s({std::stod(argv[4]), std::stod(argv[5]), 10000}, seed);
  const std::size_t count = std::stoull(argv[6]);
  Molecule mol;
  for (int i = 0; i < n; ++i) mol.atoms.push_back(Atom{"X", 1.0, 1.0});
  std::vector<double> out;
  State st;
  for (std::size_t c = 0; c < count; ++c) {
    s.sample(mol, st);
    for (const Vec3& p : st.positions) {
      out.push_back(p.x);
      out.push_back(p.y);
      out.push_back(p.z);
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
  for (int i = 0; i < 8; ++i) mol.atoms.push_back(Atom{"X", 1.0, 1.0});
  State st;
  bad += !throws<std::invalid_argument>([] { UniformSphereSampler({0.0, 0.25, 10}, 1); });
  bad += !throws<std::invalid_argument>([] { UniformSphereSampler({1.0, -0.1, 10}, 1); });
  bad += !throws<std::runtime_error>([&] {
    UniformSphereSampler s({0.5, 0.9, 50}, 1);
    s.sample(mol, st);
  });
  bad += !throws<std::invalid_argument>([] { PhiloxBallSampler({-1.0, 0.5, 10}, 1); });
  // Same seed, same draws; different seeds differ (reference test_sampler.cpp:64-86).
  UniformSphereSampler a({4.0, 0.25, 10000}, 7), b({4.0, 0.25, 10000}, 7), c({4.0, 0.25, 10000}, 8);
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
  gpu::BatchedRK45 bi(mol, 1.0, S, 1e-6, 1e-7);
  for (std::size_t l = 0; l < S; ++l) bi.set_lane_geometry(l, states[l].positions);
  RunConfig cfg;
  cfg.pe_stop_fraction = 1e-7;
  const auto res = bi.run(cfg);
  int bad = 0;
  bad += !throws<std::invalid_argument>([&] { bi.set_lane_geometry(S, states[0].positions); });
  bad += !throws<std::invalid_argument>([&] { gpu::BatchedRK45(mol, 1.0, 0, 1e-6, 1e-7); });
  auto states2 = states;
  const auto rr = gpu::run_to_convergence_batch(mol, states2, cfg, IntegratorOptions{1e-6, 1e-7});
  std::vector<double> pos, mom_driver, e0, ker;
  std::vector<std::uint32_t> steps;
  std::vector<std::uint8_t> status;
  for (std::size_t s = 0; s < S; ++s) {
    for (std::size_t i = 0; i < n; ++i) {
      pos.push_back(states[s].positions[i].x);
      pos.push_back(states[s].positions[i].y);
      pos.push_back(states[s].positions[i].z);
      const double m = mol.atoms[i].mass;
      mom_driver.push_back(states2[s].velocities[i].x * m);
      mom_driver.push_back(states2[s].velocities[i].y * m);
      mom_driver.push_back(states2[s].velocities[i].z * m);
    }
    steps.push_back(static_cast<std::uint32_t>(res.steps[s]));
    status.push_back(static_cast<std::uint8_t>(res.status[s]));
    e0.push_back(rr[s].energy_initial);
    ker.push_back(rr[s].ke_after_redist);
    bad += rr[s].converged != (res.converged[s] != 0);
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

}  // namespace

int main(int argc, char** argv) {
  try {
    const std::string mode = argc > 1 ? argv[1] : "";
    if (mode == "sampler" && argc == 8) return mode_sampler(argv);
    if (mode == "errors") return mode_errors();
    if (mode == "gpu" && argc == 4) return mode_gpu(argv);
    std::fprintf(stderr, "usage: test_host sampler|errors|gpu ...\n");
    return 2;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "exception: %s\n", e.what());
    return 3;
  }
}
