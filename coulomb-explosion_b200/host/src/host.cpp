// host.cpp -- the counter-based sampler and the dataset writer of the GPU host
// library (coulomb::gpu, include/coulomb/gpu/{philox_sampler,dataset}.hpp).
// Molecules, states and the reference's UniformSphereSampler come from the
// reference's coulomb::engine.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <stdexcept>

#include "ce_sampler.h"
#include "coulomb/gpu/dataset.hpp"
#include "coulomb/gpu/philox_sampler.hpp"
#include "coulomb/units.hpp"

namespace coulomb::gpu {

// ---- PhiloxBallSampler (counter-based; same draws as the device sampler) ----

PhiloxBallSampler::PhiloxBallSampler(Options options, std::uint64_t seed, std::uint64_t first_sim)
    : opts_(options), seed_(seed), next_(first_sim) {
  if (!(opts_.radius > 0)) throw std::invalid_argument("PhiloxBallSampler: radius must be positive");
  if (opts_.min_separation < 0) throw std::invalid_argument("PhiloxBallSampler: min_separation must be non-negative");
}

void PhiloxBallSampler::sample(const Molecule& molecule, State& state) {
  const int n = static_cast<int>(molecule.size());
  if (n < 1 || n > 10) throw std::invalid_argument("PhiloxBallSampler: 1..10 atoms");
  ce_ball_sampler c{seed_, opts_.radius, opts_.min_separation, opts_.max_attempts};
  float pos[30];
  double pos64[30];
  std::uint8_t flag = 0;
  if (ce_sample_ball_host(n, next_, 1, &c, pos, pos64, &flag) != 0)
    throw std::invalid_argument("PhiloxBallSampler: invalid options");
  if (flag) throw std::runtime_error("PhiloxBallSampler: no geometry at the requested separation");
  ++next_;
  state.positions.resize(n);
  state.velocities.assign(n, Vec3{});
  for (int i = 0; i < n; ++i)
    state.positions[i] = Vec3{static_cast<Real>(pos64[i * 3]), static_cast<Real>(pos64[i * 3 + 1]),
                              static_cast<Real>(pos64[i * 3 + 2])};
}

// ---- DatasetWriter ----

DatasetWriter::DatasetWriter(const std::string& path, const Molecule& mol) : path_(path), mol_(mol) {
  out_.open(path, std::ios::binary);
  if (!out_) throw std::runtime_error("cannot open output file: " + path);
}

void DatasetWriter::append(std::size_t count, const float* pos, const float* mom, const std::uint32_t* steps,
                           const std::uint8_t* converged) {
  const std::size_t n3 = mol_.size() * 3, rb = record_bytes(mol_.size());
  buf_.resize(count * rb);
  char* p = buf_.data();
  for (std::size_t s = 0; s < count; ++s) {
    std::memcpy(p, pos + s * n3, n3 * 4);
    std::memcpy(p + n3 * 4, mom + s * n3, n3 * 4);
    std::memcpy(p + n3 * 8, steps + s, 4);
    p[n3 * 8 + 4] = converged[s] ? 1 : 0;
    p += rb;
  }
  out_.write(buf_.data(), static_cast<std::streamsize>(buf_.size()));
  if (!out_) throw std::runtime_error("write failed: " + path_);
  written_ += count;
}

void DatasetWriter::close() {
  if (out_.is_open()) out_.close();
}

void DatasetWriter::write_metadata(const std::map<std::string, double>& numbers,
                                   const std::map<std::string, std::string>& strings) const {
  std::ofstream m(path_ + ".meta.json");
  if (!m) throw std::runtime_error("cannot open metadata file: " + path_ + ".meta.json");
  m.precision(17);
  m << "{\n  \"symbols\": [";
  for (std::size_t i = 0; i < mol_.size(); ++i) m << (i ? ", " : "") << '"' << mol_.atoms[i].symbol << '"';
  m << "],\n  \"masses_amu\": [";
  for (std::size_t i = 0; i < mol_.size(); ++i) m << (i ? ", " : "") << mol_.atoms[i].mass / units::kAmuToElectronMass;
  m << "],\n  \"charges\": [";
  for (std::size_t i = 0; i < mol_.size(); ++i) m << (i ? ", " : "") << mol_.atoms[i].charge;
  m << "],\n  \"n_atoms\": " << mol_.size();
  for (const auto& [k, v] : numbers) {
    m << ",\n  \"" << k << "\": ";
    if (std::floor(v) == v && std::fabs(v) < 9e15)
      m << static_cast<long long>(v);
    else
      m << v;
  }
  for (const auto& [k, v] : strings) m << ",\n  \"" << k << "\": \"" << v << '"';
  m << ",\n  \"record_layout\": [\"init_pos: n*3 float32 (x,y,z per atom, atom order as symbols)\", "
       "\"final_momentum: n*3 float32 (m*v per atom, post energy-redistribution)\", \"steps: uint32\", "
       "\"converged: uint8\"]\n}\n";
}

}  // namespace coulomb::gpu
