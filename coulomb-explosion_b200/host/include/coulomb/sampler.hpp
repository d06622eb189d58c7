// sampler.hpp -- initial-geometry sampler strategy of the host API.
//
// Sampler is the reference's strategy interface (include/coulomb/sampler.hpp:23-34).
// Two implementations:
//  * UniformSphereSampler -- the reference's distribution and RNG stream
//    (sampler.hpp:46-72, src/sampler.cpp:7-57): std::mt19937_64, each atom drawn
//    uniformly in the ball by cube rejection and redrawn until it clears every
//    atom already placed; std::runtime_error after max_attempts_per_atom,
//    std::invalid_argument for a non-positive radius or negative separation.
//    Seeded identically, it produces the reference's geometries bit for bit.
//  * PhiloxBallSampler -- the engine's counter-based sampler (include/ce_sampler.h):
//    sim s's geometry depends only on (seed, s), every atom independent in the
//    ball, whole-geometry redraw on a close pair; the same draws as the device
//    kernel ce_sample_ball_device.
#pragma once

#include <cstdint>
#include <random>
#include <string_view>

#include "coulomb/molecule.hpp"

namespace coulomb {

class Sampler {
 public:
  virtual ~Sampler() = default;
  virtual void sample(const Molecule& molecule, State& state) = 0;
  virtual std::string_view name() const = 0;
};

class UniformSphereSampler : public Sampler {
 public:
  struct Options {
    Real radius{4};
    Real min_separation{0.25};
    std::size_t max_attempts_per_atom{10000};
  };
  UniformSphereSampler(Options options, std::uint64_t seed);
  void sample(const Molecule& molecule, State& state) override;
  std::string_view name() const override { return "uniform-sphere"; }
  void reseed(std::uint64_t seed) { rng_.seed(seed); }
  const Options& options() const { return opts_; }

 private:
  Vec3 point_in_ball();
  Options opts_;
  std::mt19937_64 rng_;
};

class PhiloxBallSampler : public Sampler {
 public:
  struct Options {
    Real radius{3.3};
    Real min_separation{0.5};
    std::uint32_t max_attempts{1000};
  };
  PhiloxBallSampler(Options options, std::uint64_t seed, std::uint64_t first_sim = 0);
  // Draws sim `next_sim()` and advances the counter.
  void sample(const Molecule& molecule, State& state) override;
  std::string_view name() const override { return "philox-ball"; }
  std::uint64_t next_sim() const { return next_; }
  void seek(std::uint64_t sim) { next_ = sim; }

 private:
  Options opts_;
  std::uint64_t seed_;
  std::uint64_t next_;
};

}  // namespace coulomb
