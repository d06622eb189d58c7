// philox_sampler.hpp -- the engine's counter-based geometry sampler as a
// coulomb::Sampler strategy (include/coulomb/sampler.hpp:23-34 of the reference).
//
// Sim s's geometry depends only on (seed, s): every atom uniform in the ball,
// independently, and the whole geometry redrawn on a close pair. The draws are
// those of the device kernel ce_sample_ball_device (include/ce_sampler.h), so a
// host-sampled slice equals the device-sampled one bit for bit. The reference's
// own UniformSphereSampler (sequential mt19937_64, src/sampler.cpp:17-57) stays
// the host-side parity path; its stream cannot be split across threads.
#pragma once

#include <cstdint>
#include <string_view>

#include "coulomb/molecule.hpp"
#include "coulomb/sampler.hpp"
#include "coulomb/system.hpp"

namespace coulomb::gpu {

class PhiloxBallSampler : public Sampler {
 public:
  struct Options {
    double radius{3.3};
    double min_separation{0.5};
    std::uint32_t max_attempts{1000};
  };
  // std::invalid_argument for a non-positive radius or a negative separation.
  PhiloxBallSampler(Options options, std::uint64_t seed, std::uint64_t first_sim = 0);
  // Draws sim `next_sim()` and advances the counter; std::runtime_error when no
  // geometry clears the separation within max_attempts.
  void sample(const Molecule& molecule, State& state) override;
  std::string_view name() const override { return "philox-ball"; }
  std::uint64_t next_sim() const { return next_; }
  void seek(std::uint64_t sim) { next_ = sim; }

 private:
  Options opts_;
  std::uint64_t seed_;
  std::uint64_t next_;
};

}  // namespace coulomb::gpu
