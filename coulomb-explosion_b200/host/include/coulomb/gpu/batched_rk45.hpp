// batched_rk45.hpp -- the GPU drop-in for the reference's batched engine.
//
// coulomb::gpu::BatchedRK45 has the three members of the reference's
// coulomb::BatchedRK45<T> (include/coulomb/batched_integrator.hpp:61-191):
//   ctor(molecule, coulomb_k, lanes, rtol, atol), set_lane_geometry(lane, pos),
//   run(RunConfig) -> Result{momenta, steps, converged, batch_steps},
// with `lanes` any batch capacity instead of the SIMD width (the reference
// throws std::invalid_argument unless lanes equals the SIMD width,
// batched_integrator.hpp:73-75). Each lane is integrated on its own clock (no
// shared dt), so a lane's result does not depend on its batch-mates. Result adds
// the kinetic energy release, the per-sim status and the rejection count.
//
// run_to_convergence_batch is the drop-in for the scalar driver at batch
// granularity (src/driver.cpp:7-46): one RunResult per state; each state's
// velocities become the asymptotic (post-redistribution) velocities p_i / m_i.
// Final positions are not returned (the GPU engine keeps them on chip).
//
// Errors surface as exceptions on the host side, as in the reference:
// std::invalid_argument for bad arguments, std::runtime_error for device errors.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <vector>

#include "coulomb/driver.hpp"
#include "coulomb/molecule.hpp"

struct ce_engine;

namespace coulomb::gpu {

// RAII owner of one ce_engine (one per host thread and device).
class Engine {
 public:
  explicit Engine(int device = 0);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;
  ce_engine* handle() const { return e_; }
  void set_molecule(const Molecule& mol, Real coulomb_k = 1.0);
  [[noreturn]] void throw_last(int rc, const char* what) const;

 private:
  ce_engine* e_ = nullptr;
};

class BatchedRK45 {
 public:
  struct Result {
    std::vector<double> momenta;     // [(lane*n + i)*3 + c] = m_i v_i after redistribution
    std::vector<std::size_t> steps;  // accepted steps per lane
    std::vector<char> converged;     // status == Ok
    std::size_t batch_steps{0};      // max accepted steps over the lanes
    std::vector<double> ker;         // kinetic energy release per lane
    std::vector<SimStatus> status;
    std::vector<std::uint32_t> rejects;
  };

  BatchedRK45(const Molecule& mol, Real coulomb_k, std::size_t lanes, Real rtol, Real atol, int device = 0,
              int precision_mode = kKahanFP64);
  ~BatchedRK45();

  std::size_t lanes() const { return lanes_; }
  std::size_t atoms() const { return n_; }
  void set_lane_geometry(std::size_t lane, const std::vector<Vec3>& pos);
  Result run(const RunConfig& cfg);

 private:
  std::size_t n_, lanes_;
  Real rtol_, atol_;
  int mode_;
  std::unique_ptr<Engine> engine_;
  std::vector<float> pos_;
};

std::vector<RunResult> run_to_convergence_batch(const Molecule& mol, std::vector<State>& states,
                                                const RunConfig& cfg, const IntegratorOptions& opts,
                                                Real coulomb_k = 1.0, int device = 0,
                                                int precision_mode = kKahanFP64);

}  // namespace coulomb::gpu
