// batched_rk45.hpp -- the GPU drop-in for the reference's batched engine.
//
// Built on the reference's own headers (coulomb::engine: coulomb/types.hpp,
// molecule.hpp, system.hpp, driver.hpp, integrator.hpp), so coulomb::Molecule,
// State, RunConfig, RunResult and IntegratorOptions are the reference's types,
// unchanged. Everything this library adds lives in coulomb::gpu. It compiles
// with either setting of the reference's COULOMB_SINGLE_PRECISION (Real = float
// or double), which must match the engine library it is linked beside.
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
// run_to_convergence_batch is the drop-in for the scalar driver
// (src/driver.cpp:7-46, include/coulomb/driver.hpp:69-71) at batch granularity:
// one coulomb::RunResult per state, and each state's velocities become the
// asymptotic (post-redistribution) velocities p_i / m_i. The per-sim status and
// rejection counts, which RunResult does not carry, go to an optional
// BatchStatus. Final positions are not returned (the GPU keeps them on chip).
//
// Errors surface as exceptions on the host side, as in the reference:
// std::invalid_argument for bad arguments, std::runtime_error for device errors.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <vector>

#include "coulomb/driver.hpp"
#include "coulomb/integrator.hpp"
#include "coulomb/molecule.hpp"
#include "coulomb/system.hpp"
#include "coulomb/types.hpp"

struct ce_engine;

namespace coulomb::gpu {

// Precision forms of the GPU engine (include/ce_gpu.h CE_PREC_*).
enum PrecisionMode : int { kFP32 = 0, kKahan = 1, kFP64TimeEnergy = 2, kKahanFP64 = 3 };

// Per-sim outcome (include/ce_gpu.h CE_SIM_*; bench/bench_precision_sweep.cpp:80-85).
enum class SimStatus : std::uint8_t { Ok = 0, RejectLimit = 1, MaxSteps = 2, NonFinite = 3, BadInput = 4 };

// RAII owner of one ce_engine (one per host thread and device).
class Engine {
 public:
  explicit Engine(int device = 0);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;
  ce_engine* handle() const { return e_; }
  void set_molecule(const Molecule& mol, Real coulomb_k = Real{1});
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
  double rtol_, atol_;
  int mode_;
  std::unique_ptr<Engine> engine_;
  std::vector<float> pos_;
};

// What a batch run reports beyond coulomb::RunResult, one entry per state.
struct BatchStatus {
  std::vector<SimStatus> status;
  std::vector<std::uint32_t> rejects;
};

std::vector<RunResult> run_to_convergence_batch(const Molecule& mol, std::vector<State>& states,
                                                const RunConfig& cfg, const IntegratorOptions& opts,
                                                Real coulomb_k = Real{1}, int device = 0,
                                                int precision_mode = kKahanFP64, BatchStatus* extra = nullptr);

}  // namespace coulomb::gpu
