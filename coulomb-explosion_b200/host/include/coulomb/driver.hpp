// driver.hpp -- run configuration and per-run result of the host API.
//
// RunConfig / RunResult / IntegratorOptions / IntegratorKind keep the field
// names and defaults of the reference (include/coulomb/driver.hpp:141-177,
// include/coulomb/integrator.hpp:220-233) so caller code carries over. Added:
// the engine's precision mode and per-sim status.
#pragma once

#include <cstddef>
#include <cstdint>

#include "coulomb/types.hpp"

namespace coulomb {

enum class IntegratorKind { VelocityVerlet, RK45 };

struct IntegratorOptions {
  Real rtol{1e-8};
  Real atol{1e-16};
};

struct RunConfig {
  Real pe_stop_fraction{1e-9};
  bool redistribute_energy{true};
  Real max_dt{1e12};
  std::size_t max_steps{1'000'000};
};

// Precision forms of the GPU engine (include/ce_gpu.h CE_PREC_*).
enum PrecisionMode : int { kFP32 = 0, kKahan = 1, kFP64TimeEnergy = 2, kKahanFP64 = 3 };

// Per-sim outcome (include/ce_gpu.h CE_SIM_*; bench/bench_precision_sweep.cpp:80-85).
enum class SimStatus : std::uint8_t { Ok = 0, RejectLimit = 1, MaxSteps = 2, NonFinite = 3, BadInput = 4 };

struct RunResult {
  std::size_t steps{0};
  Real t_final{0};
  Real energy_initial{0};
  Real pe_final{0};
  Real ke_before_redist{0};
  Real ke_after_redist{0};
  Real redistribution_scale{1};
  bool converged{false};
  SimStatus status{SimStatus::Ok};
  std::size_t rejects{0};
};

}  // namespace coulomb
