// sampler.cu -- counter-based geometry sampler (include/ce_sampler.h): one
// thread per simulation on the device, the same code on the host. Host
// functions in this unit are compiled with -ffp-contract=off so their double
// arithmetic rounds like the device's explicitly non-fused operations.
#include <cuda_runtime.h>

#include <cmath>

#include "ce_gpu.h"
#include "ce_sampler.h"
#include "philox.h"

namespace {

constexpr double kAmuToMe = 1822.888486209;  // include/coulomb/units.hpp:13
constexpr uint32_t kDefaultAttempts = 1000;

struct MixedTables {
  double radius[CE_MAX_ATOMS + 1];  // radius_coeff * cbrt(n), formed on the host
  double mass_me[8];                // species_amu * 1822.888486209
};

bool valid_ball(int n, const ce_ball_sampler* c) {
  return c && n >= 1 && n <= CE_MAX_ATOMS && c->radius > 0.0 && std::isfinite(c->radius) && c->min_separation >= 0.0 &&
         std::isfinite(c->min_separation);
}

bool valid_mixed(const ce_mixed_sampler* c) {
  return c && c->n_min >= 1 && c->n_max <= CE_MAX_ATOMS && c->n_min <= c->n_max && c->radius_coeff > 0.0 &&
         std::isfinite(c->radius_coeff) && c->min_separation >= 0.0 && c->n_species >= 1 && c->n_species <= 8 &&
         c->q_min <= c->q_max;
}

MixedTables tables(const ce_mixed_sampler* c) {
  MixedTables t{};
  for (int n = 0; n <= CE_MAX_ATOMS; ++n) t.radius[n] = c->radius_coeff * std::cbrt(static_cast<double>(n));
  for (int s = 0; s < 8; ++s) t.mass_me[s] = c->species_amu[s] * kAmuToMe;
  return t;
}

__host__ __device__ inline void ball_one(int n, uint64_t sim, uint64_t idx, double radius, double min_sep,
                                         uint32_t attempts, uint64_t seed, float* pos, double* pos64, uint8_t* flags) {
  double g[3 * CE_MAX_ATOMS];
  const int a = ce::sample_geometry(seed, sim, n, radius, min_sep, attempts, g);
  for (int k = 0; k < 3 * n; ++k) {
    pos[idx * 3 * n + k] = static_cast<float>(g[k]);
    if (pos64) pos64[idx * 3 * n + k] = g[k];
  }
  if (flags) flags[idx] = a < 0 ? 1 : 0;
}

__host__ __device__ inline void mixed_one(uint64_t sim, uint64_t idx, const ce_mixed_sampler& c, const MixedTables& t,
                                          uint8_t* n_atoms, double* mass_me, double* charge, float* pos,
                                          double* pos64, uint8_t* flags) {
  int sp[CE_MAX_ATOMS], q[CE_MAX_ATOMS];
  const int n = ce::sample_molecule(c.seed, sim, c.n_min, c.n_max, c.n_species, c.q_min, c.q_max, sp, q);
  double g[3 * CE_MAX_ATOMS];
  const int a = ce::sample_geometry(c.seed, sim, n, t.radius[n], c.min_separation,
                                    c.max_attempts ? c.max_attempts : kDefaultAttempts, g);
  n_atoms[idx] = static_cast<uint8_t>(n);
  for (int i = 0; i < CE_MAX_ATOMS; ++i) {
    const bool real = i < n;
    mass_me[idx * CE_MAX_ATOMS + i] = real ? t.mass_me[sp[i]] : 1.0;
    charge[idx * CE_MAX_ATOMS + i] = real ? static_cast<double>(q[i]) : 0.0;
    for (int c3 = 0; c3 < 3; ++c3) {
      const double v = real ? g[i * 3 + c3] : 0.0;
      pos[(idx * CE_MAX_ATOMS + i) * 3 + c3] = static_cast<float>(v);
      if (pos64) pos64[(idx * CE_MAX_ATOMS + i) * 3 + c3] = v;
    }
  }
  if (flags) flags[idx] = a < 0 ? 1 : 0;
}

__global__ void ball_kernel(int n, uint64_t first, uint64_t S, double radius, double min_sep, uint32_t attempts,
                            uint64_t seed, float* pos, uint8_t* flags) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < S;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    ball_one(n, first + i, i, radius, min_sep, attempts, seed, pos, nullptr, flags);
}

__global__ void mixed_sample_kernel(uint64_t first, uint64_t S, const ce_mixed_sampler c, const MixedTables t,
                                    uint8_t* n_atoms, double* mass_me, double* charge, float* pos, uint8_t* flags) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < S;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    mixed_one(first + i, i, c, t, n_atoms, mass_me, charge, pos, nullptr, flags);
}

unsigned grid_for(uint64_t S) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t want = (S + 127) / 128;
  const uint64_t cap = static_cast<uint64_t>(sms) * 16;
  return static_cast<unsigned>(want < cap ? want : cap);
}

}  // namespace

extern "C" {

void ce_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  if (!ctr || !key || !out) return;
  const ce::U4 r = ce::philox4x32_10(ce::U4{ctr[0], ctr[1], ctr[2], ctr[3]}, key[0], key[1]);
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
  out[3] = r.w;
}

int ce_sample_ball_device(int n, uint64_t first_sim, uint64_t S, const ce_ball_sampler* cfg, float* pos,
                          uint8_t* flags, void* stream) {
  if (!valid_ball(n, cfg)) return CE_ERR_INVALID;
  if (S == 0) return CE_OK;
  if (!pos) return CE_ERR_INVALID;
  const uint32_t att = cfg->max_attempts ? cfg->max_attempts : kDefaultAttempts;
  ball_kernel<<<grid_for(S), 128, 0, static_cast<cudaStream_t>(stream)>>>(n, first_sim, S, cfg->radius,
                                                                           cfg->min_separation, att, cfg->seed, pos,
                                                                           flags);
  return cudaGetLastError() == cudaSuccess ? CE_OK : CE_ERR_CUDA;
}

int ce_sample_ball_host(int n, uint64_t first_sim, uint64_t S, const ce_ball_sampler* cfg, float* pos,
                        double* pos64, uint8_t* flags) {
  if (!valid_ball(n, cfg)) return CE_ERR_INVALID;
  if (S == 0) return CE_OK;
  if (!pos) return CE_ERR_INVALID;
  const uint32_t att = cfg->max_attempts ? cfg->max_attempts : kDefaultAttempts;
  for (uint64_t i = 0; i < S; ++i)
    ball_one(n, first_sim + i, i, cfg->radius, cfg->min_separation, att, cfg->seed, pos, pos64, flags);
  return CE_OK;
}

int ce_sample_mixed_device(uint64_t first_sim, uint64_t S, const ce_mixed_sampler* cfg, uint8_t* n_atoms,
                           double* mass_me, double* charge, float* pos, uint8_t* flags, void* stream) {
  if (!valid_mixed(cfg)) return CE_ERR_INVALID;
  if (S == 0) return CE_OK;
  if (!n_atoms || !mass_me || !charge || !pos) return CE_ERR_INVALID;
  mixed_sample_kernel<<<grid_for(S), 128, 0, static_cast<cudaStream_t>(stream)>>>(
      first_sim, S, *cfg, tables(cfg), n_atoms, mass_me, charge, pos, flags);
  return cudaGetLastError() == cudaSuccess ? CE_OK : CE_ERR_CUDA;
}

int ce_sample_mixed_host(uint64_t first_sim, uint64_t S, const ce_mixed_sampler* cfg, uint8_t* n_atoms,
                         double* mass_me, double* charge, float* pos, double* pos64, uint8_t* flags) {
  if (!valid_mixed(cfg)) return CE_ERR_INVALID;
  if (S == 0) return CE_OK;
  if (!n_atoms || !mass_me || !charge || !pos) return CE_ERR_INVALID;
  const MixedTables t = tables(cfg);
  for (uint64_t i = 0; i < S; ++i) mixed_one(first_sim + i, i, *cfg, t, n_atoms, mass_me, charge, pos, pos64, flags);
  return CE_OK;
}

}  // extern "C"
