/*
 * ce_sampler.h -- initial-geometry sampler of libce_gpu.so (device kernels and
 * bit-identical host twins).
 *
 * Replaces, for the GPU path, the reference's Sampler strategy
 * (include/coulomb/sampler.hpp:23-72, UniformSphereSampler, src/sampler.cpp:17-57),
 * which draws atom by atom from one sequential mt19937_64 stream. The engine's
 * sampler is counter-based (Philox4x32-10), so sim s's geometry depends only on
 * (seed, s): any chunk of a population can be generated independently, on the
 * device or the host, and regenerated later (resumable by chunk index).
 * Distribution: each atom uniform in the ball (cube rejection), the whole
 * geometry redrawn while any pair is closer than min_separation; every
 * simulation starts at rest. (The reference's sequential per-atom redraw gives
 * a different distribution; the host C++ mirror of the reference sampler is in
 * coulomb-explosion_b200/host.)
 *
 * Per-sim flags: 0 = ok, 1 = no valid geometry within max_attempts redraws.
 */
#ifndef CE_SAMPLER_H
#define CE_SAMPLER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ce_ball_sampler {
  uint64_t seed;
  double radius;         /* ball radius (bohr)                               */
  double min_separation; /* reject geometries with any pair closer (bohr)    */
  uint32_t max_attempts; /* whole-geometry redraws before flagging; 0 = 1000 */
} ce_ball_sampler;

/* Mixed population: atom count uniform in [n_min, n_max] (2..10), each atom's
 * species uniform over species_amu[0..n_species), integer charge uniform in
 * [q_min, q_max], ball radius radius_coeff * n^(1/3). */
typedef struct ce_mixed_sampler {
  uint64_t seed;
  int32_t n_min, n_max;
  double radius_coeff;
  double min_separation;
  uint32_t max_attempts;
  int32_t q_min, q_max;
  int32_t n_species;
  double species_amu[8];
} ce_mixed_sampler;

/* n atoms per sim, sims [first_sim, first_sim + S): pos [S][n][3] float.
 * flags [S] may be NULL. Device: pointers on the current device, async on
 * `stream`. Host: pos64 [S][n][3] double (may be NULL) receives the unrounded
 * draws. */
int ce_sample_ball_device(int n, uint64_t first_sim, uint64_t S, const ce_ball_sampler* cfg, float* pos,
                          uint8_t* flags, void* stream);
int ce_sample_ball_host(int n, uint64_t first_sim, uint64_t S, const ce_ball_sampler* cfg, float* pos,
                        double* pos64, uint8_t* flags);

/* Mixed rows padded to 10 atoms (the ce_mixed_batch layout of ce_gpu.h):
 * n_atoms [S], mass_me [S][10] (padding 1.0), charge [S][10] (padding 0),
 * pos [S][10][3] (padding 0). */
int ce_sample_mixed_device(uint64_t first_sim, uint64_t S, const ce_mixed_sampler* cfg, uint8_t* n_atoms,
                           double* mass_me, double* charge, float* pos, uint8_t* flags, void* stream);
int ce_sample_mixed_host(uint64_t first_sim, uint64_t S, const ce_mixed_sampler* cfg, uint8_t* n_atoms,
                         double* mass_me, double* charge, float* pos, double* pos64, uint8_t* flags);

/* The generator itself: Philox4x32-10 of counter ctr[4] under key[2] (for
 * reproducing draws and checking the published known-answer vectors). */
void ce_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint32_t* out);

#ifdef __cplusplus
}
#endif
#endif /* CE_SAMPLER_H */
