// philox.h -- Philox4x32-10 counter-based generator and the geometry draws built
// on it, shared by the device sampler kernels and their host twins (the same
// integer and IEEE double operations in the same order, so both produce
// bit-identical geometries).
//
// Philox4x32-10 is the published generator of Salmon, Moraes, Dror and Shaw,
// "Parallel random numbers: as easy as 1, 2, 3" (SC 2011): ten rounds of
// (hi, lo) = mulhilo(M, x) mixing on a 128-bit counter under a 64-bit key that
// is bumped by the Weyl constants between rounds.
//
// Geometry scheme (no counterpart in the reference, whose UniformSphereSampler
// redraws atom by atom from one mt19937_64 stream, src/sampler.cpp:28-57):
// every atom is drawn independently and uniformly in the ball by cube rejection
// (acceptance pi/6), and a geometry with any pair closer than the minimum
// separation is redrawn whole. Draw (sim s, attempt a, atom i, try t) uses
// counter (lo32(s), hi32(s), a, i << 8 | t) under key (lo32(seed), hi32(seed));
// coordinate c = R (2 u_c - 1) with u_c = word_c / 2^32.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define CE_HD __host__ __device__ __forceinline__
#else
#define CE_HD inline
#endif

namespace ce {

struct U4 {
  uint32_t x, y, z, w;
};

CE_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  const uint64_t p = static_cast<uint64_t>(a) * static_cast<uint64_t>(b);
  *hi = static_cast<uint32_t>(p >> 32);
  *lo = static_cast<uint32_t>(p);
}

CE_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(M0, c.x, &hi0, &lo0);
    mulhilo32(M1, c.z, &hi1, &lo1);
    const U4 n = {hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// IEEE double ops that a device compiler may not contract into FMAs, so the
// host twin (built with -ffp-contract=off) rounds identically.
#if defined(__CUDA_ARCH__)
CE_HD double dmul(double a, double b) { return __dmul_rn(a, b); }
CE_HD double dadd(double a, double b) { return __dadd_rn(a, b); }
CE_HD double dsub(double a, double b) { return __dsub_rn(a, b); }
#else
CE_HD double dmul(double a, double b) { return a * b; }
CE_HD double dadd(double a, double b) { return a + b; }
CE_HD double dsub(double a, double b) { return a - b; }
#endif

constexpr int kMaxPointTries = 64;

// One geometry of n (<= 16) atoms for sim `sim`: out[i*3 + c]. Returns the
// attempt index that succeeded, or -1 after max_attempts whole-geometry
// redraws (out then holds the last draw).
CE_HD int sample_geometry(uint64_t seed, uint64_t sim, int n, double radius, double min_sep, uint32_t max_attempts,
                          double* out) {
  const uint32_t k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
  const uint32_t s0 = static_cast<uint32_t>(sim), s1 = static_cast<uint32_t>(sim >> 32);
  const double r2 = dmul(radius, radius);
  const double m2 = dmul(min_sep, min_sep);
  const double inv32 = 2.3283064365386963e-10;  // 2^-32
  for (uint32_t a = 0; a < max_attempts; ++a) {
    bool ok = true;
    for (int i = 0; i < n && ok; ++i) {
      bool placed = false;
      for (int t = 0; t < kMaxPointTries; ++t) {
        const U4 w = philox4x32_10(U4{s0, s1, a, (static_cast<uint32_t>(i) << 8) | static_cast<uint32_t>(t)}, k0, k1);
        const double px = dmul(radius, dsub(dmul(2.0, dmul(static_cast<double>(w.x), inv32)), 1.0));
        const double py = dmul(radius, dsub(dmul(2.0, dmul(static_cast<double>(w.y), inv32)), 1.0));
        const double pz = dmul(radius, dsub(dmul(2.0, dmul(static_cast<double>(w.z), inv32)), 1.0));
        if (dadd(dadd(dmul(px, px), dmul(py, py)), dmul(pz, pz)) <= r2) {
          out[i * 3 + 0] = px;
          out[i * 3 + 1] = py;
          out[i * 3 + 2] = pz;
          placed = true;
          break;
        }
      }
      if (!placed) ok = false;
    }
    for (int i = 0; i < n && ok; ++i)
      for (int j = i + 1; j < n && ok; ++j) {
        const double dx = dsub(out[i * 3 + 0], out[j * 3 + 0]);
        const double dy = dsub(out[i * 3 + 1], out[j * 3 + 1]);
        const double dz = dsub(out[i * 3 + 2], out[j * 3 + 2]);
        if (dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz)) < m2) ok = false;
      }
    if (ok) return static_cast<int>(a);
  }
  return -1;
}

// Uniform integer in [0, k) from one 32-bit word (multiply-shift).
CE_HD uint32_t uniform_index(uint32_t word, uint32_t k) {
  return static_cast<uint32_t>((static_cast<uint64_t>(word) * k) >> 32);
}

// Molecule of a mixed-population sim: atom count in [n_min, n_max], then per
// atom a species index in [0, n_species) and a charge in [q_min, q_max]
// (counter (lo32(s), hi32(s), 0xFFFFFFFF, 0) for the count, (..., 1 + i) per atom).
CE_HD int sample_molecule(uint64_t seed, uint64_t sim, int n_min, int n_max, int n_species, int q_min, int q_max,
                          int* species, int* charge) {
  const uint32_t k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32);
  const uint32_t s0 = static_cast<uint32_t>(sim), s1 = static_cast<uint32_t>(sim >> 32);
  const U4 w = philox4x32_10(U4{s0, s1, 0xFFFFFFFFu, 0u}, k0, k1);
  const int n = n_min + static_cast<int>(uniform_index(w.x, static_cast<uint32_t>(n_max - n_min + 1)));
  for (int i = 0; i < n; ++i) {
    const U4 v = philox4x32_10(U4{s0, s1, 0xFFFFFFFFu, 1u + static_cast<uint32_t>(i)}, k0, k1);
    species[i] = static_cast<int>(uniform_index(v.x, static_cast<uint32_t>(n_species)));
    charge[i] = q_min + static_cast<int>(uniform_index(v.y, static_cast<uint32_t>(q_max - q_min + 1)));
  }
  return n;
}

}  // namespace ce
