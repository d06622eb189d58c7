// closure.cu -- the learned asymptotic closure around the mixed-batch engine
// (include/ce_closure.h): input features and the analytic ballistic base at a
// loose stop, the conservation gate, the fallback merge, and the serving
// pipeline loose run -> features -> network -> gate -> plain rerun of the
// doubtful sims.
//
// The reference stops at PE <= f * PE_0 and moves the residual potential energy
// into kinetic energy by one uniform velocity rescale (src/driver.cpp:38-42).
// Here the engine stops much earlier (f = 0.05) and replaces the missing tail
// of the trajectory by
//   1. the straight-line (ballistic) impulse of every pair from the stop to
//      t -> infinity, in closed form:
//        dp_i = sum_j k q_i q_j (r_ij I0 + w_ij I1),
//        I0 = int_0^inf |r + w t|^-3 dt = 1 / (|r| (|r||w| + r.w)),
//        I1 = int_0^inf t |r + w t|^-3 dt = 1 / (|w| (|r||w| + r.w)),
//      with r_ij = x_i - x_j and w_ij = v_i - v_j at the stop;
//   2. the reference's energy rescale applied to that base (KE = E_0);
//   3. the network's correction, predicted in units of Q, the RMS per-atom
//      size of the analytic step (so the network works at the same relative
//      scale at any loose stop).
// Every sim whose corrected momenta break energy or momentum conservation by
// more than the gate's bounds, or whose correction is implausibly large, is
// integrated again by plain RK45 from its initial geometry.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "ce_closure.h"
#include "ce_gpu.h"
#include "engine.hpp"

namespace {

using bf16 = __nv_bfloat16;

constexpr int kA = CE_MAX_ATOMS;  // atoms per padded row
constexpr int kFeat = CE_CLOSURE_FEATURES;
constexpr int kOut = CE_CLOSURE_OUTPUTS;
constexpr double kMassUnit = 1822.888486209;  // m_e per amu (include/coulomb/units.hpp:11)
constexpr float kInvMassUnit = static_cast<float>(1.0 / kMassUnit);
constexpr float kLogMassScale = 1.0f / 3.5f;  // ln(32.06 amu / 1 amu) ~ 3.47
constexpr int kPerAtom = 12;                  // features per atom
constexpr float kRelRef = 1e-2f;              // typical RMS residual (units of Q)
constexpr float kRelEps = 1e-4f;              // floor of the relative weighting (units of Q)

struct FeatArgs {
  uint64_t S, S_pad;
  const uint8_t* n_atoms;
  const double* mass;
  const double* charge;
  const float* x;
  const float* p;
  const double* e0;
  const double* pe_final;
  const uint8_t* status;
  double k;
  const float* p_true;  // optional [S][10][3]
  float w_scale;
  bf16* feats;     // [S_pad][kFeat]
  float* p_base;   // [S][10][3]
  float* p_scale;  // [S]
  float* target;   // optional [S_pad][kOut]
  float* weight;   // optional [S_pad][kOut]
};

// Features kernel: a block owns a tile of 128 consecutive sims, one per
// thread; the tile's feature rows and base momenta leave through shared memory
// with coalesced stores (a per-thread row write would touch one line per lane).
constexpr int kFT = 128;                 // sims per tile (= threads per block)
constexpr int kFRow = kFeat + 8;         // padded bf16 feature row in shared memory (272 B)
constexpr size_t kFeatSmem = static_cast<size_t>(kFT) * (3 * kA * 4) + static_cast<size_t>(kFT) * kFRow * 2;

// One sim's base momenta (into pb, 30 floats), features (into f, kFeat BF16),
// scale (p_scale[s]) and, for training, targets and weights. live = the row is a
// real sim (else zeros).
__device__ __forceinline__ void feat_one(const FeatArgs& A, uint64_t s, bool live, float* pb, bf16* f) {
  const float* xs = A.x + s * 3 * kA;
  const float* ps = A.p + s * 3 * kA;
  const double* ms = A.mass + s * kA;
  const double* qs = A.charge + s * kA;
  const int n = live ? A.n_atoms[s] : 0;
  bool ok = live && n >= 2 && n <= kA && A.status[s] == CE_SIM_OK;
  float scale_out = 0.0f;
  float x[kA][3], p[kA][3], im[kA], q[kA], dp[kA][3];
  float com[3] = {0.0f, 0.0f, 0.0f};
  float P = 0.0f, Q = 0.0f, L = 0.0f;
  double e0 = 1.0;
  if (ok) {
    // The rows of 30 floats (120 B) are read with 8-byte loads when their base
    // allows it (15 loads a row instead of up to 30; the padded atoms' entries
    // are valid memory and masked below).
    float xr[3 * kA], pr[3 * kA];
    if (((reinterpret_cast<uintptr_t>(xs) | reinterpret_cast<uintptr_t>(ps)) & 7u) == 0u) {
#pragma unroll
      for (int k = 0; k < 3 * kA / 2; ++k) {
        const float2 a = reinterpret_cast<const float2*>(xs)[k];
        const float2 b = reinterpret_cast<const float2*>(ps)[k];
        xr[2 * k] = a.x;
        xr[2 * k + 1] = a.y;
        pr[2 * k] = b.x;
        pr[2 * k + 1] = b.y;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 3 * kA; ++k) {
        xr[k] = xs[k];
        pr[k] = ps[k];
      }
    }
    double msum = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
#pragma unroll
    for (int i = 0; i < kA; ++i) {
      const bool on = i < n;
      const double mi = on ? ms[i] : 1.0;
      // FP32 reciprocal (IEEE, of the mass rounded to FP32): within 2 ulp of the
      // rounded FP64 quotient, and ten FP64 divisions a sim cost the kernel more
      // than its 45 pair terms
      im[i] = on ? __frcp_rn(static_cast<float>(mi)) : 0.0f;
      q[i] = on ? static_cast<float>(qs[i]) : 0.0f;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        x[i][c] = on ? xr[3 * i + c] : 0.0f;
        p[i][c] = on ? pr[3 * i + c] : 0.0f;
      }
      if (on) {
        msum += mi;
        cx += mi * x[i][0];
        cy += mi * x[i][1];
        cz += mi * x[i][2];
      }
    }
    const double imsum = 1.0 / msum;
    com[0] = static_cast<float>(cx * imsum);
    com[1] = static_cast<float>(cy * imsum);
    com[2] = static_cast<float>(cz * imsum);

    // Ballistic pair impulses from the stop to t -> infinity.
#pragma unroll
    for (int i = 0; i < kA; ++i) dp[i][0] = dp[i][1] = dp[i][2] = 0.0f;
    bool bad = false;
    const float kf = static_cast<float>(A.k);
#pragma unroll
    for (int i = 0; i < kA; ++i) {
#pragma unroll
      for (int j = i + 1; j < kA; ++j) {
        if (j < n) {
          const float rx = x[i][0] - x[j][0], ry = x[i][1] - x[j][1], rz = x[i][2] - x[j][2];
          const float wx = p[i][0] * im[i] - p[j][0] * im[j];
          const float wy = p[i][1] * im[i] - p[j][1] * im[j];
          const float wz = p[i][2] * im[i] - p[j][2] * im[j];
          const float a = wx * wx + wy * wy + wz * wz;
          const float b = rx * wx + ry * wy + rz * wz;
          const float c = rx * rx + ry * ry + rz * rz;
          // approximate reciprocal square roots / reciprocal (a few ulp; the
          // features are rounded to BF16 and the base is checked to 3e-5)
          const float rsa = rsqrtf(a), rsc = rsqrtf(c);
          const float sac = (a * rsa) * (c * rsc);
          float g;
          if (b >= 0.0f) {
            g = sac + b;
          } else {  // approaching pair: |r|^2|w|^2 - (r.w)^2 = |r x w|^2 avoids the cancellation
            const float ux = ry * wz - rz * wy, uy = rz * wx - rx * wz, uz = rx * wy - ry * wx;
            g = __fdividef(ux * ux + uy * uy + uz * uz, sac - b);
          }
          const float ig = __fdividef(1.0f, g);
          const float I0 = ig * rsc, I1 = ig * rsa;
          if (!(g > 0.0f) || !isfinite(I0) || !isfinite(I1)) bad = true;
          const float fpair = kf * q[i] * q[j];
          const float tx = fpair * (rx * I0 + wx * I1), ty = fpair * (ry * I0 + wy * I1),
                      tz = fpair * (rz * I0 + wz * I1);
          dp[i][0] += tx;
          dp[i][1] += ty;
          dp[i][2] += tz;
          dp[j][0] -= tx;
          dp[j][1] -= ty;
          dp[j][2] -= tz;
        }
      }
    }
    // Base = (p + dp) rescaled to KE = E_0 (src/driver.cpp:38-42 on the ballistic state).
    double ke = 0.0;
#pragma unroll
    for (int i = 0; i < kA; ++i) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        dp[i][c] += p[i][c];
        ke += 0.5 * static_cast<double>(dp[i][c]) * dp[i][c] * im[i];
      }
    }
    e0 = A.e0[s];
    const float scl = sqrtf(static_cast<float>(e0 / ke));
    double p2 = 0.0, r2 = 0.0, q2 = 0.0;
#pragma unroll
    for (int i = 0; i < kA; ++i) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        dp[i][c] *= scl;
        p2 += static_cast<double>(dp[i][c]) * dp[i][c];
        const double d = static_cast<double>(dp[i][c]) - p[i][c];
        q2 += d * d;
        if (i < n) {
          const double dx = x[i][c] - com[c];
          r2 += dx * dx;
        }
      }
    }
    const float in = 1.0f / static_cast<float>(n);
    P = sqrtf(static_cast<float>(p2) * in);
    Q = sqrtf(static_cast<float>(q2) * in);  // RMS per-atom size of the analytic step p -> p_base
    L = sqrtf(static_cast<float>(r2) * in);
    if (bad || !(ke > 0.0) || !isfinite(scl) || !(P > 0.0f) || !isfinite(P) || !(Q > 0.0f) || !isfinite(Q) ||
        !(L > 0.0f)) {
      ok = false;
      scale_out = __int_as_float(0x7fc00000);  // NaN: the gate sends the sim to plain integration
    } else {
      scale_out = Q;
    }
  }
  if (live) A.p_scale[s] = scale_out;
  if (ok) {
#pragma unroll
    for (int i = 0; i < kA; ++i) {
#pragma unroll
      for (int c = 0; c < 3; ++c) pb[3 * i + c] = dp[i][c];
    }
    // Features: per atom (x - x_com)/L, p/P, (p_base - p)/P, q/3,
    // ln(m/amu)/3.5, 1; then the remaining PE fraction at the stop and n/10;
    // zeros to the padded width.
    const float iL = 1.0f / L, iP = 1.0f / P;
#pragma unroll
    for (int i = 0; i < kA; ++i) {
      const bool on = i < n;
      __nv_bfloat162* f2 = reinterpret_cast<__nv_bfloat162*>(f + kPerAtom * i);
      const float v0 = on ? (x[i][0] - com[0]) * iL : 0.0f, v1 = on ? (x[i][1] - com[1]) * iL : 0.0f;
      const float v2 = on ? (x[i][2] - com[2]) * iL : 0.0f, v3 = on ? p[i][0] * iP : 0.0f;
      const float v4 = on ? p[i][1] * iP : 0.0f, v5 = on ? p[i][2] * iP : 0.0f;
      const float v6 = on ? (dp[i][0] - p[i][0]) * iP : 0.0f, v7 = on ? (dp[i][1] - p[i][1]) * iP : 0.0f;
      const float v8 = on ? (dp[i][2] - p[i][2]) * iP : 0.0f, v9 = on ? q[i] * (1.0f / 3.0f) : 0.0f;
      const float v10 = on ? logf(static_cast<float>(ms[i]) * kInvMassUnit) * kLogMassScale : 0.0f;
      const float v11 = on ? 1.0f : 0.0f;
      f2[0] = __floats2bfloat162_rn(v0, v1);
      f2[1] = __floats2bfloat162_rn(v2, v3);
      f2[2] = __floats2bfloat162_rn(v4, v5);
      f2[3] = __floats2bfloat162_rn(v6, v7);
      f2[4] = __floats2bfloat162_rn(v8, v9);
      f2[5] = __floats2bfloat162_rn(v10, v11);
    }
    __nv_bfloat162* g2 = reinterpret_cast<__nv_bfloat162*>(f + kPerAtom * kA);
    g2[0] = __floats2bfloat162_rn(static_cast<float>(A.pe_final[s] / e0) * 20.0f, static_cast<float>(n) * 0.1f);
#pragma unroll
    for (int c = 1; c < (kFeat - kPerAtom * kA) / 2; ++c) g2[c] = __floats2bfloat162_rn(0.0f, 0.0f);

    if (A.target) {
      // Targets (p_true - p_base)/Q; weights w_scale / (3n) scaled by
      // kRelRef / sqrt(rms^2 + kRelEps^2), rms = the RMS target of the sim, so
      // the loss weighs each sim's relative rather than absolute residual.
      const float iQ = 1.0f / Q;
      const float* pt = A.p_true + s * 3 * kA;
      float* t = A.target + s * kOut;
      float* w = A.weight + s * kOut;
      float ss = 0.0f;
#pragma unroll
      for (int i = 0; i < kA; ++i) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float v = i < n ? (pt[3 * i + c] - dp[i][c]) * iQ : 0.0f;
          t[3 * i + c] = v;
          ss += v * v;
        }
      }
      const float rms2 = ss / static_cast<float>(3 * n);
      const float wv = A.w_scale / static_cast<float>(3 * n) * kRelRef * rsqrtf(rms2 + kRelEps * kRelEps);
#pragma unroll
      for (int i = 0; i < kA; ++i) {
#pragma unroll
        for (int c = 0; c < 3; ++c) w[3 * i + c] = i < n ? wv : 0.0f;
      }
      for (int c = 3 * kA; c < kOut; ++c) t[c] = w[c] = 0.0f;
    }
  } else {
    for (int c = 0; c < 3 * kA; ++c) pb[c] = 0.0f;
    uint4* fz = reinterpret_cast<uint4*>(f);
#pragma unroll
    for (int c = 0; c < kFeat * 2 / 16; ++c) fz[c] = make_uint4(0u, 0u, 0u, 0u);
    if (A.target && s < A.S_pad) {
      float4* t = reinterpret_cast<float4*>(A.target + s * kOut);
      float4* w = reinterpret_cast<float4*>(A.weight + s * kOut);
#pragma unroll
      for (int c = 0; c < kOut / 4; ++c) {
        t[c] = make_float4(0.f, 0.f, 0.f, 0.f);
        w[c] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
  }
}

__global__ void __launch_bounds__(kFT, 4) closure_features_kernel(const FeatArgs A) {
  extern __shared__ __align__(16) uint8_t fsm[];
  float* spb = reinterpret_cast<float*>(fsm);              // [kFT][30]
  bf16* sf = reinterpret_cast<bf16*>(spb + kFT * 3 * kA);  // [kFT][kFRow]
  const int tid = threadIdx.x;
  for (uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * kFT; t0 < A.S_pad;
       t0 += static_cast<uint64_t>(gridDim.x) * kFT) {
    const int rows = t0 < A.S ? static_cast<int>(A.S - t0 < kFT ? A.S - t0 : kFT) : 0;
    feat_one(A, t0 + tid, tid < rows, spb + tid * 3 * kA, sf + tid * kFRow);
    __syncthreads();
    // coalesced stores of the tile: feature rows (all 128, padded rows zero) and base momenta
    {
      uint4* fo = reinterpret_cast<uint4*>(A.feats + t0 * kFeat);
      constexpr int kPerRow = kFeat * 2 / 16;  // uint4 per feature row
      for (int u = tid; u < kFT * kPerRow; u += kFT) {
        const int r = u / kPerRow, j = u - r * kPerRow;
        fo[u] = *reinterpret_cast<const uint4*>(sf + r * kFRow + j * 8);
      }
      for (int k = tid; k < rows * 3 * kA; k += kFT) A.p_base[t0 * 3 * kA + k] = spb[k];
    }
    __syncthreads();
  }
}

struct ApplyArgs {
  uint64_t S;
  const uint8_t* n_atoms;
  const double* mass;
  const double* e0;
  const uint8_t* status_loose;
  const uint32_t* steps_loose;
  const float* p_base;
  const float* p_scale;
  const float* net_out;  // [S_pad][kOut]
  float tol_e, tol_p, tol_c;
  float* momenta;     // [S][10][3]
  double* ker;        // optional
  uint32_t* steps;    // optional
  uint8_t* status;    // optional
  uint8_t* fallback;  // [S]: n for sims sent back to plain integration, else 0
  unsigned long long* counts;  // [0] accepted, [1] fallback
};

__device__ __forceinline__ void warp_count(bool pred, unsigned long long* ctr) {
  const unsigned mask = __activemask();
  const unsigned b = __ballot_sync(mask, pred);
  const int leader = __ffs(mask) - 1;
  if ((threadIdx.x & 31) == leader && b) atomicAdd(ctr, static_cast<unsigned long long>(__popc(b)));
}

__global__ void __launch_bounds__(128) closure_apply_kernel(const ApplyArgs A) {
  for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < A.S;
       s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const int n = A.n_atoms[s];
    float* mo = A.momenta + s * 3 * kA;
    bool accepted = false, fb = false;
    if (n < 2 || n > kA) {  // one-atom and invalid sims: the loose run's answer is final
      for (int c = 0; c < 3 * kA; ++c) mo[c] = 0.0f;
      if (A.ker) A.ker[s] = 0.0;
      if (A.steps) A.steps[s] = A.steps_loose[s];
      if (A.status) A.status[s] = A.status_loose[s];
    } else {
      const float P = A.p_scale[s];
      fb = A.status_loose[s] != CE_SIM_OK || !(P > 0.0f) || !isfinite(P);
      if (!fb) {
        const double* ms = A.mass + s * kA;
        const float* pb = A.p_base + s * 3 * kA;
        const float* o = A.net_out + s * kOut;
        float p[kA][3];
        double ke = 0.0, sx = 0.0, sy = 0.0, sz = 0.0, pabs = 0.0, d2 = 0.0, b2 = 0.0, msum = 0.0;
        float im[kA];
#pragma unroll
        for (int i = 0; i < kA; ++i) {
          const bool on = i < n;
          const double mi = on ? ms[i] : 1.0;
          im[i] = on ? __frcp_rn(static_cast<float>(mi)) : 0.0f;  // as in the features kernel
          if (on) msum += mi;
          double pi2 = 0.0;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float base = on ? pb[3 * i + c] : 0.0f;
            const float d = on ? P * o[3 * i + c] : 0.0f;
            p[i][c] = base + d;
            d2 += static_cast<double>(d) * d;
            b2 += static_cast<double>(base) * base;
            pi2 += static_cast<double>(p[i][c]) * p[i][c];
          }
          ke += 0.5 * pi2 * im[i];
          pabs += sqrtf(static_cast<float>(pi2));  // no cancellation in this sum: FP32 is enough
          sx += p[i][0];
          sy += p[i][1];
          sz += p[i][2];
        }
        const double e0 = A.e0[s];
        const double rho = ke / e0 - 1.0;
        const double mu = sqrt(sx * sx + sy * sy + sz * sz) / pabs;
        const double corr = sqrt(d2 / b2);
        accepted = isfinite(rho) && isfinite(mu) && isfinite(corr) && fabs(rho) <= A.tol_e && mu <= A.tol_p &&
                   corr <= A.tol_c;
        fb = !accepted;
        if (accepted) {
          // Project onto the conservation laws: remove the net momentum (mass
          // weighted, so the centre of mass stays at rest), then rescale to KE = E_0.
          double ke2 = 0.0;
          const double imsum = 1.0 / msum;
#pragma unroll
          for (int i = 0; i < kA; ++i) {
            if (i < n) {
              const double w = ms[i] * imsum;
              p[i][0] -= static_cast<float>(w * sx);
              p[i][1] -= static_cast<float>(w * sy);
              p[i][2] -= static_cast<float>(w * sz);
              ke2 += 0.5 * (static_cast<double>(p[i][0]) * p[i][0] + static_cast<double>(p[i][1]) * p[i][1] +
                            static_cast<double>(p[i][2]) * p[i][2]) * im[i];
            }
          }
          const double sc = sqrt(e0 / ke2);
          double ker = 0.0;
#pragma unroll
          for (int i = 0; i < kA; ++i) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const float v = i < n ? static_cast<float>(sc * p[i][c]) : 0.0f;
              mo[3 * i + c] = v;
              ker += 0.5 * static_cast<double>(v) * v * im[i];
            }
          }
          if (A.ker) A.ker[s] = ker;
          if (A.steps) A.steps[s] = A.steps_loose[s];
          if (A.status) A.status[s] = CE_SIM_OK;
        }
      }
    }
    A.fallback[s] = fb ? static_cast<uint8_t>(n) : static_cast<uint8_t>(0);
    warp_count(accepted, A.counts);
    warp_count(fb, A.counts + 1);
  }
}

struct MergeArgs {
  uint64_t S;
  const uint8_t* fallback;
  const float* fb_momenta;
  const double* fb_ker;
  const uint32_t* fb_steps;
  const uint8_t* fb_status;
  float* momenta;
  double* ker;
  uint32_t* steps;
  uint8_t* status;
};

__global__ void __launch_bounds__(128) closure_merge_kernel(const MergeArgs A) {
  for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < A.S;
       s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    if (!A.fallback[s]) continue;
    const float* src = A.fb_momenta + s * 3 * kA;
    float* dst = A.momenta + s * 3 * kA;
    for (int c = 0; c < 3 * kA; ++c) dst[c] = src[c];
    if (A.ker) A.ker[s] = A.fb_ker[s];
    if (A.steps) A.steps[s] = A.fb_steps[s];
    if (A.status) A.status[s] = A.fb_status[s];
  }
}

int grid_for(uint64_t S, int device) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const uint64_t need = (S + 127) / 128;
  const uint64_t cap = static_cast<uint64_t>(sms) * 16;
  return static_cast<int>(need < cap ? (need > 0 ? need : 1) : cap);
}

uint64_t pad128(uint64_t S) { return (S + 127) / 128 * 128; }

int launch_features(uint64_t S, const ce_mixed_batch* in, double k, const ce_closure_state* st, const float* p_true,
                     float w_scale, void* feats, float* p_base, float* p_scale, float* target, float* weight,
                     cudaStream_t s) {
  FeatArgs A{};
  A.S = S;
  A.S_pad = pad128(S);
  A.n_atoms = in->n_atoms;
  A.mass = in->mass_me;
  A.charge = in->charge;
  A.x = st->positions;
  A.p = st->momenta;
  A.e0 = st->e0;
  A.pe_final = st->pe_final;
  A.status = st->status;
  A.k = k;
  A.p_true = p_true;
  A.w_scale = w_scale;
  A.feats = static_cast<bf16*>(feats);
  A.p_base = p_base;
  A.p_scale = p_scale;
  A.target = target;
  A.weight = weight;
  int dev = 0;
  cudaGetDevice(&dev);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t tiles = A.S_pad / kFT;
  const uint64_t cap = static_cast<uint64_t>(sms) * 4;
  const unsigned grid = static_cast<unsigned>(tiles < cap ? tiles : cap);
  if (cudaFuncSetAttribute(closure_features_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(kFeatSmem)) != cudaSuccess)
    return CE_ERR_CUDA;
  closure_features_kernel<<<grid, kFT, kFeatSmem, s>>>(A);
  return cudaGetLastError() == cudaSuccess ? CE_OK : CE_ERR_CUDA;
}

}  // namespace

struct ce_closure {
  ce_engine* e = nullptr;
  ce_mlp* net = nullptr;
  uint64_t max_batch = 0;
  bool fused = false;  // network runs as one fused forward launch
  uint64_t cap = 0;
  void* arena = nullptr;
  // loose-stop state
  float *xs = nullptr, *ps = nullptr;
  double *e0 = nullptr, *pef = nullptr;
  uint8_t* st = nullptr;
  uint32_t* steps = nullptr;
  // the rest of the integrator state at the loose stop, from which the sims the
  // gate sends back continue
  float *vel = nullptr, *h = nullptr, *comp = nullptr;
  double* t = nullptr;
  uint32_t* rej = nullptr;
  // network
  bf16* feats = nullptr;
  float *out = nullptr, *pbase = nullptr, *pscale = nullptr;
  // fallback
  uint8_t* fb = nullptr;
  float* fb_m = nullptr;
  double* fb_ker = nullptr;
  uint32_t* fb_steps = nullptr;
  uint8_t* fb_st = nullptr;
  unsigned long long* counts = nullptr;
  cudaStream_t last_stream = nullptr;
  std::string err;
};

namespace {
int cfail(ce_closure* c, int code, const std::string& m) {
  if (c) c->err = m;
  return code;
}
}  // namespace

extern "C" {

void ce_closure_default_gate(ce_closure_gate* g) {
  if (!g) return;
  g->tol_energy = 2e-4f;
  g->tol_momentum = 2e-4f;
  g->tol_correction = 0.05f;
}

int ce_closure_features(uint64_t S, const ce_mixed_batch* in, double coulomb_k, const ce_closure_state* st,
                        const float* p_true, float weight_scale, void* feats, float* p_base, float* p_scale,
                        float* target, float* weight, void* stream) {
  if (!in || !st || !feats || !p_base || !p_scale || !in->n_atoms || !in->mass_me || !in->charge || !st->positions ||
      !st->momenta || !st->e0 || !st->pe_final || !st->status)
    return CE_ERR_INVALID;
  if ((target == nullptr) != (weight == nullptr) || (target && !p_true)) return CE_ERR_INVALID;
  if (S == 0) return CE_OK;
  return launch_features(S, in, coulomb_k, st, p_true, weight_scale, feats, p_base, p_scale, target, weight,
                         static_cast<cudaStream_t>(stream));
}

int ce_closure_apply(uint64_t S, const ce_mixed_batch* in, const ce_closure_state* st, const uint32_t* steps_loose,
                     const float* p_base, const float* p_scale, const float* net_out, const ce_closure_gate* gate,
                     const ce_outputs* out, uint8_t* fallback, unsigned long long* counts, void* stream) {
  if (!in || !st || !steps_loose || !p_base || !p_scale || !net_out || !gate || !out || !out->momenta || !fallback ||
      !counts || !in->n_atoms || !in->mass_me || !st->e0 || !st->status)
    return CE_ERR_INVALID;
  if (S == 0) return CE_OK;
  ApplyArgs A{};
  A.S = S;
  A.n_atoms = in->n_atoms;
  A.mass = in->mass_me;
  A.e0 = st->e0;
  A.status_loose = st->status;
  A.steps_loose = steps_loose;
  A.p_base = p_base;
  A.p_scale = p_scale;
  A.net_out = net_out;
  A.tol_e = gate->tol_energy;
  A.tol_p = gate->tol_momentum;
  A.tol_c = gate->tol_correction;
  A.momenta = out->momenta;
  A.ker = out->ker;
  A.steps = out->steps;
  A.status = out->status;
  A.fallback = fallback;
  A.counts = counts;
  int dev = 0;
  cudaGetDevice(&dev);
  closure_apply_kernel<<<grid_for(S, dev), 128, 0, static_cast<cudaStream_t>(stream)>>>(A);
  return cudaGetLastError() == cudaSuccess ? CE_OK : CE_ERR_CUDA;
}

int ce_closure_create(ce_closure** out, ce_engine* e, ce_mlp* net, uint64_t max_sims) {
  if (!out || !e || !net || max_sims == 0 || max_sims >= (1ull << 32)) return CE_ERR_INVALID;
  *out = nullptr;
  int in_dim = 0, out_dim = 0, hidden = 0, depth = 0;
  uint64_t mb = 0;
  if (ce_mlp_shape(net, &in_dim, &hidden, &depth, &out_dim, &mb) != CE_OK || in_dim != kFeat || out_dim != kOut)
    return CE_ERR_INVALID;
  ce_closure* c = new ce_closure;
  c->e = e;
  c->net = net;
  c->max_batch = mb;
  c->fused = hidden % 32 == 0 && depth + 1 <= 8;
  c->cap = max_sims;
  const uint64_t S = max_sims, Sp = pad128(max_sims);
  auto al = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  const size_t sizes[] = {al(S * 3 * kA * 4), al(S * 3 * kA * 4), al(S * 8), al(S * 8), al(S), al(S * 4),
                          al(Sp * kFeat * 2), al(Sp * kOut * 4), al(S * 3 * kA * 4), al(S * 4),
                          al(S), al(S * 3 * kA * 4), al(S * 8), al(S * 4), al(S), al(2 * 8),
                          al(S * 3 * kA * 4), al(S * 4), al(S * 6 * kA * 4), al(S * 8), al(S * 4)};
  constexpr int kSlots = sizeof(sizes) / sizeof(sizes[0]);
  size_t total = 0;
  for (size_t b : sizes) total += b;
  if (cudaSetDevice(e->device) != cudaSuccess || cudaMalloc(&c->arena, total) != cudaSuccess) {
    delete c;
    return CE_ERR_CUDA;
  }
  char* p = static_cast<char*>(c->arena);
  void* slot[kSlots];
  for (int i = 0; i < kSlots; ++i) {
    slot[i] = p;
    p += sizes[i];
  }
  c->xs = static_cast<float*>(slot[0]);
  c->ps = static_cast<float*>(slot[1]);
  c->e0 = static_cast<double*>(slot[2]);
  c->pef = static_cast<double*>(slot[3]);
  c->st = static_cast<uint8_t*>(slot[4]);
  c->steps = static_cast<uint32_t*>(slot[5]);
  c->feats = static_cast<bf16*>(slot[6]);
  c->out = static_cast<float*>(slot[7]);
  c->pbase = static_cast<float*>(slot[8]);
  c->pscale = static_cast<float*>(slot[9]);
  c->fb = static_cast<uint8_t*>(slot[10]);
  c->fb_m = static_cast<float*>(slot[11]);
  c->fb_ker = static_cast<double*>(slot[12]);
  c->fb_steps = static_cast<uint32_t*>(slot[13]);
  c->fb_st = static_cast<uint8_t*>(slot[14]);
  c->counts = static_cast<unsigned long long*>(slot[15]);
  c->vel = static_cast<float*>(slot[16]);
  c->h = static_cast<float*>(slot[17]);
  c->comp = static_cast<float*>(slot[18]);
  c->t = static_cast<double*>(slot[19]);
  c->rej = static_cast<uint32_t*>(slot[20]);
  // padded network rows stay finite
  cudaMemset(c->out, 0, sizes[7]);
  const int rc = ce_reserve_mixed(e, max_sims);
  if (rc != CE_OK || cudaDeviceSynchronize() != cudaSuccess) {
    cudaFree(c->arena);
    delete c;
    return rc != CE_OK ? rc : CE_ERR_CUDA;
  }
  *out = c;
  return CE_OK;
}

void ce_closure_destroy(ce_closure* c) {
  if (!c) return;
  if (c->arena) {
    cudaSetDevice(c->e->device);
    cudaFree(c->arena);
  }
  delete c;
}

const char* ce_closure_last_error(const ce_closure* c) { return c ? c->err.c_str() : "null closure"; }

int ce_closure_serve(ce_closure* c, uint64_t S, const ce_mixed_batch* in, double coulomb_k, const ce_run_config* cfg,
                     double loose_pe_stop, const ce_closure_gate* gate, const ce_outputs* out, void* stream) {
  if (!c) return CE_ERR_INVALID;
  if (!in || !cfg || !gate || !out || !out->momenta) return cfail(c, CE_ERR_INVALID, "ce_closure_serve: NULL argument");
  if (S > c->cap) return cfail(c, CE_ERR_INVALID, "ce_closure_serve: S exceeds the closure's max_sims");
  if (!(loose_pe_stop > cfg->pe_stop_fraction) || !(loose_pe_stop < 1.0))
    return cfail(c, CE_ERR_INVALID, "ce_closure_serve: loose_pe_stop must lie in (cfg->pe_stop_fraction, 1)");
  if (S == 0) return CE_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaSetDevice(c->e->device) != cudaSuccess) return cfail(c, CE_ERR_CUDA, "cudaSetDevice");
  c->last_stream = s;
  if (cudaMemsetAsync(c->counts, 0, 2 * sizeof(unsigned long long), s) != cudaSuccess)
    return cfail(c, CE_ERR_CUDA, "memset counts");

  // 1. integrate every sim to the loose stop, without the energy rescale, and
  // keep its integrator state there
  ce_run_config loose = *cfg;
  loose.pe_stop_fraction = loose_pe_stop;
  loose.redistribute_energy = 0;
  ce_outputs lo{};
  lo.momenta = c->ps;
  lo.pe_final = c->pef;
  lo.status = c->st;
  const ce_sim_state saved{c->xs, c->vel, c->h, c->t, c->steps, c->rej, c->e0, c->comp};
  const int sched = c->e->tuned_schedule;
  int rc = ce::run_mixed_device(c->e, S, in, coulomb_k, &loose, &lo, sched, stream, false, nullptr, &saved);
  if (rc != CE_OK) return cfail(c, rc, std::string("loose run: ") + ce_last_error(c->e));

  // 2. features and the ballistic base
  const ce_closure_state st{c->xs, c->ps, c->e0, c->pef, c->st};
  rc = launch_features(S, in, coulomb_k, &st, nullptr, 0.0f, c->feats, c->pbase, c->pscale, nullptr, nullptr, s);
  if (rc != CE_OK) return cfail(c, rc, "features launch");

  // 3. network correction: one fused launch over all rows when the network
  // allows it, else chunks of at most max_batch rows
  const uint64_t Sp = pad128(S);
  const uint64_t mb = c->fused ? Sp : c->max_batch;
  for (uint64_t off = 0; off < Sp; off += mb) {
    const uint64_t B = Sp - off < mb ? Sp - off : mb;
    rc = ce_mlp_forward(c->net, c->feats + off * kFeat, B, c->out + off * kOut, stream);
    if (rc != CE_OK) return cfail(c, rc, std::string("network: ") + ce_mlp_last_error(c->net));
  }

  // 4. gate; accepted sims are final, the rest are marked for plain integration
  rc = ce_closure_apply(S, in, &st, c->steps, c->pbase, c->pscale, c->out, gate, out, c->fb, c->counts, stream);
  if (rc != CE_OK) return cfail(c, rc, "apply launch");

  // 5. plain RK45 for the marked sims (n = 0 for the rest), continued from the
  // loose-stop state: bit for bit the result of an uninterrupted plain run. A
  // sim whose loose run did not finish CE_SIM_OK (saved h = 0) restarts from rest.
  const ce_mixed_batch fbin{c->fb, in->mass_me, in->charge, in->pos};
  ce_outputs fo{};
  fo.momenta = c->fb_m;
  fo.ker = c->fb_ker;
  fo.steps = c->fb_steps;
  fo.status = c->fb_st;
  rc = ce::run_mixed_device(c->e, S, &fbin, coulomb_k, cfg, &fo, sched, stream, /*skip_empty=*/true, &saved, nullptr);
  if (rc != CE_OK) return cfail(c, rc, std::string("fallback run: ") + ce_last_error(c->e));
  MergeArgs M{S, c->fb, c->fb_m, c->fb_ker, c->fb_steps, c->fb_st, out->momenta, out->ker, out->steps, out->status};
  closure_merge_kernel<<<grid_for(S, c->e->device), 128, 0, s>>>(M);
  if (cudaGetLastError() != cudaSuccess) return cfail(c, CE_ERR_CUDA, "merge launch");
  return CE_OK;
}

int ce_closure_fallback_flags(const ce_closure* c, uint8_t* dst, uint64_t S, void* stream) {
  if (!c || !dst || S > c->cap) return CE_ERR_INVALID;
  if (S == 0) return CE_OK;
  return cudaMemcpyAsync(dst, c->fb, S, cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)) == cudaSuccess
             ? CE_OK
             : CE_ERR_CUDA;
}

int ce_closure_counts(ce_closure* c, uint64_t* accepted, uint64_t* fallback) {
  if (!c) return CE_ERR_INVALID;
  unsigned long long h[2] = {0, 0};
  if (cudaSetDevice(c->e->device) != cudaSuccess ||
      cudaMemcpyAsync(h, c->counts, sizeof h, cudaMemcpyDeviceToHost, c->last_stream) != cudaSuccess ||
      cudaStreamSynchronize(c->last_stream) != cudaSuccess)
    return cfail(c, CE_ERR_CUDA, "ce_closure_counts: copy failed");
  if (accepted) *accepted = h[0];
  if (fallback) *fallback = h[1];
  return ce_mlp_check(c->net, c->last_stream);
}

}  // extern "C"
