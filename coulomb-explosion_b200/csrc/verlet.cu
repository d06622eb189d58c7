// verlet.cu -- the Velocity Verlet strategy (IntegratorKind::VelocityVerlet,
// src/integrators.cpp:14-47) under the convergence driver
// (run_to_convergence, src/driver.cpp:7-46), one thread per simulation.
//
// Fixed step dt = RunConfig::max_dt (a fixed-step scheme takes exactly the dt it
// is given, include/coulomb/integrator.hpp:24-28):
//   x += v dt + a (dt/2 * dt);  a' = a(x);  v += (a + a') (dt/2);  a = a'
// until PE <= pe_stop_fraction * PE_0 or max_steps, then the reference's energy
// rescale (driver.cpp:38-42). Every operation is an explicitly rounded IEEE FP32
// operation in the reference's order (no contraction into FMA, correctly rounded
// division and square root), so the GPU result equals the reference's scalar f32
// engine bit for bit: forces as CoulombForce::accelerations
// (src/system.cpp:5-29), potential as CoulombForce::potential_energy
// (system.cpp:31-41), kinetic energy as system.cpp:43-49.
#include <cuda_runtime.h>

#include <cmath>

#include "ce_gpu.h"
#include "engine.hpp"

namespace {

struct VVParams {
  const float* pos;
  float* momenta;
  double* ker;
  uint32_t* steps;
  uint8_t* status;
  double* t_final;
  double* pe_final;
  double* ke_before;
  uint64_t S;
  float dt;
  float pe_stop_f;
  uint64_t max_steps;
  int redistribute;
};

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
// dot(r, r) = (x*x + y*y) + z*z
__device__ __forceinline__ float dot3(float x, float y, float z) { return fa(fa(fm(x, x), fm(y, y)), fm(z, z)); }

template <int N>
__device__ __forceinline__ void vv_accel(const ce::FixedMol& M, const float (&mf)[N], const float (&x)[N][3],
                                         float (&a)[N][3]) {
#pragma unroll
  for (int i = 0; i < N; ++i) a[i][0] = a[i][1] = a[i][2] = 0.0f;
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int j = i + 1; j < N; ++j) {
      const float rx = fs(x[i][0], x[j][0]), ry = fs(x[i][1], x[j][1]), rz = fs(x[i][2], x[j][2]);
      const float d2 = dot3(rx, ry, rz);
      const float inv = __fdiv_rn(1.0f, __fsqrt_rn(d2));
      const float inv3 = __fdiv_rn(inv, d2);
      const float sc = fm(fm(fm(M.k, M.q[i]), M.q[j]), inv3);
      const float fx = fm(rx, sc), fy = fm(ry, sc), fz = fm(rz, sc);
      a[i][0] = fa(a[i][0], fx);
      a[i][1] = fa(a[i][1], fy);
      a[i][2] = fa(a[i][2], fz);
      a[j][0] = fs(a[j][0], fx);
      a[j][1] = fs(a[j][1], fy);
      a[j][2] = fs(a[j][2], fz);
    }
  }
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const float im = __fdiv_rn(1.0f, mf[i]);
    a[i][0] = fm(a[i][0], im);
    a[i][1] = fm(a[i][1], im);
    a[i][2] = fm(a[i][2], im);
  }
}

template <int N>
__device__ __forceinline__ float vv_pe(const ce::FixedMol& M, const float (&x)[N][3]) {
  float u = 0.0f;
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int j = i + 1; j < N; ++j) {
      const float rx = fs(x[i][0], x[j][0]), ry = fs(x[i][1], x[j][1]), rz = fs(x[i][2], x[j][2]);
      u = fa(u, __fdiv_rn(fm(fm(M.k, M.q[i]), M.q[j]), __fsqrt_rn(dot3(rx, ry, rz))));
    }
  }
  return u;
}

template <int N>
__device__ __forceinline__ float vv_ke(const float (&mf)[N], const float (&v)[N][3]) {
  float t = 0.0f;
#pragma unroll
  for (int i = 0; i < N; ++i) t = fa(t, fm(fm(0.5f, mf[i]), dot3(v[i][0], v[i][1], v[i][2])));
  return t;
}

template <int N>
__global__ void __launch_bounds__(128) verlet_kernel(const VVParams P, const ce::FixedMol M) {
  float mf[N];
#pragma unroll
  for (int i = 0; i < N; ++i) mf[i] = static_cast<float>(M.mass[i]);
  for (uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; s < P.S;
       s += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    float x[N][3], v[N][3], a[N][3], na[N][3];
    const float* src = P.pos + s * (3ull * N);
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        x[i][c] = src[3 * i + c];
        v[i][c] = 0.0f;
      }
    const float pe0 = vv_pe<N>(M, x);
    const float e0 = fa(pe0, vv_ke<N>(mf, v));
    const float pe_stop = fm(P.pe_stop_f, pe0);
    float pe = pe0, t = 0.0f;
    uint64_t steps = 0;
    bool converged = false, have_a = false;
    int status = isfinite(pe0) ? CE_SIM_OK : CE_SIM_NONFINITE;
    const float dt = P.dt;
    const float half_dt2 = fm(fm(0.5f, dt), dt);
    const float half_dt = fm(0.5f, dt);
    while (status == CE_SIM_OK && pe > pe_stop) {
      if (steps >= P.max_steps) {
        converged = false;
        break;
      }
      if (!have_a) {
        vv_accel<N>(M, mf, x, a);
        have_a = true;
      }
#pragma unroll
      for (int i = 0; i < N; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) x[i][c] = fa(x[i][c], fa(fm(v[i][c], dt), fm(a[i][c], half_dt2)));
      vv_accel<N>(M, mf, x, na);
#pragma unroll
      for (int i = 0; i < N; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          v[i][c] = fa(v[i][c], fm(fa(a[i][c], na[i][c]), half_dt));
          a[i][c] = na[i][c];
        }
      t = fa(t, dt);
      ++steps;
      pe = vv_pe<N>(M, x);
      converged = true;
    }
    if (steps == 0 && pe <= pe_stop) converged = true;  // already at or below the stop
    if (status == CE_SIM_OK && !converged) status = CE_SIM_MAX_STEPS;
    const float ke_before = vv_ke<N>(mf, v);
    if (P.redistribute && ke_before > 0.0f) {
      const float sc = __fsqrt_rn(__fdiv_rn(e0, ke_before));
#pragma unroll
      for (int i = 0; i < N; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) v[i][c] = fm(v[i][c], sc);
    }
    float* dst = P.momenta + s * (3ull * N);
    double ker = 0.0;
    bool finite = true;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float p = fm(v[i][c], mf[i]);  // Vec3 * m, as the reference's callers form p
        dst[3 * i + c] = p;
        finite = finite && isfinite(p);
        ker += 0.5 * static_cast<double>(p) * p / M.mass[i];
      }
    if (status == CE_SIM_OK && !finite) status = CE_SIM_NONFINITE;
    if (P.ker) P.ker[s] = ker;
    if (P.steps) P.steps[s] = static_cast<uint32_t>(steps > 0xffffffffull ? 0xffffffffull : steps);
    if (P.status) P.status[s] = static_cast<uint8_t>(status);
    if (P.t_final) P.t_final[s] = static_cast<double>(t);
    if (P.pe_final) P.pe_final[s] = static_cast<double>(pe);
    if (P.ke_before) P.ke_before[s] = static_cast<double>(ke_before);
  }
}

using VVKernel = void (*)(const VVParams, const ce::FixedMol);

VVKernel vv_kernel_for(int n) {
  switch (n) {
    case 1: return verlet_kernel<1>;
    case 2: return verlet_kernel<2>;
    case 3: return verlet_kernel<3>;
    case 4: return verlet_kernel<4>;
    case 5: return verlet_kernel<5>;
    case 6: return verlet_kernel<6>;
    case 7: return verlet_kernel<7>;
    case 8: return verlet_kernel<8>;
    case 9: return verlet_kernel<9>;
    case 10: return verlet_kernel<10>;
    default: return nullptr;
  }
}

}  // namespace

extern "C" int ce_run_verlet_device(ce_engine* e, uint64_t S, const float* pos, const ce_run_config* cfg,
                                    const ce_outputs* out, void* stream) {
  if (!e) return CE_ERR_INVALID;
  e->last_launches = 0;
  if (!cfg) return ce::fail(e, CE_ERR_INVALID, "ce_run_verlet_device: cfg is NULL");
  if (!(cfg->max_dt > 0.0) || !std::isfinite(cfg->max_dt))
    return ce::fail(e, CE_ERR_INVALID, "ce_run_verlet_device: max_dt (the fixed step) must be finite and > 0");
  if (!std::isfinite(cfg->pe_stop_fraction))
    return ce::fail(e, CE_ERR_INVALID, "ce_run_verlet_device: pe_stop_fraction must be finite");
  if (cfg->precision_mode != 0)
    return ce::fail(e, CE_ERR_INVALID, "ce_run_verlet_device: precision modes apply to the DP5(4) path only");
  if (!e->has_mol) return ce::fail(e, CE_ERR_STATE, "ce_run_verlet_device: no molecule set (ce_set_molecule)");
  if (S == 0) return CE_OK;
  if (!pos || !out || !out->momenta)
    return ce::fail(e, CE_ERR_INVALID, "ce_run_verlet_device: pos and out->momenta are required");
  if (S > (1ull << 40)) return ce::fail(e, CE_ERR_INVALID, "ce_run_verlet_device: S too large");
  cudaError_t st = cudaSetDevice(e->device);
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "cudaSetDevice");
  const VVKernel fn = vv_kernel_for(e->n);
  if (!fn) return ce::fail(e, CE_ERR_INVALID, "ce_run_verlet_device: no kernel for this atom count");
  VVParams P{};
  P.pos = pos;
  P.momenta = out->momenta;
  P.ker = out->ker;
  P.steps = out->steps;
  P.status = out->status;
  P.t_final = out->t_final;
  P.pe_final = out->pe_final;
  P.ke_before = out->ke_before;
  P.S = S;
  P.dt = static_cast<float>(cfg->max_dt);
  P.pe_stop_f = static_cast<float>(cfg->pe_stop_fraction);
  P.max_steps = cfg->max_steps;
  P.redistribute = cfg->redistribute_energy ? 1 : 0;
  const uint64_t need = (S + 127) / 128;
  const uint64_t cap = static_cast<uint64_t>(e->sms) * 8;
  const unsigned grid = static_cast<unsigned>(need < cap ? need : cap);
  fn<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(P, e->mol);
  st = cudaGetLastError();
  if (st != cudaSuccess) return ce::cuda_fail(e, st, "verlet_kernel launch");
  e->last_launches = 1;
  return CE_OK;
}
