// hwy/highway.h -- a minimal, project-written stand-in for the subset of the
// Google Highway 1.2.0 API that the reference's batched engine uses.
//
// TEST INFRASTRUCTURE ONLY (oracle/). Google Highway is an external library the
// reference fetches at configure time (bench/CMakeLists.txt:19-23,
// examples/CMakeLists.txt:12-16); it is not installed in this image. This header
// lets the reference's UNMODIFIED include/coulomb/batched_force.hpp and
// include/coulomb/batched_integrator.hpp compile, so that BatchedRK45<T> (the
// reference's SIMD hot path) can serve as the timed CPU baseline and as a parity
// oracle. It is not Highway source: it implements only the elementwise contract
// of the names the reference calls (hn::Lanes, Set, Zero, Load, LoadU, Store,
// StoreU, Add, Sub, Mul, Div, MulAdd, Sqrt, Abs, Max, ScalableTag and the
// HWY_NAMESPACE macro), with Highway's semantics on x86:
//
//   * vector width = the widest the translation unit is compiled for, as with
//     Highway's static dispatch under -march=<isa>: 512-bit with AVX-512F
//     (K = 16 float / 8 double), 256-bit with AVX2+FMA (K = 8 / 4), else 128-bit
//     SSE2 (K = 4 / 2);
//   * MulAdd(m, x, a) = m * x + a as ONE fused multiply-add where the target has
//     FMA (Highway's AVX2/AVX-512 targets), unfused multiply then add on SSE2
//     (Highway's SSE2/SSSE3/SSE4 targets have no FMA either);
//   * Div and Sqrt are the IEEE-correctly-rounded vector instructions;
//   * Max is the x86 max instruction; Abs clears the sign bit;
//   * Load/Store require alignment to the vector size, LoadU/StoreU do not.
#pragma once

#include <immintrin.h>

#include <cstddef>

#include "hwy/aligned_allocator.h"

#if defined(__AVX512F__)
#define HWY_NAMESPACE N_SHIM_AVX512
#elif defined(__AVX2__) && defined(__FMA__)
#define HWY_NAMESPACE N_SHIM_AVX2
#else
#define HWY_NAMESPACE N_SHIM_SSE2
#endif

namespace hwy {
namespace HWY_NAMESPACE {

// Native vector register type per lane type.
template <class T>
struct NativeVec;

#if defined(__AVX512F__)
inline constexpr std::size_t kVectorBytes = 64;
template <>
struct NativeVec<float> {
  using type = __m512;
};
template <>
struct NativeVec<double> {
  using type = __m512d;
};
#elif defined(__AVX2__) && defined(__FMA__)
inline constexpr std::size_t kVectorBytes = 32;
template <>
struct NativeVec<float> {
  using type = __m256;
};
template <>
struct NativeVec<double> {
  using type = __m256d;
};
#else
inline constexpr std::size_t kVectorBytes = 16;
template <>
struct NativeVec<float> {
  using type = __m128;
};
template <>
struct NativeVec<double> {
  using type = __m128d;
};
#endif

// Descriptor ("tag") of a full native vector of T.
template <class T>
struct ScalableTag {
  using T_ = T;
  static constexpr std::size_t kLanes = kVectorBytes / sizeof(T);
};

template <class T>
using Vec = typename NativeVec<T>::type;

template <class T>
constexpr std::size_t Lanes(ScalableTag<T>) {
  return ScalableTag<T>::kLanes;
}

#if defined(__AVX512F__)

inline Vec<float> Set(ScalableTag<float>, float v) { return _mm512_set1_ps(v); }
inline Vec<double> Set(ScalableTag<double>, double v) { return _mm512_set1_pd(v); }
inline Vec<float> Zero(ScalableTag<float>) { return _mm512_setzero_ps(); }
inline Vec<double> Zero(ScalableTag<double>) { return _mm512_setzero_pd(); }
inline Vec<float> Load(ScalableTag<float>, const float* p) { return _mm512_load_ps(p); }
inline Vec<double> Load(ScalableTag<double>, const double* p) { return _mm512_load_pd(p); }
inline Vec<float> LoadU(ScalableTag<float>, const float* p) { return _mm512_loadu_ps(p); }
inline Vec<double> LoadU(ScalableTag<double>, const double* p) { return _mm512_loadu_pd(p); }
inline void Store(Vec<float> v, ScalableTag<float>, float* p) { _mm512_store_ps(p, v); }
inline void Store(Vec<double> v, ScalableTag<double>, double* p) { _mm512_store_pd(p, v); }
inline void StoreU(Vec<float> v, ScalableTag<float>, float* p) { _mm512_storeu_ps(p, v); }
inline void StoreU(Vec<double> v, ScalableTag<double>, double* p) { _mm512_storeu_pd(p, v); }
inline Vec<float> Add(Vec<float> a, Vec<float> b) { return _mm512_add_ps(a, b); }
inline Vec<double> Add(Vec<double> a, Vec<double> b) { return _mm512_add_pd(a, b); }
inline Vec<float> Sub(Vec<float> a, Vec<float> b) { return _mm512_sub_ps(a, b); }
inline Vec<double> Sub(Vec<double> a, Vec<double> b) { return _mm512_sub_pd(a, b); }
inline Vec<float> Mul(Vec<float> a, Vec<float> b) { return _mm512_mul_ps(a, b); }
inline Vec<double> Mul(Vec<double> a, Vec<double> b) { return _mm512_mul_pd(a, b); }
inline Vec<float> Div(Vec<float> a, Vec<float> b) { return _mm512_div_ps(a, b); }
inline Vec<double> Div(Vec<double> a, Vec<double> b) { return _mm512_div_pd(a, b); }
inline Vec<float> MulAdd(Vec<float> m, Vec<float> x, Vec<float> a) { return _mm512_fmadd_ps(m, x, a); }
inline Vec<double> MulAdd(Vec<double> m, Vec<double> x, Vec<double> a) { return _mm512_fmadd_pd(m, x, a); }
inline Vec<float> Sqrt(Vec<float> v) { return _mm512_sqrt_ps(v); }
inline Vec<double> Sqrt(Vec<double> v) { return _mm512_sqrt_pd(v); }
inline Vec<float> Max(Vec<float> a, Vec<float> b) { return _mm512_max_ps(a, b); }
inline Vec<double> Max(Vec<double> a, Vec<double> b) { return _mm512_max_pd(a, b); }
inline Vec<float> Abs(Vec<float> v) {
  return _mm512_castsi512_ps(_mm512_and_si512(_mm512_castps_si512(v), _mm512_set1_epi32(0x7fffffff)));
}
inline Vec<double> Abs(Vec<double> v) {
  return _mm512_castsi512_pd(
      _mm512_and_si512(_mm512_castpd_si512(v), _mm512_set1_epi64(0x7fffffffffffffffLL)));
}

#elif defined(__AVX2__) && defined(__FMA__)

inline Vec<float> Set(ScalableTag<float>, float v) { return _mm256_set1_ps(v); }
inline Vec<double> Set(ScalableTag<double>, double v) { return _mm256_set1_pd(v); }
inline Vec<float> Zero(ScalableTag<float>) { return _mm256_setzero_ps(); }
inline Vec<double> Zero(ScalableTag<double>) { return _mm256_setzero_pd(); }
inline Vec<float> Load(ScalableTag<float>, const float* p) { return _mm256_load_ps(p); }
inline Vec<double> Load(ScalableTag<double>, const double* p) { return _mm256_load_pd(p); }
inline Vec<float> LoadU(ScalableTag<float>, const float* p) { return _mm256_loadu_ps(p); }
inline Vec<double> LoadU(ScalableTag<double>, const double* p) { return _mm256_loadu_pd(p); }
inline void Store(Vec<float> v, ScalableTag<float>, float* p) { _mm256_store_ps(p, v); }
inline void Store(Vec<double> v, ScalableTag<double>, double* p) { _mm256_store_pd(p, v); }
inline void StoreU(Vec<float> v, ScalableTag<float>, float* p) { _mm256_storeu_ps(p, v); }
inline void StoreU(Vec<double> v, ScalableTag<double>, double* p) { _mm256_storeu_pd(p, v); }
inline Vec<float> Add(Vec<float> a, Vec<float> b) { return _mm256_add_ps(a, b); }
inline Vec<double> Add(Vec<double> a, Vec<double> b) { return _mm256_add_pd(a, b); }
inline Vec<float> Sub(Vec<float> a, Vec<float> b) { return _mm256_sub_ps(a, b); }
inline Vec<double> Sub(Vec<double> a, Vec<double> b) { return _mm256_sub_pd(a, b); }
inline Vec<float> Mul(Vec<float> a, Vec<float> b) { return _mm256_mul_ps(a, b); }
inline Vec<double> Mul(Vec<double> a, Vec<double> b) { return _mm256_mul_pd(a, b); }
inline Vec<float> Div(Vec<float> a, Vec<float> b) { return _mm256_div_ps(a, b); }
inline Vec<double> Div(Vec<double> a, Vec<double> b) { return _mm256_div_pd(a, b); }
inline Vec<float> MulAdd(Vec<float> m, Vec<float> x, Vec<float> a) { return _mm256_fmadd_ps(m, x, a); }
inline Vec<double> MulAdd(Vec<double> m, Vec<double> x, Vec<double> a) { return _mm256_fmadd_pd(m, x, a); }
inline Vec<float> Sqrt(Vec<float> v) { return _mm256_sqrt_ps(v); }
inline Vec<double> Sqrt(Vec<double> v) { return _mm256_sqrt_pd(v); }
inline Vec<float> Max(Vec<float> a, Vec<float> b) { return _mm256_max_ps(a, b); }
inline Vec<double> Max(Vec<double> a, Vec<double> b) { return _mm256_max_pd(a, b); }
inline Vec<float> Abs(Vec<float> v) { return _mm256_andnot_ps(_mm256_set1_ps(-0.0f), v); }
inline Vec<double> Abs(Vec<double> v) { return _mm256_andnot_pd(_mm256_set1_pd(-0.0), v); }

#else

inline Vec<float> Set(ScalableTag<float>, float v) { return _mm_set1_ps(v); }
inline Vec<double> Set(ScalableTag<double>, double v) { return _mm_set1_pd(v); }
inline Vec<float> Zero(ScalableTag<float>) { return _mm_setzero_ps(); }
inline Vec<double> Zero(ScalableTag<double>) { return _mm_setzero_pd(); }
inline Vec<float> Load(ScalableTag<float>, const float* p) { return _mm_load_ps(p); }
inline Vec<double> Load(ScalableTag<double>, const double* p) { return _mm_load_pd(p); }
inline Vec<float> LoadU(ScalableTag<float>, const float* p) { return _mm_loadu_ps(p); }
inline Vec<double> LoadU(ScalableTag<double>, const double* p) { return _mm_loadu_pd(p); }
inline void Store(Vec<float> v, ScalableTag<float>, float* p) { _mm_store_ps(p, v); }
inline void Store(Vec<double> v, ScalableTag<double>, double* p) { _mm_store_pd(p, v); }
inline void StoreU(Vec<float> v, ScalableTag<float>, float* p) { _mm_storeu_ps(p, v); }
inline void StoreU(Vec<double> v, ScalableTag<double>, double* p) { _mm_storeu_pd(p, v); }
inline Vec<float> Add(Vec<float> a, Vec<float> b) { return _mm_add_ps(a, b); }
inline Vec<double> Add(Vec<double> a, Vec<double> b) { return _mm_add_pd(a, b); }
inline Vec<float> Sub(Vec<float> a, Vec<float> b) { return _mm_sub_ps(a, b); }
inline Vec<double> Sub(Vec<double> a, Vec<double> b) { return _mm_sub_pd(a, b); }
inline Vec<float> Mul(Vec<float> a, Vec<float> b) { return _mm_mul_ps(a, b); }
inline Vec<double> Mul(Vec<double> a, Vec<double> b) { return _mm_mul_pd(a, b); }
inline Vec<float> Div(Vec<float> a, Vec<float> b) { return _mm_div_ps(a, b); }
inline Vec<double> Div(Vec<double> a, Vec<double> b) { return _mm_div_pd(a, b); }
inline Vec<float> MulAdd(Vec<float> m, Vec<float> x, Vec<float> a) { return _mm_add_ps(_mm_mul_ps(m, x), a); }
inline Vec<double> MulAdd(Vec<double> m, Vec<double> x, Vec<double> a) {
  return _mm_add_pd(_mm_mul_pd(m, x), a);
}
inline Vec<float> Sqrt(Vec<float> v) { return _mm_sqrt_ps(v); }
inline Vec<double> Sqrt(Vec<double> v) { return _mm_sqrt_pd(v); }
inline Vec<float> Max(Vec<float> a, Vec<float> b) { return _mm_max_ps(a, b); }
inline Vec<double> Max(Vec<double> a, Vec<double> b) { return _mm_max_pd(a, b); }
inline Vec<float> Abs(Vec<float> v) { return _mm_andnot_ps(_mm_set1_ps(-0.0f), v); }
inline Vec<double> Abs(Vec<double> v) { return _mm_andnot_pd(_mm_set1_pd(-0.0), v); }

#endif

}  // namespace HWY_NAMESPACE
}  // namespace hwy
