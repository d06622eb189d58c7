// types.hpp -- scalar and 3-vector types of the host API.
//
// Mirrors include/coulomb/types.hpp:16-51 of the reference (Real, Vec3 with
// +, -, scalar * and dot/norm). The host API is double precision throughout;
// the GPU engine narrows positions to float at the device boundary the way the
// reference's BatchedRK45<float>::set_lane_geometry narrows to T
// (include/coulomb/batched_integrator.hpp:112-121).
#pragma once

#include <cmath>
#include <cstddef>

namespace coulomb {

using Real = double;

struct Vec3 {
  Real x{0};
  Real y{0};
  Real z{0};

  constexpr Vec3 operator+(const Vec3& o) const { return {x + o.x, y + o.y, z + o.z}; }
  constexpr Vec3 operator-(const Vec3& o) const { return {x - o.x, y - o.y, z - o.z}; }
  constexpr Vec3 operator*(Real s) const { return {x * s, y * s, z * s}; }
  constexpr Vec3& operator+=(const Vec3& o) {
    x += o.x;
    y += o.y;
    z += o.z;
    return *this;
  }
};

constexpr Vec3 operator*(Real s, const Vec3& v) { return v * s; }
constexpr Real dot(const Vec3& a, const Vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Real norm(const Vec3& v) { return std::sqrt(dot(v, v)); }

}  // namespace coulomb
