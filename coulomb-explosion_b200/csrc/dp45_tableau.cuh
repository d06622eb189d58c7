// dp45_tableau.cuh -- Dormand-Prince 5(4) coefficients for the velocity-only
// stage formulation used by the GPU kernels.
//
// The reference stores, per stage s, both the position derivative kpos_s (a
// stage velocity) and the velocity derivative kvel_s (an acceleration)
// (src/integrators.cpp:85-102, include/coulomb/batched_integrator.hpp:275-293):
//     kpos_s = v + h sum_{j<s} a_sj kvel_j          x_s = x + h sum_{j<s} a_sj kpos_j
// Substituting the first into the second gives, with c_s = sum_j a_sj,
//     x_s = x + h (c_s v + h sum_l abar_sl kvel_l),   abar_sl = sum_{l<j<s} a_sj a_jl,
// and the position half of the embedded error h sum_s E_s kpos_s becomes
//     h^2 sum_l ebar_l kvel_l,   ebar_l = sum_{s>l} E_s a_sl       (sum_s E_s = 0).
// The two forms are algebraically identical; the second needs only the
// accelerations, which halves the per-sim stage storage so a whole CH4
// simulation's stages fit in one thread's registers. The base tableau is the
// one in src/integrators.cpp:155-167 (DP5(4), scipy's RK45).
#pragma once

namespace ce {
namespace dp45 {

struct Tab {
  double a[8][8];     // a[s][j], stages 1..7 (row 7 = 5th-order weights b)
  double e[8];        // E_s = b_s - b*_s
  double c[8];        // c_s = sum_j a[s][j]
  double abar[8][8];  // abar[s][l] = sum_{l<j<s} a[s][j] a[j][l]
  double ebar[8];     // ebar[l] = sum_{s>l} E_s a[s][l]
};

constexpr Tab make_tab() {
  Tab t{};
  t.a[2][1] = 1.0 / 5;
  t.a[3][1] = 3.0 / 40;       t.a[3][2] = 9.0 / 40;
  t.a[4][1] = 44.0 / 45;      t.a[4][2] = -56.0 / 15;      t.a[4][3] = 32.0 / 9;
  t.a[5][1] = 19372.0 / 6561; t.a[5][2] = -25360.0 / 2187; t.a[5][3] = 64448.0 / 6561;
  t.a[5][4] = -212.0 / 729;
  t.a[6][1] = 9017.0 / 3168;  t.a[6][2] = -355.0 / 33;     t.a[6][3] = 46732.0 / 5247;
  t.a[6][4] = 49.0 / 176;     t.a[6][5] = -5103.0 / 18656;
  t.a[7][1] = 35.0 / 384;     t.a[7][2] = 0.0;             t.a[7][3] = 500.0 / 1113;
  t.a[7][4] = 125.0 / 192;    t.a[7][5] = -2187.0 / 6784;  t.a[7][6] = 11.0 / 84;
  t.e[1] = 71.0 / 57600;      t.e[2] = 0.0;                t.e[3] = -71.0 / 16695;
  t.e[4] = 71.0 / 1920;       t.e[5] = -17253.0 / 339200;  t.e[6] = 22.0 / 525;
  t.e[7] = -1.0 / 40;
  for (int s = 1; s <= 7; ++s) {
    double c = 0.0;
    for (int j = 1; j < s; ++j) c += t.a[s][j];
    t.c[s] = c;
    for (int l = 1; l < s; ++l) {
      double ab = 0.0;
      for (int j = l + 1; j < s; ++j) ab += t.a[s][j] * t.a[j][l];
      t.abar[s][l] = ab;
    }
  }
  for (int l = 1; l <= 7; ++l) {
    double eb = 0.0;
    for (int s = l + 1; s <= 7; ++s) eb += t.e[s] * t.a[s][l];
    t.ebar[l] = eb;
  }
  return t;
}

constexpr Tab kTab = make_tab();

}  // namespace dp45

// Float copies in constant memory (one private copy per translation unit).
// Kernels index them with compile-time (fully unrolled) indices, so each use is
// a constant-bank FFMA operand.
#define CE_AB(s, l) static_cast<float>(ce::dp45::kTab.abar[s][l])
#define CE_ROW8(M, s) M(s, 0), M(s, 1), M(s, 2), M(s, 3), M(s, 4), M(s, 5), M(s, 6), M(s, 7)
#define CE_A(s, l) static_cast<float>(ce::dp45::kTab.a[s][l])

static __constant__ float c_abar[8][8] = {{CE_ROW8(CE_AB, 0)}, {CE_ROW8(CE_AB, 1)}, {CE_ROW8(CE_AB, 2)},
                                   {CE_ROW8(CE_AB, 3)}, {CE_ROW8(CE_AB, 4)}, {CE_ROW8(CE_AB, 5)},
                                   {CE_ROW8(CE_AB, 6)}, {CE_ROW8(CE_AB, 7)}};
static __constant__ float c_b[8] = {CE_ROW8(CE_A, 7)};
static __constant__ float c_c[8] = {
    static_cast<float>(dp45::kTab.c[0]), static_cast<float>(dp45::kTab.c[1]),
    static_cast<float>(dp45::kTab.c[2]), static_cast<float>(dp45::kTab.c[3]),
    static_cast<float>(dp45::kTab.c[4]), static_cast<float>(dp45::kTab.c[5]),
    static_cast<float>(dp45::kTab.c[6]), static_cast<float>(dp45::kTab.c[7])};
static __constant__ float c_e[8] = {
    static_cast<float>(dp45::kTab.e[0]), static_cast<float>(dp45::kTab.e[1]),
    static_cast<float>(dp45::kTab.e[2]), static_cast<float>(dp45::kTab.e[3]),
    static_cast<float>(dp45::kTab.e[4]), static_cast<float>(dp45::kTab.e[5]),
    static_cast<float>(dp45::kTab.e[6]), static_cast<float>(dp45::kTab.e[7])};
static __constant__ float c_ebar[8] = {
    static_cast<float>(dp45::kTab.ebar[0]), static_cast<float>(dp45::kTab.ebar[1]),
    static_cast<float>(dp45::kTab.ebar[2]), static_cast<float>(dp45::kTab.ebar[3]),
    static_cast<float>(dp45::kTab.ebar[4]), static_cast<float>(dp45::kTab.ebar[5]),
    static_cast<float>(dp45::kTab.ebar[6]), static_cast<float>(dp45::kTab.ebar[7])};

#undef CE_AB
#undef CE_A
#undef CE_ROW8

// Step-size controller constants, src/integrators.cpp:169-175.
constexpr float kSafety = 0.9f;
constexpr float kMinFactor = 0.2f;
constexpr float kMaxFactor = 10.0f;
constexpr float kExponent = -0.2f;
constexpr int kMaxRejections = 100;

}  // namespace ce
