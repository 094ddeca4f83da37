// common.cuh -- shared device definitions of the sm_100a advection library.
//
// Arithmetic that must agree bit for bit with the reference's x86-64 build
// (baseline SSE, no FMA) uses the explicitly rounded intrinsics __fadd_rn,
// __fsub_rn, __fmul_rn and __fdiv_rn, which nvcc never contracts into FMAs.
#pragma once

#include <cstdint>
#include <initializer_list>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "dpa_b200.h"

namespace dpa {

// basic_types.hpp:51-60: invalid_value = -1 * Ones, terminal_value = -2 * Ones.
constexpr float kInvalid = -1.0f;
constexpr float kTerminal = -2.0f;

// Eigen::NumTraits<float>::dummy_precision(): isZero()'s default tolerance
// (particle_advector.cpp:363 tests |v_i| <= 1 * 1e-5 for every component).
constexpr float kZeroPrecision = 1e-5f;

// How a kernel divides a position by the spacing (per field, every axis):
//   kLocateDivide      IEEE division (__fdiv_rn);
//   kLocateReciprocal  a / h as one product and one FMA with the reciprocal
//                      split in two floats (divide_by_reciprocal), used only
//                      for divisors for which it was checked at field creation
//                      to equal __fdiv_rn for every float a;
//   kLocatePow2        power-of-two spacing: one FMA of the exact p / h and
//                      offset / h, and fmod(p - offset, h) / h = q - floor(q).
enum LocateMode : int { kLocateDivide = 0, kLocateReciprocal = 1, kLocatePow2 = 2 };

// Device view of a repacked field. Nodes are 4-wide (x, y, z, pad) so one
// vector load fetches a node: float4 for F32, four 16-bit values for F16/BF16.
// A slice holds fewer than 2^32 nodes, so a node's index within its slice is
// a 32-bit value (s0 * stride0 + s1 * stride1 + s2).
struct FieldView {
  const void* nodes;
  int32_t n[3];        // grid shape
  uint32_t stride0;    // n1 * n2
  uint32_t stride1;    // n2
  float offset[3];
  float spacing[3];
  float reciprocal[3];     // RN(1 / spacing): exact for power-of-two spacings
  float reciprocal_lo[3];  // RN(1 / spacing - reciprocal)
  float scaled_offset[3];  // offset / spacing, exact; used by kLocatePow2 only
  float upper[3];          // n - 1: inside iff 0 <= (p - offset) / h < n - 1
  uint32_t cells[3];       // n - 1, the cells per axis
  // (2^23 as float bits) * (stride0 + stride1 + 1), modulo 2^32: what the
  // cell index subtracts when it is formed from biased floors (sample.cuh).
  uint32_t node_bias;
  int32_t storage;         // dpa_storage
  // LocateMode of the spatial axes. kLocatePow2 needs every spacing a power
  // of two in [2^-20, 2^20] and every offset zero or at least 2^-100 in
  // magnitude: (p - offset) / h is then one rounding of p / h - offset / h.
  int32_t locate;
  // Time-varying fields: `slices` grids of slice_stride nodes each, slice s
  // at time time_origin + s * time_spacing; slices == 1 for a steady field.
  int32_t slices;
  int64_t slice_stride;
  float time_origin;
  float time_spacing;
  float time_reciprocal;     // RN(1 / time_spacing)
  float time_reciprocal_lo;  // RN(1 / time_spacing - time_reciprocal)
  int32_t time_fast;         // the time axis divides as kLocateReciprocal
  float time_upper;      // slices - 1: inside iff 0 <= (t - t0) / dt < slices - 1
};

// a / h by a known divisor: with y + yl = 1 / h split into two floats,
// q = RN(a * y + RN(a * yl)), one product and one FMA (Brisebarre, Muller
// and Raina, "Accelerating correctly rounded floating-point division when
// the divisor is known in advance", IEEE Trans. Computers 53(8), 2004).
// Dividends below 2^-64 or above 2^64 in magnitude (and NaN) take IEEE
// division: there the products leave the normal range. Whether the result
// equals IEEE division for every other dividend depends on the divisor; it
// is used only for divisors checked exhaustively on the device
// (verify_division_kernel, advect.cu).
__device__ __forceinline__ float divide_by_reciprocal(float a, float h, float y, float yl) {
  if (!(fabsf(a) >= 0x1p-64f && fabsf(a) <= 0x1p64f)) return __fdiv_rn(a, h);
  return __fmaf_rn(a, y, __fmul_rn(a, yl));
}

template <int kLocate>
__device__ __forceinline__ float divide_spacing(float a, float h, float y, float yl) {
  if constexpr (kLocate == kLocateDivide) return __fdiv_rn(a, h);
  else return divide_by_reciprocal(a, h, y, yl);
}

// Three divisions by known divisors (a_i / h_i, reciprocal pairs y_i, yl_i):
// one range test for all three dividends instead of one each. Inside the
// range every quotient is the reciprocal form's, as divide_by_reciprocal
// gives; otherwise each takes divide_by_reciprocal's own test. (fminf and
// fmaxf pass over NaN, but a NaN dividend gives NaN on either path.)
__device__ __forceinline__ void divide3_by_reciprocal(const float a[3], const float h[3],
                                                      const float y[3], const float yl[3],
                                                      float q[3]) {
  const float lo = fminf(fminf(fabsf(a[0]), fabsf(a[1])), fabsf(a[2]));
  const float hi = fmaxf(fmaxf(fabsf(a[0]), fabsf(a[1])), fabsf(a[2]));
  if (lo >= 0x1p-64f && hi <= 0x1p64f) {
#pragma unroll
    for (int i = 0; i < 3; ++i) q[i] = __fmaf_rn(a[i], y[i], __fmul_rn(a[i], yl[i]));
  } else {
#pragma unroll
    for (int i = 0; i < 3; ++i) q[i] = divide_by_reciprocal(a[i], h[i], y[i], yl[i]);
  }
}

// Integrator id of the kernel instantiation shared by the reference's other
// odeint steppers (modified_midpoint, runge_kutta_cash_karp54,
// runge_kutta_dopri5, runge_kutta_fehlberg78, adams_bashforth<2>,
// adams_bashforth_moulton<2>; integrators.hpp:13-28). Their coefficients come
// with the launch.
constexpr int kGeneralIntegrator = 1000;

// The reference's system ignores its state argument (particle_advector.cpp:376),
// so every stage of an odeint step sees the same derivative d and only the
// stepper's final combination shapes the result. For the general steppers:
//   kSum:       x_out = 1*x + s[0]*D0 + s[1]*D1 + ... (left to right), where
//               Di is d, or the particle's previous-step derivative for the
//               terms in prev_mask once the particle has taken a step;
//   kMidpoint:  odeint modified_midpoint with 2 sub-steps;
// and with extrapolated_start a particle's first step is the Adams methods'
// initialising stepper: extrapolation of modified midpoints with 2 and 4
// sub-steps.
enum GeneralKind : int32_t { kGeneralSum = 0, kGeneralMidpoint = 1 };

struct GeneralCoefficients {
  int32_t kind;
  int32_t terms;             // entries of s in use (<= 13)
  uint32_t prev_mask;        // bit i: term i takes the previous step's derivative
  int32_t extrapolated_start;
  float s[13];               // b_i * dt (or dt * b_i), each rounded to float
  float mm2[3];              // 2 sub-steps: h = dt/2, h2 = 2*h, 0.5*h
  float mm4[3];              // 4 sub-steps: h = dt/4, h2 = 2*h, 0.5*h
  float ex[2];               // 1 + 1/3 and -(1/3): the single extrapolation
};

struct StepCoefficients {
  float dt;
  float c0;    // float(1/6) * dt  (odeint rk4 b0 = b3)
  float c1;    // float(1/3) * dt  (odeint rk4 b1 = b2)
  float half;  // float(1/2) * dt  (stage offsets of the four-sample RK4)
  GeneralCoefficients g;
};

// True for the steppers whose step depends on the particle's previous step:
// runge_kutta_dopri5 (first-same-as-last derivative), adams_bashforth<2>
// (derivative history) and adams_bashforth_moulton<2> (different first step).
inline bool integrator_has_history(int integrator) {
  return integrator == DPA_INTEGRATOR_RUNGE_KUTTA_DORMAND_PRINCE_5 ||
         integrator == DPA_INTEGRATOR_ADAMS_BASHFORTH_2 ||
         integrator == DPA_INTEGRATOR_ADAMS_BASHFORTH_MOULTON_2;
}

// Coefficients as odeint forms them from its float value_type: tableau
// entries as quotients of floats, then products with dt in float.
inline StepCoefficients make_step_coefficients(int integrator, float dt) {
  volatile float b0 = 1.0f / 6.0f;  // computed in float as odeint does
  volatile float b1 = 1.0f / 3.0f;
  volatile float a = 1.0f / 2.0f;
  StepCoefficients k{};
  k.dt = dt;
  k.c0 = b0 * dt;
  k.c1 = b1 * dt;
  k.half = a * dt;
  GeneralCoefficients& g = k.g;
  auto q = [](float num, float den) {
    volatile float n = num, d = den;
    return n / d;
  };
  auto sum = [&](std::initializer_list<float> b, bool dt_first) {
    g.kind = kGeneralSum;
    g.terms = 0;
    for (float v : b) {
      volatile float bv = v, t = dt;
      g.s[g.terms++] = dt_first ? t * bv : bv * t;
    }
  };
  for (int m = 0; m < 2; ++m) {
    float* mm = m == 0 ? g.mm2 : g.mm4;
    volatile float steps = m == 0 ? 2.0f : 4.0f;
    const float h = dt / steps;
    mm[0] = h;
    mm[1] = 2.0f * h;
    mm[2] = 0.5f * h;
  }
  {
    volatile float four = 4.0f, two = 2.0f, one = 1.0f;
    const float r = four / two;
    const float c = one / (r * r - one);
    g.ex[0] = one + c;
    g.ex[1] = -c;
  }
  switch (integrator) {
    case DPA_INTEGRATOR_MODIFIED_MIDPOINT:
      g.kind = kGeneralMidpoint;
      break;
    case DPA_INTEGRATOR_RUNGE_KUTTA_CASH_KARP_54:
      // rk54_ck: 5th-order weights (do_step without error estimate).
      sum({q(37, 378), 0.0f, q(250, 621), q(125, 594), 0.0f, q(512, 1771)}, false);
      break;
    case DPA_INTEGRATOR_RUNGE_KUTTA_DORMAND_PRINCE_5:
      // dopri5: x + dt*c1*dxdt_in + dt*c3*k3 + dt*c4*k4 + dt*c5*k5 + dt*c6*k6;
      // dxdt_in is the derivative the previous step left behind.
      sum({q(35, 384), q(500, 1113), q(125, 192), q(-2187, 6784), q(11, 84)}, true);
      g.prev_mask = 1u;
      break;
    case DPA_INTEGRATOR_RUNGE_KUTTA_FEHLBERG_78:
      sum({0.0f, 0.0f, 0.0f, 0.0f, 0.0f, q(34, 105), q(9, 35), q(9, 35), q(9, 280), q(9, 280),
           0.0f, q(41, 840), q(41, 840)},
          false);
      break;
    case DPA_INTEGRATOR_ADAMS_BASHFORTH_2:
      // x + dt*(3/2)*d_n + dt*(-1/2)*d_(n-1)
      sum({q(3, 2), -q(1, 2)}, true);
      g.prev_mask = 2u;
      g.extrapolated_start = 1;
      break;
    case DPA_INTEGRATOR_ADAMS_BASHFORTH_MOULTON_2:
      // Corrector x + dt*(1/2)*f(predicted) + dt*(1/2)*d_n, both equal to d_n.
      sum({q(1, 2), q(1, 2)}, true);
      g.extrapolated_start = 1;
      break;
    default:
      break;
  }
  return k;
}

__device__ __forceinline__ bool equals3(float x, float y, float z, float s) {
  return x == s && y == s && z == s;
}

}  // namespace dpa

#define DPA_CUDA_TRY(expr)                                   \
  do {                                                       \
    cudaError_t dpa_err_ = (expr);                           \
    if (dpa_err_ != cudaSuccess) return dpa_err_;            \
  } while (0)
