// sample.cuh -- grid location, trilinear sampling and integrator steps.
//
// Restates, per particle step, regular_grid::contains / interpolate
// (include/dpa/types/regular_grid.hpp:41-75, corner order of
// include/dpa/math/permute_for.hpp:12-34) and the odeint euler /
// runge_kutta4 updates that particle_advector.cpp:369-385 performs, with the
// same rounding as the reference's FP32 build.
#pragma once

#include "common.cuh"

namespace dpa {

// One node of the repacked field, widened to FP32.
template <int kStorage>
__device__ __forceinline__ void load_node(const void* nodes, int64_t index, float& x, float& y,
                                          float& z) {
  if constexpr (kStorage == DPA_STORAGE_F32) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(nodes) + index);
    x = v.x;
    y = v.y;
    z = v.z;
  } else if constexpr (kStorage == DPA_STORAGE_F16) {
    const uint2 r = __ldg(reinterpret_cast<const uint2*>(nodes) + index);
    const float2 xy = __half22float2(*reinterpret_cast<const __half2*>(&r.x));
    x = xy.x;
    y = xy.y;
    z = __low2float(*reinterpret_cast<const __half2*>(&r.y));
  } else {
    const uint2 r = __ldg(reinterpret_cast<const uint2*>(nodes) + index);
    const float2 xy = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&r.x));
    x = xy.x;
    y = xy.y;
    z = __low2float(*reinterpret_cast<const __nv_bfloat162*>(&r.y));
  }
}

// Where a position falls in the grid: a = p - offset, s = floor(a / h).
// Inside iff 0 <= s <= n - 2 on every axis (NaN is outside), which is
// regular_grid::contains.
template <bool kPow2>
__device__ __forceinline__ bool locate(const FieldView& f, const float p[3], float a[3],
                                       float s[3]) {
  bool inside = true;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    a[i] = __fsub_rn(p[i], f.offset[i]);
    const float q = kPow2 ? __fmul_rn(a[i], f.inv_spacing[i]) : __fdiv_rn(a[i], f.spacing[i]);
    s[i] = floorf(q);
    inside = inside && (s[i] >= 0.0f) && (s[i] <= f.limit[i]);
  }
  return inside;
}

// fmod(a, h) / h for 0 <= a, given s = floor(fl(a / h)). The rounded quotient
// is either the true integer quotient N or N + 1 (only when a / h lies within
// half an ulp below N + 1, so fmod(a, h) >= h / 2). In both cases a - s * h is
// exactly representable, so one FMA gives it exactly; adding h back in the
// N + 1 case is exact too. fmod keeps the dividend's sign for a zero result.
template <bool kPow2>
__device__ __forceinline__ float weight(float a, float s, float h, float inv_h) {
  float r = fmaf(-s, h, a);
  if (r < 0.0f) r = __fadd_rn(r, h);
  if (r == 0.0f) r = copysignf(0.0f, a);
  return kPow2 ? __fmul_rn(r, inv_h) : __fdiv_rn(r, h);
}

// (1 - w) * lo + w * hi with every operation rounded on its own.
__device__ __forceinline__ float lerp_ref(float lo, float hi, float one_minus_w, float w) {
  return __fadd_rn(__fmul_rn(one_minus_w, lo), __fmul_rn(w, hi));
}

// The eight corners of one cell: corner[dx * 4 + dy * 2 + dz][component].
struct Corners {
  float c[8][3];
};

template <int kStorage>
__device__ __forceinline__ void gather(const FieldView& f, int i0, int i1, int i2, Corners& k) {
  const int64_t base = int64_t(i0) * f.stride0 + int64_t(i1) * f.stride1 + i2;
  const int64_t s0 = f.stride0, s1 = f.stride1;
  load_node<kStorage>(f.nodes, base, k.c[0][0], k.c[0][1], k.c[0][2]);
  load_node<kStorage>(f.nodes, base + 1, k.c[1][0], k.c[1][1], k.c[1][2]);
  load_node<kStorage>(f.nodes, base + s1, k.c[2][0], k.c[2][1], k.c[2][2]);
  load_node<kStorage>(f.nodes, base + s1 + 1, k.c[3][0], k.c[3][1], k.c[3][2]);
  load_node<kStorage>(f.nodes, base + s0, k.c[4][0], k.c[4][1], k.c[4][2]);
  load_node<kStorage>(f.nodes, base + s0 + 1, k.c[5][0], k.c[5][1], k.c[5][2]);
  load_node<kStorage>(f.nodes, base + s0 + s1, k.c[6][0], k.c[6][1], k.c[6][2]);
  load_node<kStorage>(f.nodes, base + s0 + s1 + 1, k.c[7][0], k.c[7][1], k.c[7][2]);
}

// Reduce axis 2, then 1, then 0 (regular_grid.hpp:71-73).
__device__ __forceinline__ void trilinear(const Corners& k, const float w[3], float v[3]) {
  const float tz = __fsub_rn(1.0f, w[2]);
  const float ty = __fsub_rn(1.0f, w[1]);
  const float tx = __fsub_rn(1.0f, w[0]);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float e0 = lerp_ref(k.c[0][c], k.c[1][c], tz, w[2]);
    const float e1 = lerp_ref(k.c[2][c], k.c[3][c], tz, w[2]);
    const float e2 = lerp_ref(k.c[4][c], k.c[5][c], tz, w[2]);
    const float e3 = lerp_ref(k.c[6][c], k.c[7][c], tz, w[2]);
    const float f0 = lerp_ref(e0, e1, ty, w[1]);
    const float f1 = lerp_ref(e2, e3, ty, w[1]);
    v[c] = lerp_ref(f0, f1, tx, w[0]);
  }
}

__device__ __forceinline__ bool is_zero(const float v[3]) {
  return fabsf(v[0]) <= kZeroPrecision && fabsf(v[1]) <= kZeroPrecision &&
         fabsf(v[2]) <= kZeroPrecision;
}

// A per-thread cache of the current cell's corners: a particle usually stays
// in one cell for several steps, and the sampled values do not depend on
// whether the corners came from the cache or from memory.
template <int kStorage, bool kPow2>
struct CellSampler {
  Corners corners;
  int cell[3] = {-1, -1, -1};

  // Samples at p; returns false when p is outside the grid.
  __device__ __forceinline__ bool sample(const FieldView& f, const float p[3], float v[3]) {
    float a[3], s[3];
    if (!locate<kPow2>(f, p, a, s)) return false;
    const int i0 = int(s[0]), i1 = int(s[1]), i2 = int(s[2]);
    if (i0 != cell[0] || i1 != cell[1] || i2 != cell[2]) {
      gather<kStorage>(f, i0, i1, i2, corners);
      cell[0] = i0;
      cell[1] = i1;
      cell[2] = i2;
    }
    float w[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) w[i] = weight<kPow2>(a[i], s[i], f.spacing[i], f.inv_spacing[i]);
    trilinear(corners, w, v);
    return true;
  }
};

enum StepResult : int { kStepTaken = 0, kStepOutOfBounds = 1, kStepZeroVelocity = 2 };

// One integrator step in place. The derivative is the sample with reversed
// components (particle_advector.cpp:369).
template <int kIntegrator, int kStorage, bool kPow2>
__device__ __forceinline__ int step(const FieldView& f, const StepCoefficients& k,
                                   CellSampler<kStorage, kPow2>& sampler, float p[3]) {
  float v[3];
  if (!sampler.sample(f, p, v)) return kStepOutOfBounds;
  if (is_zero(v)) return kStepZeroVelocity;
  const float d[3] = {v[2], v[1], v[0]};
  if constexpr (kIntegrator == DPA_INTEGRATOR_EULER) {
    // odeint euler: x = 1 * x + dt * dxdt
#pragma unroll
    for (int c = 0; c < 3; ++c) p[c] = __fadd_rn(p[c], __fmul_rn(k.dt, d[c]));
  } else if constexpr (kIntegrator == DPA_INTEGRATOR_RUNGE_KUTTA_4) {
    // odeint runge_kutta4, final stage with four equal stage derivatives:
    // x = 1 * x + (b0 dt) d + (b1 dt) d + (b2 dt) d + (b3 dt) d, left to right.
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float m0 = __fmul_rn(k.c0, d[c]);
      const float m1 = __fmul_rn(k.c1, d[c]);
      p[c] = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(p[c], m0), m1), m1), m0);
    }
  } else {
    // Four-sample RK4; a stage outside the grid ends the particle without
    // taking the step.
    float x[3], k2[3], k3[3], k4[3], w[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) x[c] = __fadd_rn(p[c], __fmul_rn(k.half, d[c]));
    if (!sampler.sample(f, x, w)) return kStepOutOfBounds;
    k2[0] = w[2]; k2[1] = w[1]; k2[2] = w[0];
#pragma unroll
    for (int c = 0; c < 3; ++c) x[c] = __fadd_rn(p[c], __fmul_rn(k.half, k2[c]));
    if (!sampler.sample(f, x, w)) return kStepOutOfBounds;
    k3[0] = w[2]; k3[1] = w[1]; k3[2] = w[0];
#pragma unroll
    for (int c = 0; c < 3; ++c) x[c] = __fadd_rn(p[c], __fmul_rn(k.dt, k3[c]));
    if (!sampler.sample(f, x, w)) return kStepOutOfBounds;
    k4[0] = w[2]; k4[1] = w[1]; k4[2] = w[0];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float t = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(p[c], __fmul_rn(k.c0, d[c])),
                                                    __fmul_rn(k.c1, k2[c])),
                                          __fmul_rn(k.c1, k3[c])),
                                __fmul_rn(k.c0, k4[c]));
      p[c] = t;
    }
  }
  return kStepTaken;
}

}  // namespace dpa
