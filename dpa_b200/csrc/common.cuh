// common.cuh -- shared device definitions of the sm_100a advection library.
//
// Arithmetic that must agree bit for bit with the reference's x86-64 build
// (baseline SSE, no FMA) uses the explicitly rounded intrinsics __fadd_rn,
// __fsub_rn, __fmul_rn and __fdiv_rn, which nvcc never contracts into FMAs.
#pragma once

#include <cstdint>

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

// Device view of a repacked field. Nodes are 4-wide (x, y, z, pad) so one
// vector load fetches a node: float4 for F32, four 16-bit values for F16/BF16.
struct FieldView {
  const void* nodes;
  int32_t n[3];        // grid shape
  int64_t stride0;     // n1 * n2
  int32_t stride1;     // n2
  float offset[3];
  float spacing[3];
  float inv_spacing[3];  // exact reciprocals, used only when pow2 is set
  float upper[3];        // n - 1: inside iff 0 <= (p - offset) / h < n - 1
  int32_t storage;       // dpa_storage
  int32_t pow2;          // every spacing is a power of two (division == product)
};

struct StepCoefficients {
  float dt;
  float c0;    // float(1/6) * dt  (odeint rk4 b0 = b3)
  float c1;    // float(1/3) * dt  (odeint rk4 b1 = b2)
  float half;  // float(1/2) * dt  (stage offsets of the four-sample RK4)
};

inline StepCoefficients make_step_coefficients(float dt) {
  volatile float b0 = 1.0f / 6.0f;  // computed in float as odeint does
  volatile float b1 = 1.0f / 3.0f;
  volatile float a = 1.0f / 2.0f;
  StepCoefficients k;
  k.dt = dt;
  k.c0 = b0 * dt;
  k.c1 = b1 * dt;
  k.half = a * dt;
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
