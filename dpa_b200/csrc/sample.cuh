// sample.cuh -- grid location, trilinear sampling and integrator steps.
//
// Restates, per particle step, regular_grid::contains / interpolate
// (include/dpa/types/regular_grid.hpp:41-75, corner order of
// include/dpa/math/permute_for.hpp:12-34) and the odeint euler /
// runge_kutta4 updates that particle_advector.cpp:369-385 performs, with the
// same rounding as the reference's FP32 build.
#pragma once

#include <type_traits>

#include "common.cuh"

// F32 trilinear products as packed FMUL2 pairs (1) or scalar FMULs (0).
#ifndef DPA_F32_PACKED_LERP
#define DPA_F32_PACKED_LERP 0
#endif

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

// Two FP32 lanes. Products use sm_100's packed multiply (FMUL2), whose
// lanes round exactly as __fmul_rn does. Sums that may take such a product
// as an operand stay scalar (__fadd_rn): the compiler fuses a packed multiply
// feeding a packed add into one packed FMA even when both carry explicit
// round-to-nearest, and the fused result differs from the reference's
// separately rounded product and sum. sum2 is the packed add for operands
// that are never products.
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}
__device__ __forceinline__ float2 sum2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
// Two scalar products, for lerps whose operands would need extra register
// moves to form the pairs a packed multiply reads.
__device__ __forceinline__ float2 mul2_scalar(float2 a, float2 b) {
  return make_float2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
}
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 splat(float a) { return make_float2(a, a); }

// A particle position is held as p0 and the pair p21 = (p2, p1): the
// derivative of (p2, p1) is (v0, v1), the first two components of a sample,
// because of the reversed components of particle_advector.cpp:369.
struct Position {
  float p0;
  float2 p21;
};

// Weights of one sample: w = fmod(p - offset, h) / h per axis, as (w0, (w2, w1)).
struct Weights {
  float w0;
  float2 w21;
};

// fmod(a, h) from the floor s of the rounded quotient a / h.
__device__ __forceinline__ float remainder_general(float a, float s, float h) {
  float r = fmaf(-s, h, a);
  if (r < 0.0f) r = __fadd_rn(r, h);
  if (r == 0.0f) r = copysignf(0.0f, a);
  return r;
}

// Where a position falls in the grid, per axis: the rounded quotient
// q = (p - offset) / h, its floor s (the cell subscript) and the weight
// w = fmod(p - offset, h) / h, all as the reference rounds them. The position
// is inside iff 0 <= s <= n - 2 on every axis (regular_grid::contains), which
// for any float q (NaN included) is 0 <= q < n - 1.
//
// kLocatePow2: q is one FMA of the exact p / h and offset / h, and
// fmod(a, h) / h = q - s, whose difference is representable; the sign of a
// zero weight follows q as fmod's follows a.
//
// Other spacings: the rounded quotient is either the true integer quotient N
// or N + 1 (only when a / h lies within half an ulp below N + 1, so that
// fmod(a, h) >= h / 2). In both cases a - s * h is exactly representable, so
// one FMA gives it exactly; adding h back in the N + 1 case is exact too.
// Both divisions are IEEE division (kLocateDivide) or by the verified
// reciprocal pair (kLocateReciprocal), which gives the same bits.
template <int kLocate>
__device__ __forceinline__ float weight_general(float a, float s, float h, float y, float yl) {
  return divide_spacing<kLocate>(remainder_general(a, s, h), h, y, yl);
}

// Locates p; node receives the index of the cell's first corner within its
// slice (meaningful only when p is inside).
template <int kLocate>
__device__ __forceinline__ bool locate(const FieldView& f, const Position& p, uint32_t& node,
                                       Weights& w) {
  float q0, q2, q1;
  float a0 = 0.0f;
  float2 a21 = make_float2(0.0f, 0.0f);
  if constexpr (kLocate == kLocatePow2) {
    // q = p / h - offset / h in one rounding: p / h and offset / h are exact,
    // so this is the reference's rounded (p - offset) scaled by 1 / h.
    q0 = __fmaf_rn(p.p0, f.reciprocal[0], -f.scaled_offset[0]);
    const float2 q21 =
        __ffma2_rn(p.p21, make_float2(f.reciprocal[2], f.reciprocal[1]),
                   make_float2(-f.scaled_offset[2], -f.scaled_offset[1]));
    q2 = q21.x;
    q1 = q21.y;
  } else {
    a0 = __fsub_rn(p.p0, f.offset[0]);
    a21 = sum2(p.p21, neg2(make_float2(f.offset[2], f.offset[1])));
    if constexpr (kLocate == kLocateReciprocal) {
      const float a[3] = {a0, a21.y, a21.x};
      float q[3];
      divide3_by_reciprocal(a, f.spacing, f.reciprocal, f.reciprocal_lo, q);
      q0 = q[0];
      q1 = q[1];
      q2 = q[2];
    } else {
      q0 = divide_spacing<kLocate>(a0, f.spacing[0], f.reciprocal[0], f.reciprocal_lo[0]);
      q2 = divide_spacing<kLocate>(a21.x, f.spacing[2], f.reciprocal[2], f.reciprocal_lo[2]);
      q1 = divide_spacing<kLocate>(a21.y, f.spacing[1], f.reciprocal[1], f.reciprocal_lo[1]);
    }
  }
  // floor(q) and its integer from one round-down add: for 0 <= q < 2^23,
  // RD(q + 2^23) is 2^23 + floor(q), whose low mantissa bits are floor(q),
  // and subtracting 2^23 again is exact. Inside the grid q < n - 1 <= 2^23
  // (the field's axes hold at most 2^23 nodes); outside it neither value is
  // used. (At q = -0 the floor is +0 instead of -0, which the weights' sign
  // rules below undo.)
  const float b0 = __fadd_rd(q0, 0x1p23f), b1 = __fadd_rd(q1, 0x1p23f),
              b2 = __fadd_rd(q2, 0x1p23f);
  const float s0 = __fsub_rn(b0, 0x1p23f), s1 = __fsub_rn(b1, 0x1p23f),
              s2 = __fsub_rn(b2, 0x1p23f);
  if constexpr (kLocate == kLocatePow2) {
    w.w0 = copysignf(__fsub_rn(q0, s0), q0);
    const float2 d = sum2(make_float2(q2, q1), neg2(make_float2(s2, s1)));
    w.w21 = make_float2(copysignf(d.x, q2), copysignf(d.y, q1));
  } else if constexpr (kLocate == kLocateReciprocal) {
    const float a[3] = {a0, a21.y, a21.x};
    const float s[3] = {s0, s1, s2};
    float r[3], ww[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) r[i] = remainder_general(a[i], s[i], f.spacing[i]);
    divide3_by_reciprocal(r, f.spacing, f.reciprocal, f.reciprocal_lo, ww);
    w.w0 = ww[0];
    w.w21 = make_float2(ww[2], ww[1]);
  } else {
    w.w0 = weight_general<kLocate>(a0, s0, f.spacing[0], f.reciprocal[0], f.reciprocal_lo[0]);
    w.w21 = make_float2(
        weight_general<kLocate>(a21.x, s2, f.spacing[2], f.reciprocal[2], f.reciprocal_lo[2]),
        weight_general<kLocate>(a21.y, s1, f.spacing[1], f.reciprocal[1], f.reciprocal_lo[1]));
  }
  // The integer floors (the bits of b minus those of 2^23) decide inside:
  // 0 <= q < n - 1 iff 0 <= floor(q) < n - 1, and a negative, NaN, infinite
  // or too large q gives a difference of n - 1 or more as an unsigned value
  // (-0 gives 0, inside, as the reference has it).
  constexpr uint32_t kTwo23 = 0x4B000000u;  // the bits of 2^23
  const uint32_t i0 = __float_as_uint(b0), i1 = __float_as_uint(b1), i2 = __float_as_uint(b2);
  const bool inside =
      (i0 - kTwo23 < f.cells[0]) & (i1 - kTwo23 < f.cells[1]) & (i2 - kTwo23 < f.cells[2]);
  node = i0 * f.stride0 + i1 * f.stride1 + i2 - f.node_bias;
  return inside;
}

// (1 - w) * lo + w * hi per lane, every operation rounded on its own.
__device__ __forceinline__ float2 lerp2(float2 lo, float2 hi, float2 one_minus_w, float2 w) {
  return add2(mul2(one_minus_w, lo), mul2(w, hi));
}

// The eight corners of one cell are corner j = dx * 4 + dy * 2 + dz (the
// permute_for order of permute_for.hpp:12-34). Two register layouts of them
// serve the trilinear reduction of regular_grid.hpp:71-73 (axis 2, then 1,
// then 0, with c[j] = (1 - w) * c[2j] + w * c[2j+1]); both give the same
// bits, and each storage takes the one that measured faster on the B200.
//
// CornerNodes (F32 nodes): xy[j] = (v0, v1) of corner j, and the v2
// components paired as (corner 0, corner 4), (1, 5), (2, 6), (3, 7). A
// 16-byte node load lands (v0, v1) in a register pair as it is, and the
// lerps multiply in scalar: packed products would need the weights
// duplicated into pairs, and the extra registers cost more than the packed
// multiply saves at F32's load width.
struct CornerNodes {
  float2 xy[8];
  float2 z04, z15, z26, z37;
};

// CornerEdges (F16 / BF16 nodes, F32 edge records): z[e][c] = (component c
// of corner 2e, component c of corner 2e + 1), the two ends of edge
// e = dx * 2 + dy along axis 2, formed as 16-bit values are widened or loaded
// as they are from an edge record. Each lerp is one packed multiply of
// (lo, hi) by the weight pair (1 - w, w) and one scalar sum. (F32 nodes in
// this layout, pairs formed by register moves after the loads, measured 5 %
// slower on the headline launch than CornerNodes.)
struct CornerEdges {
  float2 z[4][3];
};

template <int kStorage>
using CornersOf = std::conditional_t<kStorage == DPA_STORAGE_F32, CornerNodes, CornerEdges>;

// Node layouts (F32, F16, BF16): one 16-byte float4 (F32) or 8-byte uint2
// per node.
template <int kStorage>
using NodeOf = std::conditional_t<kStorage == DPA_STORAGE_F32, float4, uint2>;

// Pointers to the first node of the cell's four edges along axis 2 (corners
// 2e and 2e + 1 are consecutive nodes): e = dx * 2 + dy.
template <int kStorage>
struct CellEdges {
  const NodeOf<kStorage>* e[4];
  __device__ __forceinline__ CellEdges(const FieldView& f, uint32_t node, int64_t slice_base) {
    const NodeOf<kStorage>* base =
        reinterpret_cast<const NodeOf<kStorage>*>(f.nodes) + slice_base + node;
    e[0] = base;
    e[1] = base + f.stride1;
    e[2] = base + f.stride0;
    e[3] = e[2] + f.stride1;
  }
};

// Edge records (F32_EDGES): record n holds node n and node n + 1 along axis
// 2 with each component's two values side by side, (x_n, x_n+1, y_n, y_n+1,
// z_n, z_n+1, 0, 0), 32 bytes read by one 256-bit load whose registers are
// already the (lo, hi) pairs the packed lerps take.
constexpr int kEdgeRecordBytes = 32;

__device__ __forceinline__ void load_edge_record(const char* record, float2 out[3]) {
  float v[8];
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]),
        "=f"(v[7])
      : "l"(record));
  out[0] = make_float2(v[0], v[1]);
  out[1] = make_float2(v[2], v[3]);
  out[2] = make_float2(v[4], v[5]);
}

template <int kStorage>
__device__ __forceinline__ void gather(const FieldView& f, uint32_t node, CornerNodes& k,
                                       int64_t slice_base = 0) {
  const CellEdges<kStorage> c(f, node, slice_base);
  float z[8];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    load_node<kStorage>(c.e[e], 0, k.xy[2 * e].x, k.xy[2 * e].y, z[2 * e]);
    load_node<kStorage>(c.e[e], 1, k.xy[2 * e + 1].x, k.xy[2 * e + 1].y, z[2 * e + 1]);
  }
  k.z04 = make_float2(z[0], z[4]);
  k.z15 = make_float2(z[1], z[5]);
  k.z26 = make_float2(z[2], z[6]);
  k.z37 = make_float2(z[3], z[7]);
}

// gather() of F32 nodes into CornerNodes only where `need` holds, by
// predicated loads instead of a branch: elsewhere the corners keep their
// values and no load is made.
__device__ __forceinline__ void load_node_if(bool need, const float4* at, float& x, float& y,
                                             float& z) {
  float w = 0.0f;
  asm("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %5, 0;\n\t"
      "@p ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];\n\t}"
      : "+f"(x), "+f"(y), "+f"(z), "+f"(w)
      : "l"(at), "r"(need ? 1u : 0u));
}

__device__ __forceinline__ void gather_if(const FieldView& f, uint32_t node, bool need,
                                          CornerNodes& k) {
  const CellEdges<DPA_STORAGE_F32> c(f, node, 0);
  float z[8] = {k.z04.x, k.z15.x, k.z26.x, k.z37.x, k.z04.y, k.z15.y, k.z26.y, k.z37.y};
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    load_node_if(need, c.e[e], k.xy[2 * e].x, k.xy[2 * e].y, z[2 * e]);
    load_node_if(need, c.e[e] + 1, k.xy[2 * e + 1].x, k.xy[2 * e + 1].y, z[2 * e + 1]);
  }
  k.z04 = make_float2(z[0], z[4]);
  k.z15 = make_float2(z[1], z[5]);
  k.z26 = make_float2(z[2], z[6]);
  k.z37 = make_float2(z[3], z[7]);
}

template <int kStorage>
__device__ __forceinline__ void gather(const FieldView& f, uint32_t node, CornerEdges& k,
                                       int64_t slice_base = 0) {
  if constexpr (kStorage == DPA_STORAGE_F32_EDGES) {
    const char* base = static_cast<const char*>(f.nodes) +
                       (uint64_t(slice_base) + node) * uint64_t(kEdgeRecordBytes);
    const uint64_t s1 = uint64_t(f.stride1) * kEdgeRecordBytes;
    const uint64_t s0 = uint64_t(f.stride0) * kEdgeRecordBytes;
    load_edge_record(base, k.z[0]);
    load_edge_record(base + s1, k.z[1]);
    load_edge_record(base + s0, k.z[2]);
    load_edge_record(base + s0 + s1, k.z[3]);
  } else {
    const CellEdges<kStorage> c(f, node, slice_base);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float lo[3], hi[3];
      load_node<kStorage>(c.e[e], 0, lo[0], lo[1], lo[2]);
      load_node<kStorage>(c.e[e], 1, hi[0], hi[1], hi[2]);
#pragma unroll
      for (int c2 = 0; c2 < 3; ++c2) k.z[e][c2] = make_float2(lo[c2], hi[c2]);
    }
  }
}

__device__ __forceinline__ void trilinear(const CornerNodes& k, const Weights& w, float2& v01,
                                          float& v2) {
  const float2 t21 = sum2(splat(1.0f), neg2(w.w21));
  const float t0 = __fsub_rn(1.0f, w.w0);
  const float2 W2 = splat(w.w21.x), T2 = splat(t21.x);
  const float2 W1 = splat(w.w21.y), T1 = splat(t21.y);
  const float2 W0 = splat(w.w0), T0 = splat(t0);
  auto lerp = [](float2 lo, float2 hi, float2 t, float2 u) {
#if DPA_F32_PACKED_LERP
    return add2(mul2(t, lo), mul2(u, hi));
#else
    return add2(mul2_scalar(t, lo), mul2_scalar(u, hi));
#endif
  };
  const float2 e0 = lerp(k.xy[0], k.xy[1], T2, W2);
  const float2 e1 = lerp(k.xy[2], k.xy[3], T2, W2);
  const float2 e2 = lerp(k.xy[4], k.xy[5], T2, W2);
  const float2 e3 = lerp(k.xy[6], k.xy[7], T2, W2);
  const float2 f0 = lerp(e0, e1, T1, W1);
  const float2 f1 = lerp(e2, e3, T1, W1);
  v01 = lerp(f0, f1, T0, W0);
  const float2 e02 = lerp(k.z04, k.z15, T2, W2);  // (e0, e2) of component 2
  const float2 e13 = lerp(k.z26, k.z37, T2, W2);  // (e1, e3)
  const float2 f01 = lerp(e02, e13, T1, W1);      // (f0, f1)
  v2 = __fadd_rn(__fmul_rn(t0, f01.x), __fmul_rn(w.w0, f01.y));
}

// (1 - w) * lo + w * hi for the pair lohi = (lo, hi) and tw = (1 - w, w).
__device__ __forceinline__ float lerp_pair(float2 lohi, float2 tw) {
  const float2 m = mul2(tw, lohi);
  return __fadd_rn(m.x, m.y);
}

__device__ __forceinline__ void trilinear(const CornerEdges& k, const Weights& w, float2& v01,
                                          float& v2) {
  const float2 tw2 = make_float2(__fsub_rn(1.0f, w.w21.x), w.w21.x);
  const float2 tw1 = make_float2(__fsub_rn(1.0f, w.w21.y), w.w21.y);
  const float2 tw0 = make_float2(__fsub_rn(1.0f, w.w0), w.w0);
  float v[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float e0 = lerp_pair(k.z[0][c], tw2), e1 = lerp_pair(k.z[1][c], tw2);
    const float e2 = lerp_pair(k.z[2][c], tw2), e3 = lerp_pair(k.z[3][c], tw2);
    const float f0 = lerp_pair(make_float2(e0, e1), tw1);
    const float f1 = lerp_pair(make_float2(e2, e3), tw1);
    v[c] = lerp_pair(make_float2(f0, f1), tw0);
  }
  v01 = make_float2(v[0], v[1]);
  v2 = v[2];
}

// A per-thread cache of the current cell's corners: a particle usually stays
// in one cell for several steps, and the sampled values do not depend on
// whether the corners came from the cache or from memory.
template <int kStorage, int kLocate>
struct CellSampler {
  CornersOf<kStorage> corners;
  uint32_t cached = ~0u;  // first node of the cached cell (no cell starts there)

  // Samples at p (a steady field: the time t is not used); returns false
  // when p is outside the grid. The sample is returned as v01 = (v0, v1)
  // and v2.
  __device__ __forceinline__ bool sample(const FieldView& f, const Position& p, float /*t*/,
                                         float2& v01, float& v2) {
    uint32_t node;
    Weights w;
    if (!locate<kLocate>(f, p, node, w)) return false;
    if (node != cached) {
      gather<kStorage>(f, node, corners);
      cached = node;
    }
    trilinear(corners, w, v01, v2);
    return true;
  }

  // sample() without the early return, for a caller that selects its result:
  // an outside position loads no corners, and its sample (from the cached
  // ones) is to be discarded.
  __device__ __forceinline__ bool sample_selected(const FieldView& f, const Position& p,
                                                  float2& v01, float& v2) {
    uint32_t node;
    Weights w;
    const bool inside = locate<kLocate>(f, p, node, w);
    const bool need = inside && node != cached;
    if constexpr (kStorage == DPA_STORAGE_F32) {
      gather_if(f, node, need, corners);
      cached = need ? node : cached;
    } else if (need) {
      gather<kStorage>(f, node, corners);
      cached = node;
    }
    trilinear(corners, w, v01, v2);
    return inside;
  }

  static constexpr bool kSteady = true;

  __device__ __forceinline__ void reset() { cached = ~0u; }
};

// The time axis of a time-varying field, located by the spatial rule: slice
// s = floor((t - t0) / dt) of the rounded quotient, weight fmod(t - t0, dt) / dt,
// inside iff 0 <= s <= slices - 2. Returns the first node of slice s.
__device__ __forceinline__ bool locate_time(const FieldView& f, float t, int64_t& slice_base,
                                            float& w) {
  const float a = __fsub_rn(t, f.time_origin);
  const float y = f.time_reciprocal, yl = f.time_reciprocal_lo;
  const float q = f.time_fast ? divide_by_reciprocal(a, f.time_spacing, y, yl)
                              : __fdiv_rn(a, f.time_spacing);
  if (!(q >= 0.0f && q < f.time_upper)) return false;
  const float s = floorf(q);
  float r = fmaf(-s, f.time_spacing, a);
  if (r < 0.0f) r = __fadd_rn(r, f.time_spacing);
  if (r == 0.0f) r = copysignf(0.0f, a);
  w = f.time_fast ? divide_by_reciprocal(r, f.time_spacing, y, yl)
                   : __fdiv_rn(r, f.time_spacing);
  slice_base = int64_t(s) * f.slice_stride;
  return true;
}

// Sampler of a time-varying field: the trilinear samples of the two slices
// around t at p, blended as (1 - w) * a + w * b per component. It caches the
// corners of both slices for the current cell and slice pair: a pathline
// usually stays in one cell for many steps and in one slice pair for many
// more, and the sampled values do not depend on whether the corners came
// from the cache or from memory.
template <int kStorage, int kLocate>
struct TimeSampler {
  CornersOf<kStorage> lo, hi;  // slices s and s + 1
  uint32_t cached = ~0u;
  int64_t cached_slice = -1;

  __device__ __forceinline__ bool sample(const FieldView& f, const Position& p, float t,
                                         float2& v01, float& v2) {
    uint32_t node;
    Weights w;
    if (!locate<kLocate>(f, p, node, w)) return false;
    int64_t slice = 0;
    float wt = 0.0f;
    if (!locate_time(f, t, slice, wt)) return false;
    if (node != cached || slice != cached_slice) {
      gather<kStorage>(f, node, lo, slice);
      gather<kStorage>(f, node, hi, slice + f.slice_stride);
      cached = node;
      cached_slice = slice;
    }
    float2 a01, b01;
    float a2, b2;
    trilinear(lo, w, a01, a2);
    trilinear(hi, w, b01, b2);
    const float u = __fsub_rn(1.0f, wt);
    v01 = add2(mul2_scalar(splat(u), a01), mul2_scalar(splat(wt), b01));
    v2 = __fadd_rn(__fmul_rn(u, a2), __fmul_rn(wt, b2));
    return true;
  }

  static constexpr bool kSteady = false;

  __device__ __forceinline__ void reset() {
    cached = ~0u;
    cached_slice = -1;
  }
};

__device__ __forceinline__ bool is_zero(float2 v01, float v2) {
  return fabsf(v01.x) <= kZeroPrecision && fabsf(v01.y) <= kZeroPrecision &&
         fabsf(v2) <= kZeroPrecision;
}

enum StepResult : int { kStepTaken = 0, kStepOutOfBounds = 1, kStepZeroVelocity = 2 };

// What the general steppers keep of a particle's previous step: its
// derivative (as v01, v2) and whether the particle has taken a step yet.
// Every particle starts fresh, as the reference copies its integrator per
// particle (particle_advector.cpp:335).
struct StepHistory {
  float2 d01;
  float d2;
  bool started;
};

// odeint modified_midpoint with kSteps sub-steps and the state-independent
// derivative d, one component: m_x1 = x + h d; kSteps - 1 times
// (m_x1, m_x0) = (m_x0 + h2 d, m_x1); out = 0.5 m_x0 + 0.5 m_x1 + (0.5 h) d.
// mm = {h, h2, 0.5 h}.
template <int kSteps>
__device__ __forceinline__ float modified_midpoint(float x, float d, const float* mm) {
  float x1 = __fadd_rn(x, __fmul_rn(mm[0], d));
  float x0 = x;
#pragma unroll
  for (int i = 1; i < kSteps; ++i) {
    const float t = x1;
    x1 = __fadd_rn(x0, __fmul_rn(mm[1], d));
    x0 = t;
  }
  return __fadd_rn(__fadd_rn(__fmul_rn(0.5f, x0), __fmul_rn(0.5f, x1)), __fmul_rn(mm[2], d));
}

// The Adams methods' initialising stepper (an order-4 extrapolation
// stepper): modified midpoints with 2 and 4 sub-steps, one polynomial
// extrapolation x = (1 + c) mm4 + (-c) mm2, c = 1/3.
__device__ __forceinline__ float extrapolated_start(float x, float d, const GeneralCoefficients& g) {
  const float a = modified_midpoint<2>(x, d, g.mm2);
  const float b = modified_midpoint<4>(x, d, g.mm4);
  return __fadd_rn(__fmul_rn(g.ex[0], b), __fmul_rn(g.ex[1], a));
}

// One step of a general stepper (kGeneralIntegrator) given this step's
// derivative; updates the history.
__device__ __forceinline__ void general_step(const GeneralCoefficients& g, float2 v01, float v2,
                                             StepHistory& h, Position& p) {
  if (g.kind == kGeneralMidpoint) {
    p.p0 = modified_midpoint<2>(p.p0, v2, g.mm2);
    p.p21 = make_float2(modified_midpoint<2>(p.p21.x, v01.x, g.mm2),
                        modified_midpoint<2>(p.p21.y, v01.y, g.mm2));
  } else if (g.extrapolated_start && !h.started) {
    p.p0 = extrapolated_start(p.p0, v2, g);
    p.p21 = make_float2(extrapolated_start(p.p21.x, v01.x, g),
                        extrapolated_start(p.p21.y, v01.y, g));
  } else {
    float x0 = p.p0, xa = p.p21.x, xb = p.p21.y;
#pragma unroll
    for (int i = 0; i < 13; ++i) {
      if (i < g.terms) {
        const bool prev = h.started && ((g.prev_mask >> i) & 1u);
        x0 = __fadd_rn(x0, __fmul_rn(g.s[i], prev ? h.d2 : v2));
        xa = __fadd_rn(xa, __fmul_rn(g.s[i], prev ? h.d01.x : v01.x));
        xb = __fadd_rn(xb, __fmul_rn(g.s[i], prev ? h.d01.y : v01.y));
      }
    }
    p.p0 = x0;
    p.p21 = make_float2(xa, xb);
  }
  h.d01 = v01;
  h.d2 = v2;
  h.started = true;
}

// One integrator step in place. The derivative of p0 is v2 and that of
// (p2, p1) is (v0, v1) (particle_advector.cpp:369).
// t is the particle's time (used by time-varying fields only); the caller
// advances it by dt after a step is taken.
// active: false for an empty slot, which the branch-free steps below run
// through without moving it (its position is parked inside the grid).
template <int kIntegrator, class Sampler>
__device__ __forceinline__ int step(const FieldView& f, const StepCoefficients& k,
                                   Sampler& sampler, Position& p, float t,
                                   StepHistory& history, bool active = true) {
  float2 v01;
  float v2;
  if constexpr (Sampler::kSteady && (kIntegrator == DPA_INTEGRATOR_EULER ||
                                     kIntegrator == DPA_INTEGRATOR_RUNGE_KUTTA_4)) {
    // Without branches on the outcome: the step is computed whatever the
    // sample, and kept only when the position was inside and the velocity
    // not zero (a step's latency is a dependent chain; the launch's end and
    // launches of few particles wait for it).
    const bool inside = sampler.sample_selected(f, p, v01, v2);
    const bool zero = is_zero(v01, v2);
    Position n = p;
    if constexpr (kIntegrator == DPA_INTEGRATOR_EULER) {
      n.p0 = __fadd_rn(p.p0, __fmul_rn(k.dt, v2));
      n.p21 = add2(p.p21, mul2(splat(k.dt), v01));
    } else {
      const float m0 = __fmul_rn(k.c0, v2), m1 = __fmul_rn(k.c1, v2);
      n.p0 = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(p.p0, m0), m1), m1), m0);
      const float2 n0 = mul2(splat(k.c0), v01), n1 = mul2(splat(k.c1), v01);
      n.p21 = add2(add2(add2(add2(p.p21, n0), n1), n1), n0);
    }
    const bool taken = active && inside && !zero;
    p.p0 = taken ? n.p0 : p.p0;
    p.p21 = make_float2(taken ? n.p21.x : p.p21.x, taken ? n.p21.y : p.p21.y);
    return !(active && inside) ? int(kStepOutOfBounds)
           : zero              ? int(kStepZeroVelocity)
                               : int(kStepTaken);
  }
  if (!sampler.sample(f, p, t, v01, v2)) return kStepOutOfBounds;
  if (is_zero(v01, v2)) return kStepZeroVelocity;
  if constexpr (kIntegrator == DPA_INTEGRATOR_EULER) {
    // odeint euler: x = 1 * x + dt * dxdt
    p.p0 = __fadd_rn(p.p0, __fmul_rn(k.dt, v2));
    p.p21 = add2(p.p21, mul2(splat(k.dt), v01));
  } else if constexpr (kIntegrator == DPA_INTEGRATOR_RUNGE_KUTTA_4) {
    // odeint runge_kutta4, final stage with four equal stage derivatives:
    // x = 1 * x + (b0 dt) d + (b1 dt) d + (b2 dt) d + (b3 dt) d, left to right.
    const float m0 = __fmul_rn(k.c0, v2), m1 = __fmul_rn(k.c1, v2);
    p.p0 = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(p.p0, m0), m1), m1), m0);
    const float2 n0 = mul2(splat(k.c0), v01), n1 = mul2(splat(k.c1), v01);
    p.p21 = add2(add2(add2(add2(p.p21, n0), n1), n1), n0);
  } else if constexpr (kIntegrator == kGeneralIntegrator) {
    general_step(k.g, v01, v2, history, p);
  } else {
    // Four-sample RK4; a stage outside the grid ends the particle without
    // taking the step.
    float2 k2_01, k3_01, k4_01;
    float k2_2, k3_2, k4_2;
    Position x;
    x.p0 = __fadd_rn(p.p0, __fmul_rn(k.half, v2));
    x.p21 = add2(p.p21, mul2(splat(k.half), v01));
    const float t_half = __fadd_rn(t, k.half), t_end = __fadd_rn(t, k.dt);
    if (!sampler.sample(f, x, t_half, k2_01, k2_2)) return kStepOutOfBounds;
    x.p0 = __fadd_rn(p.p0, __fmul_rn(k.half, k2_2));
    x.p21 = add2(p.p21, mul2(splat(k.half), k2_01));
    if (!sampler.sample(f, x, t_half, k3_01, k3_2)) return kStepOutOfBounds;
    x.p0 = __fadd_rn(p.p0, __fmul_rn(k.dt, k3_2));
    x.p21 = add2(p.p21, mul2(splat(k.dt), k3_01));
    if (!sampler.sample(f, x, t_end, k4_01, k4_2)) return kStepOutOfBounds;
    p.p0 = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(p.p0, __fmul_rn(k.c0, v2)),
                                         __fmul_rn(k.c1, k2_2)),
                               __fmul_rn(k.c1, k3_2)),
                     __fmul_rn(k.c0, k4_2));
    const float2 C0 = splat(k.c0), C1 = splat(k.c1);
    p.p21 = add2(add2(add2(add2(p.p21, mul2(C0, v01)), mul2(C1, k2_01)), mul2(C1, k3_01)),
                 mul2(C0, k4_01));
  }
  return kStepTaken;
}

}  // namespace dpa
