// emit.cu -- curve emission: prune, index pairs and angular-velocity colors of
// one round, one warp per particle, compacted with ballot/popc.
//
// Restates, data-parallel, particle_advector::prune_integral_curves
// (particle_advector.cpp:402-408), index_generator::generate
// (index_generator.cpp:10-39) and color_generator::
// generate_from_angular_velocities (color_generator.cpp:37-58). The output is
// the reference's round curve: vertices in round-particle order, invalid
// sentinels removed, index pairs (i, i + 1) for consecutive vertices neither
// of which is the terminal sentinel, and one color per vertex.
#include "kernels.cuh"
#include "sample.cuh"

namespace dpa {

namespace {

constexpr int kEmitWarps = 8;

struct V3 {
  float x, y, z;
};

__device__ __forceinline__ V3 load3(const float* p) { return {p[0], p[1], p[2]}; }

__device__ __forceinline__ void store3(float* p, const V3& v) {
  p[0] = v.x;
  p[1] = v.y;
  p[2] = v.z;
}

// Eigen 3.3 squaredNorm / dot on 3 elements: c0 + (c1 + c2).
__device__ __forceinline__ float sum3(float a, float b, float c) {
  return __fadd_rn(a, __fadd_rn(b, c));
}

// Eigen normalized(): v / sqrt(|v|^2), or v unchanged when |v|^2 == 0.
__device__ __forceinline__ V3 normalized(V3 v) {
  const float z = sum3(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y), __fmul_rn(v.z, v.z));
  if (z > 0.0f) {
    const float n = __fsqrt_rn(z);
    v.x = __fdiv_rn(v.x, n);
    v.y = __fdiv_rn(v.y, n);
    v.z = __fdiv_rn(v.z, n);
  }
  return v;
}

// atan2(|prev x next|, prev . next) (color_generator.cpp:51-54).
__device__ __forceinline__ float angular_velocity(const V3& a, const V3& b) {
  const float cx = __fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y));
  const float cy = __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z));
  const float cz = __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x));
  const float norm = __fsqrt_rn(sum3(__fmul_rn(cx, cx), __fmul_rn(cy, cy), __fmul_rn(cz, cz)));
  const float dot = sum3(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z));
  return atan2f(norm, dot);
}

template <bool kIndex64, bool kColors>
__global__ void __launch_bounds__(kEmitWarps * 32) emit_kernel(const EmitArgs e) {
  const uint64_t k = uint64_t(blockIdx.x) * kEmitWarps + (threadIdx.x >> 5);
  if (k >= e.count) return;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lanes_below = (1u << lane) - 1u;

  // Pass 1: copy the particle's surviving raw vertices to their pruned slots.
  const float* raw = e.raw_vertices + 3 * e.raw_offsets[k];
  const uint64_t raw_count = e.steps_raw[k];
  const uint64_t first = e.vertex_offsets[k];
  uint64_t cursor = first;
  for (uint64_t j0 = 0; j0 < raw_count; j0 += 32) {
    const uint64_t j = j0 + lane;
    V3 v = {0.0f, 0.0f, 0.0f};
    bool keep = false;
    if (j < raw_count) {
      v = load3(raw + 3 * j);
      keep = !equals3(v.x, v.y, v.z, kInvalid);
    }
    const unsigned mask = __ballot_sync(0xffffffffu, keep);
    if (keep) store3(e.vertices + 3 * (cursor + __popc(mask & lanes_below)), v);
    cursor += __popc(mask);
  }
  __syncwarp();

  // Pass 2: index pairs and colors over the particle's pruned vertices. The
  // last one is always the terminal sentinel, so no pair or neighbour reaches
  // into another particle's curve; the reference's "vertex_index > 1" test
  // (color_generator.cpp:50) is applied to the round-level index.
  const uint64_t kept = e.kept_vertices[k];
  uint64_t segment = e.segment_offsets[k];
  for (uint64_t m0 = 0; m0 < kept; m0 += 32) {
    const uint64_t m = m0 + lane;
    const bool valid = m < kept;
    const uint64_t local = first + m;
    const uint64_t global = e.vertex_base + local;
    bool pair = false;
    V3 y = {0.0f, 0.0f, 0.0f};
    bool terminal = true, next_open = false, prev_open = false;
    V3 yn = y, yp = y;
    if (valid) {
      y = load3(e.vertices + 3 * local);
      terminal = equals3(y.x, y.y, y.z, kTerminal);
      if (m + 1 < kept) {
        yn = load3(e.vertices + 3 * (local + 1));
        next_open = !equals3(yn.x, yn.y, yn.z, kTerminal);
      }
      if (m > 0 && global > 1) {
        yp = load3(e.vertices + 3 * (local - 1));
        prev_open = !equals3(yp.x, yp.y, yp.z, kTerminal);
      }
      pair = !terminal && next_open;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, pair);
    if (pair) {
      const uint64_t slot = 2 * (segment + __popc(mask & lanes_below));
      if constexpr (kIndex64) {
        uint64_t* out = static_cast<uint64_t*>(e.indices);
        out[slot] = global;
        out[slot + 1] = global + 1;
      } else {
        uint32_t* out = static_cast<uint32_t*>(e.indices);
        out[slot] = uint32_t(global);
        out[slot + 1] = uint32_t(global + 1);
      }
    }
    segment += __popc(mask);
    if constexpr (kColors) {
      if (valid) {
        float color = 0.0f;
        if (!terminal) {
          V3 a = {0.0f, 0.0f, 0.0f}, b = {0.0f, 0.0f, 0.0f};
          if (prev_open)
            a = normalized({__fsub_rn(y.x, yp.x), __fsub_rn(y.y, yp.y), __fsub_rn(y.z, yp.z)});
          if (next_open)
            b = normalized({__fsub_rn(yn.x, y.x), __fsub_rn(yn.y, y.y), __fsub_rn(yn.z, y.z)});
          color = angular_velocity(a, b);
        }
        e.colors[local] = color;
      }
    }
  }
}

__global__ void raw_counts_kernel(const uint64_t* in, const uint64_t* out, uint64_t count,
                                  uint64_t* raw) {
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < count) raw[t] = in[t] - out[t] + 2;
}

// Curve offsets: the exclusive scans of the per-particle kept-vertex and
// kept-segment counts (uint32) into uint64 offsets, the data-parallel form of
// the running positions that index_generator::generate (index_generator.cpp:
// 10-39) and prune_integral_curves walk serially. Three passes over tiles of
// kScanTileItems particles: tile sums, one block's scan of the tile sums
// (which also writes the two totals), and each tile's scan plus its prefix.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;  // consecutive particles per thread
constexpr uint64_t kScanTileItems = uint64_t(kScanThreads) * kScanItems;

// Block-wide exclusive scan of one pair of values per thread; returns the
// block's totals through total.
__device__ __forceinline__ ulonglong2 block_exclusive_scan2(ulonglong2 v, ulonglong2* warp_sums,
                                                           ulonglong2* total) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  ulonglong2 x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long a = __shfl_up_sync(0xffffffffu, x.x, o);
    const unsigned long long b = __shfl_up_sync(0xffffffffu, x.y, o);
    if (lane >= unsigned(o)) {
      x.x += a;
      x.y += b;
    }
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  ulonglong2 before = make_ulonglong2(0, 0), all = make_ulonglong2(0, 0);
  for (unsigned w = 0; w < blockDim.x / 32; ++w) {
    const ulonglong2 ws = warp_sums[w];
    if (w < warp) {
      before.x += ws.x;
      before.y += ws.y;
    }
    all.x += ws.x;
    all.y += ws.y;
  }
  __syncthreads();  // warp_sums may be reused by the caller's next scan
  *total = all;
  return make_ulonglong2(before.x + x.x - v.x, before.y + x.y - v.y);
}

__device__ __forceinline__ ulonglong2 load_counts(const uint32_t* a, const uint32_t* b,
                                                  uint64_t n, uint64_t i) {
  return i < n ? make_ulonglong2(a[i], b[i]) : make_ulonglong2(0, 0);
}

__global__ void __launch_bounds__(kScanThreads) offsets_tile_sums_kernel(
    const uint32_t* a, const uint32_t* b, uint64_t n, ulonglong2* tile_sums) {
  __shared__ ulonglong2 warp_sums[kScanThreads / 32];
  const uint64_t first = uint64_t(blockIdx.x) * kScanTileItems;
  ulonglong2 sum = make_ulonglong2(0, 0);
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {  // coalesced: item j * threads + t
    const ulonglong2 v = load_counts(a, b, n, first + uint64_t(j) * kScanThreads + threadIdx.x);
    sum.x += v.x;
    sum.y += v.y;
  }
  ulonglong2 total;
  block_exclusive_scan2(sum, warp_sums, &total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// One block: tile sums -> exclusive tile prefixes in place, in chunks of
// kScanThreads with a running carry; totals receives the grand totals.
__global__ void __launch_bounds__(kScanThreads) offsets_tile_prefix_kernel(
    ulonglong2* tile_sums, uint64_t tiles, unsigned long long* totals) {
  __shared__ ulonglong2 warp_sums[kScanThreads / 32];
  ulonglong2 carry = make_ulonglong2(0, 0);
  for (uint64_t base = 0; base < tiles; base += kScanThreads) {
    const uint64_t i = base + threadIdx.x;
    const ulonglong2 v = i < tiles ? tile_sums[i] : make_ulonglong2(0, 0);
    ulonglong2 total;
    const ulonglong2 ex = block_exclusive_scan2(v, warp_sums, &total);
    if (i < tiles) tile_sums[i] = make_ulonglong2(carry.x + ex.x, carry.y + ex.y);
    carry.x += total.x;
    carry.y += total.y;
  }
  if (threadIdx.x == 0) {
    totals[0] = carry.x;
    totals[1] = carry.y;
  }
}

__global__ void __launch_bounds__(kScanThreads) offsets_tiles_kernel(
    const uint32_t* a, const uint32_t* b, uint64_t n, const ulonglong2* tile_prefix,
    uint64_t* out_a, uint64_t* out_b) {
  __shared__ ulonglong2 warp_sums[kScanThreads / 32];
  const uint64_t first = uint64_t(blockIdx.x) * kScanTileItems + uint64_t(threadIdx.x) * kScanItems;
  ulonglong2 v[kScanItems];
  ulonglong2 sum = make_ulonglong2(0, 0);
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    v[j] = load_counts(a, b, n, first + j);
    sum.x += v[j].x;
    sum.y += v[j].y;
  }
  ulonglong2 total;
  const ulonglong2 ex = block_exclusive_scan2(sum, warp_sums, &total);
  const ulonglong2 prefix = tile_prefix[blockIdx.x];
  ulonglong2 run = make_ulonglong2(prefix.x + ex.x, prefix.y + ex.y);
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    const uint64_t i = first + j;
    if (i < n) {
      out_a[i] = run.x;
      out_b[i] = run.y;
    }
    run.x += v[j].x;
    run.y += v[j].y;
  }
}

// Node layouts: one float4 (F32) or (x, y, z, 0) half/bfloat quad per node.
// F32_EDGES: record t holds nodes t and t + 1 along axis 2, each component's
// pair side by side (sample.cuh); the last node of a row repeats itself, and
// no cell reads that record's second half.
template <int kStorage>
__global__ void repack_kernel(const float* xyzv, uint64_t nodes, uint32_t n2, void* out) {
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= nodes) return;
  const float x = xyzv[3 * t], y = xyzv[3 * t + 1], z = xyzv[3 * t + 2];
  if constexpr (kStorage == DPA_STORAGE_F32_EDGES) {
    const uint64_t u = (t % n2) + 1 < n2 ? t + 1 : t;
    float4* o = reinterpret_cast<float4*>(out) + 2 * t;
    o[0] = make_float4(x, xyzv[3 * u], y, xyzv[3 * u + 1]);
    o[1] = make_float4(z, xyzv[3 * u + 2], 0.0f, 0.0f);
  } else if constexpr (kStorage == DPA_STORAGE_F32) {
    (void)n2;
    reinterpret_cast<float4*>(out)[t] = make_float4(x, y, z, 0.0f);
  } else if constexpr (kStorage == DPA_STORAGE_F16) {
    const __half2 a = __floats2half2_rn(x, y);
    const __half2 b = __floats2half2_rn(z, 0.0f);
    uint2 r;
    r.x = *reinterpret_cast<const unsigned*>(&a);
    r.y = *reinterpret_cast<const unsigned*>(&b);
    reinterpret_cast<uint2*>(out)[t] = r;
  } else {
    const __nv_bfloat162 a = __floats2bfloat162_rn(x, y);
    const __nv_bfloat162 b = __floats2bfloat162_rn(z, 0.0f);
    uint2 r;
    r.x = *reinterpret_cast<const unsigned*>(&a);
    r.y = *reinterpret_cast<const unsigned*>(&b);
    reinterpret_cast<uint2*>(out)[t] = r;
  }
}

inline unsigned blocks_for(uint64_t n, unsigned block) { return unsigned((n + block - 1) / block); }

}  // namespace

cudaError_t launch_emit(const EmitArgs& e, bool index64, bool colors, cudaStream_t stream) {
  if (e.count == 0) return cudaSuccess;
  const dim3 grid(blocks_for(e.count, kEmitWarps)), block(kEmitWarps * 32);
  if (index64) {
    if (colors) emit_kernel<true, true><<<grid, block, 0, stream>>>(e);
    else emit_kernel<true, false><<<grid, block, 0, stream>>>(e);
  } else {
    if (colors) emit_kernel<false, true><<<grid, block, 0, stream>>>(e);
    else emit_kernel<false, false><<<grid, block, 0, stream>>>(e);
  }
  return cudaGetLastError();
}

cudaError_t launch_raw_counts(const uint64_t* remaining_in, const uint64_t* remaining_out,
                              uint64_t count, uint64_t* raw_counts, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  raw_counts_kernel<<<blocks_for(count, 256), 256, 0, stream>>>(remaining_in, remaining_out, count,
                                                                raw_counts);
  return cudaGetLastError();
}

uint64_t curve_offsets_scratch_bytes(uint64_t count) {
  return ((count + kScanTileItems - 1) / kScanTileItems) * sizeof(ulonglong2) + 16;
}

cudaError_t launch_curve_offsets(const uint32_t* kept_vertices, const uint32_t* kept_segments,
                                 uint64_t count, void* scratch, uint64_t* vertex_offsets,
                                 uint64_t* segment_offsets, unsigned long long* totals,
                                 cudaStream_t stream) {
  if (count == 0) return cudaMemsetAsync(totals, 0, 16, stream);
  const uint64_t tiles = (count + kScanTileItems - 1) / kScanTileItems;
  if (tiles > 0x7fffffffull) return cudaErrorInvalidValue;
  ulonglong2* sums = static_cast<ulonglong2*>(scratch);
  offsets_tile_sums_kernel<<<unsigned(tiles), kScanThreads, 0, stream>>>(
      kept_vertices, kept_segments, count, sums);
  DPA_CUDA_TRY(cudaGetLastError());
  offsets_tile_prefix_kernel<<<1, kScanThreads, 0, stream>>>(sums, tiles, totals);
  DPA_CUDA_TRY(cudaGetLastError());
  offsets_tiles_kernel<<<unsigned(tiles), kScanThreads, 0, stream>>>(
      kept_vertices, kept_segments, count, sums, vertex_offsets, segment_offsets);
  return cudaGetLastError();
}

uint64_t field_node_bytes(int storage) {
  return storage == DPA_STORAGE_F32_EDGES ? 32 : storage == DPA_STORAGE_F32 ? 16 : 8;
}

cudaError_t launch_repack(const float* xyzv, uint64_t nodes, uint32_t n2, int storage, void* out,
                          cudaStream_t stream) {
  if (nodes == 0) return cudaSuccess;
  const unsigned grid = blocks_for(nodes, 256);
  switch (storage) {
    case DPA_STORAGE_F32:
      repack_kernel<DPA_STORAGE_F32><<<grid, 256, 0, stream>>>(xyzv, nodes, n2, out);
      break;
    case DPA_STORAGE_F16:
      repack_kernel<DPA_STORAGE_F16><<<grid, 256, 0, stream>>>(xyzv, nodes, n2, out);
      break;
    case DPA_STORAGE_BF16:
      repack_kernel<DPA_STORAGE_BF16><<<grid, 256, 0, stream>>>(xyzv, nodes, n2, out);
      break;
    case DPA_STORAGE_F32_EDGES:
      repack_kernel<DPA_STORAGE_F32_EDGES><<<grid, 256, 0, stream>>>(xyzv, nodes, n2, out);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace dpa
