// advect.cu -- the advection launch dispatch and the processing-order,
// batch and serving helper kernels.
#include <algorithm>

#include "kernels.cuh"

namespace dpa {

namespace {

// Interleaves the low 6 bits of v with two zero bits between them.
__device__ __forceinline__ uint32_t spread6(uint32_t v) {
  uint32_t r = 0;
#pragma unroll
  for (int b = 0; b < 6; ++b) r |= ((v >> b) & 1u) << (3 * b);
  return r;
}

// Processing-order bucket of a particle: the Morton code of its start cell
// on a resolution^3 coarsening of the grid, below buckets = p^3 for p the
// power of two >= resolution (<= 64), or `buckets` for particles that start
// outside the grid.
__device__ __forceinline__ uint32_t order_bucket(const FieldView& f, const float* p,
                                                 uint32_t resolution, uint32_t buckets) {
  uint32_t c[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float q = (p[i] - f.offset[i]) * (1.0f / f.spacing[i]);
    if (!(q >= 0.0f && q < f.upper[i])) return buckets;
    c[i] = uint32_t(floorf(q)) * resolution / uint32_t(f.n[i]);
  }
  return (spread6(c[0]) << 2) | (spread6(c[1]) << 1) | spread6(c[2]);
}

// Bucket ids and their counts. Lanes of a warp that share a bucket (seeds are
// often dense) add to its counter once.
__global__ void order_histogram_kernel(const FieldView f, const float* positions, uint64_t count,
                                       uint32_t* ids, uint32_t* counts, uint32_t resolution,
                                       uint32_t buckets) {
  for (uint64_t base = uint64_t(blockIdx.x) * blockDim.x; base < count;
       base += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t t = base + threadIdx.x;
    const bool live = t < count;
    const unsigned mask = __ballot_sync(0xffffffffu, live);
    if (!live) continue;
    const uint32_t b = order_bucket(f, positions + 3 * t, resolution, buckets);
    ids[t] = b;
    const unsigned same = __match_any_sync(mask, b);
    if ((threadIdx.x & 31u) == unsigned(__ffs(same) - 1))
      atomicAdd(&counts[b], uint32_t(__popc(same)));
  }
}

// Exclusive scan of the counts in tiles of kScanTile entries: tile sums,
// a scan of the sums, then each tile's scan plus its prefix. 256 threads,
// four consecutive entries each.
constexpr uint32_t kScanTile = 1024;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_sums,
                                                         uint32_t* total) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= unsigned(o)) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  uint32_t before = 0, all = 0;
  for (unsigned w = 0; w < blockDim.x / 32; ++w) {
    if (w < warp) before += warp_sums[w];
    all += warp_sums[w];
  }
  *total = all;
  return before + x - v;
}

__device__ __forceinline__ void load_tile(const uint32_t* counts, uint32_t n, uint32_t first,
                                          uint32_t v[4]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint32_t i = first + 4 * threadIdx.x + j;
    v[j] = i < n ? counts[i] : 0u;
  }
}

__global__ void __launch_bounds__(256) order_tile_sums_kernel(const uint32_t* counts, uint32_t n,
                                                              uint32_t* tile_sums) {
  __shared__ uint32_t warp_sums[8];
  uint32_t v[4];
  load_tile(counts, n, blockIdx.x * kScanTile, v);
  uint32_t total = 0;
  block_exclusive_scan(v[0] + v[1] + v[2] + v[3], warp_sums, &total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// One block: the exclusive scan of up to 256 * 4 tile sums, in place.
__global__ void __launch_bounds__(256) order_scan_sums_kernel(uint32_t* tile_sums, uint32_t tiles) {
  __shared__ uint32_t warp_sums[8];
  uint32_t v[4];
  load_tile(tile_sums, tiles, 0, v);
  uint32_t total = 0;
  uint32_t run = block_exclusive_scan(v[0] + v[1] + v[2] + v[3], warp_sums, &total);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint32_t i = 4 * threadIdx.x + j;
    if (i < tiles) tile_sums[i] = run;
    run += v[j];
  }
}

__global__ void __launch_bounds__(256) order_scan_tiles_kernel(uint32_t* counts, uint32_t n,
                                                               const uint32_t* tile_prefix) {
  __shared__ uint32_t warp_sums[8];
  uint32_t v[4];
  const uint32_t first = blockIdx.x * kScanTile;
  load_tile(counts, n, first, v);
  uint32_t total = 0;
  uint32_t run = tile_prefix[blockIdx.x] +
                 block_exclusive_scan(v[0] + v[1] + v[2] + v[3], warp_sums, &total);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint32_t i = first + 4 * threadIdx.x + j;
    if (i < n) counts[i] = run;
    run += v[j];
  }
}

__global__ void order_scatter_kernel(const uint32_t* buckets, uint64_t count, uint32_t* cursors,
                                     uint32_t* order) {
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= count) return;
  order[atomicAdd(&cursors[buckets[t]], 1u)] = uint32_t(t);
}

// One block per seed set: sum of the steps its particles took.
__global__ void set_steps_kernel(const uint64_t* in, const uint64_t* out, const uint64_t* offsets,
                                 unsigned long long* steps) {
  const uint64_t s = blockIdx.x;
  unsigned long long sum = 0;
  for (uint64_t i = offsets[s] + threadIdx.x; i < offsets[s + 1]; i += blockDim.x)
    sum += in[i] - out[i];
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
  __shared__ unsigned long long warp_sums[8];
  if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long total = 0;
    for (int w = 0; w < 8; ++w) total += warp_sums[w];
    steps[s] = total;
  }
}

__global__ void expand_ranges_kernel(const uint64_t* starts, const uint64_t* firsts,
                                     uint32_t ranges, uint64_t total, const uint32_t* order,
                                     uint32_t* list) {
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= total) return;
  uint32_t lo = 0, hi = ranges;  // last range whose first entry is <= t
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (firsts[mid] <= t) lo = mid;
    else hi = mid;
  }
  const uint64_t start = starts[lo];
  list[t] = uint32_t(start + order[start + (t - firsts[lo])]);
}

// Counts the dividends a (every 32-bit pattern) for which
// divide_by_reciprocal(a, h, y, yl) and __fdiv_rn(a, h) differ in their bits.
__global__ void verify_division_kernel(float h, float y, float yl, unsigned int* mismatches) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  unsigned int bad = 0;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < (1ull << 32);
       i += stride) {
    const float a = __uint_as_float(uint32_t(i));
    const float want = __fdiv_rn(a, h);
    const float got = divide_by_reciprocal(a, h, y, yl);
    const bool same = __float_as_uint(want) == __float_as_uint(got) || (isnan(want) && isnan(got));
    bad += same ? 0u : 1u;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) bad += __shfl_down_sync(0xffffffffu, bad, o);
  if ((threadIdx.x & 31u) == 0 && bad) atomicAdd(mismatches, bad);
}

// Data-path probe: every lane loads, per iteration, the eight 16-byte nodes
// of one cell (four edges of two consecutive nodes, the advection kernel's
// gather), from a table of mask + 1 nodes laid out as a cube of side 2^side.
// Random: each lane's cell is drawn by xorshift32 (Marsaglia, "Xorshift
// RNGs", 2003). Coalesced: the warp's lanes read consecutive cells, so each
// load instruction covers four 128-byte lines (the data path's ceiling).
__global__ void __launch_bounds__(256) gather_probe_kernel(const float4* table, uint32_t mask,
                                                           uint32_t side, uint32_t iterations,
                                                           int random, float* sink) {
  const uint32_t s1 = 1u << side, s0 = 1u << (2 * side);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u + 1u;
  uint32_t cursor = warp * 64u;
  // Random: the second node of an edge follows the first; coalesced: the
  // warp's first loads cover 32 consecutive nodes and its second loads the
  // next 32.
  const uint32_t pair = random ? 1u : 32u;
  float acc = 0.0f;
  for (uint32_t i = 0; i < iterations; ++i) {
    uint32_t c;
    if (random) {
      x ^= x << 13;
      x ^= x >> 17;
      x ^= x << 5;
      c = x;
    } else {
      c = cursor + lane;
      cursor += 64u * warps;
    }
    const uint32_t e[4] = {c, c + s1, c + s0, c + s0 + s1};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float4 a = __ldg(table + (e[k] & mask));
      const float4 b = __ldg(table + ((e[k] + pair) & mask));
      acc += a.x + a.y + a.z + b.x + b.y + b.z;
    }
  }
  if (acc == 1.5f) *sink = acc;  // keeps the loads; the table holds no such sum
}

}  // namespace

cudaError_t launch_gather_probe(const float4* table, uint32_t mask, uint32_t side,
                                uint32_t iterations, int random, float* sink, uint32_t blocks,
                                cudaStream_t stream) {
  gather_probe_kernel<<<blocks, 256, 0, stream>>>(table, mask, side, iterations, random, sink);
  return cudaGetLastError();
}

cudaError_t launch_verify_division(float h, float y, float yl, unsigned int* mismatches,
                                   cudaStream_t stream) {
  DPA_CUDA_TRY(cudaMemsetAsync(mismatches, 0, sizeof(unsigned int), stream));
  verify_division_kernel<<<148 * 8, 256, 0, stream>>>(h, y, yl, mismatches);
  return cudaGetLastError();
}

cudaError_t launch_expand_ranges(const uint64_t* starts, const uint64_t* firsts, uint32_t ranges,
                                 uint64_t total, const uint32_t* order, uint32_t* list,
                                 cudaStream_t stream) {
  if (total == 0 || ranges == 0) return cudaSuccess;
  expand_ranges_kernel<<<unsigned((total + 255) / 256), 256, 0, stream>>>(starts, firsts, ranges,
                                                                          total, order, list);
  return cudaGetLastError();
}

cudaError_t launch_set_steps(const uint64_t* remaining_in, const uint64_t* remaining_out,
                             const uint64_t* offsets, uint64_t sets, unsigned long long* steps,
                             cudaStream_t stream) {
  if (sets == 0) return cudaSuccess;
  set_steps_kernel<<<unsigned(sets), 256, 0, stream>>>(remaining_in, remaining_out, offsets, steps);
  return cudaGetLastError();
}

cudaError_t launch_advect(const FieldView& f, const AdvectArgs& a, int integrator, bool record,
                          cudaStream_t stream) {
  const bool unsteady = f.slices > 1;
  switch (f.storage) {
    case DPA_STORAGE_F32:
      return unsteady ? launch_advect_storage<DPA_STORAGE_F32, true>(f, a, integrator, record, stream)
                      : launch_advect_storage<DPA_STORAGE_F32, false>(f, a, integrator, record, stream);
    case DPA_STORAGE_F16:
      return unsteady ? launch_advect_storage<DPA_STORAGE_F16, true>(f, a, integrator, record, stream)
                      : launch_advect_storage<DPA_STORAGE_F16, false>(f, a, integrator, record, stream);
    case DPA_STORAGE_BF16:
      return unsteady ? launch_advect_storage<DPA_STORAGE_BF16, true>(f, a, integrator, record, stream)
                      : launch_advect_storage<DPA_STORAGE_BF16, false>(f, a, integrator, record, stream);
    case DPA_STORAGE_F32_EDGES:
      return unsteady
                 ? launch_advect_storage<DPA_STORAGE_F32_EDGES, true>(f, a, integrator, record, stream)
                 : launch_advect_storage<DPA_STORAGE_F32_EDGES, false>(f, a, integrator, record,
                                                                        stream);
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t prepare_advect(const FieldView& f, const AdvectArgs& launch, int integrator,
                           bool record) {
  AdvectArgs a = launch;
  a.count = 0;
  return launch_advect(f, a, integrator, record, nullptr);
}

cudaError_t launch_order(const FieldView& f, const float* positions, uint64_t count,
                         uint32_t* ids, uint32_t* counts, uint32_t* order, cudaStream_t stream,
                         uint32_t resolution) {
  if (count == 0) return cudaSuccess;
  if (resolution < 1 || resolution > kOrderMaxResolution) resolution = kOrderDefaultResolution;
  uint32_t p = 1;
  while (p < resolution) p *= 2;
  const uint32_t buckets = p * p * p;
  const uint32_t n = buckets + 1;  // the last counts the particles outside the grid
  const uint32_t tiles = (n + kScanTile - 1) / kScanTile;
  uint32_t* tile_sums = counts + kOrderBuckets + 1;
  DPA_CUDA_TRY(cudaMemsetAsync(counts, 0, n * sizeof(uint32_t), stream));
  const uint64_t blocks = std::min<uint64_t>((count + 255) / 256, 4 * 148);
  order_histogram_kernel<<<unsigned(blocks), 256, 0, stream>>>(f, positions, count, ids, counts,
                                                               resolution, buckets);
  order_tile_sums_kernel<<<tiles, 256, 0, stream>>>(counts, n, tile_sums);
  order_scan_sums_kernel<<<1, 256, 0, stream>>>(tile_sums, tiles);
  order_scan_tiles_kernel<<<tiles, 256, 0, stream>>>(counts, n, tile_sums);
  order_scatter_kernel<<<unsigned((count + 255) / 256), 256, 0, stream>>>(ids, count, counts,
                                                                           order);
  return cudaGetLastError();
}

}  // namespace dpa
