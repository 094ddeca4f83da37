// advect.cu -- steady-field advection launches and the processing-order,
// batch and serving helper kernels.
#include <algorithm>

#include "advect_kernel.cuh"

namespace dpa {

namespace {

// Interleaves the low 4 bits of v with two zero bits between them.
__device__ __forceinline__ uint32_t spread4(uint32_t v) {
  v &= 0xfu;
  v = (v | (v << 4)) & 0x0c3u;
  v = (v | (v << 2)) & 0x249u;
  return v;
}

// Processing-order bucket of a particle: the Morton code of its start cell
// on a resolution^3 coarsening of the grid (resolution <= 16, so at most 4096
// buckets), or kOrderBuckets for particles that start outside the grid.
__device__ __forceinline__ uint32_t order_bucket(const FieldView& f, const float* p,
                                                 uint32_t resolution) {
  uint32_t c[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float q = (p[i] - f.offset[i]) * (1.0f / f.spacing[i]);
    if (!(q >= 0.0f && q < f.upper[i])) return kOrderBuckets;
    c[i] = uint32_t(floorf(q)) * resolution / uint32_t(f.n[i]);
  }
  return (spread4(c[0]) << 2) | (spread4(c[1]) << 1) | spread4(c[2]);
}

__global__ void order_clear_kernel(uint32_t* counts) {
  for (int i = threadIdx.x; i <= kOrderBuckets; i += blockDim.x) counts[i] = 0;
}

__global__ void order_histogram_kernel(const FieldView f, const float* positions, uint64_t count,
                                       uint16_t* buckets, uint32_t* counts, uint32_t resolution) {
  __shared__ uint32_t local[kOrderBuckets + 1];
  for (int i = threadIdx.x; i <= kOrderBuckets; i += blockDim.x) local[i] = 0;
  __syncthreads();
  for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < count;
       t += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t b = order_bucket(f, positions + 3 * t, resolution);
    buckets[t] = uint16_t(b);
    atomicAdd(&local[b], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i <= kOrderBuckets; i += blockDim.x)
    if (local[i]) atomicAdd(&counts[i], local[i]);
}

// Exclusive scan of the bucket counts in one block; counts become cursors.
__global__ void __launch_bounds__(1024) order_scan_kernel(uint32_t* counts) {
  constexpr int kPer = (kOrderBuckets + 1 + 1023) / 1024;
  __shared__ uint32_t sums[1024];
  uint32_t v[kPer];
  uint32_t total = 0;
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int i = threadIdx.x * kPer + j;
    v[j] = i <= kOrderBuckets ? counts[i] : 0u;
    total += v[j];
  }
  sums[threadIdx.x] = total;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const uint32_t add = threadIdx.x >= off ? sums[threadIdx.x - off] : 0u;
    __syncthreads();
    sums[threadIdx.x] += add;
    __syncthreads();
  }
  uint32_t run = sums[threadIdx.x] - total;
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int i = threadIdx.x * kPer + j;
    if (i <= kOrderBuckets) counts[i] = run;
    run += v[j];
  }
}

__global__ void order_scatter_kernel(const uint16_t* buckets, uint64_t count, uint32_t* cursors,
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
                                     uint32_t ranges, uint64_t total, uint32_t* list) {
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= total) return;
  uint32_t lo = 0, hi = ranges;  // last range whose first entry is <= t
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (firsts[mid] <= t) lo = mid;
    else hi = mid;
  }
  list[t] = uint32_t(starts[lo] + (t - firsts[lo]));
}

}  // namespace

cudaError_t launch_expand_ranges(const uint64_t* starts, const uint64_t* firsts, uint32_t ranges,
                                 uint64_t total, uint32_t* list, cudaStream_t stream) {
  if (total == 0 || ranges == 0) return cudaSuccess;
  expand_ranges_kernel<<<unsigned((total + 255) / 256), 256, 0, stream>>>(starts, firsts, ranges,
                                                                          total, list);
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
  if (f.slices > 1) return launch_advect_unsteady(f, a, integrator, record, stream);
  return launch_family<false>(f, a, integrator, record, stream);
}

cudaError_t prepare_advect(const FieldView& f, int integrator, bool record) {
  AdvectArgs a{};
  a.count = 0;
  return launch_advect(f, a, integrator, record, nullptr);
}

cudaError_t launch_order(const FieldView& f, const float* positions, uint64_t count,
                         uint16_t* buckets, uint32_t* counts, uint32_t* order, cudaStream_t stream,
                         uint32_t resolution) {
  if (count == 0) return cudaSuccess;
  if (resolution < 1 || resolution > 16) resolution = 16;
  order_clear_kernel<<<1, 1024, 0, stream>>>(counts);
  const uint64_t blocks = std::min<uint64_t>((count + 255) / 256, 4 * 148);
  order_histogram_kernel<<<unsigned(blocks), 256, 0, stream>>>(f, positions, count, buckets, counts,
                                                               resolution);
  order_scan_kernel<<<1, 1024, 0, stream>>>(counts);
  order_scatter_kernel<<<unsigned((count + 255) / 256), 256, 0, stream>>>(buckets, count, counts,
                                                                           order);
  return cudaGetLastError();
}

}  // namespace dpa
