// advect.cu -- the advection kernel: one thread per particle, every step of
// that particle in registers (particle_advector.cpp:325-396).
#include <algorithm>

#include "kernels.cuh"
#include "sample.cuh"

namespace dpa {

namespace {

// Appends one vertex to the count of the pruned curve: invalid-sentinel
// vertices are dropped by prune_integral_curves (particle_advector.cpp:402-408),
// and index_generator (index_generator.cpp:10-39) pairs consecutive kept
// vertices of which neither equals the terminal sentinel.
struct CurveCounter {
  uint32_t kept = 0;
  uint32_t segments = 0;
  bool prev_open = false;  // previous kept vertex is not terminal-valued

  __device__ __forceinline__ void append(float x, float y, float z) {
    if (equals3(x, y, z, kInvalid)) return;
    const bool terminal = equals3(x, y, z, kTerminal);
    if (!terminal && prev_open) ++segments;
    prev_open = !terminal;
    ++kept;
  }
};

template <int kIntegrator, int kStorage, bool kPow2, bool kRecord>
__global__ void __launch_bounds__(kAdvectBlock)
advect_kernel(const FieldView f, const AdvectArgs a) {
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= a.count) return;
  const uint64_t k = a.order ? a.order[t] : t;

  float p[3] = {a.positions[3 * k], a.positions[3 * k + 1], a.positions[3 * k + 2]};
  const uint64_t remaining = a.remaining[k];

  float* curve = nullptr;
  CurveCounter counter;
  if constexpr (kRecord) {
    curve = a.raw_vertices + 3 * a.raw_offsets[k];
    curve[0] = p[0];
    curve[1] = p[1];
    curve[2] = p[2];
    counter.append(p[0], p[1], p[2]);
  }

  CellSampler<kStorage, kPow2> sampler;
  uint64_t it = 0;
  int reason = DPA_TERMINATION_COMPLETE;
  for (; it < remaining; ++it) {
    const int r = step<kIntegrator, kStorage, kPow2>(f, a.coefficients, sampler, p);
    if (r != kStepTaken) {
      reason = r == kStepOutOfBounds ? DPA_TERMINATION_OUT_OF_BOUNDS : DPA_TERMINATION_ZERO_VELOCITY;
      break;
    }
    if constexpr (kRecord) {
      float* v = curve + 3 * (it + 1);
      v[0] = p[0];
      v[1] = p[1];
      v[2] = p[2];
      counter.append(p[0], p[1], p[2]);
    }
  }
  if constexpr (kRecord) {
    float* v = curve + 3 * (it + 1);
    v[0] = kTerminal;
    v[1] = kTerminal;
    v[2] = kTerminal;
    counter.append(kTerminal, kTerminal, kTerminal);
    a.kept_vertices[k] = counter.kept;
    a.kept_segments[k] = counter.segments;
  }
  a.positions[3 * k] = p[0];
  a.positions[3 * k + 1] = p[1];
  a.positions[3 * k + 2] = p[2];
  a.remaining[k] = remaining - it;
  if (a.termination) a.termination[k] = uint8_t(reason);
}

template <int kIntegrator, int kStorage, bool kPow2, bool kRecord>
cudaError_t launch_typed(const FieldView& f, const AdvectArgs& a, cudaStream_t stream) {
  const uint64_t blocks = (a.count + kAdvectBlock - 1) / kAdvectBlock;
  advect_kernel<kIntegrator, kStorage, kPow2, kRecord>
      <<<dim3(unsigned(blocks)), dim3(kAdvectBlock), 0, stream>>>(f, a);
  return cudaGetLastError();
}

template <int kIntegrator, int kStorage>
cudaError_t launch_pow2(const FieldView& f, const AdvectArgs& a, bool record, cudaStream_t s) {
  if (f.pow2) {
    return record ? launch_typed<kIntegrator, kStorage, true, true>(f, a, s)
                  : launch_typed<kIntegrator, kStorage, true, false>(f, a, s);
  }
  return record ? launch_typed<kIntegrator, kStorage, false, true>(f, a, s)
                : launch_typed<kIntegrator, kStorage, false, false>(f, a, s);
}

template <int kIntegrator>
cudaError_t launch_storage(const FieldView& f, const AdvectArgs& a, bool record, cudaStream_t s) {
  switch (f.storage) {
    case DPA_STORAGE_F32: return launch_pow2<kIntegrator, DPA_STORAGE_F32>(f, a, record, s);
    case DPA_STORAGE_F16: return launch_pow2<kIntegrator, DPA_STORAGE_F16>(f, a, record, s);
    case DPA_STORAGE_BF16: return launch_pow2<kIntegrator, DPA_STORAGE_BF16>(f, a, record, s);
    default: return cudaErrorInvalidValue;
  }
}

// Interleaves the low 4 bits of v with two zero bits between them.
__device__ __forceinline__ uint32_t spread4(uint32_t v) {
  v &= 0xfu;
  v = (v | (v << 4)) & 0x0c3u;
  v = (v | (v << 2)) & 0x249u;
  return v;
}

// Processing-order bucket of a particle: the Morton code of its start cell
// on a 16 x 16 x 16 coarsening of the grid (4096 buckets), or kOrderBuckets
// for particles that start outside the grid.
__device__ __forceinline__ uint32_t order_bucket(const FieldView& f, const float* p) {
  uint32_t c[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float q = (p[i] - f.offset[i]) * (1.0f / f.spacing[i]);
    const float s = floorf(q);
    if (!(s >= 0.0f && s <= f.limit[i])) return kOrderBuckets;
    c[i] = uint32_t(s) * 16u / uint32_t(f.n[i]);
  }
  return (spread4(c[0]) << 2) | (spread4(c[1]) << 1) | spread4(c[2]);
}

__global__ void order_clear_kernel(uint32_t* counts) {
  for (int i = threadIdx.x; i <= kOrderBuckets; i += blockDim.x) counts[i] = 0;
}

__global__ void order_histogram_kernel(const FieldView f, const float* positions, uint64_t count,
                                       uint16_t* buckets, uint32_t* counts) {
  __shared__ uint32_t local[kOrderBuckets + 1];
  for (int i = threadIdx.x; i <= kOrderBuckets; i += blockDim.x) local[i] = 0;
  __syncthreads();
  for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < count;
       t += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t b = order_bucket(f, positions + 3 * t);
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

}  // namespace

cudaError_t launch_advect(const FieldView& f, const AdvectArgs& a, int integrator, bool record,
                          cudaStream_t stream) {
  if (a.count == 0) return cudaSuccess;
  switch (integrator) {
    case DPA_INTEGRATOR_EULER:
      return launch_storage<DPA_INTEGRATOR_EULER>(f, a, record, stream);
    case DPA_INTEGRATOR_RUNGE_KUTTA_4:
      return launch_storage<DPA_INTEGRATOR_RUNGE_KUTTA_4>(f, a, record, stream);
    case DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE:
      return launch_storage<DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE>(f, a, record, stream);
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t launch_order(const FieldView& f, const float* positions, uint64_t count,
                         uint16_t* buckets, uint32_t* counts, uint32_t* order, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  order_clear_kernel<<<1, 1024, 0, stream>>>(counts);
  const uint64_t blocks = std::min<uint64_t>((count + 255) / 256, 4 * 148);
  order_histogram_kernel<<<unsigned(blocks), 256, 0, stream>>>(f, positions, count, buckets, counts);
  order_scan_kernel<<<1, 1024, 0, stream>>>(counts);
  order_scatter_kernel<<<unsigned((count + 255) / 256), 256, 0, stream>>>(buckets, count, counts,
                                                                           order);
  return cudaGetLastError();
}

}  // namespace dpa
