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

// Persistent advection: every lane owns one particle at a time and, when it
// finishes, takes the next one from its warp's claim of a.claim consecutive
// entries of the processing order; the warp claims a new batch with one
// atomic when its batch runs out. Lanes therefore stay busy while particles
// of one warp end after very different numbers of steps. A particle takes at
// most a.max_steps steps per launch; one stopped by that budget alone is
// reported as in flight and resumes in a later launch.
template <int kIntegrator, int kStorage, bool kPow2, bool kRecord>
__global__ void __launch_bounds__(kAdvectBlock, kAdvectMinBlocks)
advect_kernel(const FieldView f, const AdvectArgs a) {
  constexpr unsigned kFull = 0xffffffffu;
  const uint32_t claim = a.claim;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lanes_below = (1u << lane) - 1u;

  // Warp-uniform claim: entries [claim_next, claim_end) of the order.
  uint64_t claim_next = 0, claim_end = 0;
  bool exhausted = false;

  bool active = false;
  uint64_t k = 0, remaining = 0, budget = 0, it = 0;
  Position p{0.0f, make_float2(0.0f, 0.0f)};
  float* curve = nullptr;
  CurveCounter counter;
  CellSampler<kStorage, kPow2> sampler;
  StepHistory history{};

  while (true) {
    // Hand new particles to idle lanes.
    unsigned idle = __ballot_sync(kFull, !active);
    while (idle && !exhausted) {
      if (claim_next == claim_end) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(a.work_counter, (unsigned long long)claim);
        base = __shfl_sync(kFull, base, 0);
        if (base >= a.count) {
          exhausted = true;
          break;
        }
        claim_next = base;
        claim_end = base + claim < a.count ? base + claim : a.count;
      }
      const uint32_t left = uint32_t(claim_end - claim_next);
      const uint32_t take = uint32_t(__popc(idle)) < left ? uint32_t(__popc(idle)) : left;
      const uint32_t rank = __popc(idle & lanes_below);
      // Lanes still in the idle set take entries claim_next + rank. (A lane
      // that drew a finished particle earlier in this round is inactive but
      // no longer idle, and must not take one again.)
      const bool took = ((idle >> lane) & 1u) && rank < take;
      bool mine = took;
      if (mine) {
        const uint64_t t = claim_next + rank;
        k = a.order ? a.order[t] : t;
        // Serving: a finished particle stays finished.
        if (a.resume_only && a.termination[k] != DPA_TERMINATION_IN_FLIGHT) mine = false;
      }
      if (mine) {
        p.p0 = a.positions[3 * k];
        p.p21 = make_float2(a.positions[3 * k + 2], a.positions[3 * k + 1]);
        remaining = a.remaining[k];
        budget = remaining < a.max_steps ? remaining : a.max_steps;
        it = 0;
        sampler.reset();
        history.started = false;
        active = true;
        if constexpr (kRecord) {
          // A particle resumed from an earlier launch continues its curve
          // where that launch left it.
          const uint64_t done = a.remaining_initial ? a.remaining_initial[k] - remaining : 0;
          curve = a.raw_vertices + 3 * (a.raw_offsets[k] + done);
          counter = CurveCounter();
          if (done == 0) {
            curve[0] = p.p0;
            curve[1] = p.p21.y;
            curve[2] = p.p21.x;
            counter.append(p.p0, p.p21.y, p.p21.x);
          } else {
            counter.kept = a.kept_vertices[k];
            counter.segments = a.kept_segments[k];
            counter.prev_open = a.curve_open[k] != 0;
          }
        }
      }
      claim_next += take;
      // Every lane that took an entry leaves this round of hand-outs; one that
      // drew a finished particle (serving) stays inactive until the next.
      idle &= ~__ballot_sync(kFull, took);
    }
    if (!__any_sync(kFull, active)) {
      if (exhausted) break;
      continue;  // every lane drew a finished particle (serving): claim again
    }

    if (active) {
      int r = kStepTaken;
      if (it < budget) {
        r = step<kIntegrator, kStorage, kPow2>(f, a.coefficients, sampler, p, history);
        if (r == kStepTaken) {
          ++it;
          if constexpr (kRecord) {
            float* v = curve + 3 * it;
            v[0] = p.p0;
            v[1] = p.p21.y;
            v[2] = p.p21.x;
            counter.append(p.p0, p.p21.y, p.p21.x);
          }
        }
      }
      if (r != kStepTaken || it >= budget) {
        const int reason = r == kStepOutOfBounds    ? DPA_TERMINATION_OUT_OF_BOUNDS
                           : r == kStepZeroVelocity ? DPA_TERMINATION_ZERO_VELOCITY
                           : it >= remaining        ? DPA_TERMINATION_COMPLETE
                                                    : DPA_TERMINATION_IN_FLIGHT;
        if constexpr (kRecord) {
          if (reason != DPA_TERMINATION_IN_FLIGHT) {
            float* v = curve + 3 * (it + 1);
            v[0] = kTerminal;
            v[1] = kTerminal;
            v[2] = kTerminal;
            counter.append(kTerminal, kTerminal, kTerminal);
          } else {
            a.curve_open[k] = counter.prev_open ? 1 : 0;
          }
          a.kept_vertices[k] = counter.kept;
          a.kept_segments[k] = counter.segments;
        }
        a.positions[3 * k] = p.p0;
        a.positions[3 * k + 1] = p.p21.y;
        a.positions[3 * k + 2] = p.p21.x;
        a.remaining[k] = remaining - it;
        if (a.termination) a.termination[k] = uint8_t(reason);
        if (a.in_flight && reason != DPA_TERMINATION_IN_FLIGHT)
          atomicSub(a.in_flight + a.request_of[k], 1u);
        active = false;
      }
    }
  }
}

template <int kIntegrator, int kStorage, bool kPow2, bool kRecord>
cudaError_t resident_blocks(int* blocks_per_sm, int* sms) {
  // Per instantiation and process; every device of a process is a B200 here.
  static int resident = 0;
  static int count = 0;
  if (resident == 0) {
    int device = 0;
    DPA_CUDA_TRY(cudaGetDevice(&device));
    DPA_CUDA_TRY(cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, device));
    int r = 0;
    DPA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &r, advect_kernel<kIntegrator, kStorage, kPow2, kRecord>, kAdvectBlock, 0));
    resident = r < 1 ? 1 : r;
  }
  *blocks_per_sm = resident;
  *sms = count;
  return cudaSuccess;
}

template <int kIntegrator, int kStorage, bool kPow2, bool kRecord>
cudaError_t launch_typed(const FieldView& f, const AdvectArgs& a, cudaStream_t stream) {
  // Persistent grid: as many blocks as fit on the device at once (or as the
  // tuning asks), fewer when there are fewer particles than lanes.
  int resident = 0, sms = 0;
  DPA_CUDA_TRY((resident_blocks<kIntegrator, kStorage, kPow2, kRecord>(&resident, &sms)));
  if (a.count == 0) return cudaSuccess;  // nothing to do, or preparation only
  if (a.blocks_per_sm && int(a.blocks_per_sm) < resident) resident = int(a.blocks_per_sm);
  const uint64_t needed = (a.count + kAdvectBlock - 1) / kAdvectBlock;
  const uint64_t blocks = std::min<uint64_t>(needed, uint64_t(resident) * uint64_t(sms));
  if (blocks == 0) return cudaSuccess;
  DPA_CUDA_TRY(cudaMemsetAsync(a.work_counter, 0, sizeof(unsigned long long), stream));
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
  switch (integrator) {
    case DPA_INTEGRATOR_EULER:
      return launch_storage<DPA_INTEGRATOR_EULER>(f, a, record, stream);
    case DPA_INTEGRATOR_RUNGE_KUTTA_4:
      return launch_storage<DPA_INTEGRATOR_RUNGE_KUTTA_4>(f, a, record, stream);
    case DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE:
      return launch_storage<DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE>(f, a, record, stream);
    case DPA_INTEGRATOR_MODIFIED_MIDPOINT:
    case DPA_INTEGRATOR_RUNGE_KUTTA_CASH_KARP_54:
    case DPA_INTEGRATOR_RUNGE_KUTTA_DORMAND_PRINCE_5:
    case DPA_INTEGRATOR_RUNGE_KUTTA_FEHLBERG_78:
    case DPA_INTEGRATOR_ADAMS_BASHFORTH_2:
    case DPA_INTEGRATOR_ADAMS_BASHFORTH_MOULTON_2:
      // The coefficients in a.coefficients.g select the stepper.
      return launch_storage<kGeneralIntegrator>(f, a, record, stream);
    default:
      return cudaErrorInvalidValue;
  }
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
