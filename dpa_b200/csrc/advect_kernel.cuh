// advect_kernel.cuh -- the advection kernel template and its launchers:
// every step of a particle in registers (particle_advector.cpp:325-396), one
// or two particles per lane. advect_f32.cu, advect_f32e.cu, advect_f16.cu and
// advect_bf16.cu instantiate it per field storage, for steady and
// time-varying fields.
#pragma once

#include <algorithm>
#include <atomic>
#include <type_traits>

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

  __device__ __forceinline__ void append(float x, float y, float z, bool taken = true) {
    const bool valid = taken && !equals3(x, y, z, kInvalid);
    const bool terminal = equals3(x, y, z, kTerminal);
    segments += valid && !terminal && prev_open ? 1u : 0u;
    prev_open = valid ? !terminal : prev_open;
    kept += valid ? 1u : 0u;
  }
};

template <int kIntegrator, bool kUnsteady, int kPPT>
constexpr int advect_min_blocks() {
  return kPPT == 2                                       ? kAdvectPpt2MinBlocks
         : kUnsteady                                     ? kAdvectUnsteadyMinBlocks
         : kIntegrator == DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE ? kAdvectTrueRk4MinBlocks
                                                         : kAdvectMinBlocks;
}

// Persistent advection. Every lane owns kPPT slots, each holding one particle
// at a time; a slot whose particle finishes takes the next one from its
// warp's claim of a.claim consecutive entries of the processing order, and
// the warp claims a new batch with one atomic when its batch runs out. Lanes
// therefore stay busy while particles of one warp end after very different
// numbers of steps. A particle takes at most a.max_steps steps per launch;
// one stopped by that budget alone is reported as in flight and resumes in a
// later launch.
//
// Between hand-outs the warp runs stretches: every slot steps until one of
// the warp's particles stops, with one vote per step and a 32-bit step
// counter per stretch (a stretch ends at 2^32 - 1 steps at the latest). The
// kPPT slots of a lane step in lock-step, so one particle's corner gather is
// in flight while the other's arithmetic issues. An empty slot holds a parked
// position, the centre of the first cell (never NaN, which would send the
// division of a step into its slow path for the whole warp). With one
// particle per lane the branch-free steady Euler and RK4 steppers step a
// parked slot and discard the result; otherwise an empty slot takes no steps.
template <int kIntegrator, int kStorage, int kLocate, bool kRecord, bool kUnsteady, int kPPT>
__global__ void __launch_bounds__(kAdvectBlock, advect_min_blocks<kIntegrator, kUnsteady, kPPT>())
advect_kernel(const FieldView f, const AdvectArgs a) {
  using Sampler = std::conditional_t<kUnsteady, TimeSampler<kStorage, kLocate>,
                                     CellSampler<kStorage, kLocate>>;
  constexpr unsigned kFull = 0xffffffffu;
  // State touched only when particles are handed out or finish lives in
  // shared memory, leaving the registers to the stepping loop: the warp's
  // claim [next, end) of the order and, per slot, the particle index, its
  // remaining iterations and the steps it may still take in this launch
  // (its remaining iterations or the launch's step budget).
  __shared__ uint64_t claims[kAdvectBlock / 32][2];
  __shared__ uint64_t particle[kPPT][kAdvectBlock];
  __shared__ uint64_t remaining[kPPT][kAdvectBlock];
  __shared__ uint64_t budget[kPPT][kAdvectBlock];
  const uint32_t claim = a.claim;
  const unsigned tid = threadIdx.x;
  const unsigned lane = tid & 31u;
  uint64_t* const warp_claim = claims[tid >> 5];
  if (lane == 0) warp_claim[0] = warp_claim[1] = 0;
  __syncwarp();
  bool exhausted = false;
  // Where an empty slot waits: the centre of the first cell, so that a step
  // run for it (branch-free steppers) divides normal numbers and loads its
  // corners once.
  const Position parked{__fmaf_rn(0.5f, f.spacing[0], f.offset[0]),
                        make_float2(__fmaf_rn(0.5f, f.spacing[2], f.offset[2]),
                                    __fmaf_rn(0.5f, f.spacing[1], f.offset[1]))};
  // (One particle per lane only: with two, skipping a pair's empty slot by a
  // branch measured 1.7x faster on the 512^3 batch than stepping it.)
  constexpr bool kStepAll = kPPT == 1 && !kUnsteady &&
                            (kIntegrator == DPA_INTEGRATOR_EULER ||
                             kIntegrator == DPA_INTEGRATOR_RUNGE_KUTTA_4);

  bool active[kPPT];
  Position p[kPPT];
  Sampler sampler[kPPT];
  StepHistory history[kPPT];
  float t[kPPT];          // particle time (a.times)
  float* curve[kPPT];     // the particle's last written vertex
  CurveCounter counter[kPPT];
#pragma unroll
  for (int j = 0; j < kPPT; ++j) {
    active[j] = false;
    p[j] = parked;
    history[j] = StepHistory{};
    t[j] = 0.0f;
    curve[j] = nullptr;
  }

  while (true) {
    // Hand new particles to idle slots.
#pragma unroll
    for (int j = 0; j < kPPT; ++j) {
      unsigned idle = __ballot_sync(kFull, !active[j]);
      while (idle && !exhausted) {
        uint64_t next = warp_claim[0], end = warp_claim[1];
        if (next == end) {
          unsigned long long base = 0;
          if (lane == 0) base = atomicAdd(a.work_counter, (unsigned long long)claim);
          base = __shfl_sync(kFull, base, 0);
          if (base >= a.count) {
            exhausted = true;
            break;
          }
          next = base;
          end = base + claim < a.count ? base + claim : a.count;
        }
        const uint32_t avail = uint32_t(end - next);
        const uint32_t take = uint32_t(__popc(idle)) < avail ? uint32_t(__popc(idle)) : avail;
        const uint32_t rank = __popc(idle & ((1u << lane) - 1u));
        // Lanes still in the idle set take entries next + rank. (A slot that
        // drew a finished particle earlier in this round is inactive but no
        // longer idle, and must not take one again.)
        const bool took = ((idle >> lane) & 1u) && rank < take;
        bool mine = took;
        uint64_t k = 0;
        if (mine) {
          const uint64_t e = next + rank;
          k = a.order ? a.order[e] : e;
          // Serving: a finished particle stays finished.
          if (a.resume_only && a.termination[k] != DPA_TERMINATION_IN_FLIGHT) mine = false;
        }
        if (mine) {
          particle[j][tid] = k;
          p[j].p0 = a.positions[3 * k];
          p[j].p21 = make_float2(a.positions[3 * k + 2], a.positions[3 * k + 1]);
          const uint64_t rem = a.remaining[k];
          remaining[j][tid] = rem;
          budget[j][tid] = rem < a.max_steps ? rem : a.max_steps;
          if (a.times) t[j] = a.times[k];
          sampler[j].reset();
          history[j].started = false;
          active[j] = true;
          if constexpr (kRecord) {
            // A particle resumed from an earlier launch continues its curve
            // where that launch left it.
            const uint64_t done = a.remaining_initial ? a.remaining_initial[k] - rem : 0;
            curve[j] = a.raw_vertices + 3 * (a.raw_offsets[k] + done);
            counter[j] = CurveCounter();
            if (done == 0) {
              curve[j][0] = p[j].p0;
              curve[j][1] = p[j].p21.y;
              curve[j][2] = p[j].p21.x;
              counter[j].append(p[j].p0, p[j].p21.y, p[j].p21.x);
            } else {
              counter[j].kept = a.kept_vertices[k];
              counter[j].segments = a.kept_segments[k];
              counter[j].prev_open = a.curve_open[k] != 0;
            }
          }
        }
        __syncwarp();
        if (lane == 0) {
          warp_claim[0] = next + take;
          warp_claim[1] = end;
        }
        __syncwarp();
        // Every lane that took an entry leaves this round of hand-outs; one
        // that drew a finished particle (serving) stays inactive until the next.
        idle &= ~__ballot_sync(kFull, took);
      }
    }
    bool any = false;
#pragma unroll
    for (int j = 0; j < kPPT; ++j) any = any || active[j];
    if (!__any_sync(kFull, any)) {
      if (exhausted) break;
      continue;  // every lane drew a finished particle (serving): claim again
    }

    // One stretch.
    uint32_t it[kPPT], limit[kPPT];
    int r[kPPT];
    bool stop[kPPT];
    bool halt = false;
#pragma unroll
    for (int j = 0; j < kPPT; ++j) {
      const uint64_t allowed = active[j] ? budget[j][tid] : 0;
      limit[j] = allowed < 0xffffffffull ? uint32_t(allowed) : 0xffffffffu;
      it[j] = 0;
      r[j] = kStepTaken;
      stop[j] = active[j] && limit[j] == 0;
      halt = halt || stop[j];
    }
    while (!__any_sync(kFull, halt)) {
      // Branch-free steppers run every slot, an empty one without moving it;
      // the others skip empty slots.
#pragma unroll
      for (int j = 0; j < kPPT; ++j) {
        if constexpr (kStepAll)
          r[j] = step<kIntegrator>(f, a.coefficients, sampler[j], p[j], t[j], history[j],
                                   active[j]);
        else
          r[j] = active[j]
                     ? step<kIntegrator>(f, a.coefficients, sampler[j], p[j], t[j], history[j])
                     : int(kStepOutOfBounds);
      }
      halt = false;
#pragma unroll
      for (int j = 0; j < kPPT; ++j) {
        const bool taken = r[j] == kStepTaken;  // never for an empty slot
        it[j] += taken ? 1u : 0u;
        if constexpr (kUnsteady) t[j] = taken ? __fadd_rn(t[j], a.coefficients.dt) : t[j];
        if constexpr (kRecord) {
          // The step's vertex, stored by predicated stores rather than a
          // branch (a launch of few particles waits on each step's chain).
          float* v = curve[j] + 3 * uint64_t(it[j]);
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %4, 0;\n\t"
              "@p st.global.f32 [%0], %1;\n\t@p st.global.f32 [%0+4], %2;\n\t"
              "@p st.global.f32 [%0+8], %3;\n\t}" ::"l"(v),
              "f"(p[j].p0), "f"(p[j].p21.y), "f"(p[j].p21.x), "r"(taken ? 1u : 0u));
          counter[j].append(p[j].p0, p[j].p21.y, p[j].p21.x, taken);
        }
        stop[j] = !taken || it[j] >= limit[j];
        halt = halt || (active[j] && stop[j]);
      }
    }

#pragma unroll
    for (int j = 0; j < kPPT; ++j) {
      if (!active[j]) continue;
      const uint64_t rem = remaining[j][tid] - it[j];
      const uint64_t left = budget[j][tid] - it[j];
      remaining[j][tid] = rem;
      budget[j][tid] = left;
      if constexpr (!kUnsteady) {
        // A steady field's particles carry their time only when asked to; it
        // advances by dt per step taken, rounded step by step as a
        // time-varying field's does.
        if (a.times)
          for (uint32_t i = 0; i < it[j]; ++i) t[j] = __fadd_rn(t[j], a.coefficients.dt);
      }
      if constexpr (kRecord) curve[j] += 3 * uint64_t(it[j]);
      // A particle that only reached the end of a stretch carries on.
      if (!stop[j] || (r[j] == kStepTaken && left > 0)) continue;

      const uint64_t k = particle[j][tid];
      const int reason = r[j] == kStepOutOfBounds    ? DPA_TERMINATION_OUT_OF_BOUNDS
                         : r[j] == kStepZeroVelocity ? DPA_TERMINATION_ZERO_VELOCITY
                         : rem == 0                  ? DPA_TERMINATION_COMPLETE
                                                     : DPA_TERMINATION_IN_FLIGHT;
      if constexpr (kRecord) {
        if (reason != DPA_TERMINATION_IN_FLIGHT) {
          float* v = curve[j] + 3;
          v[0] = kTerminal;
          v[1] = kTerminal;
          v[2] = kTerminal;
          counter[j].append(kTerminal, kTerminal, kTerminal);
        } else {
          a.curve_open[k] = counter[j].prev_open ? 1 : 0;
        }
        a.kept_vertices[k] = counter[j].kept;
        a.kept_segments[k] = counter[j].segments;
      }
      a.positions[3 * k] = p[j].p0;
      a.positions[3 * k + 1] = p[j].p21.y;
      a.positions[3 * k + 2] = p[j].p21.x;
      a.remaining[k] = rem;
      if (a.times) a.times[k] = t[j];
      if (a.termination) a.termination[k] = uint8_t(reason);
      if (a.in_flight && reason != DPA_TERMINATION_IN_FLIGHT)
        atomicSub(a.in_flight + a.request_of[k], 1u);
      active[j] = false;
      p[j] = parked;
    }
  }
}

// Resident blocks per SM of one instantiation at one block size, and the SM
// count, looked up once per process (every device of a process is a B200
// here) and published as one atomic value, so that threads making their
// first launches at once each see either nothing or both figures.
template <int kIntegrator, int kStorage, int kLocate, bool kRecord, bool kUnsteady, int kPPT>
cudaError_t resident_blocks(uint32_t block, int* blocks_per_sm, int* sms) {
  static std::atomic<uint64_t> cache[kAdvectBlock / 32 + 1] = {};
  std::atomic<uint64_t>& slot = cache[block / 32];
  uint64_t packed = slot.load(std::memory_order_acquire);
  if (packed == 0) {
    int device = 0, count = 0, r = 0;
    DPA_CUDA_TRY(cudaGetDevice(&device));
    DPA_CUDA_TRY(cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, device));
    DPA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &r, advect_kernel<kIntegrator, kStorage, kLocate, kRecord, kUnsteady, kPPT>, int(block),
        0));
    packed = (uint64_t(uint32_t(count)) << 32) | uint32_t(r < 1 ? 1 : r);
    slot.store(packed, std::memory_order_release);
  }
  *blocks_per_sm = int(uint32_t(packed));
  *sms = int(packed >> 32);
  return cudaSuccess;
}

// Threads per block of a launch: the tuning's choice, else kAdvectBlock, or
// fewer (a multiple of 32) when the particles would fill fewer blocks than
// the device has SMs, so that a small launch still spreads over every SM.
inline uint32_t advect_block(const AdvectArgs& a, uint64_t lanes, int sms) {
  if (a.block) return a.block;
  uint32_t block = uint32_t(kAdvectBlock);
#if DPA_ADVECT_SPREAD
  const uint64_t per_sm = (lanes + uint64_t(sms) - 1) / uint64_t(sms);
  if (per_sm < uint64_t(kAdvectBlock)) block = uint32_t(std::max<uint64_t>(32, (per_sm + 31) / 32 * 32));
#else
  (void)lanes;
  (void)sms;
#endif
  return block;
}

template <int kIntegrator, int kStorage, int kLocate, bool kRecord, bool kUnsteady, int kPPT>
cudaError_t launch_typed(const FieldView& f, const AdvectArgs& a, cudaStream_t stream) {
  // Persistent grid: as many blocks as fit on the device at once (or as the
  // tuning asks), fewer when there are fewer particles than lanes.
  const uint64_t lanes = (a.count + kPPT - 1) / kPPT;
  int sms = 0, resident = 0;
  DPA_CUDA_TRY((resident_blocks<kIntegrator, kStorage, kLocate, kRecord, kUnsteady, kPPT>(
      kAdvectBlock, &resident, &sms)));
  const uint32_t block = advect_block(a, lanes, sms);
  if (block == 0 || block % 32 != 0 || block > uint32_t(kAdvectBlock)) return cudaErrorInvalidValue;
  DPA_CUDA_TRY((resident_blocks<kIntegrator, kStorage, kLocate, kRecord, kUnsteady, kPPT>(
      block, &resident, &sms)));
  if (a.count == 0) return cudaSuccess;  // nothing to do, or preparation only
  if (a.blocks_per_sm && int(a.blocks_per_sm) < resident) resident = int(a.blocks_per_sm);
  const uint64_t needed = (lanes + block - 1) / block;
  const uint64_t blocks = std::min<uint64_t>(needed, uint64_t(resident) * uint64_t(sms));
  if (blocks == 0) return cudaSuccess;
  DPA_CUDA_TRY(cudaMemsetAsync(a.work_counter, 0, sizeof(unsigned long long), stream));
  advect_kernel<kIntegrator, kStorage, kLocate, kRecord, kUnsteady, kPPT>
      <<<dim3(unsigned(blocks)), dim3(block), 0, stream>>>(f, a);
  return cudaGetLastError();
}

// Two particles per lane for steady fields without recording; everything
// else runs one.
template <int kIntegrator, int kStorage, int kLocate, bool kRecord, bool kUnsteady>
cudaError_t launch_ppt(const FieldView& f, const AdvectArgs& a, cudaStream_t s) {
  if constexpr (!kRecord && !kUnsteady && kIntegrator != DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE) {
    if (a.particles_per_thread == 2)
      return launch_typed<kIntegrator, kStorage, kLocate, kRecord, kUnsteady, 2>(f, a, s);
  }
  return launch_typed<kIntegrator, kStorage, kLocate, kRecord, kUnsteady, 1>(f, a, s);
}

template <int kIntegrator, int kStorage, bool kUnsteady>
cudaError_t launch_locate(const FieldView& f, const AdvectArgs& a, bool record, cudaStream_t s) {
  switch (f.locate) {
    case kLocatePow2:
      return record ? launch_ppt<kIntegrator, kStorage, kLocatePow2, true, kUnsteady>(f, a, s)
                    : launch_ppt<kIntegrator, kStorage, kLocatePow2, false, kUnsteady>(f, a, s);
    case kLocateReciprocal:
      return record ? launch_ppt<kIntegrator, kStorage, kLocateReciprocal, true, kUnsteady>(f, a, s)
                    : launch_ppt<kIntegrator, kStorage, kLocateReciprocal, false, kUnsteady>(f, a, s);
    default:
      return record ? launch_ppt<kIntegrator, kStorage, kLocateDivide, true, kUnsteady>(f, a, s)
                    : launch_ppt<kIntegrator, kStorage, kLocateDivide, false, kUnsteady>(f, a, s);
  }
}

}  // namespace

// Every integrator for one storage and kind of field (steady or time-varying).
template <int kStorage, bool kUnsteady>
cudaError_t launch_advect_storage(const FieldView& f, const AdvectArgs& a, int integrator,
                                  bool record, cudaStream_t stream) {
  switch (integrator) {
    case DPA_INTEGRATOR_EULER:
      return launch_locate<DPA_INTEGRATOR_EULER, kStorage, kUnsteady>(f, a, record, stream);
    case DPA_INTEGRATOR_RUNGE_KUTTA_4:
      return launch_locate<DPA_INTEGRATOR_RUNGE_KUTTA_4, kStorage, kUnsteady>(f, a, record, stream);
    case DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE:
      return launch_locate<DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE, kStorage, kUnsteady>(f, a, record,
                                                                                  stream);
    case DPA_INTEGRATOR_MODIFIED_MIDPOINT:
    case DPA_INTEGRATOR_RUNGE_KUTTA_CASH_KARP_54:
    case DPA_INTEGRATOR_RUNGE_KUTTA_DORMAND_PRINCE_5:
    case DPA_INTEGRATOR_RUNGE_KUTTA_FEHLBERG_78:
    case DPA_INTEGRATOR_ADAMS_BASHFORTH_2:
    case DPA_INTEGRATOR_ADAMS_BASHFORTH_MOULTON_2:
      // The coefficients in a.coefficients.g select the stepper.
      return launch_locate<kGeneralIntegrator, kStorage, kUnsteady>(f, a, record, stream);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace dpa
