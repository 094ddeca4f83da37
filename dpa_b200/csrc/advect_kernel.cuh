// advect_kernel.cuh -- the advection kernel template and its launchers:
// one thread per particle, every step of that particle in registers
// (particle_advector.cpp:325-396). advect.cu instantiates it for steady
// fields, advect_unsteady.cu for time-varying ones.
#pragma once

#include <algorithm>
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
//
// Between hand-outs the warp runs stretches: every active lane steps until
// one of the warp's particles stops, with one vote per step and a 32-bit step
// counter per stretch (a stretch ends at 2^32 - 1 steps at the latest).
template <int kIntegrator, int kStorage, bool kPow2, bool kRecord, bool kUnsteady>
__global__ void __launch_bounds__(kAdvectBlock,
                                  kUnsteady ? kAdvectUnsteadyMinBlocks
                                  : kIntegrator == DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE
                                      ? kAdvectTrueRk4MinBlocks
                                      : kAdvectMinBlocks)
advect_kernel(const FieldView f, const AdvectArgs a) {
  using Sampler = std::conditional_t<kUnsteady, TimeSampler<kStorage, kPow2>,
                                     CellSampler<kStorage, kPow2>>;
  constexpr unsigned kFull = 0xffffffffu;
  // State touched only when particles are handed out or finish lives in
  // shared memory, leaving the registers to the stepping loop: the warp's
  // claim [next, end) of the order, and each lane's particle index.
  __shared__ uint64_t claims[kAdvectBlock / 32][2];
  __shared__ uint64_t particle[kAdvectBlock];
  const uint32_t claim = a.claim;
  const unsigned lane = threadIdx.x & 31u;
  uint64_t* const warp_claim = claims[threadIdx.x >> 5];
  if (lane == 0) warp_claim[0] = warp_claim[1] = 0;
  __syncwarp();
  bool exhausted = false;

  bool active = false;
  // rem: the particle's remaining iterations; left: steps it may still take
  // in this launch (its remaining iterations or the launch's step budget).
  uint64_t rem = 0, left = 0;
  Position p{0.0f, make_float2(0.0f, 0.0f)};
  float* curve = nullptr;  // the particle's last written vertex
  CurveCounter counter;
  Sampler sampler;
  StepHistory history{};
  float t = 0.0f;  // particle time (a.times)

  while (true) {
    // Hand new particles to idle lanes.
    unsigned idle = __ballot_sync(kFull, !active);
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
      // Lanes still in the idle set take entries next + rank. (A lane that
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
        particle[threadIdx.x] = k;
        p.p0 = a.positions[3 * k];
        p.p21 = make_float2(a.positions[3 * k + 2], a.positions[3 * k + 1]);
        rem = a.remaining[k];
        if (a.times) t = a.times[k];
        left = rem < a.max_steps ? rem : a.max_steps;
        sampler.reset();
        history.started = false;
        active = true;
        if constexpr (kRecord) {
          // A particle resumed from an earlier launch continues its curve
          // where that launch left it.
          const uint64_t done = a.remaining_initial ? a.remaining_initial[k] - rem : 0;
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
      __syncwarp();
      if (lane == 0) {
        warp_claim[0] = next + take;
        warp_claim[1] = end;
      }
      __syncwarp();
      // Every lane that took an entry leaves this round of hand-outs; one that
      // drew a finished particle (serving) stays inactive until the next.
      idle &= ~__ballot_sync(kFull, took);
    }
    if (!__any_sync(kFull, active)) {
      if (exhausted) break;
      continue;  // every lane drew a finished particle (serving): claim again
    }

    // One stretch. Inactive lanes (the order ran out) only vote.
    const uint64_t allowed = active ? left : 0;
    const uint32_t limit = allowed < 0xffffffffull ? uint32_t(allowed) : 0xffffffffu;
    uint32_t it = 0;
    int r = kStepTaken;
    bool stop = active && limit == 0;
    while (!__any_sync(kFull, stop)) {
      if (active) {
        r = step<kIntegrator>(f, a.coefficients, sampler, p, t, history);
        if (r == kStepTaken) {
          ++it;
          if constexpr (kUnsteady) t = __fadd_rn(t, a.coefficients.dt);
          if constexpr (kRecord) {
            float* v = curve + 3 * uint64_t(it);
            v[0] = p.p0;
            v[1] = p.p21.y;
            v[2] = p.p21.x;
            counter.append(p.p0, p.p21.y, p.p21.x);
          }
          stop = it >= limit;
        } else {
          stop = true;
        }
      }
    }
    if (!active) continue;
    rem -= it;
    left -= it;
    if constexpr (!kUnsteady) {
      // A steady field's particles carry their time only when asked to; it
      // advances by dt per step taken, rounded step by step as a
      // time-varying field's does.
      if (a.times)
        for (uint32_t i = 0; i < it; ++i) t = __fadd_rn(t, a.coefficients.dt);
    }
    if constexpr (kRecord) curve += 3 * uint64_t(it);
    // A particle that only reached the end of a stretch carries on.
    if (!stop || (r == kStepTaken && left > 0)) continue;

    const uint64_t k = particle[threadIdx.x];
    const int reason = r == kStepOutOfBounds    ? DPA_TERMINATION_OUT_OF_BOUNDS
                       : r == kStepZeroVelocity ? DPA_TERMINATION_ZERO_VELOCITY
                       : rem == 0               ? DPA_TERMINATION_COMPLETE
                                                : DPA_TERMINATION_IN_FLIGHT;
    if constexpr (kRecord) {
      if (reason != DPA_TERMINATION_IN_FLIGHT) {
        float* v = curve + 3;
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
    a.remaining[k] = rem;
    if (a.times) a.times[k] = t;
    if (a.termination) a.termination[k] = uint8_t(reason);
    if (a.in_flight && reason != DPA_TERMINATION_IN_FLIGHT)
      atomicSub(a.in_flight + a.request_of[k], 1u);
    active = false;
  }
}

template <int kIntegrator, int kStorage, bool kPow2, bool kRecord, bool kUnsteady>
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
        &r, advect_kernel<kIntegrator, kStorage, kPow2, kRecord, kUnsteady>, kAdvectBlock, 0));
    resident = r < 1 ? 1 : r;
  }
  *blocks_per_sm = resident;
  *sms = count;
  return cudaSuccess;
}

template <int kIntegrator, int kStorage, bool kPow2, bool kRecord, bool kUnsteady>
cudaError_t launch_typed(const FieldView& f, const AdvectArgs& a, cudaStream_t stream) {
  // Persistent grid: as many blocks as fit on the device at once (or as the
  // tuning asks), fewer when there are fewer particles than lanes.
  int resident = 0, sms = 0;
  DPA_CUDA_TRY((resident_blocks<kIntegrator, kStorage, kPow2, kRecord, kUnsteady>(&resident, &sms)));
  if (a.count == 0) return cudaSuccess;  // nothing to do, or preparation only
  if (a.blocks_per_sm && int(a.blocks_per_sm) < resident) resident = int(a.blocks_per_sm);
  const uint64_t needed = (a.count + kAdvectBlock - 1) / kAdvectBlock;
  const uint64_t blocks = std::min<uint64_t>(needed, uint64_t(resident) * uint64_t(sms));
  if (blocks == 0) return cudaSuccess;
  DPA_CUDA_TRY(cudaMemsetAsync(a.work_counter, 0, sizeof(unsigned long long), stream));
  advect_kernel<kIntegrator, kStorage, kPow2, kRecord, kUnsteady>
      <<<dim3(unsigned(blocks)), dim3(kAdvectBlock), 0, stream>>>(f, a);
  return cudaGetLastError();
}

template <int kIntegrator, int kStorage, bool kUnsteady>
cudaError_t launch_pow2(const FieldView& f, const AdvectArgs& a, bool record, cudaStream_t s) {
  if (f.pow2) {
    return record ? launch_typed<kIntegrator, kStorage, true, true, kUnsteady>(f, a, s)
                  : launch_typed<kIntegrator, kStorage, true, false, kUnsteady>(f, a, s);
  }
  return record ? launch_typed<kIntegrator, kStorage, false, true, kUnsteady>(f, a, s)
                : launch_typed<kIntegrator, kStorage, false, false, kUnsteady>(f, a, s);
}

template <int kIntegrator, bool kUnsteady>
cudaError_t launch_storage(const FieldView& f, const AdvectArgs& a, bool record, cudaStream_t s) {
  switch (f.storage) {
    case DPA_STORAGE_F32:
      return launch_pow2<kIntegrator, DPA_STORAGE_F32, kUnsteady>(f, a, record, s);
    case DPA_STORAGE_F16:
      return launch_pow2<kIntegrator, DPA_STORAGE_F16, kUnsteady>(f, a, record, s);
    case DPA_STORAGE_BF16:
      return launch_pow2<kIntegrator, DPA_STORAGE_BF16, kUnsteady>(f, a, record, s);
    default: return cudaErrorInvalidValue;
  }
}

// Every integrator for one kind of field (steady or time-varying).
template <bool kUnsteady>
cudaError_t launch_family(const FieldView& f, const AdvectArgs& a, int integrator, bool record,
                          cudaStream_t stream) {
  switch (integrator) {
    case DPA_INTEGRATOR_EULER:
      return launch_storage<DPA_INTEGRATOR_EULER, kUnsteady>(f, a, record, stream);
    case DPA_INTEGRATOR_RUNGE_KUTTA_4:
      return launch_storage<DPA_INTEGRATOR_RUNGE_KUTTA_4, kUnsteady>(f, a, record, stream);
    case DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE:
      return launch_storage<DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE, kUnsteady>(f, a, record, stream);
    case DPA_INTEGRATOR_MODIFIED_MIDPOINT:
    case DPA_INTEGRATOR_RUNGE_KUTTA_CASH_KARP_54:
    case DPA_INTEGRATOR_RUNGE_KUTTA_DORMAND_PRINCE_5:
    case DPA_INTEGRATOR_RUNGE_KUTTA_FEHLBERG_78:
    case DPA_INTEGRATOR_ADAMS_BASHFORTH_2:
    case DPA_INTEGRATOR_ADAMS_BASHFORTH_MOULTON_2:
      // The coefficients in a.coefficients.g select the stepper.
      return launch_storage<kGeneralIntegrator, kUnsteady>(f, a, record, stream);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace
}  // namespace dpa
