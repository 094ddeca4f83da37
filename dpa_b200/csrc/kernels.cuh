// kernels.cuh -- kernel argument blocks and launchers shared by the .cu files.
#pragma once

#include "common.cuh"

namespace dpa {

#ifndef DPA_ADVECT_BLOCK
#define DPA_ADVECT_BLOCK 256
#endif
constexpr int kAdvectBlock = DPA_ADVECT_BLOCK;
#ifndef DPA_ADVECT_MIN_BLOCKS
#define DPA_ADVECT_MIN_BLOCKS 4
#endif
constexpr int kAdvectMinBlocks = DPA_ADVECT_MIN_BLOCKS;
// Time-varying fields: the corner cache holds two slices, so fewer, larger
// threads (up to 128 registers) per SM.
#ifndef DPA_ADVECT_UNSTEADY_MIN_BLOCKS
#define DPA_ADVECT_UNSTEADY_MIN_BLOCKS 2
#endif
constexpr int kAdvectUnsteadyMinBlocks = DPA_ADVECT_UNSTEADY_MIN_BLOCKS;
// Four-sample RK4 keeps three more stage derivatives alive: up to 80
// registers (3 blocks per SM) instead of spilling at 64.
#ifndef DPA_ADVECT_TRUE_RK4_MIN_BLOCKS
#define DPA_ADVECT_TRUE_RK4_MIN_BLOCKS 3
#endif
constexpr int kAdvectTrueRk4MinBlocks = DPA_ADVECT_TRUE_RK4_MIN_BLOCKS;
// Two particles per lane, stepped in lock-step so that one particle's gather
// overlaps the other's arithmetic: twice the particle state per thread.
#ifndef DPA_ADVECT_PPT2_MIN_BLOCKS
#define DPA_ADVECT_PPT2_MIN_BLOCKS 2
#endif
constexpr int kAdvectPpt2MinBlocks = DPA_ADVECT_PPT2_MIN_BLOCKS;
// Launches whose particles would fill fewer blocks than the device has SMs
// use smaller blocks (1) or keep kAdvectBlock threads per block (0).
#ifndef DPA_ADVECT_SPREAD
#define DPA_ADVECT_SPREAD 1
#endif

struct AdvectArgs {
  uint64_t count;
  const uint32_t* order;  // processing order (Morton); null = identity
  float* positions;       // [count][3], updated in place
  uint64_t* remaining;    // [count], updated in place
  uint8_t* termination;   // [count] or null
  float* times;           // [count] particle times, updated in place; required by
                          // time-varying fields, optional (null) for steady ones
  StepCoefficients coefficients;
  uint64_t max_steps;                // step budget of this launch (~0: none)
  uint32_t claim;                    // order entries a warp claims at once
  uint32_t blocks_per_sm;            // persistent grid per SM (0: occupancy maximum)
  uint32_t block;                    // threads per block: a multiple of 32 up to
                                     // kAdvectBlock; 0 = kAdvectBlock, or fewer when
                                     // the particles would not reach every SM
  uint32_t particles_per_thread;     // 1 or 2 (2: steady fields without recording)
  unsigned long long* work_counter;  // zeroed by the launcher; claims of the order
  // Recording only.
  float* raw_vertices;          // unpruned curve of particle k at raw_offsets[k]
  const uint64_t* raw_offsets;  // exclusive scan of remaining + 2
  uint32_t* kept_vertices;      // per particle: vertices surviving the prune
  uint32_t* kept_segments;      // per particle: index pairs it contributes
  // Resumed recording (null for a curve recorded in one launch).
  const uint64_t* remaining_initial;  // remaining iterations when the curve began
  uint8_t* curve_open;                // last kept vertex is not terminal-valued
  // Serving: skip order entries whose termination is not in flight, and count
  // each particle's finish down in its request's counter (null when unused).
  bool resume_only;
  const uint32_t* request_of;         // per particle
  unsigned int* in_flight;            // per request
};

// Launch defaults: no step budget, 16-entry claims.
inline void set_launch_defaults(AdvectArgs& a) {
  a.times = nullptr;
  a.max_steps = ~0ull;
  a.claim = 16;
  a.blocks_per_sm = 0;
  a.block = 0;
  a.particles_per_thread = 1;
  a.resume_only = false;
  a.request_of = nullptr;
  a.in_flight = nullptr;
}

// list[t] = starts[r] + order[starts[r] + (t - firsts[r])] for the range r
// holding t, where firsts is the exclusive scan of the range lengths (ranges
// of arena slots) and order holds, per slot, a permutation of each range's
// offsets (its processing order).
cudaError_t launch_expand_ranges(const uint64_t* starts, const uint64_t* firsts, uint32_t ranges,
                                 uint64_t total, const uint32_t* order, uint32_t* list,
                                 cudaStream_t stream);

// Picks the kernel instantiation for the field (steady or time-varying,
// storage, locate mode), the integrator, recording and particles per lane.
cudaError_t launch_advect(const FieldView& f, const AdvectArgs& a, int integrator, bool record,
                          cudaStream_t stream);
// The instantiations of one storage for steady or time-varying fields
// (advect_f32.cu, advect_f32e.cu, advect_f16.cu, advect_bf16.cu).
template <int kStorage, bool kUnsteady>
cudaError_t launch_advect_storage(const FieldView& f, const AdvectArgs& a, int integrator,
                                  bool record, cudaStream_t stream);

// Resolves, outside any stream capture, what launch_advect looks up on its
// first use of a kernel instantiation (its occupancy at the given launch
// parameters).
cudaError_t prepare_advect(const FieldView& f, const AdvectArgs& a, int integrator, bool record);

// Processing order: a counting sort of the particles by the Morton code of
// their start cell on a resolution^3 coarsening of the grid (a memset and
// five kernels). Within a bucket the order is arbitrary; results never depend
// on processing order. ids holds count bucket ids; counts holds
// kOrderCountsSize counters (the buckets of the finest resolution, one for
// particles outside the grid, and the scan's tile sums).
constexpr uint32_t kOrderMaxResolution = 64;
constexpr uint32_t kOrderDefaultResolution = 64;
constexpr uint32_t kOrderBuckets = kOrderMaxResolution * kOrderMaxResolution * kOrderMaxResolution;
constexpr uint32_t kOrderCountsSize = kOrderBuckets + 1 + (kOrderBuckets + 1 + 1023) / 1024;
constexpr int kOrderLaunches = 5;
// Calls with fewer particles run in input order: their warps share few cells,
// and the sort's six launches cost more than the locality gains (4096 seeds of
// the recording configuration: 0.90 ms per round unsorted, 0.94 sorted).
constexpr uint64_t kOrderMinParticles = 8192;

cudaError_t launch_order(const FieldView& f, const float* positions, uint64_t count,
                         uint32_t* ids, uint32_t* counts, uint32_t* order, cudaStream_t stream,
                         uint32_t resolution = kOrderDefaultResolution);

// Particle-steps each seed set took: sum over [offsets[s], offsets[s+1]) of
// remaining_in - remaining_out.
cudaError_t launch_set_steps(const uint64_t* remaining_in, const uint64_t* remaining_out,
                             const uint64_t* offsets, uint64_t sets, unsigned long long* steps,
                             cudaStream_t stream);

struct EmitArgs {
  uint64_t count;                 // particles in this piece, in round order
  const float* raw_vertices;
  const uint64_t* raw_offsets;    // per particle
  const uint64_t* steps_raw;      // per particle: raw vertex count (steps + 2)
  const uint64_t* vertex_offsets; // exclusive scan of kept vertices (piece-local)
  const uint64_t* segment_offsets;// exclusive scan of kept segments (piece-local)
  const uint32_t* kept_vertices;
  uint64_t vertex_base;           // round-level index of the piece's first vertex
  float* vertices;                // piece output
  float* colors;                  // piece output or null
  void* indices;                  // piece output (uint32 or uint64)
};

cudaError_t launch_emit(const EmitArgs& e, bool index64, bool colors, cudaStream_t stream);

// Raw vertex count per particle: remaining_in - remaining_out + 2.
cudaError_t launch_raw_counts(const uint64_t* remaining_in, const uint64_t* remaining_out,
                              uint64_t count, uint64_t* raw_counts, cudaStream_t stream);

// Exclusive scans of the per-particle kept-vertex and kept-segment counts
// into vertex_offsets and segment_offsets (three kernels); totals (device,
// two entries) receives the sums of both. scratch holds
// curve_offsets_scratch_bytes(count) bytes.
uint64_t curve_offsets_scratch_bytes(uint64_t count);
cudaError_t launch_curve_offsets(const uint32_t* kept_vertices, const uint32_t* kept_segments,
                                 uint64_t count, void* scratch, uint64_t* vertex_offsets,
                                 uint64_t* segment_offsets, unsigned long long* totals,
                                 cudaStream_t stream);
constexpr int kCurveOffsetsLaunches = 3;

// The data-path probe of dpa_measure_gather_bandwidth: blocks x 256 lanes,
// each loading 8 16-byte nodes per iteration from table (mask + 1 nodes).
cudaError_t launch_gather_probe(const float4* table, uint32_t mask, uint32_t side,
                                uint32_t iterations, int random, float* sink, uint32_t blocks,
                                cudaStream_t stream);

// Counts into *mismatches (zeroed first) the 32-bit dividends for which
// divide_by_reciprocal(a, h, y, yl) differs from IEEE division by h.
cudaError_t launch_verify_division(float h, float y, float yl, unsigned int* mismatches,
                                   cudaStream_t stream);

// Field repack: XYZV float [n][3] (rows of n2 nodes along axis 2) -> the
// device layout of the given storage; field_node_bytes is its size per node.
uint64_t field_node_bytes(int storage);
cudaError_t launch_repack(const float* xyzv, uint64_t nodes, uint32_t n2, int storage, void* out,
                          cudaStream_t stream);

struct FtleArgs {
  uint64_t count;
  const float* original_positions;
  const float* final_positions;
  int mapping;
  uint64_t shape[3];       // flow-map lattice
  float offset[3];
  float spacing[3];        // field spacing * stride
  float two_spacing[3];
  double horizon;          // |step_size * iterations| as the reference rounds it
  unsigned long long* winners;  // [cells], scratch
  float* flow;             // [cells][3], scratch
  float* ftle;             // [cells]
};

cudaError_t launch_ftle(const FtleArgs& a, cudaStream_t stream);

// Uniform seeds offset + size * u, u from splitmix64(key ^ (3 i + axis)) >> 40
// scaled by 2^-24; key = splitmix64(seed).
cudaError_t launch_random_seeds(const float offset[3], const float size[3], uint64_t count,
                                uint64_t key, float* out, cudaStream_t stream);

cudaError_t launch_lattice_seeds(const float offset[3], const float stride[3],
                                 const uint64_t shape[3], float* out, cudaStream_t stream);

}  // namespace dpa
