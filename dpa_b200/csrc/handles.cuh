// handles.cuh -- definitions of the opaque handles of include/dpa_b200.h
// (dpa_context, dpa_field) and the device/pinned buffers they own.
#pragma once

#include <string>

#include "kernels.cuh"

namespace dpa {

// Grow-only device buffer; freed by release() or when it goes out of scope
// (with its device current).
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() { release(); }
  cudaError_t reserve(size_t n) {
    if (n <= bytes && ptr) return cudaSuccess;
    release();
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
      ptr = nullptr;
      return e;
    }
    bytes = n;
    return cudaSuccess;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  template <class T>
  T* as() const { return static_cast<T*>(ptr); }
};

struct PinnedBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  PinnedBuffer() = default;
  PinnedBuffer(const PinnedBuffer&) = delete;
  PinnedBuffer& operator=(const PinnedBuffer&) = delete;
  ~PinnedBuffer() { release(); }
  cudaError_t reserve(size_t n) {
    if (n <= bytes && ptr) return cudaSuccess;
    release();
    if (n == 0) n = 16;
    cudaError_t e = cudaMallocHost(&ptr, n);
    if (e != cudaSuccess) {
      ptr = nullptr;
      return e;
    }
    bytes = n;
    return cudaSuccess;
  }
  void release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  template <class T>
  T* as() const { return static_cast<T*>(ptr); }
};

}  // namespace dpa

using dpa::DeviceBuffer;
using dpa::PinnedBuffer;

// Launch parameters an autotuner may change per context.
struct dpa_tuning_state {
  uint32_t claim = 16;        // order entries a warp claims at once
  uint32_t blocks_per_sm = 0; // persistent grid: 0 = as many as fit
  uint32_t order = 64;        // processing order: Morton buckets of an order^3
                              // coarsening of the grid (1..64); 0: input order
  uint32_t block = 0;         // threads per block (multiple of 32, <= 256); 0: 256, or
                              // fewer so that a small launch reaches every SM
  uint32_t particles_per_thread = 1;  // 1 or 2 (steady fields without recording)
};

namespace dpa {
// The launch parameters of a tuning.
inline void apply_tuning(const dpa_tuning_state& t, AdvectArgs& a) {
  a.claim = t.claim;
  a.blocks_per_sm = t.blocks_per_sm;
  a.block = t.block;
  a.particles_per_thread = t.particles_per_thread;
}
}  // namespace dpa

// Scratch of one processing-order + advection launch sequence: bucket ids,
// the order, the counting sort's counters and the claim counter. A context
// keeps one for its calls; a CUDA graph keeps its own, because a later call
// with more particles reallocates the context's.
struct dpa_launch_scratch {
  DeviceBuffer keys, values, sort_temp, work_counter;
  void release() {
    keys.release();
    values.release();
    sort_temp.release();
    work_counter.release();
  }
};

struct dpa_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string error;
  uint64_t staging_limit = 1ull << 30;
  uint64_t host_chunk_bytes = 256ull << 20;  // per pinned half (vertices + colors; indices)
  cudaEvent_t chunk_events[2] = {nullptr, nullptr};
  bool ieee_division = false;  // fields created now divide by __fdiv_rn only

  DeviceBuffer positions, remaining, remaining_in, termination;
  dpa_launch_scratch scratch;
  uint64_t launches = 0;  // kernels this context launched (advection path)
  bool profiling = false;
  // order begin, advect begin, advect end, emission begin, emission end
  cudaEvent_t events[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  bool timed_order = false;
  // A profiled recording round: its pieces' times, summed as they finish.
  bool timed_round = false;
  float round_order_ms = 0.0f, round_advect_ms = 0.0f, round_emit_ms = 0.0f;
  dpa_tuning_state tuning;
  DeviceBuffer raw, raw_offsets, raw_counts, kept_vertices, kept_segments;
  DeviceBuffer wide, vertex_offsets, segment_offsets, scan_temp, totals;
  DeviceBuffer out_vertices, out_colors, out_indices;
  PinnedBuffer host_vertices, host_colors, host_indices, host_totals, host_offsets;
  DeviceBuffer ftle_winners, ftle_flow, ftle_out, ftle_original, ftle_final;

  void release_all() {
    scratch.release();
    DeviceBuffer* d[] = {&positions, &remaining, &remaining_in, &termination, &raw, &raw_offsets,
                         &raw_counts,
                         &kept_vertices, &kept_segments, &wide, &vertex_offsets,
                         &segment_offsets, &scan_temp, &totals, &out_vertices, &out_colors,
                         &out_indices, &ftle_winners, &ftle_flow, &ftle_out, &ftle_original,
                         &ftle_final};
    for (DeviceBuffer* b : d) b->release();
    PinnedBuffer* h[] = {&host_vertices, &host_colors, &host_indices, &host_totals,
                         &host_offsets};
    for (PinnedBuffer* b : h) b->release();
  }
};

struct dpa_field {
  dpa_context* owner = nullptr;
  DeviceBuffer nodes;
  dpa::FieldView view{};
  uint64_t shape[3] = {0, 0, 0};
  float offset[3] = {0, 0, 0};
  float spacing[3] = {0, 0, 0};
  int32_t storage = DPA_STORAGE_F32;
  uint32_t slices = 1;  // > 1: a time-varying field
  float time_origin = 0.0f;
  float time_spacing = 0.0f;
};

