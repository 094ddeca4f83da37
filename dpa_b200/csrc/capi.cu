// capi.cu -- the C ABI of include/dpa_b200.h: contexts, fields, rounds, FTLE.
//
// Host orchestration only; the kernels live in advect.cu, emit.cu and ftle.cu.
// Every entry point returns a dpa_status, records a message on failure and
// never lets a C++ exception cross the boundary.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "checks.cuh"
#include "handles.cuh"
#include "kernels.cuh"

struct dpa_graph {
  dpa_context* owner = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t launches = 0;        // kernels per replay
  dpa_launch_scratch scratch;   // the captured launches' own scratch
};

namespace {

using dpa::check_options;
using dpa::check_steady;
using dpa::fail;
using dpa::fail_cuda;

#define DPA_TRY_CUDA(ctx, expr)                                  \
  do {                                                           \
    cudaError_t dpa_e_ = (expr);                                 \
    if (dpa_e_ != cudaSuccess) return fail_cuda(ctx, dpa_e_, #expr); \
  } while (0)

template <class F>
int guarded(dpa_context* ctx, F&& body) {
  try {
    return body();
  } catch (const std::bad_alloc&) {
    return fail(ctx, DPA_ERROR_OUT_OF_MEMORY, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(ctx, DPA_ERROR_INTERNAL, e.what());
  } catch (...) {
    return fail(ctx, DPA_ERROR_INTERNAL, "unknown exception");
  }
}

bool is_power_of_two(float h) {
  if (!(h > 0.0f) || !std::isfinite(h)) return false;
  int e = 0;
  return std::frexp(h, &e) == 0.5f && std::ldexp(1.0f, e - 1) == h &&
         std::isnormal(1.0f / h);
}

// Axes on which the kernels may locate with q = fma(p, 1 / h, -offset / h):
// h a power of two in [2^-20, 2^20] and offset zero or at least 2^-100 in
// magnitude. Then offset / h is an exact float and the fma's one rounding of
// (p - offset) / h equals the reference's rounded p - offset scaled exactly by
// 1 / h: whenever the scaled quotient could fall below the normal range,
// p - offset is itself exact (p is then within a factor of two of offset, or
// offset is zero).
bool exact_scaled_axis(float h, float offset) {
  if (!is_power_of_two(h) || h < std::ldexp(1.0f, -20) || h > std::ldexp(1.0f, 20)) return false;
  if (offset != 0.0f && !(std::fabs(offset) >= std::ldexp(1.0f, -100))) return false;
  const float scaled = offset * (1.0f / h);
  return std::isfinite(scaled) && double(scaled) * double(h) == double(offset);
}

cudaStream_t pick_stream(dpa_context* ctx, void* stream) {
  return stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
}

// Builds the processing order of `count` device positions (coarse Morton
// buckets, see launch_order) in scratch.values. Returns it through *order.
int build_order(dpa_context* ctx, dpa_launch_scratch& scratch, const dpa_field* field,
                const float* positions, uint64_t count, cudaStream_t stream,
                const uint32_t** order) {
  *order = nullptr;
  if (count < dpa::kOrderMinParticles) return DPA_OK;
  DPA_TRY_CUDA(ctx, scratch.keys.reserve(count * 4));
  DPA_TRY_CUDA(ctx, scratch.values.reserve(count * 4));
  DPA_TRY_CUDA(ctx, scratch.sort_temp.reserve(dpa::kOrderCountsSize * 4));
  DPA_TRY_CUDA(ctx, dpa::launch_order(field->view, positions, count, scratch.keys.as<uint32_t>(),
                                      scratch.sort_temp.as<uint32_t>(),
                                      scratch.values.as<uint32_t>(), stream, ctx->tuning.order));
  ctx->launches += dpa::kOrderLaunches;
  *order = scratch.values.as<uint32_t>();
  return DPA_OK;
}

// Order (optional) + advection kernel over device arrays, no recording.
// times (may be null for a steady field) are the particles' times.
// The processing order and the advection launch for device arrays, with the
// context's scratch or, for a graph's capture, the graph's own.
int advect_device_impl(dpa_context* ctx, const dpa_field* field, const dpa_advect_options* o,
                       uint64_t count, float* positions, uint64_t* remaining, uint8_t* termination,
                       cudaStream_t s, float* times = nullptr,
                       dpa_launch_scratch* own_scratch = nullptr) {
  if (!times) {
    const int st = check_steady(ctx, field);
    if (st != DPA_OK) return st;
  }
  if (count == 0) return DPA_OK;
  dpa_launch_scratch& scratch = own_scratch ? *own_scratch : ctx->scratch;
  if (ctx->profiling) DPA_TRY_CUDA(ctx, cudaEventRecord(ctx->events[0], s));
  const uint32_t* order = nullptr;
  if (o->morton_order && ctx->tuning.order) {
    const int st = build_order(ctx, scratch, field, positions, count, s, &order);
    if (st != DPA_OK) return st;
  }
  if (ctx->profiling) DPA_TRY_CUDA(ctx, cudaEventRecord(ctx->events[1], s));
  DPA_TRY_CUDA(ctx, scratch.work_counter.reserve(sizeof(unsigned long long)));
  dpa::AdvectArgs a{};
  dpa::set_launch_defaults(a);
  if (o->max_steps) a.max_steps = o->max_steps;
  dpa::apply_tuning(ctx->tuning, a);
  a.work_counter = scratch.work_counter.as<unsigned long long>();
  a.count = count;
  a.order = order;
  a.positions = positions;
  a.remaining = remaining;
  a.termination = termination;
  a.times = times;
  a.coefficients = dpa::make_step_coefficients(o->integrator, o->step_size);
  DPA_TRY_CUDA(ctx, dpa::launch_advect(field->view, a, o->integrator, false, s));
  ctx->launches += 1;
  if (ctx->profiling) {
    DPA_TRY_CUDA(ctx, cudaEventRecord(ctx->events[2], s));
    ctx->timed_order = true;
    ctx->timed_round = false;
  }
  return DPA_OK;
}

// Advects and emits particles [begin, end) of a recording round. The device
// arrays ctx->positions / remaining hold the whole round.
int record_piece(dpa_context* ctx, const dpa_field* field, const dpa_advect_options* o,
                 const dpa::StepCoefficients& k, uint64_t begin, uint64_t end,
                 const uint64_t* host_remaining, uint64_t* round_vertices,
                 uint64_t* round_indices, bool final_piece, dpa_curve_sink sink, void* user) {
  cudaStream_t s = ctx->stream;
  const uint64_t n = end - begin;
  // Raw (unpruned) vertex offsets: remaining + 2 slots per particle.
  DPA_TRY_CUDA(ctx, ctx->host_offsets.reserve(n * 8));
  uint64_t* offsets = ctx->host_offsets.as<uint64_t>();
  uint64_t raw_total = 0;
  for (uint64_t i = 0; i < n; ++i) {
    offsets[i] = raw_total;
    raw_total += host_remaining[begin + i] + 2;
  }
  DPA_TRY_CUDA(ctx, ctx->raw.reserve(raw_total * 12));
  DPA_TRY_CUDA(ctx, ctx->raw_offsets.reserve(n * 8));
  DPA_TRY_CUDA(ctx, ctx->raw_counts.reserve(n * 8));
  DPA_TRY_CUDA(ctx, ctx->kept_vertices.reserve(n * 4));
  DPA_TRY_CUDA(ctx, ctx->kept_segments.reserve(n * 4));
  DPA_TRY_CUDA(ctx, ctx->vertex_offsets.reserve(n * 8));
  DPA_TRY_CUDA(ctx, ctx->segment_offsets.reserve(n * 8));
  DPA_TRY_CUDA(ctx, ctx->totals.reserve(32));
  DPA_TRY_CUDA(ctx, ctx->host_totals.reserve(32));
  // The pinned offsets of the previous piece are free: its copies finished
  // before the previous piece returned.
  DPA_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->raw_offsets.ptr, offsets, n * 8, cudaMemcpyHostToDevice,
                                    s));

  float* positions = ctx->positions.as<float>() + 3 * begin;
  uint64_t* remaining = ctx->remaining.as<uint64_t>() + begin;
  uint8_t* termination = ctx->termination.as<uint8_t>() + begin;
  if (ctx->profiling) DPA_TRY_CUDA(ctx, cudaEventRecord(ctx->events[0], s));
  const uint32_t* order = nullptr;
  if (o->morton_order && ctx->tuning.order) {
    const int st = build_order(ctx, ctx->scratch, field, positions, n, s, &order);
    if (st != DPA_OK) return st;
  }
  if (ctx->profiling) DPA_TRY_CUDA(ctx, cudaEventRecord(ctx->events[1], s));
  DPA_TRY_CUDA(ctx, ctx->scratch.work_counter.reserve(sizeof(unsigned long long)));
  dpa::AdvectArgs a{};
  dpa::set_launch_defaults(a);
  dpa::apply_tuning(ctx->tuning, a);
  a.work_counter = ctx->scratch.work_counter.as<unsigned long long>();
  a.count = n;
  a.order = order;
  a.positions = positions;
  a.remaining = remaining;
  a.termination = termination;
  a.coefficients = k;
  a.raw_vertices = ctx->raw.as<float>();
  a.raw_offsets = ctx->raw_offsets.as<uint64_t>();
  a.kept_vertices = ctx->kept_vertices.as<uint32_t>();
  a.kept_segments = ctx->kept_segments.as<uint32_t>();
  DPA_TRY_CUDA(ctx, dpa::launch_advect(field->view, a, o->integrator, true, s));
  ctx->launches += 1;
  if (ctx->profiling) {
    DPA_TRY_CUDA(ctx, cudaEventRecord(ctx->events[2], s));
    DPA_TRY_CUDA(ctx, cudaEventRecord(ctx->events[3], s));
  }

  // Per-particle raw counts, then piece-local offsets of kept vertices and
  // kept segments and their totals.
  DPA_TRY_CUDA(ctx, dpa::launch_raw_counts(ctx->remaining_in.as<uint64_t>() + begin, remaining, n,
                                           ctx->raw_counts.as<uint64_t>(), s));
  DPA_TRY_CUDA(ctx, ctx->scan_temp.reserve(dpa::curve_offsets_scratch_bytes(n)));
  DPA_TRY_CUDA(ctx, dpa::launch_curve_offsets(
                        ctx->kept_vertices.as<uint32_t>(), ctx->kept_segments.as<uint32_t>(), n,
                        ctx->scan_temp.ptr, ctx->vertex_offsets.as<uint64_t>(),
                        ctx->segment_offsets.as<uint64_t>(),
                        ctx->totals.as<unsigned long long>(), s));
  ctx->launches += 1 + dpa::kCurveOffsetsLaunches;
  uint64_t* ht = ctx->host_totals.as<uint64_t>();
  DPA_TRY_CUDA(ctx, cudaMemcpyAsync(ht, ctx->totals.ptr, 16, cudaMemcpyDeviceToHost, s));
  DPA_TRY_CUDA(ctx, cudaStreamSynchronize(s));
  const uint64_t piece_vertices = ht[0];
  const uint64_t piece_segments = ht[1];
  const uint64_t piece_indices = 2 * piece_segments;
  if (!o->index64 && *round_vertices + piece_vertices > 0xffffffffull)
    return fail(ctx, DPA_ERROR_UNSUPPORTED,
                "the round's curve has more vertices than 32-bit indices can address; "
                "set index64");

  const size_t index_bytes = o->index64 ? 8 : 4;
  DPA_TRY_CUDA(ctx, ctx->out_vertices.reserve(piece_vertices * 12));
  DPA_TRY_CUDA(ctx, ctx->out_colors.reserve(piece_vertices * 4));
  DPA_TRY_CUDA(ctx, ctx->out_indices.reserve(piece_indices * index_bytes));

  dpa::EmitArgs e{};
  e.count = n;
  e.raw_vertices = ctx->raw.as<float>();
  e.raw_offsets = ctx->raw_offsets.as<uint64_t>();
  e.steps_raw = ctx->raw_counts.as<uint64_t>();
  e.vertex_offsets = ctx->vertex_offsets.as<uint64_t>();
  e.segment_offsets = ctx->segment_offsets.as<uint64_t>();
  e.kept_vertices = ctx->kept_vertices.as<uint32_t>();
  e.vertex_base = *round_vertices;
  e.vertices = ctx->out_vertices.as<float>();
  e.colors = o->colors ? ctx->out_colors.as<float>() : nullptr;
  e.indices = ctx->out_indices.ptr;
  DPA_TRY_CUDA(ctx, dpa::launch_emit(e, o->index64 != 0, o->colors != 0, s));
  ctx->launches += 1;
  if (ctx->profiling) DPA_TRY_CUDA(ctx, cudaEventRecord(ctx->events[4], s));

  // The piece's curve crosses to the host in chunks through two pinned
  // halves, so that chunk j + 1 copies while the sink takes chunk j and the
  // pinned memory stays bounded (dpa_context_set_host_chunk_limit).
  if (sink) {
    const uint64_t cap_v = std::max<uint64_t>(ctx->host_chunk_bytes / 16, 1);
    const uint64_t cap_i = std::max<uint64_t>(ctx->host_chunk_bytes / index_bytes, 2) & ~1ull;
    const uint64_t chunks = std::max<uint64_t>(
        {1, (piece_vertices + cap_v - 1) / cap_v, (piece_indices + cap_i - 1) / cap_i});
    const uint64_t half_v = std::min(piece_vertices, cap_v);
    const uint64_t half_i = std::min(piece_indices, cap_i);
    DPA_TRY_CUDA(ctx, ctx->host_vertices.reserve(2 * half_v * 12));
    DPA_TRY_CUDA(ctx, ctx->host_colors.reserve(2 * half_v * 4));
    DPA_TRY_CUDA(ctx, ctx->host_indices.reserve(2 * half_i * index_bytes));
    for (cudaEvent_t& ev : ctx->chunk_events)
      if (!ev) DPA_TRY_CUDA(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    auto span = [](uint64_t j, uint64_t cap, uint64_t total, uint64_t* first, uint64_t* count) {
      *first = std::min(j * cap, total);
      *count = std::min(cap, total - *first);
    };
    auto issue = [&](uint64_t j) -> int {
      const uint64_t h = j & 1;
      uint64_t v0, vn, i0, in;
      span(j, cap_v, piece_vertices, &v0, &vn);
      span(j, cap_i, piece_indices, &i0, &in);
      if (vn) {
        DPA_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->host_vertices.as<float>() + 3 * h * half_v,
                                          ctx->out_vertices.as<float>() + 3 * v0, vn * 12,
                                          cudaMemcpyDeviceToHost, s));
        if (o->colors)
          DPA_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->host_colors.as<float>() + h * half_v,
                                            ctx->out_colors.as<float>() + v0, vn * 4,
                                            cudaMemcpyDeviceToHost, s));
      }
      if (in)
        DPA_TRY_CUDA(ctx, cudaMemcpyAsync(
                              ctx->host_indices.as<char>() + h * half_i * index_bytes,
                              ctx->out_indices.as<char>() + i0 * index_bytes, in * index_bytes,
                              cudaMemcpyDeviceToHost, s));
      DPA_TRY_CUDA(ctx, cudaEventRecord(ctx->chunk_events[h], s));
      return DPA_OK;
    };
    int st = issue(0);
    if (st != DPA_OK) return st;
    for (uint64_t j = 0; j < chunks; ++j) {
      if (j + 1 < chunks) {
        st = issue(j + 1);  // into the half whose chunk the sink has returned
        if (st != DPA_OK) return st;
      }
      const uint64_t h = j & 1;
      DPA_TRY_CUDA(ctx, cudaEventSynchronize(ctx->chunk_events[h]));
      uint64_t v0, vn, i0, in;
      span(j, cap_v, piece_vertices, &v0, &vn);
      span(j, cap_i, piece_indices, &i0, &in);
      dpa_curve_chunk c{};
      c.vertex_offset = *round_vertices + v0;
      c.vertex_count = vn;
      c.vertices = ctx->host_vertices.as<float>() + 3 * h * half_v;
      c.colors = o->colors ? ctx->host_colors.as<float>() + h * half_v : nullptr;
      c.index_offset = *round_indices + i0;
      c.index_count = in;
      c.indices = ctx->host_indices.as<char>() + h * half_i * index_bytes;
      c.last = (final_piece && j + 1 == chunks) ? 1 : 0;
      if (sink(user, &c) != 0) {
        cudaStreamSynchronize(s);  // no copy may still target the halves
        return fail(ctx, DPA_ERROR_SINK, "curve sink aborted the round");
      }
    }
  }
  DPA_TRY_CUDA(ctx, cudaStreamSynchronize(s));
  if (ctx->profiling) {
    float order_ms = 0.0f, advect_ms = 0.0f, emit_ms = 0.0f;
    DPA_TRY_CUDA(ctx, cudaEventElapsedTime(&order_ms, ctx->events[0], ctx->events[1]));
    DPA_TRY_CUDA(ctx, cudaEventElapsedTime(&advect_ms, ctx->events[1], ctx->events[2]));
    DPA_TRY_CUDA(ctx, cudaEventElapsedTime(&emit_ms, ctx->events[3], ctx->events[4]));
    ctx->round_order_ms += order_ms;
    ctx->round_advect_ms += advect_ms;
    ctx->round_emit_ms += emit_ms;
  }
  *round_vertices += piece_vertices;
  *round_indices += piece_indices;
  return DPA_OK;
}

}  // namespace

extern "C" {

const char* dpa_version(void) { return "dpa_b200 0.1.0 (sm_100a)"; }

int dpa_device_count(int* count) {
  if (!count) return DPA_ERROR_INVALID_ARGUMENT;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  *count = n;
  return DPA_OK;
}

int dpa_context_create(int device, dpa_context** out) {
  if (!out) return DPA_ERROR_INVALID_ARGUMENT;
  *out = nullptr;
  return guarded(nullptr, [&]() -> int {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
      cudaGetLastError();
      return DPA_ERROR_CUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess) return DPA_ERROR_CUDA;
    dpa_context* ctx = new dpa_context();
    ctx->device = device;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete ctx;
      return DPA_ERROR_CUDA;
    }
    *out = ctx;
    return DPA_OK;
  });
}

int dpa_context_destroy(dpa_context* ctx) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->release_all();
  for (cudaEvent_t e : ctx->events)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : ctx->chunk_events)
    if (e) cudaEventDestroy(e);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return DPA_OK;
}

const char* dpa_last_error(const dpa_context* ctx) {
  if (!ctx) return "no context";
  return ctx->error.c_str();
}

void* dpa_context_stream(dpa_context* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int dpa_context_synchronize(dpa_context* ctx) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  DPA_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return DPA_OK;
}

int dpa_context_set_staging_limit(dpa_context* ctx, uint64_t bytes) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  if (bytes < 4096) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "staging limit below 4 KiB");
  ctx->staging_limit = bytes;
  return DPA_OK;
}

int dpa_context_set_host_chunk_limit(dpa_context* ctx, uint64_t bytes) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  if (bytes < 4096) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "host chunk limit below 4 KiB");
  ctx->host_chunk_bytes = bytes;
  return DPA_OK;
}

int dpa_context_set_profiling(dpa_context* ctx, int32_t enabled) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  if (enabled && !ctx->events[0])
    for (cudaEvent_t& e : ctx->events) DPA_TRY_CUDA(ctx, cudaEventCreate(&e));
  ctx->profiling = enabled != 0;
  ctx->timed_order = false;
  ctx->timed_round = false;
  return DPA_OK;
}

int dpa_context_last_timing(dpa_context* ctx, float* order_ms, float* advect_ms) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  if (ctx->profiling && ctx->timed_round) {
    if (order_ms) *order_ms = ctx->round_order_ms;
    if (advect_ms) *advect_ms = ctx->round_advect_ms;
    return DPA_OK;
  }
  if (!ctx->profiling || !ctx->timed_order)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "no profiled advection since profiling was enabled");
  DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  DPA_TRY_CUDA(ctx, cudaEventSynchronize(ctx->events[2]));
  float a = 0.0f, b = 0.0f;
  DPA_TRY_CUDA(ctx, cudaEventElapsedTime(&a, ctx->events[0], ctx->events[1]));
  DPA_TRY_CUDA(ctx, cudaEventElapsedTime(&b, ctx->events[1], ctx->events[2]));
  if (order_ms) *order_ms = a;
  if (advect_ms) *advect_ms = b;
  return DPA_OK;
}

int dpa_context_last_emit_timing(dpa_context* ctx, float* emit_ms) {
  if (!ctx || !emit_ms) return DPA_ERROR_INVALID_ARGUMENT;
  if (!ctx->profiling || !ctx->timed_round)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT,
                "no profiled recording round since profiling was enabled");
  *emit_ms = ctx->round_emit_ms;
  return DPA_OK;
}

int dpa_measure_gather_bandwidth(dpa_context* ctx, uint64_t table_bytes, int32_t pattern,
                                 double* gigabytes_per_second) {
  if (!ctx || !gigabytes_per_second) return DPA_ERROR_INVALID_ARGUMENT;
  if (pattern != 0 && pattern != 1)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "pattern must be 0 (coalesced) or 1 (random)");
  // A cube of 2^(3 side) 16-byte nodes, the largest that fits table_bytes.
  uint32_t side = 1;
  while (side < 10 && (16ull << (3 * (side + 1))) <= table_bytes) ++side;
  const uint64_t nodes = 1ull << (3 * side);
  if ((16ull << 3) > table_bytes)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "table_bytes below 128");
  return guarded(ctx, [&]() -> int {
    DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    DeviceBuffer table, sink;
    DPA_TRY_CUDA(ctx, table.reserve(nodes * 16));
    DPA_TRY_CUDA(ctx, sink.reserve(16));
    DPA_TRY_CUDA(ctx, cudaMemsetAsync(table.ptr, 0, nodes * 16, s));
    int sms = 0;
    DPA_TRY_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    const uint32_t blocks = uint32_t(sms) * 8, iterations = 512;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    DPA_TRY_CUDA(ctx, cudaEventCreate(&e0));
    const cudaError_t made = cudaEventCreate(&e1);
    if (made != cudaSuccess) {
      cudaEventDestroy(e0);
      return fail_cuda(ctx, made, "cudaEventCreate");
    }
    float best = 0.0f;
    cudaError_t e = cudaSuccess;
    for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
      e = cudaEventRecord(e0, s);
      if (e == cudaSuccess)
        e = dpa::launch_gather_probe(table.as<float4>(), uint32_t(nodes - 1), side, iterations,
                                     pattern, sink.as<float>(), blocks, s);
      if (e == cudaSuccess) e = cudaEventRecord(e1, s);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.0f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e == cudaSuccess && rep > 0 && (best == 0.0f || ms < best)) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return fail_cuda(ctx, e, "gather probe");
    const double bytes = double(blocks) * 256.0 * iterations * 8.0 * 16.0;
    *gigabytes_per_second = bytes / (double(best) * 1e-3) / 1e9;
    return DPA_OK;
  });
}

int dpa_context_launch_count(const dpa_context* ctx, uint64_t* launches) {
  if (!ctx || !launches) return DPA_ERROR_INVALID_ARGUMENT;
  *launches = ctx->launches;
  return DPA_OK;
}

int dpa_integrator_from_name(const char* name, int32_t* integrator) {
  if (!name || !integrator) return DPA_ERROR_INVALID_ARGUMENT;
  static const struct {
    const char* name;
    int32_t code;
  } table[] = {
      {"euler", DPA_INTEGRATOR_EULER},
      {"modified_midpoint", DPA_INTEGRATOR_MODIFIED_MIDPOINT},
      {"runge_kutta_4", DPA_INTEGRATOR_RUNGE_KUTTA_4},
      {"runge_kutta_cash_karp_54", DPA_INTEGRATOR_RUNGE_KUTTA_CASH_KARP_54},
      {"runge_kutta_dormand_prince_5", DPA_INTEGRATOR_RUNGE_KUTTA_DORMAND_PRINCE_5},
      {"runge_kutta_fehlberg_78", DPA_INTEGRATOR_RUNGE_KUTTA_FEHLBERG_78},
      {"adams_bashforth_2", DPA_INTEGRATOR_ADAMS_BASHFORTH_2},
      {"adams_bashforth_moulton_2", DPA_INTEGRATOR_ADAMS_BASHFORTH_MOULTON_2},
      {"runge_kutta_4_true", DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE},
  };
  for (const auto& e : table) {
    if (std::strcmp(e.name, name) == 0) {
      *integrator = e.code;
      return DPA_OK;
    }
  }
  return DPA_ERROR_INVALID_ARGUMENT;
}

// The reciprocal of h split into two floats: hi = RN(1 / h), lo =
// RN(1 / h - hi), with 1 / h taken in the host's extended precision.
static void split_reciprocal(float h, float* hi, float* lo) {
  const long double inv = 1.0L / static_cast<long double>(h);
  *hi = static_cast<float>(inv);
  *lo = static_cast<float>(inv - static_cast<long double>(*hi));
}

// Whether dividing by h through its split reciprocal (divide_by_reciprocal)
// gives IEEE division's bits for every float dividend: checked once per
// divisor and process on the device, over all 2^32 bit patterns (a few
// milliseconds), and remembered.
static int reciprocal_divides_exactly(dpa_context* ctx, float h, bool* exact) {
  static std::mutex lock;
  static std::map<uint32_t, bool> known;
  uint32_t bits = 0;
  std::memcpy(&bits, &h, sizeof bits);
  {
    std::lock_guard<std::mutex> guard(lock);
    const auto it = known.find(bits);
    if (it != known.end()) {
      *exact = it->second;
      return DPA_OK;
    }
  }
  DeviceBuffer counter;
  DPA_TRY_CUDA(ctx, counter.reserve(sizeof(unsigned int)));
  float hi = 0.0f, lo = 0.0f;
  split_reciprocal(h, &hi, &lo);
  DPA_TRY_CUDA(ctx, dpa::launch_verify_division(h, hi, lo, counter.as<unsigned int>(),
                                                ctx->stream));
  unsigned int mismatches = 0;
  DPA_TRY_CUDA(ctx, cudaMemcpyAsync(&mismatches, counter.ptr, sizeof mismatches,
                                    cudaMemcpyDeviceToHost, ctx->stream));
  DPA_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *exact = mismatches == 0;
  std::lock_guard<std::mutex> guard(lock);
  known[bits] = *exact;
  return DPA_OK;
}

static int create_field(dpa_context* ctx, const float* xyzv, bool device_input,
                        const uint64_t shape[3], const float offset[3], const float spacing[3],
                        int32_t storage, dpa_field** out, uint32_t slices = 1,
                        float time_origin = 0.0f, float time_spacing = 0.0f) {
  if (!ctx || !out || !shape || !offset || !spacing)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  if (storage != DPA_STORAGE_F32 && storage != DPA_STORAGE_F16 && storage != DPA_STORAGE_BF16 &&
      storage != DPA_STORAGE_F32_EDGES)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "unknown storage");
  for (int i = 0; i < 3; ++i) {
    if (shape[i] == 0 || shape[i] > (1u << 23))
      return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "field shape must be in [1, 2^23] per axis");
    if (!(spacing[i] > 0.0f) || !std::isfinite(spacing[i]) || !std::isfinite(offset[i]))
      return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "spacing must be positive and finite");
  }
  if (slices == 0) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "no time slices");
  if (slices > 1 && (!(time_spacing > 0.0f) || !std::isfinite(time_spacing) ||
                     !std::isfinite(time_origin)))
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "time spacing must be positive and finite");
  const uint64_t slice_nodes = shape[0] * shape[1] * shape[2];
  if (slice_nodes >= (1ull << 32) || slice_nodes * slices > (1ull << 36))
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT,
                "field too large: at most 2^32 - 1 nodes per slice and 2^36 in all");
  const uint64_t nodes = slice_nodes * slices;
  if (nodes && !xyzv) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "field data is NULL");
  return guarded(ctx, [&]() -> int {
    DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    dpa_field* f = new dpa_field();
    f->owner = ctx;
    f->storage = storage;
    const size_t node_bytes = dpa::field_node_bytes(storage);
    cudaError_t e = f->nodes.reserve(nodes * node_bytes);
    const float* src = xyzv;
    DeviceBuffer staging;
    if (e == cudaSuccess && !device_input) {
      e = staging.reserve(nodes * 12);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(staging.ptr, xyzv, nodes * 12, cudaMemcpyHostToDevice, ctx->stream);
      src = staging.as<float>();
    }
    if (e == cudaSuccess)
      e = dpa::launch_repack(src, nodes, uint32_t(shape[2]), storage, f->nodes.ptr, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    staging.release();
    if (e != cudaSuccess) {
      f->nodes.release();
      delete f;
      return fail_cuda(ctx, e, "field upload");
    }
    bool pow2 = true;
    for (int i = 0; i < 3; ++i) {
      f->shape[i] = shape[i];
      f->offset[i] = offset[i];
      f->spacing[i] = spacing[i];
      pow2 = pow2 && exact_scaled_axis(spacing[i], offset[i]);
    }
    dpa::FieldView& v = f->view;
    v.nodes = f->nodes.ptr;
    for (int i = 0; i < 3; ++i) {
      v.n[i] = int32_t(shape[i]);
      v.offset[i] = offset[i];
      v.spacing[i] = spacing[i];
      float hi = 0.0f, lo = 0.0f;
      split_reciprocal(spacing[i], &hi, &lo);
      v.reciprocal[i] = hi;
      v.reciprocal_lo[i] = lo;
      v.scaled_offset[i] = offset[i] * v.reciprocal[i];
      v.upper[i] = float(int64_t(shape[i]) - 1);
      v.cells[i] = uint32_t(shape[i] - 1);
    }
    v.stride0 = uint32_t(shape[1] * shape[2]);
    v.stride1 = uint32_t(shape[2]);
    v.node_bias = 0x4B000000u * (v.stride0 + v.stride1 + 1u);
    v.storage = storage;
    v.locate = dpa::kLocatePow2;
    if (!pow2 && ctx->ieee_division) {
      v.locate = dpa::kLocateDivide;
    } else if (!pow2) {
      bool exact = true;
      for (int i = 0; i < 3 && exact; ++i) {
        const int st = reciprocal_divides_exactly(ctx, spacing[i], &exact);
        if (st != DPA_OK) {
          f->nodes.release();
          delete f;
          return st;
        }
      }
      v.locate = exact ? dpa::kLocateReciprocal : dpa::kLocateDivide;
    }
    f->slices = slices;
    f->time_origin = time_origin;
    f->time_spacing = time_spacing;
    v.slices = int32_t(slices);
    v.slice_stride = int64_t(slice_nodes);
    v.time_origin = time_origin;
    v.time_spacing = slices > 1 ? time_spacing : 1.0f;
    split_reciprocal(v.time_spacing, &v.time_reciprocal, &v.time_reciprocal_lo);
    v.time_fast = 0;
    if (slices > 1 && !ctx->ieee_division) {
      bool exact = false;
      const int st = reciprocal_divides_exactly(ctx, v.time_spacing, &exact);
      if (st != DPA_OK) {
        f->nodes.release();
        delete f;
        return st;
      }
      v.time_fast = exact ? 1 : 0;
    }
    v.time_upper = float(int64_t(slices) - 1);
    *out = f;
    return DPA_OK;
  });
}

int dpa_field_create(dpa_context* ctx, const float* xyzv, const uint64_t shape[3],
                     const float offset[3], const float spacing[3], int32_t storage,
                     dpa_field** out) {
  return create_field(ctx, xyzv, false, shape, offset, spacing, storage, out);
}

int dpa_field_create_device(dpa_context* ctx, const float* device_xyzv, const uint64_t shape[3],
                            const float offset[3], const float spacing[3], int32_t storage,
                            dpa_field** out) {
  return create_field(ctx, device_xyzv, true, shape, offset, spacing, storage, out);
}

int dpa_field_create_unsteady(dpa_context* ctx, const float* xyzv, const uint64_t shape[3],
                              uint32_t slices, const float offset[3], const float spacing[3],
                              float time_origin, float time_spacing, int32_t storage,
                              dpa_field** out) {
  if (ctx && slices < 2)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "a time-varying field needs 2 or more slices");
  return create_field(ctx, xyzv, false, shape, offset, spacing, storage, out, slices, time_origin,
                      time_spacing);
}

int dpa_context_set_ieee_division(dpa_context* ctx, int32_t enabled) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  ctx->ieee_division = enabled != 0;
  return DPA_OK;
}

int dpa_field_locate_mode(const dpa_field* field, int32_t* mode) {
  if (!field || !mode) return DPA_ERROR_INVALID_ARGUMENT;
  *mode = field->view.locate;
  return DPA_OK;
}

int dpa_field_time_info(const dpa_field* field, uint32_t* slices, float* time_origin,
                        float* time_spacing) {
  if (!field) return DPA_ERROR_INVALID_ARGUMENT;
  if (slices) *slices = field->slices;
  if (time_origin) *time_origin = field->time_origin;
  if (time_spacing) *time_spacing = field->time_spacing;
  return DPA_OK;
}

int dpa_field_destroy(dpa_context* ctx, dpa_field* field) {
  if (!ctx || !field) return DPA_ERROR_INVALID_ARGUMENT;
  if (field->owner != ctx) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "field belongs to another context");
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  field->nodes.release();
  delete field;
  return DPA_OK;
}

int dpa_field_info(const dpa_field* field, uint64_t shape[3], float offset[3], float spacing[3],
                   int32_t* storage, uint64_t* device_bytes) {
  if (!field) return DPA_ERROR_INVALID_ARGUMENT;
  for (int i = 0; i < 3; ++i) {
    if (shape) shape[i] = field->shape[i];
    if (offset) offset[i] = field->offset[i];
    if (spacing) spacing[i] = field->spacing[i];
  }
  if (storage) *storage = field->storage;
  if (device_bytes) *device_bytes = field->nodes.bytes;
  return DPA_OK;
}

int dpa_advect_round(dpa_context* ctx, const dpa_field* field, const dpa_advect_options* options,
                     uint64_t count, float* positions, uint64_t* remaining,
                     uint8_t* termination, dpa_curve_sink sink, void* sink_user) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  int st = check_options(ctx, options);
  if (st != DPA_OK) return st;
  if (!field || field->owner != ctx) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "bad field");
  st = check_steady(ctx, field);
  if (st != DPA_OK) return st;
  if (count && (!positions || !remaining))
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "positions or remaining is NULL");
  if (count > 0xffffffffull)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "at most 2^32-1 particles per round");
  return guarded(ctx, [&]() -> int {
    DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const dpa::StepCoefficients k = dpa::make_step_coefficients(options->integrator, options->step_size);
    if (options->record) {
      for (uint64_t i = 0; i < count; ++i)
        if (remaining[i] > 0xfffffff0ull)
          return fail(ctx, DPA_ERROR_INVALID_ARGUMENT,
                      "recording supports at most 2^32-16 iterations per particle");
    }
    if (count == 0) {
      if (options->record && sink) {
        dpa_curve_chunk c{};
        c.last = 1;
        if (sink(sink_user, &c) != 0) return fail(ctx, DPA_ERROR_SINK, "curve sink aborted the round");
      }
      return DPA_OK;
    }
    DPA_TRY_CUDA(ctx, ctx->positions.reserve(count * 12));
    DPA_TRY_CUDA(ctx, ctx->remaining.reserve(count * 8));
    DPA_TRY_CUDA(ctx, ctx->termination.reserve(count));
    DPA_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->positions.ptr, positions, count * 12,
                                      cudaMemcpyHostToDevice, s));
    DPA_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->remaining.ptr, remaining, count * 8,
                                      cudaMemcpyHostToDevice, s));
    if (!options->record) {
      st = advect_device_impl(ctx, field, options, count, ctx->positions.as<float>(),
                              ctx->remaining.as<uint64_t>(), ctx->termination.as<uint8_t>(), s);
      if (st != DPA_OK) return st;
    } else {
      DPA_TRY_CUDA(ctx, ctx->remaining_in.reserve(count * 8));
      DPA_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->remaining_in.ptr, ctx->remaining.ptr, count * 8,
                                        cudaMemcpyDeviceToDevice, s));
      ctx->round_order_ms = ctx->round_advect_ms = ctx->round_emit_ms = 0.0f;
      // Pieces of the round whose unpruned curves fit the staging limit.
      const uint64_t limit_vertices = std::max<uint64_t>(ctx->staging_limit / 12, 1);
      uint64_t round_vertices = 0, round_indices = 0;
      uint64_t begin = 0;
      while (begin < count) {
        uint64_t end = begin, raw = 0;
        while (end < count && (end == begin || raw + remaining[end] + 2 <= limit_vertices)) {
          raw += remaining[end] + 2;
          ++end;
        }
        st = record_piece(ctx, field, options, k, begin, end, remaining, &round_vertices,
                          &round_indices, end == count, sink, sink_user);
        if (st != DPA_OK) return st;
        begin = end;
      }
      if (ctx->profiling) {
        ctx->timed_round = true;
        ctx->timed_order = false;
      }
    }
    DPA_TRY_CUDA(ctx, cudaMemcpyAsync(positions, ctx->positions.ptr, count * 12,
                                      cudaMemcpyDeviceToHost, s));
    DPA_TRY_CUDA(ctx, cudaMemcpyAsync(remaining, ctx->remaining.ptr, count * 8,
                                      cudaMemcpyDeviceToHost, s));
    if (termination)
      DPA_TRY_CUDA(ctx, cudaMemcpyAsync(termination, ctx->termination.ptr, count,
                                        cudaMemcpyDeviceToHost, s));
    DPA_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    return DPA_OK;
  });
}

int dpa_advect_device(dpa_context* ctx, const dpa_field* field, const dpa_advect_options* options,
                      uint64_t count, float* device_positions, uint64_t* device_remaining,
                      uint8_t* device_termination, void* stream) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  int st = check_options(ctx, options);
  if (st != DPA_OK) return st;
  if (options->record)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT,
                "dpa_advect_device does not record; use dpa_advect_round");
  if (!field || field->owner != ctx) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "bad field");
  if (count && (!device_positions || !device_remaining))
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "positions or remaining is NULL");
  if (count > 0xffffffffull)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "at most 2^32-1 particles per call");
  return guarded(ctx, [&]() -> int {
    DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    return advect_device_impl(ctx, field, options, count, device_positions, device_remaining,
                              device_termination, pick_stream(ctx, stream));
  });
}

int dpa_advect_pathlines_device(dpa_context* ctx, const dpa_field* field,
                                const dpa_advect_options* options, uint64_t count,
                                float* device_positions, float* device_times,
                                uint64_t* device_remaining, uint8_t* device_termination,
                                void* stream) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  int st = check_options(ctx, options);
  if (st != DPA_OK) return st;
  if (options->record)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "dpa_advect_pathlines_device does not record");
  if (!field || field->owner != ctx) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "bad field");
  if (count && (!device_positions || !device_remaining || !device_times))
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "positions, times or remaining is NULL");
  if (count > 0xffffffffull)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "at most 2^32-1 particles per call");
  return guarded(ctx, [&]() -> int {
    DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    return advect_device_impl(ctx, field, options, count, device_positions, device_remaining,
                              device_termination, pick_stream(ctx, stream), device_times);
  });
}

int dpa_seed_lattice_device(dpa_context* ctx, const float offset_in[3], const float size_in[3],
                            const float stride[3], const float* aabb, uint64_t* count,
                            uint64_t shape_out[3], float* device_positions, void* stream) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  if (!offset_in || !size_in || !stride || !count)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "NULL argument");
  float offset[3] = {offset_in[0], offset_in[1], offset_in[2]};
  float size[3] = {size_in[0], size_in[1], size_in[2]};
  uint64_t shape[3] = {0, 0, 0};
  bool empty = false;
  if (aabb) {
    // Eigen AlignedBox intersection and isEmpty (uniform_seed_generator.cpp:18-27).
    float lo[3], hi[3];
    for (int i = 0; i < 3; ++i) {
      lo[i] = std::max(aabb[i], offset[i]);
      hi[i] = std::min(aabb[3 + i], offset[i] + size[i]);
      if (lo[i] > hi[i]) empty = true;
    }
    if (!empty)
      for (int i = 0; i < 3; ++i) {
        offset[i] = lo[i];
        size[i] = hi[i] - lo[i];
      }
  }
  if (!empty)
    for (int i = 0; i < 3; ++i) {
      if (!(stride[i] > 0.0f)) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "stride must be positive");
      const float q = size[i] / stride[i];
      shape[i] = q > 0.0f ? uint64_t(q) : 0;
    }
  *count = shape[0] * shape[1] * shape[2];
  if (shape_out)
    for (int i = 0; i < 3; ++i) shape_out[i] = shape[i];
  if (!device_positions || *count == 0) return DPA_OK;
  return guarded(ctx, [&]() -> int {
    DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    DPA_TRY_CUDA(ctx, dpa::launch_lattice_seeds(offset, stride, shape, device_positions,
                                                pick_stream(ctx, stream)));
    return DPA_OK;
  });
}

int dpa_seed_random_device(dpa_context* ctx, const float offset_in[3], const float size_in[3],
                           uint64_t count, uint64_t seed, const float* aabb, uint64_t* count_out,
                           float* device_positions, void* stream) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  if (!offset_in || !size_in) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "NULL argument");
  float offset[3] = {offset_in[0], offset_in[1], offset_in[2]};
  float size[3] = {size_in[0], size_in[1], size_in[2]};
  if (aabb) {
    float lo[3], hi[3];
    for (int i = 0; i < 3; ++i) {
      lo[i] = std::max(aabb[i], offset[i]);
      hi[i] = std::min(aabb[3 + i], offset[i] + size[i]);
      if (lo[i] > hi[i]) count = 0;
    }
    if (count)
      for (int i = 0; i < 3; ++i) {
        offset[i] = lo[i];
        size[i] = hi[i] - lo[i];
      }
  }
  if (count_out) *count_out = count;
  if (!device_positions || count == 0) return DPA_OK;
  return guarded(ctx, [&]() -> int {
    DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    uint64_t key = seed;
    key += 0x9e3779b97f4a7c15ull;
    key = (key ^ (key >> 30)) * 0xbf58476d1ce4e5b9ull;
    key = (key ^ (key >> 27)) * 0x94d049bb133111ebull;
    key ^= key >> 31;
    DPA_TRY_CUDA(ctx, dpa::launch_random_seeds(offset, size, count, key, device_positions,
                                               pick_stream(ctx, stream)));
    return DPA_OK;
  });
}

static int ftle_common(dpa_context* ctx, const dpa_field* field, const float seed_stride[3],
                       uint64_t iterations, float step_size, uint64_t count,
                       const float* original, const float* final_positions, int32_t mapping,
                       float* ftle, uint64_t shape_out[3], cudaStream_t s, dpa::FtleArgs* a,
                       uint64_t* cells) {
  if (!field || field->owner != ctx) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "bad field");
  if (!seed_stride) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "seed_stride is NULL");
  if (mapping != DPA_FTLE_MAPPING_REFERENCE && mapping != DPA_FTLE_MAPPING_LATTICE)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "unknown FTLE mapping");
  (void)s;
  for (int i = 0; i < 3; ++i) {
    if (!(seed_stride[i] > 0.0f)) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "stride must be positive");
    // size(scalar(shape) / stride) (ftle_estimator.cpp:16-22).
    const float q = float(field->shape[i]) / seed_stride[i];
    a->shape[i] = q > 0.0f ? uint64_t(q) : 0;
    a->offset[i] = field->offset[i];
    a->spacing[i] = field->spacing[i] * seed_stride[i];
    a->two_spacing[i] = 2.0f * a->spacing[i];
  }
  if (shape_out)
    for (int i = 0; i < 3; ++i) shape_out[i] = a->shape[i];
  *cells = a->shape[0] * a->shape[1] * a->shape[2];
  if (mapping == DPA_FTLE_MAPPING_LATTICE && count != *cells)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "lattice mapping needs one particle per cell");
  if (count && (!original || !final_positions))
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "positions are NULL");
  (void)ftle;
  const float horizon = std::fabs(step_size * float(iterations));
  a->count = count;
  a->mapping = mapping;
  a->horizon = double(horizon);
  return DPA_OK;
}

int dpa_ftle_estimate(dpa_context* ctx, const dpa_field* field, const float seed_stride[3],
                      uint64_t iterations, float step_size, uint64_t count,
                      const float* original_positions, const float* final_positions,
                      int32_t mapping, float* ftle, uint64_t shape_out[3]) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  return guarded(ctx, [&]() -> int {
    dpa::FtleArgs a{};
    uint64_t cells = 0;
    int st = ftle_common(ctx, field, seed_stride, iterations, step_size, count, original_positions,
                         final_positions, mapping, ftle, shape_out, ctx->stream, &a, &cells);
    if (st != DPA_OK || !ftle || cells == 0) return st;
    DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    DPA_TRY_CUDA(ctx, ctx->ftle_original.reserve(count * 12));
    DPA_TRY_CUDA(ctx, ctx->ftle_final.reserve(count * 12));
    DPA_TRY_CUDA(ctx, ctx->ftle_winners.reserve(cells * 8));
    DPA_TRY_CUDA(ctx, ctx->ftle_flow.reserve(cells * 12));
    DPA_TRY_CUDA(ctx, ctx->ftle_out.reserve(cells * 4));
    if (count) {
      DPA_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->ftle_original.ptr, original_positions, count * 12,
                                        cudaMemcpyHostToDevice, s));
      DPA_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->ftle_final.ptr, final_positions, count * 12,
                                        cudaMemcpyHostToDevice, s));
    }
    a.original_positions = ctx->ftle_original.as<float>();
    a.final_positions = ctx->ftle_final.as<float>();
    a.winners = ctx->ftle_winners.as<unsigned long long>();
    a.flow = ctx->ftle_flow.as<float>();
    a.ftle = ctx->ftle_out.as<float>();
    DPA_TRY_CUDA(ctx, dpa::launch_ftle(a, s));
    DPA_TRY_CUDA(ctx, cudaMemcpyAsync(ftle, ctx->ftle_out.ptr, cells * 4, cudaMemcpyDeviceToHost, s));
    DPA_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    return DPA_OK;
  });
}

int dpa_ftle_estimate_device(dpa_context* ctx, const dpa_field* field, const float seed_stride[3],
                             uint64_t iterations, float step_size, uint64_t count,
                             const float* device_original_positions,
                             const float* device_final_positions, int32_t mapping,
                             float* device_ftle, uint64_t shape_out[3], void* stream) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  return guarded(ctx, [&]() -> int {
    cudaStream_t s = pick_stream(ctx, stream);
    dpa::FtleArgs a{};
    uint64_t cells = 0;
    int st = ftle_common(ctx, field, seed_stride, iterations, step_size, count,
                         device_original_positions, device_final_positions, mapping, device_ftle,
                         shape_out, s, &a, &cells);
    if (st != DPA_OK || !device_ftle || cells == 0) return st;
    DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    DPA_TRY_CUDA(ctx, ctx->ftle_winners.reserve(cells * 8));
    DPA_TRY_CUDA(ctx, ctx->ftle_flow.reserve(cells * 12));
    a.original_positions = device_original_positions;
    a.final_positions = device_final_positions;
    a.winners = ctx->ftle_winners.as<unsigned long long>();
    a.flow = ctx->ftle_flow.as<float>();
    a.ftle = device_ftle;
    DPA_TRY_CUDA(ctx, dpa::launch_ftle(a, s));
    return DPA_OK;
  });
}

int dpa_context_set_tuning(dpa_context* ctx, const dpa_tuning* tuning) {
  if (!ctx || !tuning) return DPA_ERROR_INVALID_ARGUMENT;
  if (tuning->claim < 1 || tuning->claim > 4096)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "claim must be in [1, 4096]");
  if (tuning->order > dpa::kOrderMaxResolution)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "order resolution must be in [0, 64]");
  if (tuning->block_size % 32 != 0 || tuning->block_size > uint32_t(dpa::kAdvectBlock))
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT,
                "block_size must be 0 or a multiple of 32 up to " +
                    std::to_string(dpa::kAdvectBlock));
  if (tuning->particles_per_thread > 2)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "particles_per_thread must be 0, 1 or 2");
  ctx->tuning.claim = tuning->claim;
  ctx->tuning.blocks_per_sm = tuning->blocks_per_sm;
  ctx->tuning.order = tuning->order;
  ctx->tuning.block = tuning->block_size;
  ctx->tuning.particles_per_thread = tuning->particles_per_thread ? tuning->particles_per_thread : 1;
  return DPA_OK;
}

int dpa_context_get_tuning(const dpa_context* ctx, dpa_tuning* tuning) {
  if (!ctx || !tuning) return DPA_ERROR_INVALID_ARGUMENT;
  tuning->claim = ctx->tuning.claim;
  tuning->blocks_per_sm = ctx->tuning.blocks_per_sm;
  tuning->order = ctx->tuning.order;
  tuning->measured_ms = 0.0f;
  tuning->block_size = ctx->tuning.block;
  tuning->particles_per_thread = ctx->tuning.particles_per_thread;
  return DPA_OK;
}

int dpa_autotune_advect(dpa_context* ctx, const dpa_field* field, const dpa_advect_options* options,
                        uint64_t count, const float* device_positions,
                        const uint64_t* device_remaining, uint64_t sample_steps,
                        dpa_tuning* best) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  int st = check_options(ctx, options);
  if (st != DPA_OK) return st;
  if (options->record)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "autotune measures calls without recording");
  if (!field || field->owner != ctx) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "bad field");
  st = check_steady(ctx, field);
  if (st != DPA_OK) return st;
  if (count == 0 || !device_positions || !device_remaining)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "autotune needs particles");
  return guarded(ctx, [&]() -> int {
    DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    // A sample of the particles, run for at most sample_steps steps each.
    const uint64_t n = std::min<uint64_t>(count, 1ull << 22);
    DeviceBuffer pos, rem, pos0, rem0, term;
    DPA_TRY_CUDA(ctx, pos.reserve(n * 12));
    DPA_TRY_CUDA(ctx, rem.reserve(n * 8));
    DPA_TRY_CUDA(ctx, pos0.reserve(n * 12));
    DPA_TRY_CUDA(ctx, rem0.reserve(n * 8));
    DPA_TRY_CUDA(ctx, term.reserve(n));
    DPA_TRY_CUDA(ctx, cudaMemcpyAsync(pos0.ptr, device_positions, n * 12, cudaMemcpyDeviceToDevice, s));
    DPA_TRY_CUDA(ctx, cudaMemcpyAsync(rem0.ptr, device_remaining, n * 8, cudaMemcpyDeviceToDevice, s));
    dpa_advect_options o = *options;
    if (sample_steps && (o.max_steps == 0 || sample_steps < o.max_steps)) o.max_steps = sample_steps;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const cudaError_t made = cudaEventCreate(&e0);
    const cudaError_t made1 = made == cudaSuccess ? cudaEventCreate(&e1) : made;
    if (made1 != cudaSuccess) {
      if (e0) cudaEventDestroy(e0);
      return fail_cuda(ctx, made1, "cudaEventCreate");
    }
    const dpa_tuning_state saved = ctx->tuning;
    const bool profiling = ctx->profiling;
    ctx->profiling = false;
    dpa_tuning_state winner = saved;
    float winner_ms = 0.0f;
    bool first = true;
    int rc = DPA_OK;
    // Best of three timed runs (after one untimed) of the sample at the
    // current ctx->tuning; keeps it as the winner when it is the fastest yet.
    auto trial = [&]() {
      float best_ms = 0.0f;
      for (int rep = 0; rep < 3 && rc == DPA_OK; ++rep) {
        cudaMemcpyAsync(pos.ptr, pos0.ptr, n * 12, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(rem.ptr, rem0.ptr, n * 8, cudaMemcpyDeviceToDevice, s);
        cudaEventRecord(e0, s);
        rc = advect_device_impl(ctx, field, &o, n, pos.as<float>(), rem.as<uint64_t>(),
                                term.as<uint8_t>(), s);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && (best_ms == 0.0f || ms < best_ms)) best_ms = ms;
      }
      // A later setting replaces the winner only if it is at least 3 %
      // faster: timings of a sample vary by about that much, and the search
      // tries the defaults first.
      if (rc == DPA_OK && (first || best_ms < 0.97f * winner_ms)) {
        winner = ctx->tuning;
        winner_ms = best_ms;
        first = false;
      }
    };
    // Coordinate search from the defaults: processing order, then the launch
    // shape (threads per block and particles per lane), then claim size and
    // blocks per SM, each step keeping the best setting so far. Claims stay
    // small: a warp that claimed many entries works through them one lifetime
    // after another once the order runs out, which a sample with a step cap
    // does not show.
    for (uint32_t order : {64u, 16u, 0u}) {
      if (rc != DPA_OK) break;
      ctx->tuning = dpa_tuning_state{};
      ctx->tuning.order = order;
      trial();
    }
    const dpa_tuning_state after_order = winner;
    for (uint32_t block : {256u, 128u, 64u})
      for (uint32_t ppt : {1u, 2u}) {
        if (rc != DPA_OK) break;
        ctx->tuning = after_order;
        ctx->tuning.block = block;
        ctx->tuning.particles_per_thread = ppt;
        trial();
      }
    const dpa_tuning_state after_shape = winner;
    for (uint32_t grid : {0u, 3u, 2u})
      for (uint32_t claim : {16u, 32u}) {
        if (rc != DPA_OK) break;
        ctx->tuning = after_shape;
        ctx->tuning.blocks_per_sm = grid;
        ctx->tuning.claim = claim;
        trial();
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->profiling = profiling;
    ctx->tuning = rc == DPA_OK ? winner : saved;
    if (rc != DPA_OK) return rc;
    if (best) {
      best->claim = winner.claim;
      best->blocks_per_sm = winner.blocks_per_sm;
      best->order = winner.order;
      best->measured_ms = winner_ms;
      best->block_size = winner.block;
      best->particles_per_thread = winner.particles_per_thread;
    }
    return DPA_OK;
  });
}

int dpa_advect_batch_device(dpa_context* ctx, const dpa_field* field,
                            const dpa_advect_options* options, uint64_t set_count,
                            const uint64_t* set_offsets, float* device_positions,
                            uint64_t* device_remaining, uint8_t* device_termination,
                            uint64_t* set_steps, void* stream) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  int st = check_options(ctx, options);
  if (st != DPA_OK) return st;
  if (options->record)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "batched launches do not record");
  if (!field || field->owner != ctx) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "bad field");
  st = check_steady(ctx, field);
  if (st != DPA_OK) return st;
  if (set_count && !set_offsets) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "set_offsets is NULL");
  for (uint64_t i = 0; i < set_count; ++i)
    if (set_offsets[i + 1] < set_offsets[i])
      return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "set_offsets must not decrease");
  const uint64_t total = set_count ? set_offsets[set_count] - set_offsets[0] : 0;
  if (set_count && set_offsets[0] != 0)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "set_offsets must start at 0");
  if (total > 0xffffffffull)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "at most 2^32-1 particles per batch");
  if (total && (!device_positions || !device_remaining))
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "positions or remaining is NULL");
  return guarded(ctx, [&]() -> int {
    DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = pick_stream(ctx, stream);
    if (set_steps) {
      DPA_TRY_CUDA(ctx, ctx->remaining_in.reserve(total * 8 + 8));
      DPA_TRY_CUDA(ctx, ctx->raw_offsets.reserve((set_count + 1) * 8));
      DPA_TRY_CUDA(ctx, ctx->wide.reserve(set_count * 8 + 8));
      DPA_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->remaining_in.ptr, device_remaining, total * 8,
                                        cudaMemcpyDeviceToDevice, s));
    }
    // One persistent launch over every set: each particle carries its own
    // remaining iteration count, so sets of any size and iteration count mix.
    st = advect_device_impl(ctx, field, options, total, device_positions, device_remaining,
                            device_termination, s);
    if (st != DPA_OK) return st;
    if (set_steps && set_count) {
      DPA_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->raw_offsets.ptr, set_offsets, (set_count + 1) * 8,
                                        cudaMemcpyHostToDevice, s));
      DPA_TRY_CUDA(ctx, dpa::launch_set_steps(ctx->remaining_in.as<uint64_t>(), device_remaining,
                                              ctx->raw_offsets.as<uint64_t>(), set_count,
                                              ctx->wide.as<unsigned long long>(), s));
      DPA_TRY_CUDA(ctx, cudaMemcpyAsync(set_steps, ctx->wide.ptr, set_count * 8,
                                        cudaMemcpyDeviceToHost, s));
      DPA_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    }
    return DPA_OK;
  });
}

int dpa_graph_create_advect(dpa_context* ctx, const dpa_field* field,
                            const dpa_advect_options* options, uint64_t count,
                            float* device_positions, uint64_t* device_remaining,
                            uint8_t* device_termination, dpa_graph** out) {
  if (!ctx || !out) return DPA_ERROR_INVALID_ARGUMENT;
  *out = nullptr;
  int st = check_options(ctx, options);
  if (st != DPA_OK) return st;
  if (options->record) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "graphs do not record");
  if (!field || field->owner != ctx) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "bad field");
  st = check_steady(ctx, field);
  if (st != DPA_OK) return st;
  if (count == 0 || count > 0xffffffffull || !device_positions || !device_remaining)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "graphs need 1 to 2^32-1 particles");
  return guarded(ctx, [&]() -> int {
    DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    auto g = std::make_unique<dpa_graph>();
    g->owner = ctx;
    // Everything the launch sequence allocates or looks up, before capture.
    // The graph's scratch is its own: the captured kernels keep its
    // addresses for every replay.
    DPA_TRY_CUDA(ctx, g->scratch.keys.reserve(count * 4));
    DPA_TRY_CUDA(ctx, g->scratch.values.reserve(count * 4));
    DPA_TRY_CUDA(ctx, g->scratch.sort_temp.reserve(dpa::kOrderCountsSize * 4));
    DPA_TRY_CUDA(ctx, g->scratch.work_counter.reserve(sizeof(unsigned long long)));
    {
      dpa::AdvectArgs launch{};
      dpa::set_launch_defaults(launch);
      dpa::apply_tuning(ctx->tuning, launch);
      DPA_TRY_CUDA(ctx, dpa::prepare_advect(field->view, launch, options->integrator, false));
    }
    DPA_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    const bool profiling = ctx->profiling;
    ctx->profiling = false;
    const uint64_t launches0 = ctx->launches;
    cudaGraph_t graph = nullptr;
    DPA_TRY_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    st = advect_device_impl(ctx, field, options, count, device_positions, device_remaining,
                            device_termination, s, nullptr, &g->scratch);
    const cudaError_t end = cudaStreamEndCapture(s, &graph);
    ctx->profiling = profiling;
    const uint64_t captured = ctx->launches - launches0;
    ctx->launches = launches0;  // capture launched nothing
    if (st != DPA_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (end != cudaSuccess) return fail_cuda(ctx, end, "cudaStreamEndCapture");
    cudaGraphExec_t exec = nullptr;
    const cudaError_t inst = cudaGraphInstantiate(&exec, graph, 0);
    if (inst != cudaSuccess) {
      cudaGraphDestroy(graph);
      return fail_cuda(ctx, inst, "cudaGraphInstantiate");
    }
    g->graph = graph;
    g->exec = exec;
    g->launches = captured;
    *out = g.release();
    return DPA_OK;
  });
}

int dpa_graph_launch(dpa_context* ctx, dpa_graph* graph, void* stream) {
  if (!ctx || !graph || graph->owner != ctx) return DPA_ERROR_INVALID_ARGUMENT;
  DPA_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  DPA_TRY_CUDA(ctx, cudaGraphLaunch(graph->exec, pick_stream(ctx, stream)));
  ctx->launches += graph->launches;
  return DPA_OK;
}

int dpa_graph_destroy(dpa_context* ctx, dpa_graph* graph) {
  if (!ctx || !graph || graph->owner != ctx) return DPA_ERROR_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  // Replays may run on any stream; the scratch goes only once they are done.
  cudaDeviceSynchronize();
  if (graph->exec) cudaGraphExecDestroy(graph->exec);
  if (graph->graph) cudaGraphDestroy(graph->graph);
  delete graph;
  return DPA_OK;
}

}  // extern "C"
