// serve.cu -- the request server: resident fields, admission by device
// memory, continuous batching of advection / FTLE requests.
//
// No counterpart in the reference (a batch MPI program). A worker thread owns
// two device arenas: particle slots (position, remaining iterations and the
// per-particle state of resumable launches) and raw curve staging (the
// unpruned vertices of recording requests, remaining + 2 per particle). A
// request is admitted, first in first out, when the arenas have room for it:
// its seeds take `count` slots, and a recording request also takes
// count * (iterations + 2) staging vertices -- its output buffer. Admitted
// requests advance together: each tick is one persistent advection launch per
// (field, integrator, step, recording) group over every in-flight particle of
// the group's requests, with a step budget, so requests that arrive while
// others run join at the next tick and share the launches. A request whose
// particles have all finished leaves the ticks at once; a second thread with
// its own stream copies its results out, emits its curve and FTLE and returns
// it, while the worker's ticks go on.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "admission.hpp"
#include "handles.cuh"
#include "kernels.cuh"
#include "range_allocator.hpp"

namespace {

using clock_type = std::chrono::steady_clock;

constexpr size_t kMaxServerFields = 256;

using dpa::range_allocator;

struct pending {
  uint64_t id;
  dpa_request request;
  std::vector<float> positions;
  double queued;
  double deadline;  // seconds since the server started; 0: none
};

struct active_request {
  pending p;
  uint32_t slot;         // index of its in-flight counter
  uint64_t first;        // first particle slot
  uint64_t raw_first;    // first staging vertex (recording)
  uint64_t raw_count;
  double admitted;
  uint64_t first_tick;   // the first tick that advances it
  int32_t dropped = DPA_OK;  // DPA_ERROR_TIMEOUT / CANCELLED once dropped while running
};

// A returned request: one block holds all its arrays, in the server's pinned
// response arena when it has room (the copies then run at the link's speed),
// else in pageable heap memory.
struct response_storage {
  dpa_response r{};
  char* data = nullptr;
  uint64_t arena_offset = ~0ull;  // in units of kResponseUnit; ~0: heap
  uint64_t arena_units = 0;
  std::unique_ptr<char[]> heap;
};

constexpr uint64_t kResponseUnit = 256;

}  // namespace

struct dpa_server {
  dpa_context* ctx = nullptr;
  dpa_server_options options{};
  // The context's launch tuning when the server was created: the worker
  // reads it without the context, which other threads may retune.
  dpa_tuning_state tuning;
  std::vector<const dpa_field*> fields;
  cudaStream_t stream = nullptr;

  // Particle arena (per slot) and curve staging arena (per vertex).
  DeviceBuffer positions, times, remaining, remaining_initial, termination, raw_offsets,
      kept_vertices, kept_segments, curve_open, request_of, raw, in_flight;
  // Processing order of each request's particles, relative to its first slot
  // (a Morton sort of its seeds at admission), and the sort's bucket ids and
  // counters.
  DeviceBuffer seed_order, order_ids, order_counts;
  // Per tick. Two ticks may be in flight, so the host-side buffers a tick's
  // copies read or write come in two halves, one per tick parity.
  DeviceBuffer list, starts, firsts, work_counter;
  PinnedBuffer host_ranges[2], host_in_flight;
  cudaStream_t upload_stream = nullptr;  // seed copies, beside the running tick
  cudaEvent_t seeds_copied = nullptr, readback[2] = {nullptr, nullptr};
  cudaEvent_t tick_start[2] = {nullptr, nullptr};  // device time of each tick
  // Emission scratch.
  DeviceBuffer raw_counts, curve_totals, vertex_offsets, segment_offsets, scan_temp, out_vertices,
      out_colors, out_indices;
  DeviceBuffer ftle_original, ftle_winners, ftle_flow, ftle_out;
  range_allocator slots, vertices;
  PinnedBuffer response_arena;
  range_allocator response_units;  // of response_arena, in kResponseUnit bytes
  std::vector<uint32_t> free_counters;

  std::mutex mutex;
  std::condition_variable wake, done_signal;
  std::deque<pending> queue;
  std::vector<active_request> active;
  uint64_t used_slots = 0;
  uint64_t small_slots = 0;  // of used_slots, held by small requests
  uint64_t used_vertices = 0;
  dpa::admission_config admission;
  std::map<uint64_t, int32_t> drop_requests;  // id -> status, from dpa_server_cancel
  std::map<uint64_t, std::unique_ptr<response_storage>> done, handed_out;
  std::deque<uint64_t> done_order;
  std::thread worker, finisher;
  cudaStream_t finish_stream = nullptr;
  std::deque<active_request> finishing;  // handed from the worker to the finisher
  std::condition_variable finish_wake;
  bool stopping = false;
  bool worker_done = false;
  std::string failure;
  uint64_t next_id = 1;
  dpa_server_stats stats{};
  clock_type::time_point start = clock_type::now();

  double now() const { return std::chrono::duration<double>(clock_type::now() - start).count(); }
  void run();
  void run_finisher();
  void destroy_streams() {
    for (cudaStream_t st : {stream, finish_stream, upload_stream})
      if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
      }
    for (cudaEvent_t ev : {seeds_copied, readback[0], readback[1], tick_start[0], tick_start[1]})
      if (ev) cudaEventDestroy(ev);
    stream = finish_stream = upload_stream = nullptr;
    seeds_copied = readback[0] = readback[1] = tick_start[0] = tick_start[1] = nullptr;
  }
  uint32_t tick(uint64_t steps, int parity);
  void select(std::vector<active_request>& out);
  void drop_waiting(double t);
  void drop_running(double t);
  void upload(std::vector<active_request>& admitted, uint64_t first_tick);
  void finish(active_request& a, response_storage& out);
};

namespace {

#define SERVER_TRY(expr)                                                   \
  do {                                                                     \
    const cudaError_t e_ = (expr);                                         \
    if (e_ != cudaSuccess)                                                 \
      throw std::runtime_error(std::string(#expr) + ": " + cudaGetErrorName(e_)); \
  } while (0)

// Per-particle state of a newly admitted request in slots [first, first + n):
// remaining (and its initial copy) = iterations, in flight, owned by counter
// `slot`, at time t0, with curve staging at raw_first + i (iterations + 2);
// the request's in-flight counter = n.
__global__ void serve_init_kernel(uint64_t first, uint64_t n, uint64_t iterations, float t0,
                                  uint32_t slot, bool record, uint64_t raw_first, bool ordered,
                                  uint64_t* remaining, uint64_t* remaining_initial,
                                  uint8_t* termination, uint32_t* request_of, float* times,
                                  uint64_t* raw_offsets, uint32_t* seed_order,
                                  unsigned int* in_flight) {
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i == 0) in_flight[slot] = unsigned(n);
  if (i >= n) return;
  const uint64_t k = first + i;
  remaining[k] = iterations;
  remaining_initial[k] = iterations;
  termination[k] = DPA_TERMINATION_IN_FLIGHT;
  request_of[k] = slot;
  times[k] = t0;
  if (record) raw_offsets[k] = raw_first + i * (iterations + 2);
  if (!ordered) seed_order[k] = uint32_t(i);
}

// Drops a running request between ticks: its particles still in flight are
// marked cancelled (later ticks skip them) and its in-flight counter is
// zeroed, so the next read of the counters hands it to the finisher.
__global__ void serve_drop_kernel(uint64_t first, uint64_t n, uint32_t slot, uint8_t* termination,
                                  unsigned int* in_flight) {
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i == 0) in_flight[slot] = 0;
  if (i < n && termination[first + i] == DPA_TERMINATION_IN_FLIGHT)
    termination[first + i] = DPA_TERMINATION_CANCELLED;
}

// Requests of fewer seeds run in submission order: sorting them would cost
// more launches than their few warps gain in locality.
constexpr uint64_t kServeOrderMin = 4096;

// Requests advance in step budgets of steps_per_tick, so a particle resumes
// in a later tick: integrators that carry a derivative from one step to the
// next (dpa::integrator_has_history) are not served.
bool integrator_ok(int32_t i) {
  const bool known = (i >= DPA_INTEGRATOR_EULER && i <= DPA_INTEGRATOR_ADAMS_BASHFORTH_MOULTON_2) ||
                     i == DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE;
  return known && !dpa::integrator_has_history(i);
}

}  // namespace

// Called with the mutex held: moves the waiting requests that may start now
// into `out` (the policy of admission.hpp: oldest first, younger requests
// that fit may pass one that does not, within the reserve and bypass limits).
void dpa_server::select(std::vector<active_request>& out) {
  const double t = now();
  uint64_t first = 0, raw_first = 0;
  dpa::admit_waiting(
      queue, admission, used_slots, small_slots, [](const pending& p) { return p.request.count; },
      [&](const pending& p) { return t - p.queued; },
      [&](const pending& p) {
        const dpa_request& q = p.request;
        const uint64_t raw_need = q.record ? q.count * (q.iterations + 2) : 0;
        if (!slots.allocate(q.count, &first)) {
          ++stats.slot_refusals;
          return false;
        }
        if (!vertices.allocate(raw_need, &raw_first)) {
          slots.release(first, q.count);
          ++stats.vertex_refusals;
          return false;
        }
        return true;
      },
      [&](pending& p) {
        active_request a;
        a.raw_count = p.request.record ? p.request.count * (p.request.iterations + 2) : 0;
        a.p = std::move(p);
        a.slot = free_counters.back();
        free_counters.pop_back();
        a.first = first;
        a.raw_first = raw_first;
        a.admitted = t;
        used_vertices += a.raw_count;
        out.push_back(std::move(a));
      },
      [&] { return !free_counters.empty(); });
  stats.peak_slots = std::max(stats.peak_slots, used_slots);
  stats.peak_vertices = std::max(stats.peak_vertices, used_vertices);
  if (!queue.empty() && t - queue.front().queued >= admission.max_bypass_seconds)
    ++stats.overdue_scans;
}

// Called with the mutex held: returns the waiting requests that have passed
// their deadline or were cancelled, without arrays.
void dpa_server::drop_waiting(double t) {
  for (auto it = queue.begin(); it != queue.end();) {
    int32_t status = DPA_OK;
    const auto c = drop_requests.find(it->id);
    if (c != drop_requests.end()) {
      status = c->second;
      drop_requests.erase(c);
    } else if (it->deadline > 0.0 && t >= it->deadline) {
      status = DPA_ERROR_TIMEOUT;
    }
    if (status == DPA_OK) {
      ++it;
      continue;
    }
    auto out = std::make_unique<response_storage>();
    dpa_response& r = out->r;
    r.id = it->id;
    r.user = it->request.user;
    r.status = status;
    r.count = it->request.count;
    r.queued_seconds = it->queued;
    r.admitted_seconds = t;
    r.finished_seconds = t;
    done_order.push_back(r.id);
    done[r.id] = std::move(out);
    stats.completed += 1;
    it = queue.erase(it);
    done_signal.notify_all();
  }
}

// Called with the mutex held, in the worker between ticks: a running request
// past its deadline or cancelled is dropped on the ticks' stream before the
// next tick (serve_drop_kernel) and finishes through the usual read of the
// in-flight counters.
void dpa_server::drop_running(double t) {
  for (active_request& a : active) {
    if (a.dropped != DPA_OK) continue;
    int32_t status = DPA_OK;
    const auto c = drop_requests.find(a.p.id);
    if (c != drop_requests.end()) {
      status = c->second;
      drop_requests.erase(c);
    } else if (a.p.deadline > 0.0 && t >= a.p.deadline) {
      status = DPA_ERROR_TIMEOUT;
    }
    if (status == DPA_OK) continue;
    a.dropped = status;
    const uint64_t n = a.p.request.count;
    serve_drop_kernel<<<unsigned(std::max<uint64_t>((n + 255) / 256, 1)), 256, 0, stream>>>(
        a.first, n, a.slot, termination.as<uint8_t>(), in_flight.as<unsigned int>());
    SERVER_TRY(cudaGetLastError());
  }
}

// Starts admitted requests on the device: their seeds are copied in on the
// upload stream, beside the running tick (whose particles never share slots
// with them: a slot is reused only after its request has finished and been
// returned, and ticks skip finished particles). Then, in the ticks' stream
// order, a request of kServeOrderMin seeds or more is sorted into its
// processing order, so that the lanes of a tick sweep its seeds in Morton
// order of their start cells, and an init kernel per request sets its
// per-particle state (every particle in flight) and its in-flight counter.
// The sort stays in the ticks' stream: a running tick may still expand the
// slot range of a request that finished in the tick before (ticks skip its
// particles, but read its processing order), and a new request may reuse
// that range. Worker thread, without the mutex.
void dpa_server::upload(std::vector<active_request>& admitted, uint64_t first_tick) {
  for (active_request& a : admitted) {
    a.first_tick = first_tick;
    const uint64_t n = a.p.request.count;
    if (n)
      SERVER_TRY(cudaMemcpyAsync(positions.as<float>() + 3 * a.first, a.p.positions.data(),
                                 n * 12, cudaMemcpyHostToDevice, upload_stream));
  }
  SERVER_TRY(cudaEventRecord(seeds_copied, upload_stream));
  SERVER_TRY(cudaStreamWaitEvent(stream, seeds_copied, 0));
  for (const active_request& a : admitted) {
    const uint64_t n = a.p.request.count;
    if (n >= kServeOrderMin && tuning.order)
      SERVER_TRY(dpa::launch_order(fields[size_t(a.p.request.field)]->view,
                                   positions.as<float>() + 3 * a.first, n,
                                   order_ids.as<uint32_t>() + a.first,
                                   order_counts.as<uint32_t>(),
                                   seed_order.as<uint32_t>() + a.first, stream,
                                   tuning.order));
  }
  for (const active_request& a : admitted) {
    const dpa_request& q = a.p.request;
    const uint64_t n = q.count;
    serve_init_kernel<<<unsigned(std::max<uint64_t>((n + 255) / 256, 1)), 256, 0, stream>>>(
        a.first, n, q.iterations, q.start_time, a.slot, q.record != 0, a.raw_first,
        n >= kServeOrderMin && tuning.order, remaining.as<uint64_t>(),
        remaining_initial.as<uint64_t>(), termination.as<uint8_t>(), request_of.as<uint32_t>(),
        times.as<float>(), raw_offsets.as<uint64_t>(), seed_order.as<uint32_t>(),
        in_flight.as<unsigned int>());
    SERVER_TRY(cudaGetLastError());
  }
}

// One tick: a step-budgeted launch per group of requests that can share one.
// Returns false when nothing was in flight.
uint32_t dpa_server::tick(uint64_t steps, int parity) {
  using key_type = std::tuple<int32_t, int32_t, float, int32_t>;  // field, integrator, step, record
  std::map<key_type, std::vector<const active_request*>> groups;
  for (const active_request& a : active) {
    const dpa_request& q = a.p.request;
    if (q.count == 0) continue;
    groups[{q.field, q.integrator, q.step_size, q.record ? 1 : 0}].push_back(&a);
  }
  if (groups.empty()) return 0;
  // Every group's ranges get their own part of the pinned buffer, so no copy
  // has to finish before the next group's ranges are written.
  uint64_t all_ranges = 0;
  for (auto& g : groups) all_ranges += g.second.size();
  uint32_t launched = 0;
  PinnedBuffer& host = host_ranges[parity];
  SERVER_TRY(host.reserve(all_ranges * 16));
  uint64_t range_base = 0;
  for (auto& [key, members] : groups) {
    const auto [field_id, integrator, step_size, record] = key;
    const dpa_field* field = fields[size_t(field_id)];
    const uint32_t ranges = uint32_t(members.size());
    SERVER_TRY(starts.reserve(uint64_t(ranges) * 8));
    SERVER_TRY(firsts.reserve(uint64_t(ranges) * 8));
    uint64_t* h = host.as<uint64_t>() + 2 * range_base;
    range_base += ranges;
    uint64_t total = 0;
    for (uint32_t r = 0; r < ranges; ++r) {
      h[r] = members[r]->first;
      h[ranges + r] = total;
      total += members[r]->p.request.count;
    }
    SERVER_TRY(list.reserve(total * 4));
    SERVER_TRY(cudaMemcpyAsync(starts.ptr, h, uint64_t(ranges) * 8, cudaMemcpyHostToDevice, stream));
    SERVER_TRY(cudaMemcpyAsync(firsts.ptr, h + ranges, uint64_t(ranges) * 8, cudaMemcpyHostToDevice,
                               stream));
    SERVER_TRY(dpa::launch_expand_ranges(starts.as<uint64_t>(), firsts.as<uint64_t>(), ranges,
                                         total, seed_order.as<uint32_t>(), list.as<uint32_t>(),
                                         stream));
    dpa::AdvectArgs a{};
    dpa::set_launch_defaults(a);
    a.count = total;
    a.order = list.as<uint32_t>();
    a.positions = positions.as<float>();
    a.times = times.as<float>();
    a.remaining = remaining.as<uint64_t>();
    a.termination = termination.as<uint8_t>();
    a.coefficients = dpa::make_step_coefficients(integrator, step_size);
    a.max_steps = steps;
    dpa::apply_tuning(tuning, a);
    a.work_counter = work_counter.as<unsigned long long>();
    a.resume_only = true;
    a.request_of = request_of.as<uint32_t>();
    a.in_flight = in_flight.as<unsigned int>();
    if (record) {
      a.raw_vertices = raw.as<float>();
      a.raw_offsets = raw_offsets.as<uint64_t>();
      a.kept_vertices = kept_vertices.as<uint32_t>();
      a.kept_segments = kept_segments.as<uint32_t>();
      a.remaining_initial = remaining_initial.as<uint64_t>();
      a.curve_open = curve_open.as<uint8_t>();
    }
    SERVER_TRY(dpa::launch_advect(field->view, a, integrator, record != 0, stream));
    ++launched;
  }
  return launched;
}

// A request whose particles have all finished: copies its end states out,
// emits its curve and FTLE; finisher thread, on its own stream, without the
// mutex. The worker no longer touches the request's arena ranges.
void dpa_server::finish(active_request& a, response_storage& out) {
  const dpa_request& q = a.p.request;
  const uint64_t n = q.count, first = a.first;
  // A request the worker dropped is returned as it stood, without curve or
  // FTLE -- unless every particle had finished before the drop took effect.
  int32_t status = DPA_OK;
  if (a.dropped != DPA_OK && n) {
    std::vector<uint8_t> term(n);
    SERVER_TRY(cudaMemcpyAsync(term.data(), termination.as<uint8_t>() + first, n,
                               cudaMemcpyDeviceToHost, finish_stream));
    SERVER_TRY(cudaStreamSynchronize(finish_stream));
    for (uint64_t i = 0; i < n && status == DPA_OK; ++i)
      if (term[i] == DPA_TERMINATION_CANCELLED) status = a.dropped;
  }
  const bool record = q.record && n && status == DPA_OK;
  const bool ftle = q.ftle && n && status == DPA_OK;
  uint64_t vertex_count = 0, index_count = 0;
  const size_t index_bytes = q.index64 ? 8 : 4;
  if (record) {
    // Emission of the request's curve, as one round of the reference:
    // offsets and totals first, to size the response.
    SERVER_TRY(raw_counts.reserve(n * 8));
    SERVER_TRY(vertex_offsets.reserve(n * 8));
    SERVER_TRY(segment_offsets.reserve(n * 8));
    SERVER_TRY(dpa::launch_raw_counts(remaining_initial.as<uint64_t>() + first,
                                      remaining.as<uint64_t>() + first, n,
                                      raw_counts.as<uint64_t>(), finish_stream));
    SERVER_TRY(scan_temp.reserve(dpa::curve_offsets_scratch_bytes(n)));
    SERVER_TRY(curve_totals.reserve(16));
    SERVER_TRY(dpa::launch_curve_offsets(kept_vertices.as<uint32_t>() + first,
                                         kept_segments.as<uint32_t>() + first, n, scan_temp.ptr,
                                         vertex_offsets.as<uint64_t>(),
                                         segment_offsets.as<uint64_t>(),
                                         curve_totals.as<unsigned long long>(), finish_stream));
    uint64_t totals[2];
    SERVER_TRY(cudaMemcpyAsync(totals, curve_totals.ptr, 16, cudaMemcpyDeviceToHost,
                               finish_stream));
    SERVER_TRY(cudaStreamSynchronize(finish_stream));
    vertex_count = totals[0];
    index_count = 2 * totals[1];
  }
  dpa_response& r = out.r;
  dpa::FtleArgs f{};
  uint64_t cells = 0;
  if (ftle) {
    // Lattice FTLE of the final positions (ftle_estimator.cpp:7-65); the
    // seeds should be the lattice of seed_stride on the request's field.
    const dpa_field* field = fields[size_t(q.field)];
    for (int i = 0; i < 3; ++i) {
      const float stride = q.seed_stride[i] > 0.0f ? q.seed_stride[i] : 1.0f;
      const float c = float(field->shape[i]) / stride;
      f.shape[i] = c > 0.0f ? uint64_t(c) : 0;
      f.offset[i] = field->offset[i];
      f.spacing[i] = field->spacing[i] * stride;
      f.two_spacing[i] = 2.0f * f.spacing[i];
      r.ftle_shape[i] = f.shape[i];
    }
    cells = f.shape[0] * f.shape[1] * f.shape[2];
  }
  // One block for every array, each part 16-byte aligned.
  auto pad = [](uint64_t b) { return (b + 15) / 16 * 16; };
  const uint64_t part[8] = {pad(12 * n),           pad(4 * n),
                            pad(8 * n),            pad(n),
                            pad(12 * vertex_count), pad(4 * vertex_count),
                            pad(index_bytes * index_count), pad(4 * cells)};
  uint64_t at[8], bytes = 0;
  for (int i = 0; i < 8; ++i) {
    at[i] = bytes;
    bytes += part[i];
  }
  {
    std::lock_guard<std::mutex> lock(mutex);
    const uint64_t units = (bytes + kResponseUnit - 1) / kResponseUnit;
    uint64_t offset = 0;
    if (bytes && response_units.allocate(units, &offset)) {
      out.arena_offset = offset;
      out.arena_units = units;
      out.data = response_arena.as<char>() + offset * kResponseUnit;
    }
  }
  if (!out.data) {
    out.heap.reset(new char[std::max<uint64_t>(bytes, 16)]);  // not zero-filled
    out.data = out.heap.get();
  }
  char* d = out.data;
  if (n) {
    SERVER_TRY(cudaMemcpyAsync(d + at[0], positions.as<float>() + 3 * first, n * 12,
                               cudaMemcpyDeviceToHost, finish_stream));
    SERVER_TRY(cudaMemcpyAsync(d + at[1], times.as<float>() + first, n * 4,
                               cudaMemcpyDeviceToHost, finish_stream));
    SERVER_TRY(cudaMemcpyAsync(d + at[2], remaining.as<uint64_t>() + first, n * 8,
                               cudaMemcpyDeviceToHost, finish_stream));
    SERVER_TRY(cudaMemcpyAsync(d + at[3], termination.as<uint8_t>() + first, n,
                               cudaMemcpyDeviceToHost, finish_stream));
  }
  if (record) {
    SERVER_TRY(out_vertices.reserve(vertex_count * 12));
    SERVER_TRY(out_colors.reserve(vertex_count * 4));
    SERVER_TRY(out_indices.reserve(index_count * index_bytes));
    dpa::EmitArgs e{};
    e.count = n;
    e.raw_vertices = raw.as<float>();
    e.raw_offsets = raw_offsets.as<uint64_t>() + first;
    e.steps_raw = raw_counts.as<uint64_t>();
    e.vertex_offsets = vertex_offsets.as<uint64_t>();
    e.segment_offsets = segment_offsets.as<uint64_t>();
    e.kept_vertices = kept_vertices.as<uint32_t>() + first;
    e.vertex_base = 0;
    e.vertices = out_vertices.as<float>();
    e.colors = out_colors.as<float>();
    e.indices = out_indices.ptr;
    SERVER_TRY(dpa::launch_emit(e, q.index64 != 0, true, finish_stream));
    SERVER_TRY(cudaMemcpyAsync(d + at[4], out_vertices.ptr, vertex_count * 12,
                               cudaMemcpyDeviceToHost, finish_stream));
    SERVER_TRY(cudaMemcpyAsync(d + at[5], out_colors.ptr, vertex_count * 4,
                               cudaMemcpyDeviceToHost, finish_stream));
    SERVER_TRY(cudaMemcpyAsync(d + at[6], out_indices.ptr, index_count * index_bytes,
                               cudaMemcpyDeviceToHost, finish_stream));
  }
  if (ftle && cells) {
    SERVER_TRY(ftle_original.reserve(n * 12));
    SERVER_TRY(ftle_winners.reserve(cells * 8));
    SERVER_TRY(ftle_flow.reserve(cells * 12));
    SERVER_TRY(ftle_out.reserve(cells * 4));
    SERVER_TRY(cudaMemcpyAsync(ftle_original.ptr, a.p.positions.data(), n * 12,
                               cudaMemcpyHostToDevice, finish_stream));
    f.count = n;
    f.original_positions = ftle_original.as<float>();
    f.final_positions = positions.as<float>() + 3 * first;
    f.mapping = DPA_FTLE_MAPPING_REFERENCE;
    f.horizon = double(std::fabs(q.step_size * float(q.iterations)));
    f.winners = ftle_winners.as<unsigned long long>();
    f.flow = ftle_flow.as<float>();
    f.ftle = ftle_out.as<float>();
    SERVER_TRY(dpa::launch_ftle(f, finish_stream));
    SERVER_TRY(cudaMemcpyAsync(d + at[7], ftle_out.ptr, cells * 4, cudaMemcpyDeviceToHost,
                               finish_stream));
  }
  SERVER_TRY(cudaStreamSynchronize(finish_stream));
  const uint64_t* rem_out = reinterpret_cast<const uint64_t*>(d + at[2]);
  uint64_t steps = 0;
  for (uint64_t i = 0; i < n; ++i) steps += q.iterations - rem_out[i];
  r.status = status;
  r.id = a.p.id;
  r.user = q.user;
  r.count = n;
  r.positions = reinterpret_cast<const float*>(d + at[0]);
  r.times = reinterpret_cast<const float*>(d + at[1]);
  r.remaining = rem_out;
  r.termination = reinterpret_cast<const uint8_t*>(d + at[3]);
  r.vertex_count = vertex_count;
  r.vertices = record ? reinterpret_cast<const float*>(d + at[4]) : nullptr;
  r.colors = record ? reinterpret_cast<const float*>(d + at[5]) : nullptr;
  r.index_count = index_count;
  r.indices = record ? static_cast<const void*>(d + at[6]) : nullptr;
  r.ftle = (ftle && cells) ? reinterpret_cast<const float*>(d + at[7]) : nullptr;
  r.particle_steps = steps;
  r.queued_seconds = a.p.queued;
  r.admitted_seconds = a.admitted;
  r.finished_seconds = now();
}

// The worker keeps the GPU fed: it launches tick k and only then looks at
// tick k - 1's in-flight counters, so tick k runs while the host admits,
// uploads and hands finished requests to the finisher. A request finishing in
// tick k - 1 may still be in tick k's launch list; tick k skips its finished
// particles.
void dpa_server::run() {
  try {
    SERVER_TRY(cudaSetDevice(ctx->device));
    const uint64_t counters = options.max_requests;
    SERVER_TRY(host_in_flight.reserve(2 * 4 * counters));
    uint64_t next_tick = 0;
    bool pending = false;  // a launched tick whose counters are not read yet
    uint64_t pending_tick = 0;
    while (true) {
      std::vector<active_request> admitted;
      bool waiting = false;
      {
        std::unique_lock<std::mutex> lock(mutex);
        if (!failure.empty()) break;  // the finisher failed
        const double t = now();
        drop_waiting(t);
        drop_running(t);
        select(admitted);
        waiting = !queue.empty();
        if (active.empty() && admitted.empty() && !pending) {
          if (stopping && queue.empty()) break;
          wake.wait_for(lock, std::chrono::milliseconds(2));
          continue;
        }
      }
      const auto t0 = clock_type::now();
      if (!admitted.empty()) {
        upload(admitted, next_tick);
        std::lock_guard<std::mutex> lock(mutex);
        for (active_request& a : admitted) active.push_back(std::move(a));
        stats.admitted += admitted.size();
      }
      bool launched = false;
      const int parity = int(next_tick & 1);
      if (!active.empty()) {
        // While no request waits for admission, ticks run four times as many
        // steps: fewer launches per step for the same latency to the next
        // arrival's admission, which only a waiting request could use.
        const uint64_t base = options.steps_per_tick ? options.steps_per_tick : 64;
        SERVER_TRY(cudaEventRecord(tick_start[parity], stream));
        const uint32_t launches = tick(waiting ? base : 4 * base, parity);
        {
          std::lock_guard<std::mutex> lock(mutex);
          stats.launches += launches;
          stats.ticks += 1;
        }
        // Which requests have no particle in flight any more?
        SERVER_TRY(cudaMemcpyAsync(host_in_flight.as<unsigned int>() + parity * counters,
                                   in_flight.ptr, 4 * counters, cudaMemcpyDeviceToHost, stream));
        SERVER_TRY(cudaEventRecord(readback[parity], stream));
        launched = true;
      }
      if (pending) {
        SERVER_TRY(cudaEventSynchronize(readback[pending_tick & 1]));
        const unsigned int* left =
            host_in_flight.as<unsigned int>() + (pending_tick & 1) * counters;
        float tick_ms = 0.0f;
        SERVER_TRY(cudaEventElapsedTime(&tick_ms, tick_start[pending_tick & 1],
                                        readback[pending_tick & 1]));
        std::lock_guard<std::mutex> lock(mutex);
        stats.tick_device_seconds += 1e-3 * double(tick_ms);
        bool handed = false;
        for (size_t i = active.size(); i-- > 0;) {
          // Requests admitted after that tick have not been counted yet.
          if (active[i].first_tick > pending_tick || left[active[i].slot] != 0) continue;
          finishing.push_back(std::move(active[i]));
          active.erase(active.begin() + long(i));
          handed = true;
        }
        stats.peak_finishing = std::max(stats.peak_finishing, uint32_t(finishing.size()));
        if (handed) finish_wake.notify_one();
        pending = false;
      }
      if (launched) {
        pending = true;
        pending_tick = next_tick++;
      }
      std::lock_guard<std::mutex> lock(mutex);
      stats.busy_seconds += std::chrono::duration<double>(clock_type::now() - t0).count();
    }
  } catch (const std::exception& e) {
    std::lock_guard<std::mutex> lock(mutex);
    failure = e.what();
    stopping = true;
    done_signal.notify_all();
  }
  std::lock_guard<std::mutex> lock(mutex);
  worker_done = true;
  finish_wake.notify_all();
}

void dpa_server::run_finisher() {
  try {
    SERVER_TRY(cudaSetDevice(ctx->device));
    while (true) {
      active_request a;
      {
        std::unique_lock<std::mutex> lock(mutex);
        finish_wake.wait(lock, [&] { return !finishing.empty() || worker_done; });
        if (finishing.empty()) break;
        a = std::move(finishing.front());
        finishing.pop_front();
      }
      auto out = std::make_unique<response_storage>();
      const auto f0 = clock_type::now();
      finish(a, *out);
      std::lock_guard<std::mutex> lock(mutex);
      stats.finish_seconds += std::chrono::duration<double>(clock_type::now() - f0).count();
      slots.release(a.first, a.p.request.count);
      used_slots -= a.p.request.count;
      if (a.p.request.count <= admission.small_seeds) small_slots -= a.p.request.count;
      vertices.release(a.raw_first, a.raw_count);
      used_vertices -= a.raw_count;
      free_counters.push_back(a.slot);
      stats.particle_steps += out->r.particle_steps;
      stats.completed += 1;
      const uint64_t id = out->r.id;
      drop_requests.erase(id);  // a cancel that arrived after the request finished
      done_order.push_back(id);
      done[id] = std::move(out);
      done_signal.notify_all();
      wake.notify_one();  // the worker may admit into the freed room
    }
  } catch (const std::exception& e) {
    std::lock_guard<std::mutex> lock(mutex);
    failure = e.what();
    stopping = true;
    done_signal.notify_all();
  }
}

extern "C" {

int dpa_server_create(dpa_context* ctx, const dpa_server_options* options, dpa_server** out) {
  if (!ctx || !options || !out) return DPA_ERROR_INVALID_ARGUMENT;
  *out = nullptr;
  if (options->particle_capacity == 0 || options->max_requests == 0) {
    ctx->error = "server needs particle_capacity and max_requests";
    return DPA_ERROR_INVALID_ARGUMENT;
  }
  try {
    auto s = std::make_unique<dpa_server>();
    s->ctx = ctx;
    s->options = *options;
    s->tuning = ctx->tuning;
    if (cudaSetDevice(ctx->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
      ctx->error = "server: cannot create a stream";
      return DPA_ERROR_CUDA;
    }
    if (cudaStreamCreateWithFlags(&s->finish_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->upload_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->seeds_copied, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&s->readback[0]) != cudaSuccess ||
        cudaEventCreate(&s->readback[1]) != cudaSuccess ||
        cudaEventCreate(&s->tick_start[0]) != cudaSuccess ||
        cudaEventCreate(&s->tick_start[1]) != cudaSuccess) {
      s->destroy_streams();
      ctx->error = "server: cannot create a stream";
      return DPA_ERROR_CUDA;
    }
    const uint64_t p = options->particle_capacity, v = options->vertex_capacity;
    cudaError_t e = cudaSuccess;
    DeviceBuffer* per_slot[] = {&s->positions, &s->times, &s->remaining, &s->remaining_initial,
                                &s->termination, &s->raw_offsets, &s->kept_vertices,
                                &s->kept_segments, &s->curve_open, &s->request_of,
                                &s->seed_order, &s->order_ids};
    const size_t bytes[] = {12, 4, 8, 8, 1, 8, 4, 4, 1, 4, 4, 4};
    for (size_t i = 0; i < 12 && e == cudaSuccess; ++i) e = per_slot[i]->reserve(p * bytes[i]);
    if (e == cudaSuccess) e = s->order_counts.reserve(dpa::kOrderCountsSize * 4);
    if (e == cudaSuccess) e = s->raw.reserve(std::max<uint64_t>(v, 1) * 12);
    if (e == cudaSuccess) e = s->in_flight.reserve(4 * uint64_t(options->max_requests));
    if (e == cudaSuccess) e = s->work_counter.reserve(8);
    const uint64_t response_bytes =
        (options->response_bytes ? options->response_bytes : (256ull << 20)) / kResponseUnit *
        kResponseUnit;
    if (e == cudaSuccess) e = s->response_arena.reserve(response_bytes);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(s->in_flight.ptr, 0, 4 * uint64_t(options->max_requests), s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) {
      s->destroy_streams();
      ctx->error = std::string("server: device arenas: ") + cudaGetErrorName(e);
      return e == cudaErrorMemoryAllocation ? DPA_ERROR_OUT_OF_MEMORY : DPA_ERROR_CUDA;
    }
    s->fields.reserve(kMaxServerFields);
    s->slots.reset(p);
    s->vertices.reset(v);
    s->response_units.reset(response_bytes / kResponseUnit);
    s->admission.slot_capacity = p;
    s->admission.small_seeds = options->small_request_seeds ? options->small_request_seeds : 65536;
    s->admission.reserved_slots = p / 100 * std::min<uint32_t>(options->reserved_percent, 90);
    s->admission.max_bypass_seconds =
        1e-3 * double(options->max_bypass_ms ? options->max_bypass_ms : 250);
    for (uint32_t i = options->max_requests; i-- > 0;) s->free_counters.push_back(i);
    dpa_server* raw_ptr = s.get();
    s->worker = std::thread([raw_ptr] { raw_ptr->run(); });
    s->finisher = std::thread([raw_ptr] { raw_ptr->run_finisher(); });
    *out = s.release();
    return DPA_OK;
  } catch (const std::exception& e) {
    ctx->error = e.what();
    return DPA_ERROR_INTERNAL;
  }
}

int dpa_server_add_field(dpa_server* s, const dpa_field* field, int32_t* id) {
  if (!s || !field || !id || field->owner != s->ctx) return DPA_ERROR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mutex);
  // The worker and the finisher read fields[] without the lock: the vector
  // never reallocates (its capacity is reserved at creation).
  if (s->fields.size() == s->fields.capacity()) {
    s->ctx->error = "server: at most " + std::to_string(kMaxServerFields) + " fields";
    return DPA_ERROR_INVALID_ARGUMENT;
  }
  s->fields.push_back(field);
  *id = int32_t(s->fields.size() - 1);
  return DPA_OK;
}

int dpa_server_submit(dpa_server* s, const dpa_request* request, uint64_t* id) {
  if (!s || !request || !id) return DPA_ERROR_INVALID_ARGUMENT;
  const dpa_request& q = *request;
  {
    std::lock_guard<std::mutex> lock(s->mutex);
    if (q.field < 0 || size_t(q.field) >= s->fields.size()) return DPA_ERROR_INVALID_ARGUMENT;
  }
  if (!integrator_ok(q.integrator)) return DPA_ERROR_UNSUPPORTED;
  if (q.count && !q.positions) return DPA_ERROR_INVALID_ARGUMENT;
  // The range checks come first: they bound count * (iterations + 2) below 2^64.
  if (q.count > 0xffffffffull) return DPA_ERROR_INVALID_ARGUMENT;
  if (q.record && q.iterations > 0xfffffff0ull) return DPA_ERROR_INVALID_ARGUMENT;
  if (q.count > s->options.particle_capacity) return DPA_ERROR_OUT_OF_MEMORY;
  if (q.record && q.count * (q.iterations + 2) > s->options.vertex_capacity)
    return DPA_ERROR_OUT_OF_MEMORY;
  try {
    pending p;
    p.request = q;
    p.positions.assign(q.positions, q.positions + 3 * q.count);
    std::lock_guard<std::mutex> lock(s->mutex);
    if (!s->failure.empty() || s->stopping) return DPA_ERROR_INTERNAL;
    p.id = s->next_id++;
    p.queued = s->now();
    p.deadline = q.deadline_ms ? p.queued + 1e-3 * double(q.deadline_ms) : 0.0;
    *id = p.id;
    s->queue.push_back(std::move(p));
    s->stats.submitted += 1;
  } catch (const std::bad_alloc&) {
    return DPA_ERROR_OUT_OF_MEMORY;
  }
  s->wake.notify_one();
  return DPA_OK;
}

int dpa_server_poll(dpa_server* s, int32_t wait_ms, dpa_response* out, int32_t* got) {
  if (!s || !out || !got) return DPA_ERROR_INVALID_ARGUMENT;
  *got = 0;
  std::unique_lock<std::mutex> lock(s->mutex);
  const auto ready = [&] { return !s->done_order.empty() || !s->failure.empty(); };
  if (wait_ms > 0) s->done_signal.wait_for(lock, std::chrono::milliseconds(wait_ms), ready);
  if (s->done_order.empty()) {
    if (!s->failure.empty()) {
      s->ctx->error = "server: " + s->failure;
      return DPA_ERROR_CUDA;
    }
    return DPA_OK;
  }
  const uint64_t id = s->done_order.front();
  s->done_order.pop_front();
  auto it = s->done.find(id);
  *out = it->second->r;
  s->handed_out[id] = std::move(it->second);
  s->done.erase(it);
  *got = 1;
  return DPA_OK;
}

int dpa_server_cancel(dpa_server* s, uint64_t id) {
  if (!s) return DPA_ERROR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(s->mutex);
    bool known = false;
    for (const pending& p : s->queue) known = known || p.id == id;
    for (const active_request& a : s->active) known = known || a.p.id == id;
    if (!known) return DPA_ERROR_INVALID_ARGUMENT;  // unknown, finishing or finished
    s->drop_requests[id] = DPA_ERROR_CANCELLED;
  }
  s->wake.notify_one();
  return DPA_OK;
}

int dpa_server_release(dpa_server* s, uint64_t id) {
  if (!s) return DPA_ERROR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mutex);
  const auto it = s->handed_out.find(id);
  if (it == s->handed_out.end()) return DPA_ERROR_INVALID_ARGUMENT;
  if (it->second->arena_offset != ~0ull)
    s->response_units.release(it->second->arena_offset, it->second->arena_units);
  s->handed_out.erase(it);
  return DPA_OK;
}

int dpa_server_get_stats(dpa_server* s, dpa_server_stats* out) {
  if (!s || !out) return DPA_ERROR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mutex);
  *out = s->stats;
  out->queued = uint32_t(s->queue.size());
  out->active = uint32_t(s->active.size());
  return DPA_OK;
}

int dpa_server_destroy(dpa_server* s) {
  if (!s) return DPA_ERROR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(s->mutex);
    s->stopping = true;
  }
  s->wake.notify_all();
  if (s->worker.joinable()) s->worker.join();
  if (s->finisher.joinable()) s->finisher.join();
  cudaSetDevice(s->ctx->device);
  s->destroy_streams();
  delete s;
  return DPA_OK;
}

}  // extern "C"
