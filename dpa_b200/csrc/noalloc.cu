// noalloc.cu -- dpa_advect_device_no_alloc: the device advection entry point
// for callers that must not allocate device memory once they are running.
//
// Who needs it: a host program whose device memory is reserved up front by
// another owner (a framework's caching allocator, or a service that fixes its
// HBM budget at start-up) cannot count on a cudaMalloc succeeding later, and a
// latency-bound loop cannot afford one: cudaMalloc and cudaFree may
// synchronize the whole device and so stall work queued on other streams.
// dpa_advect_device grows its ordering scratch with cudaMalloc; this variant
// takes it from a fixed array compiled into the library instead.
//
// The array below is a file-scope __device__ array of kScratchBytes (about
// 9 MiB). Every GPU on which the library's code is loaded holds its own copy
// until the process exits. Host code cannot use the name g_scratch as a device
// address (on the host it names a host-side stand-in), so the device address
// is looked up once per device with cudaGetSymbolAddress, with that device
// current, and handed to the kernels.
#include <mutex>

#include "checks.cuh"
#include "handles.cuh"
#include "kernels.cuh"

namespace {

constexpr uint64_t kMaxParticles = DPA_NO_ALLOC_MAX_PARTICLES;
constexpr size_t kAlign = 256;
constexpr size_t round_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

// Scratch layout: the advection kernel's work counter, the bucket counters,
// the processing order, the per-particle bucket ids.
constexpr size_t kCounterOffset = 0;
constexpr size_t kCountsOffset = kAlign;
constexpr size_t kOrderOffset =
    kCountsOffset + round_up(size_t(dpa::kOrderCountsSize) * sizeof(uint32_t));
constexpr size_t kBucketsOffset = kOrderOffset + round_up(kMaxParticles * sizeof(uint32_t));
constexpr size_t kScratchBytes = kBucketsOffset + round_up(kMaxParticles * sizeof(uint32_t));

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_lock;
void* g_device_address[kMaxDevices] = {};

// Device address of g_scratch on `device`, which must be current. The first
// call per device resolves it (and, with lazy module loading, loads this
// file's module on that device); later calls return the cached address.
cudaError_t scratch_on(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> guard(g_lock);
  if (!g_device_address[device]) {
    void* address = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&address, g_scratch);
    if (e != cudaSuccess) return e;
    g_device_address[device] = address;
  }
  *out = static_cast<unsigned char*>(g_device_address[device]);
  return cudaSuccess;
}

}  // namespace

extern "C" int dpa_advect_device_no_alloc(dpa_context* ctx, const dpa_field* field,
                                          const dpa_advect_options* options, uint64_t count,
                                          float* device_positions, uint64_t* device_remaining,
                                          uint8_t* device_termination, void* stream) {
  if (!ctx) return DPA_ERROR_INVALID_ARGUMENT;
  try {
    // The same checks, in the same order, as dpa_advect_device.
    int st = dpa::check_options(ctx, options);
    if (st != DPA_OK) return st;
    if (options->record)
      return dpa::fail(ctx, DPA_ERROR_INVALID_ARGUMENT,
                       "dpa_advect_device_no_alloc does not record; use dpa_advect_round");
    if (!field || field->owner != ctx) return dpa::fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "bad field");
    if (count && (!device_positions || !device_remaining))
      return dpa::fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "positions or remaining is NULL");
    st = dpa::check_steady(ctx, field);
    if (st != DPA_OK) return st;
    if (count > kMaxParticles)
      return dpa::fail(ctx, DPA_ERROR_INVALID_ARGUMENT,
                       "dpa_advect_device_no_alloc: count exceeds DPA_NO_ALLOC_MAX_PARTICLES "
                       "(1048576); split the particles or use dpa_advect_device");
    if (count == 0) return DPA_OK;

    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return dpa::fail_cuda(ctx, e, "cudaSetDevice");
    unsigned char* scratch = nullptr;
    e = scratch_on(ctx->device, &scratch);
    if (e != cudaSuccess) return dpa::fail_cuda(ctx, e, "cudaGetSymbolAddress");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;

    // The context's tuning applies as it does to dpa_advect_device: launch
    // shape, claims and processing order (resolution, or input order when 0).
    if (ctx->profiling) {
      e = cudaEventRecord(ctx->events[0], s);
      if (e != cudaSuccess) return dpa::fail_cuda(ctx, e, "cudaEventRecord");
    }
    const uint32_t* order = nullptr;
    if (options->morton_order && ctx->tuning.order && count >= dpa::kOrderMinParticles) {
      // launch_order starts by zeroing the counters, so what an earlier call
      // left in the shared array does not matter.
      uint32_t* counts = reinterpret_cast<uint32_t*>(scratch + kCountsOffset);
      uint32_t* order_out = reinterpret_cast<uint32_t*>(scratch + kOrderOffset);
      uint32_t* buckets = reinterpret_cast<uint32_t*>(scratch + kBucketsOffset);
      e = dpa::launch_order(field->view, device_positions, count, buckets, counts, order_out, s,
                            ctx->tuning.order);
      if (e != cudaSuccess) return dpa::fail_cuda(ctx, e, "ordering kernels");
      ctx->launches += dpa::kOrderLaunches;
      order = order_out;
    }
    if (ctx->profiling) {
      e = cudaEventRecord(ctx->events[1], s);
      if (e != cudaSuccess) return dpa::fail_cuda(ctx, e, "cudaEventRecord");
    }
    dpa::AdvectArgs a{};
    dpa::set_launch_defaults(a);
    if (options->max_steps) a.max_steps = options->max_steps;
    dpa::apply_tuning(ctx->tuning, a);
    // launch_advect zeroes the work counter before the kernel starts.
    a.work_counter = reinterpret_cast<unsigned long long*>(scratch + kCounterOffset);
    a.count = count;
    a.order = order;
    a.positions = device_positions;
    a.remaining = device_remaining;
    a.termination = device_termination;
    a.coefficients = dpa::make_step_coefficients(options->integrator, options->step_size);
    e = dpa::launch_advect(field->view, a, options->integrator, false, s);
    if (e != cudaSuccess) return dpa::fail_cuda(ctx, e, "advection kernel");
    ctx->launches += 1;
    if (ctx->profiling) {
      e = cudaEventRecord(ctx->events[2], s);
      if (e != cudaSuccess) return dpa::fail_cuda(ctx, e, "cudaEventRecord");
      ctx->timed_order = true;
    }
    return DPA_OK;
  } catch (...) {
    return dpa::fail(ctx, DPA_ERROR_INTERNAL, "unexpected exception");
  }
}
