// checks.cuh -- failure reporting and argument checks shared by the C ABI's
// entry points (capi.cu, noalloc.cu), so that every advection entry point
// refuses the same inputs with the same messages.
#pragma once

#include <cmath>
#include <string>

#include "handles.cuh"

namespace dpa {

inline int fail(dpa_context* ctx, int status, const std::string& message) {
  if (ctx) ctx->error = message;
  return status;
}

inline int fail_cuda(dpa_context* ctx, cudaError_t e, const char* where) {
  const int status = (e == cudaErrorMemoryAllocation) ? DPA_ERROR_OUT_OF_MEMORY : DPA_ERROR_CUDA;
  return fail(ctx, status, std::string(where) + ": " + cudaGetErrorName(e) + " (" +
                               cudaGetErrorString(e) + ")");
}

inline int check_options(dpa_context* ctx, const dpa_advect_options* o) {
  if (!o) return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "options is NULL");
  switch (o->integrator) {
    case DPA_INTEGRATOR_EULER:
    case DPA_INTEGRATOR_RUNGE_KUTTA_4:
    case DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE:
    case DPA_INTEGRATOR_MODIFIED_MIDPOINT:
    case DPA_INTEGRATOR_RUNGE_KUTTA_CASH_KARP_54:
    case DPA_INTEGRATOR_RUNGE_KUTTA_DORMAND_PRINCE_5:
    case DPA_INTEGRATOR_RUNGE_KUTTA_FEHLBERG_78:
    case DPA_INTEGRATOR_ADAMS_BASHFORTH_2:
    case DPA_INTEGRATOR_ADAMS_BASHFORTH_MOULTON_2:
      break;
    default:
      return fail(ctx, DPA_ERROR_INVALID_ARGUMENT,
                  "unknown integrator " + std::to_string(o->integrator));
  }
  if (!std::isfinite(o->step_size))
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "step_size is not finite");
  if (o->record && o->max_steps)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT, "max_steps applies to calls without recording");
  if (o->max_steps && dpa::integrator_has_history(o->integrator))
    return fail(ctx, DPA_ERROR_UNSUPPORTED,
                "max_steps: this integrator carries a derivative from one step to the next, "
                "so a particle cannot resume in a later call");
  return DPA_OK;
}

// A time-varying field needs particle times, which only the pathline entry
// points (and the request server) carry.
inline int check_steady(dpa_context* ctx, const dpa_field* field) {
  if (field->slices > 1)
    return fail(ctx, DPA_ERROR_INVALID_ARGUMENT,
                "the field varies in time: advect it with dpa_advect_pathlines_device");
  return DPA_OK;
}

}  // namespace dpa
