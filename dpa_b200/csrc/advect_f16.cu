// advect_f16.cu -- the advection kernels of F16 fields, steady and time-varying
// (a compile split: each storage's instantiations build in parallel).
#include "advect_kernel.cuh"

namespace dpa {
template cudaError_t launch_advect_storage<DPA_STORAGE_F16, false>(const FieldView&, const AdvectArgs&,
                                                                   int, bool, cudaStream_t);
template cudaError_t launch_advect_storage<DPA_STORAGE_F16, true>(const FieldView&, const AdvectArgs&,
                                                                  int, bool, cudaStream_t);
}  // namespace dpa
