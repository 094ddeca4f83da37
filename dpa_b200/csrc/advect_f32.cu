// advect_f32.cu -- the advection kernels of F32 fields, steady and time-varying
// (a compile split: each storage's instantiations build in parallel).
#include "advect_kernel.cuh"

namespace dpa {
template cudaError_t launch_advect_storage<DPA_STORAGE_F32, false>(const FieldView&, const AdvectArgs&,
                                                                   int, bool, cudaStream_t);
template cudaError_t launch_advect_storage<DPA_STORAGE_F32, true>(const FieldView&, const AdvectArgs&,
                                                                  int, bool, cudaStream_t);
}  // namespace dpa
