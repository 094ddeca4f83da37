// advect_f32e.cu -- the advection kernels of F32 edge-record fields, steady
// and time-varying (a compile split: each storage's instantiations build in
// parallel).
#include "advect_kernel.cuh"

namespace dpa {
template cudaError_t launch_advect_storage<DPA_STORAGE_F32_EDGES, false>(const FieldView&,
                                                                         const AdvectArgs&, int,
                                                                         bool, cudaStream_t);
template cudaError_t launch_advect_storage<DPA_STORAGE_F32_EDGES, true>(const FieldView&,
                                                                        const AdvectArgs&, int,
                                                                        bool, cudaStream_t);
}  // namespace dpa
