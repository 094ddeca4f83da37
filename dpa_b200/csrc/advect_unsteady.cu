// advect_unsteady.cu -- advection launches over time-varying fields
// (pathlines): the kernel of advect_kernel.cuh with the two-slice sampler.
#include "advect_kernel.cuh"

namespace dpa {

cudaError_t launch_advect_unsteady(const FieldView& f, const AdvectArgs& a, int integrator,
                                   bool record, cudaStream_t stream) {
  return launch_family<true>(f, a, integrator, record, stream);
}

}  // namespace dpa
