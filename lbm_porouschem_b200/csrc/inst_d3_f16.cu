// Launchers for D3Q19 + D3Q7 with FP16 deviation storage.
#include "launch.cuh"

namespace lbm {
namespace capi {

template int dispatch_batch<Lattice<3>, __half>(lbm_batch*, cudaStream_t);
template int dispatch_step<Lattice<3>, __half>(lbm_handle*, StepParams<__half>, cudaStream_t);
template int dispatch_init<Lattice<3>, __half>(lbm_handle*, StepParams<__half>, const float*, const float*, const float*,
                                     const float*, int, cudaStream_t);

}  // namespace capi
}  // namespace lbm
