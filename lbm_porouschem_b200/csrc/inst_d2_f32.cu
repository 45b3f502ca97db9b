// Launchers for D2Q9 + D2Q5 with FP32 storage.
#include "launch.cuh"

namespace lbm {
namespace capi {

template int dispatch_batch<Lattice<2>, float>(lbm_batch*, cudaStream_t);
template int dispatch_step<Lattice<2>, float>(lbm_handle*, StepParams<float>, cudaStream_t);
template int dispatch_init<Lattice<2>, float>(lbm_handle*, StepParams<float>, const float*, const float*, const float*,
                                     const float*, int, cudaStream_t);

}  // namespace capi
}  // namespace lbm
