// Multi-plan kernels (networks of different sizes in one launch) of one
// factor precision (WDS_FP32 = 0: FP64, 1: FP32).
#include "wds_device.cuh"

namespace wds {
const void* WDS_KSEL(forward_multi_kernel)() { return (const void*)k_forward_multi<KFT>; }
const void* WDS_KSEL(adjoint_multi_kernel)() { return (const void*)k_adjoint_multi<KFT>; }
}  // namespace wds
