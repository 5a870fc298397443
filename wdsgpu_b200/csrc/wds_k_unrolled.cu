// k_unrolled instances of one factor precision (WDS_FP32 = 0: FP64, 1: FP32);
// the reverse pass runs at most 3 scenario groups per CTA.
#include "wds_device.cuh"

namespace wds {
const void* WDS_KSEL(unrolled_kernel)(int wide, int groups) {
  if (wide) return (const void*)k_unrolled<256, 1, LTab, KFT>;
  switch (groups) {
    case 1: return (const void*)k_unrolled<256, 1, STab, KFT>;
    case 2: return (const void*)k_unrolled<256, 2, STab, KFT>;
    default: return (const void*)k_unrolled<256, 3, STab, KFT>;
  }
}
}  // namespace wds
