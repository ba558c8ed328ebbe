// FP16-storage instantiation: f stored as f * 2^k, g as (g - w_q c) * 256, both in FP16;
// c and u in FP32; arithmetic as in the FP32 instantiation.
#include "launch.cuh"

namespace clipb {
using PrecFP16 = Prec<__half, __half, float, float, float, true>;
KernelTable kernels_fp16() { return Launch<PrecFP16, true, true>::table(); }
}  // namespace clipb
