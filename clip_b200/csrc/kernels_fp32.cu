// FP32 instantiation: f and g stored in FP32, g as the deviation g - w_q c; c and u stored
// in FP32; all arithmetic of the step in FP32 (lean_update; the stencils run on c as an
// unevaluated (stored, remainder) pair).
#include "launch.cuh"

namespace clipb {
using PrecFP32 = Prec<float, float, float, float, float, true>;
KernelTable kernels_fp32() { return Launch<PrecFP32, true, true>::table(); }
}  // namespace clipb
