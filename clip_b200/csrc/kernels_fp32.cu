// FP32 instantiation: f and g stored in FP32, g as the deviation g - w_q c; c and u stored
// in FP32; hydrodynamics (f, WMRT) in FP32 arithmetic, the phase field (c sums, stencils,
// g relaxation) in FP64 registers.
#include "launch.cuh"

namespace clipb {
using PrecFP32 = Prec<float, float, float, float, float, true>;
KernelTable kernels_fp32() { return Launch<PrecFP32, true, true>::table(); }
}  // namespace clipb
