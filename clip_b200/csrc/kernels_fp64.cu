// FP64 instantiation (parity path): every array and every operation in FP64.  Compiled
// with -fmad=false so that each product and sum is rounded separately, which matches the
// CPU oracle and the reference built without FMA contraction bit for bit.
#include "launch.cuh"

namespace clipb {
using PrecFP64 = Prec<double, double, double, double, double, false>;
KernelTable kernels_fp64() { return Launch<PrecFP64, false, false>::table(); }
}  // namespace clipb
