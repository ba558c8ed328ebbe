// FP64 instantiation (parity path): every array and every operation in FP64.  Compiled
// with -fmad=false so that each product and sum is rounded separately, which matches the
// CPU oracle and the reference built without FMA contraction bit for bit.
#include "launch.cuh"

namespace clipb {
using PrecFP64 = Prec<double, double, double, double, double, false>;
KernelTable kernels_fp64() { return Launch<PrecFP64, false, false>::table(); }

// NSAllen::initialCondition (NsAllen.cu:768-824) on the device: c = 1/2 +- 1/2 tanh(2 sdf / W)
// at every node of the ghosted extent (a z slab at its global z), written into the
// device-layout initial field c0.  Products and sums round one at a time (this unit is
// compiled without FMA contraction), like the host evaluation; tanh is CUDA's, so values
// can differ from the host's (the C library's tanh) in the last bits.
__global__ void initial_condition_kernel(Geom g, GeometryTable geo, int case_type, double W, int zoff,
                                         double* __restrict__ c0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = (int)blockIdx.z;
    if (i >= g.e[0] || j >= g.e[1]) return;
    const double x = (double)i, y = (double)j, z = g.dim == 3 ? (double)(k + zoff) : 0.0;
    const double sd = signed_distance(geo, 0, x, y, z, g.dim);
    double v;
    if (case_type == kBubble) v = 0.50 + 0.50 * tanh(2.0 * sd / W);
    else if (case_type == kDrop || case_type == kJet) v = 0.50 - 0.50 * tanh(2.0 * sd / W);
    else if (case_type == kRTI) v = 0.5 + 0.5 * tanh(2.0 * sd / W);
    else v = 0.0;
    c0[g.base + i + (long long)j * g.sy + (long long)k * g.sz] = v;
}

cudaError_t launch_initial_condition(const DevState& st, int case_type, double W, int zoff, cudaStream_t s) {
    const Geom& g = st.g;
    const dim3 b(32, 8, 1);
    const dim3 gr((g.e[0] + 31) / 32, (g.e[1] + 7) / 8, g.dim == 3 ? g.e[2] : 1);
    initial_condition_kernel<<<gr, b, 0, s>>>(g, st.geo, case_type, W, zoff, st.c0);
    return cudaGetLastError();
}
}  // namespace clipb
