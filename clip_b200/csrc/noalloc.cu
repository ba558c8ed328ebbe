// Allocation-free variant of the mass / kinetic-energy reduction (clipb_monitors).
//
// Some callers cannot allocate device memory at the point where they need the monitors:
// code running under a memory pool or arena that owns the whole device, real-time loops
// that must not enter the CUDA allocator (cudaMalloc can synchronise the device and its
// latency is unbounded), or hosts that hand the library nothing but their own buffers.
// clipb_field_sums_noalloc serves them: it reads caller-owned device arrays, writes a
// caller-owned device result, and keeps its per-block partial sums in a fixed array in
// the library's own device image instead of a cudaMalloc'd buffer.  It calls no
// cudaMalloc, cudaFree or other allocating routine.
#include <cuda_runtime.h>

#include <string>

#include "clipb.h"

namespace clipb {
void set_last_error(const std::string& msg);  // capi.cu
}

namespace {

// Per-block partial sums (mass, kinetic) of one call.  Every GPU that loads the library
// holds this array (16 KiB) until the process exits.  All calls share it: each call writes
// the partials of the blocks it launches before reading them back, so nothing needs
// clearing, but calls whose kernels overlap on the GPU race on it.
constexpr int kMaxBlocks = 1024;
constexpr int kThreads = 256;
static __device__ __align__(256) double g_partials[2 * kMaxBlocks];

constexpr int kMaxDevices = 64;
double* g_partials_addr[kMaxDevices] = {};  // device address of g_partials, per device

__global__ void sums_partials(const double* __restrict__ c, const double* __restrict__ u, int dim, long long n,
                              double rho_l, double drho, double* partials) {
    double m = 0.0, ke = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double ci = c[i];
        double u2 = 0.0;
        for (int d = 0; d < dim; ++d) {
            const double v = u[d * n + i];
            u2 += v * v;
        }
        m += ci;
        ke += 0.5 * (rho_l + ci * drho) * u2;
    }
    for (int off = 16; off > 0; off >>= 1) {
        m += __shfl_down_sync(0xffffffffu, m, off);
        ke += __shfl_down_sync(0xffffffffu, ke, off);
    }
    __shared__ double sm[32], sk[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sm[warp] = m;
        sk[warp] = ke;
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        m = lane < nw ? sm[lane] : 0.0;
        ke = lane < nw ? sk[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) {
            m += __shfl_down_sync(0xffffffffu, m, off);
            ke += __shfl_down_sync(0xffffffffu, ke, off);
        }
        if (lane == 0) {
            partials[2 * blockIdx.x] = m;
            partials[2 * blockIdx.x + 1] = ke;
        }
    }
}

__global__ void sums_final(const double* __restrict__ partials, int nblocks, double* out2) {
    double m = 0.0, ke = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += 32) {
        m += partials[2 * i];
        ke += partials[2 * i + 1];
    }
    for (int off = 16; off > 0; off >>= 1) {
        m += __shfl_down_sync(0xffffffffu, m, off);
        ke += __shfl_down_sync(0xffffffffu, ke, off);
    }
    if (threadIdx.x == 0) {
        out2[0] = m;
        out2[1] = ke;
    }
}

int fail(int code, const std::string& msg) {
    clipb::set_last_error(msg);
    return code;
}

}  // namespace

extern "C" {

int clipb_field_sums_noalloc(const double* dev_c, const double* dev_u, int dim, long long n, double rho_l,
                             double drho, double* dev_out2, int nblocks, void* stream) {
    if (!dev_c || !dev_u || !dev_out2) return fail(CLIPB_E_ARG, "null device pointer");
    if (dim != 2 && dim != 3) return fail(CLIPB_E_ARG, "dim must be 2 or 3");
    if (n < 0) return fail(CLIPB_E_ARG, "negative node count");
    if (nblocks == 0) nblocks = 4 * 148;
    if (nblocks < 1 || nblocks > kMaxBlocks)
        return fail(CLIPB_E_ARG, "nblocks must be in [1, " + std::to_string(kMaxBlocks) +
                                     "]: the partial sums live in a fixed array of that many blocks");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(CLIPB_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(CLIPB_E_ARG, "device ordinal beyond the supported range");
    // First call on this device (with it current): look up the array's device address.
    if (!g_partials_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_partials);
        if (e != cudaSuccess) return fail(CLIPB_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_partials_addr[dev] = static_cast<double*>(p);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    sums_partials<<<nblocks, kThreads, 0, s>>>(dev_c, dev_u, dim, n, rho_l, drho, g_partials_addr[dev]);
    sums_final<<<1, 32, 0, s>>>(g_partials_addr[dev], nblocks, dev_out2);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(CLIPB_E_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return CLIPB_OK;
}

}  // extern "C"
