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
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
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

// Per-device set-up: the device address of g_partials in the context that was current
// when it was looked up, and the default block count (4 per SM).  A context that is torn
// down and recreated (cudaDeviceReset in the caller) reloads the library's device image,
// possibly at another address, so the entry is keyed by the context's unique id and looked
// up again when that id changes.
constexpr int kMaxDevices = 64;
struct DeviceSetup {
    unsigned long long ctx_id = 0;  // 0: not set up
    double* partials = nullptr;
    int default_blocks = 0;
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the current context (0 if the driver cannot tell).
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(p);
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

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

std::string cuda_msg(const char* what, cudaError_t e) { return std::string(what) + ": " + cudaGetErrorString(e); }

// Set-up of the current device `dev` (with it current): look up g_partials' address and
// the SM count once per context.
int setup_device(int dev, DeviceSetup& out) {
    const unsigned long long id = current_context_id();
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup& d = g_setup[dev];
    if (d.ctx_id == 0 || id == 0 || d.ctx_id != id) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_partials);
        if (e != cudaSuccess) return fail(CLIPB_E_CUDA, cuda_msg("cudaGetSymbolAddress", e));
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return fail(CLIPB_E_CUDA, cuda_msg("cudaDeviceGetAttribute", e));
        d.partials = static_cast<double*>(p);
        d.default_blocks = sms > 0 ? (4 * sms < kMaxBlocks ? 4 * sms : kMaxBlocks) : kMaxBlocks;
        // without a context id (old driver) the address is looked up on every call
        d.ctx_id = id;
    }
    out = d;
    return CLIPB_OK;
}

}  // namespace

extern "C" {

int clipb_field_sums_noalloc(const double* dev_c, const double* dev_u, int dim, long long n, double rho_l,
                             double drho, double* dev_out2, int nblocks, void* stream) {
    if (!dev_c || !dev_u || !dev_out2) return fail(CLIPB_E_ARG, "null device pointer");
    if (dim != 2 && dim != 3) return fail(CLIPB_E_ARG, "dim must be 2 or 3");
    if (n < 0) return fail(CLIPB_E_ARG, "negative node count");
    if (nblocks < 0 || nblocks > kMaxBlocks)
        return fail(CLIPB_E_ARG, "nblocks must be in [1, " + std::to_string(kMaxBlocks) +
                                     "]: the partial sums live in a fixed array of that many blocks");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(CLIPB_E_CUDA, cuda_msg("cudaGetDevice", e));
    if (dev < 0 || dev >= kMaxDevices) return fail(CLIPB_E_ARG, "device ordinal beyond the supported range");
    DeviceSetup d;
    const int rc = setup_device(dev, d);
    if (rc) return rc;
    if (nblocks == 0) nblocks = d.default_blocks;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    sums_partials<<<nblocks, kThreads, 0, s>>>(dev_c, dev_u, dim, n, rho_l, drho, d.partials);
    sums_final<<<1, 32, 0, s>>>(d.partials, nblocks, dev_out2);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(CLIPB_E_CUDA, cuda_msg("launch", e));
    // divergence check of clipb_monitors (Reporter.cu:130-142): wait for the two sums
    double h[2];
    e = cudaMemcpyAsync(h, dev_out2, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(CLIPB_E_CUDA, cuda_msg("result read-back", e));
    if (std::isnan(h[0]) || std::isnan(h[1])) return fail(CLIPB_E_DIVERGED, "Solver has diverged.");
    return CLIPB_OK;
}

}  // extern "C"
