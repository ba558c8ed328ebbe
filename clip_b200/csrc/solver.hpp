// Internal: the solver object behind the C ABI's clipb_solver handle, shared by the
// single-case entry points (capi.cu) and the batched ones (batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "clipb.h"
#include "config.hpp"
#include "engine.hpp"

namespace clipb {
// Record `msg` for clipb_last_error and return `code`.
int fail(int code, const std::string& msg);
// Background VTS writer of a solver (vts.cu): joins its thread after the pending writes.
struct VtsQueue;
void vts_release(VtsQueue* q);
// Device workspace of clipb_adjoint (adjoint_rev.cu), kept for later calls.
struct AdjWork;
void adj_release(AdjWork* w);
}  // namespace clipb

#define CLIPB_CUDA(call)                                                                                      \
    do {                                                                                                      \
        const cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return clipb::fail(CLIPB_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct clipb_solver {
    clipb::CaseConfig cfg;
    clipb::DevState st{};
    clipb::KernelTable kt{};
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    // Host array of doubles that is not zero-filled on allocation, so that the threads
    // writing it touch its pages first (in parallel).
    struct HostArray {
        std::unique_ptr<double[]> p;
        size_t n = 0;
        void alloc(size_t m) {
            if (m != n) p.reset(new double[m]);
            n = m;
        }
        double* data() { return p.get(); }
        const double* data() const { return p.get(); }
        size_t size() const { return n; }
        bool empty() const { return n == 0; }
    };
    HostArray host_c;  // reference layout, ghosted
    // Pinned staging of a large initial-field upload (device layout), kept for later uploads.
    double* h_stage = nullptr;
    size_t h_stage_elems = 0;
    // per-plane table of the uniform rows of a large upload (pinned host copy, device copy)
    void* h_plane_tab = nullptr;
    void* d_plane_tab = nullptr;
    size_t plane_tab_elems = 0;
    long long upload_bytes = 0;  // host-to-device bytes of the last initial-field upload
    double* mon_rows = nullptr;  // row-segment monitor partials of clipb_solve_monitored (2 per row)
    long long steps = 0;
    bool initialized = false;
    double* d_stage = nullptr;
    size_t stage_elems = 0;
    double* d_mon = nullptr;
    double* h_mon = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    size_t device_bytes = 0;
    std::vector<void*> allocations;
    // CUDA graph of kGraphSteps consecutive steps starting at an even step (launch
    // arguments depend only on the step's parity), replayed by clipb_solve.
    static constexpr int kGraphSteps = 16;
    cudaGraphExec_t graph = nullptr;
    bool use_graphs = true;
    clipb::VtsQueue* vts = nullptr;  // created by the first VTS write
    clipb::AdjWork* adjw = nullptr;  // created by the first clipb_adjoint
    bool slab_half = false;          // a slab step's first part ran (clipb_slab_step_part)
    size_t fc_bytes = 0;             // bytes of each parity's free-convect state (st.g.fc)

    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }

    long long ref_nodes() const { return (long long)cfg.extent[0] * cfg.extent[1] * cfg.extent[2]; }
    int ncomp(int field) const {
        switch (field) {
            case CLIPB_FIELD_C:
            case CLIPB_FIELD_P:
            case CLIPB_FIELD_RHO: return 1;
            case CLIPB_FIELD_VEL: return cfg.dim;
            default: return cfg.dim == 3 ? 19 : 9;
        }
    }
    // element index of reference node (i, j, k) in the device layout
    long long dev_index(int i, int j, int k) const { return st.g.base + i + (long long)j * st.g.sy + (long long)k * st.g.sz; }

    int alloc(void** p, size_t bytes) {
        const cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) return clipb::fail(CLIPB_E_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e));
        allocations.push_back(*p);
        device_bytes += bytes;
        CLIPB_CUDA(cudaMemsetAsync(*p, 0, bytes, stream));
        return 0;
    }

    ~clipb_solver() {
        if (stream) cudaStreamSynchronize(stream);
        clipb::vts_release(vts);
        clipb::adj_release(adjw);
        drop_graph();
        if (kt.release) kt.release(st);
        for (void* p : allocations) cudaFree(p);
        if (h_mon) cudaFreeHost(h_mon);
        if (h_stage) cudaFreeHost(h_stage);
        if (h_plane_tab) cudaFreeHost(h_plane_tab);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (own_stream) cudaStreamDestroy(own_stream);
    }
};


namespace clipb {
// clipb_create from an already parsed case.
int solver_create(const CaseConfig& cfg, int precision, clipb_solver** out);
// Launch step `steps` of one solver (velocity-inlet kernel if any, then the fused step)
// on its stream, without a CUDA graph, and advance its step count.
int solver_launch_one(clipb_solver* s);
}  // namespace clipb
