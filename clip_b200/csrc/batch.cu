// Batched 2D cases (C ABI in include/clipb.h): many independent small cases advanced by one
// persistent launch per time step (step2d_batch_kernel), replayed from a CUDA graph.  Each
// case is an ordinary solver (its own buffers, geometry and physics); the batch keeps a
// device table of every case's step arguments for both buffer parities and a list of work
// items (case, tile, row segment) built for the current launch shape.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "clipb.h"
#include "config.hpp"
#include "engine.hpp"
#include "solver.hpp"

using namespace clipb;

struct clipb_batch {
    int precision = CLIPB_FP32;
    std::vector<clipb_solver*> cases;  // owned
    KernelTable kt{};
    cudaStream_t stream = nullptr;
    void* d_args[2] = {nullptr, nullptr};  // StepArgs of every case, input parity 0 / 1
    int* d_items = nullptr;
    int nitems = 0;
    int variant = 0, seg = 8, blocks_per_sm = 0;
    long long steps = 0;
    bool initialized = false;
    static constexpr int kGraphSteps = 16;
    cudaGraphExec_t graph = nullptr;
    bool use_graphs = true;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double* d_mon = nullptr;  // 3 doubles per case
    std::vector<double> h_mon;

    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }
    ~clipb_batch() {
        if (stream) cudaStreamSynchronize(stream);
        drop_graph();
        for (auto* c : cases) clipb_destroy(c);
        for (void* p : d_args) cudaFree(p);
        cudaFree(d_items);
        cudaFree(d_mon);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// Work items (case, tile bx, row segment by) for a tile width and segment length, case by
// case so that CTAs running at the same time work on neighbouring tiles of one case.
int build_items(clipb_batch* b) {
    const int TX = b->kt.tile2(b->variant);
    std::vector<int> items;
    for (size_t c = 0; c < b->cases.size(); ++c) {
        const Geom& g = b->cases[c]->st.g;
        const int nbx = (g.n[0] + TX - 1) / TX, nby = (g.n[1] + b->seg - 1) / b->seg;
        for (int by = 0; by < nby; ++by)
            for (int bx = 0; bx < nbx; ++bx) {
                items.push_back((int)c);
                items.push_back(bx);
                items.push_back(by);
            }
    }
    CLIPB_CUDA(cudaStreamSynchronize(b->stream));
    cudaFree(b->d_items);
    b->d_items = nullptr;
    CLIPB_CUDA(cudaMalloc((void**)&b->d_items, items.size() * sizeof(int)));
    CLIPB_CUDA(cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(int), cudaMemcpyHostToDevice));
    b->nitems = (int)(items.size() / 3);
    return CLIPB_OK;
}

int launch_batched(clipb_batch* b) {
    CLIPB_CUDA(b->kt.step2_batch(b->d_args[b->steps & 1], b->d_items, b->nitems, b->variant, b->seg,
                                 b->blocks_per_sm, b->stream));
    ++b->steps;
    for (auto* c : b->cases) ++c->steps;
    return CLIPB_OK;
}

int build_graph(clipb_batch* b) {
    cudaGraph_t g = nullptr;
    CLIPB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < clipb_batch::kGraphSteps; ++i) {
        const cudaError_t e =
            b->kt.step2_batch(b->d_args[i & 1], b->d_items, b->nitems, b->variant, b->seg, b->blocks_per_sm, b->stream);
        if (e != cudaSuccess) {
            cudaStreamEndCapture(b->stream, &g);
            if (g) cudaGraphDestroy(g);
            return fail(CLIPB_E_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(e));
        }
    }
    CLIPB_CUDA(cudaStreamEndCapture(b->stream, &g));
    const cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(CLIPB_E_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return CLIPB_OK;
}

// Uniform double in [0, 1) from the top 53 bits of one generator output.
double unit(std::mt19937_64& rng) { return (double)(rng() >> 11) * (1.0 / 9007199254740992.0); }

std::string seeded_config(uint64_t seed, int index) {
    std::mt19937_64 rng(seed);
    int nx = 0, ny = 0;
    double we = 0, re = 0, rho = 0;
    for (int i = 0; i <= index; ++i) {  // five draws per case, in this order
        nx = 32 * (1 + (int)(rng() % 8));         // 32 .. 256
        ny = 64 + 32 * (int)(rng() % 15);         // 64 .. 512
        we = 1.0 + 19.0 * unit(rng);              // U[1, 20]
        re = 50.0 + 450.0 * unit(rng);            // U[50, 500]
        rho = std::exp(std::log(10.0) + unit(rng) * (std::log(1000.0) - std::log(10.0)));  // log-uniform
    }
    const double R = 0.2 * std::min(nx, ny);
    char buf[2048];
    std::snprintf(buf, sizeof(buf),
                  "case = %s\n\nfinalStep = 5000\noutputInterval = 5000\nreportInterval = 5000\n\n"
                  "N = [%d, %d, 1]\nreferenceLength = %.17g\nWe = %.17g\nRe = %.17g\n"
                  "gravity = [0, -1e-06, 0]\nmobility = 0.02\ninterfaceWidth = 4\nmuRatio = %.17g\nrhoRatio = %.17g\n\n"
                  "geometry = [\n  {\n    type = \"circle\"\n    center = [%.17g, %.17g, 0]\n    radius = %.17g\n    id = 0\n  }\n]\n\n"
                  "boundary = [\n  {\n    side = \"x-\"\n    type = \"periodic\"\n  },\n  {\n    side = \"x+\"\n"
                  "    type = \"periodic\"\n  },\n  {\n    side = \"y-\"\n    type = \"wall\"\n  },\n  {\n"
                  "    side = \"y+\"\n    type = \"wall\"\n  },\n]\n",
                  index % 2 == 0 ? "drop" : "bubble", nx, ny, 2.0 * R, we, re, rho / 10.0, rho, nx / 2.0 + 0.5,
                  ny / 2.0 + 0.5, R);
    return buf;
}

}  // namespace

extern "C" {

int clipb_seeded_case_config(unsigned long long seed, int index, char* buf, size_t len) {
    if (index < 0) return fail(CLIPB_E_ARG, "negative case index");
    const std::string t = seeded_config(seed, index);
    if (buf && len > 0) {
        const size_t n = std::min(len - 1, t.size());
        std::memcpy(buf, t.data(), n);
        buf[n] = '\0';
    }
    return (int)t.size();
}

int clipb_batch_create(const char* const* configs, int ncases, int kind, int precision, clipb_batch** out) {
    if (!configs || !out || ncases < 1) return fail(CLIPB_E_ARG, "need a non-empty list of configs");
    if (kind != CLIPB_CONFIG_PATH && kind != CLIPB_CONFIG_TEXT) return fail(CLIPB_E_ARG, "unknown config kind");
    *out = nullptr;
    std::unique_ptr<clipb_batch> b(new clipb_batch());
    b->precision = precision;
    CLIPB_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    for (int i = 0; i < ncases; ++i) {
        if (!configs[i]) return fail(CLIPB_E_ARG, "null config " + std::to_string(i));
        CaseConfig cfg;
        try {
            cfg = kind == CLIPB_CONFIG_PATH ? load_config(configs[i])
                                            : load_config_text(configs[i], "case " + std::to_string(i));
        } catch (const std::exception& e) {
            return fail(CLIPB_E_CONFIG, "case " + std::to_string(i) + ": " + e.what());
        }
        if (cfg.dim != 2) return fail(CLIPB_E_CONFIG, "case " + std::to_string(i) + ": batches hold 2D cases");
        for (int sd = 0; sd < 4; ++sd)
            if (cfg.bc.type[sd] == kVelocity || cfg.bc.type[sd] == kFreeConvect || cfg.bc.type[sd] == kNeumann)
                return fail(CLIPB_E_CONFIG, "case " + std::to_string(i) +
                                                ": batched cases take wall, slip-wall and periodic sides");
        clipb_solver* s = nullptr;
        const int rc = solver_create(cfg, precision, &s);
        if (rc) return fail(rc, "case " + std::to_string(i) + ": " + clipb_last_error());
        b->cases.push_back(s);
        CLIPB_CUDA(cudaStreamSynchronize(s->stream));
        s->stream = b->stream;  // every case runs on the batch's stream
    }
    b->kt = b->cases[0]->kt;
    // step arguments of every case for both buffer parities
    const size_t ab = b->kt.args_bytes;
    std::vector<unsigned char> host(ab * ncases);
    for (int p = 0; p < 2; ++p) {
        for (int i = 0; i < ncases; ++i) b->kt.make_args(b->cases[i]->st, p, host.data() + ab * i);
        CLIPB_CUDA(cudaMalloc(&b->d_args[p], host.size()));
        CLIPB_CUDA(cudaMemcpy(b->d_args[p], host.data(), host.size(), cudaMemcpyHostToDevice));
    }
    CLIPB_CUDA(cudaMalloc((void**)&b->d_mon, 3 * sizeof(double) * ncases));
    b->h_mon.resize(3 * (size_t)ncases);
    CLIPB_CUDA(cudaEventCreate(&b->ev0));
    CLIPB_CUDA(cudaEventCreate(&b->ev1));
    int rc = build_items(b.get());
    if (rc) return rc;
    *out = b.release();
    return CLIPB_OK;
}

void clipb_batch_destroy(clipb_batch* b) { delete b; }

int clipb_batch_size(const clipb_batch* b) { return b ? (int)b->cases.size() : 0; }

int clipb_batch_case(clipb_batch* b, int index, clipb_solver** out) {
    if (!b || !out) return fail(CLIPB_E_ARG, "null argument");
    if (index < 0 || index >= (int)b->cases.size()) return fail(CLIPB_E_ARG, "case index out of range");
    *out = b->cases[index];
    return CLIPB_OK;
}

int clipb_batch_init(clipb_batch* b) {
    if (!b) return fail(CLIPB_E_ARG, "null batch");
    CLIPB_CUDA(cudaStreamSynchronize(b->stream));
    for (auto* c : b->cases) {
        const int rc = clipb_init(c);
        if (rc) return rc;
    }
    b->steps = 0;
    b->initialized = true;
    return CLIPB_OK;
}

int clipb_batch_solve(clipb_batch* b, int nsteps) {
    if (!b) return fail(CLIPB_E_ARG, "null batch");
    if (!b->initialized) return fail(CLIPB_E_STATE, "solve before init");
    if (nsteps < 0) return fail(CLIPB_E_ARG, "negative step count");
    int rc;
    long long left = nsteps;
    const int G = clipb_batch::kGraphSteps;
    if (b->use_graphs && left > G) {
        if (b->steps & 1) {  // the graph starts on an even step
            if ((rc = launch_batched(b))) return rc;
            --left;
        }
        if (!b->graph && (rc = build_graph(b))) return rc;
        for (; left >= G; left -= G) {
            CLIPB_CUDA(cudaGraphLaunch(b->graph, b->stream));
            b->steps += G;
            for (auto* c : b->cases) c->steps += G;
        }
    }
    for (; left > 0; --left)
        if ((rc = launch_batched(b))) return rc;
    return CLIPB_OK;
}

int clipb_batch_solve_sequential(clipb_batch* b, int nsteps) {
    if (!b) return fail(CLIPB_E_ARG, "null batch");
    if (!b->initialized) return fail(CLIPB_E_STATE, "solve before init");
    if (nsteps < 0) return fail(CLIPB_E_ARG, "negative step count");
    for (int k = 0; k < nsteps; ++k) {
        for (auto* c : b->cases) {
            const int rc = solver_launch_one(c);
            if (rc) return rc;
        }
        ++b->steps;
    }
    return CLIPB_OK;
}

int clipb_batch_set_launch(clipb_batch* b, int variant, int seg, int blocks_per_sm) {
    if (!b) return fail(CLIPB_E_ARG, "null batch");
    if (variant < 0 || variant >= b->kt.variants2 || !b->kt.available(b->cases[0]->st, variant))
        return fail(CLIPB_E_ARG, "variant must be in [0, " + std::to_string(b->kt.variants2) + ")");
    if (seg < 1) return fail(CLIPB_E_ARG, "rows per work item must be positive");
    if (blocks_per_sm < 0) return fail(CLIPB_E_ARG, "negative blocks per SM");
    CLIPB_CUDA(cudaStreamSynchronize(b->stream));
    b->drop_graph();
    b->variant = variant;
    b->seg = seg;
    b->blocks_per_sm = blocks_per_sm;
    return build_items(b);
}

int clipb_batch_get_launch(const clipb_batch* b, int* variant, int* seg, int* blocks_per_sm, int* nitems) {
    if (!b) return fail(CLIPB_E_ARG, "null batch");
    if (variant) *variant = b->variant;
    if (seg) *seg = b->seg;
    if (blocks_per_sm) *blocks_per_sm = b->blocks_per_sm;
    if (nitems) *nitems = b->nitems;
    return CLIPB_OK;
}

int clipb_batch_set_graphs(clipb_batch* b, int enable) {
    if (!b) return fail(CLIPB_E_ARG, "null batch");
    b->use_graphs = enable != 0;
    if (!b->use_graphs) b->drop_graph();
    return CLIPB_OK;
}

int clipb_batch_time_steps(clipb_batch* b, int nsteps, int sequential, float* ms) {
    if (!b || !ms) return fail(CLIPB_E_ARG, "null argument");
    // a graph the steps will replay is captured before the first event, not timed
    if (!sequential && b->initialized && b->use_graphs && nsteps > clipb_batch::kGraphSteps && !b->graph) {
        const int rc = build_graph(b);
        if (rc) return rc;
    }
    CLIPB_CUDA(cudaEventRecord(b->ev0, b->stream));
    const int rc = sequential ? clipb_batch_solve_sequential(b, nsteps) : clipb_batch_solve(b, nsteps);
    if (rc) return rc;
    CLIPB_CUDA(cudaEventRecord(b->ev1, b->stream));
    CLIPB_CUDA(cudaEventSynchronize(b->ev1));
    CLIPB_CUDA(cudaEventElapsedTime(ms, b->ev0, b->ev1));
    return CLIPB_OK;
}

// Time every tile width, rows per work item and persistent-grid size on the batch's own
// freshly initialised state, keep the fastest and rebuild the initial state.
int clipb_batch_autotune(clipb_batch* b, int trial_steps, int* best_variant, int* best_seg, int* best_bps,
                         float* best_ms) {
    if (!b) return fail(CLIPB_E_ARG, "null batch");
    if (!b->initialized || b->steps != 0) return fail(CLIPB_E_STATE, "autotune needs a freshly initialised batch");
    if (trial_steps < 1) trial_steps = 4;
    const bool graphs = b->use_graphs;
    b->use_graphs = false;
    float best = 1e30f;
    int bv = b->variant, bs = b->seg, bb = b->blocks_per_sm, rc;
    for (int v = 0; v < b->kt.variants2; ++v) {
        if (!b->kt.available(b->cases[0]->st, v)) continue;
        for (int seg : {4, 8, 16, 32, 64})
            for (int bps : {1, 2, 0}) {
                if ((rc = clipb_batch_set_launch(b, v, seg, bps))) return rc;
                if ((rc = clipb_batch_solve(b, 1))) return rc;  // warm-up
                float ms = 0.f;
                if ((rc = clipb_batch_time_steps(b, trial_steps, 0, &ms))) return rc;
                if (ms < best) {
                    best = ms;
                    bv = v;
                    bs = seg;
                    bb = bps;
                }
            }
    }
    b->use_graphs = graphs;
    if ((rc = clipb_batch_set_launch(b, bv, bs, bb))) return rc;
    for (auto* c : b->cases) {
        CLIPB_CUDA(c->kt.init(c->st, b->stream));
        c->steps = 0;
    }
    CLIPB_CUDA(cudaStreamSynchronize(b->stream));
    b->steps = 0;
    if (best_variant) *best_variant = bv;
    if (best_seg) *best_seg = bs;
    if (best_bps) *best_bps = bb;
    if (best_ms) *best_ms = best / (float)trial_steps;
    return CLIPB_OK;
}

int clipb_batch_monitors(clipb_batch* b, double* mass, double* kinetic) {
    if (!b) return fail(CLIPB_E_ARG, "null batch");
    if (!b->initialized) return fail(CLIPB_E_STATE, "monitors before init");
    const size_t n = b->cases.size();
    for (size_t i = 0; i < n; ++i) {
        clipb_solver* c = b->cases[i];
        CLIPB_CUDA(c->kt.monitors(c->st, c->steps, b->d_mon + 3 * i, b->stream));
    }
    CLIPB_CUDA(cudaMemcpyAsync(b->h_mon.data(), b->d_mon, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    CLIPB_CUDA(cudaStreamSynchronize(b->stream));
    bool nan = false;
    for (size_t i = 0; i < n; ++i) {
        if (mass) mass[i] = b->h_mon[3 * i];
        if (kinetic) kinetic[i] = b->h_mon[3 * i + 1];
        nan = nan || std::isnan(b->h_mon[3 * i]) || std::isnan(b->h_mon[3 * i + 1]);
    }
    if (nan) return fail(CLIPB_E_DIVERGED, "Solver has diverged.");
    return CLIPB_OK;
}

}  // extern "C"
