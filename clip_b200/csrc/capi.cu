// C ABI of libclipb.so (declared in include/clipb.h): solver lifetime, host-side
// initial condition, device memory, launch sequencing and host/device transfers.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "clipb.h"
#include "config.hpp"
#include "engine.hpp"
#include "solver.hpp"

using namespace clipb;

namespace {

long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

// Host threads for the one-off host loops (initial condition, layout conversion).
template <class F>
// fn(i) for i in [0, n) on the host's threads, at least `grain` items per thread.
void host_parallel(long long n, F&& fn, long long grain = 4096) {
    const long long T = std::max<long long>(1, std::min<long long>(std::thread::hardware_concurrency(), n / grain));
    if (T <= 1) {
        for (long long i = 0; i < n; ++i) fn(i);
        return;
    }
    std::vector<std::thread> pool;
    for (long long t = 0; t < T; ++t)
        pool.emplace_back([&, t] {
            for (long long i = n * t / T; i < n * (t + 1) / T; ++i) fn(i);
        });
    for (auto& th : pool) th.join();
}

int side_code(int t) {
    switch (t) {
        case kPeriodic: return kSidePeriodic;
        case kVelocity: return kSideVelocity;
        case kFreeConvect: return kSideFreeConvect;
        case kNeumann: return kSideNeumann;
        case kExchange: return kSideExchange;
        case kWrap: return kSideWrap;
        default: return kSideWall;  // wall, and slip wall (bounced back like a wall)
    }
}

}  // namespace

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace clipb {
// Lets other translation units of the library report through clipb_last_error.
void set_last_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
}  // namespace clipb

int clipb::solver_create(const CaseConfig& cfg, int precision, clipb_solver** out) {
    *out = nullptr;
    if (precision < CLIPB_FP64 || precision > CLIPB_FP16) return fail(CLIPB_E_ARG, "unknown precision");
    std::unique_ptr<clipb_solver> s(new clipb_solver());
    s->cfg = cfg;
    const CaseConfig& c = s->cfg;
    int vel_sides = 0;
    for (int i = 0; i < 2 * c.dim; ++i) vel_sides += c.bc.type[i] == kVelocity;
    if (vel_sides > 1) return fail(CLIPB_E_CONFIG, "at most one velocity side is supported");

    int dev = 0;
    CLIPB_CUDA(cudaGetDevice(&dev));
    CLIPB_CUDA(cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking));
    s->stream = s->own_stream;

    DevState& st = s->st;
    st.precision = precision;
    Geom& g = st.g;
    g.dim = c.dim;
    for (int a = 0; a < 3; ++a) {
        g.n[a] = a < c.dim ? c.interior[a] : 1;
        g.e[a] = a < c.dim ? c.interior[a] + 2 : 1;
    }
    for (int i = 0; i < 6; ++i) g.side[i] = i < 2 * c.dim ? side_code(c.bc.type[i]) : kSideWall;
    g.vel_side = -1;
    for (int i = 0; i < 2 * c.dim; ++i)
        if (g.side[i] == kSideVelocity) g.vel_side = i;
    for (int a = 0; a < 3; ++a) g.per[a] = a < c.dim && g.side[2 * a] == kSidePeriodic;
    g.xch = 0;
    for (int i = 0; i < 2 * c.dim; ++i)
        if (g.side[i] == kSideExchange || g.side[i] == kSideWrap) g.xch = 1;
    g.zlo = c.dim == 3 ? c.zlo : 1;
    g.zhi = c.dim == 3 && c.zhi > 0 ? c.zhi : g.n[2];
    g.open = 0;
    for (int i = 0; i < 6; ++i) {
        g.fc_off[i] = -1;
        if (i < 2 * c.dim && (g.side[i] == kSideFreeConvect || g.side[i] == kSideNeumann)) g.open = 1;
    }
    g.fc[0] = g.fc[1] = nullptr;
    // x = 1 of every row starts on a 32-element boundary
    g.base = 31;
    g.sy = round_up(31 + g.e[0], 32);
    g.sz = g.sy * g.e[1];
    g.ps = round_up(g.sz * g.e[2], 32);

    const Physics& P = c.phys;
    PhysD& d = st.phys;
    d.RhoL = P.RhoL;
    d.RhoH = P.RhoH;
    d.drho = P.RhoH - P.RhoL;
    d.drho3 = (P.RhoH - P.RhoL) / 3.0;
    d.tauL = P.tauL;
    d.tauH = P.tauH;
    d.dtau = P.tauH - P.tauL;
    d.kappa = P.kConstant;
    d.beta4 = 4.0 * P.betaConstant;
    d.mobility = P.mobility;
    d.W = P.interfaceWidth;
    d.wc = 1.0 / (0.50 + 3.0 * P.mobility);
    d.one_minus_wc = 1.0 - d.wc;
    d.amob3 = 3.0 * P.mobility;
    for (int a = 0; a < 3; ++a) d.g[a] = P.gravity[a];
    d.sigma = P.sigma;
    d.refLen = P.referenceLength;
    d.caseType = P.caseType;
    st.geo = c.geo;
    for (int a = 0; a < 3; ++a) st.inlet[a] = c.bc.value[kYPlus][a];

    // FP16: power-of-two scale for f so that its typical magnitude (pressure-scaled
    // deviations, w (p + 3 e.u)) sits well inside the FP16 normal range.
    st.pop_scale = 1.0;
    if (precision == CLIPB_FP16) {
        const double grav = std::sqrt(std::fabs(P.gravity[1]) * std::max(P.referenceLength, 1.0));
        const double lap = std::fabs(P.sigma) / std::max(P.referenceLength / 2.0, 1e-30) * 3.0 / std::max(P.RhoL, 1e-30);
        const double fchar = std::max({grav, lap, 1e-8});
        st.pop_scale = std::ldexp(1.0, (int)std::floor(std::log2(64.0 / fchar)));
    }
    s->kt = precision == CLIPB_FP64 ? kernels_fp64() : (precision == CLIPB_FP32 ? kernels_fp32() : kernels_fp16());
    st.seg = 0;
    // default launch variant: FP32/FP16 keep g of the next plane in registers (2D), FP64
    // re-pulls it; clipb_autotune can pick another one
    st.variant = 0;

    const int Q = c.dim == 3 ? 19 : 9;
    // the step kernels index every buffer with 32-bit element offsets
    if ((unsigned long long)Q * (unsigned long long)g.ps >= (1ull << 32))
        return fail(CLIPB_E_CONFIG, "grid too large for one solver: Q x padded nodes must stay below 2^32 (about "
                                    "226 million nodes for D3Q19)");
    const size_t pop = (size_t)Q * g.ps * s->kt.pop_bytes, aux = (size_t)g.ps * s->kt.aux_bytes;
    int rc;
    for (int b = 0; b < 2; ++b) {
        if ((rc = s->alloc(&st.f[b], pop))) return rc;
        if ((rc = s->alloc(&st.gp[b], pop))) return rc;
        if ((rc = s->alloc(&st.c[b], aux))) return rc;
    }
    if ((rc = s->alloc(&st.u, aux * c.dim))) return rc;
    // free-convect state: per such side (2 A + 1) planes of the arithmetic type, per parity
    {
        const int A = c.dim == 3 ? 5 : 3;
        long long total = 0;
        for (int i = 0; i < 2 * c.dim; ++i)
            if (g.side[i] == kSideFreeConvect) {
                g.fc_off[i] = total;
                total += (2LL * A + 1) * side_plane(g, i);
            }
        if (total > 0) {
            const size_t bytes = (size_t)total * (precision == CLIPB_FP64 ? sizeof(double) : sizeof(float));
            for (int b = 0; b < 2; ++b)
                if ((rc = s->alloc(&g.fc[b], bytes))) return rc;
            s->fc_bytes = bytes;
        }
    }
    if ((rc = s->alloc(&st.p, aux))) return rc;
    if ((rc = s->alloc((void**)&st.c0, (size_t)g.ps * sizeof(double)))) return rc;
    st.red_blocks = 8 * 148;  // monitor blocks: a fixed count keeps the sums deterministic
    if ((rc = s->alloc((void**)&st.red, (size_t)2 * st.red_blocks * sizeof(double)))) return rc;
    if ((rc = s->alloc((void**)&s->d_mon, 3 * sizeof(double)))) return rc;
    if ((rc = s->alloc((void**)&st.err, sizeof(int)))) return rc;
    CLIPB_CUDA(cudaMallocHost((void**)&s->h_mon, 3 * sizeof(double)));
    // staged variants need tensor maps of the buffers; without them they are unavailable
    if (s->kt.prepare(st) != cudaSuccess) {
        (void)cudaGetLastError();
        s->kt.release(st);
    }
    CLIPB_CUDA(cudaEventCreate(&s->ev0));
    CLIPB_CUDA(cudaEventCreate(&s->ev1));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    *out = s.release();
    return CLIPB_OK;
}


int clipb::solver_launch_one(clipb_solver* s) {
    CLIPB_CUDA(s->kt.ghost(s->st, s->steps, s->stream));
    CLIPB_CUDA(s->kt.step(s->st, s->steps, s->stream));
    ++s->steps;
    return CLIPB_OK;
}

extern "C" {

const char* clipb_last_error(void) { return g_last_error.c_str(); }

int clipb_create(const char* config_path, int precision, clipb_solver** out) {
    if (!config_path || !out) return fail(CLIPB_E_ARG, "null argument");
    *out = nullptr;
    CaseConfig cfg;
    try {
        cfg = load_config(config_path);
    } catch (const std::exception& e) {
        return fail(CLIPB_E_CONFIG, e.what());
    }
    return solver_create(cfg, precision, out);
}

void clipb_destroy(clipb_solver* s) { delete s; }

int clipb_set_stream(clipb_solver* s, void* stream) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    s->stream = stream ? static_cast<cudaStream_t>(stream) : s->own_stream;
    return CLIPB_OK;
}

int clipb_get_info(const clipb_solver* s, clipb_info* out) {
    if (!s || !out) return fail(CLIPB_E_ARG, "null argument");
    out->dim = s->cfg.dim;
    out->q = s->cfg.dim == 3 ? 19 : 9;
    out->precision = s->st.precision;
    for (int a = 0; a < 3; ++a) {
        out->extent[a] = s->cfg.extent[a];
        out->interior[a] = s->cfg.interior[a];
    }
    out->steps = s->steps;
    out->device_bytes = s->device_bytes;
    out->pop_scale = s->st.pop_scale;
    return CLIPB_OK;
}

int clipb_config_summary(const char* path, int* dim, int* extent3, int* sides6, double* params16) {
    if (!path) return fail(CLIPB_E_ARG, "null path");
    try {
        const CaseConfig c = load_config(path);
        if (dim) *dim = c.dim;
        if (extent3)
            for (int a = 0; a < 3; ++a) extent3[a] = c.extent[a];
        if (sides6)
            for (int i = 0; i < 6; ++i) sides6[i] = i < 2 * c.dim ? c.bc.type[i] : -1;
        if (params16) {
            const Physics& P = c.phys;
            const double v[16] = {P.RhoL, P.RhoH, P.sigma, P.muH, P.muL, P.tauH, P.tauL, P.kConstant,
                                  P.betaConstant, P.mobility, P.interfaceWidth, P.referenceLength, P.gravity[0],
                                  P.gravity[1], P.gravity[2], (double)P.caseType};
            std::memcpy(params16, v, sizeof(v));
        }
    } catch (const std::exception& e) {
        return fail(CLIPB_E_CONFIG, e.what());
    }
    return CLIPB_OK;
}

int clipb_get_intervals(const clipb_solver* s, long long* o) {
    if (!s || !o) return fail(CLIPB_E_ARG, "null argument");
    const Physics& P = s->cfg.phys;
    o[0] = P.finalStep;
    o[1] = P.outputInterval;
    o[2] = P.reportInterval;
    o[3] = P.checkpointInterval;
    return CLIPB_OK;
}

int clipb_get_checkpoint_copies(const clipb_solver* s, long long* copies) {
    if (!s || !copies) return fail(CLIPB_E_ARG, "null argument");
    *copies = s->cfg.phys.checkpointCopy;
    return CLIPB_OK;
}

int clipb_get_upload_bytes(const clipb_solver* s, long long* bytes) {
    if (!s || !bytes) return fail(CLIPB_E_ARG, "null argument");
    *bytes = s->upload_bytes;
    return CLIPB_OK;
}

int clipb_get_params(const clipb_solver* s, double* o) {
    if (!s || !o) return fail(CLIPB_E_ARG, "null argument");
    const Physics& P = s->cfg.phys;
    const double v[16] = {P.RhoL, P.RhoH, P.sigma, P.muH, P.muL, P.tauH, P.tauL, P.kConstant, P.betaConstant,
                          P.mobility, P.interfaceWidth, P.referenceLength, P.gravity[0], P.gravity[1], P.gravity[2],
                          (double)P.caseType};
    std::memcpy(o, v, sizeof(v));
    return CLIPB_OK;
}

// NSAllen::initialCondition (NsAllen.cu:768-824): c = 1/2 +- 1/2 tanh(2 sdf / W) at ghosted
// node (i, j, k), evaluated on the host like the reference.  A z slab evaluates its planes
// at their global z (its ghost planes on the case's boundary at 0 and N + 1, as the whole
// case's ghost planes).  For |2 sdf / W| >= 22 the C library's tanh returns exactly +-1
// (1 - tanh(22) is below half a unit in the last place of 1), so that value is used
// without the call: the result is the same, and most nodes of a large grid lie there.
static inline double c_of_profile(const CaseConfig& c, double t) {
    const int ct = c.phys.caseType;
    if (ct == kBubble) return 0.50 + 0.50 * t;
    if (ct == kDrop || ct == kJet) return 0.50 - 0.50 * t;
    if (ct == kRTI) return 0.5 + 0.5 * t;
    return 0.0;
}

static inline double initial_c(const CaseConfig& c, int i, int j, int k) {
    const double x = (double)i, y = (double)j, z = c.dim == 3 ? (double)(k + c.zoff) : 0.0;
    const double sd = signed_distance(c.geo, 0, x, y, z, c.dim);
    const double a = 2.0 * sd / c.phys.interfaceWidth;
    const double t = a >= 22.0 ? 1.0 : (a <= -22.0 ? -1.0 : std::tanh(a));
    return c_of_profile(c, t);
}

// Row (j, k) of the initial field when every one of its points has |2 sd / W| >= 22 (tanh
// taken as +-1 there, as initial_c does): true and its value.  The distance bound carries a
// margin of 1e-9 relative, far above the rounding of sd and of 2 sd / W.
static inline bool initial_row_uniform(const CaseConfig& c, int j, int k, double& v) {
    const double d = 11.0 * c.phys.interfaceWidth * (1.0 + 1e-9) + 1e-9;
    const double z = c.dim == 3 ? (double)(k + c.zoff) : 0.0;
    const int sgn = row_distance_sign(c.geo, 0, 0.0, (double)(c.extent[0] - 1), (double)j, z, c.dim, d);
    if (sgn == 0) return false;
    v = c_of_profile(c, sgn > 0 ? 1.0 : -1.0);
    return true;
}

int clipb_initial_condition(clipb_solver* s, double* c_out) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    const CaseConfig& c = s->cfg;
    const int E0 = c.extent[0], E1 = c.extent[1], E2 = c.extent[2];
    s->host_c.alloc((size_t)E0 * E1 * E2);
    double* hc = s->host_c.data();
    host_parallel(E0, [&](long long i) {
        for (int j = 0; j < E1; ++j)
            for (int k = 0; k < E2; ++k) hc[((size_t)i * E1 + j) * E2 + k] = initial_c(c, (int)i, j, k);
    }, 1);
    if (c_out) std::memcpy(c_out, hc, s->host_c.size() * sizeof(double));
    return CLIPB_OK;
}

int clipb_init_device(clipb_solver* s) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    const CaseConfig& c = s->cfg;
    CLIPB_CUDA(launch_initial_condition(s->st, c.phys.caseType, c.phys.interfaceWidth, c.zoff, s->stream));
    s->upload_bytes = 0;
    CLIPB_CUDA(s->kt.init(s->st, s->stream));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    s->steps = 0;
    s->initialized = true;
    return CLIPB_OK;
}

// Upload of the initial field into st.c0 (device layout: x fastest, padded rows) and the
// initial state.  row(j, k, out) writes the E0 values of ghosted row (j, k) through
// out(i, value).  Large fields go through pinned staging kept with the solver, in chunks
// of z planes: the host threads fill chunk n + 1 while chunk n is copied.  Small fields
// are staged in pageable memory (no page-locking per case of a batch), in one copy.
// In a large field most rows hold one value (the bulk of each phase, exactly 0 or 1): the
// threads mark every uniform row as they write it, each plane sends only its rows from the
// first to the last one that is not uniform with the plane's first or last row, and one
// kernel writes the uniform rows above and below from a per-plane table.  The device field
// holds the same bits either way.  After each chunk the initial state of the planes whose
// neighbours have arrived is computed (init_planes), so that kernel runs while the host
// threads evaluate the next chunks.
}  // extern "C"

namespace {
struct PlaneFill {
    int jlo, jhi;  // rows jlo .. jhi were copied; rows below take a, rows above take b
    double a, b;
};

__global__ void fill_uniform_rows(double* __restrict__ c0, const PlaneFill* __restrict__ tab, long long base,
                                  long long sy, long long sz, int E0, int k_first) {
    const int j = (int)blockIdx.x, k = k_first + (int)blockIdx.y;
    const PlaneFill t = tab[k];
    if (j >= t.jlo && j <= t.jhi) return;
    const double v = j < t.jlo ? t.a : t.b;
    double* row = c0 + base + (long long)j * sy + (long long)k * sz;
    for (int i = (int)threadIdx.x; i < E0; i += (int)blockDim.x) row[i] = v;
}
}  // namespace

template <class Row, class Uniform>
static int upload_initial(clipb_solver* s, Row&& row, Uniform&& uniform_row) {
    const CaseConfig& c = s->cfg;
    const int E0 = c.extent[0], E1 = c.extent[1], E2 = c.extent[2];
    const Geom& g = s->st.g;
    constexpr size_t kPinnedFrom = size_t(1) << 22;  // doubles (32 MB)
    clipb_solver::HostArray dev;
    double* dv;
    bool fresh = true;  // the padding, which the rows never write, needs zeros
    const bool pinned = (size_t)g.ps >= kPinnedFrom;
    if (pinned) {
        if (s->h_stage_elems < (size_t)g.ps) {
            if (s->h_stage) cudaFreeHost(s->h_stage);
            s->h_stage = nullptr;
            s->h_stage_elems = 0;
            CLIPB_CUDA(cudaHostAlloc((void**)&s->h_stage, (size_t)g.ps * sizeof(double), cudaHostAllocDefault));
            s->h_stage_elems = (size_t)g.ps;
        } else {
            fresh = false;  // zero padding from the first upload
        }
        dv = s->h_stage;
    } else {
        dev.alloc((size_t)g.ps);
        dv = dev.data();
    }
    constexpr long long kChunk = 1 << 20;
    if (fresh)
        host_parallel((g.ps + kChunk - 1) / kChunk, [&](long long b) {
            std::fill(dv + b * kChunk, dv + std::min<long long>(g.ps, (b + 1) * kChunk), 0.0);
        }, 1);
    // chunks of planes; chunk [k0, k1) owns elements [lo(k0), lo(k1)) of the layout
    const int planes = pinned && E2 > 1 ? 8 : E2;
    const int nchunks = (E2 + planes - 1) / planes;
    auto lo = [&](int k) -> long long { return k == 0 ? 0 : (k >= E2 ? g.ps : g.base + (long long)k * g.sz); };
    const long long T = std::max<long long>(
        1, std::min<long long>(std::min<long long>(std::thread::hardware_concurrency(), 32), (long long)E1 * E2 / 16));
    std::unique_ptr<std::atomic<int>[]> done(new std::atomic<int>[nchunks]);
    for (int n = 0; n < nchunks; ++n) done[n].store(0);
    std::atomic<int> copy_error{0};
    // uniform rows (pinned uploads): per row 0 (not uniform), 1 (uniform, written to the
    // staging) or 2 (uniform by uniform_row, not written), and its first value
    const bool sparse = pinned;
    std::vector<unsigned char> uniform(sparse ? (size_t)E1 * E2 : 0);
    std::vector<double> rowval(sparse ? (size_t)E1 * E2 : 0);
    if (sparse && s->plane_tab_elems < (size_t)E2) {
        if (s->h_plane_tab) cudaFreeHost(s->h_plane_tab);
        s->h_plane_tab = nullptr;
        s->plane_tab_elems = 0;
        CLIPB_CUDA(cudaHostAlloc(&s->h_plane_tab, (size_t)E2 * sizeof(PlaneFill), cudaHostAllocDefault));
        void* d = nullptr;
        const int rc = s->alloc(&d, (size_t)E2 * sizeof(PlaneFill));
        if (rc) return rc;
        s->d_plane_tab = d;
        s->plane_tab_elems = (size_t)E2;
    }
    PlaneFill* tab = static_cast<PlaneFill*>(s->h_plane_tab);
    std::atomic<long long> sent{0};
    int init_done = 0;  // planes [0, init_done) have their initial state (thread 0 only)
    auto bits = [](double v) {
        unsigned long long u;
        std::memcpy(&u, &v, sizeof(u));
        return u;
    };
    // plane k of a filled chunk: rows jlo .. jhi go by copy, the uniform rows around them
    // are written by fill_uniform_rows
    auto send_plane = [&](int k) {
        const unsigned char* u = uniform.data() + (size_t)k * E1;
        const double* rv = rowval.data() + (size_t)k * E1;
        auto first = [&](int j) { return bits(rv[j]); };
        int jlo = 0;
        while (jlo < E1 && u[jlo] && first(jlo) == first(0)) ++jlo;
        int jhi = E1 - 1;
        while (jhi >= jlo && u[jhi] && first(jhi) == first(E1 - 1)) --jhi;
        tab[k] = PlaneFill{jlo, jhi, rv[0], rv[E1 - 1]};
        if (jlo > jhi) return;
        for (int j = jlo; j <= jhi; ++j)  // rows inside the copied range that were not written
            if (u[j] == 2) std::fill_n(dv + s->dev_index(0, j, k), E0, rv[j]);
        const long long a = s->dev_index(0, jlo, k), b = s->dev_index(0, jhi + 1, k);
        if (cudaMemcpyAsync(s->st.c0 + a, dv + a, (size_t)(b - a) * sizeof(double), cudaMemcpyHostToDevice, s->stream) !=
            cudaSuccess)
            copy_error.store(1);
        sent.fetch_add((b - a) * (long long)sizeof(double));
    };
    auto work = [&](long long t) {
        for (int n = 0; n < nchunks; ++n) {
            const int k0 = n * planes, k1 = std::min(E2, k0 + planes);
            const long long rows = (long long)E1 * (k1 - k0);
            for (long long r = rows * t / T; r < rows * (t + 1) / T; ++r) {
                const int j = (int)(r % E1), k = k0 + (int)(r / E1);
                const size_t rid = (size_t)k * E1 + j;
                if (sparse && uniform_row(j, k, rowval[rid])) {
                    uniform[rid] = 2;
                    continue;
                }
                double* base = dv + s->dev_index(0, j, k);
                row(j, k, [base](int i, double v) { base[i] = v; });
                if (sparse) {
                    bool same = true;
                    for (int i = 1; i < E0 && same; ++i) same = bits(base[i]) == bits(base[0]);
                    uniform[rid] = same;
                    rowval[rid] = base[0];
                }
            }
            done[n].fetch_add(1, std::memory_order_acq_rel);
            if (t == 0) {  // thread 0 copies each chunk once every thread has filled its part
                while (done[n].load(std::memory_order_acquire) < T) std::this_thread::yield();
                if (sparse) {
                    for (int k = k0; k < k1; ++k) send_plane(k);
                    // the chunk's uniform rows, then the initial state of every plane whose
                    // neighbours have arrived: the GPU works while the host fills the next chunk
                    const size_t tb = (size_t)(k1 - k0) * sizeof(PlaneFill);
                    if (cudaMemcpyAsync(static_cast<PlaneFill*>(s->d_plane_tab) + k0, tab + k0, tb,
                                        cudaMemcpyHostToDevice, s->stream) != cudaSuccess)
                        copy_error.store(1);
                    sent.fetch_add((long long)tb);
                    fill_uniform_rows<<<dim3((unsigned)E1, (unsigned)(k1 - k0)), 128, 0, s->stream>>>(
                        s->st.c0, static_cast<const PlaneFill*>(s->d_plane_tab), s->st.g.base, s->st.g.sy,
                        s->st.g.sz, E0, k0);
                    const int ready = k1 >= E2 ? E2 : k1 - 1;
                    if (cudaGetLastError() != cudaSuccess ||
                        s->kt.init_planes(s->st, init_done, ready, s->stream) != cudaSuccess)
                        copy_error.store(1);
                    init_done = std::max(init_done, ready);
                } else {
                    const long long a = lo(k0), b = lo(k1);
                    if (cudaMemcpyAsync(s->st.c0 + a, dv + a, (size_t)(b - a) * sizeof(double),
                                        cudaMemcpyHostToDevice, s->stream) != cudaSuccess)
                        copy_error.store(1);
                    sent.fetch_add((b - a) * (long long)sizeof(double));
                }
            }
        }
    };
    if (T == 1) {
        work(0);
    } else {
        std::vector<std::thread> pool;
        for (long long t = 1; t < T; ++t) pool.emplace_back(work, t);
        work(0);
        for (auto& th : pool) th.join();
    }
    if (copy_error.load()) {
        CLIPB_CUDA(cudaGetLastError());
        return fail(CLIPB_E_CUDA, "initial-field upload or initial state failed");
    }
    s->upload_bytes = sent.load();
    if (!sparse) CLIPB_CUDA(s->kt.init(s->st, s->stream));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    s->steps = 0;
    s->initialized = true;
    return CLIPB_OK;
}

extern "C" {

int clipb_device_initializer(clipb_solver* s, const double* c_host) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    const CaseConfig& c = s->cfg;
    const int E0 = c.extent[0], E1 = c.extent[1], E2 = c.extent[2];
    if (!c_host) {
        if (s->host_c.empty()) {
            const int rc = clipb_initial_condition(s, nullptr);
            if (rc) return rc;
        }
        c_host = s->host_c.data();
    }
    return upload_initial(
        s, [&](int j, int k, auto&& out) {
            for (int i = 0; i < E0; ++i) out(i, c_host[((size_t)i * E1 + j) * E2 + k]);
        },
        [](int, int, double&) { return false; });
}

// clipb_initial_condition + clipb_device_initializer, with the field evaluated straight
// into the device layout (the same values, without the reference-layout copy).
int clipb_init(clipb_solver* s) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    const CaseConfig& c = s->cfg;
    const int E0 = c.extent[0];
    return upload_initial(
        s, [&](int j, int k, auto&& out) {
            for (int i = 0; i < E0; ++i) out(i, initial_c(c, i, j, k));
        },
        [&](int j, int k, double& v) { return initial_row_uniform(c, j, k, v); });
}

static const char* const kWaitMessage =
    "a bounded wait for a bulk copy in the staged step gave up; results of this solver are invalid";

// Synchronise the stream and report the staged step's wait flag.
static int check_wait_flag(clipb_solver* s) {
    int flag = 0;
    CLIPB_CUDA(cudaMemcpyAsync(&flag, s->st.err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    return flag ? fail(CLIPB_E_CUDA, kWaitMessage) : CLIPB_OK;
}

static int launch_one(clipb_solver* s) { return solver_launch_one(s); }

// Capture kGraphSteps steps (starting at an even step) into s->graph.
static int build_graph(clipb_solver* s) {
    cudaGraph_t g = nullptr;
    CLIPB_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    long long k = 0;
    for (int i = 0; i < clipb_solver::kGraphSteps; ++i, ++k) {
        const cudaError_t e1 = s->kt.ghost(s->st, k, s->stream);
        const cudaError_t e2 = s->kt.step(s->st, k, s->stream);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            cudaStreamEndCapture(s->stream, &g);
            if (g) cudaGraphDestroy(g);
            return fail(CLIPB_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
        }
    }
    CLIPB_CUDA(cudaStreamEndCapture(s->stream, &g));
    const cudaError_t e = cudaGraphInstantiate(&s->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(CLIPB_E_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return CLIPB_OK;
}

int clipb_solve(clipb_solver* s, int nsteps) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    if (!s->initialized) return fail(CLIPB_E_STATE, "solve before init");
    if (s->slab_half) return fail(CLIPB_E_STATE, "part 2 of a slab step is due (clipb_slab_step_part)");
    if (nsteps < 0) return fail(CLIPB_E_ARG, "negative step count");
    int rc;
    long long left = nsteps;
    const int G = clipb_solver::kGraphSteps;
    if (s->use_graphs && left > G) {
        if (s->steps & 1) {  // the graph starts on an even step
            if ((rc = launch_one(s))) return rc;
            --left;
        }
        if (!s->graph && (rc = build_graph(s))) return rc;
        for (; left >= G; left -= G) {
            CLIPB_CUDA(cudaGraphLaunch(s->graph, s->stream));
            s->steps += G;
        }
    }
    for (; left > 0; --left)
        if ((rc = launch_one(s))) return rc;
    return CLIPB_OK;
}

int clipb_set_launch(clipb_solver* s, int variant, int seg) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    const int nv = s->cfg.dim == 3 ? s->kt.variants3 : s->kt.variants2;
    if (variant < 0 || variant >= nv) return fail(CLIPB_E_ARG, "variant must be in [0, " + std::to_string(nv) + ")");
    if (!s->kt.available(s->st, variant))
        return fail(CLIPB_E_ARG, "variant " + std::to_string(variant) + " is unavailable on this solver");
    if (seg < 0) return fail(CLIPB_E_ARG, "negative segment length");
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    s->st.variant = variant;
    s->st.seg = seg;
    s->drop_graph();
    return CLIPB_OK;
}

int clipb_get_launch(const clipb_solver* s, int* variant, int* seg, int* nvariants) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    if (variant) *variant = s->st.variant;
    if (seg) *seg = s->st.seg;
    if (nvariants) *nvariants = s->cfg.dim == 3 ? s->kt.variants3 : s->kt.variants2;
    return CLIPB_OK;
}

int clipb_set_wait_limit(clipb_solver* s, long long cycles, unsigned inject_bytes) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    if (cycles < 0) return fail(CLIPB_E_ARG, "negative wait limit");
    if (inject_bytes >= (1u << 16)) return fail(CLIPB_E_ARG, "inject_bytes must stay below 65536");
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    s->st.wait_limit = cycles;
    s->st.wait_inject = inject_bytes;
    s->drop_graph();  // the graph holds the old kernel arguments
    return CLIPB_OK;
}

int clipb_set_graphs(clipb_solver* s, int enable) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    s->use_graphs = enable != 0;
    if (!s->use_graphs) s->drop_graph();
    else if (s->initialized && !s->graph) return build_graph(s);  // now, not inside a later solve
    return CLIPB_OK;
}

// Time every launch variant and segment length on this solver's own state, keep the
// fastest and rebuild the initial state (the initial c stays on the device, so the
// rebuilt state equals the one before tuning).
int clipb_autotune(clipb_solver* s, int trial_steps, int* best_variant, int* best_seg, float* best_ms) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    if (!s->initialized || s->steps != 0) return fail(CLIPB_E_STATE, "autotune needs a freshly initialised solver");
    if (trial_steps < 1) trial_steps = 4;
    const int dim = s->cfg.dim;
    const int nv = dim == 3 ? s->kt.variants3 : s->kt.variants2;
    const int n_march = dim == 3 ? s->st.g.n[2] : s->st.g.n[1];
    std::vector<int> segs = dim == 3 ? std::vector<int>{8, 16, 32, 64} : std::vector<int>{1, 2, 4, 8, 16, 32, 64};
    float best = 1e30f;
    int bv = s->st.variant, bs = s->st.seg;
    const bool graphs = s->use_graphs;
    s->use_graphs = false;
    int rc;
    // The trials run on one evolving state, whose step time can drift as the flow develops;
    // the candidates are timed twice, in order and then in reverse, and each keeps its best,
    // so that a drift favours none of them.
    std::vector<std::pair<int, int>> cands;
    for (int v = 0; v < nv; ++v) {
        if (!s->kt.available(s->st, v)) continue;
        for (int seg : segs)
            if (seg <= n_march || seg == segs.front()) cands.emplace_back(v, seg);
    }
    std::vector<float> ms_best(cands.size(), 1e30f);
    for (int pass = 0; pass < 2; ++pass) {
        for (size_t i = 0; i < cands.size(); ++i) {
            const size_t c = pass == 0 ? i : cands.size() - 1 - i;
            if ((rc = clipb_set_launch(s, cands[c].first, cands[c].second))) return rc;
            if ((rc = clipb_solve(s, 1))) return rc;  // warm-up
            float ms = 0.f;
            if ((rc = clipb_time_steps(s, trial_steps, &ms))) return rc;
            ms_best[c] = std::min(ms_best[c], ms);
        }
    }
    for (size_t c = 0; c < cands.size(); ++c)
        if (ms_best[c] < best) {
            best = ms_best[c];
            bv = cands[c].first;
            bs = cands[c].second;
        }
    s->use_graphs = graphs;
    if ((rc = clipb_set_launch(s, bv, bs))) return rc;
    CLIPB_CUDA(s->kt.init(s->st, s->stream));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    s->steps = 0;
    // capture the winner's graph now, so that the first long solve does not pay for it
    if (s->use_graphs && (rc = build_graph(s))) return rc;
    if (best_variant) *best_variant = bv;
    if (best_seg) *best_seg = bs;
    if (best_ms) *best_ms = best / (float)trial_steps;
    return CLIPB_OK;
}

static int ensure_stage(clipb_solver* s, size_t elems) {
    if (s->stage_elems >= elems) return 0;
    if (s->d_stage) {
        CLIPB_CUDA(cudaStreamSynchronize(s->stream));
        cudaFree(s->d_stage);
        s->allocations.erase(std::remove(s->allocations.begin(), s->allocations.end(), (void*)s->d_stage), s->allocations.end());
        s->d_stage = nullptr;
    }
    const int rc = s->alloc((void**)&s->d_stage, elems * sizeof(double));
    if (rc) return rc;
    s->stage_elems = elems;
    return 0;
}

int clipb_get_field(clipb_solver* s, int field, double* host_out, size_t count) {
    if (!s || !host_out) return fail(CLIPB_E_ARG, "null argument");
    if (!s->initialized) return fail(CLIPB_E_STATE, "get_field before init");
    if (field < CLIPB_FIELD_C || field > CLIPB_FIELD_G_POST) return fail(CLIPB_E_ARG, "unknown field");
    const size_t need = (size_t)s->ref_nodes() * s->ncomp(field);
    if (count != need) return fail(CLIPB_E_ARG, "count must be " + std::to_string(need));
    int rc = ensure_stage(s, need);
    if (rc) return rc;
    const int last = s->steps > 0 ? (int)((s->steps - 1) & 1) : -1;
    CLIPB_CUDA(s->kt.field(s->st, field, last, s->steps, s->d_stage, s->stream));
    CLIPB_CUDA(cudaMemcpyAsync(host_out, s->d_stage, need * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    return check_wait_flag(s);
}

int clipb_get_fields(clipb_solver* s, double* c, double* p, double* rho, double* u) {
    const size_t n = s ? (size_t)s->ref_nodes() : 0;
    int rc = 0;
    if (c && (rc = clipb_get_field(s, CLIPB_FIELD_C, c, n))) return rc;
    if (p && (rc = clipb_get_field(s, CLIPB_FIELD_P, p, n))) return rc;
    if (rho && (rc = clipb_get_field(s, CLIPB_FIELD_RHO, rho, n))) return rc;
    if (u && (rc = clipb_get_field(s, CLIPB_FIELD_VEL, u, n * (s ? s->cfg.dim : 0)))) return rc;
    return CLIPB_OK;
}

int clipb_get_field_device(clipb_solver* s, int field, double* dev_out, size_t count) {
    if (!s || !dev_out) return fail(CLIPB_E_ARG, "null argument");
    if (!s->initialized) return fail(CLIPB_E_STATE, "get_field_device before init");
    if (field != CLIPB_FIELD_C && field != CLIPB_FIELD_RHO && field != CLIPB_FIELD_VEL)
        return fail(CLIPB_E_ARG, "device copies support c, rho and u");
    const size_t nn = (size_t)s->st.g.n[0] * s->st.g.n[1] * s->st.g.n[2];
    const size_t need = nn * (field == CLIPB_FIELD_VEL ? s->cfg.dim : 1);
    if (count != need) return fail(CLIPB_E_ARG, "count must be " + std::to_string(need));
    const int last = s->steps > 0 ? (int)((s->steps - 1) & 1) : -1;
    CLIPB_CUDA(s->kt.interior(s->st, field, last, s->steps, dev_out, s->stream));
    return CLIPB_OK;
}

int clipb_monitors(clipb_solver* s, double* mass, double* kinetic) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    if (!s->initialized) return fail(CLIPB_E_STATE, "monitors before init");
    CLIPB_CUDA(s->kt.monitors(s->st, s->steps, s->d_mon, s->stream));
    CLIPB_CUDA(cudaMemcpyAsync(s->h_mon, s->d_mon, 3 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    if (s->h_mon[2] != 0.0) return fail(CLIPB_E_CUDA, kWaitMessage);
    if (mass) *mass = s->h_mon[0];
    if (kinetic) *kinetic = s->h_mon[1];
    if (std::isnan(s->h_mon[0]) || std::isnan(s->h_mon[1])) return fail(CLIPB_E_DIVERGED, "Solver has diverged.");
    return CLIPB_OK;
}

int clipb_solve_monitored(clipb_solver* s, int nsteps, double* mass, double* kinetic) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    if (!s->initialized) return fail(CLIPB_E_STATE, "solve before init");
    if (nsteps < 1) return fail(CLIPB_E_ARG, "a monitored solve takes at least one step");
    if (!s->kt.fused_monitors(s->st)) {
        const int rc = clipb_solve(s, nsteps);
        return rc ? rc : clipb_monitors(s, mass, kinetic);
    }
    int rc = clipb_solve(s, nsteps - 1);
    if (rc) return rc;
    if (!s->mon_rows) {
        const Geom& g = s->st.g;
        const size_t rows = (size_t)((g.n[0] + 31) / 32) * g.n[1] * (g.zhi - g.zlo + 1);
        if ((rc = s->alloc((void**)&s->mon_rows, 2 * rows * sizeof(double)))) return rc;
    }
    s->st.mon_rows = s->mon_rows;
    rc = launch_one(s);
    s->st.mon_rows = nullptr;
    if (rc) return rc;
    CLIPB_CUDA(s->kt.monitor_rows(s->st, s->mon_rows, s->d_mon, s->stream));
    CLIPB_CUDA(cudaMemcpyAsync(s->h_mon, s->d_mon, 3 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    if (s->h_mon[2] != 0.0) return fail(CLIPB_E_CUDA, kWaitMessage);
    if (mass) *mass = s->h_mon[0];
    if (kinetic) *kinetic = s->h_mon[1];
    if (std::isnan(s->h_mon[0]) || std::isnan(s->h_mon[1])) return fail(CLIPB_E_DIVERGED, "Solver has diverged.");
    return CLIPB_OK;
}

int clipb_time_steps(clipb_solver* s, int nsteps, float* ms) {
    if (!s || !ms) return fail(CLIPB_E_ARG, "null argument");
    // a graph the steps will replay is captured before the first event, not timed
    if (s->initialized && s->use_graphs && nsteps > clipb_solver::kGraphSteps && !s->graph) {
        const int rc = build_graph(s);
        if (rc) return rc;
    }
    CLIPB_CUDA(cudaEventRecord(s->ev0, s->stream));
    const int rc = clipb_solve(s, nsteps);
    if (rc) return rc;
    CLIPB_CUDA(cudaEventRecord(s->ev1, s->stream));
    CLIPB_CUDA(cudaEventSynchronize(s->ev1));
    CLIPB_CUDA(cudaEventElapsedTime(ms, s->ev0, s->ev1));
    return check_wait_flag(s);
}

}  // extern "C"
