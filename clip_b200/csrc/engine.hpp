// Device state of one solver and the per-precision kernel table (host side).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "config.hpp"

namespace clipb {

// Side codes of the device geometry.  A slip wall is a wall here: the reference bounces
// slip-wall populations back with the no-slip wall map (kernelHalfBounceBack with
// wallBCMap, Solver.cu:248-333, 997-1004; its slipWallBCMap kernel is never launched).
// kSideExchange: a z face of a slab inside the case (its last plane and the ghost plane hold
// the neighbouring slab's first two planes); kSideWrap: a z face of a slab on the case's
// periodic z boundary (its ghost plane holds the periodic image, the other end's boundary
// plane, from the slab there).
enum : int { kSideWall = 0, kSideFreeConvect = 2, kSidePeriodic = 3, kSideNeumann = 4, kSideVelocity = 5,
             kSideExchange = 6, kSideWrap = 7 };

// Sides whose ghost c mirrors the adjacent interior node (Boundary::isMirrorType).
__host__ __device__ inline bool mirror_side(int t) {
    return t == kSideWall || t == kSideFreeConvect || t == kSideNeumann;
}

// Lattice geometry in the device layout: structure of arrays, x fastest, ghost layer
// kept (so velocity-inlet planes have storage), rows padded so that interior x = 1 starts
// on a 128-element boundary.  Node (x, y, z) (ghost coordinates 0 and n+1 included) lives
// at element base + x + y*sy + z*sz of every per-node array; population q of a node at
// q*ps further.
struct Geom {
    int dim;
    int n[3];       // interior nodes per axis (n[2] = 1 in 2D)
    int e[3];       // ghosted extent per axis (n + 2; e[2] = 1 in 2D)
    long long sy, sz, base, ps;
    int side[6];    // kSide* per side
    int per[3];     // axis periodic
    int vel_side;   // the velocity side (-1 if none)
    int open;       // any free-convect or Neumann side
    int xch;        // any exchange side (a z slab of a larger case)
    int zlo, zhi;   // 3D: planes updated by the step (1 .. n[2] for a whole case)
    // Free-convect state (kernelFreeConvect reads the last step's populations on the side's
    // boundary layer and the previous velocity of the layer inside it): per free-convect
    // side s a block at element fc_off[s] (-1: not free convect) of fc[parity], elements of
    // the step's arithmetic type: for each of the side's entering directions (wallBCMap
    // order) a plane of f, then one of g (shifted storage: g - w_q c of the node), then the
    // plane of the inner layer's velocity along the side's axis.  Parity b is read by step b
    // and written by step b - 1.
    long long fc_off[6];
    void* fc[2];
};

// Nodes of the plane of side s (the two other axes).
__host__ __device__ inline long long side_plane(const Geom& g, int s) {
    const int a = s / 2;
    long long p = 1;
    for (int b = 0; b < g.dim; ++b)
        if (b != a) p *= g.n[b];
    return p;
}
// Index of interior node (x, y, z) in the plane of side s (lower other axis fastest).
__host__ __device__ inline long long side_plane_index(const Geom& g, int s, int x, int y, int z) {
    const int a = s / 2;
    const int c[3] = {x - 1, y - 1, z - 1};
    long long idx = 0, stride = 1;
    for (int b = 0; b < g.dim; ++b) {
        if (b == a) continue;
        idx += c[b] * stride;
        stride *= g.n[b];
    }
    return idx;
}

// Physical parameters in FP64; kernels cast them to their arithmetic type.
struct PhysD {
    double RhoL, RhoH, drho, drho3, tauL, tauH, dtau, kappa, beta4, mobility, W, wc, one_minus_wc, amob3;
    double g[3];
    double sigma, refLen;
    int caseType;
};

struct DevState {
    int precision;       // CLIPB_FP64 / FP32 / FP16
    Geom g;
    PhysD phys;
    GeometryTable geo;   // for the velocity-inlet mask
    double inlet[3];     // inlet velocity (the reference reads the y+ entry, Solver.cu:587-588)
    void* f[2];          // population buffers (storage type), f[k % 2] is the input of step k
    void* gp[2];
    void* c[2];          // order parameter (aux type), same parity rule
    void* u;             // velocity, DIM planes (aux type)
    void* uin;           // velocity the step reads, when not null (else u): the adjoint's
                         // recomputation writes each step's u into the next tape entry
    void* p;             // pressure (aux type)
    double* c0;          // initial c, device layout (double)
    double* red;         // reduction partials
    int red_blocks;
    // monitor partials written by a monitored 3D step (mass and kinetic energy of each row
    // segment of 32 nodes, 2 doubles each), or null: set only for that step's launch
    double* mon_rows;
    double pop_scale;    // FP16: power-of-two scale of stored f
    int variant;         // launch variant of the fused step (Launch::step)
    int seg;             // planes (3D) / rows (2D) per CTA; 0 = default
    int* err;            // device flag: a bounded wait in a staged kernel gave up
    long long wait_limit;   // cycles a staged kernel's wait lasts before it gives up (0: default)
    unsigned wait_inject;   // test hook: bytes the first bulk load of each block expects in excess
    void* stage;         // host: tensor maps of the staged 3D step (StageHost), or null
};

using InitFn = cudaError_t (*)(const DevState&, cudaStream_t);
using InitPlanesFn = cudaError_t (*)(const DevState&, int z0, int z1, cudaStream_t);
using StepFn = cudaError_t (*)(const DevState&, long long step, cudaStream_t);
// Reference-layout field output: which = CLIPB_FIELD_*; `last` is the parity of the last
// step's input buffer (or -1 right after init).
using FieldFn = cudaError_t (*)(const DevState&, int which, int last, long long steps, double* out, cudaStream_t);
using InteriorFn = cudaError_t (*)(const DevState&, int which, int last, long long steps, double* out, cudaStream_t);
using MonitorFn = cudaError_t (*)(const DevState&, long long steps, double* out2, cudaStream_t);
// Sums of the row-segment partials that a monitored 3D step wrote (mon_rows) into out2.
using MonitorRowsFn = cudaError_t (*)(const DevState&, const double* rows, double* out2, cudaStream_t);
// Interior fields packed for a .vts file (vts_pack_kernel): FP64, or FP32 when `single`.
using VtsPackFn = cudaError_t (*)(const DevState&, int last, void* out, bool single, cudaStream_t);

struct KernelTable {
    // one-off host set-up after allocation (tensor maps, shared-memory limits)
    cudaError_t (*prepare)(DevState&);
    void (*release)(DevState&);
    bool (*available)(const DevState&, int variant);  // launch variant usable on this solver
    InitFn init;
    InitPlanesFn init_planes;  // the initial state of ghosted planes [z0, z1) only
    StepFn ghost;      // velocity-inlet ghost planes before step k (nullptr-safe: no-op without inlet)
    StepFn step;       // fused step k
    FieldFn field;
    InteriorFn interior;
    MonitorFn monitors;
    MonitorRowsFn monitor_rows;
    // launch variant whose step can write monitor partials (the 3D direct-load kernels)
    bool (*fused_monitors)(const DevState&);
    VtsPackFn vts_pack;
    // batched 2D step (many cases, one persistent launch; see step2d_batch_kernel)
    size_t args_bytes;                                          // bytes of one case's step arguments
    void (*make_args)(const DevState&, long long step, void* out);  // host: arguments of step `step`
    cudaError_t (*step2_batch)(const void* args, const int* items, int nitems, int variant, int seg,
                               int blocks_per_sm, cudaStream_t);
    int (*tile2)(int variant);                                  // tile width (x nodes) of a 2D variant
    // state read by step with input parity b from reference-layout FP64 fields (f, g, c, u)
    cudaError_t (*set_state)(const DevState&, int b, const double* f, const double* g, const double* c,
                             const double* u, cudaStream_t);
    int aux_bytes;     // bytes of c/u/p elements
    int pop_bytes;     // bytes of a stored population
    int variants2, variants3;  // launch variants of the fused step (2D, 3D)
};

KernelTable kernels_fp64();
// Initial field of NSAllen::initialCondition evaluated on the device into st.c0 (FP64).
cudaError_t launch_initial_condition(const DevState& st, int case_type, double W, int zoff, cudaStream_t s);
KernelTable kernels_fp32();
KernelTable kernels_fp16();

}  // namespace clipb
