// sm_100a kernels of the CLIP lattice update (templated on a precision policy;
// instantiated in kernels_fp64.cu / kernels_fp32.cu / kernels_fp16.cu).
//
// One fused pass per time step replaces the reference's ~15 launches
// (NsAllen.cu:881-892): pull-streaming of f and g with half-way bounce-back and periodic
// wrap, the Allen-Cahn order parameter on a shared-memory tile with halo, the chemical
// potential / isotropic gradient stencils, the macroscopic update, and the collision of
// the next step.  Only the minimal state crosses HBM: f and g (read + write once), u
// (read + write) and c (read for the lagged ghost layer, write).
//
// Step k (k = 0, 1, ...) reads f[k%2], g[k%2], c[k%2] and u, and writes f[(k+1)%2],
// g[(k+1)%2], c[(k+1)%2] and u.  After step k the interior c, u equal the reference's
// after k+1 calls of NSAllen::solve; f[k%2] holds the reference's post-collision f of
// that call, whose pull gives its f_post and p.
#pragma once

#include <utility>

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "engine.hpp"
#include "lattice.cuh"

namespace clipb {

// ---------------------------------------------------------------- precision policy
// Sf, Sg: storage of f and g.  T: arithmetic of the hydrodynamic part (f, WMRT).
// TP: arithmetic of the phase-field part (c sums, stencils, g relaxation).  A: storage of
// c and u.  kShift: g is stored as the deviation g - w_q c_s, about 1% of g, where c_s is
// the stored c (of the same step) of the node that will pull the value: the writer uses
// c of the destination node s + e_q when that node is interior, else its own c (the value
// then comes back to it by bounce-back, or reaches another node through a periodic wrap or
// a velocity-inlet plane, whose readers use the source's c).  So a reader needs only its
// own c for every direction that does not cross the domain boundary, and the deviations
// it pulls sum to c - c_old directly.
// FP16 storage additionally scales f by a power of two (DevState::pop_scale) and g by 256.
template <typename Sf_, typename Sg_, typename T_, typename TP_, typename A_, bool kShift_>
struct Prec {
    using Sf = Sf_;
    using Sg = Sg_;
    using T = T_;
    using TP = TP_;
    using A = A_;
    static constexpr bool kShift = kShift_;
    static constexpr bool kHalf = std::is_same<Sf_, __half>::value;
    // FP64: the reference's literal operation sequence (bit-exact); otherwise the FP32
    // update on shifted storage (lean_update).
    static constexpr bool kExact = std::is_same<T_, double>::value;
    static_assert(kExact || (std::is_same<T_, float>::value && std::is_same<TP_, float>::value && kShift_),
                  "reduced-precision paths compute in FP32 on shifted g storage");
    // c of a node in the shared-memory ring: the FP64 value, or (stored FP32 c, remainder)
    using Ring = typename std::conditional<kExact, T_, float2>::type;
};

constexpr double kGScaleHalf = 256.0;

// Products that must not be contracted into a neighbouring add: the power-of-two FP16
// scalings are exact on their own, so writing them with round-to-nearest intrinsics keeps
// every kernel that inlines the codec on one rounding sequence.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

template <class PR>
struct Codec {
    using T = typename PR::T;
    using TP = typename PR::TP;
    using A = typename PR::A;
    T finv, fscale;
    TP ginv, gscale;
    __device__ __forceinline__ explicit Codec(double pop_scale) {
        fscale = T(PR::kHalf ? pop_scale : 1.0);
        finv = T(PR::kHalf ? 1.0 / pop_scale : 1.0);
        gscale = TP(PR::kHalf ? kGScaleHalf : 1.0);
        ginv = TP(PR::kHalf ? 1.0 / kGScaleHalf : 1.0);
    }
    __device__ __forceinline__ T load_f(const typename PR::Sf* p) const {
        if constexpr (PR::kHalf) return mul_rn(T(__half2float(*p)), finv);
        else return T(*p);
    }
    __device__ __forceinline__ void store_f(typename PR::Sf* p, T v) const {
        if constexpr (PR::kHalf) *p = __float2half_rn(float(mul_rn(v, fscale)));
        else *p = typename PR::Sf(v);
    }
    // stored g as it is kept: the deviation g - w_q c_s with kShift, else g itself
    __device__ __forceinline__ TP load_dev(const typename PR::Sg* p) const {
        if constexpr (PR::kHalf) return mul_rn(TP(__half2float(*p)), ginv);
        else return TP(*p);
    }
    __device__ __forceinline__ void store_dev(typename PR::Sg* p, TP v) const {
        if constexpr (PR::kHalf) *p = __float2half_rn(float(mul_rn(v, gscale)));
        else *p = typename PR::Sg(v);
    }
    // g itself, in FP64, from a value stored shifted by cs (output and inlet paths)
    template <int DIM>
    __device__ __forceinline__ double load_g_abs(const typename PR::Sg* p, int q, double cs) const {
        const double v = double(load_dev(p));
        return PR::kShift ? v + double(Lat<DIM>::ws(q)) * cs : v;
    }
    // store g (FP64 value) shifted by cs
    template <int DIM>
    __device__ __forceinline__ void store_g_abs(typename PR::Sg* p, int q, double v, double cs) const {
        store_dev(p, TP(PR::kShift ? v - double(Lat<DIM>::ws(q)) * cs : v));
    }
};

template <typename T>
__host__ __device__ __forceinline__ Phys<T> phys_cast(const PhysD& d) {
    Phys<T> p;
    p.RhoL = T(d.RhoL); p.RhoH = T(d.RhoH); p.drho = T(d.drho); p.drho3 = T(d.drho3);
    p.tauL = T(d.tauL); p.tauH = T(d.tauH); p.dtau = T(d.dtau);
    p.kappa = T(d.kappa); p.beta4 = T(d.beta4); p.mobility = T(d.mobility); p.W = T(d.W);
    p.wc = T(d.wc); p.one_minus_wc = T(d.one_minus_wc); p.amob3 = T(d.amob3);
    p.g[0] = T(d.g[0]); p.g[1] = T(d.g[1]); p.g[2] = T(d.g[2]);
    p.caseType = d.caseType;
    return p;
}

__device__ __forceinline__ long long nidx(const Geom& g, int x, int y, int z) {
    return g.base + x + (long long)y * g.sy + (long long)z * g.sz;
}

// 32-bit element index for the step kernels: every buffer holds fewer than 2^32 elements
// (Q * ps, checked when the solver is created), so index sums are exact modulo 2^32 and a
// load address is one 32 x 32 -> 64-bit multiply-add on the buffer base.
__device__ __forceinline__ unsigned nidx32(const Geom& g, int x, int y, int z) {
    return unsigned(g.base + x) + unsigned(y) * unsigned(g.sy) + unsigned(z) * unsigned(g.sz);
}
// offset from a node's index to the source of direction q in plane q of a population buffer
template <int DIM>
__device__ __forceinline__ unsigned pull_offset(const Geom& g, int q) {
    using L = Lat<DIM>;
    return unsigned(q) * unsigned(g.ps) - unsigned(L::ex(q)) - unsigned(L::ey(q)) * unsigned(g.sy) -
           (DIM == 3 ? unsigned(L::ez(q)) * unsigned(g.sz) : 0u);
}

// Value of c at a coordinate outside the interior, as the reference's ghost layer holds it
// when the macroscopic stencils run: mirror sides copy the adjacent interior node
// (Solver.cu:927-978), periodic axes copy the opposite interior node (Solver.cu:75-141),
// both from the previous step's c; a velocity-inlet plane keeps its own stored value.  A
// slab's exchange or wrap face keeps the stored value of its ghost plane (the neighbouring
// slab's c of the previous step), wrapped on the other periodic axes.
template <int DIM, typename A>
__device__ __forceinline__ A ghost_c(const A* C, const Geom& g, int x, int y, int z) {
    int s[3] = {x, y, z};
    bool vel = false;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        s[a] = s[a] < 0 ? 0 : (s[a] > g.n[a] + 1 ? g.n[a] + 1 : s[a]);
        if (s[a] < 1) {
            if (mirror_side(g.side[2 * a])) s[a] = 1;
            else if (g.side[2 * a] == kSideVelocity) vel = true;
        } else if (s[a] > g.n[a]) {
            if (mirror_side(g.side[2 * a + 1])) s[a] = g.n[a];
            else if (g.side[2 * a + 1] == kSideVelocity) vel = true;
        }
    }
    if (!vel) {
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            if (g.per[a]) {
                if (s[a] < 1) s[a] += g.n[a];
                else if (s[a] > g.n[a]) s[a] -= g.n[a];
            }
        }
    }
    return C[nidx(g, s[0], s[1], DIM == 3 ? s[2] : 0)];
}

// Source of population q streamed into interior node (x,y,z) (kernelStreaming,
// NsAllen.cu:327-364, followed by kernelHalfBounceBack, Solver.cu:248-333):
//   * if the source lies behind a wall: half-way bounce-back, the node's own opposite
//     population (qsrc = opposite(q), source = self);
//   * if it lies in a velocity-inlet plane: that ghost cell (corner cells included);
//   * otherwise the periodic image.
// `crossed` tells whether the source lies across the domain boundary (periodic image or
// inlet ghost cell): such values were stored shifted by the source's own c.
template <int DIM>
__device__ __forceinline__ long long pull_source(const Geom& g, int q, int x, int y, int z, long long self, int& qsrc,
                                                 bool& crossed) {
    using L = Lat<DIM>;
    int s[3] = {x - L::ex(q), y - L::ey(q), DIM == 3 ? z - L::ez(q) : 0};
    bool vel = false, out = false;
    crossed = false;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
        if (s[a] < 1) {
            if (g.side[2 * a] == kSideWall) {
                qsrc = opposite<DIM>(q);
                return self;
            }
            if (g.side[2 * a] == kSideVelocity) vel = true;
            // an exchange plane holds the neighbouring slab's values, stored as that slab's
            // interior stores them (shifted by this node's c): not a crossing
            if (g.side[2 * a] != kSideExchange) out = true;
        } else if (s[a] > g.n[a]) {
            if (g.side[2 * a + 1] == kSideWall) {
                qsrc = opposite<DIM>(q);
                return self;
            }
            if (g.side[2 * a + 1] == kSideVelocity) vel = true;
            if (g.side[2 * a + 1] != kSideExchange) out = true;
        }
    }
    if (!vel) {
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
            if (g.per[a]) {
                if (s[a] < 1) s[a] += g.n[a];
                else if (s[a] > g.n[a]) s[a] -= g.n[a];
            }
        }
    }
    crossed = out;
    qsrc = q;
    return nidx(g, s[0], s[1], s[2]);
}

// Directions with e_q along axis a equal to s, as a bit mask (bit q).
template <int DIM>
__host__ __device__ constexpr unsigned dir_mask(int a, int s) {
    unsigned m = 0;
    for (int q = 0; q < Lat<DIM>::Q; ++q) {
        const int e = a == 0 ? Lat<DIM>::ex(q) : (a == 1 ? Lat<DIM>::ey(q) : Lat<DIM>::ez(q));
        if (e == s) m |= 1u << q;
    }
    return m;
}

// Directions q whose source x - e_q (kDest: destination x + e_q) lies outside the interior.
// Zero for every node not next to the domain boundary.
template <int DIM, bool kDest = false>
__device__ __forceinline__ unsigned cross_mask(const Geom& g, int x, int y, int z) {
    constexpr int s = kDest ? -1 : 1;
    constexpr unsigned xp = dir_mask<DIM>(0, s), xm = dir_mask<DIM>(0, -s);
    constexpr unsigned yp = dir_mask<DIM>(1, s), ym = dir_mask<DIM>(1, -s);
    constexpr unsigned zp = dir_mask<DIM>(2, s), zm = dir_mask<DIM>(2, -s);
    unsigned m = (x == 1 ? xp : 0u) | (x == g.n[0] ? xm : 0u) | (y == 1 ? yp : 0u) | (y == g.n[1] ? ym : 0u);
    if (DIM == 3) m |= (z == 1 ? zp : 0u) | (z == g.n[2] ? zm : 0u);
    return m;
}

// Pull-streaming reads every direction at the fixed lattice offset (for a direction that
// crosses the domain boundary that read lands in the ghost layer, inside the allocation),
// then rereads the directions set in `mask` (cross_mask) with the source pull_source would
// give.  Per node (only when mask != 0) the boundary is summarised once:
//   bb      directions whose source lies behind a wall: the node's own opposite population
//   vel     directions whose source lies in a velocity-inlet plane: the ghost cell itself, no
//           periodic wrap on the other axes (the fixed-offset read is already right)
//   lo, hi  index corrections for a source beyond the low / high side of a periodic axis
//   open    directions entering across a free-convect or Neumann side (open_value)
//   corr    directions whose source lies across a side other than a slab's exchange face:
//           those values were stored shifted by the source's own c
// so that each reread costs a few integer operations.  A slab's exchange and wrap faces
// need no index correction: their ghost plane holds the neighbouring slab's values at the
// fixed offset (stored as an interior node's on an exchange face; as a periodic image on a
// wrap face, which is a crossing like the periodic wrap itself).
struct EdgeFix {
    unsigned bb, vel, open, corr;
    int lo[3], hi[3];
};

template <int DIM>
__device__ __forceinline__ EdgeFix edge_fix(const Geom& g, int x, int y, int z) {
    EdgeFix e;
    e.bb = 0u;
    e.vel = 0u;
    e.open = 0u;
    e.corr = 0u;
    const int c[3] = {x, y, z};
    const long long stride[3] = {1, g.sy, g.sz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        e.lo[a] = e.hi[a] = 0;
        if (a >= DIM) continue;
        const unsigned up = dir_mask<DIM>(a, 1), down = dir_mask<DIM>(a, -1);
        if (c[a] == 1) {  // sources at coordinate 0: directions with e_a = +1
            const int t = g.side[2 * a];
            if (t != kSideExchange) e.corr |= up;
            if (t == kSideWall) e.bb |= up;
            else if (t == kSideVelocity) e.vel |= up;
            else if (t == kSidePeriodic) e.lo[a] = int(g.n[a] * stride[a]);
            else if (t < kSideExchange) e.open |= up;
        }
        if (c[a] == g.n[a]) {  // sources at coordinate n + 1: directions with e_a = -1
            const int t = g.side[2 * a + 1];
            if (t != kSideExchange) e.corr |= down;
            if (t == kSideWall) e.bb |= down;
            else if (t == kSideVelocity) e.vel |= down;
            else if (t == kSidePeriodic) e.hi[a] = -int(g.n[a] * stride[a]);
            else if (t < kSideExchange) e.open |= down;
        }
    }
    // the free-convect and Neumann passes run after the bounce-back (NsAllen.cu:881-892)
    e.bb &= ~e.open;
    e.vel &= ~(e.bb | e.open);
    return e;
}

// Corrected source index of direction q (not bounce-back) for a node with summary e.
template <int DIM>
__device__ __forceinline__ unsigned fixed_source(const Geom& g, const EdgeFix& e, int q, unsigned self) {
    using L = Lat<DIM>;
    unsigned src = self + pull_offset<DIM>(g, q) - unsigned(q) * unsigned(g.ps);
    if (e.vel & (1u << q)) return src;
    const int ex = L::ex(q), ey = L::ey(q), ez = DIM == 3 ? L::ez(q) : 0;
    if (ex) src += unsigned(ex > 0 ? e.lo[0] : e.hi[0]);
    if (ey) src += unsigned(ey > 0 ? e.lo[1] : e.hi[1]);
    if (DIM == 3 && ez) src += unsigned(ez > 0 ? e.lo[2] : e.hi[2]);
    return src;
}

// Population q of interior node (x, y, z) as the reference leaves it after its
// free-convect and Neumann passes (kernelFreeConvect, kernelNeumann, Solver.cu:342-542), for
// a direction in EdgeFix::open.  The passes run in this order after streaming and the
// bounce-back (NsAllen.cu:881-892), each on the first interior layer of its sides:
//   * Neumann: the node takes the population of its inner neighbour x + n_s as the passes
//     before left it (when q enters across two Neumann sides, the side that the
//     reference's loop writes last: largest wallBCMap slot, then largest side);
//   * free convect (the last such side in the order x-, x+, y-, ...):
//     (prev + U pre) / (1 + U) with prev = the node's value of the last step (state in
//     Geom::fc[par]), pre = the inner neighbour's streamed or bounced value, U = |u_s| of
//     the inner neighbour's previous velocity;
//   * otherwise the streamed or bounced value (pull_source).
// kG: g, returned relative to cref, the reading node's stored c (shifted storage): every
// stored g is corrected by w_q (c of the node it was shifted by - cref).  Not inlined: the
// kernels reach it only for nodes on such sides.
template <int DIM, class PR, bool kG>
__device__ __noinline__ typename PR::TP open_value(const void* P, const typename PR::A* __restrict__ C,
                                                   const Codec<PR> cd, const Geom g, int par, int x, int y, int z,
                                                   int q, typename PR::TP cref) {
    using L = Lat<DIM>;
    using TP = typename PR::TP;
    const int e[3] = {L::ex(q), L::ey(q), L::ez(q)};
    int m[3] = {x, y, DIM == 3 ? z : 0};
    auto crossed = [&]() {
        unsigned sides = 0u;
        for (int a = 0; a < DIM; ++a) {
            if (m[a] - e[a] < 1) sides |= 1u << (2 * a);
            else if (m[a] - e[a] > g.n[a]) sides |= 1u << (2 * a + 1);
        }
        return sides;
    };
    unsigned cs = crossed();
    int best = -1, key = -1;
    for (int s = 0; s < 2 * DIM; ++s)
        if (((cs >> s) & 1u) && g.side[s] == kSideNeumann && wall_slot<DIM>(s, q) * 8 + s > key) {
            key = wall_slot<DIM>(s, q) * 8 + s;
            best = s;
        }
    if (best >= 0) {
        m[best / 2] += (best & 1) ? -1 : 1;
        cs = crossed();
    }
    // streamed or bounced value at node c, relative to cref
    auto level2 = [&](const int* c) -> TP {
        const long long ci = nidx(g, c[0], c[1], c[2]);
        int qs;
        bool out;
        const long long src = pull_source<DIM>(g, q, c[0], c[1], c[2], ci, qs, out);
        if constexpr (kG) {
            TP v = cd.load_dev(static_cast<const typename PR::Sg*>(P) + (src + (long long)qs * g.ps));
            if constexpr (PR::kShift) v = v + TP(L::ws(q)) * (TP(C[out ? src : ci]) - cref);
            return v;
        } else {
            (void)C;
            return cd.load_f(static_cast<const typename PR::Sf*>(P) + (src + (long long)qs * g.ps));
        }
    };
    best = -1;
    for (int s = 0; s < 2 * DIM; ++s)
        if (((cs >> s) & 1u) && g.side[s] == kSideFreeConvect) best = s;
    if (best < 0) return level2(m);
    const long long np = side_plane(g, best), pi = side_plane_index(g, best, m[0], m[1], m[2]);
    const TP* blk = static_cast<const TP*>(g.fc[par]) + g.fc_off[best];
    const int slot = wall_slot<DIM>(best, q);
    TP prev = blk[(kG ? L::A + slot : slot) * np + pi];
    if constexpr (kG && PR::kShift) prev = prev + TP(L::ws(q)) * (TP(C[nidx(g, m[0], m[1], m[2])]) - cref);
    const TP U = fabs(blk[2 * L::A * np + pi]);
    int nb[3] = {m[0], m[1], m[2]};
    nb[best / 2] += (best & 1) ? -1 : 1;
    const TP pre = level2(nb);
    return (prev + U * pre) / (TP(1.0) + U);
}

// Free-convect state that interior node (x, y, z) leaves for the next step (Geom::fc[par ^
// 1]): on a free-convect side's boundary layer, its entering populations after this step's
// boundary passes (the reference copies dev_f_post / dev_g_post to dev_f_prev / dev_g_prev
// before the next streaming, NsAllen.cu:849-853); g relative to this step's stored c.
template <int DIM, class PR, class Gq>
__device__ __forceinline__ void store_open(const Geom& g, int par, int x, int y, int z, const typename PR::T* fpost,
                                           Gq gpost, typename PR::TP c_old, typename PR::TP c_new) {
    using L = Lat<DIM>;
    using TP = typename PR::TP;
    const int c[3] = {x, y, z};
#pragma unroll
    for (int s = 0; s < 2 * DIM; ++s) {
        const int a = s / 2;
        if (g.side[s] != kSideFreeConvect || c[a] != ((s & 1) ? g.n[a] : 1)) continue;
        const long long np = side_plane(g, s), pi = side_plane_index(g, s, x, y, z);
        TP* blk = static_cast<TP*>(g.fc[par ^ 1]) + g.fc_off[s];
#pragma unroll
        for (int q = 0; q < L::Q; ++q) {
            const int slot = wall_slot<DIM>(s, q);
            if (slot < 0) continue;
            blk[slot * np + pi] = TP(fpost[q]);
            blk[(L::A + slot) * np + pi] = PR::kShift ? gpost(q) + TP(L::ws(q)) * (c_old - c_new) : gpost(q);
        }
    }
}

// The inner layer's velocity along a free-convect side's axis, read by the next step's
// free-convect pass as the previous velocity (Solver.cu:364); U holds this node's velocity
// of this step.
template <int DIM, class PR>
__device__ __forceinline__ void store_open_u(const Geom& g, int par, int x, int y, int z,
                                             const typename PR::A* __restrict__ U, unsigned self) {
    using TP = typename PR::TP;
    const int c[3] = {x, y, z};
#pragma unroll
    for (int s = 0; s < 2 * DIM; ++s) {
        const int a = s / 2;
        if (g.side[s] != kSideFreeConvect || c[a] != ((s & 1) ? g.n[a] - 1 : 2)) continue;
        const long long np = side_plane(g, s), pi = side_plane_index(g, s, x, y, z);
        TP* blk = static_cast<TP*>(g.fc[par ^ 1]) + g.fc_off[s];
        blk[2 * Lat<DIM>::A * np + pi] = TP(U[self + unsigned(a) * unsigned(g.ps)]);
    }
}

template <int DIM, class PR>
__device__ __forceinline__ void fix_f(const typename PR::Sf* __restrict__ F, const Codec<PR>& cd, const Geom& g, int x,
                                      int y, int z, unsigned self, unsigned mask, typename PR::T* v) {
    const EdgeFix e = edge_fix<DIM>(g, x, y, z);
#pragma unroll
    for (int q = 0; q < Lat<DIM>::Q; ++q) {
        if (!(mask & (1u << q))) continue;
        if (e.bb & (1u << q)) v[q] = cd.load_f(F + (self + unsigned(opposite<DIM>(q)) * unsigned(g.ps)));
        else v[q] = cd.load_f(F + (fixed_source<DIM>(g, e, q, self) + unsigned(q) * unsigned(g.ps)));
    }
}

template <int DIM, class PR>
__device__ __forceinline__ void fix_g(const typename PR::Sg* __restrict__ G, const typename PR::A* __restrict__ C,
                                      const Codec<PR>& cd, const Geom& g, int x, int y, int z, unsigned self,
                                      unsigned mask, typename PR::TP cself, typename PR::TP* v) {
    using TP = typename PR::TP;
    const EdgeFix e = edge_fix<DIM>(g, x, y, z);
#pragma unroll
    for (int q = 0; q < Lat<DIM>::Q; ++q) {
        if (!(mask & (1u << q))) continue;
        if (e.bb & (1u << q)) {
            v[q] = cd.load_dev(G + (self + unsigned(opposite<DIM>(q)) * unsigned(g.ps)));
        } else {
            // a source across the domain boundary (periodic image or inlet ghost) was
            // stored shifted by its own c
            const unsigned src = fixed_source<DIM>(g, e, q, self);
            v[q] = cd.load_dev(G + (src + unsigned(q) * unsigned(g.ps)));
            if (PR::kShift) v[q] = fma(TP(Lat<DIM>::ws(q)), TP(C[src]) - cself, v[q]);
        }
    }
}

// Pull the Q streamed populations of f (arithmetic T) into node (x,y,z); `mask` =
// cross_mask of the node.  A warp whose nodes are all away from the boundary reads the
// fixed offsets; any other warp reads the corrected sources (EdgeFix) in one round.
template <int DIM, class PR, bool kOpen = false>
__device__ __forceinline__ void pull_f(const typename PR::Sf* __restrict__ F, const Codec<PR>& cd, const Geom& g, int x,
                                       int y, int z, unsigned self, unsigned mask, typename PR::T* v, int par) {
    using L = Lat<DIM>;
    if (__any_sync(__activemask(), mask != 0u)) {
        // a warp holding a node next to the boundary reads every lane's corrected sources in
        // one round (zero corrections for its interior lanes)
        const EdgeFix e = edge_fix<DIM>(g, x, y, z);
#pragma unroll
        for (int q = 0; q < L::Q; ++q) {
            const unsigned idx = (e.bb & (1u << q)) ? self + unsigned(opposite<DIM>(q)) * unsigned(g.ps)
                                                    : fixed_source<DIM>(g, e, q, self) + unsigned(q) * unsigned(g.ps);
            v[q] = cd.load_f(F + idx);
        }
        if constexpr (kOpen) {
            if (e.open) {
#pragma unroll
                for (int q = 0; q < L::Q; ++q)
                    if (e.open & (1u << q))
                        v[q] = open_value<DIM, PR, false>(F, nullptr, cd, g, par, x, y, z, q, typename PR::TP(0));
            }
        } else {
            (void)par;
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < L::Q; ++q) v[q] = cd.load_f(F + (self + pull_offset<DIM>(g, q)));
}

// The same for g (arithmetic TP).  FP64 (no shift): v = g.  Shifted storage: v = g - w_q
// c_self (c_self = the node's stored c of the previous step, returned in `cself`); a
// source that crossed the domain boundary was shifted by its own c instead.
template <int DIM, class PR, bool kOpen = false>
__device__ __forceinline__ void pull_g(const typename PR::Sg* __restrict__ G, const typename PR::A* __restrict__ C,
                                       const Codec<PR>& cd, const Geom& g, int x, int y, int z, unsigned self,
                                       unsigned mask, typename PR::TP* v, typename PR::TP& cself, int par) {
    using L = Lat<DIM>;
    using TP = typename PR::TP;
    cself = PR::kShift ? TP(C[self]) : TP(0);
    if (__any_sync(__activemask(), mask != 0u)) {
        const EdgeFix e = edge_fix<DIM>(g, x, y, z);
#pragma unroll
        for (int q = 0; q < L::Q; ++q) {
            const bool bbq = e.bb & (1u << q);
            const unsigned src = fixed_source<DIM>(g, e, q, self);
            v[q] = cd.load_dev(G + (bbq ? self + unsigned(opposite<DIM>(q)) * unsigned(g.ps) : src + unsigned(q) * unsigned(g.ps)));
            // a source across the domain boundary was stored shifted by its own c
            if (PR::kShift && !bbq && (e.corr & (1u << q))) v[q] = fma(TP(L::ws(q)), TP(C[src]) - cself, v[q]);
        }
        if constexpr (kOpen) {
            if (e.open) {
#pragma unroll
                for (int q = 0; q < L::Q; ++q)
                    if (e.open & (1u << q)) v[q] = open_value<DIM, PR, true>(G, C, cd, g, par, x, y, z, q, cself);
            }
        } else {
            (void)par;
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < L::Q; ++q) v[q] = cd.load_dev(G + (self + pull_offset<DIM>(g, q)));
}

// c of a node from the sum of its pulled g in ascending q (kernelMacroscopicg,
// NsAllen.cu:516-540): the plain sum (FP64), or c_old + the sum of deviations as an
// unevaluated (stored c, remainder) pair (shifted storage).
template <class PR>
__device__ __forceinline__ typename PR::Ring ring_c(typename PR::TP sum, typename PR::TP cself) {
    if constexpr (PR::kExact) {
        (void)cself;
        return sum;
    } else {
        return two_sum(cself, sum);
    }
}
template <class PR>
__device__ __forceinline__ typename PR::Ring ring_of(typename PR::A c) {
    if constexpr (PR::kExact) return c;
    else return make_float2(c, 0.f);
}
// the stored c of a ring entry
template <class PR>
__device__ __forceinline__ typename PR::TP ring_hi(typename PR::Ring r) {
    if constexpr (PR::kExact) return r;
    else return r.x;
}

// mu and grad c: the reference's expression (FP64) or the difference form (FP32).
template <int DIM, class PR, class Cfun>
__device__ __forceinline__ void phase_stencil(const Phys<typename PR::TP>& P, Cfun C, typename PR::TP& mu,
                                              typename PR::TP* dc) {
    if constexpr (PR::kExact) stencil<DIM, typename PR::TP>(P, C, mu, dc);
    else stencil_hilo<DIM>(P, C, mu, dc);
}

// Shift values for the g written by an interior node (see Prec): c of each destination
// node x + e_q when it is interior, else the node's own stored c.  Cd(dx,dy,dz) returns
// this step's stored c around the node; dmask = cross_mask<DIM, true> of the node.
template <int DIM, class PR, typename V, class Cfun>
__device__ __forceinline__ void dest_shift(unsigned dmask, V cown, Cfun Cd, V* cs) {
    using L = Lat<DIM>;
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        if constexpr (!PR::kShift) cs[q] = cown;
        else cs[q] = Cd(L::ex(q), L::ey(q), DIM == 3 ? L::ez(q) : 0);
    }
    if (PR::kShift && dmask) {
#pragma unroll
        for (int q = 0; q < L::Q; ++q)
            if (dmask & (1u << q)) cs[q] = cown;
    }
}

template <class PR>
struct StepArgs {
    const typename PR::Sf* fin;
    const typename PR::Sg* gin;
    typename PR::Sf* fout;
    typename PR::Sg* gout;
    const typename PR::A* cin;
    typename PR::A* cout;
    typename PR::A* u;          // velocity written by the step
    const typename PR::A* uin;  // velocity read by the step (u itself, or another buffer)
    Geom g;
    PhysD phys;
    // the parameters in the step's arithmetic types, cast on the host: the kernels read them
    // from the parameter space, so they hold no registers
    Phys<typename PR::T> pt;
    Phys<typename PR::TP> pp;
    double pop_scale;
    int par;  // parity of the input buffers (step k reads parity k % 2)
    // 3D direct-load step only, when not null: per row segment of 32 nodes (x-tile, y, z)
    // the mass and kinetic energy of the step's stored c and u, as monitor_partials forms
    // them per node
    double* mon;
};

// Shift of direction q as dest_shift computes it, evaluated when it is needed.
template <int DIM, class PR, typename V, class Cfun>
__device__ __forceinline__ V dest_shift_q(int q, unsigned dmask, V cown, Cfun Cd) {
    using L = Lat<DIM>;
    if constexpr (!PR::kShift) return cown;
    else return (dmask & (1u << q)) ? cown : Cd(L::ex(q), L::ey(q), DIM == 3 ? L::ez(q) : 0);
}

// Macroscopic update and the next collision of one interior node, then its stores.
//   fpost (T): streamed f;  gpost(q) (TP): streamed g as pull_g returns it;
//   delta: sum of gpost(q) over q in ascending order (shifted storage only; the phase-field
//   sum of the node's c);  c_old: the node's stored c of the previous step (shifted storage
//   only);  c, mu, dc (TP): phase field of this step;  u: previous velocity in, this step's
//   out;  cdest(q): shift of each stored g (dest_shift_q).
// The FP32 path stores each output as soon as lean_update forms it.
// mon (not null): receives the node's mass and kinetic energy from its stored c and u, in
// FP64 as monitor_partials forms them.
template <int DIM, class PR, class Gq, class Cq>
__device__ __forceinline__ void update_node(const StepArgs<PR>& a, const Codec<PR>& cd, const Phys<typename PR::T>& PT,
                                            const Phys<typename PR::TP>& PP, unsigned self,
                                            const typename PR::T* fpost, Gq gpost, typename PR::TP delta,
                                            typename PR::TP c_old, typename PR::TP c, typename PR::TP mu,
                                            const typename PR::TP* dc, Cq cdest, double* mon = nullptr) {
    using T = typename PR::T;
    using TP = typename PR::TP;
    using A = typename PR::A;
    constexpr int Q = Lat<DIM>::Q;
    const Geom& g = a.g;
    A* U = a.u;
    T u[3];
#pragma unroll
    for (int d = 0; d < DIM; ++d) u[d] = T(a.uin[self + unsigned(d) * unsigned(g.ps)]);
    if constexpr (PR::kExact) {
        (void)c_old;
        (void)delta;
        (void)cdest;
        T fo[Q], p, rho;
        TP go[Q], gp[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) gp[q] = gpost(q);
        macroscopic<DIM, T>(PT, fpost, c, mu, dc, u, p, rho);
        collide_g<DIM, TP>(PP, gp, c, dc, u, go);  // Allen-Cahn relaxation
        // g is stored before the f collision, so its 19 values are not live through it
#pragma unroll
        for (int q = 0; q < Q; ++q) cd.store_dev(a.gout + (self + unsigned(q) * unsigned(g.ps)), go[q]);
        collide_f<DIM, T>(PT, fpost, c, mu, dc, rho, p, u, fo);  // force-corrected WMRT relaxation
#pragma unroll
        for (int q = 0; q < Q; ++q) cd.store_f(a.fout + (self + unsigned(q) * unsigned(g.ps)), fo[q]);
    } else {
        T p;
        lean_update<DIM>(PT, fpost, gpost, delta, c_old, c, mu, dc, u, cdest, p, [&](int q, T fo, TP go) {
            cd.store_dev(a.gout + (self + unsigned(q) * unsigned(g.ps)), go);
            cd.store_f(a.fout + (self + unsigned(q) * unsigned(g.ps)), fo);
        });
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d) U[self + unsigned(d) * unsigned(g.ps)] = A(u[d]);
    a.cout[self] = A(c);
    if (mon) {
        const double cs = double(A(c));
        double u2 = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
            const double v = double(A(u[d]));
            u2 += v * v;
        }
        mon[0] = cs;
        mon[1] = 0.5 * (a.phys.RhoL + cs * a.phys.drho) * u2;
    }
}

// Sum of the Q pulled values in ascending q (the order of ring_c and of lean_update's delta).
template <class PR, int Q>
__device__ __forceinline__ typename PR::TP pulled_sum(const typename PR::TP* v) {
    typename PR::TP c = v[0];
#pragma unroll
    for (int q = 1; q < Q; ++q) c = c + v[q];
    return c;
}

// ---------------------------------------------------------------- init + first collision
// Initial state of one node from the uploaded c (read through `C0`): chemical potential,
// gradient and normal on interior nodes (NsAllen.cu:897-905; ghost nodes keep zero
// normals), then KernelInitializeDistributions (NsAllen.cu:137-202).
template <int DIM, typename T, class Cfun>
__device__ __forceinline__ void initial_state(const PhysD& pd, T sigma, const Phys<T>& P, Cfun C0, bool interior, T& c,
                                              T& mu, T* dc, T& rho, T& p, T* f0, T* g0) {
    using L = Lat<DIM>;
    c = C0(0, 0, 0);
    mu = T(0);
    dc[0] = dc[1] = dc[2] = T(0);
    T nrm[3] = {T(0), T(0), T(0)};
    if (interior) {
        stencil<DIM, T>(P, C0, mu, dc);
        interface_normal<DIM>(P, c, dc, nrm);
    }
    rho = (P.RhoL) + c * P.drho;
    if (pd.caseType == 0) p = T(0) - c * sigma / (T(pd.refLen) / T(2.0)) / (rho / T(3.0));
    else if (pd.caseType == 1) p = T(0) + c * sigma / (T(pd.refLen) / T(2.0)) / (rho / T(3.0));
    else p = T(0);
    const T zero = T(0);
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        const T ga_wa = equilibrium<DIM, T>(q, zero, zero, zero, zero);
        const T hlp = T(L::w(q)) * ((T(1.0) - T(4.0) * ((c - T(0.50)) * (c - T(0.50)))) / P.W *
                                    edot<DIM, T>(q, nrm[0], nrm[1], nrm[2]));
        const T Gamma = ga_wa + T(L::w(q));
        g0[q] = c * Gamma - T(0.50) * hlp;
        f0[q] = p * T(L::w(q)) + ga_wa;
    }
}

// Every node: initial state (FP64); interior nodes then take the first collision of
// solve() (NsAllen.cu:830-842) into buffer 0, ghost nodes keep the initial populations in
// both buffers (their storage only matters on a velocity-inlet plane).  The f collision is
// the reference's literal sequence for the FP64 path and its closed form at u = 0
// (first_collide_f) for the FP32/FP16 paths.
template <int DIM, class PR>
// z_first: ghosted plane of blockIdx.z = 0 (3D; the initial state of a range of planes,
// which needs the initial c of the planes next to it).
__global__ void __launch_bounds__(256, 2) init_kernel(DevState st, int z_first) {
    using T = typename PR::T;
    using A = typename PR::A;
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    const Geom& g = st.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = DIM == 3 ? z_first + (int)blockIdx.z : 0;
    if (x >= g.e[0] || y >= g.e[1]) return;
    const Phys<double> PD = phys_cast<double>(st.phys);
    const long long self = nidx(g, x, y, z);
    const double* C0 = st.c0;
    const bool interior = x >= 1 && x <= g.n[0] && y >= 1 && y <= g.n[1] && (DIM == 2 || (z >= 1 && z <= g.n[2]));
    auto Cf = [&](int dx, int dy, int dz) { return C0[nidx(g, x + dx, y + dy, z + dz)]; };
    double c, mu, dc[3], rho, p, f0[Q], g0[Q];
    initial_state<DIM, double>(st.phys, st.phys.sigma, PD, Cf, interior, c, mu, dc, rho, p, f0, g0);
    const Codec<PR> cd(st.pop_scale);
    A* U = static_cast<A*>(st.u);
    for (int d = 0; d < DIM; ++d) U[(long long)d * g.ps + self] = A(0);
    static_cast<A*>(st.p)[self] = A(p);
    const A c_store = A(c);
    static_cast<A*>(st.c[0])[self] = c_store;
    static_cast<A*>(st.c[1])[self] = c_store;
    if (interior && g.fc[0]) {
        // free-convect state read by step 0: the initial populations on each free-convect
        // boundary layer (the reference's dev_f_post / dev_g_post after init) and the
        // initial velocity (zero) of the layer inside it
        using TP = typename PR::TP;
        for (int s = 0; s < 2 * DIM; ++s) {
            if (g.side[s] != kSideFreeConvect) continue;
            const int a = s / 2, ca = a == 0 ? x : (a == 1 ? y : z);
            const long long np = side_plane(g, s), pi = side_plane_index(g, s, x, y, z);
            TP* blk = static_cast<TP*>(g.fc[0]) + g.fc_off[s];
            if (ca == ((s & 1) ? g.n[a] : 1)) {
                // q runs over compile-time indices (f0, g0 stay in registers)
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const int i = wall_slot<DIM>(s, q);
                    if (i < 0) continue;
                    blk[i * np + pi] = TP(f0[q]);
                    blk[(L::A + i) * np + pi] = PR::kShift ? TP(g0[q] - double(L::ws(q)) * double(c_store)) : TP(g0[q]);
                }
            }
            if (ca == ((s & 1) ? g.n[a] - 1 : 2)) blk[2 * L::A * np + pi] = TP(0);
        }
    }
    auto* F0 = static_cast<typename PR::Sf*>(st.f[0]);
    auto* G0 = static_cast<typename PR::Sg*>(st.gp[0]);
    if (interior) {
        // first collision in FP64 for every precision (FP64: the reference's sequence)
        const double u0[3] = {0.0, 0.0, 0.0};
        double go[Q], fo[Q], cdest[Q];
        collide_g<DIM, double>(PD, g0, c, dc, u0, go);
        auto Cd = [&](int dx, int dy, int dz) { return double(A(Cf(dx, dy, dz))); };
        dest_shift<DIM, PR>(cross_mask<DIM, true>(g, x, y, z), double(c_store), Cd, cdest);
#pragma unroll
        for (int q = 0; q < Q; ++q) cd.template store_g_abs<DIM>(G0 + (long long)q * g.ps + self, q, go[q], cdest[q]);
        if constexpr (PR::kExact) collide_f<DIM, double>(PD, f0, c, mu, dc, rho, p, u0, fo);
        else first_collide_f<DIM, double>(PD, mu, dc, rho, p, fo);
#pragma unroll
        for (int q = 0; q < Q; ++q) cd.store_f(F0 + (long long)q * g.ps + self, T(fo[q]));
    } else {
        for (int b = 0; b < 2; ++b) {
            auto* Fb = static_cast<typename PR::Sf*>(st.f[b]);
            auto* Gb = static_cast<typename PR::Sg*>(st.gp[b]);
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                cd.store_f(Fb + (long long)q * g.ps + self, T(f0[q]));
                cd.template store_g_abs<DIM>(Gb + (long long)q * g.ps + self, q, g0[q], double(c_store));
            }
        }
    }
}

// ---------------------------------------------------------------- chained launches
// Programmatic dependent launch for chains of short kernels (the adjoint's reverse sweep;
// the fused steps of a small 2D grid measured slower chained): launch_chained lets the
// next kernel of the stream be dispatched while this one runs (launch_dependents), and
// chain_wait, first in such a kernel, waits until its predecessor has completed with its
// writes visible (griddepcontrol.wait: a hardware dependency, not a spin; after an
// ordinary launch it returns at once).
__device__ __forceinline__ void chain_wait() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename... P, typename... Args>
cudaError_t launch_chained(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// ---------------------------------------------------------------- fused step, 3D
// CTA = TX x TY tile of an (x,y) plane, marching in z over a segment of `seg` planes.
// Per plane: (1) pull g of plane z+1 for the tile and its one-node halo ring and reduce it
// to c (halo values recomputed, domain ghosts mapped from the previous c) into a 3-plane
// shared-memory ring; (2) for plane z: mu and grad c from the ring, pull f, macroscopic
// update, collision, store.  The ring has four plane slots: the slot written for plane
// z+2 was last read by the update of plane z-1, which every thread finished before the
// barrier of plane z, so one barrier per plane suffices.
// Ring-slot index of halo node h of a TX x TY tile (the ring of the (TX+2) x (TY+2) box).
template <int TX, int TY>
__device__ __forceinline__ void halo_coords(int h, int& hx, int& hy) {
    constexpr int HX = TX + 2, HY = TY + 2;
    if (h < HX) { hx = h; hy = 0; }
    else if (h < 2 * HX) { hx = h - HX; hy = HY - 1; }
    else if (h < 2 * HX + TY) { hx = 0; hy = 1 + (h - 2 * HX); }
    else { hx = HX - 1; hy = 1 + (h - 2 * HX - TY); }
}

// The 3D step of one CTA with loads straight from global memory.  `ring` is the CTA's
// 4-plane phase-field ring of (TX+2)*(TY+2) values.  Only nodes next to a boundary take the
// boundary-aware pull.  Every per-node code path appears once (one box loop, one update),
// which keeps the kernel's code small enough for the instruction caches.
// kKeep: 0 the update pulls g again; 1 the c phase keeps the node's pulled g (and c_old)
// in registers for the update of the next iteration; 2 the same in shared memory
// (keep_s: 2 x (Q + 1) x TX*TY values, private to each thread), which leaves registers
// for a higher occupancy.
// kOpen: the instance for cases with free-convect or Neumann sides (open_value calls and
// free-convect state); the other instance carries neither.
// kMon: the instance of a monitored step (writes a.mon); plain steps carry none of it.
template <class PR, int TX, int TY, int kKeep, bool kOpen = false, bool kMon = false>
__device__ __forceinline__ void step3d_body(const StepArgs<PR>& a, int seg, int bx, int by, int bz,
                                            typename PR::Ring (*ring)[(TX + 2) * (TY + 2)],
                                            typename PR::TP* keep_s = nullptr) {
    constexpr bool kKeepG = kKeep == 1;
    using TP = typename PR::TP;
    using R = typename PR::Ring;
    using T = typename PR::T;
    using A = typename PR::A;
    using L = Lat<3>;
    constexpr int Q = L::Q;
    constexpr int HX = TX + 2, NT = TX * TY;
    const Geom& g = a.g;
    const Phys<T>& PT = a.pt;
    const Phys<TP>& PP = a.pp;
    const Codec<PR> cd(a.pop_scale);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int x0 = 1 + bx * TX, y0 = 1 + by * TY;
    const int x = x0 + tx, y = y0 + ty;
    const int z0 = g.zlo + bz * seg;
    const int z1 = min(z0 + seg, g.zhi + 1);
    const bool active = x <= g.n[0] && y <= g.n[1];

    constexpr int NBOX = HX * (TY + 2);
    TP gcur[kKeepG ? Q : 1], gnext[kKeepG ? Q : 1], ccur = TP(0), cnext = TP(0), dcur = TP(0), dnext = TP(0);
    // Iteration cz: phase field of plane cz for the tile and its halo (box index k: the
    // tile's own nodes first, k = tid, then the halo ring), then the update of plane cz - 1.
    for (int cz = z0 - 1; cz <= z1; ++cz) {
        {
            const bool keep = kKeepG && cz >= z0 && cz < z1;
            R* slot = ring[cz & 3];
            for (int k = tid; k < NBOX; k += NT) {
                int hx, hy;
                if (k < NT) {
                    hx = tx + 1;
                    hy = ty + 1;
                } else {
                    halo_coords<TX, TY>(k - NT, hx, hy);
                }
                const int cx = x0 - 1 + hx, cy = y0 - 1 + hy;
                R cval;
                if (cx < 1 || cx > g.n[0] || cy < 1 || cy > g.n[1] || cz < 1 || cz > g.n[2]) {
                    cval = ring_of<PR>(ghost_c<3, A>(a.cin, g, cx, cy, cz));
                } else {
                    TP v[Q], cs;
                    pull_g<3, PR, kOpen>(a.gin, a.cin, cd, g, cx, cy, cz, nidx32(g, cx, cy, cz), cross_mask<3>(g, cx, cy, cz),
                                         v, cs, a.par);
                    const TP sum = pulled_sum<PR, Q>(v);
                    if (keep && k < NT) {
#pragma unroll
                        for (int q = 0; q < (kKeepG ? Q : 1); ++q) gnext[q] = v[q];
                        cnext = cs;
                        dnext = sum;
                    }
                    if (kKeep == 2 && cz >= z0 && cz < z1 && k < NT) {
                        TP* ks = keep_s + (cz & 1) * (Q + 2) * NT + tid;
#pragma unroll
                        for (int q = 0; q < Q; ++q) ks[q * NT] = v[q];
                        ks[Q * NT] = cs;
                        ks[(Q + 1) * NT] = sum;
                    }
                    cval = ring_c<PR>(sum, cs);
                }
                slot[hy * HX + hx] = cval;
            }
        }
        __syncthreads();
        const int z = cz - 1;  // plane updated in this iteration
        double mon2[2] = {0.0, 0.0};
        if (z >= z0 && active) {
            const unsigned self = nidx32(g, x, y, z);
            const unsigned mask = cross_mask<3>(g, x, y, z);
            auto Cf = [&](int dx, int dy, int dz) -> R { return ring[(z + dz) & 3][(ty + 1 + dy) * HX + tx + 1 + dx]; };
            auto Ch = [&](int dx, int dy, int dz) -> TP { return ring_hi<PR>(Cf(dx, dy, dz)); };
            TP mu, dc[3];
            phase_stencil<3, PR>(PP, Cf, mu, dc);
            T fpost[Q];
            pull_f<3, PR, kOpen>(a.fin, cd, g, x, y, z, self, mask, fpost, a.par);
            const unsigned dmask = cross_mask<3, true>(g, x, y, z);
            const TP cown = Ch(0, 0, 0);
            auto cdest = [&](int q) { return dest_shift_q<3, PR>(q, dmask, cown, Ch); };
            if constexpr (kKeepG) {
                auto gq = [&](int q) { return gcur[q]; };
                // next to the boundary the kept values are the boundary-aware pull as well
                if (kOpen && g.fc[0]) store_open<3, PR>(g, a.par, x, y, z, fpost, gq, ccur, cown);
                update_node<3, PR>(a, cd, PT, PP, self, fpost, gq, dcur, ccur, cown, mu, dc, cdest, kMon ? mon2 : nullptr);
            } else if constexpr (kKeep == 2) {
                const TP* ks = keep_s + (z & 1) * (Q + 2) * NT + tid;
                auto gq = [&](int q) { return ks[q * NT]; };
                if (kOpen && g.fc[0]) store_open<3, PR>(g, a.par, x, y, z, fpost, gq, ks[Q * NT], cown);
                update_node<3, PR>(a, cd, PT, PP, self, fpost, gq, ks[(Q + 1) * NT], ks[Q * NT], cown, mu, dc, cdest,
                                   kMon ? mon2 : nullptr);
            } else {
                TP gpost[Q], cold;
                pull_g<3, PR, kOpen>(a.gin, a.cin, cd, g, x, y, z, self, mask, gpost, cold, a.par);
                auto gq = [&](int q) { return gpost[q]; };
                if (kOpen && g.fc[0]) store_open<3, PR>(g, a.par, x, y, z, fpost, gq, cold, cown);
                update_node<3, PR>(a, cd, PT, PP, self, fpost, gq, pulled_sum<PR, Q>(gpost), cold, cown, mu, dc,
                                   cdest, kMon ? mon2 : nullptr);
            }
            if (kOpen && g.fc[0]) store_open_u<3, PR>(g, a.par, x, y, z, a.u, self);
        }
        // monitored step: each warp (32 consecutive x of one row) sums its nodes' mass and
        // kinetic energy in a fixed tree into one entry per row segment, so the result does
        // not depend on the tile shape or the planes per CTA
        if (kMon && z >= z0) {
            double m = mon2[0], k = mon2[1];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                m += __shfl_down_sync(0xffffffffu, m, off);
                k += __shfl_down_sync(0xffffffffu, k, off);
            }
            const int nxs = (g.n[0] + 31) / 32, xs = (x0 - 1 + (tx & ~31)) / 32;
            if ((tx & 31) == 0 && y <= g.n[1] && xs < nxs) {
                const long long row = ((long long)(z - g.zlo) * g.n[1] + (y - 1)) * nxs + xs;
                a.mon[2 * row] = m;
                a.mon[2 * row + 1] = k;
            }
        }
        if constexpr (kKeepG) {
#pragma unroll
            for (int q = 0; q < Q; ++q) gcur[q] = gnext[q];
            ccur = cnext;
            dcur = dnext;
        }
    }
}

template <class PR, int TX, int TY, bool kKeepG, bool kOpen = false, bool kMon = false>
__global__ void __launch_bounds__(TX * TY) step3d_kernel(StepArgs<PR> a, int seg) {
    __shared__ typename PR::Ring ring[4][(TX + 2) * (TY + 2)];
    step3d_body<PR, TX, TY, kKeepG ? 1 : 0, kOpen, kMon>(a, seg, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z,
                                                         ring);
}

// The same with the kept g in dynamic shared memory (2 x (Q + 1) x TX*TY values) and at
// least kMinBlocks resident blocks per SM.
template <class PR, int TX, int TY, int kMinBlocks, bool kOpen = false, bool kMon = false>
__global__ void __launch_bounds__(TX * TY, kMinBlocks) step3d_smemkeep_kernel(StepArgs<PR> a, int seg) {
    __shared__ typename PR::Ring ring[4][(TX + 2) * (TY + 2)];
    extern __shared__ __align__(16) unsigned char keep_raw[];
    step3d_body<PR, TX, TY, 2, kOpen, kMon>(a, seg, (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, ring,
                                      reinterpret_cast<typename PR::TP*>(keep_raw));
}

// ---------------------------------------------------------------- fused step, 2D
// CTA = TX consecutive x of a row (tile bx), marching in y over the `seg` rows of segment
// by; the c ring holds four rows of TX + 2 values (one barrier per row, as in the 3D
// kernel).  Used by the single-case kernel and by the batched kernel.
template <class PR, int TX, bool kKeepG, bool kOpen = false>
__device__ __forceinline__ void step2d_body(const StepArgs<PR>& a, int seg, int bx, int by,
                                            typename PR::Ring (*ring)[TX + 2]) {
    using TP = typename PR::TP;
    using T = typename PR::T;
    using A = typename PR::A;
    using L = Lat<2>;
    constexpr int Q = L::Q;
    using R = typename PR::Ring;
    constexpr int HX = TX + 2;
    const Geom& g = a.g;
    // the parameters as locals: the batched step passes `a` in shared memory, where every
    // use through a reference would be a load
    const Phys<T> PT = a.pt;
    const Phys<TP> PP = a.pp;
    const Codec<PR> cd(a.pop_scale);
    const int tx = threadIdx.x;
    const int x0 = 1 + bx * TX;
    const int x = x0 + tx;
    const int y0 = 1 + by * seg;
    const int y1 = min(y0 + seg, g.n[1] + 1);
    const bool active = x <= g.n[0];

    TP gcur[kKeepG ? Q : 1], gnext[kKeepG ? Q : 1], ccur = TP(0), cnext = TP(0), dcur = TP(0), dnext = TP(0);
    // Iteration cy: c of row cy for the segment and its two halo nodes (threads 0 and 1),
    // then the update of row cy - 1.
    for (int cy = y0 - 1; cy <= y1; ++cy) {
        {
            const bool keep = kKeepG && cy >= y0 && cy < y1;
            R* slot = ring[cy & 3];
            for (int k = tx; k < TX + 2; k += TX) {
                const int hx = k < TX ? tx + 1 : (k == TX ? 0 : TX + 1);
                const int cx = x0 - 1 + hx;
                R cval;
                if (cx < 1 || cx > g.n[0] || cy < 1 || cy > g.n[1]) {
                    cval = ring_of<PR>(ghost_c<2, A>(a.cin, g, cx, cy, 0));
                } else {
                    TP v[Q], cs;
                    pull_g<2, PR, kOpen>(a.gin, a.cin, cd, g, cx, cy, 0, nidx32(g, cx, cy, 0), cross_mask<2>(g, cx, cy, 0), v,
                                         cs, a.par);
                    const TP sum = pulled_sum<PR, Q>(v);
                    if (keep && k < TX) {
#pragma unroll
                        for (int q = 0; q < (kKeepG ? Q : 1); ++q) gnext[q] = v[q];
                        cnext = cs;
                        dnext = sum;
                    }
                    cval = ring_c<PR>(sum, cs);
                }
                slot[hx] = cval;
            }
        }
        __syncthreads();
        const int y = cy - 1;  // row updated in this iteration
        if (y >= y0 && active) {
            const unsigned self = nidx32(g, x, y, 0);
            const unsigned mask = cross_mask<2>(g, x, y, 0);
            auto Cf = [&](int dx, int dy, int) -> R { return ring[(y + dy) & 3][tx + 1 + dx]; };
            auto Ch = [&](int dx, int dy, int dz) -> TP { return ring_hi<PR>(Cf(dx, dy, dz)); };
            TP mu, dc[3] = {TP(0), TP(0), TP(0)};
            phase_stencil<2, PR>(PP, Cf, mu, dc);
            T fpost[Q];
            pull_f<2, PR, kOpen>(a.fin, cd, g, x, y, 0, self, mask, fpost, a.par);
            const unsigned dmask = cross_mask<2, true>(g, x, y, 0);
            const TP cown = Ch(0, 0, 0);
            auto cdest = [&](int q) { return dest_shift_q<2, PR>(q, dmask, cown, Ch); };
            if constexpr (kKeepG) {
                auto gq = [&](int q) { return gcur[q]; };
                if (kOpen && g.fc[0]) store_open<2, PR>(g, a.par, x, y, 0, fpost, gq, ccur, cown);
                update_node<2, PR>(a, cd, PT, PP, self, fpost, gq, dcur, ccur, cown, mu, dc, cdest);
            } else {
                TP gpost[Q], cold;
                pull_g<2, PR, kOpen>(a.gin, a.cin, cd, g, x, y, 0, self, mask, gpost, cold, a.par);
                auto gq = [&](int q) { return gpost[q]; };
                if (kOpen && g.fc[0]) store_open<2, PR>(g, a.par, x, y, 0, fpost, gq, cold, cown);
                update_node<2, PR>(a, cd, PT, PP, self, fpost, gq, pulled_sum<PR, Q>(gpost), cold, cown, mu, dc,
                                   cdest);
            }
            if (kOpen && g.fc[0]) store_open_u<2, PR>(g, a.par, x, y, 0, a.u, self);
        }
        if constexpr (kKeepG) {
#pragma unroll
            for (int q = 0; q < Q; ++q) gcur[q] = gnext[q];
            ccur = cnext;
            dcur = dnext;
        }
    }
}

// FP32/FP16: at most 64 registers, so that 1024 threads (32 warps) fit on an SM: the 2D
// grids are small and latency-bound (256x1024 RTI: 25% faster than at the compiler's 80-96
// registers, no spills).  FP64 keeps its registers.
template <class PR, int TX>
constexpr int kMinBlocks2 = PR::kExact ? 1 : 1024 / TX;

template <class PR, int TX, bool kKeepG, bool kOpen = false>
__global__ void __launch_bounds__(TX, (kMinBlocks2<PR, TX>)) step2d_kernel(StepArgs<PR> a, int seg) {
    __shared__ typename PR::Ring ring[4][TX + 2];
    step2d_body<PR, TX, kKeepG, kOpen>(a, seg, (int)blockIdx.x, (int)blockIdx.y, ring);
}

// One step of many independent 2D cases in one persistent launch.  A work item is
// (case, tile bx, row segment by); CTA b takes items b, b + gridDim.x, ...  The case's step
// arguments (this step's buffers, geometry, physics) are copied from the device table into
// shared memory per item.  items: 3 ints per item.
template <class PR, int TX, bool kKeepG>
__global__ void __launch_bounds__(TX, (kMinBlocks2<PR, TX>)) step2d_batch_kernel(const StepArgs<PR>* __restrict__ args,
                                                          const int* __restrict__ items, int nitems, int seg) {
    __shared__ typename PR::Ring ring[4][TX + 2];
    __shared__ StepArgs<PR> sa;
    static_assert(sizeof(StepArgs<PR>) % 4 == 0, "copied in 4-byte words");
    constexpr int W = sizeof(StepArgs<PR>) / 4;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int c = items[3 * it], bx = items[3 * it + 1], by = items[3 * it + 2];
        const unsigned* src = reinterpret_cast<const unsigned*>(args + c);
        unsigned* dst = reinterpret_cast<unsigned*>(&sa);
        for (int w = threadIdx.x; w < W; w += TX) dst[w] = src[w];
        __syncthreads();
        step2d_body<PR, TX, kKeepG>(sa, seg, bx, by, ring);
        __syncthreads();  // ring and sa are reused by the next item
    }
}

// ---------------------------------------------------------------- velocity inlet
// JetBoundary (Solver.cu:550-921) on the ghost plane of the velocity side, before step k,
// in FP64.  Old ghost state is read from buffer (k+1)%2 (written before step k-1) and the
// new state is written into buffer k%2, the input of step k.  Periodic copies into the
// plane's edge cells (Solver.cu:75-141, which run first in the reference) are taken from
// the wrapped plane cell's old state.  Every inlet value comes from the y+ entry of the
// boundary list, as in the reference (Solver.cu:587-588).
template <int DIM, class PR>
__global__ void inlet_kernel(DevState st, long long k) {
    using A = typename PR::A;
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    const Geom& g = st.g;
    const int side = g.vel_side;
    const int ax = side / 2;
    const bool plus = side & 1;
    const int a1 = ax == 0 ? 1 : 0;
    const int a2 = DIM == 3 ? (ax == 2 ? 1 : 2) : -1;
    const int i1 = blockIdx.x * blockDim.x + threadIdx.x;
    const int i2 = DIM == 3 ? (int)(blockIdx.y * blockDim.y + threadIdx.y) : 0;
    if (i1 > g.n[a1] + 1) return;
    if (DIM == 3 && i2 > g.n[a2] + 1) return;
    int cell[3] = {0, 0, 0};
    cell[ax] = plus ? g.n[ax] + 1 : 0;
    cell[a1] = i1;
    if (DIM == 3) cell[a2] = i2;
    const int cur = (int)(k & 1), old = cur ^ 1;
    const Codec<PR> cd(st.pop_scale);
    const auto* Fo = static_cast<const typename PR::Sf*>(st.f[old]);
    const auto* Go = static_cast<const typename PR::Sg*>(st.gp[old]);
    const A* Co = static_cast<const A*>(st.c[old]);
    auto* Fn = static_cast<typename PR::Sf*>(st.f[cur]);
    auto* Gn = static_cast<typename PR::Sg*>(st.gp[cur]);
    A* Cn = static_cast<A*>(st.c[cur]);

    int src[3] = {cell[0], cell[1], cell[2]};
    for (int b = 0; b < DIM; ++b) {
        if (b == ax || !g.per[b]) continue;
        if (src[b] < 1) src[b] += g.n[b];
        else if (src[b] > g.n[b]) src[b] -= g.n[b];
    }
    const long long sidx = nidx(g, src[0], src[1], DIM == 3 ? src[2] : 0);
    const long long self = nidx(g, cell[0], cell[1], DIM == 3 ? cell[2] : 0);
    double f[Q], gg[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        f[q] = double(cd.load_f(Fo + (long long)q * g.ps + sidx));
        gg[q] = cd.template load_g_abs<DIM>(Go + (long long)q * g.ps + sidx, q, double(Co[sidx]));
    }
    double c = double(Co[sidx]);
    auto e_ax = [&](int q) { return ax == 0 ? L::ex(q) : (ax == 1 ? L::ey(q) : L::ez(q)); };
    const int inward = plus ? -1 : 1;
    if (signed_distance(st.geo, 0, double(cell[0]), double(cell[1]), DIM == 3 ? double(cell[2]) : 0.0, DIM) <= 0) {
        const double V[3] = {st.inlet[0], st.inlet[1], st.inlet[2]};
        const double V2 = usq<DIM, double>(V[0], V[1], V[2]);
        double feq[Q], geq[Q];
        double M1 = 0.0, M2 = 0.0, N = 0.0;
        bool m1f = true, m2f = true, nf = true;
        // tangential axes in index order (Solver.cu:580-599, 700-719, 823-837)
        const int t1 = ax == 0 ? 1 : 0;
        const int t2 = ax == 2 ? 1 : 2;
#pragma unroll
        for (int q = 1; q < Q; ++q) {
            const double fa_wa = equilibrium<DIM, double>(q, V[0], V[1], V[2], V2);
            feq[q] = 0.0 * L::w(q) + fa_wa;
            geq[q] = c * (fa_wa + L::w(q));
            if (e_ax(q) == 0) {
                const int e1 = t1 == 0 ? L::ex(q) : L::ey(q);
                const double d1 = f[q] - feq[q];
                if (e1 != 0) {
                    const double t = e1 > 0 ? d1 : -d1;
                    M1 = m1f ? t : M1 + t;
                    m1f = false;
                }
                if (DIM == 3) {
                    const int e2 = t2 == 1 ? L::ey(q) : L::ez(q);
                    if (e2 != 0) {
                        const double t = e2 > 0 ? d1 : -d1;
                        M2 = m2f ? t : M2 + t;
                        m2f = false;
                    }
                }
                const double dn = gg[q] - geq[q];
                N = nf ? dn : N + dn;
                nf = false;
            }
        }
        const double invw = 1.0 / double(L::kWeight);
#pragma unroll
        for (int q = 1; q < Q; ++q) {
            if (e_ax(q) != inward) continue;
            const int od = opposite<DIM>(q);
            const int e1 = t1 == 0 ? L::ex(q) : L::ey(q);
            double corr = e1 == 0 ? 0.0 : (e1 > 0 ? M1 : -M1);
            if (DIM == 3) {
                const int e2 = t2 == 1 ? L::ey(q) : L::ez(q);
                if (e2 != 0) corr = (e1 == 0) ? (e2 > 0 ? M2 : -M2) : corr + (e2 > 0 ? M2 : -M2);
            }
            f[q] = f[od] + feq[q] - feq[od] - invw * corr;
            // the first direction of each wall map is the axis-aligned one (WMRT.cuh:220-234)
            const bool axis_aligned = (L::ex(q) != 0) + (L::ey(q) != 0) + (L::ez(q) != 0) == 1;
            gg[q] = axis_aligned ? geq[q] - (gg[od] - geq[od]) : geq[q] - (gg[od] - geq[od]) - N / double(L::kWeight);
        }
    } else {
        // outside the inlet mask: copy the adjacent interior node (Solver.cu:618-631)
        int adj[3] = {cell[0], cell[1], cell[2]};
        adj[ax] = plus ? g.n[ax] : 1;
        for (int b = 0; b < DIM; ++b) {
            if (b == ax) continue;
            if (adj[b] < 1) adj[b] = g.per[b] ? adj[b] + g.n[b] : 1;
            else if (adj[b] > g.n[b]) adj[b] = g.per[b] ? adj[b] - g.n[b] : g.n[b];
        }
        const long long aidx = nidx(g, adj[0], adj[1], DIM == 3 ? adj[2] : 0);
        const auto* Fi = static_cast<const typename PR::Sf*>(st.f[cur]);
        const auto* Gi = static_cast<const typename PR::Sg*>(st.gp[cur]);
        const A* Ci = static_cast<const A*>(st.c[cur]);
#pragma unroll
        for (int q = 1; q < Q; ++q) {
            if (e_ax(q) != inward) continue;
            const int od = opposite<DIM>(q);
            f[q] = double(cd.load_f(Fi + (long long)od * g.ps + aidx));
            // written by the interior node towards the boundary: shifted by its own c
            gg[q] = cd.template load_g_abs<DIM>(Gi + (long long)od * g.ps + aidx, od, double(Ci[aidx]));
        }
        c = double(Ci[aidx]);
    }
    const A c_store = A(c);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        cd.store_f(Fn + (long long)q * g.ps + self, typename PR::T(f[q]));
        cd.template store_g_abs<DIM>(Gn + (long long)q * g.ps + self, q, gg[q], double(c_store));
    }
    Cn[self] = c_store;
}

// ---------------------------------------------------------------- fields and monitors
// p of an interior node after `last` (the parity of the last step's input buffer, or -1
// right after init): the sum of the pulled f of that step (the reference's dev_p after
// kernelMacroscopicf), or the stored p (zero) before the first step.
template <int DIM, class PR>
__device__ __forceinline__ double node_p(const DevState& st, int x, int y, int z, long long self, int last) {
    using T = typename PR::T;
    using A = typename PR::A;
    constexpr int Q = Lat<DIM>::Q;
    if (last < 0) return double(static_cast<const A*>(st.p)[self]);
    const Codec<PR> cd(st.pop_scale);
    T v[Q];
    pull_f<DIM, PR, true>(static_cast<const typename PR::Sf*>(st.f[last]), cd, st.g, x, y, z, (unsigned)self,
                    cross_mask<DIM>(st.g, x, y, z), v, last);
    T p = v[0];
#pragma unroll
    for (int q = 1; q < Q; ++q) p = p + v[q];
    return double(p);
}
// rho of a node from its c (kernelMacroscopicg form, NsAllen.cu:538)
template <class PR>
__device__ __forceinline__ double node_rho(const DevState& st, double c) {
    using T = typename PR::T;
    return double(T(st.phys.RhoL) + (T(c) * T(st.phys.drho)));
}

// Reference-layout output ((x * EY + y) * EZ + z) * ncomp + comp over the reference's
// ghosted extent.  p, f_post and g_post come from the pull of the last step's input buffer
// (the reference's dev_p, dev_f_post, dev_g_post after the same number of solve calls).
template <int DIM, class PR>
__global__ void field_kernel(DevState st, int which, int last, double* out) {
    using T = typename PR::T;
    using A = typename PR::A;
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    const Geom& g = st.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = DIM == 3 ? (int)blockIdx.z : 0;
    if (x >= g.e[0] || y >= g.e[1]) return;
    const long long self = nidx(g, x, y, z);
    const bool interior = x >= 1 && x <= g.n[0] && y >= 1 && y <= g.n[1] && (DIM == 2 || (z >= 1 && z <= g.n[2]));
    const long long ro = ((long long)x * g.e[1] + y) * (DIM == 3 ? g.e[2] : 1) + (DIM == 3 ? z : 0);
    const int cbuf = last < 0 ? 0 : ((last + 1) & 1);  // c written by the last step
    const A* C = static_cast<const A*>(st.c[cbuf]);
    const A* Cin = static_cast<const A*>(st.c[last < 0 ? 0 : last]);
    const A* U = static_cast<const A*>(st.u);
    const Codec<PR> cd(st.pop_scale);
    switch (which) {
        case 0: {  // c: interior from the last step, ghosts as the reference's ghost layer
            out[ro] = (interior || last < 0) ? double(C[self]) : double(ghost_c<DIM, A>(Cin, g, x, y, z));
            break;
        }
        case 2: {  // rho
            const double c = interior ? double(C[self]) : double(static_cast<const A*>(st.c[0])[self]);
            out[ro] = node_rho<PR>(st, c);
            break;
        }
        case 3: {  // u
            for (int d = 0; d < DIM; ++d) out[ro * DIM + d] = double(U[(long long)d * g.ps + self]);
            break;
        }
        case 1: {  // p
            out[ro] = interior ? node_p<DIM, PR>(st, x, y, z, self, last) : double(static_cast<const A*>(st.p)[self]);
            break;
        }
        default: {  // 4 f, 5 g (post-collision input of the last step), 6 f_post, 7 g_post
            const bool isg = which == 5 || which == 7;
            if (last < 0) {  // right after init the reference holds the initial populations
                const Phys<double> PD = phys_cast<double>(st.phys);
                auto Cf = [&](int dx, int dy, int dz) { return st.c0[nidx(g, x + dx, y + dy, z + dz)]; };
                double c, mu, dc[3], rho, p, f0[Q], g0[Q];
                initial_state<DIM, double>(st.phys, st.phys.sigma, PD, Cf, interior, c, mu, dc, rho, p, f0, g0);
                for (int q = 0; q < Q; ++q) out[ro * Q + q] = isg ? g0[q] : f0[q];
                break;
            }
            const auto* F = static_cast<const typename PR::Sf*>(st.f[last]);
            const auto* G = static_cast<const typename PR::Sg*>(st.gp[last]);
            const A* Cs = static_cast<const A*>(st.c[last]);
            if (which >= 6 && interior) {
                if (isg) {
                    typename PR::TP v[Q], cs;
                    pull_g<DIM, PR, true>(G, Cs, cd, g, x, y, z, self, cross_mask<DIM>(g, x, y, z), v, cs, last);
                    for (int q = 0; q < Q; ++q) out[ro * Q + q] = PR::kShift ? double(v[q]) + double(L::ws(q)) * double(cs) : double(v[q]);
                } else {
                    T v[Q];
                    pull_f<DIM, PR, true>(F, cd, g, x, y, z, self, cross_mask<DIM>(g, x, y, z), v, last);
                    for (int q = 0; q < Q; ++q) out[ro * Q + q] = double(v[q]);
                }
                break;
            }
            // stored populations; ghost cells of periodic axes hold the periodic image
            // (Solver.cu:75-141); the reference never rewrites ghost f_post/g_post.
            long long src = self;
            int s3[3] = {x, y, z};
            bool src_interior = interior;
            if (which < 6 && !interior) {
                bool periodic_only = true;
                for (int a2 = 0; a2 < DIM; ++a2)
                    if ((s3[a2] < 1 || s3[a2] > g.n[a2]) && !g.per[a2]) periodic_only = false;
                if (periodic_only) {
                    for (int a2 = 0; a2 < DIM; ++a2) {
                        if (s3[a2] < 1) s3[a2] += g.n[a2];
                        else if (s3[a2] > g.n[a2]) s3[a2] -= g.n[a2];
                    }
                    src = nidx(g, s3[0], s3[1], s3[2]);
                    src_interior = true;
                }
            }
            for (int q = 0; q < Q; ++q) {
                if (!isg) {
                    out[ro * Q + q] = double(cd.load_f(F + (long long)q * g.ps + src));
                    continue;
                }
                // shift used by the writer: c of the destination if interior, else its own
                long long sh = src;
                if (src_interior) {
                    const int d0 = s3[0] + L::ex(q), d1 = s3[1] + L::ey(q), d2 = DIM == 3 ? s3[2] + L::ez(q) : 0;
                    if (d0 >= 1 && d0 <= g.n[0] && d1 >= 1 && d1 <= g.n[1] && (DIM == 2 || (d2 >= 1 && d2 <= g.n[2])))
                        sh = nidx(g, d0, d1, d2);
                }
                out[ro * Q + q] = cd.template load_g_abs<DIM>(G + (long long)q * g.ps + src, q, double(Cs[sh]));
            }
            break;
        }
    }
}

// Set the state that step k (input parity b) reads from fields in the reference layout
// (FP64, ghosted extent): post-collision f and g (F, G: Q components), c (C) and u (U:
// DIM components).  g is stored as the writer of the previous step would have stored it
// (shifted by the destination's stored c, see Prec).  Used to resume from a checkpoint.
template <int DIM, class PR>
__global__ void state_kernel(DevState st, int b, const double* F, const double* G, const double* C, const double* U) {
    using A = typename PR::A;
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    const Geom& g = st.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = DIM == 3 ? (int)blockIdx.z : 0;
    if (x >= g.e[0] || y >= g.e[1]) return;
    const long long self = nidx(g, x, y, z);
    auto ro = [&](int i, int j, int k) { return ((long long)i * g.e[1] + j) * (DIM == 3 ? g.e[2] : 1) + (DIM == 3 ? k : 0); };
    const long long r = ro(x, y, z);
    const bool interior = x >= 1 && x <= g.n[0] && y >= 1 && y <= g.n[1] && (DIM == 2 || (z >= 1 && z <= g.n[2]));
    const Codec<PR> cd(st.pop_scale);
    auto* Fb = static_cast<typename PR::Sf*>(st.f[b]);
    auto* Gb = static_cast<typename PR::Sg*>(st.gp[b]);
    const double cown = double(A(C[r]));
    static_cast<A*>(st.c[b])[self] = A(C[r]);
    for (int q = 0; q < Q; ++q) {
        cd.store_f(Fb + (long long)q * g.ps + self, typename PR::T(F[r * Q + q]));
        double cs = cown;
        if (interior) {
            const int d0 = x + L::ex(q), d1 = y + L::ey(q), d2 = DIM == 3 ? z + L::ez(q) : 0;
            if (d0 >= 1 && d0 <= g.n[0] && d1 >= 1 && d1 <= g.n[1] && (DIM == 2 || (d2 >= 1 && d2 <= g.n[2])))
                cs = double(A(C[ro(d0, d1, d2)]));
        }
        cd.template store_g_abs<DIM>(Gb + (long long)q * g.ps + self, q, G[r * Q + q], cs);
    }
    if (interior)
        for (int d = 0; d < DIM; ++d) static_cast<A*>(st.u)[(long long)d * g.ps + self] = A(U[r * DIM + d]);
}

// Interior field into a dense device array (x fastest, components as planes).
template <int DIM, typename A>
__global__ void interior_kernel(DevState st, int which, int last, double* out) {
    const Geom& g = st.g;
    const int x = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int y = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int z = DIM == 3 ? 1 + (int)blockIdx.z : 0;
    if (x > g.n[0] || y > g.n[1]) return;
    const long long self = nidx(g, x, y, z);
    const long long nn = (long long)g.n[0] * g.n[1] * (DIM == 3 ? g.n[2] : 1);
    const long long o = (x - 1) + (long long)(y - 1) * g.n[0] + (DIM == 3 ? (long long)(z - 1) * g.n[0] * g.n[1] : 0);
    const int cbuf = last < 0 ? 0 : ((last + 1) & 1);
    const A* C = static_cast<const A*>(st.c[cbuf]);
    if (which == 0) out[o] = double(C[self]);
    else if (which == 2) out[o] = st.phys.RhoL + double(C[self]) * st.phys.drho;
    else if (which == 3)
        for (int d = 0; d < DIM; ++d) out[d * nn + o] = double(static_cast<const A*>(st.u)[(long long)d * g.ps + self]);
}

// The interior fields in VTK point order (x fastest, then y, then z) as the consecutive
// arrays of a .vts file: Velocity (DIM components per point), C, P, Rho
// (VTSwriter.cu:124-135).  Each value equals field_kernel's output at the same node; O is
// double, or float for the single-precision files.
template <int DIM, class PR, typename O>
__global__ void vts_pack_kernel(DevState st, int last, O* __restrict__ out) {
    using A = typename PR::A;
    const Geom& g = st.g;
    const int x = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int y = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    // 3D: the updated planes zlo .. zhi (all interior planes of a whole case, a slab's own)
    const int z = DIM == 3 ? g.zlo + (int)blockIdx.z : 0;
    if (x > g.n[0] || y > g.n[1]) return;
    const long long self = nidx(g, x, y, z);
    const long long nn = (long long)g.n[0] * g.n[1] * (DIM == 3 ? g.zhi - g.zlo + 1 : 1);
    const long long o = (x - 1) + (long long)(y - 1) * g.n[0] + (DIM == 3 ? (long long)(z - g.zlo) * g.n[0] * g.n[1] : 0);
    const int cbuf = last < 0 ? 0 : ((last + 1) & 1);
    const double c = double(static_cast<const A*>(st.c[cbuf])[self]);
    const A* U = static_cast<const A*>(st.u);
#pragma unroll
    for (int d = 0; d < DIM; ++d) out[o * DIM + d] = O(double(U[(long long)d * g.ps + self]));
    O* scal = out + nn * DIM;
    scal[o] = O(c);
    scal[nn + o] = O(node_p<DIM, PR>(st, x, y, z, self, last));
    scal[2 * nn + o] = O(node_rho<PR>(st, c));
}

// Mass sum(c) and kinetic energy sum(rho |u|^2 / 2) over the interior: per-thread FP64
// accumulation over a grid-stride range, warp shuffles, one partial per block; a second
// single-warp pass adds the partials in a fixed order (deterministic result).
template <int DIM, typename A>
__global__ void monitor_partials(DevState st, int cbuf) {
    const Geom& g = st.g;
    // 3D: the updated planes zlo .. zhi (all interior planes of a whole case).  Blocks take
    // rows (y, z) in turn, threads the x of a row: coalesced loads, one division per row,
    // and a fixed summation order for a fixed grid.
    const int ny = g.n[1], nrows = ny * (DIM == 3 ? g.zhi - g.zlo + 1 : 1);
    const A* C = static_cast<const A*>(st.c[cbuf]);
    const A* U = static_cast<const A*>(st.u);
    double m = 0.0, ke = 0.0;
#pragma unroll 4
    for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
        const int y = 1 + r % ny, z = DIM == 3 ? g.zlo + r / ny : 0;
        const long long row = nidx(g, 0, y, z);
        for (int x = 1 + (int)threadIdx.x; x <= g.n[0]; x += blockDim.x) {
            const long long s = row + x;
            const double c = double(C[s]);
            double u2 = 0.0;
            for (int d = 0; d < DIM; ++d) {
                const double v = double(U[(long long)d * g.ps + s]);
                u2 += v * v;
            }
            m += c;
            ke += 0.5 * (st.phys.RhoL + c * st.phys.drho) * u2;
        }
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
            st.red[2 * blockIdx.x] = m;
            st.red[2 * blockIdx.x + 1] = ke;
        }
    }
}

// First pass over the row-segment partials of a monitored step: a grid-stride range per
// thread in a fixed order, warp shuffles, one partial per block (monitor_final adds them).
// A: the instantiating precision's aux type (one instance per unit, like monitor_final).
template <typename A>
__global__ void monitor_rows_partials(const double* __restrict__ rows, long long n, double* red) {
    double m = 0.0, ke = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        m += rows[2 * i];
        ke += rows[2 * i + 1];
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
            red[2 * blockIdx.x] = m;
            red[2 * blockIdx.x + 1] = ke;
        }
    }
}

// out2[2] reports the staged step's wait flag (nonzero: a bounded wait gave up).
template <typename A>
__global__ void monitor_final(const double* red, int nblocks, const int* err, double* out2) {
    double m = 0.0, ke = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += 32) {
        m += red[2 * i];
        ke += red[2 * i + 1];
    }
    for (int off = 16; off > 0; off >>= 1) {
        m += __shfl_down_sync(0xffffffffu, m, off);
        ke += __shfl_down_sync(0xffffffffu, ke, off);
    }
    if (threadIdx.x == 0) {
        out2[0] = m;
        out2[1] = ke;
        out2[2] = *err ? 1.0 : 0.0;
    }
}

}  // namespace clipb
