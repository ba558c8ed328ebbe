// Hand-written adjoint of the FP64 2D step (clipb_adjoint, C ABI in include/clipb.h).
//
// Objective and parameters as in adjoint.cu.  Per reverse step k:
//   (1) adj_node_kernel takes the adjoint of each of the node's stored outputs from the
//       value it became when pulled at step k+1 (the transposed pull streaming, bounce-back
//       and periodic wrap included), recomputes the node's update from the stored state of
//       step k in the moment form of the collision (lean_update: the same
//       operator as the reference's WMRT sequence) and applies its transposed Jacobian;
//   (2) adj_c_kernel applies the transposed mu / grad c stencils, giving the full adjoint
//       of the node's c (which every pulled g of the node receives, c = sum g_post);
//       ghost-layer reads scatter into the adjoint of the lagged c of step k.
// Forward states are kept on the device in segments of K steps (a checkpoint every K
// steps).  The forward run stores the last segment's states directly; while one segment
// is reversed, a second stream recomputes the one before it from its checkpoint into a
// second tape.  (On small grids the two seldom share SMs: each kernel's threads, one per
// node, hold most of the register file.)  Each node kernel brings the next reverse step's
// tape entry into L2.  The workspace stays allocated with the solver and is reused by
// later calls.
//
// Compiled with FMA contraction: the reverse recomputes forward quantities only as
// coefficients of the Jacobian, so it need not round like the forward step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "adjoint.cuh"
#include "clipb.h"
#include "dual.cuh"
#include "kernels.cuh"
#include "solver.hpp"

using namespace clipb;
using namespace clipb::adj;

namespace {


// Block sum of three doubles into partials[3 * blockIdx.x + i] (fixed order).
__device__ __forceinline__ void block_sum3(double v0, double v1, double v2, double* partials) {
    __shared__ double sh[3][32];
    double v[3] = {v0, v1, v2};
    const int lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31, warp = (threadIdx.x + threadIdx.y * blockDim.x) >> 5;
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
    for (int i = 0; i < 3; ++i) {
        for (int off = 16; off > 0; off >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], off);
        if (lane == 0) sh[i][warp] = v[i];
    }
    __syncthreads();
    if (warp == 0) {
        for (int i = 0; i < 3; ++i) {
            double t = lane < nw ? sh[i][lane] : 0.0;
            for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
            if (lane == 0) partials[3 * (blockIdx.x + blockIdx.y * gridDim.x) + i] = t;
        }
    }
}

// acc[i] += sum of partials[3 b + i] over b < n, in a fixed order (one warp per component).
__global__ void accumulate3(const double* partials, int n, double* acc) {
    const int i = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (i >= 3) return;
    double s = 0.0;
    for (int b = lane; b < n; b += 32) s += partials[3 * b + i];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (lane == 0) acc[i] += s;
}

struct Tape {  // one stored forward state (the input of a step), device layout
    double* f;
    double* g;
    double* c;
    double* u;
};

struct AdjBufs {
    double* lf;      // adjoint of the stored f of step 0's input (Q planes), for the initial state
    double* lg;
    double* lu;      // adjoint of U (2 planes), updated in place
    double* lclag;   // adjoint of the stored c of step k+1 (read and cleared by the node kernel),
                     // then of step k's input c (the ghost-layer scatter of adj_c_kernel)
    double* lcf;     // full adjoint of step k's c
    double* lfp[2];  // adjoint of the pulled f (Q planes), by the parity of the step
    double* lgp[2];  // adjoint of the pulled g through the node's g outputs (Q planes), by parity
    double* lcl;     // adjoint of c from the node's own update
    double* llap;    // adjoint of the Laplacian of c at the node
    double* ldc;     // adjoint of grad c (2 planes)
    double* partials;
};

// Where the value stored for node (x, y) in direction q is pulled at the next step: node
// (x, y) + e_q in direction q (wrapped on periodic axes), or (x, y) itself in the opposite
// direction when e_q leads behind a wall (bounce-back).
__device__ __forceinline__ long long stream_dest(const Geom& g, int x, int y, int q, int& qd) {
    int d[2] = {x + L2::ex(q), y + L2::ey(q)};
    bool bb = false;
    for (int a = 0; a < 2; ++a) {
        if (d[a] < 1) {
            if (g.per[a]) d[a] += g.n[a];
            else bb = true;
        } else if (d[a] > g.n[a]) {
            if (g.per[a]) d[a] -= g.n[a];
            else bb = true;
        }
    }
    if (bb) {
        qd = opposite<2>(q);
        return nidx(g, x, y, 0);
    }
    qd = q;
    return nidx(g, d[0], d[1], 0);
}

// Moment-form forward of one node, kept for its reverse (2D).
// Moment-form forward of one node, kept for its reverse (2D).
struct Force {
    double S[2][2], dev[2][2], R[2][2], F[2];
};

__device__ __forceinline__ void force_fwd(const double* uu, const double (*Pi)[2], double p3, double s9, double kvis,
                                          double fcap, const double* dc, const double* grav, Force& o) {
    for (int a = 0; a < 2; ++a)
        for (int bb = 0; bb < 2; ++bb) o.S[a][bb] = Pi[a][bb] - (a == bb ? p3 : 0.0) - uu[a] * uu[bb];
    const double trd = (o.S[0][0] + o.S[1][1]) * 0.5;
    for (int a = 0; a < 2; ++a)
        for (int bb = 0; bb < 2; ++bb) {
            o.dev[a][bb] = o.S[a][bb] - (a == bb ? trd : 0.0);
            o.R[a][bb] = (a == bb ? trd : 0.0) + s9 * o.dev[a][bb];
        }
    for (int a = 0; a < 2; ++a) o.F[a] = fcap * dc[a] + kvis * (o.R[a][0] * dc[0] + o.R[a][1] * dc[1]) + grav[a];
}

struct ForceAdj {
    double lPi[2][2], lp3, ls9, lkvis, lfcap, ldc[2], lgrav[2], luu[2];
};

// Reverse of force_fwd: lF (adjoint of F) and ldev_extra (adjoint of dev from elsewhere).
__device__ __forceinline__ void force_rev(const double* uu, const Force& o, double s9, double kvis, double fcap,
                                          const double* dc, const double* lF, const double (*ldev_extra)[2],
                                          ForceAdj& A) {
    double lR[2][2];
    for (int a = 0; a < 2; ++a) {
        A.lfcap += lF[a] * dc[a];
        A.ldc[a] += lF[a] * fcap;
        A.lgrav[a] += lF[a];
        A.lkvis += lF[a] * (o.R[a][0] * dc[0] + o.R[a][1] * dc[1]);
        for (int bb = 0; bb < 2; ++bb) {
            lR[a][bb] = kvis * lF[a] * dc[bb];
            A.ldc[bb] += kvis * lF[a] * o.R[a][bb];
        }
    }
    double ltrd = lR[0][0] + lR[1][1], ldev[2][2], lS[2][2];
    for (int a = 0; a < 2; ++a)
        for (int bb = 0; bb < 2; ++bb) {
            A.ls9 += lR[a][bb] * o.dev[a][bb];
            ldev[a][bb] = s9 * lR[a][bb] + (ldev_extra ? ldev_extra[a][bb] : 0.0);
        }
    for (int a = 0; a < 2; ++a)
        for (int bb = 0; bb < 2; ++bb) lS[a][bb] = ldev[a][bb];
    ltrd -= ldev[0][0] + ldev[1][1];
    lS[0][0] += ltrd * 0.5;
    lS[1][1] += ltrd * 0.5;
    for (int a = 0; a < 2; ++a)
        for (int bb = 0; bb < 2; ++bb) A.lPi[a][bb] += lS[a][bb];
    A.lp3 -= lS[0][0] + lS[1][1];
    for (int cidx = 0; cidx < 2; ++cidx)
        A.luu[cidx] -= (lS[cidx][0] + lS[0][cidx]) * uu[0] + (lS[cidx][1] + lS[1][cidx]) * uu[1];
}

// Block shape of the node kernel, and the operands each thread stages in shared memory
// before it computes: the adjoints of its 9 f and 9 g outputs (taken where the next step
// pulls them), its 9 pulled f and 9 pulled g, and c over its 3 x 3 neighbourhood.  Staging
// issues these 45 scattered loads together; nodes one away from every side (whole warps,
// mostly) find them at fixed offsets.
constexpr int kNodeThreads = 256;
constexpr int kSlf = 0, kSlg = Q, kSgp = 2 * Q, kSfp = 3 * Q, kSc = 4 * Q, kStage = 4 * Q + 9;
constexpr int kNodeSmem = kStage * kNodeThreads * (int)sizeof(double);

// acc += k v for a lattice factor k in {-1, 0, 1}, known once the direction loops are
// unrolled: a zero factor adds nothing (as x * 0 would, infinities aside).
__device__ __forceinline__ void acc_k(double& acc, int k, double v) {
    if (k > 0) acc += v;
    else if (k < 0) acc -= v;
}

// Stage the node's operands into its column st[row * kNodeThreads] of the stage.
__device__ __forceinline__ void stage_node(const Geom& g, int x, int y, const Tape& in, const double* c_out,
                                           const AdjBufs& A, int par, double* st) {
    constexpr int NT = kNodeThreads;
    const double* lfp_in = par ? A.lfp[0] : A.lfp[1];
    const double* lgp_in = par ? A.lgp[0] : A.lgp[1];
    const long long self = nidx(g, x, y, 0), ps = g.ps;
    if (x > 1 && x < g.n[0] && y > 1 && y < g.n[1]) {
        // every neighbour is interior: fixed 32-bit offsets (Q planes hold fewer than 2^32
        // elements, as the step kernels require)
        const unsigned s32 = (unsigned)self, p32 = (unsigned)ps, sy = (unsigned)g.sy;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const unsigned off = unsigned(L2::ex(q)) + unsigned(L2::ey(q)) * sy;
            const unsigned d = s32 + off, s = s32 - off, qo = unsigned(q) * p32;
            st[(kSlf + q) * NT] = lfp_in[qo + d];
            st[(kSlg + q) * NT] = lgp_in[qo + d] + A.lcf[d];
            st[(kSgp + q) * NT] = in.g[qo + s];
            st[(kSfp + q) * NT] = in.f[qo + s];
        }
#pragma unroll
        for (int oy = -1; oy <= 1; ++oy)
#pragma unroll
            for (int ox = -1; ox <= 1; ++ox)
                st[(kSc + 3 * (oy + 1) + ox + 1) * NT] = c_out[s32 + unsigned(ox) + unsigned(oy) * sy];
    } else {
        for (int q = 0; q < Q; ++q) {
            int qd, qs;
            bool crossed;
            const long long d = stream_dest(g, x, y, q, qd);
            const long long s = pull_source<2>(g, q, x, y, 0, self, qs, crossed);
            st[(kSlf + q) * NT] = lfp_in[qd * ps + d];
            st[(kSlg + q) * NT] = lgp_in[qd * ps + d] + A.lcf[d];
            st[(kSgp + q) * NT] = in.g[qs * ps + s];
            st[(kSfp + q) * NT] = in.f[qs * ps + s];
        }
        // interior: this step's c; ghosts: the lagged c of step k
        for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) {
                const int xx = x + ox, yy = y + oy;
                st[(kSc + 3 * (oy + 1) + ox + 1) * NT] =
                    interior2(g, xx, yy) ? c_out[nidx(g, xx, yy, 0)] : in.c[ghost_source(g, xx, yy)];
            }
    }
}

__device__ __forceinline__ void prefetch_l2(const double* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }


// (1) node-local reverse of step k (parity par) at every interior node.  `next`: the tape
// entry the next kernel of the sweep reads (step k - 1), whose populations are brought into
// L2 while this step computes (null when it lies in another tape).
__global__ void __launch_bounds__(kNodeThreads, 2) adj_node_kernel(Geom g, PhysD pd, ParamChain pc, Tape in,
                                                                   const double* c_out, AdjBufs A, int par, Tape next) {
    constexpr int NT = kNodeThreads;
    extern __shared__ double stage[];  // [kStage][kNodeThreads], each thread its own column
    chain_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1, y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    double pg = 0.0, psig = 0.0, pmob = 0.0;
    if (x <= g.n[0] && y <= g.n[1]) {
        const long long self = nidx(g, x, y, 0);
        const long long ps = g.ps;
        const double* st = stage + threadIdx.y * blockDim.x + threadIdx.x;
        stage_node(g, x, y, in, c_out, A, par, stage + threadIdx.y * blockDim.x + threadIdx.x);
        if (next.f) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                prefetch_l2(next.f + q * ps + self);
                prefetch_l2(next.g + q * ps + self);
            }
        }
        double lc = A.lclag[self];
        A.lclag[self] = 0.0;  // receives the ghost-layer scatter of this step (adj_c_kernel)
        // stencils of c
        double lap = 0.0, dc[2] = {0.0, 0.0};
#pragma unroll
        for (int oy = -1; oy <= 1; ++oy)
#pragma unroll
            for (int ox = -1; ox <= 1; ++ox) {
                const double cv = st[(kSc + 3 * (oy + 1) + ox + 1) * NT];
                double a, bx, by;
                coef2(ox, oy, a, bx, by);
                lap += a * cv;
                if (ox) dc[0] += bx * cv;
                if (oy) dc[1] += by * cv;
            }
        const double c = st[(kSc + 4) * NT];
        const double poly = c * (c - 1.0) * (c - 0.5), dpoly = (3.0 * c - 3.0) * c + 0.5;
        const double mu = pd.beta4 * poly - pd.kappa * lap;
        // hydrodynamic moments
        double p = 0.0, j[2] = {0.0, 0.0}, Pi[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int e[2] = {L2::ex(q), L2::ey(q)};
            const double fq = st[(kSfp + q) * NT];
            p += fq;
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                acc_k(j[a], e[a], fq);
#pragma unroll
                for (int bb = 0; bb < 2; ++bb) acc_k(Pi[a][bb], e[a] * e[bb], fq);
            }
        }
        const double rho = pd.RhoL + c * pd.drho, irho = 1.0 / rho;
        double tau, dtdc;
        if (c < 0.0) { tau = pd.tauL; dtdc = 0.0; }
        else if (c > 1.0) { tau = pd.tauH; dtdc = 0.0; }
        else { tau = pd.tauL + c * pd.dtau; dtdc = pd.dtau; }
        const double s9 = 1.0 / (tau + 0.5), kvis = -tau * pd.drho, fcap = mu - p * pd.drho3, p3 = p * (1.0 / 3.0);
        const double gfac = pd.caseType == 2 ? rho : rho - pc.rref;
        const double grav[2] = {gfac * pd.g[0], gfac * pd.g[1]};
        const double uprev[2] = {in.u[self], in.u[ps + self]};
        Force f1, f2;
        force_fwd(uprev, Pi, p3, s9, kvis, fcap, dc, grav, f1);
        const double h = 0.5 * irho;
        const double u[2] = {j[0] + f1.F[0] * h, j[1] + f1.F[1] * h};
        force_fwd(u, Pi, p3, s9, kvis, fcap, dc, grav, f2);
        const double U2 = u[0] * u[0] + u[1] * u[1], sm1 = s9 - 1.0;
        // phase field
        const double mag = sqrt(dc[0] * dc[0] + dc[1] * dc[1]), m = mag + 1e-32, im = 1.0 / m, iW = 1.0 / pd.W;
        const double nrm[2] = {dc[0] * im, dc[1] * im};
        const double cm = c - 0.5, pf = 1.0 - 4.0 * cm * cm, pref = pd.amob3 * pf * iW;
        const double f15 = 1.5 * irho, f15r = f15 * irho;

        // ---- reverse
        double lmu = 0.0, ldcv[2] = {0.0, 0.0}, lu[2] = {A.lu[self], A.lu[ps + self]};
        double lp = 0.0, lrho = 0.0, ls9 = 0.0, lU2 = 0.0, lwc = 0.0, lamob3 = 0.0, lpref = 0.0;
        double lnrm[2] = {0.0, 0.0}, lF2[2] = {0.0, 0.0}, ldev2[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
        double* lgp_out = par ? A.lgp[1] : A.lgp[0];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int e[2] = {L2::ex(q), L2::ey(q)};
            const double w = L2::w(q);
            double eu = 0.0, eF = 0.0, en = 0.0, phi = 0.0;
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                acc_k(eu, e[a], u[a]);
                acc_k(eF, e[a], f2.F[a]);
                acc_k(en, e[a], nrm[a]);
#pragma unroll
                for (int bb = 0; bb < 2; ++bb) acc_k(phi, e[a] * e[bb], f2.dev[a][bb]);
            }
            phi *= 4.5;
            // g output
            const double lg_q = st[(kSlg + q) * NT];
            const double ga = w * (3.0 * eu + 4.5 * eu * eu - 1.5 * U2);
            const double H = c * (ga + w) + w * pref * en;
            lgp_out[q * ps + self] = lg_q * pd.one_minus_wc;
            lwc += lg_q * (H - st[(kSgp + q) * NT]);  // pulled g
            const double lH = lg_q * pd.wc;
            lc += lH * (ga + w);
            const double lga = lH * c;
            double leu = lga * w * (3.0 + 9.0 * eu);
            lU2 += lga * w * -1.5;
            lpref += lH * w * en;
            const double len = lH * w * pref;
            // f output
            const double lf_q = st[(kSlf + q) * NT];
            lp += w * lf_q;
            leu += w * lf_q * (3.0 + 9.0 * eu);
            lU2 += w * lf_q * -1.5;
            const double leF = w * lf_q * f15;
            lrho -= w * lf_q * eF * f15r;
            ls9 += -w * lf_q * phi;  // d/d(s9) of -(s9 - 1) phi
            const double lphi = -w * lf_q * sm1 * 4.5;
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                acc_k(lnrm[a], e[a], len);
                acc_k(lF2[a], e[a], leF);
                acc_k(lu[a], e[a], leu);
#pragma unroll
                for (int bb = 0; bb < 2; ++bb) acc_k(ldev2[a][bb], e[a] * e[bb], lphi);
            }
        }
        lu[0] += 2.0 * u[0] * lU2;
        lu[1] += 2.0 * u[1] * lU2;
        lc += lpref * pd.amob3 * (-8.0 * cm) * iW;
        lamob3 += lpref * pf * iW;
        {  // interface normal, derivative damped as in the tangent-linear model (dual.cuh)
            const double sc = normal_damping(mag, c, pd.W);
            const double t = mag > 0.0 ? (lnrm[0] * dc[0] + lnrm[1] * dc[1]) * (im * im) / mag : 0.0;
            for (int bb = 0; bb < 2; ++bb) ldcv[bb] += sc * (lnrm[bb] * im - t * dc[bb]);
        }
        // force at this step's velocity
        ForceAdj FA{};
        force_rev(u, f2, s9, kvis, fcap, dc, lF2, ldev2, FA);
        lu[0] += FA.luu[0];
        lu[1] += FA.luu[1];
        // u = j + F(uprev) h
        double lj[2] = {lu[0], lu[1]}, lF1[2] = {lu[0] * h, lu[1] * h};
        lrho += (lu[0] * f1.F[0] + lu[1] * f1.F[1]) * (-0.5 * irho * irho);
        FA.luu[0] = FA.luu[1] = 0.0;
        force_rev(uprev, f1, s9, kvis, fcap, dc, lF1, nullptr, FA);
        A.lu[self] = FA.luu[0];
        A.lu[ps + self] = FA.luu[1];
        // scalars
        lp += FA.lp3 * (1.0 / 3.0) - pd.drho3 * FA.lfcap;
        lmu += FA.lfcap;
        ls9 += FA.ls9;
        double ltau = -pd.drho * FA.lkvis - s9 * s9 * ls9;
        lc += dtdc * ltau;
        for (int a = 0; a < 2; ++a) {
            lrho += FA.lgrav[a] * pd.g[a];
            ldcv[a] += FA.ldc[a];
        }
        pg = FA.lgrav[1] * gfac;
        lc += pd.drho * lrho;
        // mu = beta4 poly(c) - kappa lap
        lc += lmu * pd.beta4 * dpoly;
        psig = (lmu * poly) * pc.dbeta4_dsigma + (-lmu * lap) * pc.dkappa_dsigma;
        pmob = lwc * pc.dwc_dM + lamob3 * 3.0;
        A.llap[self] = -pd.kappa * lmu;
        A.ldc[self] = ldcv[0];
        A.ldc[ps + self] = ldcv[1];
        A.lcl[self] = lc;
        double* lfp_out = par ? A.lfp[1] : A.lfp[0];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int e[2] = {L2::ex(q), L2::ey(q)};
            double v = lp;
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                acc_k(v, e[a], lj[a]);
#pragma unroll
                for (int bb = 0; bb < 2; ++bb) acc_k(v, e[a] * e[bb], FA.lPi[a][bb]);
            }
            lfp_out[q * ps + self] = v;
        }
    }
    block_sum3(pg, psig, pmob, A.partials);
}

// (2) transposed stencils: the full adjoint of c at every interior node (the node's own
// part plus the stencils of its neighbours that read it); the node's own stencil reads of
// ghost positions scatter into the adjoint of the lagged c.
__global__ void adj_c_kernel(Geom g, AdjBufs A) {
    chain_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1, y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (x > g.n[0] || y > g.n[1]) return;
    const long long self = nidx(g, x, y, 0), ps = g.ps;
    double lc = A.lcl[self];
    if (x > 1 && x < g.n[0] && y > 1 && y < g.n[1]) {
        // every neighbour is interior and no stencil of this node reads a ghost position
        const unsigned s32 = (unsigned)self, p32 = (unsigned)ps, sy = (unsigned)g.sy;
#pragma unroll
        for (int oy = -1; oy <= 1; ++oy)
#pragma unroll
            for (int ox = -1; ox <= 1; ++ox) {
                double a, bx, by;
                coef2(ox, oy, a, bx, by);
                const unsigned n = s32 - unsigned(ox) - unsigned(oy) * sy;
                lc += A.llap[n] * a;
                if (ox) lc += A.ldc[n] * bx;
                if (oy) lc += A.ldc[p32 + n] * by;
            }
        A.lcf[self] = lc;
        return;
    }
    for (int oy = -1; oy <= 1; ++oy)
        for (int ox = -1; ox <= 1; ++ox) {
            double a, bx, by;
            coef2(ox, oy, a, bx, by);
            // node n = m - o reads m at offset o
            const int nx = x - ox, ny = y - oy;
            if (interior2(g, nx, ny)) {
                const long long n = nidx(g, nx, ny, 0);
                lc += A.llap[n] * a + A.ldc[n] * bx + A.ldc[ps + n] * by;
            }
            // this node's own stencil reading a ghost position
            const int gx = x + ox, gy = y + oy;
            if (!interior2(g, gx, gy))
                atomicAdd(&A.lclag[ghost_source(g, gx, gy)], A.llap[self] * a + A.ldc[self] * bx + A.ldc[ps + self] * by);
        }
    A.lcf[self] = lc;
}

// Adjoint of the stored populations of step 0's input (the initial state's outputs): those
// of the values they became when pulled at step 0 (adjoints of parity 0).
__global__ void adj_stream_kernel(Geom g, AdjBufs A) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1, y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (x > g.n[0] || y > g.n[1]) return;
    const long long self = nidx(g, x, y, 0), ps = g.ps;
    for (int q = 0; q < Q; ++q) {
        int qd;
        const long long n = stream_dest(g, x, y, q, qd);
        A.lf[q * ps + self] = A.lfp[0][qd * ps + n];
        A.lg[q * ps + self] = A.lgp[0][qd * ps + n] + A.lcf[n];
    }
}

// Reverse of the initial state + first collision: adjoint of the initial c field.
__global__ void adj_init_node_kernel(Geom g, PhysD pd, ParamChain pc, const double* c0, AdjBufs A) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1, y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    double pg = 0.0, psig = 0.0, pmob = 0.0;
    if (x <= g.n[0] && y <= g.n[1]) {
        const long long self = nidx(g, x, y, 0), ps = g.ps;
        double lap = 0.0, dc[2] = {0.0, 0.0};
        for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) {
                double a, bx, by;
                coef2(ox, oy, a, bx, by);
                const double cv = c0[nidx(g, x + ox, y + oy, 0)];
                lap += a * cv;
                dc[0] += bx * cv;
                dc[1] += by * cv;
            }
        const double c = c0[self];
        const double poly = c * (c - 1.0) * (c - 0.5), dpoly = (3.0 * c - 3.0) * c + 0.5;
        const double mu = pd.beta4 * poly - pd.kappa * lap;
        const double mag = sqrt(dc[0] * dc[0] + dc[1] * dc[1]), m = mag + 1e-32;
        const double nrm[2] = {dc[0] / m, dc[1] / m};
        const double rho = pd.RhoL + c * pd.drho;
        const double sgn = pd.caseType == 0 ? -1.0 : (pd.caseType == 1 ? 1.0 : 0.0);
        const double kp = sgn * pd.sigma / (pd.refLen / 2.0) / (rho / 3.0);  // p = c kp
        const double p = c * kp;
        const double cm = c - 0.5, pf = 1.0 - 4.0 * cm * cm, pref = pd.amob3 * pf / pd.W;
        const double gfac = pd.caseType == 2 ? rho : rho - pc.rref;
        const double F[2] = {(mu - p * pd.drho3) * dc[0] + gfac * pd.g[0], (mu - p * pd.drho3) * dc[1] + gfac * pd.g[1]};
        double lc = 0.0, lrho = 0.0, lp = 0.0, lmu = 0.0, ldcv[2] = {0.0, 0.0}, lnrm[2] = {0.0, 0.0};
        double lF[2] = {0.0, 0.0}, lwc = 0.0, lamob3 = 0.0, lpref = 0.0;
        for (int q = 0; q < Q; ++q) {
            const int e[2] = {L2::ex(q), L2::ey(q)};
            const double w = L2::w(q);
            const double en = e[0] * nrm[0] + e[1] * nrm[1];
            // fo = w (p + 1.5 e.F / rho)
            const double lfo = A.lf[q * ps + self];
            const double eF = e[0] * F[0] + e[1] * F[1];
            lp += w * lfo;
            lF[0] += w * lfo * 1.5 * e[0] / rho;
            lF[1] += w * lfo * 1.5 * e[1] / rho;
            lrho += -w * lfo * 1.5 * eF / (rho * rho);
            // g0 = c w - w pf en / (2 W);  go = g0 (1 - wc) + wc (c w + w pref en)
            const double lgo = A.lg[q * ps + self];
            const double g0 = c * w - 0.5 * w * pf / pd.W * en;
            const double lg0 = lgo * pd.one_minus_wc;
            lwc += lgo * (-g0 + c * w + w * pref * en);
            lc += lgo * pd.wc * w + lg0 * w;
            lpref += lgo * pd.wc * w * en;
            const double len = lgo * pd.wc * w * pref - lg0 * 0.5 * w * pf / pd.W;
            lc += -lg0 * 0.5 * w / pd.W * en * (-8.0 * cm);
            lnrm[0] += len * e[0];
            lnrm[1] += len * e[1];
        }
        lc += lpref * pd.amob3 * (-8.0 * cm) / pd.W;
        lamob3 += lpref * pf / pd.W;
        // F = (mu - p drho3) dc + gfac g
        for (int a = 0; a < 2; ++a) {
            lmu += lF[a] * dc[a];
            lp += -pd.drho3 * lF[a] * dc[a];
            ldcv[a] += lF[a] * (mu - p * pd.drho3);
            lrho += lF[a] * pd.g[a];
        }
        pg = lF[1] * gfac;
        // p = c kp(rho), kp = sgn sigma / (L/2) / (rho/3)
        lc += lp * kp;
        lrho += lp * (-p / rho);
        psig = lp * (sgn * c / (pd.refLen / 2.0) / (rho / 3.0));
        lc += lrho * pd.drho;
        {  // interface normal, derivative damped as in the tangent-linear model (dual.cuh)
            const double sc = normal_damping(mag, c, pd.W);
            const double t = mag > 0.0 ? (lnrm[0] * dc[0] + lnrm[1] * dc[1]) / (mag * m * m) : 0.0;
            for (int bb = 0; bb < 2; ++bb) ldcv[bb] += sc * (lnrm[bb] / m - t * dc[bb]);
        }
        lc += lmu * pd.beta4 * dpoly;
        psig += (lmu * poly) * pc.dbeta4_dsigma + (-lmu * lap) * pc.dkappa_dsigma;
        pmob = lwc * pc.dwc_dM + lamob3 * 3.0;
        A.llap[self] = -pd.kappa * lmu;
        A.ldc[self] = ldcv[0];
        A.ldc[ps + self] = ldcv[1];
        A.lcl[self] = lc;
    }
    block_sum3(pg, psig, pmob, A.partials);
}

// Adjoint of the initial c over the ghosted extent (into out, device layout).
__global__ void adj_init_c_kernel(Geom g, AdjBufs A, const double* lc0_lag, double* out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= g.e[0] || y >= g.e[1]) return;
    const long long self = nidx(g, x, y, 0), ps = g.ps;
    double lc = interior2(g, x, y) ? A.lcl[self] + lc0_lag[self] : 0.0;
    for (int oy = -1; oy <= 1; ++oy)
        for (int ox = -1; ox <= 1; ++ox) {
            const int nx = x - ox, ny = y - oy;
            if (!interior2(g, nx, ny)) continue;
            double a, bx, by;
            coef2(ox, oy, a, bx, by);
            const long long n = nidx(g, nx, ny, 0);
            lc += A.llap[n] * a + A.ldc[n] * bx + A.ldc[ps + n] * by;
        }
    out[self] = lc;
}

}  // namespace

namespace clipb {

// Device workspace of clipb_adjoint, kept with its solver and grown when a call needs more
// (tapes, checkpoints, adjoint planes, partial sums), plus the stream that recomputes
// segments beside the reverse sweep.
struct AdjWork {
    void* mem = nullptr;
    size_t bytes = 0;
    cudaStream_t s2 = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    ~AdjWork() {
        if (s2) cudaStreamSynchronize(s2);
        if (mem) cudaFree(mem);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (s2) cudaStreamDestroy(s2);
    }
};

void adj_release(AdjWork* w) { delete w; }

}  // namespace clipb

namespace {

int ensure_work(clipb_solver* s, size_t bytes) {
    if (!s->adjw) {
        s->adjw = new AdjWork();
        AdjWork* w = s->adjw;
        CLIPB_CUDA(cudaStreamCreateWithFlags(&w->s2, cudaStreamNonBlocking));
        CLIPB_CUDA(cudaEventCreateWithFlags(&w->fork, cudaEventDisableTiming));
        CLIPB_CUDA(cudaEventCreateWithFlags(&w->join, cudaEventDisableTiming));
    }
    AdjWork* w = s->adjw;
    if (w->bytes >= bytes) return CLIPB_OK;
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    if (w->mem) cudaFree(w->mem);
    w->mem = nullptr;
    w->bytes = 0;
    const cudaError_t e = cudaMalloc(&w->mem, bytes);
    if (e != cudaSuccess)
        return fail(CLIPB_E_NOMEM, "adjoint workspace of " + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e) +
                                       " (a smaller checkpoint interval needs less)");
    w->bytes = bytes;
    // tape entries are written at interior nodes only: keep the rest defined
    CLIPB_CUDA(cudaMemsetAsync(w->mem, 0, bytes, s->stream));
    return CLIPB_OK;
}

}  // namespace

extern "C" {

int clipb_adjoint(clipb_solver* s, const double* c0_host, int nsteps, const double* target, int checkpoint_every,
                  double* J, double* grad_c0, double* grad_params3) {
    if (!s || !target || !J) return fail(CLIPB_E_ARG, "null argument");
    if (nsteps < 1) return fail(CLIPB_E_ARG, "need at least one step");
    int rc = check_case(s);
    if (rc) return rc;
    const Geom& g = s->st.g;
    const size_t ps = (size_t)g.ps;
    const size_t state = (2 * Q + 1 + 2) * ps;  // f, g, c, u
    int K = checkpoint_every;
    if (K <= 0) {
        // every state of the run in one tape (no recomputation) when the tape takes at most
        // half of the device memory that is free, counting the workspace this solver holds
        size_t free_b = 0, total_b = 0;
        CLIPB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const size_t held = s->adjw ? s->adjw->bytes : 0;
        K = ((size_t)nsteps + 1) * state * sizeof(double) <= (free_b + held) / 2 ? nsteps : 100;
    }
    const int nck = (nsteps + K - 1) / K, last = nck - 1, len_last = nsteps - last * K;
    static_assert(kNodeThreads == 32 * 8, "node kernel blocks are 32 x 8");
    const dim3 blk(32, 8), gi((g.n[0] + 31) / 32, (g.n[1] + 7) / 8), ge((g.e[0] + 31) / 32, (g.e[1] + 7) / 8);
    const int nblocks = (int)(gi.x * gi.y);
    // workspace: a tape of K + 1 states (two when there are several segments), a checkpoint
    // per segment but the last, the adjoint planes, the parameter partial sums of a
    // segment, the initial c and its adjoint
    const int ntapes = last > 0 ? 2 : 1;
    const size_t n_tape = (size_t)(std::min(K, nsteps) + 1) * state, n_ck = (size_t)last * state;
    const size_t n_adj = (6 * Q + 8) * ps;
    const size_t n_part = 3 * (size_t)nblocks * K;
    if ((rc = upload_c0(s, c0_host))) return rc;
    if ((rc = ensure_work(s, (ntapes * n_tape + n_ck + n_adj + n_part + 3 + 2 * ps) * sizeof(double)))) return rc;
    AdjWork* W = s->adjw;
    static const cudaError_t smem_ok =
        cudaFuncSetAttribute(adj_node_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kNodeSmem);
    if (smem_ok != cudaSuccess) return fail(CLIPB_E_CUDA, std::string("adjoint node kernel: ") + cudaGetErrorString(smem_ok));
    double* tape[2] = {static_cast<double*>(W->mem), static_cast<double*>(W->mem) + (ntapes - 1) * n_tape};
    double* ck = static_cast<double*>(W->mem) + ntapes * n_tape;
    double* a0 = ck + n_ck;
    double* partials = a0 + n_adj;
    double* acc = partials + n_part;
    double* c0dev = acc + 3;
    double* gc0 = c0dev + ps;
    CLIPB_CUDA(cudaMemcpyAsync(c0dev, s->st.c0, ps * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
    auto view = [&](double* p) {
        Tape t;
        t.f = p;
        t.g = p + Q * ps;
        t.c = p + 2 * Q * ps;
        t.u = p + (2 * Q + 1) * ps;
        return t;
    };
    auto save = [&](const Tape& t) -> int {  // solver state (input of step s->steps) -> t
        const int b = (int)(s->steps & 1);
        CLIPB_CUDA(cudaMemcpyAsync(t.f, s->st.f[b], Q * ps * 8, cudaMemcpyDeviceToDevice, s->stream));
        CLIPB_CUDA(cudaMemcpyAsync(t.g, s->st.gp[b], Q * ps * 8, cudaMemcpyDeviceToDevice, s->stream));
        CLIPB_CUDA(cudaMemcpyAsync(t.c, s->st.c[b], ps * 8, cudaMemcpyDeviceToDevice, s->stream));
        CLIPB_CUDA(cudaMemcpyAsync(t.u, s->st.u, 2 * ps * 8, cudaMemcpyDeviceToDevice, s->stream));
        return CLIPB_OK;
    };
    // interior rows of `planes` planes (tape entries hold defined values there only; the
    // solver's ghost nodes keep theirs)
    auto copy_interior = [&](void* dst, const double* src, int planes) -> int {
        const size_t first = (size_t)(g.base + 1 + g.sy), pitch = (size_t)g.sy * 8;  // node (1, 1)
        for (int q = 0; q < planes; ++q)
            CLIPB_CUDA(cudaMemcpy2DAsync(static_cast<double*>(dst) + q * ps + first, pitch, src + q * ps + first, pitch,
                                         (size_t)g.n[0] * 8, (size_t)g.n[1], cudaMemcpyDeviceToDevice, s->stream));
        return CLIPB_OK;
    };
    // tape entry t (the state after `step` steps) into the solver's buffers of that parity
    auto restore = [&](const Tape& t, long long step, bool with_u) -> int {
        const int b = (int)(step & 1);
        int r = copy_interior(s->st.f[b], t.f, Q);
        if (!r) r = copy_interior(s->st.gp[b], t.g, Q);
        if (!r) r = copy_interior(s->st.c[b], t.c, 1);
        if (!r && with_u) r = copy_interior(s->st.u, t.u, 2);
        return r;
    };
    // steps k0 .. k0 + len - 1 from tape entry 0 (their input states and the state after
    // them) into tape tp, by pointing the solver's buffers at tape entries (each step reads
    // u from its entry and writes it into the next)
    const DevState saved = s->st;
    auto recompute = [&](double* tp, int k0, int len, cudaStream_t strm) -> int {
        for (int i = 0; i < len; ++i) {
            const int k = k0 + i, b = k & 1;
            const Tape ti = view(tp + (size_t)i * state), tn = view(tp + (size_t)(i + 1) * state);
            s->st.f[b] = ti.f;
            s->st.gp[b] = ti.g;
            s->st.c[b] = ti.c;
            s->st.f[b ^ 1] = tn.f;
            s->st.gp[b ^ 1] = tn.g;
            s->st.c[b ^ 1] = tn.c;
            s->st.uin = ti.u;
            s->st.u = tn.u;
            const cudaError_t e = s->kt.step(s->st, k, strm);
            if (e != cudaSuccess) {
                s->st = saved;
                return fail(CLIPB_E_CUDA, std::string("adjoint recomputation: ") + cudaGetErrorString(e));
            }
        }
        s->st = saved;
        return CLIPB_OK;
    };
    // ---- forward: segments 0 .. last-1 in the solver's buffers with a checkpoint each (graph
    // replays), the last segment straight into its tape
    for (int seg = 0; seg < last; ++seg) {
        if ((rc = save(view(ck + (size_t)seg * state)))) return rc;
        if ((rc = clipb_solve(s, K))) return rc;
    }
    double* tl = tape[last & 1];
    if ((rc = save(view(tl)))) return rc;
    if ((rc = recompute(tl, last * K, len_last, s->stream))) return rc;
    // the solver is left at the end of the forward run: its last state and, in the other
    // parity, the input of its last step (which the p and rho outputs pull)
    if ((rc = restore(view(tl + (size_t)(len_last - 1) * state), nsteps - 1, false))) return rc;
    if ((rc = restore(view(tl + (size_t)len_last * state), nsteps, true))) return rc;
    s->steps = nsteps;
    std::vector<double> c((size_t)ps), dJ;
    CLIPB_CUDA(cudaMemcpyAsync(c.data(), tl + (size_t)len_last * state + 2 * Q * ps, ps * 8, cudaMemcpyDeviceToHost,
                               s->stream));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    *J = objective(s, c, target, &dJ);
    // ---- adjoint buffers (the adjoints of the final populations and velocity are zero)
    AdjBufs A;
    A.lf = a0;
    A.lg = a0 + Q * ps;
    A.lfp[0] = a0 + 2 * Q * ps;
    A.lfp[1] = a0 + 3 * Q * ps;
    A.lgp[0] = a0 + 4 * Q * ps;
    A.lgp[1] = a0 + 5 * Q * ps;
    A.lu = a0 + 6 * Q * ps;
    A.ldc = a0 + 6 * Q * ps + 2 * ps;
    A.lclag = a0 + 6 * Q * ps + 4 * ps;
    A.lcf = a0 + 6 * Q * ps + 5 * ps;
    A.lcl = a0 + 6 * Q * ps + 6 * ps;
    A.llap = a0 + 6 * Q * ps + 7 * ps;
    A.partials = partials;
    CLIPB_CUDA(cudaMemsetAsync(a0, 0, n_adj * sizeof(double), s->stream));
    CLIPB_CUDA(cudaMemsetAsync(acc, 0, 3 * sizeof(double), s->stream));
    CLIPB_CUDA(cudaMemcpyAsync(A.lclag, dJ.data(), ps * 8, cudaMemcpyHostToDevice, s->stream));
    const PhysD pd = s->st.phys;
    const ParamChain pc = chain(pd);
    // reverse sweep of segment seg (tape tp) on the solver's stream, then its partial sums
    auto reverse = [&](double* tp, int k0, int len) -> int {
        for (int i = len - 1; i >= 0; --i) {
            const Tape in = view(tp + (size_t)i * state);
            const double* c_out = tp + (size_t)(i + 1) * state + 2 * Q * ps;
            A.partials = partials + 3 * (size_t)nblocks * i;
            const Tape next = i > 0 ? view(tp + (size_t)(i - 1) * state) : Tape{nullptr, nullptr, nullptr, nullptr};
            CLIPB_CUDA(launch_chained(adj_node_kernel, gi, blk, kNodeSmem, s->stream, g, pd, pc, in, c_out, A,
                                      (k0 + i) & 1, next));
            CLIPB_CUDA(launch_chained(adj_c_kernel, gi, blk, 0, s->stream, g, A));
        }
        accumulate3<<<1, 96, 0, s->stream>>>(partials, len * nblocks, acc);
        CLIPB_CUDA(cudaGetLastError());
        return CLIPB_OK;
    };
    // one iteration: segment seg reversed on the solver's stream while the second stream
    // recomputes segment seg - 1 into the other tape (its entry 0 already holds the checkpoint)
    auto iteration = [&](int seg) -> int {
        const int len = seg == last ? len_last : K;
        if (seg > 0) {
            CLIPB_CUDA(cudaEventRecord(W->fork, s->stream));
            CLIPB_CUDA(cudaStreamWaitEvent(W->s2, W->fork, 0));
            int r = recompute(tape[(seg - 1) & 1], (seg - 1) * K, K, W->s2);
            // the join is recorded even after a failed launch, so that a capture can end
            const cudaError_t e = cudaEventRecord(W->join, W->s2);
            if (e == cudaSuccess) CLIPB_CUDA(cudaStreamWaitEvent(s->stream, W->join, 0));
            if (r) return r;
            if (e != cudaSuccess) return fail(CLIPB_E_CUDA, std::string("adjoint join: ") + cudaGetErrorString(e));
        }
        return reverse(tape[seg & 1], seg * K, len);
    };
    // the middle segments (full length, both parts) replay one captured graph per tape
    // parity when K is even: same tape entries, same step parities, same partial sums
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};
    auto drop_graphs = [&]() {
        for (auto& x : graphs)
            if (x) cudaGraphExecDestroy(x);
        graphs[0] = graphs[1] = nullptr;
    };
    for (int seg = last; seg >= 0; --seg) {
        cudaError_t ce = cudaSuccess;
        if (seg > 0)
            ce = cudaMemcpyAsync(tape[(seg - 1) & 1], ck + (size_t)(seg - 1) * state, state * 8,
                                 cudaMemcpyDeviceToDevice, s->stream);
        if (ce != cudaSuccess) {
            drop_graphs();
            return fail(CLIPB_E_CUDA, std::string("checkpoint restore: ") + cudaGetErrorString(ce));
        }
        if (K % 2 == 0 && seg > 0 && seg < last) {
            cudaGraphExec_t& ex = graphs[seg & 1];
            if (!ex) {
                cudaGraph_t gr = nullptr;
                ce = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
                const int r = ce == cudaSuccess ? iteration(seg) : 0;
                const cudaError_t ee = ce == cudaSuccess ? cudaStreamEndCapture(s->stream, &gr) : ce;
                if (ce == cudaSuccess && !r && ee == cudaSuccess) ce = cudaGraphInstantiate(&ex, gr, 0);
                else if (ce == cudaSuccess) ce = ee != cudaSuccess ? ee : cudaErrorUnknown;
                if (gr) cudaGraphDestroy(gr);
                if (ce != cudaSuccess) {
                    drop_graphs();
                    return r ? r : fail(CLIPB_E_CUDA, std::string("adjoint segment graph: ") + cudaGetErrorString(ce));
                }
            }
            ce = cudaGraphLaunch(ex, s->stream);
            if (ce != cudaSuccess) {
                drop_graphs();
                return fail(CLIPB_E_CUDA, std::string("adjoint segment: ") + cudaGetErrorString(ce));
            }
        } else if ((rc = iteration(seg))) {
            drop_graphs();
            return rc;
        }
    }
    drop_graphs();
    // ---- initial state and first collision
    adj_stream_kernel<<<gi, blk, 0, s->stream>>>(g, A);
    A.partials = partials;
    adj_init_node_kernel<<<gi, blk, 0, s->stream>>>(g, pd, pc, c0dev, A);
    accumulate3<<<1, 96, 0, s->stream>>>(partials, nblocks, acc);
    adj_init_c_kernel<<<ge, blk, 0, s->stream>>>(g, A, A.lclag, gc0);
    CLIPB_CUDA(cudaGetLastError());
    double hacc[3];
    CLIPB_CUDA(cudaMemcpyAsync(hacc, acc, sizeof(hacc), cudaMemcpyDeviceToHost, s->stream));
    std::vector<double> hg(ps);
    CLIPB_CUDA(cudaMemcpyAsync(hg.data(), gc0, ps * 8, cudaMemcpyDeviceToHost, s->stream));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    if (grad_params3) std::memcpy(grad_params3, hacc, sizeof(hacc));
    if (grad_c0) {
        const CaseConfig& cfg = s->cfg;
        for (int i = 0; i < cfg.extent[0]; ++i)
            for (int j = 0; j < cfg.extent[1]; ++j) grad_c0[(size_t)i * cfg.extent[1] + j] = hg[s->dev_index(i, j, 0)];
    }
    return CLIPB_OK;
}

}  // extern "C"
