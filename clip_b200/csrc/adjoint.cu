// Tangent-linear model and hand-written adjoint of the FP64 2D step (C ABI in include/clipb.h).
//
// Objective: J = |X(c_N) - target|^2, X = sum(x c) / sum(c) over the interior (node
// coordinates in the reference's ghosted index convention), after N steps of the FP64
// forward from an initial c field.  Parameters: the body-force acceleration g_y, the
// surface tension sigma (kappa = 1.5 sigma W, beta = 8 sigma / W, and the initial pressure
// jump) and the mobility M (w_c = 1 / (1/2 + 3M)).  Walls and periodic sides.
//
// Tangent-linear model: the FP64 lattice functions instantiated on dual numbers (dual.cuh)
// in an unfused form of the step (c kernel, then update kernel); its value part equals the
// FP64 forward bit for bit.
//
// Adjoint: per reverse step k, (1) a node kernel recomputes the node's update from the
// stored state of step k in the moment form of the collision (moment_hydro/lean_update:
// the same operator as the reference's WMRT sequence) and applies its transposed Jacobian
// to the adjoints of the node's outputs (f, g, u, c); (2) a kernel applies the transposed
// mu / grad c stencils and the c = sum g_post reduction (ghost-layer reads go to the
// lagged c of step k); (3) a kernel applies the transposed pull streaming (bounce-back
// and periodic wrap included).  The forward states of a segment of K steps are recomputed
// from a checkpoint (every K steps) and kept on the device while the segment is reversed.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "clipb.h"
#include "kernels.cuh"
#include "dual.cuh"
#include "solver.hpp"

using namespace clipb;

namespace {

using L2 = Lat<2>;
constexpr int Q = 9;

// ---------------------------------------------------------------- shared helpers
// Laplacian (a) and gradient (bx, by) weights of the 9-point stencils (NsAllen.cu:207-236,
// 280-322) for offset (ox, oy).
__device__ __forceinline__ void coef2(int ox, int oy, double& a, double& bx, double& by) {
    const int n = (ox != 0) + (oy != 0);
    a = n == 0 ? -20.0 / 6.0 : (n == 1 ? 4.0 / 6.0 : 1.0 / 6.0);
    bx = ox == 0 ? 0.0 : (oy == 0 ? ox / 3.0 : ox / 12.0);
    by = oy == 0 ? 0.0 : (ox == 0 ? oy / 3.0 : oy / 12.0);
}

// Interior node whose c a ghost position holds (mirror on walls, wrap on periodic axes).
__device__ __forceinline__ long long ghost_source(const Geom& g, int x, int y) {
    int s[2] = {x, y};
    for (int a = 0; a < 2; ++a) {
        s[a] = s[a] < 0 ? 0 : (s[a] > g.n[a] + 1 ? g.n[a] + 1 : s[a]);
        if (s[a] < 1) s[a] = g.per[a] ? s[a] + g.n[a] : 1;
        else if (s[a] > g.n[a]) s[a] = g.per[a] ? s[a] - g.n[a] : g.n[a];
    }
    return nidx(g, s[0], s[1], 0);
}

__device__ __forceinline__ bool interior2(const Geom& g, int x, int y) {
    return x >= 1 && x <= g.n[0] && y >= 1 && y <= g.n[1];
}

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

// Parameter chain factors: d(beta4)/d(sigma), d(kappa)/d(sigma), d(wc)/dM.
struct ParamChain {
    double dbeta4_dsigma, dkappa_dsigma, dwc_dM, rref;
};

// ---------------------------------------------------------------- tangent-linear model
struct DualBufs {
    Dual* f[2];
    Dual* g[2];
    Dual* c[2];
    Dual* u;
};

__global__ void tlm_init_kernel(Geom g, PhysD pd, Phys<Dual> P, Dual sigma, const double* c0v, const double* c0d,
                                DualBufs b) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= g.e[0] || y >= g.e[1]) return;
    const long long self = nidx(g, x, y, 0);
    const bool interior = interior2(g, x, y);
    auto Cf = [&](int dx, int dy, int) {
        const long long i = nidx(g, x + dx, y + dy, 0);
        return Dual(c0v[i], c0d[i]);
    };
    Dual c, mu, dc[3], rho, p, f0[Q], g0[Q];
    initial_state<2, Dual>(pd, sigma, P, Cf, interior, c, mu, dc, rho, p, f0, g0);
    b.c[0][self] = c;
    b.c[1][self] = c;
    b.u[self] = Dual(0.0);
    b.u[g.ps + self] = Dual(0.0);
    if (interior) {
        const Dual u0[3] = {Dual(0.0), Dual(0.0), Dual(0.0)};
        Dual go[Q], fo[Q];
        collide_g<2, Dual>(P, g0, c, dc, u0, go);
        collide_f<2, Dual>(P, f0, c, mu, dc, rho, p, u0, fo);
        for (int q = 0; q < Q; ++q) {
            b.f[0][q * g.ps + self] = fo[q];
            b.g[0][q * g.ps + self] = go[q];
        }
    } else {
        for (int q = 0; q < Q; ++q)
            for (int k = 0; k < 2; ++k) {
                b.f[k][q * g.ps + self] = f0[q];
                b.g[k][q * g.ps + self] = g0[q];
            }
    }
}

// c of step k: sum of the pulled g of buffer `in`, into c[out]
__global__ void tlm_c_kernel(Geom g, DualBufs b, int in) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1, y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (x > g.n[0] || y > g.n[1]) return;
    const long long self = nidx(g, x, y, 0);
    Dual c;
    for (int q = 0; q < Q; ++q) {
        int qs;
        bool crossed;
        const long long src = pull_source<2>(g, q, x, y, 0, self, qs, crossed);
        const Dual v = b.g[in][qs * g.ps + src];
        c = q == 0 ? v : c + v;
    }
    b.c[in ^ 1][self] = c;
}

__global__ void tlm_step_kernel(Geom g, Phys<Dual> P, DualBufs b, int in) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1, y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (x > g.n[0] || y > g.n[1]) return;
    const int out = in ^ 1;
    const long long self = nidx(g, x, y, 0);
    Dual fp[Q], gp[Q];
    for (int q = 0; q < Q; ++q) {
        int qs;
        bool crossed;
        const long long src = pull_source<2>(g, q, x, y, 0, self, qs, crossed);
        fp[q] = b.f[in][qs * g.ps + src];
        gp[q] = b.g[in][qs * g.ps + src];
    }
    auto Cf = [&](int dx, int dy, int) {
        const int xx = x + dx, yy = y + dy;
        return interior2(g, xx, yy) ? b.c[out][nidx(g, xx, yy, 0)] : b.c[in][ghost_source(g, xx, yy)];
    };
    const Dual c = Cf(0, 0, 0);
    Dual mu, dc[3];
    dc[2] = Dual(0.0);
    stencil<2, Dual>(P, Cf, mu, dc);
    Dual u[3] = {b.u[self], b.u[g.ps + self], Dual(0.0)}, p, rho, go[Q], fo[Q];
    macroscopic<2, Dual>(P, fp, c, mu, dc, u, p, rho);
    collide_g<2, Dual>(P, gp, c, dc, u, go);
    collide_f<2, Dual>(P, fp, c, mu, dc, rho, p, u, fo);
    for (int q = 0; q < Q; ++q) {
        b.f[out][q * g.ps + self] = fo[q];
        b.g[out][q * g.ps + self] = go[q];
    }
    b.u[self] = u[0];
    b.u[g.ps + self] = u[1];
}

// ---------------------------------------------------------------- adjoint
struct Tape {  // one stored forward state (the input of a step), device layout
    double* f;
    double* g;
    double* c;
    double* u;
};

struct AdjBufs {
    double* lf;    // adjoint of F (Q planes): of step k+1's input on entry, of step k's on exit
    double* lg;
    double* lu;    // adjoint of U (2 planes), updated in place
    double* lc[2]; // adjoint of the stored c: [0] of step k+1 (read), [1] of step k (scattered)
    double* lfp;   // adjoint of the pulled f of every node (Q planes)
    double* lgp;   // adjoint of the pulled g (Q planes), then plus the adjoint of c
    double* lcl;   // adjoint of c from the node's own update
    double* llap;  // adjoint of the Laplacian of c at the node
    double* ldc;   // adjoint of grad c (2 planes)
    double* partials;
};

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

// (1) node-local reverse of step k at every interior node.
__global__ void adj_node_kernel(Geom g, PhysD pd, ParamChain pc, Tape in, const double* c_out, AdjBufs A) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1, y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    double pg = 0.0, psig = 0.0, pmob = 0.0;
    if (x <= g.n[0] && y <= g.n[1]) {
        const long long self = nidx(g, x, y, 0);
        const long long ps = g.ps;
        A.lc[1][self] = 0.0;  // receives the ghost-layer scatter of this step (adj_c_kernel)
        double fp[Q], gp[Q];
        for (int q = 0; q < Q; ++q) {
            int qs;
            bool crossed;
            const long long src = pull_source<2>(g, q, x, y, 0, self, qs, crossed);
            fp[q] = in.f[qs * ps + src];
            gp[q] = in.g[qs * ps + src];
        }
        // stencils of c (interior: this step's c, ghosts: the lagged c of step k)
        double lap = 0.0, dc[2] = {0.0, 0.0};
        for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) {
                const int xx = x + ox, yy = y + oy;
                const double cv = interior2(g, xx, yy) ? c_out[nidx(g, xx, yy, 0)] : in.c[ghost_source(g, xx, yy)];
                double a, bx, by;
                coef2(ox, oy, a, bx, by);
                lap += a * cv;
                dc[0] += bx * cv;
                dc[1] += by * cv;
            }
        const double c = c_out[self];
        const double poly = c * (c - 1.0) * (c - 0.5), dpoly = (3.0 * c - 3.0) * c + 0.5;
        const double mu = pd.beta4 * poly - pd.kappa * lap;
        // hydrodynamic moments
        double p = 0.0, j[2] = {0.0, 0.0}, Pi[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
        for (int q = 0; q < Q; ++q) {
            const int e[2] = {L2::ex(q), L2::ey(q)};
            p += fp[q];
            for (int a = 0; a < 2; ++a) {
                j[a] += e[a] * fp[q];
                for (int bb = 0; bb < 2; ++bb) Pi[a][bb] += e[a] * e[bb] * fp[q];
            }
        }
        const double rho = pd.RhoL + c * pd.drho;
        double tau, dtdc;
        if (c < 0.0) { tau = pd.tauL; dtdc = 0.0; }
        else if (c > 1.0) { tau = pd.tauH; dtdc = 0.0; }
        else { tau = pd.tauL + c * pd.dtau; dtdc = pd.dtau; }
        const double s9 = 1.0 / (tau + 0.5), kvis = -tau * pd.drho, fcap = mu - p * pd.drho3, p3 = p / 3.0;
        const double gfac = pd.caseType == 2 ? rho : rho - pc.rref;
        const double grav[2] = {gfac * pd.g[0], gfac * pd.g[1]};
        const double uprev[2] = {in.u[self], in.u[ps + self]};
        Force f1, f2;
        force_fwd(uprev, Pi, p3, s9, kvis, fcap, dc, grav, f1);
        const double h = 0.5 / rho;
        const double u[2] = {j[0] + f1.F[0] * h, j[1] + f1.F[1] * h};
        force_fwd(u, Pi, p3, s9, kvis, fcap, dc, grav, f2);
        const double U2 = u[0] * u[0] + u[1] * u[1], sm1 = s9 - 1.0;
        // phase field
        const double mag = sqrt(dc[0] * dc[0] + dc[1] * dc[1]), m = mag + 1e-32;
        const double nrm[2] = {dc[0] / m, dc[1] / m};
        const double cm = c - 0.5, pf = 1.0 - 4.0 * cm * cm, pref = pd.amob3 * pf / pd.W;

        // ---- reverse
        double lc = A.lc[0][self], lmu = 0.0, ldcv[2] = {0.0, 0.0}, lu[2] = {A.lu[self], A.lu[ps + self]};
        double lp = 0.0, lrho = 0.0, ls9 = 0.0, lU2 = 0.0, lwc = 0.0, lamob3 = 0.0, lpref = 0.0;
        double lnrm[2] = {0.0, 0.0}, lF2[2] = {0.0, 0.0}, ldev2[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
        for (int q = 0; q < Q; ++q) {
            const int e[2] = {L2::ex(q), L2::ey(q)};
            const double w = L2::w(q);
            const double eu = e[0] * u[0] + e[1] * u[1], eF = e[0] * f2.F[0] + e[1] * f2.F[1];
            const double en = e[0] * nrm[0] + e[1] * nrm[1];
            double phi = 0.0;
            for (int a = 0; a < 2; ++a)
                for (int bb = 0; bb < 2; ++bb) phi += 4.5 * e[a] * e[bb] * f2.dev[a][bb];
            // g output
            const double lgo = A.lg[q * ps + self];
            const double ga = w * (3.0 * eu + 4.5 * eu * eu - 1.5 * U2);
            const double H = c * (ga + w) + w * pref * en;
            A.lgp[q * ps + self] = lgo * pd.one_minus_wc;
            lwc += lgo * (H - gp[q]);
            const double lH = lgo * pd.wc;
            lc += lH * (ga + w);
            const double lga = lH * c;
            double leu = lga * w * (3.0 + 9.0 * eu);
            lU2 += lga * w * -1.5;
            lpref += lH * w * en;
            const double len = lH * w * pref;
            lnrm[0] += len * e[0];
            lnrm[1] += len * e[1];
            // f output
            const double lfo = A.lf[q * ps + self];
            lp += w * lfo;
            leu += w * lfo * (3.0 + 9.0 * eu);
            lU2 += w * lfo * -1.5;
            const double leF = w * lfo * 1.5 / rho;
            lF2[0] += leF * e[0];
            lF2[1] += leF * e[1];
            lrho += -w * lfo * 1.5 * eF / (rho * rho);
            ls9 += -w * lfo * phi;  // d/d(s9) of -(s9 - 1) phi
            const double lphi = -w * lfo * sm1;
            for (int a = 0; a < 2; ++a)
                for (int bb = 0; bb < 2; ++bb) ldev2[a][bb] += lphi * 4.5 * e[a] * e[bb];
            lu[0] += leu * e[0];
            lu[1] += leu * e[1];
        }
        lu[0] += 2.0 * u[0] * lU2;
        lu[1] += 2.0 * u[1] * lU2;
        lc += lpref * pd.amob3 * (-8.0 * cm) / pd.W;
        lamob3 += lpref * pf / pd.W;
        {  // interface normal, derivative damped as in the tangent-linear model (dual.cuh)
            const double sc = normal_damping(mag, c, pd.W);
            const double t = mag > 0.0 ? (lnrm[0] * dc[0] + lnrm[1] * dc[1]) / (mag * m * m) : 0.0;
            for (int bb = 0; bb < 2; ++bb) ldcv[bb] += sc * (lnrm[bb] / m - t * dc[bb]);
        }
        // force at this step's velocity
        ForceAdj FA{};
        force_rev(u, f2, s9, kvis, fcap, dc, lF2, ldev2, FA);
        lu[0] += FA.luu[0];
        lu[1] += FA.luu[1];
        // u = j + F(uprev) h
        double lj[2] = {lu[0], lu[1]}, lF1[2] = {lu[0] * h, lu[1] * h};
        lrho += (lu[0] * f1.F[0] + lu[1] * f1.F[1]) * (-0.5 / (rho * rho));
        FA.luu[0] = FA.luu[1] = 0.0;
        force_rev(uprev, f1, s9, kvis, fcap, dc, lF1, nullptr, FA);
        A.lu[self] = FA.luu[0];
        A.lu[ps + self] = FA.luu[1];
        // scalars
        lp += FA.lp3 / 3.0 - pd.drho3 * FA.lfcap;
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
        for (int q = 0; q < Q; ++q) {
            const int e[2] = {L2::ex(q), L2::ey(q)};
            double v = lp + e[0] * lj[0] + e[1] * lj[1];
            for (int a = 0; a < 2; ++a)
                for (int bb = 0; bb < 2; ++bb) v += e[a] * e[bb] * FA.lPi[a][bb];
            A.lfp[q * ps + self] = v;
        }
    }
    block_sum3(pg, psig, pmob, A.partials);
}

// (2) transposed stencils and c = sum g_post: adjoint of c at every interior node, added to
// the adjoint of each pulled g; ghost-layer reads scatter into the adjoint of the lagged c.
__global__ void adj_c_kernel(Geom g, AdjBufs A) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1, y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (x > g.n[0] || y > g.n[1]) return;
    const long long self = nidx(g, x, y, 0), ps = g.ps;
    double lc = A.lcl[self];
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
                atomicAdd(&A.lc[1][ghost_source(g, gx, gy)], A.llap[self] * a + A.ldc[self] * bx + A.ldc[ps + self] * by);
        }
    for (int q = 0; q < Q; ++q) A.lgp[q * ps + self] += lc;
}

// (3) transposed pull: the adjoint of stored value (s, q) is that of the pulled value it
// became: (s + e_q, q), wrapped on periodic axes, or (s, opposite(q)) by bounce-back.
__global__ void adj_stream_kernel(Geom g, AdjBufs A) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1, y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (x > g.n[0] || y > g.n[1]) return;
    const long long self = nidx(g, x, y, 0), ps = g.ps;
    for (int q = 0; q < Q; ++q) {
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
        long long n;
        int qd;
        if (bb) {
            n = self;
            qd = opposite<2>(q);
        } else {
            n = nidx(g, d[0], d[1], 0);
            qd = q;
        }
        A.lf[q * ps + self] = A.lfp[qd * ps + n];
        A.lg[q * ps + self] = A.lgp[qd * ps + n];
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

// ---------------------------------------------------------------- host side
int check_case(clipb_solver* s) {
    if (s->st.precision != CLIPB_FP64) return fail(CLIPB_E_ARG, "the tangent-linear and adjoint paths run in FP64");
    if (s->cfg.dim != 2) return fail(CLIPB_E_ARG, "the tangent-linear and adjoint paths are 2D");
    if (s->st.g.vel_side >= 0 || s->st.g.open)
        return fail(CLIPB_E_ARG, "the tangent-linear and adjoint paths take wall and periodic sides");
    return CLIPB_OK;
}

// Host objective and its gradient with respect to c (device layout) from the interior c.
double objective(clipb_solver* s, const std::vector<double>& c_dev, const double* target, std::vector<double>* dJ) {
    const Geom& g = s->st.g;
    double M = 0.0, X[2] = {0.0, 0.0};
    for (int y = 1; y <= g.n[1]; ++y)
        for (int x = 1; x <= g.n[0]; ++x) {
            const double c = c_dev[g.base + x + (long long)y * g.sy];
            M += c;
            X[0] += x * c;
            X[1] += y * c;
        }
    X[0] /= M;
    X[1] /= M;
    const double r[2] = {X[0] - target[0], X[1] - target[1]};
    if (dJ) {
        dJ->assign((size_t)g.ps, 0.0);
        for (int y = 1; y <= g.n[1]; ++y)
            for (int x = 1; x <= g.n[0]; ++x)
                (*dJ)[g.base + x + (long long)y * g.sy] = 2.0 * (r[0] * (x - X[0]) + r[1] * (y - X[1])) / M;
    }
    return r[0] * r[0] + r[1] * r[1];
}

int upload_c0(clipb_solver* s, const double* c0_host) {
    return clipb_device_initializer(s, c0_host);
}

ParamChain chain(const PhysD& d) {
    ParamChain pc;
    pc.dbeta4_dsigma = 4.0 * 8.0 / d.W;
    pc.dkappa_dsigma = 1.50 * d.W;
    pc.dwc_dM = -3.0 * d.wc * d.wc;
    pc.rref = d.caseType == 0 ? d.RhoH : (d.caseType == 1 ? d.RhoL : 0.0);
    return pc;
}

struct DevVec {  // owned device allocation
    void* p = nullptr;
    ~DevVec() { cudaFree(p); }
    cudaError_t alloc(size_t bytes) {
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) e = cudaMemset(p, 0, bytes);
        return e;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

}  // namespace

extern "C" {

int clipb_set_params(clipb_solver* s, double gy, double sigma, double mobility) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    Physics& P = s->cfg.phys;
    PhysD& d = s->st.phys;
    P.gravity[1] = gy;
    P.sigma = sigma;
    P.kConstant = 1.50 * P.sigma * P.interfaceWidth;
    P.betaConstant = 8.0 * P.sigma / P.interfaceWidth;
    P.mobility = mobility;
    d.g[1] = gy;
    d.sigma = sigma;
    d.kappa = P.kConstant;
    d.beta4 = 4.0 * P.betaConstant;
    d.mobility = mobility;
    d.wc = 1.0 / (0.50 + 3.0 * mobility);
    d.one_minus_wc = 1.0 - d.wc;
    d.amob3 = 3.0 * mobility;
    s->drop_graph();  // kernel arguments are captured by value
    return CLIPB_OK;
}

int clipb_objective(clipb_solver* s, const double* c0_host, int nsteps, const double* target, double* J) {
    if (!s || !target || !J) return fail(CLIPB_E_ARG, "null argument");
    int rc = check_case(s);
    if (rc) return rc;
    if ((rc = upload_c0(s, c0_host))) return rc;
    if ((rc = clipb_solve(s, nsteps))) return rc;
    std::vector<double> c((size_t)s->st.g.ps);
    CLIPB_CUDA(cudaMemcpyAsync(c.data(), s->st.c[nsteps & 1], c.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    *J = objective(s, c, target, nullptr);
    return CLIPB_OK;
}

int clipb_tangent(clipb_solver* s, const double* c0_host, int nsteps, const double* target, const double* dc0_host,
                  const double* dparams3, double* J, double* dJ) {
    if (!s || !target || !J || !dJ) return fail(CLIPB_E_ARG, "null argument");
    int rc = check_case(s);
    if (rc) return rc;
    // initial c on the host (reference layout) -> device layout values and tangents
    const CaseConfig& cfg = s->cfg;
    if (!c0_host) {
        if ((rc = clipb_initial_condition(s, nullptr))) return rc;
        c0_host = s->host_c.data();
    }
    const Geom& g = s->st.g;
    std::vector<double> cv((size_t)g.ps, 0.0), cd((size_t)g.ps, 0.0);
    for (int i = 0; i < cfg.extent[0]; ++i)
        for (int j = 0; j < cfg.extent[1]; ++j) {
            const size_t r = (size_t)i * cfg.extent[1] + j;
            cv[s->dev_index(i, j, 0)] = c0_host[r];
            if (dc0_host) cd[s->dev_index(i, j, 0)] = dc0_host[r];
        }
    const double dp[3] = {dparams3 ? dparams3[0] : 0.0, dparams3 ? dparams3[1] : 0.0, dparams3 ? dparams3[2] : 0.0};
    const PhysD& d = s->st.phys;
    Phys<Dual> P;
    {
        const Phys<double> PD = [&] {
            Phys<double> t;
            t.RhoL = d.RhoL; t.RhoH = d.RhoH; t.drho = d.drho; t.drho3 = d.drho3;
            t.tauL = d.tauL; t.tauH = d.tauH; t.dtau = d.dtau; t.kappa = d.kappa; t.beta4 = d.beta4;
            t.mobility = d.mobility; t.W = d.W; t.wc = d.wc; t.one_minus_wc = d.one_minus_wc; t.amob3 = d.amob3;
            t.g[0] = d.g[0]; t.g[1] = d.g[1]; t.g[2] = d.g[2]; t.caseType = d.caseType;
            return t;
        }();
        P.RhoL = PD.RhoL; P.RhoH = PD.RhoH; P.drho = PD.drho; P.drho3 = PD.drho3;
        P.tauL = PD.tauL; P.tauH = PD.tauH; P.dtau = PD.dtau;
        P.kappa = Dual(PD.kappa, 1.50 * d.W * dp[1]);
        P.beta4 = Dual(PD.beta4, 4.0 * 8.0 / d.W * dp[1]);
        P.mobility = Dual(PD.mobility, dp[2]);
        P.W = PD.W;
        const double dwc = -3.0 * d.wc * d.wc * dp[2];
        P.wc = Dual(PD.wc, dwc);
        P.one_minus_wc = Dual(PD.one_minus_wc, -dwc);
        P.amob3 = Dual(PD.amob3, 3.0 * dp[2]);
        P.g[0] = PD.g[0];
        P.g[1] = Dual(PD.g[1], dp[0]);
        P.g[2] = PD.g[2];
        P.caseType = PD.caseType;
    }
    const Dual sigma(d.sigma, dp[1]);
    const size_t ps = (size_t)g.ps;
    DevVec mem, c0v, c0d;
    const size_t nd = 4 * Q * ps + 2 * ps + 2 * ps;
    cudaError_t e = mem.alloc(nd * sizeof(Dual));
    if (e == cudaSuccess) e = c0v.alloc(ps * sizeof(double));
    if (e == cudaSuccess) e = c0d.alloc(ps * sizeof(double));
    if (e != cudaSuccess) return fail(CLIPB_E_NOMEM, std::string("tangent-linear buffers: ") + cudaGetErrorString(e));
    CLIPB_CUDA(cudaMemcpy(c0v.p, cv.data(), ps * sizeof(double), cudaMemcpyHostToDevice));
    CLIPB_CUDA(cudaMemcpy(c0d.p, cd.data(), ps * sizeof(double), cudaMemcpyHostToDevice));
    DualBufs b;
    Dual* base = mem.as<Dual>();
    b.f[0] = base;
    b.f[1] = base + Q * ps;
    b.g[0] = base + 2 * Q * ps;
    b.g[1] = base + 3 * Q * ps;
    b.c[0] = base + 4 * Q * ps;
    b.c[1] = base + 4 * Q * ps + ps;
    b.u = base + 4 * Q * ps + 2 * ps;
    const dim3 blk(32, 8);
    const dim3 ge((g.e[0] + 31) / 32, (g.e[1] + 7) / 8), gi((g.n[0] + 31) / 32, (g.n[1] + 7) / 8);
    tlm_init_kernel<<<ge, blk, 0, s->stream>>>(g, d, P, sigma, c0v.as<double>(), c0d.as<double>(), b);
    CLIPB_CUDA(cudaGetLastError());
    for (int k = 0; k < nsteps; ++k) {
        tlm_c_kernel<<<gi, blk, 0, s->stream>>>(g, b, k & 1);
        tlm_step_kernel<<<gi, blk, 0, s->stream>>>(g, P, b, k & 1);
    }
    CLIPB_CUDA(cudaGetLastError());
    std::vector<Dual> c(ps);
    CLIPB_CUDA(cudaMemcpyAsync(c.data(), b.c[nsteps & 1], ps * sizeof(Dual), cudaMemcpyDeviceToHost, s->stream));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    std::vector<double> val(ps), grad;
    for (size_t i = 0; i < ps; ++i) val[i] = c[i].v;
    *J = objective(s, val, target, &grad);
    double t = 0.0;
    for (int y = 1; y <= g.n[1]; ++y)
        for (int x = 1; x <= g.n[0]; ++x) {
            const size_t i = g.base + x + (size_t)y * g.sy;
            t += grad[i] * c[i].d;
        }
    *dJ = t;
    return CLIPB_OK;
}

int clipb_adjoint(clipb_solver* s, const double* c0_host, int nsteps, const double* target, int checkpoint_every,
                  double* J, double* grad_c0, double* grad_params3) {
    if (!s || !target || !J) return fail(CLIPB_E_ARG, "null argument");
    if (nsteps < 1) return fail(CLIPB_E_ARG, "need at least one step");
    int rc = check_case(s);
    if (rc) return rc;
    const int K = checkpoint_every > 0 ? checkpoint_every : 100;
    const Geom& g = s->st.g;
    const size_t ps = (size_t)g.ps;
    const size_t state = (2 * Q + 1 + 2) * ps;  // f, g, c, u
    const int nck = (nsteps + K - 1) / K;
    // ---- forward with checkpoints (the input state of steps 0, K, 2K, ...)
    if ((rc = upload_c0(s, c0_host))) return rc;
    DevVec ck, tape, adj, c0dev, gc0, fin;
    cudaError_t e = ck.alloc((size_t)nck * state * sizeof(double));
    if (e == cudaSuccess) e = fin.alloc(state * sizeof(double));
    if (e == cudaSuccess) e = tape.alloc((size_t)(K + 1) * state * sizeof(double));
    const size_t nadj = 4 * Q * ps + 2 * ps + 2 * ps + 5 * ps;
    const dim3 blk(32, 8), gi((g.n[0] + 31) / 32, (g.n[1] + 7) / 8), ge((g.e[0] + 31) / 32, (g.e[1] + 7) / 8);
    const int nblocks = (int)(gi.x * gi.y);
    if (e == cudaSuccess) e = adj.alloc((nadj + 3 * (size_t)nblocks * K + 3) * sizeof(double));
    if (e == cudaSuccess) e = c0dev.alloc(ps * sizeof(double));
    if (e == cudaSuccess) e = gc0.alloc(ps * sizeof(double));
    if (e != cudaSuccess) return fail(CLIPB_E_NOMEM, std::string("adjoint buffers: ") + cudaGetErrorString(e));
    CLIPB_CUDA(cudaMemcpyAsync(c0dev.p, s->st.c0, ps * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
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
    auto restore = [&](const Tape& t, long long step) -> int {
        const int b = (int)(step & 1);
        CLIPB_CUDA(cudaMemcpyAsync(s->st.f[b], t.f, Q * ps * 8, cudaMemcpyDeviceToDevice, s->stream));
        CLIPB_CUDA(cudaMemcpyAsync(s->st.gp[b], t.g, Q * ps * 8, cudaMemcpyDeviceToDevice, s->stream));
        CLIPB_CUDA(cudaMemcpyAsync(s->st.c[b], t.c, ps * 8, cudaMemcpyDeviceToDevice, s->stream));
        CLIPB_CUDA(cudaMemcpyAsync(s->st.u, t.u, 2 * ps * 8, cudaMemcpyDeviceToDevice, s->stream));
        s->steps = step;
        return CLIPB_OK;
    };
    // forward: checkpoints at steps 0, K, 2K, ... (graph replays between them)
    for (int seg = 0; seg < nck; ++seg) {
        if ((rc = save(view(ck.as<double>() + (size_t)seg * state)))) return rc;
        if ((rc = clipb_solve(s, std::min(K, nsteps - seg * K)))) return rc;
    }
    if ((rc = save(view(fin.as<double>())))) return rc;
    std::vector<double> c((size_t)ps), dJ;
    CLIPB_CUDA(cudaMemcpyAsync(c.data(), s->st.c[nsteps & 1], ps * 8, cudaMemcpyDeviceToHost, s->stream));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    *J = objective(s, c, target, &dJ);
    // ---- adjoint buffers
    double* a0 = adj.as<double>();
    AdjBufs A;
    A.lf = a0;
    A.lg = a0 + Q * ps;
    A.lfp = a0 + 2 * Q * ps;
    A.lgp = a0 + 3 * Q * ps;
    A.lu = a0 + 4 * Q * ps;
    A.ldc = a0 + 4 * Q * ps + 2 * ps;
    A.lc[0] = a0 + 4 * Q * ps + 4 * ps;
    A.lc[1] = a0 + 4 * Q * ps + 5 * ps;
    A.lcl = a0 + 4 * Q * ps + 6 * ps;
    A.llap = a0 + 4 * Q * ps + 7 * ps;
    double* partials = a0 + nadj;  // 3 x nblocks per reverse step of a segment
    double* acc = partials + 3 * (size_t)nblocks * K;
    CLIPB_CUDA(cudaMemcpyAsync(A.lc[0], dJ.data(), ps * 8, cudaMemcpyHostToDevice, s->stream));
    const PhysD pd = s->st.phys;
    const ParamChain pc = chain(pd);
    double* tp = tape.as<double>();
    // recompute the inputs of steps k0 .. k0 + len - 1 (and the state after them) into the
    // tape, by pointing the solver's buffers at tape entries; u is updated in place, so
    // each step first copies it forward
    const DevState saved = s->st;
    auto recompute = [&](int k0, int len) -> int {
        for (int i = 0; i < len; ++i) {
            const int k = k0 + i, b = k & 1;
            const Tape ti = view(tp + (size_t)i * state), tn = view(tp + (size_t)(i + 1) * state);
            s->st.f[b] = ti.f;
            s->st.gp[b] = ti.g;
            s->st.c[b] = ti.c;
            s->st.f[b ^ 1] = tn.f;
            s->st.gp[b ^ 1] = tn.g;
            s->st.c[b ^ 1] = tn.c;
            s->st.u = tn.u;
            CLIPB_CUDA(cudaMemcpyAsync(tn.u, ti.u, 2 * ps * 8, cudaMemcpyDeviceToDevice, s->stream));
            CLIPB_CUDA(s->kt.step(s->st, k, s->stream));
        }
        return CLIPB_OK;
    };
    auto reverse = [&](int k0, int len) -> int {
        for (int i = len - 1; i >= 0; --i) {
            const Tape in = view(tp + (size_t)i * state);
            const double* c_out = tp + (size_t)(i + 1) * state + 2 * Q * ps;
            A.partials = partials + 3 * (size_t)nblocks * i;
            adj_node_kernel<<<gi, blk, 0, s->stream>>>(g, pd, pc, in, c_out, A);
            adj_c_kernel<<<gi, blk, 0, s->stream>>>(g, A);
            adj_stream_kernel<<<gi, blk, 0, s->stream>>>(g, A);
            CLIPB_CUDA(cudaGetLastError());
            std::swap(A.lc[0], A.lc[1]);  // the scattered adjoint of c_k is the next step's input
        }
        (void)k0;
        return CLIPB_OK;
    };
    // full segments of even length replay one captured graph (same tape entries, same
    // parities, and the adjoint-of-c buffers back in place after an even number of swaps)
    cudaGraphExec_t seg_graph = nullptr;
    auto drop_seg_graph = [&]() {
        if (seg_graph) cudaGraphExecDestroy(seg_graph);
        seg_graph = nullptr;
    };
    const bool graphs = K % 2 == 0 && nsteps >= 2 * K;
    for (int seg = nck - 1; seg >= 0; --seg) {
        const int k0 = seg * K, len = std::min(nsteps, k0 + K) - k0;
        cudaError_t ce = cudaMemcpyAsync(tp, ck.as<double>() + (size_t)seg * state, state * 8, cudaMemcpyDeviceToDevice,
                                         s->stream);
        if (ce != cudaSuccess) {
            drop_seg_graph();
            s->st = saved;
            return fail(CLIPB_E_CUDA, std::string("checkpoint restore: ") + cudaGetErrorString(ce));
        }
        if (graphs && len == K) {
            if (!seg_graph) {
                cudaGraph_t gr = nullptr;
                ce = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
                int r1 = ce == cudaSuccess ? recompute(k0, len) : 0;
                int r2 = (ce == cudaSuccess && !r1) ? reverse(k0, len) : 0;
                const cudaError_t ee = cudaStreamEndCapture(s->stream, &gr);
                if (ce == cudaSuccess && !r1 && !r2 && ee == cudaSuccess) ce = cudaGraphInstantiate(&seg_graph, gr, 0);
                else if (ce == cudaSuccess) ce = ee != cudaSuccess ? ee : cudaErrorUnknown;
                if (gr) cudaGraphDestroy(gr);
                if (ce != cudaSuccess) {
                    drop_seg_graph();
                    s->st = saved;
                    return fail(CLIPB_E_CUDA, std::string("adjoint segment graph: ") + cudaGetErrorString(ce));
                }
            }
            ce = cudaGraphLaunch(seg_graph, s->stream);
        } else {
            rc = recompute(k0, len);
            if (!rc) rc = reverse(k0, len);
            ce = rc ? cudaErrorUnknown : cudaSuccess;
        }
        if (ce == cudaSuccess) {
            accumulate3<<<1, 96, 0, s->stream>>>(partials, len * nblocks, acc);
            ce = cudaGetLastError();
        }
        if (ce != cudaSuccess) {
            drop_seg_graph();
            s->st = saved;
            return rc ? rc : fail(CLIPB_E_CUDA, std::string("adjoint segment: ") + cudaGetErrorString(ce));
        }
    }
    drop_seg_graph();
    s->st = saved;
    // ---- initial state
    A.partials = partials;
    adj_init_node_kernel<<<gi, blk, 0, s->stream>>>(g, pd, pc, c0dev.as<double>(), A);
    accumulate3<<<1, 96, 0, s->stream>>>(partials, nblocks, acc);
    adj_init_c_kernel<<<ge, blk, 0, s->stream>>>(g, A, A.lc[0], gc0.as<double>());
    CLIPB_CUDA(cudaGetLastError());
    double hacc[3];
    CLIPB_CUDA(cudaMemcpyAsync(hacc, acc, sizeof(hacc), cudaMemcpyDeviceToHost, s->stream));
    std::vector<double> hg(ps);
    CLIPB_CUDA(cudaMemcpyAsync(hg.data(), gc0.p, ps * 8, cudaMemcpyDeviceToHost, s->stream));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    if (grad_params3) std::memcpy(grad_params3, hacc, sizeof(hacc));
    if (grad_c0) {
        const CaseConfig& cfg = s->cfg;
        for (int i = 0; i < cfg.extent[0]; ++i)
            for (int j = 0; j < cfg.extent[1]; ++j) grad_c0[(size_t)i * cfg.extent[1] + j] = hg[s->dev_index(i, j, 0)];
    }
    // leave the solver at the end of the forward run
    if ((rc = restore(view(fin.as<double>()), nsteps))) return rc;
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    return CLIPB_OK;
}

}  // extern "C"
