// Tangent-linear model of the FP64 2D step, the forward objective and the parameter
// setter (C ABI in include/clipb.h); the adjoint is in adjoint_rev.cu.
//
// Objective: J = |X(c_N) - target|^2, X = sum(x c) / sum(c) over the interior (node
// coordinates in the reference's ghosted index convention), after N steps of the FP64
// forward from an initial c field.  Parameters: the body-force acceleration g_y, the
// surface tension sigma (kappa = 1.5 sigma W, beta = 8 sigma / W, and the initial pressure
// jump) and the mobility M (w_c = 1 / (1/2 + 3M)).  Walls and periodic sides.
//
// Tangent-linear model: the FP64 lattice functions instantiated on dual numbers (dual.cuh)
// in an unfused form of the step (c kernel, then update kernel); compiled without FMA
// contraction, its value part equals the FP64 forward bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "adjoint.cuh"
#include "clipb.h"
#include "dual.cuh"
#include "kernels.cuh"
#include "solver.hpp"

using namespace clipb;
using namespace clipb::adj;

namespace {

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

}  // namespace

namespace clipb {
namespace adj {

int check_case(clipb_solver* s) {
    if (s->st.precision != CLIPB_FP64) return fail(CLIPB_E_ARG, "the tangent-linear and adjoint paths run in FP64");
    if (s->cfg.dim != 2) return fail(CLIPB_E_ARG, "the tangent-linear and adjoint paths are 2D");
    if (s->st.g.vel_side >= 0 || s->st.g.open)
        return fail(CLIPB_E_ARG, "the tangent-linear and adjoint paths take wall and periodic sides");
    if (s->cfg.phys.caseType == kJet)
        return fail(CLIPB_E_ARG, "the tangent-linear and adjoint paths take drop, bubble and RTI cases");
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

}  // namespace adj
}  // namespace clipb

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

}  // extern "C"
