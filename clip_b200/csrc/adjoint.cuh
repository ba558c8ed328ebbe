// Internal: pieces shared by the tangent-linear model (adjoint.cu, compiled without FMA
// contraction so that its value part rounds like the FP64 step) and the adjoint
// (adjoint_rev.cu, compiled with contraction).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "clipb.h"
#include "kernels.cuh"
#include "solver.hpp"

namespace clipb {
namespace adj {

using L2 = Lat<2>;
constexpr int Q = 9;

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

// Parameter chain factors: d(beta4)/d(sigma), d(kappa)/d(sigma), d(wc)/dM.
struct ParamChain {
    double dbeta4_dsigma, dkappa_dsigma, dwc_dM, rref;
};

inline ParamChain chain(const PhysD& d) {
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

// FP64, 2D, walls and periodic sides only.
int check_case(clipb_solver* s);
// Host objective and its gradient with respect to c (device layout) from the interior c.
double objective(clipb_solver* s, const std::vector<double>& c_dev, const double* target, std::vector<double>* dJ);
int upload_c0(clipb_solver* s, const double* c0_host);

}  // namespace adj
}  // namespace clipb
