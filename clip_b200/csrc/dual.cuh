// Forward-mode dual numbers (value, tangent) for the tangent-linear model: the FP64
// lattice functions of lattice.cuh are templates on their arithmetic type, so instantiating
// them on Dual propagates a directional derivative through exactly the operations (and,
// compiled without FMA contraction, the rounding) of the FP64 step.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "lattice.cuh"

namespace clipb {

using ::sqrt;  // keep the double overload visible beside the Dual one below

struct Dual {
    double v, d;
    __host__ __device__ Dual() : v(0.0), d(0.0) {}
    __host__ __device__ Dual(double x) : v(x), d(0.0) {}  // NOLINT: constants enter as T(x)
    __host__ __device__ Dual(double x, double t) : v(x), d(t) {}
};

__host__ __device__ inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__host__ __device__ inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__host__ __device__ inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__host__ __device__ inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__host__ __device__ inline Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
__host__ __device__ inline Dual& operator+=(Dual& a, Dual b) { return a = a + b; }
__host__ __device__ inline Dual& operator-=(Dual& a, Dual b) { return a = a - b; }
__host__ __device__ inline Dual& operator*=(Dual& a, Dual b) { return a = a * b; }
__host__ __device__ inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
__host__ __device__ inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
__host__ __device__ inline Dual sqrt(Dual a) {
    const double r = ::sqrt(a.v);
    return Dual(r, r > 0.0 ? a.d / (2.0 * r) : 0.0);
}

// Damping of the normal's derivative: below this fraction of the gradient that an
// equilibrium interface profile has at the same c (4 c (1 - c) / W), grad c is set by the
// rounding noise of a nearly uniform field, and the derivative of grad c / |grad c| there
// (of order 1 / |grad c|) describes no physical sensitivity: the normal's effect on the
// step is bounded by the vanishing prefactor 1 - 4 (c - 1/2)^2, which finite differences
// see, while the exact derivative of the discrete map grows without bound.  Both the
// tangent-linear model and the adjoint scale the normal's derivative by
// min(1, |grad c| / (kNormalDamp 4 c (1 - c) / W)); the forward itself is unchanged.
constexpr double kNormalDamp = 0.1;

__host__ __device__ inline double normal_damping(double mag, double c, double W) {
    const double ref = kNormalDamp * 4.0 * fabs(c * (1.0 - c)) / W;
    return mag >= ref ? 1.0 : mag / ref;
}

// interface_normal (lattice.cuh) on dual numbers: the same values, the damped derivative.
template <int DIM>
__device__ __forceinline__ void interface_normal(const Phys<Dual>& P, Dual c, const Dual* dc, Dual* nrm) {
    const double ss = DIM == 2 ? (dc[0].v * dc[0].v) + (dc[1].v * dc[1].v)
                               : (dc[0].v * dc[0].v) + (dc[1].v * dc[1].v) + (dc[2].v * dc[2].v);
    const double mag = ::sqrt(ss), m = mag + 1e-32;
    double dmag = 0.0;
    if (mag > 0.0) {
        for (int d = 0; d < DIM; ++d) dmag += dc[d].v * dc[d].d;
        dmag /= mag;
    }
    const double sc = normal_damping(mag, c.v, P.W.v);
    for (int d = 0; d < DIM; ++d) {
        const double n = dc[d].v / m;
        nrm[d] = Dual(n, sc * (dc[d].d - n * dmag) / m);
    }
}

}  // namespace clipb
