// Lattice tables and per-node physics of the two-phase Allen-Cahn / weighted-MRT LBM.
//
// Every formula keeps the operation order of the reference (mshadkhah/CLIP) so that the
// FP64 instantiation, compiled without FMA contraction, rounds exactly like the
// reference's own arithmetic:
//   equilibrium            NsAllen.cu:77-94
//   viscous force (VF)     NsAllen.cu:102-132
//   macroscopic f          NsAllen.cu:369-511
//   g collision            NsAllen.cu:545-584
//   f collision            NsAllen.cu:589-763
//   WMRT transforms        WMRT.cuh:54-184
//   stencils               NsAllen.cu:207-236 (mu), 280-322 (grad c), 241-275 (normal)
// Products with a zero lattice component are skipped: x*0 contributes +-0 to a sum and
// x*(+-1) is exact, so the skipped form returns the same values as the reference's dense
// form while the FP32/FP16 instantiations avoid the dead arithmetic.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

namespace clipb {

template <int DIM> struct Lat;

// D2Q9, WMRT.cuh:193-196.
template <> struct Lat<2> {
    static constexpr int Q = 9;
    static constexpr int A = 3;       // directions per wall (wallBCMap::Q)
    static constexpr int kWeight = 2;  // wallBCMap::weight
    __host__ __device__ static constexpr int ex(int q) { return q == 1 || q == 5 || q == 8 ? 1 : (q == 3 || q == 6 || q == 7 ? -1 : 0); }
    __host__ __device__ static constexpr int ey(int q) { return q == 2 || q == 5 || q == 6 ? 1 : (q == 4 || q == 7 || q == 8 ? -1 : 0); }
    __host__ __device__ static constexpr int ez(int) { return 0; }
    __host__ __device__ static constexpr double w(int q) { return q == 0 ? 4.0 / 9.0 : (q < 5 ? 1.0 / 9.0 : 1.0 / 36.0); }
    // FP32 weights (see Lat<3>): 4/9 (1 + 7.5e-8), 1/9 (1 - 6e-8), 1/36 (1 - 6e-8);
    // 3 w: 1/3 (1 + 3e-8), 1/12 (1 - 6e-8)
    __host__ __device__ static constexpr float ws(int q) {
        return q == 0 ? 0x1.c71c74p-2f : (q < 5 ? 0x1.c71c70p-4f : 0x1.c71c70p-6f);
    }
    __host__ __device__ static constexpr float wo(int q) { return q == 0 ? 0.f : (q < 5 ? 0x1.555556p-2f : 0x1.555554p-4f); }
};

// D3Q19, WMRT.cuh:199-204.
template <> struct Lat<3> {
    static constexpr int Q = 19;
    static constexpr int A = 5;
    static constexpr int kWeight = 4;
    __host__ __device__ static constexpr int ex(int q) {
        return (q == 1 || q == 7 || q == 9 || q == 11 || q == 13) ? 1 : ((q == 2 || q == 8 || q == 10 || q == 12 || q == 14) ? -1 : 0);
    }
    __host__ __device__ static constexpr int ey(int q) {
        return (q == 3 || q == 7 || q == 10 || q == 15 || q == 17) ? 1 : ((q == 4 || q == 8 || q == 9 || q == 16 || q == 18) ? -1 : 0);
    }
    __host__ __device__ static constexpr int ez(int q) {
        return (q == 5 || q == 11 || q == 14 || q == 15 || q == 18) ? 1 : ((q == 6 || q == 12 || q == 13 || q == 16 || q == 17) ? -1 : 0);
    }
    __host__ __device__ static constexpr double w(int q) { return q == 0 ? 1.0 / 3.0 : (q < 7 ? 1.0 / 18.0 : 1.0 / 36.0); }
    // FP32 weights of the reduced-precision update, chosen so that the moments it conserves
    // come out exact.  ws (equilibrium and storage shift): sum ws_q = 1 exactly, so that the
    // zeroth moments of the relaxed populations are c and p themselves; with the weights
    // rounded to nearest the sum is 1 + 1.5e-8, which multiplies c and p by that factor at
    // every step (a drift of 1.5e-4 of c in the heavy phase over 10^4 steps).  wo (3 w_q, for
    // the parts odd in e_q): sum wo_q e_qx^2 = 1 exactly, so the first moments are j and
    // the phase-field flux themselves.  ws: 1/3 (1 + 1.2e-7), 1/18 (1 - 6e-8), 1/36 (1 - 6e-8);
    // wo: 1/6 (1 - 6e-8), 1/12 (1 + 3e-8).
    __host__ __device__ static constexpr float ws(int q) {
        return q == 0 ? 0x1.555558p-2f : (q < 7 ? 0x1.c71c70p-5f : 0x1.c71c70p-6f);
    }
    __host__ __device__ static constexpr float wo(int q) { return q == 0 ? 0.f : (q < 7 ? 0x1.555554p-3f : 0x1.555556p-4f); }
};

// The FP32 weight sums, evaluated in FP64 where every term is exact.
static_assert(double(Lat<2>::ws(0)) + 4.0 * double(Lat<2>::ws(1)) + 4.0 * double(Lat<2>::ws(5)) == 1.0, "D2Q9 ws");
static_assert(2.0 * double(Lat<2>::wo(1)) + 4.0 * double(Lat<2>::wo(5)) == 1.0, "D2Q9 wo");
static_assert(double(Lat<3>::ws(0)) + 6.0 * double(Lat<3>::ws(1)) + 12.0 * double(Lat<3>::ws(7)) == 1.0, "D3Q19 ws");
static_assert(2.0 * double(Lat<3>::wo(1)) + 8.0 * double(Lat<3>::wo(7)) == 1.0, "D3Q19 wo");

// Opposite direction (the partner that half-way bounce-back reflects into; the wall maps of
// WMRT.cuh:214-237 pair every incoming direction with its exact opposite).
template <int DIM>
__host__ __device__ constexpr int opposite(int q) {
    if (DIM == 2) {
        constexpr int t[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
        return t[q];
    } else {
        constexpr int t[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
        return t[q];
    }
}

// e_q . v with zero components skipped (see file comment).
// Directions entering the domain across side s (x-, x+, y-, y+, z-, z+), in the order of the
// reference's wallBCMap (include/solver/WMRT.cuh:214-237), and the inverse: the slot of q
// in that list, -1 if q does not enter across s.  Needed where the reference's loop order
// decides which side writes an edge node's population last (kernelNeumann).
template <int DIM>
__host__ __device__ constexpr int wall_dir(int s, int i) {
    if (DIM == 2) {
        constexpr int t[4][3] = {{1, 5, 8}, {3, 7, 6}, {2, 5, 6}, {4, 7, 8}};
        return t[s][i];
    } else {
        constexpr int t[6][5] = {{1, 9, 7, 13, 11}, {2, 10, 8, 14, 12}, {3, 10, 7, 17, 15},
                                 {4, 9, 8, 18, 16}, {5, 14, 11, 18, 15}, {6, 13, 12, 17, 16}};
        return t[s][i];
    }
}
template <int DIM>
__host__ __device__ constexpr int wall_slot(int s, int q) {
    for (int i = 0; i < (DIM == 2 ? 3 : 5); ++i)
        if (wall_dir<DIM>(s, i) == q) return i;
    return -1;
}

template <int DIM, typename T>
__device__ __forceinline__ T edot(int q, T vx, T vy, T vz) {
    using L = Lat<DIM>;
    T s = T(0);
    bool first = true;
    auto acc = [&](int e, T v) {
        if (e == 0) return;
        const T t = e > 0 ? v : -v;
        s = first ? t : s + t;
        first = false;
    };
    acc(L::ex(q), vx);
    acc(L::ey(q), vy);
    if (DIM == 3) acc(L::ez(q), vz);
    return s;
}

// w_q (3 e.u + 4.5 (e.u)^2 - 1.5 u^2)  (NsAllen.cu:77-94)
template <int DIM, typename T>
__device__ __forceinline__ T equilibrium(int q, T ux, T uy, T uz, T U2) {
    const T eU = edot<DIM, T>(q, ux, uy, uz);
    return T(Lat<DIM>::w(q)) * (T(3.0) * eU + T(4.5) * eU * eU - T(1.5) * U2);
}

template <int DIM, typename T>
__device__ __forceinline__ T usq(T ux, T uy, T uz) {
    return DIM == 2 ? ux * ux + uy * uy : ux * ux + uy * uy + uz * uz;
}

// ---------------------------------------------------------------- WMRT (WMRT.cuh:54-184)
template <typename T>
__device__ __forceinline__ void wmrt_forward9(const T* in, T* out) {
    const T in0 = in[0], in1 = in[1], in2 = in[2], in3 = in[3], in4 = in[4], in5 = in[5], in6 = in[6], in7 = in[7], in8 = in[8];
    out[0] = in0 + in1 + in2 + in3 + in4 + in5 + in6 + in7 + in8;
    out[1] = -T(4.0) * in0 - in1 - in2 - in3 - in4 + T(2.0) * in5 + T(2.0) * in6 + T(2.0) * in7 + T(2.0) * in8;
    out[2] = T(4.0) * in0 - T(2.0) * in1 - T(2.0) * in2 - T(2.0) * in3 - T(2.0) * in4 + in5 + in6 + in7 + in8;
    out[3] = in1 - in3 + in5 - in6 - in7 + in8;
    out[4] = -T(2.0) * in1 + T(2.0) * in3 + in5 - in6 - in7 + in8;
    out[5] = in2 - in4 + in5 + in6 - in7 - in8;
    out[6] = -T(2.0) * in2 + T(2.0) * in4 + in5 + in6 - in7 - in8;
    out[7] = in1 - in2 + in3 - in4;
    out[8] = in5 - in6 + in7 - in8;
}

template <typename T>
__device__ __forceinline__ void wmrt_inverse9(const T* in, T* out) {
    const T in0 = in[0], in1 = in[1], in2 = in[2], in3 = in[3], in4 = in[4], in5 = in[5], in6 = in[6], in7 = in[7], in8 = in[8];
    const T d = T(36.0);
    out[0] = (T(4.0) * in0 - T(4.0) * in1 + T(4.0) * in2) / d;
    out[1] = (T(4.0) * in0 - in1 - T(2.0) * in2 + T(6.0) * in3 - T(6.0) * in4 + T(9.0) * in7) / d;
    out[2] = (T(4.0) * in0 - in1 - T(2.0) * in2 + T(6.0) * in5 - T(6.0) * in6 - T(9.0) * in7) / d;
    out[3] = (T(4.0) * in0 - in1 - T(2.0) * in2 - T(6.0) * in3 + T(6.0) * in4 + T(9.0) * in7) / d;
    out[4] = (T(4.0) * in0 - in1 - T(2.0) * in2 - T(6.0) * in5 + T(6.0) * in6 - T(9.0) * in7) / d;
    out[5] = (T(4.0) * in0 + T(2.0) * in1 + in2 + T(6.0) * in3 + T(3.0) * in4 + T(6.0) * in5 + T(3.0) * in6 + T(9.0) * in8) / d;
    out[6] = (T(4.0) * in0 + T(2.0) * in1 + in2 - T(6.0) * in3 - T(3.0) * in4 + T(6.0) * in5 + T(3.0) * in6 - T(9.0) * in8) / d;
    out[7] = (T(4.0) * in0 + T(2.0) * in1 + in2 - T(6.0) * in3 - T(3.0) * in4 - T(6.0) * in5 - T(3.0) * in6 + T(9.0) * in8) / d;
    out[8] = (T(4.0) * in0 + T(2.0) * in1 + in2 + T(6.0) * in3 + T(3.0) * in4 - T(6.0) * in5 - T(3.0) * in6 - T(9.0) * in8) / d;
}

template <typename T>
__device__ __forceinline__ void wmrt_forward19(const T* in, T* out) {
    const T in0 = in[0], in1 = in[1], in2 = in[2], in3 = in[3], in4 = in[4], in5 = in[5], in6 = in[6], in7 = in[7],
            in8 = in[8], in9 = in[9], in10 = in[10], in11 = in[11], in12 = in[12], in13 = in[13], in14 = in[14],
            in15 = in[15], in16 = in[16], in17 = in[17], in18 = in[18];
    out[0] = in0 + in1 + in2 + in3 + in4 + in5 + in6 + in7 + in8 + in9 + in10 + in11 + in12 + in13 + in14 + in15 + in16 + in17 + in18;
    out[1] = in1 - in2 + in7 - in8 + in9 - in10 + in11 - in12 + in13 - in14;
    out[2] = in3 - in4 + in7 - in8 - in9 + in10 + in15 - in16 + in17 - in18;
    out[3] = in5 - in6 + in11 - in12 - in13 + in14 + in15 - in16 - in17 + in18;
    out[4] = in7 + in8 - in9 - in10;
    out[5] = in15 + in16 - in17 - in18;
    out[6] = in11 + in12 - in13 - in14;
    out[7] = T(2.0) * in1 + T(2.0) * in2 - in3 - in4 - in5 - in6 + in7 + in8 + in9 + in10 + in11 + in12 + in13 + in14 -
             T(2.0) * in15 - T(2.0) * in16 - T(2.0) * in17 - T(2.0) * in18;
    out[8] = in3 + in4 - in5 - in6 + in7 + in8 + in9 + in10 - in11 - in12 - in13 - in14;
    out[9] = -in0 + in7 + in8 + in9 + in10 + in11 + in12 + in13 + in14 + in15 + in16 + in17 + in18;
    out[10] = -T(2.0) * in1 + T(2.0) * in2 + in7 - in8 + in9 - in10 + in11 - in12 + in13 - in14;
    out[11] = -T(2.0) * in3 + T(2.0) * in4 + in7 - in8 - in9 + in10 + in15 - in16 + in17 - in18;
    out[12] = -T(2.0) * in5 + T(2.0) * in6 + in11 - in12 - in13 + in14 + in15 - in16 - in17 + in18;
    out[13] = in7 - in8 + in9 - in10 - in11 + in12 - in13 + in14;
    out[14] = -in7 + in8 + in9 - in10 + in15 - in16 + in17 - in18;
    out[15] = in11 - in12 - in13 + in14 - in15 + in16 + in17 - in18;
    out[16] = in0 - T(2.0) * in1 - T(2.0) * in2 - T(2.0) * in3 - T(2.0) * in4 - T(2.0) * in5 - T(2.0) * in6 + in7 + in8 +
              in9 + in10 + in11 + in12 + in13 + in14 + in15 + in16 + in17 + in18;
    out[17] = -T(2.0) * in1 - T(2.0) * in2 + in3 + in4 + in5 + in6 + in7 + in8 + in9 + in10 + in11 + in12 + in13 + in14 -
              T(2.0) * in15 - T(2.0) * in16 - T(2.0) * in17 - T(2.0) * in18;
    out[18] = -in3 - in4 + in5 + in6 + in7 + in8 + in9 + in10 - in11 - in12 - in13 - in14;
}

template <typename T>
__device__ __forceinline__ void wmrt_inverse19(const T* in, T* out) {
    const T in0 = in[0], in1 = in[1], in2 = in[2], in3 = in[3], in4 = in[4], in5 = in[5], in6 = in[6], in7 = in[7],
            in8 = in[8], in9 = in[9], in10 = in[10], in11 = in[11], in12 = in[12], in13 = in[13], in14 = in[14],
            in15 = in[15], in16 = in[16], in17 = in[17], in18 = in[18];
    const T d6 = T(6.0), d36 = T(36.0), d72 = T(72.0), d144 = T(144.0);
    out[0] = (T(2.0) * in0 - T(3.0) * in9 + in16) / d6;
    out[1] = (T(2.0) * in0 + T(6.0) * in1 + T(3.0) * in7 - T(6.0) * in10 - T(2.0) * in16 - T(3.0) * in17) / d36;
    out[2] = (T(2.0) * in0 - T(6.0) * in1 + T(3.0) * in7 + T(6.0) * in10 - T(2.0) * in16 - T(3.0) * in17) / d36;
    out[3] = (T(4.0) * in0 + T(12.0) * in2 - T(3.0) * in7 + T(9.0) * in8 - T(12.0) * in11 - T(4.0) * in16 + T(3.0) * in17 - T(9.0) * in18) / d72;
    out[4] = (T(4.0) * in0 - T(12.0) * in2 - T(3.0) * in7 + T(9.0) * in8 + T(12.0) * in11 - T(4.0) * in16 + T(3.0) * in17 - T(9.0) * in18) / d72;
    out[5] = (T(4.0) * in0 + T(12.0) * in3 - T(3.0) * in7 - T(9.0) * in8 - T(12.0) * in12 - T(4.0) * in16 + T(3.0) * in17 + T(9.0) * in18) / d72;
    out[6] = (T(4.0) * in0 - T(12.0) * in3 - T(3.0) * in7 - T(9.0) * in8 + T(12.0) * in12 - T(4.0) * in16 + T(3.0) * in17 + T(9.0) * in18) / d72;
    out[7] = (T(4.0) * in0 + T(12.0) * in1 + T(12.0) * in2 + T(36.0) * in4 + T(3.0) * in7 + T(9.0) * in8 + T(6.0) * in9 + T(6.0) * in10 + T(6.0) * in11 + T(18.0) * in13 - T(18.0) * in14 + T(2.0) * in16 + T(3.0) * in17 + T(9.0) * in18) / d144;
    out[8] = (T(4.0) * in0 - T(12.0) * in1 - T(12.0) * in2 + T(36.0) * in4 + T(3.0) * in7 + T(9.0) * in8 + T(6.0) * in9 - T(6.0) * in10 - T(6.0) * in11 - T(18.0) * in13 + T(18.0) * in14 + T(2.0) * in16 + T(3.0) * in17 + T(9.0) * in18) / d144;
    out[9] = (T(4.0) * in0 + T(12.0) * in1 - T(12.0) * in2 - T(36.0) * in4 + T(3.0) * in7 + T(9.0) * in8 + T(6.0) * in9 + T(6.0) * in10 - T(6.0) * in11 + T(18.0) * in13 + T(18.0) * in14 + T(2.0) * in16 + T(3.0) * in17 + T(9.0) * in18) / d144;
    out[10] = (T(4.0) * in0 - T(12.0) * in1 + T(12.0) * in2 - T(36.0) * in4 + T(3.0) * in7 + T(9.0) * in8 + T(6.0) * in9 - T(6.0) * in10 + T(6.0) * in11 - T(18.0) * in13 - T(18.0) * in14 + T(2.0) * in16 + T(3.0) * in17 + T(9.0) * in18) / d144;
    out[11] = (T(4.0) * in0 + T(12.0) * in1 + T(12.0) * in3 + T(36.0) * in6 + T(3.0) * in7 - T(9.0) * in8 + T(6.0) * in9 + T(6.0) * in10 + T(6.0) * in12 - T(18.0) * in13 + T(18.0) * in15 + T(2.0) * in16 + T(3.0) * in17 - T(9.0) * in18) / d144;
    out[12] = (T(4.0) * in0 - T(12.0) * in1 - T(12.0) * in3 + T(36.0) * in6 + T(3.0) * in7 - T(9.0) * in8 + T(6.0) * in9 - T(6.0) * in10 - T(6.0) * in12 + T(18.0) * in13 - T(18.0) * in15 + T(2.0) * in16 + T(3.0) * in17 - T(9.0) * in18) / d144;
    out[13] = (T(4.0) * in0 + T(12.0) * in1 - T(12.0) * in3 - T(36.0) * in6 + T(3.0) * in7 - T(9.0) * in8 + T(6.0) * in9 + T(6.0) * in10 - T(6.0) * in12 - T(18.0) * in13 - T(18.0) * in15 + T(2.0) * in16 + T(3.0) * in17 - T(9.0) * in18) / d144;
    out[14] = (T(4.0) * in0 - T(12.0) * in1 + T(12.0) * in3 - T(36.0) * in6 + T(3.0) * in7 - T(9.0) * in8 + T(6.0) * in9 - T(6.0) * in10 + T(6.0) * in12 + T(18.0) * in13 + T(18.0) * in15 + T(2.0) * in16 + T(3.0) * in17 - T(9.0) * in18) / d144;
    out[15] = (T(4.0) * in0 + T(12.0) * in2 + T(12.0) * in3 + T(36.0) * in5 - T(6.0) * in7 + T(6.0) * in9 + T(6.0) * in11 + T(6.0) * in12 + T(18.0) * in14 - T(18.0) * in15 + T(2.0) * in16 - T(6.0) * in17) / d144;
    out[16] = (T(4.0) * in0 - T(12.0) * in2 - T(12.0) * in3 + T(36.0) * in5 - T(6.0) * in7 + T(6.0) * in9 - T(6.0) * in11 - T(6.0) * in12 - T(18.0) * in14 + T(18.0) * in15 + T(2.0) * in16 - T(6.0) * in17) / d144;
    out[17] = (T(4.0) * in0 + T(12.0) * in2 - T(12.0) * in3 - T(36.0) * in5 - T(6.0) * in7 + T(6.0) * in9 + T(6.0) * in11 - T(6.0) * in12 + T(18.0) * in14 + T(18.0) * in15 + T(2.0) * in16 - T(6.0) * in17) / d144;
    out[18] = (T(4.0) * in0 - T(12.0) * in2 + T(12.0) * in3 - T(36.0) * in5 - T(6.0) * in7 + T(6.0) * in9 - T(6.0) * in11 + T(6.0) * in12 - T(18.0) * in14 - T(18.0) * in15 + T(2.0) * in16 - T(6.0) * in17) / d144;
}

// Relax the viscous moments (2D: 7,8; 3D: 4..8) by s, all others at rate 1
// (NsAllen.cu:416-431, 435-454): gneq <- M^-1 S M gneq.
template <int DIM, typename T>
__device__ __forceinline__ void wmrt_relax(T* gneq, T s) {
    T m[Lat<DIM>::Q];
    if (DIM == 2) {
        wmrt_forward9<T>(gneq, m);
        m[7] = m[7] * s;
        m[8] = m[8] * s;
        wmrt_inverse9<T>(m, gneq);
    } else {
        wmrt_forward19<T>(gneq, m);
        m[4] = m[4] * s;
        m[5] = m[5] * s;
        m[6] = m[6] * s;
        m[7] = m[7] * s;
        m[8] = m[8] * s;
        wmrt_inverse19<T>(m, gneq);
    }
}

// ---------------------------------------------------------------- scalar physics

// Parameters of one case, already cast to the arithmetic type T.
template <typename T>
struct Phys {
    T RhoL, RhoH, drho, drho3;  // drho = RhoH - RhoL, drho3 = (RhoH - RhoL) / 3
    T tauL, tauH, dtau;         // dtau = tauH - tauL
    T kappa, beta4;             // kConstant, 4 * betaConstant
    T mobility, W;              // mobility, interfaceWidth
    T wc, one_minus_wc;         // Allen-Cahn rate 1/(1/2 + 3M) and 1 - wc (NsAllen.cu:549)
    T amob3;                    // 3 * mobility
    T g[3];                     // gravity
    int caseType;               // 0 bubble, 1 drop, 2 RTI
};

template <typename T>
__device__ __forceinline__ T relax_tau(const Phys<T>& P, T c) {  // NsAllen.cu:418-425
    if (c < T(0.0)) return P.tauL;
    if (c > T(1.0)) return P.tauH;
    return P.tauL + c * P.dtau;
}

// Gravity body force per case (NsAllen.cu:460-474).  For case 'jet' the reference sets no
// value (its local force array stays uninitialised); here a jet has no body force.
template <typename T>
__device__ __forceinline__ T gravity_force(const Phys<T>& P, T rho, int d) {
    if (P.caseType == 2) return (rho)*P.g[d];
    if (P.caseType == 0) return (rho - P.RhoH) * P.g[d];
    if (P.caseType == 1) return (rho - P.RhoL) * P.g[d];
    return T(0);
}

// Viscous force from the relaxed non-equilibrium moments (NsAllen.cu:102-132).
template <int DIM, typename T>
__device__ __forceinline__ void viscous_force(const Phys<T>& P, const T* gneq, T tau, T dcx, T dcy, T dcz, T* fv) {
    using L = Lat<DIM>;
    T sxx = T(0), sxy = T(0), syy = T(0), szy = T(0), szx = T(0), szz = T(0);
    bool fxx = true, fxy = true, fyy = true, fzy = true, fzx = true, fzz = true;
    auto acc = [](T& s, bool& first, int e, T v) {
        if (e == 0) return;
        const T t = e > 0 ? v : -v;
        s = first ? t : s + t;
        first = false;
    };
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        acc(sxx, fxx, L::ex(i) * L::ex(i), gneq[i]);
        acc(sxy, fxy, L::ex(i) * L::ey(i), gneq[i]);
        acc(syy, fyy, L::ey(i) * L::ey(i), gneq[i]);
        if (DIM == 3) {
            acc(szy, fzy, L::ez(i) * L::ey(i), gneq[i]);
            acc(szx, fzx, L::ez(i) * L::ex(i), gneq[i]);
            acc(szz, fzz, L::ez(i) * L::ez(i), gneq[i]);
        }
    }
    if (DIM == 2) {
        fv[0] = -tau * (sxx * dcx + sxy * dcy) * P.drho;
        fv[1] = -tau * (sxy * dcx + syy * dcy) * P.drho;
    } else {
        fv[0] = -tau * (sxx * dcx + sxy * dcy + szx * dcz) * P.drho;
        fv[1] = -tau * (sxy * dcx + syy * dcy + szy * dcz) * P.drho;
        fv[2] = -tau * (szz * dcz + szx * dcx + szy * dcy) * P.drho;
    }
}

// Total force mu grad c - p (rhoH-rhoL)/3 grad c + F_visc + F_gravity (NsAllen.cu:476-485).
template <int DIM, typename T>
__device__ __forceinline__ void total_force(const Phys<T>& P, const T* fpost, T p, T ux, T uy, T uz, T tau, T s9,
                                            T mu, T rho, const T* dc, T* F) {
    using L = Lat<DIM>;
    T gneq[L::Q];
    const T U2 = usq<DIM, T>(ux, uy, uz);
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        const T geq = p * T(L::w(q)) + equilibrium<DIM, T>(q, ux, uy, uz, U2);
        gneq[q] = fpost[q] - geq;
    }
    wmrt_relax<DIM, T>(gneq, s9);
    T fv[3];
    viscous_force<DIM, T>(P, gneq, tau, dc[0], dc[1], DIM == 3 ? dc[2] : T(0), fv);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        const T Fp = -p * P.drho3 * dc[d];
        F[d] = mu * dc[d] + Fp + fv[d] + gravity_force<T>(P, rho, d);
    }
}

// kernelMacroscopicg + kernelMacroscopicf at one node (NsAllen.cu:369-540).
//   in : fpost (streamed, bounced), c, mu, dc of this step, u (previous step)
//   out: u (this step), p, rho
template <int DIM, typename T>
__device__ __forceinline__ void macroscopic(const Phys<T>& P, const T* fpost, T c, T mu, const T* dc, T* u, T& p_out,
                                            T& rho_out) {
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    const T rho = (P.RhoL + (c * P.drho));  // NsAllen.cu:538
    T p = fpost[0];
#pragma unroll
    for (int q = 1; q < Q; ++q) p = p + fpost[q];
    const T tau = relax_tau<T>(P, c);
    const T s9 = T(1.0) / (tau + T(0.50));
    T F[3];
    total_force<DIM, T>(P, fpost, p, u[0], u[1], DIM == 3 ? u[2] : T(0), tau, s9, mu, rho, dc, F);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        T s = T(0);
        bool first = true;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int e = d == 0 ? L::ex(q) : (d == 1 ? L::ey(q) : L::ez(q));
            if (e == 0) continue;
            const T t = e > 0 ? fpost[q] : -fpost[q];
            s = first ? t : s + t;
            first = false;
        }
        u[d] = s + T(0.50) * F[d] / rho;
    }
    p_out = p;
    rho_out = rho;
}

// Interface normal grad c / (|grad c| + 1e-32) (normal_FD, NsAllen.cu:241-275).  The
// tangent-linear model overloads it for dual numbers (dual.cuh).
template <int DIM, typename T>
__device__ __forceinline__ void interface_normal(const Phys<T>& P, T c, const T* dc, T* nrm) {
    (void)P;
    (void)c;
    const T mag = (DIM == 2 ? sqrt((dc[0] * dc[0]) + (dc[1] * dc[1]))
                            : sqrt((dc[0] * dc[0]) + (dc[1] * dc[1]) + (dc[2] * dc[2]))) + T(1e-32);
#pragma unroll
    for (int d = 0; d < DIM; ++d) nrm[d] = dc[d] / mag;
}

// normal_FD + kernelCollisionMRTg at one node (NsAllen.cu:241-275, 545-584): the
// single-rate Allen-Cahn relaxation with this step's c, grad c and u.
template <int DIM, typename T>
__device__ __forceinline__ void collide_g(const Phys<T>& P, const T* gpost, T c, const T* dc, const T* u, T* gout) {
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    const T ux = u[0], uy = u[1], uz = DIM == 3 ? u[2] : T(0);
    const T U2 = usq<DIM, T>(ux, uy, uz);
    T nrm[3];
    interface_normal<DIM>(P, c, dc, nrm);
    const T cm = c - T(0.50);
    const T pref = ((P.amob3 * (T(1.0) - T(4.0) * (cm * cm))) / P.W);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const T ga_wa = equilibrium<DIM, T>(q, ux, uy, uz, U2);
        const T eF = pref * edot<DIM, T>(q, nrm[0], nrm[1], DIM == 3 ? nrm[2] : T(0));
        const T hlp = T(L::w(q)) * eF;
        const T heq = c * (ga_wa + T(L::w(q))) + hlp;
        gout[q] = gpost[q] * P.one_minus_wc + heq * P.wc;
    }
}

// kernelCollisionMRTf at one node (NsAllen.cu:589-763): force-corrected WMRT relaxation
// with this step's p, c, mu, grad c, rho and u.
template <int DIM, typename T>
__device__ __forceinline__ void collide_f(const Phys<T>& P, const T* fpost, T c, T mu, const T* dc, T rho, T p,
                                          const T* u, T* fout) {
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    const T ux = u[0], uy = u[1], uz = DIM == 3 ? u[2] : T(0);
    const T U2 = usq<DIM, T>(ux, uy, uz);
    const T tau = relax_tau<T>(P, c);
    const T s9 = T(1.0) / (tau + T(0.50));
    {
        T F[3];
        total_force<DIM, T>(P, fpost, p, ux, uy, uz, tau, s9, mu, rho, dc, F);
        T gneq[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const T eF = edot<DIM, T>(q, F[0], F[1], DIM == 3 ? F[2] : T(0));
            const T hlp = T(3.0 * L::w(q)) * eF / rho;
            const T feq = p * T(L::w(q)) + equilibrium<DIM, T>(q, ux, uy, uz, U2) - T(0.50) * hlp;
            gneq[q] = fpost[q] - feq;
        }
        wmrt_relax<DIM, T>(gneq, s9);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const T eF = edot<DIM, T>(q, F[0], F[1], DIM == 3 ? F[2] : T(0));
            const T hlp = T(3.0 * L::w(q)) * eF / rho;
            fout[q] = fpost[q] - gneq[q] + hlp;
        }
    }
}

// kernelCollisionMRTf (NsAllen.cu:589-763) on the initial populations f_q = p w_q at u = 0
// (KernelInitializeDistributions, NsAllen.cu:137-202): their non-equilibrium part is zero, so
// the viscous force vanishes and F = (mu - p drho/3) grad c + gravity; the part the collision
// relaxes is then the force term alone, odd in e_q, which the weighted-MRT relaxation
// returns at rate 1, leaving f_q = p w_q + (3/2) w_q (e_q . F) / rho.  Equal to collide_f on
// those populations up to FP64 rounding, without its two pairs of 19x19 transforms; the
// initial state of the FP32/FP16 paths, which store the result rounded, uses it.
template <int DIM, typename T>
__device__ __forceinline__ void first_collide_f(const Phys<T>& P, T mu, const T* dc, T rho, T p, T* fout) {
    using L = Lat<DIM>;
    T F[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
        const T Fp = -p * P.drho3 * dc[d];
        F[d] = mu * dc[d] + Fp + gravity_force<T>(P, rho, d);
    }
    const T h = T(1.5) / rho;
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
        const T eF = edot<DIM, T>(q, F[0], F[1], DIM == 3 ? F[2] : T(0));
        fout[q] = p * T(L::w(q)) + T(L::w(q)) * (eF * h);
    }
}


// ---------------------------------------------------------------- FP32 update
// The FP32/FP16 storage paths keep g as deviations from w_q c (see Prec in kernels.cuh) and
// compute in FP32 without losing the digits that FP64 would keep: every quantity that is
// rounded is small (a deviation, a difference of neighbouring c values, a population of
// the pressure-based f), never a sum that cancels.

// Unit normal grad c / (|grad c| + 1e-32) (NsAllen.cu:241-275) with the gradient scaled by
// its largest component first, so that FP32 squares neither underflow nor overflow.
template <int DIM>
__device__ __forceinline__ void unit_normal(const float* dc, float* n) {
    const float m = fmaxf(fmaxf(fabsf(dc[0]), fabsf(dc[1])), DIM == 3 ? fabsf(dc[2]) : 0.f);
    const float im = 1.f / fmaxf(m, 1e-30f);
    const float sx = dc[0] * im, sy = dc[1] * im, sz = DIM == 3 ? dc[2] * im : 0.f;
    const float r = 1.f / (sqrtf(fmaf(sz, sz, fmaf(sy, sy, sx * sx))) + 1e-32f * im);
    n[0] = sx * r;
    n[1] = sy * r;
    n[2] = sz * r;
}

// Macroscopic update and both collisions of one node (kernelMacroscopicf + normal_FD +
// kernelCollisionMRTg + kernelCollisionMRTf, NsAllen.cu:369-763), FP32, for the shifted
// storage of the FP32/FP16 paths, in moment form.
// The weighted-MRT relaxation only rescales the five (3D) / two (2D) traceless stress
// moments by s = 1/(tau + 1/2); every other moment of gneq relaxes at rate 1.  Hence
//   * the second moments of the relaxed gneq are  tr(S)/D I + s dev(S), with S the second
//     moments of gneq = Pi - p/3 I - u u^T (Pi = sum e e f_post; the equilibrium's second
//     moments are p/3 I + u u^T on D2Q9/D3Q19), which gives the viscous force without the
//     19x19 transforms;
//   * the post-collision populations are  f_q = p w_q + feq_q(u) + hlp_q / 2
//     - (s - 1) w_q Phi_q(dev S), Phi_q being the rank-5 (rank-2) image of the relaxed
//     moments (the columns of the inverse transform for moments 4..8, resp. 7..8, are
//     w_q (9 e_a e_b, 0.75 (2e_x^2 - e_y^2 - e_z^2), 2.25 (e_y^2 - e_z^2)) in 3D and
//     w_q (2.25 (e_x^2 - e_y^2), 9 e_x e_y) in 2D).
// The result equals the reference's operator up to rounding; the FP64 path keeps the
// literal transforms (macroscopic / collide_f) for bit-exact parity.
// The update is arranged per pair (q, opposite q): the pair's sum and difference give the
// moments, and each output splits into a part even in e_q and a part odd in e_q.
//   f       : streamed f (p, j and Pi moments)
//   d(q)    : streamed g minus w_q c_old (c_old: this node's stored c of the previous step)
//   delta   : sum d in the order d_0 + d_1 + ... (the phase-field sum of the node's c)
//   c       : this step's c (= c_old + delta, rounded as stored);  mu, dc: its stencils
// The conserved part of the update uses delta itself, not c - c_old: the rounding of the
// stored c cancels between writer and reader (both use the same stored value), so the
// transported g keeps the sum of the deviations to FP32 accuracy of that small number.
//   u       : previous velocity in, this step's velocity out
//   cdest(q): stored c of the node each g_q is written for (dest_shift)
//   out     : receives (q, post-collision f_q, post-collision g_q minus w_q cdest_q)
// With gpost = d + w c_old and heq = c (ga + w) + hlp the stored value is
//   go_q = (1 - wc) d_q + wc (c ga_q + hlp_q) + w_q ((c_old - cdest_q) + wc delta).
// The weights are Lat::ws (even parts, storage shift) and Lat::wo = 3 w (odd parts), whose
// sums are exact in FP32, so that the relaxation leaves c, p, j and the phase-field flux
// unscaled.  Each f output is formed as wo_q (e_q.u) + (w_q (p + even terms) +- wo_q
// (e_q.F) / (2 rho)): the velocity term, the largest, enters through the last fused
// multiply-add, so f is rounded once at its own magnitude (twice for a diagonal q, whose
// e_q.u is a rounded sum); forming the odd part first and adding it rounds there four
// times, and over 10^4 steps of a slowly moving interface those roundings repeat and
// accumulate into the momentum.
// d(q) and cdest(q) are read only where the outputs of pair (q, opposite q) are formed, and
// every output goes to out() as soon as it is known, so that neither the 19 deviations nor
// the 19 shifts stay in registers through the moment and force computation.  Every fused
// multiply-add is written out (fmaf) and the FP32 units are compiled without contraction, so
// each launch shape rounds the same way; the three quotients are the units' fast division
// (-prec-div=false), one fixed instruction sequence wherever the update is inlined.
template <int DIM, class Dq, class Cq, class Out>
__device__ __forceinline__ void lean_update(const Phys<float>& P, const float* f, Dq d, float delta, float c_old,
                                            float c, float mu, const float* dc, float* u, Cq cdest, float& p_out,
                                            Out out) {
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    float p = f[0], j[3] = {0.f, 0.f, 0.f};
    float Pi[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // xx yy zz xy xz yz
#pragma unroll
    for (int q = 1; q < Q; ++q) {
        const int o = opposite<DIM>(q);
        if (o < q) continue;
        const float s = f[q] + f[o], a = f[q] - f[o];
        const int ex = L::ex(q), ey = L::ey(q), ez = L::ez(q);
        p += s;
        if (ex) j[0] += ex > 0 ? a : -a;
        if (ey) j[1] += ey > 0 ? a : -a;
        if (DIM == 3 && ez) j[2] += ez > 0 ? a : -a;
        if (ex) Pi[0] += s;
        if (ey) Pi[1] += s;
        if (DIM == 3 && ez) Pi[2] += s;
        if (ex * ey) Pi[3] += ex * ey > 0 ? s : -s;
        if (DIM == 3 && ex * ez) Pi[4] += ex * ez > 0 ? s : -s;
        if (DIM == 3 && ey * ez) Pi[5] += ey * ez > 0 ? s : -s;
    }
    const float rho = fmaf(c, P.drho, P.RhoL);
    // relaxation time, clamped outside [0, 1] (NsAllen.cu:418-425)
    const float tau = c < 0.f ? P.tauL : (c > 1.f ? P.tauH : fmaf(c, P.dtau, P.tauL));
    const float s9 = 1.f / (tau + 0.5f);
    const float p3 = p * (1.f / 3.f);
    const float kvis = -tau * P.drho;
    const float fcap = fmaf(-p, P.drho3, mu);
    // 1 - c from the node's stored c of the last step and the sum of its pulled deviations:
    // 1 - c_old is exact for c_old in [1/2, 2], so 1 - c keeps its relative precision next to
    // c = 1, where 1 - (stored c) would keep a few bits
    const float omc = (1.f - c_old) - delta;
    // body force (NsAllen.cu:460-474) with rho - RhoH = -(1 - c) drho and rho - RhoL = c drho:
    // the same values, without the cancellation of rho - RhoH against the rounded rho
    const float gf = P.caseType == 2 ? rho : (P.caseType == 0 ? -omc * P.drho : (P.caseType == 1 ? c * P.drho : 0.f));
    float grav[3];
#pragma unroll
    for (int dd = 0; dd < DIM; ++dd) grav[dd] = gf * P.g[dd];
    float dev[6], F[3];
    // relaxed second moments of gneq -> total force (NsAllen.cu:102-132, 476-485)
    auto force = [&](const float* uu) {
        const float sxx = fmaf(-uu[0], uu[0], Pi[0] - p3);
        const float syy = fmaf(-uu[1], uu[1], Pi[1] - p3);
        const float szz = DIM == 3 ? fmaf(-uu[2], uu[2], Pi[2] - p3) : 0.f;
        const float trd = DIM == 3 ? (sxx + syy + szz) * (1.f / 3.f) : (sxx + syy) * 0.5f;
        dev[0] = sxx - trd;
        dev[1] = syy - trd;
        dev[2] = DIM == 3 ? szz - trd : 0.f;
        dev[3] = fmaf(-uu[0], uu[1], Pi[3]);
        dev[4] = DIM == 3 ? fmaf(-uu[0], uu[2], Pi[4]) : 0.f;
        dev[5] = DIM == 3 ? fmaf(-uu[1], uu[2], Pi[5]) : 0.f;
        const float rxx = fmaf(s9, dev[0], trd), ryy = fmaf(s9, dev[1], trd), rzz = fmaf(s9, dev[2], trd);
        const float rxy = s9 * dev[3], rxz = s9 * dev[4], ryz = s9 * dev[5];
        float fv[3];
        if (DIM == 3) {
            fv[0] = kvis * fmaf(rxz, dc[2], fmaf(rxy, dc[1], rxx * dc[0]));
            fv[1] = kvis * fmaf(ryz, dc[2], fmaf(ryy, dc[1], rxy * dc[0]));
            fv[2] = kvis * fmaf(rzz, dc[2], fmaf(ryz, dc[1], rxz * dc[0]));
        } else {
            fv[0] = kvis * fmaf(rxy, dc[1], rxx * dc[0]);
            fv[1] = kvis * fmaf(ryy, dc[1], rxy * dc[0]);
        }
#pragma unroll
        for (int dd = 0; dd < DIM; ++dd) F[dd] = fmaf(fcap, dc[dd], fv[dd] + grav[dd]);
    };
    force(u);  // previous velocity (kernelMacroscopicf)
    const float half_inv_rho = 0.5f / rho;
#pragma unroll
    for (int dd = 0; dd < DIM; ++dd) u[dd] = fmaf(F[dd], half_inv_rho, j[dd]);
    force(u);  // this step's velocity (kernelCollisionMRTf)
    const float U2 = DIM == 3 ? fmaf(u[2], u[2], fmaf(u[1], u[1], u[0] * u[0])) : fmaf(u[1], u[1], u[0] * u[0]);
    const float sm1 = s9 - 1.f;
    float axy, axz, ayz, a7, a8;
    if (DIM == 3) {
        axy = 9.f * dev[3];
        axz = 9.f * dev[4];
        ayz = 9.f * dev[5];
        a7 = 0.75f * ((2.f * dev[0] - dev[1]) - dev[2]);
        a8 = 2.25f * (dev[1] - dev[2]);
    } else {
        axy = 9.f * dev[3];
        axz = ayz = 0.f;
        a7 = 2.25f * (dev[0] - dev[1]);
        a8 = 0.f;
    }
    float nrm[3];
    {
        const float dl[3] = {dc[0], dc[1], DIM == 3 ? dc[2] : 0.f};
        unit_normal<DIM>(dl, nrm);
    }
    // 1 - 4 (c - 1/2)^2 as 4 c (1 - c), with 1 - c as above: the prefactor keeps its
    // relative precision in the bulk phases, where the form with (c - 1/2)^2 cancels.  The
    // odd parts carry wo = 3 w (Lat::wo), so the flux terms enter over 3: wc M 4 c (1 - c) / W
    // along the normal and wc c along the velocity.
    const float wc = P.wc, omw = P.one_minus_wc;
    const float wpref = wc * ((1.f / P.W) * (P.mobility * (4.f * (c * omc))));
    const float t = wc * delta;
    const float wcc = wc * c;
    const float eq0 = -1.5f * U2;
    {
        const float w = L::ws(0);
        out(0, fmaf(w, p, w * eq0), fmaf(omw, d(0), w * (fmaf(wcc, eq0, t) + (c_old - cdest(0)))));
    }
#pragma unroll
    for (int q = 1; q < Q; ++q) {
        const int o = opposite<DIM>(q);
        if (o < q) continue;
        const int ex = L::ex(q), ey = L::ey(q), ez = L::ez(q);
        const float w = L::ws(q), w3 = L::wo(q);
        const float eU = edot<DIM, float>(q, u[0], u[1], DIM == 3 ? u[2] : 0.f);
        const float eF = edot<DIM, float>(q, F[0], F[1], DIM == 3 ? F[2] : 0.f);
        const float en = edot<DIM, float>(q, nrm[0], nrm[1], nrm[2]);
        float phi = 0.f;
        if (ex * ey) phi += ex * ey > 0 ? axy : -axy;
        if (DIM == 3) {
            if (ex * ez) phi += ex * ez > 0 ? axz : -axz;
            if (ey * ez) phi += ey * ez > 0 ? ayz : -ayz;
            const int k7 = 2 * ex * ex - ey * ey - ez * ez, k8 = ey * ey - ez * ez;
            if (k7) phi = fmaf(float(k7), a7, phi);
            if (k8) phi = fmaf(float(k8), a8, phi);
        } else {
            const int k7 = ex * ex - ey * ey;
            if (k7) phi = fmaf(float(k7), a7, phi);
        }
        const float symg = fmaf(4.5f * eU, eU, eq0);        // even part of ga / w
        const float pe = p + fmaf(-sm1, phi, symg);         // even part of f / w
        const float fF = w3 * (half_inv_rho * eF);          // force part of the odd f
        const float ge = fmaf(wcc, symg, t);                // even part of g / w
        const float ga = w3 * fmaf(wpref, en, wcc * eU);    // odd part of g
        out(q, fmaf(w3, eU, fmaf(w, pe, fF)), fmaf(omw, d(q), fmaf(w, ge + (c_old - cdest(q)), ga)));
        out(o, fmaf(-w3, eU, fmaf(w, pe, -fF)), fmaf(omw, d(o), fmaf(w, ge + (c_old - cdest(o)), -ga)));
    }
    p_out = p;
}

// Error-free sum: hi + lo == a + b exactly (Knuth's TwoSum, round-to-nearest).
__device__ __forceinline__ float2 two_sum(float a, float b) {
    const float s = __fadd_rn(a, b);
    const float bb = __fadd_rn(s, -a);
    const float e = __fadd_rn(__fadd_rn(a, -__fadd_rn(s, -bb)), __fadd_rn(b, -bb));
    return make_float2(s, e);
}

// Paired FP32 arithmetic of sm_100 (FADD2 / FMUL2 / FFMA2: two lanes per instruction,
// each rounded as its scalar form).  a - b is b * -1 + a in one rounding.
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
__device__ __forceinline__ float2 fma2(float2 a, float s, float2 c) { return __ffma2_rn(a, make_float2(s, s), c); }

// Laplacian and isotropic gradient of `stencil` below for FP32, summed over differences
// (to the centre node for the Laplacian, across the node for the gradient), so that no sum
// of O(1) values cancels; both lanes of a float2 at once (the stored c and its remainder).
template <int DIM, class Cfun>
__device__ __forceinline__ void lap_grad_diff2(Cfun C, float2& D2C, float2* dc) {
    const float2 c0 = C(0, 0, 0);
    auto D = [&](int dx, int dy, int dz) { return sub2(C(dx, dy, dz), c0); };
    auto Gx = [&](int j, int k) { return sub2(C(1, j, k), C(-1, j, k)); };
    auto Gy = [&](int i, int k) { return sub2(C(i, 1, k), C(i, -1, k)); };
    auto Gz = [&](int i, int j) { return sub2(C(i, j, 1), C(i, j, -1)); };
    if (DIM == 2) {
        const float2 diag = add2(add2(D(-1, -1, 0), D(1, -1, 0)), add2(D(-1, 1, 0), D(1, 1, 0)));
        const float2 axis = add2(add2(D(0, -1, 0), D(-1, 0, 0)), add2(D(1, 0, 0), D(0, 1, 0)));
        D2C = mul2(fma2(axis, 4.f, diag), 1.f / 6.f);
        dc[0] = fma2(add2(Gx(-1, 0), Gx(1, 0)), 1.f / 12.f, mul2(Gx(0, 0), 1.f / 3.f));
        dc[1] = fma2(add2(Gy(-1, 0), Gy(1, 0)), 1.f / 12.f, mul2(Gy(0, 0), 1.f / 3.f));
    } else {
        const float2 s6 = add2(add2(add2(D(1, 0, 0), D(-1, 0, 0)), add2(D(0, 1, 0), D(0, -1, 0))),
                               add2(D(0, 0, 1), D(0, 0, -1)));
        const float2 s12 = add2(add2(add2(add2(D(1, 1, 0), D(-1, -1, 0)), add2(D(-1, 1, 0), D(1, -1, 0))),
                                     add2(add2(D(1, 0, 1), D(-1, 0, -1)), add2(D(1, 0, -1), D(-1, 0, 1)))),
                                add2(add2(D(0, 1, 1), D(0, -1, -1)), add2(D(0, 1, -1), D(0, -1, 1))));
        const float2 s8 = add2(add2(add2(D(1, 1, 1), D(-1, -1, -1)), add2(D(1, 1, -1), D(-1, -1, 1))),
                               add2(add2(D(1, -1, 1), D(-1, 1, -1)), add2(D(-1, 1, 1), D(1, -1, -1))));
        D2C = mul2(fma2(s6, 20.f, fma2(s12, 6.f, s8)), 1.f / 48.f);
        const float a = 4.f / 9.f, b = 1.f / 9.f, e = 1.f / 36.f;
        dc[0] = mul2(fma2(Gx(0, 0), a,
                          fma2(add2(add2(Gx(0, 1), Gx(0, -1)), add2(Gx(1, 0), Gx(-1, 0))), b,
                               mul2(add2(add2(Gx(1, 1), Gx(-1, 1)), add2(Gx(1, -1), Gx(-1, -1))), e))),
                     0.5f);
        dc[1] = mul2(fma2(Gy(0, 0), a,
                          fma2(add2(add2(Gy(1, 0), Gy(-1, 0)), add2(Gy(0, 1), Gy(0, -1))), b,
                               mul2(add2(add2(Gy(1, 1), Gy(-1, 1)), add2(Gy(1, -1), Gy(-1, -1))), e))),
                     0.5f);
        dc[2] = mul2(fma2(Gz(0, 0), a,
                          fma2(add2(add2(Gz(1, 0), Gz(-1, 0)), add2(Gz(0, 1), Gz(0, -1))), b,
                               mul2(add2(add2(Gz(1, 1), Gz(1, -1)), add2(Gz(-1, 1), Gz(-1, -1))), e))),
                     0.5f);
    }
}

// mu and grad c of `stencil` below in FP32 from an unevaluated sum c = hi + lo per node:
// hi is the stored c, lo the part of this step's c that FP32 storage rounds away.  The
// stencils are linear, so they run on hi and on lo, as the two lanes of paired FP32
// instructions; mu's polynomial takes lo through its derivative.
template <int DIM, class Cfun>
__device__ __forceinline__ void stencil_hilo(const Phys<float>& P, Cfun C, float& mu, float* dc) {
    float2 l2, d2[3];
    lap_grad_diff2<DIM>(C, l2, d2);
#pragma unroll
    for (int d = 0; d < DIM; ++d) dc[d] = d2[d].x + d2[d].y;
    const float2 c0 = C(0, 0, 0);
    const float h = c0.x;
    const float poly = h * (h - 1.f) * (h - 0.5f), dpoly = fmaf(3.f * h - 3.f, h, 0.5f);
    mu = fmaf(P.beta4, fmaf(dpoly, c0.y, poly), -P.kappa * (l2.x + l2.y));
}

// Chemical potential mu = 4 beta c (c-1)(c-1/2) - kappa lap(c) and the isotropic
// gradient of c from the 3^DIM neighbourhood `C(dx, dy, dz)` (NsAllen.cu:207-236, 280-322).
template <int DIM, typename T, class Cfun>
__device__ __forceinline__ void stencil(const Phys<T>& P, Cfun C, T& mu, T* dc) {
    const T c0 = C(0, 0, 0);
    T D2C;
    if (DIM == 2) {
        D2C = (C(-1, -1, 0) + C(1, -1, 0) + C(-1, 1, 0) + C(1, 1, 0) +
               T(4.0) * (C(0, -1, 0) + C(-1, 0, 0) + C(1, 0, 0) + C(0, 1, 0)) - T(20) * c0) / T(6.0);
        dc[0] = (C(1, 0, 0) - C(-1, 0, 0)) / T(3.0) + (C(1, -1, 0) + C(1, 1, 0) - C(-1, -1, 0) - C(-1, 1, 0)) / T(12.0);
        dc[1] = (C(0, 1, 0) - C(0, -1, 0)) / T(3.0) + (C(-1, 1, 0) + C(1, 1, 0) - C(-1, -1, 0) - C(1, -1, 0)) / T(12.0);
    } else {
        D2C = (T(20.0) * (C(1, 0, 0) + C(-1, 0, 0) + C(0, 1, 0) + C(0, -1, 0) + C(0, 0, 1) + C(0, 0, -1)) +
               T(6.0) * (C(1, 1, 0) + C(0, 1, -1) + C(-1, 1, 0) + C(0, 1, 1) + C(1, 0, 1) + C(1, 0, -1) + C(-1, 0, -1) +
                         C(-1, 0, 1) + C(0, -1, 1) + C(1, -1, 0) + C(0, -1, -1) + C(-1, -1, 0)) +
               (C(1, 1, 1) + C(1, 1, -1) + C(-1, 1, -1) + C(-1, 1, 1) + C(1, -1, 1) + C(1, -1, -1) + C(-1, -1, -1) +
                C(-1, -1, 1)) -
               T(200.0) * c0) /
              T(48.0);
        const T a = T(4.0 / 9.0), b = T(1.0 / 9.0), e = T(1.0 / 36.0);
        dc[0] = (T(0.50)) * (a * (C(1, 0, 0) - C(-1, 0, 0)) +
                             b * ((C(1, 0, 1) + C(1, 0, -1) + C(1, 1, 0) + C(1, -1, 0)) - (C(-1, 0, 1) + C(-1, 0, -1) + C(-1, 1, 0) + C(-1, -1, 0))) +
                             e * ((C(1, 1, 1) + C(1, -1, 1) + C(1, 1, -1) + C(1, -1, -1)) - (C(-1, 1, 1) + C(-1, -1, 1) + C(-1, 1, -1) + C(-1, -1, -1))));
        dc[1] = (T(0.50)) * (a * (C(0, 1, 0) - C(0, -1, 0)) +
                             b * ((C(1, 1, 0) + C(-1, 1, 0) + C(0, 1, 1) + C(0, 1, -1)) - (C(0, -1, 1) + C(0, -1, -1) + C(1, -1, 0) + C(-1, -1, 0))) +
                             e * ((C(1, 1, 1) + C(-1, 1, 1) + C(1, 1, -1) + C(-1, 1, -1)) - (C(1, -1, 1) + C(-1, -1, 1) + C(1, -1, -1) + C(-1, -1, -1))));
        dc[2] = (T(0.50)) * (a * (C(0, 0, 1) - C(0, 0, -1)) +
                             b * ((C(1, 0, 1) + C(-1, 0, 1) + C(0, 1, 1) + C(0, -1, 1)) - (C(1, 0, -1) + C(-1, 0, -1) + C(0, 1, -1) + C(0, -1, -1))) +
                             e * ((C(1, 1, 1) + C(1, -1, 1) + C(-1, 1, 1) + C(-1, -1, 1)) - (C(1, 1, -1) + C(-1, 1, -1) + C(1, -1, -1) + C(-1, -1, -1))));
    }
    mu = P.beta4 * c0 * (c0 - T(1.0)) * (c0 - T(0.50)) - P.kappa * D2C;
}

}  // namespace clipb
