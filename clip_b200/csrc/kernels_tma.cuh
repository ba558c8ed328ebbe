// Staged 3D step: the g and f tiles of coming planes are brought into shared memory by
// bulk tensor copies (TMA) while the CTA computes the current plane.
//
// CTA = 32 x TY tile of an (x,y) plane marching in z over a segment of planes (the work
// split of step3d_body).  Iteration cz (z0 - 1 <= cz <= z1):
//   wait g(cz) -> phase field of plane cz for the tile and its halo (ring slot cz % 4)
//   barrier    -> thread 0 issues g(cz + 2) into the slot just read and f(cz)
//   wait f(cz - 1) -> update of plane cz - 1, stores to global memory
// A g slot holds, per direction q, the (TX+2) x (TY+2) box of source nodes of the tile and
// its halo, shifted by -e_q, plus the box of the readers' own stored c; an f slot the
// TX x TY box.  A box starts at an x element rounded down to 16 bytes, so the lattice shift
// -e_x becomes a column offset in shared memory.  For nodes next to the domain boundary
// the directions that cross it are reread through the boundary-aware path (fix_g, fix_f);
// ghost nodes map c as ghost_c does.  Every per-node code path appears once in the kernel
// (one box loop, one update), which keeps the kernel's code small.
//
// Bounded waits: every wait gives up after `limit` cycles.  The block agrees on failure at
// the next barrier (__syncthreads_and), issues no further copy, waits (bounded by
// kWaitCycles) for every copy it has in flight, so that none lands in shared memory after
// the block has exited, records the device flag and returns.  `inject` > 0 is the test
// hook of that path: the first g load expects `inject` bytes more than its copies bring,
// so its phase cannot complete and the first wait runs out; thread 0 completes those bytes
// itself before the block drains.
#pragma once

#include "kernels.cuh"
#include "tma.cuh"

namespace clipb {

struct StageMaps {
    CUtensorMap f, g, c;  // input buffers of this step
};

// Host-side tensor maps of one solver: [variant (TY = 8, 4)][input parity].
struct StageHost {
    StageMaps maps[2][2];
};

template <class PR, int TY, bool kStageF = true>
struct StageShape {
    static constexpr int TX = 32;
    static constexpr int Q = 19;
    static constexpr int EB = sizeof(typename PR::Sf);  // population element bytes
    static constexpr int XA = 16 / EB;                  // x alignment in elements
    // populations: element of node x in a row is 31 + x; a tile starting at x0 = 1 + 32 bx
    // needs elements [32 bx + 30, 32 bx + 65]
    static constexpr int XOFF = 30 - 30 % XA;           // box start - 32 bx
    static constexpr int BW = ((TX + 34 - XOFF) + XA - 1) / XA * XA;
    static constexpr int XOFFC = 28, BWC = 40;          // c (4-byte elements)
    static constexpr int HY = TY + 2;
    static constexpr int GBOX = (BW * HY * EB + 127) / 128 * 128;  // bytes per direction
    static constexpr int FBOX = (BW * TY * EB + 127) / 128 * 128;
    static constexpr int CBOX = (BWC * HY * 4 + 127) / 128 * 128;
    static constexpr int GSLOT = Q * GBOX + CBOX;
    static constexpr int FSLOT = Q * FBOX;
    static constexpr int BARS = 128;                    // 4 mbarriers, padded
    static constexpr int SMEM = BARS + 2 * GSLOT + (kStageF ? 2 * FSLOT : 0);
    static constexpr uint32_t GBYTES = Q * BW * HY * EB + BWC * HY * 4;  // bytes landing per g load
    static constexpr uint32_t FBYTES = Q * BW * TY * EB;
};

// kStageF: f of the updated plane comes by bulk copies too (2 more slots); otherwise the
// update pulls it from global memory (pull_f), which leaves room for kMinBlocks resident
// blocks per SM.
template <class PR, int TY, bool kStageF = true, int kMinBlocks = 1>
__global__ void __launch_bounds__(32 * TY, kMinBlocks) step3d_staged_kernel(StepArgs<PR> a, int seg,
                                                                 const __grid_constant__ StageMaps maps, int* err,
                                                                 long long limit, unsigned inject) {
    using SH = StageShape<PR, TY, kStageF>;
    using TP = typename PR::TP;
    using T = typename PR::T;
    using A = typename PR::A;
    using R = typename PR::Ring;
    using Sg = typename PR::Sg;
    using Sf = typename PR::Sf;
    using L = Lat<3>;
    constexpr int Q = 19, TX = 32, HX = TX + 2, NT = TX * TY, NBOX = HX * (TY + 2);
    __shared__ R ring[4][NBOX];
    extern __shared__ __align__(128) unsigned char dsm_raw[];
    // bulk tensor copies need 128-byte aligned shared destinations (launch adds 128 bytes)
    unsigned char* dsm = dsm_raw + ((128u - (smem_addr(dsm_raw) & 127u)) & 127u);

    const Geom& g = a.g;
    const Phys<T>& PT = a.pt;
    const Phys<TP>& PP = a.pp;
    const Codec<PR> cd(a.pop_scale);
    const int bx = (int)blockIdx.x, by = (int)blockIdx.y;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int x0 = 1 + bx * TX, y0 = 1 + by * TY;
    const int x = x0 + tx, y = y0 + ty;
    const int z0 = 1 + (int)blockIdx.z * seg;
    const int z1 = min(z0 + seg, g.n[2] + 1);
    const bool active = x <= g.n[0] && y <= g.n[1];
    const int xs = 32 * bx + SH::XOFF, xsc = 32 * bx + SH::XOFFC;

    uint64_t* bars = reinterpret_cast<uint64_t*>(dsm);  // 0,1: g slots; 2,3: f slots
    unsigned char* gbase = dsm + SH::BARS;
    unsigned char* fbase = gbase + 2 * SH::GSLOT;
    auto gbox = [&](int s, int q) { return reinterpret_cast<const Sg*>(gbase + s * SH::GSLOT + q * SH::GBOX); };
    auto cbox = [&](int s) { return reinterpret_cast<const A*>(gbase + s * SH::GSLOT + Q * SH::GBOX); };
    auto fbox = [&](int s, int q) { return reinterpret_cast<const Sf*>(fbase + s * SH::FSLOT + q * SH::FBOX); };

    if (tid == 0) {
        for (int i = 0; i < 4; ++i) mbar_init(&bars[i], 1);
        mbar_fence_init();
    }
    __syncthreads();

    auto issue_g = [&](int cz, unsigned extra) {  // thread 0
        const int s = cz & 1;
        uint64_t* b = &bars[s];
        mbar_arrive_expect_tx(b, SH::GBYTES + extra);
#pragma unroll
        for (int q = 0; q < Q; ++q)
            tma_load_4d(gbase + s * SH::GSLOT + q * SH::GBOX, &maps.g, xs, y0 - 1 - L::ey(q), cz - L::ez(q), q, b);
        tma_load_3d(gbase + s * SH::GSLOT + Q * SH::GBOX, &maps.c, xsc, y0 - 1, cz, b);
    };
    auto issue_f = [&](int z) {  // thread 0
        const int s = z & 1;
        uint64_t* b = &bars[2 + s];
        mbar_arrive_expect_tx(b, SH::FBYTES);
#pragma unroll
        for (int q = 0; q < Q; ++q)
            tma_load_4d(fbase + s * SH::FSLOT + q * SH::FBOX, &maps.f, xs, y0 - L::ey(q), z - L::ez(q), q, b);
    };
    // bit s: parity of the next phase of slot s (registers, no dynamic indexing); gout /
    // fout bit s: slot s has copies issued whose phase this thread has not yet seen complete
    // (every thread tracks the issues of thread 0, which depend on cz only)
    unsigned gph = 0u, fph = 0u, gout = 0u, fout = 0u;
    bool ok = true;
    auto wait_g = [&](int cz) {
        const int s = cz & 1;
        if (ok && mbar_wait(&bars[s], (gph >> s) & 1u, limit)) {
            gph ^= 1u << s;
            gout &= ~(1u << s);
        } else {
            ok = false;
        }
    };
    auto wait_f = [&](int z) {
        const int s = z & 1;
        if (ok && mbar_wait(&bars[2 + s], (fph >> s) & 1u, limit)) {
            fph ^= 1u << s;
            fout &= ~(1u << s);
        } else {
            ok = false;
        }
    };

    TP gcur[Q], gnext[Q];
    TP ccur = TP(0), cnext = TP(0), dcur = TP(0), dnext = TP(0);
    if (tid == 0) {
        issue_g(z0 - 1, inject);
        issue_g(z0, 0u);
    }
    gout = (1u << ((z0 - 1) & 1)) | (1u << (z0 & 1));
    // Iteration cz: phase field of plane cz (box of the tile and its halo), then the update
    // of plane cz - 1.  Loads in flight: g of planes cz + 1, cz + 2 and f of plane cz.
    for (int cz = z0 - 1; cz <= z1; ++cz) {
        wait_g(cz);
        {
            const int s = cz & 1;
            const bool keep = cz >= z0 && cz < z1;
            R* slot = ring[cz & 3];
            // box index k: the tile's own nodes first (k = tid), then the halo ring
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
                    TP v[Q];
                    const TP cs = TP(cbox(s)[hy * SH::BWC + 31 + hx - SH::XOFFC]);
#pragma unroll
                    for (int q = 0; q < Q; ++q) v[q] = cd.load_dev(&gbox(s, q)[hy * SH::BW + 31 + hx - L::ex(q) - SH::XOFF]);
                    // directions crossing the domain boundary: boundary-aware reread
                    const unsigned m = cross_mask<3>(g, cx, cy, cz);
                    if (m) fix_g<3, PR>(a.gin, a.cin, cd, g, cx, cy, cz, nidx32(g, cx, cy, cz), m, cs, v);
                    const TP sum = pulled_sum<PR, Q>(v);
                    if (keep && k < NT) {
#pragma unroll
                        for (int q = 0; q < Q; ++q) gnext[q] = v[q];
                        cnext = cs;
                        dnext = sum;
                    }
                    cval = ring_c<PR>(sum, cs);
                }
                slot[hy * HX + hx] = cval;
            }
        }
        // g slot of plane cz and f slot of plane cz - 2 are free; a wait of any thread that
        // gave up stops the block here
        if (!__syncthreads_and(ok)) {
            ok = false;
            break;
        }
        const bool more_g = cz + 2 <= z1, more_f = kStageF && cz >= z0 && cz < z1;
        if (tid == 0) {
            if (more_g) issue_g(cz + 2, 0u);
            if (more_f) issue_f(cz);
        }
        if (more_g) gout |= 1u << ((cz + 2) & 1);
        if (more_f) fout |= 1u << (cz & 1);
        const int z = cz - 1;  // plane updated in this iteration
        if (z >= z0) {
            if constexpr (kStageF) wait_f(z);
            if (active) {
                const unsigned self = nidx32(g, x, y, z);
                auto Cf = [&](int dx, int dy, int dz) -> R { return ring[(z + dz) & 3][(ty + 1 + dy) * HX + tx + 1 + dx]; };
                auto Ch = [&](int dx, int dy, int dz) -> TP { return ring_hi<PR>(Cf(dx, dy, dz)); };
                TP mu, dc[3];
                phase_stencil<3, PR>(PP, Cf, mu, dc);
                T fpost[Q];
                const unsigned m = cross_mask<3>(g, x, y, z);
                if constexpr (kStageF) {
                    const int s = z & 1;
#pragma unroll
                    for (int q = 0; q < Q; ++q)
                        fpost[q] = cd.load_f(&fbox(s, q)[ty * SH::BW + 32 + tx - L::ex(q) - SH::XOFF]);
                    if (m) fix_f<3, PR>(a.fin, cd, g, x, y, z, self, m, fpost);
                } else {
                    pull_f<3, PR>(a.fin, cd, g, x, y, z, self, m, fpost, a.par);
                }
                const unsigned dmask = cross_mask<3, true>(g, x, y, z);
                const TP cown = Ch(0, 0, 0);
                auto cdest = [&](int q) { return dest_shift_q<3, PR>(q, dmask, cown, Ch); };
                update_node<3, PR>(a, cd, PT, PP, self, fpost, [&](int q) { return gcur[q]; }, dcur, ccur, cown, mu,
                                   dc, cdest);
            }
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) gcur[q] = gnext[q];
        ccur = cnext;
        dcur = dnext;
    }
    if (__syncthreads_and(ok)) return;
    // A wait gave up: release the injected bytes, wait for the copies still in flight, then
    // record the failure.
    if (tid == 0 && inject) mbar_complete_tx(&bars[(z0 - 1) & 1], inject);
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        if ((gout >> s) & 1u) (void)mbar_wait(&bars[s], (gph >> s) & 1u);
        if ((fout >> s) & 1u) (void)mbar_wait(&bars[2 + s], (fph >> s) & 1u);
    }
    if (tid == 0) atomicOr(err, 1);
}

}  // namespace clipb
