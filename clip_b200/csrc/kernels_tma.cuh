// Staged 3D step: the g and f tiles of coming planes are brought into shared memory by
// bulk tensor copies (TMA) while the CTA computes the current plane.
//
// CTA = 32 x TY tile of an (x,y) plane marching in z (same work split and results as
// step3d_body).  Tiles next to the domain boundary in x or y run step3d_body instead.
// Per iteration (update of plane z):
//   wait g(z+1) -> phase field of plane z+1 (tile + halo ring) from the staged g box
//   barrier
//   thread 0 issues g(z+2) and f(z+1) (their slots were last read before the barrier)
//   wait f(z)   -> update of plane z from the staged f box, stores to global memory
// g slots hold, per direction q, the (TX+2) x (TY+2) box of source nodes of the tile and
// its halo, shifted by -e_q; f slots the TX x TY box; a c slot the readers' own c.  A box
// starts at an x element rounded down to 16 bytes, so the lattice shift -e_x becomes a
// column offset in shared memory.  Planes 1 and n (next to a z boundary) pull from global
// memory with the boundary-aware path; ghost planes map c as in step3d_body.
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

template <class PR, int TY>
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
    static constexpr int SMEM = BARS + 2 * GSLOT + 2 * FSLOT;
    static constexpr uint32_t GBYTES = Q * BW * HY * EB + BWC * HY * 4;  // bytes landing per g load
    static constexpr uint32_t FBYTES = Q * BW * TY * EB;
};

template <class PR, int TY>
__global__ void __launch_bounds__(32 * TY) step3d_staged_kernel(StepArgs<PR> a, int seg,
                                                                 const __grid_constant__ StageMaps maps, int* err) {
    using SH = StageShape<PR, TY>;
    using TP = typename PR::TP;
    using T = typename PR::T;
    using A = typename PR::A;
    using Sg = typename PR::Sg;
    using Sf = typename PR::Sf;
    using L = Lat<3>;
    constexpr int Q = 19, TX = 32, HX = TX + 2, NHALO = 2 * HX + 2 * TY, NT = TX * TY;
    __shared__ TP ring[4][HX * (TY + 2)];
    extern __shared__ __align__(128) unsigned char dsm_raw[];
    // bulk tensor copies need 128-byte aligned shared destinations (launch adds 128 bytes)
    unsigned char* dsm = dsm_raw + ((128u - (smem_addr(dsm_raw) & 127u)) & 127u);

    const Geom& g = a.g;
    const int bx = (int)blockIdx.x, by = (int)blockIdx.y, bz = (int)blockIdx.z;
    const int x0 = 1 + bx * TX, y0 = 1 + by * TY;
    const bool deep_xy = x0 - 1 >= 2 && x0 + TX <= g.n[0] - 1 && y0 - 1 >= 2 && y0 + TY <= g.n[1] - 1;
    if (!deep_xy) {
        step3d_body<PR, TX, TY, false>(a, seg, bx, by, bz, ring);
        return;
    }
    const Phys<T> PT = phys_cast<T>(a.phys);
    const Phys<TP> PP = phys_cast<TP>(a.phys);
    const Codec<PR> cd(a.pop_scale);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int x = x0 + tx, y = y0 + ty;
    const int z0 = 1 + bz * seg;
    const int z1 = min(z0 + seg, g.n[2] + 1);
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

    auto issue_g = [&](int cz) {  // thread 0
        const int s = cz & 1;
        uint64_t* b = &bars[s];
        mbar_arrive_expect_tx(b, SH::GBYTES);
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
    // bit s: parity of the next phase of slot s (registers, no dynamic indexing)
    unsigned gph = 0u, fph = 0u;
    bool ok = true;
    auto wait_g = [&](int cz) {
        const int s = cz & 1;
        ok = ok && mbar_wait(&bars[s], (gph >> s) & 1u);
        gph ^= 1u << s;
    };
    auto wait_f = [&](int z) {
        const int s = z & 1;
        ok = ok && mbar_wait(&bars[2 + s], (fph >> s) & 1u);
        fph ^= 1u << s;
    };

    // phase field of one node of plane cz (tile coordinates hx, hy in the halo box)
    auto node_c = [&](int hx, int hy, int cz, Sg* keep, TP* keep_c) -> TP {
        const int cx = x0 - 1 + hx, cy = y0 - 1 + hy;
        if (cz < 1 || cz > g.n[2]) return TP(ghost_c<3, A>(a.cin, g, cx, cy, cz));
        if (cz == 1 || cz == g.n[2]) {  // next to a z boundary: boundary-aware global pull
            TP v[Q];
            pull_g<3, PR>(a.gin, a.cin, cd, g, cx, cy, cz, nidx(g, cx, cy, cz), true, v);
            TP c = v[0];
#pragma unroll
            for (int q = 1; q < Q; ++q) c = c + v[q];
            if (keep) {
                // keep the rebuilt values as raw storage plus a zero shift
#pragma unroll
                for (int q = 0; q < Q; ++q) keep[q] = Sg(0);
                *keep_c = TP(0);
            }
            return c;
        }
        const int s = cz & 1;
        const TP cself = TP(cbox(s)[hy * SH::BWC + 31 + hx - SH::XOFFC]);
        TP c = TP(0);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const Sg raw = gbox(s, q)[hy * SH::BW + 31 + hx - L::ex(q) - SH::XOFF];
            c = c + cd.template load_g<3>(&raw, q, cself);
            if (keep) keep[q] = raw;
        }
        if (keep) *keep_c = cself;
        return c;
    };
    // keep[] holds raw stored g of the own node (and keep_c its shift); for the boundary
    // planes the update pulls again from global memory.
    auto plane_c = [&](int cz, Sg* keep, TP* keep_c) {
        TP* slot = ring[cz & 3];
        slot[(ty + 1) * HX + tx + 1] = node_c(tx + 1, ty + 1, cz, keep, keep_c);
        for (int h = tid; h < NHALO; h += NT) {
            int hx, hy;
            halo_coords<TX, TY>(h, hx, hy);
            slot[hy * HX + hx] = node_c(hx, hy, cz, nullptr, nullptr);
        }
    };

    Sg gcur[Q], gnext[Q];
    TP ccur = TP(0), cnext = TP(0);
    if (tid == 0) {
        issue_g(z0 - 1);
        issue_g(z0);
        issue_f(z0);
    }
    wait_g(z0 - 1);
    plane_c(z0 - 1, nullptr, nullptr);
    wait_g(z0);
    plane_c(z0, gcur, &ccur);
    __syncthreads();  // slot of plane z0-1 is free
    if (tid == 0 && z0 + 1 <= z1) issue_g(z0 + 1);

    for (int z = z0; z < z1; ++z) {
        wait_g(z + 1);
        plane_c(z + 1, z + 1 < z1 ? gnext : nullptr, &cnext);
        __syncthreads();
        if (tid == 0) {
            if (z + 2 <= z1) issue_g(z + 2);
            if (z + 1 < z1) issue_f(z + 1);
        }
        wait_f(z);
        {
            const long long self = nidx(g, x, y, z);
            auto Cf = [&](int dx, int dy, int dz) -> TP { return ring[(z + dz) & 3][(ty + 1 + dy) * HX + tx + 1 + dx]; };
            TP mu, dc[3];
            stencil<3, TP>(PP, Cf, mu, dc);
            T fpost[Q];
            TP gpost[Q];
            if (z == 1 || z == g.n[2]) {
                pull_f<3, PR>(a.fin, cd, g, x, y, z, self, true, fpost);
                pull_g<3, PR>(a.gin, a.cin, cd, g, x, y, z, self, true, gpost);
            } else {
                const int s = z & 1;
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    fpost[q] = cd.load_f(&fbox(s, q)[ty * SH::BW + 32 + tx - L::ex(q) - SH::XOFF]);
                    gpost[q] = cd.template load_g<3>(&gcur[q], q, ccur);
                }
            }
            TP cdest[Q];
            auto Cd = [&](int dx, int dy, int dz) { return TP(A(Cf(dx, dy, dz))); };
            dest_shift<3, PR>(g, x, y, z, Cd(0, 0, 0), Cd, cdest);
            update_node<3, PR>(a, cd, PT, PP, self, fpost, gpost, Cf(0, 0, 0), mu, dc, cdest);
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) gcur[q] = gnext[q];
        ccur = cnext;
    }
    if (!ok && tid == 0) atomicOr(err, 1);
}

}  // namespace clipb
