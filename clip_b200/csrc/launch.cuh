// Host launchers of the kernels in kernels.cuh for one precision policy PR.  Included
// once by each kernels_fp*.cu translation unit, which compiles it with that precision's
// floating-point flags.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstring>

#include "kernels.cuh"
#include "kernels_tma.cuh"

namespace clipb {

// SM count of the current device (looked up once per device).
inline int sm_count() {
    constexpr int kDevs = 64;
    static std::atomic<int> of[kDevs];
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    if (dev >= 0 && dev < kDevs && (v = of[dev].load(std::memory_order_acquire)) > 0) return v;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v < 1) v = 148;
    if (dev >= 0 && dev < kDevs) of[dev].store(v, std::memory_order_release);
    return v;
}

// Rows per CTA of the 2D step when none is set: the largest of 16, 8, 4, 2 that still
// gives eight CTAs per SM.  A CTA's rows run one after another, so on a small grid the
// step lasts as long as that chain and short segments fill the GPU (256 x 256 FP64: 17.5
// us per step at 2 rows, 105 us at 16).
inline int default_rows2(const Geom& g, int TX) {
    const long long tiles = (g.n[0] + TX - 1) / TX;
    int seg = 16;
    while (seg > 2 && tiles * ((g.n[1] + seg - 1) / seg) < 8LL * sm_count()) seg /= 2;
    return seg;
}

template <class PR, bool kKeepG2, bool kKeepG3>
struct Launch {
    using A = typename PR::A;

    static StepArgs<PR> args(const DevState& st, long long k) {
        StepArgs<PR> a;
        const int in = (int)(k & 1), out = in ^ 1;
        a.fin = static_cast<const typename PR::Sf*>(st.f[in]);
        a.gin = static_cast<const typename PR::Sg*>(st.gp[in]);
        a.fout = static_cast<typename PR::Sf*>(st.f[out]);
        a.gout = static_cast<typename PR::Sg*>(st.gp[out]);
        a.cin = static_cast<const A*>(st.c[in]);
        a.cout = static_cast<A*>(st.c[out]);
        a.u = static_cast<A*>(st.u);
        a.uin = static_cast<const A*>(st.uin ? st.uin : st.u);
        a.g = st.g;
        a.phys = st.phys;
        a.pt = phys_cast<typename PR::T>(st.phys);
        a.pp = phys_cast<typename PR::TP>(st.phys);
        a.pop_scale = st.pop_scale;
        a.par = in;
        a.mon = st.mon_rows;
        return a;
    }

    static cudaError_t init(const DevState& st, cudaStream_t s) { return init_planes(st, 0, st.g.dim == 3 ? st.g.e[2] : 1, s); }
    // initial state of the ghosted planes [z0, z1) (2D: the one plane)
    static cudaError_t init_planes(const DevState& st, int z0, int z1, cudaStream_t s) {
        const Geom& g = st.g;
        if (z1 <= z0) return cudaSuccess;
        const dim3 b(32, 8, 1);
        const dim3 gr((g.e[0] + 31) / 32, (g.e[1] + 7) / 8, g.dim == 3 ? z1 - z0 : 1);
        if (g.dim == 2) init_kernel<2, PR><<<gr, b, 0, s>>>(st, 0);
        else init_kernel<3, PR><<<gr, b, 0, s>>>(st, z0);
        return cudaGetLastError();
    }

    static cudaError_t ghost(const DevState& st, long long k, cudaStream_t s) {
        const Geom& g = st.g;
        if (g.vel_side < 0) return cudaSuccess;
        const int ax = g.vel_side / 2;
        if (g.dim == 2) {
            const int n1 = g.n[ax == 0 ? 1 : 0] + 2;
            inlet_kernel<2, PR><<<(n1 + 127) / 128, 128, 0, s>>>(st, k);
        } else {
            const int n1 = g.n[ax == 0 ? 1 : 0] + 2, n2 = g.n[ax == 2 ? 1 : 2] + 2;
            inlet_kernel<3, PR><<<dim3((n1 + 31) / 32, (n2 + 7) / 8), dim3(32, 8), 0, s>>>(st, k);
        }
        return cudaGetLastError();
    }

    template <int TX, int TY, bool kKeep, bool kOpen>
    static void go3(const DevState& st, const StepArgs<PR>& a, cudaStream_t s) {
        const Geom& g = st.g;
        const int seg = st.seg > 0 ? st.seg : 64;
        const dim3 gr((g.n[0] + TX - 1) / TX, (g.n[1] + TY - 1) / TY, (g.zhi - g.zlo + seg) / seg);
        if constexpr (!kOpen) {
            if (a.mon) {
                step3d_kernel<PR, TX, TY, kKeep, false, true><<<gr, dim3(TX, TY), 0, s>>>(a, seg);
                return;
            }
        }
        step3d_kernel<PR, TX, TY, kKeep, kOpen><<<gr, dim3(TX, TY), 0, s>>>(a, seg);
    }
    // Staged 3D step (FP32/FP16 storage): tensor maps [TY = 8, 4][input parity].
    static constexpr bool kStaged = !PR::kExact;
    template <int TY, bool kStageF = true>
    static constexpr int staged_smem() { return StageShape<PR, TY, kStageF>::SMEM + 128; }

    template <int TY>
    static cudaError_t encode_stage(const DevState& st, StageMaps* m) {
        using SH = StageShape<PR, TY>;
        const Geom& g = st.g;
        const CUtensorMapDataType pt = PR::kHalf ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
        const cuuint64_t eb = sizeof(typename PR::Sf), ab = sizeof(A);
        const cuuint64_t pd[4] = {(cuuint64_t)g.sy, (cuuint64_t)g.e[1], (cuuint64_t)g.e[2], 19};
        const cuuint64_t ps[3] = {g.sy * eb, g.sz * eb, g.ps * eb};
        const cuuint32_t gbox[4] = {SH::BW, SH::HY, 1, 1}, fbox[4] = {SH::BW, TY, 1, 1};
        const cuuint64_t cd[3] = {(cuuint64_t)g.sy, (cuuint64_t)g.e[1], (cuuint64_t)g.e[2]};
        const cuuint64_t cs[2] = {g.sy * ab, g.sz * ab};
        const cuuint32_t cbox[3] = {SH::BWC, SH::HY, 1};
        for (int b = 0; b < 2; ++b) {
            cudaError_t e;
            if ((e = encode_tiled(&m[b].f, pt, 4, st.f[b], pd, ps, fbox)) != cudaSuccess) return e;
            if ((e = encode_tiled(&m[b].g, pt, 4, st.gp[b], pd, ps, gbox)) != cudaSuccess) return e;
            if ((e = encode_tiled(&m[b].c, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, st.c[b], cd, cs, cbox)) != cudaSuccess)
                return e;
        }
        cudaError_t e = cudaFuncSetAttribute(step3d_staged_kernel<PR, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             staged_smem<TY>());
        if (e == cudaSuccess && TY == 8)
            e = cudaFuncSetAttribute(step3d_staged_kernel<PR, 8, false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     staged_smem<8, false>());
        return e;
    }

    // Tensor maps and shared-memory limits of the staged variants; without them (FP64, 2D,
    // or a driver that cannot encode the maps) those variants are unavailable.
    static cudaError_t prepare(DevState& st) {
        if constexpr (kStaged) {
            static_assert(sizeof(A) == 4, "the c tensor map is FP32");
            if (st.g.dim != 3) return cudaSuccess;
            cudaError_t ek = cudaSuccess;
            auto allow = [&](auto kernel, int bytes) {
                if (ek == cudaSuccess)
                    ek = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            };
            allow(step3d_smemkeep_kernel<PR, 32, 8, 2, false>, smemkeep_bytes<8>());
            allow(step3d_smemkeep_kernel<PR, 32, 8, 3, false>, smemkeep_bytes<8>());
            allow(step3d_smemkeep_kernel<PR, 32, 8, 2, true>, smemkeep_bytes<8>());
            allow(step3d_smemkeep_kernel<PR, 32, 8, 3, true>, smemkeep_bytes<8>());
            allow(step3d_smemkeep_kernel<PR, 32, 8, 2, false, true>, smemkeep_bytes<8>());
            allow(step3d_smemkeep_kernel<PR, 32, 8, 3, false, true>, smemkeep_bytes<8>());
            if (ek != cudaSuccess) return ek;
            auto* h = new StageHost();
            cudaError_t e = encode_stage<8>(st, h->maps[0]);
            if (e == cudaSuccess) e = encode_stage<4>(st, h->maps[1]);
            if (e != cudaSuccess) {
                delete h;
                return e;
            }
            st.stage = h;
        }
        return cudaSuccess;
    }
    static void release(DevState& st) {
        delete static_cast<StageHost*>(st.stage);
        st.stage = nullptr;
    }
    static bool available(const DevState& st, int variant) {
        if (st.g.dim != 3) return variant >= 0 && variant < kVariants2;
        if (variant < 5) return variant >= 0;
        // the staged kernel resolves wall, periodic and inlet sides of a whole case only
        if ((variant == 5 || variant == 6 || variant == 9) && (st.g.open || st.g.xch)) return false;
        if (variant == 7 || variant == 8) return kStaged;
        return kStaged && variant < kVariants3 && st.stage != nullptr;
    }

    template <int TY, bool kStageF = true>
    static void go3s(const DevState& st, const StepArgs<PR>& a, long long k, cudaStream_t s) {
        if constexpr (kStaged) {
            const Geom& g = st.g;
            const int seg = st.seg > 0 ? st.seg : 64;
            const dim3 gr((g.n[0] + 31) / 32, (g.n[1] + TY - 1) / TY, (g.n[2] + seg - 1) / seg);
            const StageMaps& m = static_cast<const StageHost*>(st.stage)->maps[TY == 8 ? 0 : 1][k & 1];
            const long long limit = st.wait_limit > 0 ? st.wait_limit : kWaitCycles;
            if (kStageF)
                step3d_staged_kernel<PR, TY><<<gr, dim3(32, TY), staged_smem<TY>(), s>>>(a, seg, m, st.err, limit,
                                                                                         st.wait_inject);
            else
                step3d_staged_kernel<PR, 8, false, 2><<<gr, dim3(32, 8), staged_smem<8, false>(), s>>>(
                    a, seg, m, st.err, limit, st.wait_inject);
        }
    }

    // Batched 2D step: args = device table of StepArgs<PR> (one per case, this step's
    // parity), items = (case, bx, by) triples built for the variant's tile width and `seg`.
    // The grid is persistent: SM count x blocks_per_sm (0: as many as fit).
    template <int TX, bool kKeep>
    static cudaError_t go2_batch(const void* args, const int* items, int nitems, int seg, int blocks_per_sm,
                                 cudaStream_t s) {
        // resident blocks per SM and SM count, per device (looked up once per device; the
        // lookup is idempotent, so concurrent first calls may both do it)
        constexpr int kDevs = 64;
        static std::atomic<int> fit_of[kDevs], sms_of[kDevs];
        int dev = 0;
        cudaGetDevice(&dev);
        int fit = dev >= 0 && dev < kDevs ? fit_of[dev].load(std::memory_order_acquire) : 0;
        int sms = dev >= 0 && dev < kDevs ? sms_of[dev].load(std::memory_order_acquire) : 0;
        if (!fit || !sms) {
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 1;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, step2d_batch_kernel<PR, TX, kKeep>, TX, 0) !=
                    cudaSuccess || fit < 1)
                fit = 1;
            if (dev >= 0 && dev < kDevs) {
                sms_of[dev].store(sms, std::memory_order_release);
                fit_of[dev].store(fit, std::memory_order_release);
            }
        }
        const int bps = blocks_per_sm > 0 && blocks_per_sm < fit ? blocks_per_sm : fit;
        const int grid = std::max(1, std::min(nitems, sms * bps));
        step2d_batch_kernel<PR, TX, kKeep><<<grid, TX, 0, s>>>(static_cast<const StepArgs<PR>*>(args), items, nitems,
                                                                 seg);
        return cudaGetLastError();
    }
    static cudaError_t step2_batch(const void* args, const int* items, int nitems, int variant, int seg,
                                   int blocks_per_sm, cudaStream_t s) {
        switch (variant) {
            case 1: return go2_batch<32, kKeepG2>(args, items, nitems, seg, blocks_per_sm, s);
            case 2: return go2_batch<128, kKeepG2>(args, items, nitems, seg, blocks_per_sm, s);
            case 3: return go2_batch<64, false>(args, items, nitems, seg, blocks_per_sm, s);
            default: return go2_batch<64, kKeepG2>(args, items, nitems, seg, blocks_per_sm, s);
        }
    }
    static int tile2(int variant) { return variant == 1 ? 32 : (variant == 2 ? 128 : 64); }
    static void make_args(const DevState& st, long long k, void* out) {
        const StepArgs<PR> a = args(st, k);
        std::memcpy(out, &a, sizeof(a));
    }

    // kept g of a 32 x TY tile: two planes of (Q + 2) values per node (the 19 pulled
    // deviations, c_old and their sum)
    template <int TY>
    static constexpr int smemkeep_bytes() {
        return 2 * 21 * 32 * TY * (int)sizeof(typename PR::TP);
    }
    template <int TY, int kMinBlocks, bool kOpen>
    static void go3k(const DevState& st, const StepArgs<PR>& a, cudaStream_t s) {
        if constexpr (kStaged) {
            const Geom& g = st.g;
            const int seg = st.seg > 0 ? st.seg : 16;
            const dim3 gr((g.n[0] + 31) / 32, (g.n[1] + TY - 1) / TY, (g.zhi - g.zlo + seg) / seg);
            if constexpr (!kOpen) {
                if (a.mon) {
                    step3d_smemkeep_kernel<PR, 32, TY, kMinBlocks, false, true>
                        <<<gr, dim3(32, TY), smemkeep_bytes<TY>(), s>>>(a, seg);
                    return;
                }
            }
            step3d_smemkeep_kernel<PR, 32, TY, kMinBlocks, kOpen>
                <<<gr, dim3(32, TY), smemkeep_bytes<TY>(), s>>>(a, seg);
        }
    }

    template <int TX, bool kKeep, bool kOpen>
    static void go2(const DevState& st, const StepArgs<PR>& a, cudaStream_t s) {
        const Geom& g = st.g;
        const int seg = st.seg > 0 ? st.seg : default_rows2(g, TX);
        const dim3 gr((g.n[0] + TX - 1) / TX, (g.n[1] + seg - 1) / seg);
        step2d_kernel<PR, TX, kKeep, kOpen><<<gr, TX, 0, s>>>(a, seg);
    }

    // Launch variants (tile shape, whether g of the next plane stays in registers); the
    // autotuner in capi.cu picks one per solver.  kKeepG2/kKeepG3 = false restricts a
    // precision to the re-pulling variants (FP64: registers).
    // Variants 5 and 6 (FP32/FP16) are the staged step with 32 x 8 and 32 x 4 tiles.
    // Variants 7 and 8 (FP32/FP16) keep the next plane's g in shared memory, with at least
    // 2 and 3 resident 32 x 8 blocks per SM.
    // Variant 9 (FP32/FP16) is the staged step with g by bulk copies and f pulled from global
    // memory, at least 2 resident 32 x 8 blocks per SM.
    static constexpr int kVariants3 = kStaged ? 10 : 5, kVariants2 = 4;

    // kOpen: the kernel instances for cases with free-convect or Neumann sides.
    template <bool kOpen>
    static void step_shape(const DevState& st, const StepArgs<PR>& a, long long k, cudaStream_t s) {
        if (st.g.dim == 3) {
            switch (st.variant) {
                case 1: go3<32, 8, kKeepG3, kOpen>(st, a, s); break;
                case 2: go3<32, 16, false, kOpen>(st, a, s); break;
                case 3: go3<64, 8, false, kOpen>(st, a, s); break;
                case 4: go3<32, 4, kKeepG3, kOpen>(st, a, s); break;
                case 5:
                    if constexpr (!kOpen) go3s<8>(st, a, k, s);
                    break;
                case 6:
                    if constexpr (!kOpen) go3s<4>(st, a, k, s);
                    break;
                case 7: go3k<8, 2, kOpen>(st, a, s); break;
                case 8: go3k<8, 3, kOpen>(st, a, s); break;
                case 9:
                    if constexpr (!kOpen) go3s<8, false>(st, a, k, s);
                    break;
                default: go3<32, 8, false, kOpen>(st, a, s); break;
            }
        } else {
            switch (st.variant) {
                case 1: go2<32, kKeepG2, kOpen>(st, a, s); break;
                case 2: go2<128, kKeepG2, kOpen>(st, a, s); break;
                case 3: go2<64, false, kOpen>(st, a, s); break;
                default: go2<64, kKeepG2, kOpen>(st, a, s); break;
            }
        }
    }

    static cudaError_t step(const DevState& st, long long k, cudaStream_t s) {
        const StepArgs<PR> a = args(st, k);
        if (st.g.open) step_shape<true>(st, a, k, s);
        else step_shape<false>(st, a, k, s);
        return cudaGetLastError();
    }

    static cudaError_t field(const DevState& st, int which, int last, long long, double* out, cudaStream_t s) {
        const Geom& g = st.g;
        const dim3 b(32, 8, 1);
        const dim3 gr((g.e[0] + 31) / 32, (g.e[1] + 7) / 8, g.dim == 3 ? g.e[2] : 1);
        if (g.dim == 2) field_kernel<2, PR><<<gr, b, 0, s>>>(st, which, last, out);
        else field_kernel<3, PR><<<gr, b, 0, s>>>(st, which, last, out);
        return cudaGetLastError();
    }

    static cudaError_t set_state(const DevState& st, int b, const double* F, const double* G, const double* C,
                                 const double* U, cudaStream_t s) {
        const Geom& g = st.g;
        const dim3 bl(32, 8, 1);
        const dim3 gr((g.e[0] + 31) / 32, (g.e[1] + 7) / 8, g.dim == 3 ? g.e[2] : 1);
        if (g.dim == 2) state_kernel<2, PR><<<gr, bl, 0, s>>>(st, b, F, G, C, U);
        else state_kernel<3, PR><<<gr, bl, 0, s>>>(st, b, F, G, C, U);
        return cudaGetLastError();
    }

    static cudaError_t interior(const DevState& st, int which, int last, long long, double* out, cudaStream_t s) {
        const Geom& g = st.g;
        const dim3 b(32, 8, 1);
        const dim3 gr((g.n[0] + 31) / 32, (g.n[1] + 7) / 8, g.dim == 3 ? g.n[2] : 1);
        if (g.dim == 2) interior_kernel<2, A><<<gr, b, 0, s>>>(st, which, last, out);
        else interior_kernel<3, A><<<gr, b, 0, s>>>(st, which, last, out);
        return cudaGetLastError();
    }

    static cudaError_t vts_pack(const DevState& st, int last, void* out, bool single, cudaStream_t s) {
        const Geom& g = st.g;
        const dim3 b(32, 8, 1);
        const dim3 gr((g.n[0] + 31) / 32, (g.n[1] + 7) / 8, g.dim == 3 ? g.zhi - g.zlo + 1 : 1);
        if (g.dim == 2) {
            if (single) vts_pack_kernel<2, PR, float><<<gr, b, 0, s>>>(st, last, static_cast<float*>(out));
            else vts_pack_kernel<2, PR, double><<<gr, b, 0, s>>>(st, last, static_cast<double*>(out));
        } else {
            if (single) vts_pack_kernel<3, PR, float><<<gr, b, 0, s>>>(st, last, static_cast<float*>(out));
            else vts_pack_kernel<3, PR, double><<<gr, b, 0, s>>>(st, last, static_cast<double*>(out));
        }
        return cudaGetLastError();
    }

    static cudaError_t monitors(const DevState& st, long long steps, double* out2, cudaStream_t s) {
        const int cbuf = (int)(steps & 1);  // c written by the last step (c[0] right after init)
        if (st.g.dim == 2) monitor_partials<2, A><<<st.red_blocks, 256, 0, s>>>(st, cbuf);
        else monitor_partials<3, A><<<st.red_blocks, 256, 0, s>>>(st, cbuf);
        monitor_final<A><<<1, 32, 0, s>>>(st.red, st.red_blocks, st.err, out2);
        return cudaGetLastError();
    }

    static cudaError_t monitor_rows(const DevState& st, const double* rows, double* out2, cudaStream_t s) {
        const Geom& g = st.g;
        const long long n = (long long)((g.n[0] + 31) / 32) * g.n[1] * (g.zhi - g.zlo + 1);
        monitor_rows_partials<A><<<st.red_blocks, 256, 0, s>>>(rows, n, st.red);
        monitor_final<A><<<1, 32, 0, s>>>(st.red, st.red_blocks, st.err, out2);
        return cudaGetLastError();
    }
    // the variants whose 3D step runs step3d_body (all but the staged ones), on cases without
    // free-convect or Neumann sides (the monitored instances carry no open-side code)
    static bool fused_monitors(const DevState& st) {
        return st.g.dim == 3 && !st.g.open && st.variant != 5 && st.variant != 6 && st.variant != 9;
    }

    static KernelTable table() {
        KernelTable t;
        t.prepare = &prepare;
        t.release = &release;
        t.available = &available;
        t.args_bytes = sizeof(StepArgs<PR>);
        t.make_args = &make_args;
        t.step2_batch = &step2_batch;
        t.tile2 = &tile2;
        t.set_state = &set_state;
        t.init = &init;
        t.init_planes = &init_planes;
        t.monitor_rows = &monitor_rows;
        t.fused_monitors = &fused_monitors;
        t.ghost = &ghost;
        t.step = &step;
        t.field = &field;
        t.interior = &interior;
        t.monitors = &monitors;
        t.vts_pack = &vts_pack;
        t.aux_bytes = (int)sizeof(A);
        t.pop_bytes = (int)sizeof(typename PR::Sf);
        t.variants2 = kVariants2;
        t.variants3 = kVariants3;
        return t;
    }
};

}  // namespace clipb
