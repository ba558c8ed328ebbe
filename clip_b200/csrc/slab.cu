// Slab decomposition along z (C ABI in include/clipb.h).
//
// A 3D case is split into slabs of whole z planes, one per GPU.  A slab solver owns global
// planes z_begin .. z_end.  On each face inside the case (an exchange face) it keeps one
// extra plane (E, the neighbour's boundary plane) and the ghost plane beyond it (G, the
// plane after that).  Its step updates only the owned planes; it computes c on E by
// pulling g there (sources on E, G and its own boundary plane), exactly as the whole case
// computes c on that plane, so the owned planes see the same phase field, stencils and
// streamed populations as in the whole case.  Before every step each exchange face
// receives, from the neighbour's stored state of that step: f, g and c of E, and g and c of
// G, in the directions that the step reads there (plane_copies).  A population read from G or E
// carries the shift that the neighbour's interior writer gave it (the c of its
// destination), so it is read like an interior value (EdgeFix::corr, pull_source).
// On the case's periodic z boundary the whole case reads the periodic image instead: the
// other end's boundary plane, its populations of this step but its c of the step before
// (the reference's ghost layer is filled before the macroscopic update), and a population
// crossing that boundary was shifted by its writer's own c.  A slab's face there (a wrap
// face) therefore has no extra plane: its ghost plane receives the other end's boundary
// plane (f, g, c) and is read like the periodic image.  With slabs of at least two planes
// the result equals the whole case's bit for bit.
//
// The exchange itself is the caller's: clipb_slab_pack writes the planes a neighbour needs
// into a device packet (one kernel), clipb_slab_unpack writes a received packet into the
// face's E and G planes; the packet travels between GPUs by any means (NCCL send/recv over
// NVLink, a peer copy).  No kernel here waits on another GPU.  clipb_slab_step_part splits
// a step so that the packets can be packed and moved on another stream while the planes
// away from the faces update.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "clipb.h"
#include "config.hpp"
#include "engine.hpp"
#include "lattice.cuh"
#include "solver.hpp"

using namespace clipb;

namespace {

constexpr int kMaxSegments = 64;

// Up to kMaxSegments contiguous copies of 16-byte multiples (blockIdx.y = copy).
struct CopyList {
    const char* src[kMaxSegments];
    char* dst[kMaxSegments];
    unsigned long long bytes[kMaxSegments];
    int n;
};

__global__ void plane_copy_kernel(CopyList L) {
    const int k = (int)blockIdx.y;
    if (k >= L.n) return;
    const uint4* s = reinterpret_cast<const uint4*>(L.src[k]);
    uint4* d = reinterpret_cast<uint4*>(L.dst[k]);
    const unsigned long long n16 = L.bytes[k] / 16;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n16;
         i += (unsigned long long)gridDim.x * blockDim.x)
        d[i] = s[i];
}

// Bytes of one z plane (padded rows, ghost rows and columns included) of a population
// array and of an aux (c) array.
size_t plane_bytes(const clipb_solver* s, bool pop) {
    return (size_t)s->st.g.sz * (pop ? s->kt.pop_bytes : s->kt.aux_bytes);
}

// The directions a face's step reads, with ez = +1 for a z- face (the planes below the
// owned ones) and -1 for a z+ face: f of E in the directions entering the owned plane
// (e_z = ez, 5 of 19); g of E in every direction (E's own c pulls its in-plane g, and next
// to a wall its bounce-back reads the node's opposite populations, which point either
// way); g of G in the directions entering E (5); plus c of E and G.
bool f_of_e(int q, int ez) { return Lat<3>::ez(q) == ez; }
bool g_of_e(int, int) { return true; }
bool g_of_g(int q, int ez) { return Lat<3>::ez(q) == ez; }

size_t packet_bytes(const clipb_solver* s) {
    int npop = 0;
    for (int q = 0; q < 19; ++q) npop += f_of_e(q, 1) + g_of_e(q, 1) + g_of_g(q, 1);
    return (size_t)npop * plane_bytes(s, true) + 2 * plane_bytes(s, false);
}

// Copies between the planes E (its f, g, c) and G (its g, c; skipped when plane_g < 0) of
// the input buffers of the next step (parity steps % 2) and the packet, in the packet's
// order, for the directions that a face of side ez (see f_of_e) reads.
int plane_copies(clipb_solver* s, int plane_e, int plane_g, int ez, char* packet, bool to_packet,
                 cudaStream_t strm) {
    const DevState& st = s->st;
    const Geom& g = st.g;
    // the input of the next step: after the first part of a step, its output
    const int b = (int)((s->steps + (s->slab_half ? 1 : 0)) & 1);
    const int Q = 19;
    const size_t pp = plane_bytes(s, true), pa = plane_bytes(s, false);
    const size_t pop_stride = (size_t)g.ps * s->kt.pop_bytes;  // bytes between directions
    CopyList L{};
    size_t off = 0;
    auto add = [&](char* buf, size_t buf_off, size_t bytes) {
        char* dev = buf + buf_off;
        L.src[L.n] = to_packet ? dev : packet + off;
        L.dst[L.n] = to_packet ? packet + off : dev;
        L.bytes[L.n] = bytes;
        ++L.n;
        off += bytes;
    };
    char* F = static_cast<char*>(st.f[b]);
    char* G = static_cast<char*>(st.gp[b]);
    char* C = static_cast<char*>(st.c[b]);
    for (int q = 0; q < Q; ++q)
        if (f_of_e(q, ez)) add(F, q * pop_stride + (size_t)plane_e * pp, pp);
    for (int q = 0; q < Q; ++q)
        if (g_of_e(q, ez)) add(G, q * pop_stride + (size_t)plane_e * pp, pp);
    add(C, (size_t)plane_e * pa, pa);
    if (plane_g >= 0) {
        for (int q = 0; q < Q; ++q)
            if (g_of_g(q, ez)) add(G, q * pop_stride + (size_t)plane_g * pp, pp);
        add(C, (size_t)plane_g * pa, pa);
    }
    const dim3 grid(64, L.n);
    plane_copy_kernel<<<grid, 256, 0, strm>>>(L);
    CLIPB_CUDA(cudaGetLastError());
    return CLIPB_OK;
}

}  // namespace

int clipb_slab_create(const char* config_path, int precision, int z_begin, int z_end, int exchange_faces,
                      clipb_solver** out) {
    if (!config_path || !out) return fail(CLIPB_E_ARG, "null argument");
    *out = nullptr;
    CaseConfig cfg;
    try {
        cfg = load_config(config_path);
    } catch (const std::exception& e) {
        return fail(CLIPB_E_CONFIG, e.what());
    }
    if (cfg.dim != 3) return fail(CLIPB_E_CONFIG, "slabs split 3D cases along z");
    const int N = cfg.interior[2];
    if (z_begin < 1 || z_end > N || z_end - z_begin + 1 < 2)
        return fail(CLIPB_E_ARG, "a slab owns at least two of the planes 1.." + std::to_string(N));
    for (int i = 0; i < 6; ++i) {
        const int t = cfg.bc.type[i];
        if (t == kVelocity || t == kFreeConvect || t == kNeumann)
            return fail(CLIPB_E_CONFIG, "slabs take wall, slip-wall and periodic sides");
    }
    const bool zper = cfg.bc.type[kZMinus] == kPeriodic;
    const bool lo = exchange_faces & 1, hi = exchange_faces & 2;
    if ((z_begin > 1 && !lo) || (z_end < N && !hi))
        return fail(CLIPB_E_ARG, "a face inside the case must be an exchange face");
    if ((z_begin == 1 && lo && !zper) || (z_end == N && hi && !zper))
        return fail(CLIPB_E_ARG, "a face on a non-periodic boundary of the case cannot be exchanged");
    if (zper && (lo != hi || (!lo && (z_begin != 1 || z_end != N))))
        return fail(CLIPB_E_ARG, "on a periodic z axis a slab either holds the whole axis or exchanges both faces");
    const int own = z_end - z_begin + 1;
    // an exchange face inside the case keeps the neighbour's boundary plane; a face on the
    // periodic boundary (wrap) keeps only the ghost plane
    const bool lo_in = lo && z_begin > 1, hi_in = hi && z_end < N;
    cfg.interior[2] = own + (lo_in ? 1 : 0) + (hi_in ? 1 : 0);
    cfg.extent[2] = cfg.interior[2] + 2;
    cfg.phys.N[2] = cfg.extent[2];
    cfg.zlo = lo_in ? 2 : 1;
    cfg.zhi = cfg.zlo + own - 1;
    cfg.zoff = z_begin - cfg.zlo;
    cfg.zglobal = N;
    if (lo) cfg.bc.type[kZMinus] = lo_in ? kExchange : kWrap;
    if (hi) cfg.bc.type[kZPlus] = hi_in ? kExchange : kWrap;
    return solver_create(cfg, precision, out);
}

int clipb_slab_info(const clipb_solver* s, int* z_begin, int* z_end, int* zlo, int* zhi, long long* packet_bytes_out) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    const CaseConfig& c = s->cfg;
    const int lo = c.zlo, hi = c.zhi > 0 ? c.zhi : c.interior[2];
    if (z_begin) *z_begin = lo + c.zoff;
    if (z_end) *z_end = hi + c.zoff;
    if (zlo) *zlo = lo;
    if (zhi) *zhi = hi;
    if (packet_bytes_out) *packet_bytes_out = (long long)packet_bytes(s);
    return CLIPB_OK;
}

int clipb_slab_pack(clipb_solver* s, int toward, void* dev_packet, void* stream) {
    if (!s || !dev_packet) return fail(CLIPB_E_ARG, "null argument");
    if (!s->initialized) return fail(CLIPB_E_STATE, "pack before init");
    if (toward != 0 && toward != 1) return fail(CLIPB_E_ARG, "toward: 0 = the z- neighbour, 1 = the z+ neighbour");
    const Geom& g = s->st.g;
    if (g.dim != 3 || (g.side[4 + toward] != kSideExchange && g.side[4 + toward] != kSideWrap))
        return fail(CLIPB_E_ARG, "that face does not border another slab");
    // the neighbour below needs this slab's first two owned planes, the one above its last
    // two (a wrap face there reads only the first of them)
    const int e = toward == 0 ? g.zlo : g.zhi, gg = toward == 0 ? g.zlo + 1 : g.zhi - 1;
    // the neighbour below reads them through its z+ face, the one above through its z- face
    return plane_copies(s, e, gg, toward == 0 ? -1 : 1, static_cast<char*>(dev_packet), true,
                        stream ? static_cast<cudaStream_t>(stream) : s->stream);
}

int clipb_slab_unpack(clipb_solver* s, int face, const void* dev_packet, void* stream) {
    if (!s || !dev_packet) return fail(CLIPB_E_ARG, "null argument");
    if (!s->initialized) return fail(CLIPB_E_STATE, "unpack before init");
    if (face != 0 && face != 1) return fail(CLIPB_E_ARG, "face: 0 = z-, 1 = z+");
    const Geom& g = s->st.g;
    const int t = g.dim == 3 ? g.side[4 + face] : -1;
    if (t != kSideExchange && t != kSideWrap) return fail(CLIPB_E_ARG, "that face does not border another slab");
    // exchange face: planes E and G; wrap face: the ghost plane only
    const int e = face == 0 ? g.zlo - 1 : g.zhi + 1;
    const int gg = t == kSideWrap ? -1 : (face == 0 ? g.zlo - 2 : g.zhi + 2);
    return plane_copies(s, e, gg, face == 0 ? 1 : -1, const_cast<char*>(static_cast<const char*>(dev_packet)), false,
                        stream ? static_cast<cudaStream_t>(stream) : s->stream);
}

int clipb_slab_step_part(clipb_solver* s, int part) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    if (!s->initialized) return fail(CLIPB_E_STATE, "step before init");
    if (s->cfg.zglobal <= 0) return fail(CLIPB_E_ARG, "not a slab (clipb_slab_create)");
    if (part != 1 && part != 2) return fail(CLIPB_E_ARG, "part: 1 = the planes next to the faces, 2 = the rest");
    if ((part == 1) == s->slab_half) return fail(CLIPB_E_STATE, part == 1 ? "part 2 of the step is due" : "part 2 before part 1");
    const int lo = s->st.g.zlo, hi = s->st.g.zhi;
    // the same step kernel over a range of owned planes (the ring recomputes c on the
    // planes either side, as it does at every segment boundary)
    auto planes = [&](int a, int b) -> int {
        if (a > b) return CLIPB_OK;
        DevState st = s->st;
        st.g.zlo = a;
        st.g.zhi = b;
        CLIPB_CUDA(s->kt.ghost(st, s->steps, s->stream));
        CLIPB_CUDA(s->kt.step(st, s->steps, s->stream));
        return CLIPB_OK;
    };
    int rc;
    const bool split = hi - lo + 1 > 4;
    if (part == 1) {
        if (split) {
            if ((rc = planes(lo, lo + 1)) || (rc = planes(hi - 1, hi))) return rc;
        } else if ((rc = planes(lo, hi))) {
            return rc;
        }
        s->slab_half = true;
    } else {
        if (split && (rc = planes(lo + 2, hi - 2))) return rc;
        s->slab_half = false;
        ++s->steps;
    }
    return CLIPB_OK;
}
