// Checkpoint and resume (C ABI in include/clipb.h).
//
// clipb_save writes, into one folder, the files of the reference's CheckPointer::save
// (src/io/CheckPointer.cu:53-80; raw host arrays as DataArray::writeHostToFile writes them,
// include/data/DataArray.cuh:195-205):
//   dev_f.bin, dev_g.bin, dev_f_post.bin, dev_g_post.bin  Q doubles per node, reference layout
//   dev_f_prev.bin, dev_g_prev.bin (free-convect cases)     the same layout
//   timeInfo.bin   TimeInfo::simInfo {double currentTime; int currentStep; double dt; bool dtIsSet}
//   domainSize.bin N[3] as doubles;  info.txt  the summary lines
// plus clipb_state.bin, libclipb's own state (every device buffer the step reads, in its
// storage precision), so that clipb_load resumes bit for bit.  The reference saves no c or
// u, so its own resume restarts them from the initial condition.  clipb_load of a folder
// without clipb_state.bin sets dev_f and dev_g as the input of the last step and replays
// that step, with c = sum of g_post for the lagged ghost layer and u = sum of e_q f_post
// (the force half-step of the velocity is not in the files) as the previous velocity:
// c comes out exact, u approximate.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <string>
#include <vector>

#include "clipb.h"
#include "config.hpp"
#include "engine.hpp"
#include "solver.hpp"

using namespace clipb;

namespace {

struct SimInfo {  // layout of the reference's TimeInfo::simInfo (include/utils/TimeInfo.cuh:37-43)
    double currentTime;
    int currentStep;
    double dt;
    bool dtIsSet;
};

struct StateHeader {
    char magic[8];
    int version, precision, dim;
    int extent[3];
    long long steps, ps;
    int pop_bytes, aux_bytes, q;
    double pop_scale;
};
constexpr char kMagic[8] = {'C', 'L', 'I', 'P', 'B', 'S', 'T', '1'};

int write_file(const std::string& path, const void* data, size_t bytes) {
    std::ofstream out(path, std::ios::binary);
    if (!out.is_open()) return fail(CLIPB_E_ARG, "cannot write " + path);
    out.write(static_cast<const char*>(data), (std::streamsize)bytes);
    return out.good() ? CLIPB_OK : fail(CLIPB_E_ARG, "write failed: " + path);
}

int read_file(const std::string& path, void* data, size_t bytes) {
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) return fail(CLIPB_E_ARG, "cannot read " + path);
    in.read(static_cast<char*>(data), (std::streamsize)bytes);
    if ((size_t)in.gcount() != bytes) return fail(CLIPB_E_ARG, path + " is shorter than this case needs");
    return CLIPB_OK;
}

// (pointer, bytes) of every device buffer of the native state, in file order
std::vector<std::pair<void*, size_t>> state_buffers(clipb_solver* s) {
    const DevState& st = s->st;
    const int Q = s->cfg.dim == 3 ? 19 : 9;
    const size_t pop = (size_t)Q * st.g.ps * s->kt.pop_bytes, aux = (size_t)st.g.ps * s->kt.aux_bytes;
    std::vector<std::pair<void*, size_t>> b = {{st.f[0], pop},  {st.f[1], pop},          {st.gp[0], pop},
                                               {st.gp[1], pop}, {st.c[0], aux},          {st.c[1], aux},
                                               {st.u, aux * s->cfg.dim}, {st.p, aux},
                                               {st.c0, (size_t)st.g.ps * sizeof(double)}};
    if (s->fc_bytes) {  // free-convect state of both parities
        b.push_back({st.g.fc[0], s->fc_bytes});
        b.push_back({st.g.fc[1], s->fc_bytes});
    }
    return b;
}

}  // namespace

extern "C" {

int clipb_save(clipb_solver* s, const char* dir) {
    if (!s || !dir) return fail(CLIPB_E_ARG, "null argument");
    if (!s->initialized) return fail(CLIPB_E_STATE, "save before init");
    const std::string folder(dir);
    std::error_code ec;
    std::filesystem::create_directories(folder, ec);
    if (ec) return fail(CLIPB_E_ARG, "cannot create " + folder + ": " + ec.message());
    const int Q = s->cfg.dim == 3 ? 19 : 9;
    const size_t nodes = (size_t)s->ref_nodes();
    std::vector<double> host(nodes * Q);
    int rc;
    const struct {
        int field;
        const char* name;
    } pops[] = {{CLIPB_FIELD_G_POST, "dev_g_post"}, {CLIPB_FIELD_F_POST, "dev_f_post"}, {CLIPB_FIELD_G, "dev_g"},
                {CLIPB_FIELD_F, "dev_f"}};
    for (const auto& p : pops) {
        if ((rc = clipb_get_field(s, p.field, host.data(), host.size()))) return rc;
        if ((rc = write_file(folder + "/" + p.name + ".bin", host.data(), host.size() * sizeof(double)))) return rc;
        // A free-convect case also saves dev_g_prev / dev_f_prev (CheckPointer.cu:69-73), which
        // the reference's load reads.  Its next step copies dev_*_post over dev_*_prev before
        // the free-convect pass reads them (NsAllen.cu:849-853), so their saved values are
        // never read after a resume: the files carry the post-streaming values, which is what
        // dev_*_prev holds once that copy has run.
        if (s->fc_bytes && (p.field == CLIPB_FIELD_G_POST || p.field == CLIPB_FIELD_F_POST)) {
            const std::string prev = p.field == CLIPB_FIELD_G_POST ? "/dev_g_prev.bin" : "/dev_f_prev.bin";
            if ((rc = write_file(folder + prev, host.data(), host.size() * sizeof(double)))) return rc;
        }
    }
    SimInfo ti{};
    ti.currentTime = 0.0;
    ti.currentStep = (int)s->steps;
    ti.dt = 0.0;
    ti.dtIsSet = false;
    if ((rc = write_file(folder + "/timeInfo.bin", &ti, sizeof(ti)))) return rc;
    const double N[3] = {s->cfg.phys.N[0], s->cfg.phys.N[1], s->cfg.phys.N[2]};
    if ((rc = write_file(folder + "/domainSize.bin", N, sizeof(N)))) return rc;
    {
        std::ofstream info(folder + "/info.txt");
        info << "# Summary Info\nCurrentTime: 0\nCurrentStep: " << s->steps << "\nDomainSize (N): " << N[0] << ", "
             << N[1] << ", " << N[2] << "\n";
    }
    // native state
    StateHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = 1;
    h.precision = s->st.precision;
    h.dim = s->cfg.dim;
    for (int a = 0; a < 3; ++a) h.extent[a] = s->cfg.extent[a];
    h.steps = s->steps;
    h.ps = s->st.g.ps;
    h.pop_bytes = s->kt.pop_bytes;
    h.aux_bytes = s->kt.aux_bytes;
    h.q = Q;
    h.pop_scale = s->st.pop_scale;
    std::ofstream out(folder + "/clipb_state.bin", std::ios::binary);
    if (!out.is_open()) return fail(CLIPB_E_ARG, "cannot write " + folder + "/clipb_state.bin");
    out.write(reinterpret_cast<const char*>(&h), sizeof(h));
    for (const auto& b : state_buffers(s)) {
        std::vector<char> buf(b.second);
        CLIPB_CUDA(cudaMemcpyAsync(buf.data(), b.first, b.second, cudaMemcpyDeviceToHost, s->stream));
        CLIPB_CUDA(cudaStreamSynchronize(s->stream));
        out.write(buf.data(), (std::streamsize)buf.size());
    }
    return out.good() ? CLIPB_OK : fail(CLIPB_E_ARG, "write failed: " + folder + "/clipb_state.bin");
}

int clipb_load(clipb_solver* s, const char* dir) {
    if (!s || !dir) return fail(CLIPB_E_ARG, "null argument");
    const std::string folder(dir);
    const int Q = s->cfg.dim == 3 ? 19 : 9;
    int rc;
    // CheckPointer::checkDomainSize (CheckPointer.cu:228-246)
    double N[3];
    if ((rc = read_file(folder + "/domainSize.bin", N, sizeof(N)))) return rc;
    for (int a = 0; a < 3; ++a)
        if (N[a] != s->cfg.phys.N[a])
            return fail(CLIPB_E_CONFIG, "checkpoint domain size mismatch at dimension " + std::to_string(a));
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    s->drop_graph();
    const std::string native = folder + "/clipb_state.bin";
    if (std::filesystem::exists(native)) {
        std::ifstream in(native, std::ios::binary);
        StateHeader h{};
        in.read(reinterpret_cast<char*>(&h), sizeof(h));
        if (!in || std::memcmp(h.magic, kMagic, 8) != 0 || h.version != 1)
            return fail(CLIPB_E_ARG, native + " is not a state file of this library");
        if (h.precision != s->st.precision || h.dim != s->cfg.dim || h.ps != s->st.g.ps || h.q != Q ||
            h.pop_bytes != s->kt.pop_bytes || h.aux_bytes != s->kt.aux_bytes || h.pop_scale != s->st.pop_scale)
            return fail(CLIPB_E_CONFIG, "the state in " + native + " was written for another precision or grid");
        for (const auto& b : state_buffers(s)) {
            std::vector<char> buf(b.second);
            in.read(buf.data(), (std::streamsize)buf.size());
            if ((size_t)in.gcount() != buf.size()) return fail(CLIPB_E_ARG, native + " is truncated");
            CLIPB_CUDA(cudaMemcpyAsync(b.first, buf.data(), b.second, cudaMemcpyHostToDevice, s->stream));
            CLIPB_CUDA(cudaStreamSynchronize(s->stream));
        }
        s->steps = h.steps;
        s->initialized = true;
        return CLIPB_OK;
    }
    // the reference's files only: rebuild c and u from the streamed populations
    if (s->fc_bytes)
        return fail(CLIPB_E_STATE, "a free-convect case resumes from clipb_state.bin only: replaying the last step "
                                   "needs the populations of the step before it");
    SimInfo ti{};
    if ((rc = read_file(folder + "/timeInfo.bin", &ti, sizeof(ti)))) return rc;
    if (ti.currentStep < 1) return fail(CLIPB_E_ARG, "a checkpoint of step 0 holds no streamed populations");
    const size_t nodes = (size_t)s->ref_nodes();
    std::vector<double> f(nodes * Q), g(nodes * Q), fp(nodes * Q), gp(nodes * Q), c(nodes), u(nodes * s->cfg.dim, 0.0);
    if ((rc = read_file(folder + "/dev_f.bin", f.data(), f.size() * 8))) return rc;
    if ((rc = read_file(folder + "/dev_g.bin", g.data(), g.size() * 8))) return rc;
    if ((rc = read_file(folder + "/dev_f_post.bin", fp.data(), fp.size() * 8))) return rc;
    if ((rc = read_file(folder + "/dev_g_post.bin", gp.data(), gp.size() * 8))) return rc;
    const int dim = s->cfg.dim;
    auto e = [&](int q, int d) {
        static const int ex2[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1}, ey2[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
        static const int ex3[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
        static const int ey3[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
        static const int ez3[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
        if (dim == 2) return d == 0 ? ex2[q] : ey2[q];
        return d == 0 ? ex3[q] : (d == 1 ? ey3[q] : ez3[q]);
    };
    for (size_t n = 0; n < nodes; ++n) {
        double sc = gp[n * Q];  // kernelMacroscopicg's sum order (NsAllen.cu:516-540)
        for (int q = 1; q < Q; ++q) sc += gp[n * Q + q];
        c[n] = sc;
        for (int d = 0; d < dim; ++d) {
            double j = 0.0;
            for (int q = 0; q < Q; ++q) j += e(q, d) * fp[n * Q + q];
            u[n * dim + d] = j;
        }
    }
    double* d = nullptr;
    const size_t pq = nodes * Q;
    CLIPB_CUDA(cudaMalloc((void**)&d, (2 * pq + nodes + nodes * dim) * sizeof(double)));
    auto upload = [&](size_t off, const std::vector<double>& v) {
        return cudaMemcpyAsync(d + off, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream);
    };
    cudaError_t err = upload(0, f);
    if (err == cudaSuccess) err = upload(pq, g);
    if (err == cudaSuccess) err = upload(2 * pq, c);
    if (err == cudaSuccess) err = upload(2 * pq + nodes, u);
    // dev_f, dev_g are the collision output of the reference's last solve, i.e. the input of
    // libclipb's launch currentStep - 1: set that input, then replay the launch (its pull
    // and sums give c exactly; u uses the rebuilt u as the previous velocity)
    const int b = (ti.currentStep - 1) & 1;
    if (err == cudaSuccess) err = s->kt.set_state(s->st, b, d, d + pq, d + 2 * pq, d + 2 * pq + nodes, s->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s->stream);
    cudaFree(d);
    if (err != cudaSuccess) return fail(CLIPB_E_CUDA, std::string("loading the reference checkpoint: ") + cudaGetErrorString(err));
    s->steps = ti.currentStep - 1;
    s->initialized = true;
    if ((rc = solver_launch_one(s))) return rc;
    CLIPB_CUDA(cudaStreamSynchronize(s->stream));
    return CLIPB_OK;
}

}  // extern "C"
