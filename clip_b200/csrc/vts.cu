// VTS output of a solver's fields (C ABI in include/clipb.h).
//
// The reference's VTSwriter (src/io/VTSwriter.cu:72-205) copies every field to the host on
// every step (DataArray::updateHost) and, when step % outputInterval == 0, writes
// <folder>/<baseName>_t<step>.vts: a VTK XML structured grid over the interior nodes with
// the point arrays Velocity (DIM components), C, P and Rho as Float64 text.
//
// Here one kernel (vts_pack_kernel) packs the interior fields in point order on the
// solver's stream; a dedicated copy stream moves them into pinned host memory after an
// event, and a writer thread formats and writes the file.  The solver's stream carries only
// the pack kernel, so the copy and the file write overlap the following steps.  Two buffers
// are in flight at most: a third write waits for the oldest one.
//
// Formats: the reference's text form (numbers printed as %g with 6 significant digits, as
// its default-formatted std::ofstream prints them), or the same arrays as raw Float64 or
// Float32 in an appended block (VTK XML 1.0, UInt64 block headers).
#include <cuda_runtime.h>
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <filesystem>
#include <fstream>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "clipb.h"
#include "solver.hpp"

namespace clipb {

namespace {

constexpr int kSlots = 2;

// Number formatting of the reference's ofstream (default flags, precision 6).
inline int put_num(char* p, double v) { return std::snprintf(p, 32, "%g", v); }

// Appends the text of points [i0, i1) produced by `row(i, buf) -> length` to `out`,
// formatting slices of the range on `threads` threads.
template <class Row>
void format_rows(long long i0, long long i1, int threads, Row row, std::string& out) {
    const long long n = i1 - i0;
    if (n <= 0) return;
    const int t = (int)std::max<long long>(1, std::min<long long>(threads, n / 4096 + 1));
    std::vector<std::string> parts(t);
    auto work = [&](int k) {
        const long long a = i0 + n * k / t, b = i0 + n * (k + 1) / t;
        std::string& s = parts[k];
        s.reserve((size_t)(b - a) * 16);
        char buf[160];
        for (long long i = a; i < b; ++i) s.append(buf, (size_t)row(i, buf));
    };
    std::vector<std::thread> pool;
    for (int k = 1; k < t; ++k) pool.emplace_back(work, k);
    work(0);
    for (auto& th : pool) th.join();
    for (auto& s : parts) out += s;
}

struct Grid {
    int dim;
    int n[3];   // nodes written per axis (n[2] = 1 in 2D)
    int z1 = 1;  // 3D: global index of the first plane written (a slab's first own plane)
    long long points() const { return (long long)n[0] * n[1] * n[2]; }
    // reference index of point i (x fastest): interior indices start at 1, z = 0 in 2D
    void coords(long long i, long long& x, long long& y, long long& z) const {
        x = 1 + i % n[0];
        y = 1 + (i / n[0]) % n[1];
        z = dim == 3 ? z1 + i / ((long long)n[0] * n[1]) : 0;
    }
    std::string extent() const {
        const std::string zr =
            dim == 3 ? std::to_string(z1) + " " + std::to_string(z1 + n[2] - 1) : std::string("0 0");
        return "1 " + std::to_string(n[0]) + " 1 " + std::to_string(n[1]) + " " + zr;
    }
};

const char* const kScalarNames[3] = {"C", "P", "Rho"};

// The text file of VTSwriter::writeVTSBinaryFile (VTSwriter.cu:100-139).
template <typename V>
bool write_ascii(std::ofstream& f, const Grid& gr, const V* data) {
    const long long nn = gr.points();
    const int threads = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    constexpr long long kBlock = 1 << 22;  // points formatted per write
    f << "<?xml version=\"1.0\"?>\n";
    f << "<VTKFile type=\"StructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
    f << "<StructuredGrid WholeExtent=\"" << gr.extent() << "\">\n";
    f << "<Piece Extent=\"" << gr.extent() << "\">\n";
    f << "<Points>\n<DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    std::string text;
    auto emit = [&](auto row) {
        for (long long b = 0; b < nn; b += kBlock) {
            text.clear();
            format_rows(b, std::min(nn, b + kBlock), threads, row, text);
            f.write(text.data(), (std::streamsize)text.size());
        }
    };
    emit([&](long long i, char* p) {
        long long x, y, z;
        gr.coords(i, x, y, z);
        int k = put_num(p, (double)x);
        p[k++] = ' ';
        k += put_num(p + k, (double)y);
        p[k++] = ' ';
        k += put_num(p + k, (double)z);
        p[k++] = '\n';
        return k;
    });
    f << "</DataArray>\n</Points>\n";
    f << "<PointData Scalars=\"scalars\" Vectors=\"velocity\">\n";
    f << "<DataArray type=\"Float64\" Name=\"Velocity\" NumberOfComponents=\"" << gr.dim << "\" format=\"ascii\">\n";
    emit([&](long long i, char* p) {
        int k = 0;
        for (int d = 0; d < gr.dim; ++d) {
            if (d) p[k++] = ' ';
            k += put_num(p + k, (double)data[i * gr.dim + d]);
        }
        p[k++] = '\n';
        return k;
    });
    f << "</DataArray>\n";
    for (int a = 0; a < 3; ++a) {
        const V* col = data + nn * gr.dim + nn * a;
        f << "<DataArray type=\"Float64\" Name=\"" << kScalarNames[a] << "\" format=\"ascii\">\n";
        emit([&](long long i, char* p) {
            int k = put_num(p, (double)col[i]);
            p[k++] = '\n';
            return k;
        });
        f << "</DataArray>\n";
    }
    f << "</PointData>\n";
    f << "</Piece>\n</StructuredGrid>\n</VTKFile>\n";
    return f.good();
}

// Writes `bytes` at `off` of file descriptor fd (pwrite until done).
bool put_at(int fd, const void* data, size_t bytes, uint64_t off) {
    const char* p = static_cast<const char*>(data);
    while (bytes > 0) {
        const ssize_t w = ::pwrite(fd, p, bytes, (off_t)off);
        if (w <= 0) return false;
        p += w;
        bytes -= (size_t)w;
        off += (uint64_t)w;
    }
    return true;
}

// The same arrays as raw little-endian values in one appended block.  Every offset is known
// in advance, so slices of the points (generated per thread) and of the packed fields are
// written in parallel at their positions.
template <typename V>
bool write_binary(const std::string& path, const Grid& gr, const V* data) {
    const long long nn = gr.points();
    const char* type = sizeof(V) == 8 ? "Float64" : "Float32";
    const uint64_t bytes[5] = {(uint64_t)nn * 3 * sizeof(V), (uint64_t)nn * gr.dim * sizeof(V),
                               (uint64_t)nn * sizeof(V), (uint64_t)nn * sizeof(V), (uint64_t)nn * sizeof(V)};
    uint64_t off[5];
    off[0] = 0;
    for (int a = 1; a < 5; ++a) off[a] = off[a - 1] + sizeof(uint64_t) + bytes[a - 1];
    std::string h;
    h += "<?xml version=\"1.0\"?>\n";
    h += "<VTKFile type=\"StructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n";
    h += "<StructuredGrid WholeExtent=\"" + gr.extent() + "\">\n";
    h += "<Piece Extent=\"" + gr.extent() + "\">\n";
    h += std::string("<Points>\n<DataArray type=\"") + type +
         "\" NumberOfComponents=\"3\" format=\"appended\" offset=\"0\"/>\n</Points>\n";
    h += "<PointData Scalars=\"scalars\" Vectors=\"velocity\">\n";
    h += std::string("<DataArray type=\"") + type + "\" Name=\"Velocity\" NumberOfComponents=\"" +
         std::to_string(gr.dim) + "\" format=\"appended\" offset=\"" + std::to_string(off[1]) + "\"/>\n";
    for (int a = 0; a < 3; ++a)
        h += std::string("<DataArray type=\"") + type + "\" Name=\"" + kScalarNames[a] +
             "\" format=\"appended\" offset=\"" + std::to_string(off[2 + a]) + "\"/>\n";
    h += "</PointData>\n</Piece>\n</StructuredGrid>\n";
    h += "<AppendedData encoding=\"raw\">\n_";
    const std::string tail = "\n</AppendedData>\n</VTKFile>\n";
    const uint64_t base = h.size();
    const uint64_t end = base + off[4] + sizeof(uint64_t) + bytes[4];

    const int fd = ::open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0) return false;
    bool ok = put_at(fd, h.data(), h.size(), 0) && put_at(fd, tail.data(), tail.size(), end);
    for (int a = 0; a < 5 && ok; ++a) ok = put_at(fd, &bytes[a], sizeof(uint64_t), base + off[a]);
    const int threads = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<char> good(threads, 1);
    auto work = [&](int t) {
        // points [p0, p1) of this thread, generated in blocks
        const long long p0 = nn * t / threads, p1 = nn * (t + 1) / threads;
        constexpr long long kBlock = 1 << 16;
        std::vector<V> pts((size_t)kBlock * 3);
        for (long long b = p0; b < p1 && good[t]; b += kBlock) {
            const long long e = std::min(p1, b + kBlock);
            for (long long i = b; i < e; ++i) {
                long long x, y, z;
                gr.coords(i, x, y, z);
                V* q = &pts[(size_t)(i - b) * 3];
                q[0] = (V)x;
                q[1] = (V)y;
                q[2] = (V)z;
            }
            good[t] = put_at(fd, pts.data(), (size_t)(e - b) * 3 * sizeof(V),
                             base + off[0] + sizeof(uint64_t) + (uint64_t)b * 3 * sizeof(V));
        }
        // this thread's slice of the packed fields (Velocity, C, P, Rho back to back)
        const uint64_t total = bytes[1] + bytes[2] + bytes[3] + bytes[4];
        const uint64_t s0 = total * t / threads, s1 = total * (t + 1) / threads;
        uint64_t src = 0;
        for (int a = 1; a < 5 && good[t]; ++a) {
            const uint64_t lo = std::max(s0, src), hi = std::min(s1, src + bytes[a]);
            if (lo < hi)
                good[t] = put_at(fd, reinterpret_cast<const char*>(data) + lo, hi - lo,
                                 base + off[a] + sizeof(uint64_t) + (lo - src));
            src += bytes[a];
        }
    };
    if (ok) {
        std::vector<std::thread> pool;
        for (int t = 1; t < threads; ++t) pool.emplace_back(work, t);
        work(0);
        for (auto& th : pool) th.join();
        for (char g : good) ok = ok && g;
    }
    return (::close(fd) == 0) && ok;
}

}  // namespace

struct VtsQueue {
    struct Slot {
        void* dev = nullptr;
        void* host = nullptr;
        size_t bytes = 0;
        cudaEvent_t copied = nullptr;
        bool busy = false;
    };
    struct Job {
        int slot;
        std::string path;
        int format;
    };
    int device = 0;
    Grid grid{};
    cudaStream_t copy = nullptr;
    cudaEvent_t packed = nullptr;
    Slot slots[kSlots];
    std::mutex m;
    std::condition_variable cv;
    std::deque<Job> jobs;
    int pending = 0;
    bool stop = false;
    std::string error;  // first error of a background write, reported by clipb_vts_wait
    std::thread worker;

    void run() {
        cudaSetDevice(device);
        for (;;) {
            Job job;
            {
                std::unique_lock<std::mutex> lk(m);
                cv.wait(lk, [&] { return stop || !jobs.empty(); });
                if (jobs.empty()) return;
                job = jobs.front();
                jobs.pop_front();
            }
            Slot& sl = slots[job.slot];
            std::string err;
            const cudaError_t e = cudaEventSynchronize(sl.copied);
            if (e != cudaSuccess) {
                err = std::string("device-to-host copy of the fields: ") + cudaGetErrorString(e);
            } else {
                bool ok = false;
                if (job.format == CLIPB_VTS_ASCII) {
                    std::ofstream f(job.path, std::ios::binary);
                    ok = f.is_open() && write_ascii(f, grid, static_cast<const double*>(sl.host));
                    f.close();
                    ok = ok && !f.fail();
                } else if (job.format == CLIPB_VTS_BINARY64) {
                    ok = write_binary(job.path, grid, static_cast<const double*>(sl.host));
                } else {
                    ok = write_binary(job.path, grid, static_cast<const float*>(sl.host));
                }
                if (!ok) err = "Failed to write file: " + job.path;
            }
            {
                std::lock_guard<std::mutex> lk(m);
                if (!err.empty() && error.empty()) error = err;
                sl.busy = false;
                --pending;
            }
            cv.notify_all();
        }
    }

    ~VtsQueue() {
        {
            std::lock_guard<std::mutex> lk(m);
            stop = true;
        }
        cv.notify_all();
        if (worker.joinable()) worker.join();
        for (Slot& sl : slots) {
            if (sl.dev) cudaFree(sl.dev);
            if (sl.host) cudaFreeHost(sl.host);
            if (sl.copied) cudaEventDestroy(sl.copied);
        }
        if (packed) cudaEventDestroy(packed);
        if (copy) cudaStreamDestroy(copy);
    }
};

void vts_release(VtsQueue* q) { delete q; }

}  // namespace clipb

using namespace clipb;

namespace {

int vts_queue(clipb_solver* s, VtsQueue** out) {
    if (!s->vts) {
        auto* q = new VtsQueue();
        s->vts = q;
        CLIPB_CUDA(cudaGetDevice(&q->device));
        q->grid.dim = s->cfg.dim;
        for (int a = 0; a < 3; ++a) q->grid.n[a] = s->st.g.n[a];
        if (s->cfg.dim == 3) {  // the updated planes, at their global z (a slab's own planes)
            q->grid.n[2] = s->st.g.zhi - s->st.g.zlo + 1;
            q->grid.z1 = s->st.g.zlo + s->cfg.zoff;
        }
        CLIPB_CUDA(cudaStreamCreateWithFlags(&q->copy, cudaStreamNonBlocking));
        CLIPB_CUDA(cudaEventCreateWithFlags(&q->packed, cudaEventDisableTiming));
        for (auto& sl : q->slots) CLIPB_CUDA(cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming));
        q->worker = std::thread([q] { q->run(); });
    }
    *out = s->vts;
    return CLIPB_OK;
}

}  // namespace

int clipb_write_vts_async(clipb_solver* s, const char* folder, const char* base_name, int format) {
    if (!s || !folder || !base_name) return fail(CLIPB_E_ARG, "null argument");
    if (!s->initialized) return fail(CLIPB_E_STATE, "write_vts before init");
    if (format != CLIPB_VTS_ASCII && format != CLIPB_VTS_BINARY64 && format != CLIPB_VTS_BINARY32)
        return fail(CLIPB_E_ARG, "unknown VTS format");
    std::error_code ec;
    std::filesystem::create_directories(folder, ec);
    if (ec) return fail(CLIPB_E_ARG, std::string("cannot create ") + folder + ": " + ec.message());
    VtsQueue* q = nullptr;
    int rc = vts_queue(s, &q);
    if (rc) return rc;
    const bool single = format == CLIPB_VTS_BINARY32;
    const size_t bytes = (size_t)q->grid.points() * (q->grid.dim + 3) * (single ? sizeof(float) : sizeof(double));
    int k = -1;
    {
        std::unique_lock<std::mutex> lk(q->m);
        q->cv.wait(lk, [&] { return !q->slots[0].busy || !q->slots[1].busy; });
        k = q->slots[0].busy ? 1 : 0;
        q->slots[k].busy = true;
        ++q->pending;
    }
    VtsQueue::Slot& sl = q->slots[k];
    auto release = [&](int code) {
        {
            std::lock_guard<std::mutex> lk(q->m);
            sl.busy = false;
            --q->pending;
        }
        q->cv.notify_all();
        return code;
    };
    if (sl.bytes < bytes) {
        if (sl.dev) cudaFree(sl.dev);
        if (sl.host) cudaFreeHost(sl.host);
        sl.dev = sl.host = nullptr;
        sl.bytes = 0;
        if (cudaMalloc(&sl.dev, bytes) != cudaSuccess || cudaMallocHost(&sl.host, bytes) != cudaSuccess) {
            cudaGetLastError();
            return release(fail(CLIPB_E_NOMEM, "VTS buffers of " + std::to_string(bytes) + " bytes"));
        }
        sl.bytes = bytes;
    }
    const int last = s->steps > 0 ? (int)((s->steps - 1) & 1) : -1;
    cudaError_t e = s->kt.vts_pack(s->st, last, sl.dev, single, s->stream);
    if (e == cudaSuccess) e = cudaEventRecord(q->packed, s->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(q->copy, q->packed, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sl.host, sl.dev, bytes, cudaMemcpyDeviceToHost, q->copy);
    if (e == cudaSuccess) e = cudaEventRecord(sl.copied, q->copy);
    if (e != cudaSuccess) return release(fail(CLIPB_E_CUDA, std::string("VTS field copy: ") + cudaGetErrorString(e)));
    std::string path = std::string(folder) + "/" + base_name + "_t" + std::to_string(s->steps) + ".vts";
    {
        std::lock_guard<std::mutex> lk(q->m);
        q->jobs.push_back(VtsQueue::Job{k, std::move(path), format});
    }
    q->cv.notify_all();
    return CLIPB_OK;
}

int clipb_vts_wait(clipb_solver* s) {
    if (!s) return fail(CLIPB_E_ARG, "null solver");
    VtsQueue* q = s->vts;
    if (!q) return CLIPB_OK;
    std::string err;
    {
        std::unique_lock<std::mutex> lk(q->m);
        q->cv.wait(lk, [&] { return q->pending == 0; });
        err.swap(q->error);
    }
    return err.empty() ? CLIPB_OK : fail(CLIPB_E_ARG, err);
}

int clipb_write_vts(clipb_solver* s, const char* folder, const char* base_name, int format) {
    const int rc = clipb_write_vts_async(s, folder, base_name, format);
    if (rc) return rc;
    return clipb_vts_wait(s);
}
