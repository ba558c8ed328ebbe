// Test harness around the reference CLIP build (mshadkhah/CLIP), compiled from the
// reference's own sources by oracle/Makefile into oracle/_ref/.  It is test
// infrastructure: it drives the reference's unmodified NSAllen solver through its
// public C++ interface and dumps raw FP64 fields, so the CPU oracle and the CUDA
// product can be pinned to the reference's own results, and it times
// NSAllen::solve() for the reference arm of bench.py.
//
// Call sequence mirrors src/main.cu:53-89 of the reference:
//   InputData -> Domain -> Geometry -> Boundary -> DataArray::createVectors ->
//   NSAllen -> initialCondition -> DataArray::updateDevice -> deviceInitializer ->
//   loop { solve }.
// Differences from the reference's main:
//   * every device buffer is zeroed after createVectors (DataArray.cu:79-121 leaves
//     them uninitialised; KernelInitializeDistributions reads dev_p, NsAllen.cu:159,163);
//   * no checkpoint / report side effects; fields are dumped in binary instead;
//   * --bc SIDE=TYPE[,SIDE=TYPE...] (SIDE x- x+ y- y+ z- z+; TYPE wall, slipwall,
//     freeconvect, neumann, periodic) sets a side's type after the config is parsed and
//     before any solver object reads it: the reference's parser strips every space from a
//     block line (Boundary.cu:282-288) and then looks for "slip wall" and "free convect"
//     (Boundary.cu:57-75), so those types are otherwise unreachable.  The flags isWall,
//     isSlipWall, ... are recomputed from the side types, as Boundary::updateFlags does;
//   * VTS output only with --vts DIR: then the reference's own TimeInfo and VTSwriter
//     (folder DIR, base name "results") run exactly as in main.cu:64,78-86 -- writeToFile
//     after the initial state and after every solve + increment, writing a file whenever
//     the step is a multiple of the config's outputInterval.
//
// Usage:
//   ref_harness CONFIG OUTDIR NSTEPS [--dump s0,s1,...] [--full] [--vts DIR] [--bc SIDE=TYPE,...]
//   ref_harness CONFIG - 0 --time WARMUP STEPS [--mainloop]
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <string>
#include <vector>

#include "Boundary.cuh"
#include "DataArray.cuh"
#include "Domain.cuh"
#include "Geometry.cuh"
#include "InputData.cuh"
#include "NsAllen.cuh"
#include "TimeInfo.cuh"
#include "VTSwriter.cuh"

namespace {

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "ref_harness: %s: %s\n", what, cudaGetErrorString(e));
        std::exit(3);
    }
}

void dump(const std::string& dir, const std::string& name, int step, const double* dev, size_t n) {
    std::vector<double> host(n);
    check(cudaMemcpy(host.data(), dev, n * sizeof(double), cudaMemcpyDeviceToHost), "dump memcpy");
    char path[1024];
    std::snprintf(path, sizeof(path), "%s/%s_%06d.bin", dir.c_str(), name.c_str(), step);
    FILE* fp = std::fopen(path, "wb");
    if (!fp) {
        std::fprintf(stderr, "ref_harness: cannot open %s\n", path);
        std::exit(4);
    }
    std::fwrite(host.data(), sizeof(double), n, fp);
    std::fclose(fp);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s CONFIG OUTDIR NSTEPS [--dump a,b,..] [--full] [--time W K] [--mainloop]\n", argv[0]);
        return 2;
    }
    const std::string config = argv[1];
    const std::string outdir = argv[2];
    const long nsteps = std::atol(argv[3]);
    std::set<long> dumps;
    bool full = false, mainloop = false;
    std::string vts_dir, bc_override;
    long warm = -1, timed = -1;
    for (int a = 4; a < argc; ++a) {
        std::string s = argv[a];
        if (s == "--dump" && a + 1 < argc) {
            std::string list = argv[++a];
            size_t pos = 0;
            while (pos < list.size()) {
                size_t comma = list.find(',', pos);
                if (comma == std::string::npos) comma = list.size();
                dumps.insert(std::atol(list.substr(pos, comma - pos).c_str()));
                pos = comma + 1;
            }
        } else if (s == "--full") {
            full = true;
        } else if (s == "--time" && a + 2 < argc) {
            warm = std::atol(argv[++a]);
            timed = std::atol(argv[++a]);
        } else if (s == "--mainloop") {
            mainloop = true;
        } else if (s == "--vts" && a + 1 < argc) {
            vts_dir = argv[++a];
        } else if (s == "--bc" && a + 1 < argc) {
            bc_override = argv[++a];
        }
    }

    clip::InputData inputData(config);
    clip::Domain simDomain(inputData);
    clip::Geometry geometry(inputData);
    clip::Boundary boundaryConditions(inputData, simDomain);
    if (!bc_override.empty()) {
        using T = clip::Boundary::Type;
        const char* sides[6] = {"x-", "x+", "y-", "y+", "z-", "z+"};
        size_t pos = 0;
        while (pos < bc_override.size()) {
            size_t comma = bc_override.find(',', pos);
            if (comma == std::string::npos) comma = bc_override.size();
            const std::string item = bc_override.substr(pos, comma - pos);
            pos = comma + 1;
            const size_t eq = item.find('=');
            const std::string side = item.substr(0, eq), type = eq == std::string::npos ? "" : item.substr(eq + 1);
            int si = -1;
            for (int k = 0; k < 6; ++k)
                if (side == sides[k]) si = k;
            T t = T::Unknown;
            if (type == "wall") t = T::Wall;
            else if (type == "slipwall") t = T::SlipWall;
            else if (type == "freeconvect") t = T::FreeConvect;
            else if (type == "neumann") t = T::Neumann;
            else if (type == "periodic") t = T::Periodic;
            if (si < 0 || t == T::Unknown) {
                std::fprintf(stderr, "ref_harness: bad --bc item %s\n", item.c_str());
                return 2;
            }
            boundaryConditions.BCMap.types[si] = t;
        }
        auto& b = boundaryConditions;
        b.isWall = b.isSlipWall = b.isFreeConvect = b.isNeumann = b.isPeriodic = b.isVelocity = false;
        for (int k = 0; k < 2 * DIM; ++k) {
            switch (b.BCMap.types[k]) {
                case T::Wall: b.isWall = true; break;
                case T::SlipWall: b.isSlipWall = true; break;
                case T::FreeConvect: b.isFreeConvect = true; break;
                case T::Neumann: b.isNeumann = true; break;
                case T::Periodic: b.isPeriodic = true; break;
                case T::Velocity: b.isVelocity = true; break;
                default: break;
            }
        }
    }
    clip::DataArray dataArray(inputData, simDomain, boundaryConditions);
    dataArray.createVectors();

    constexpr unsigned Q = clip::WMRT::WMRTvelSet::Q;
    const size_t n = simDomain.domainSize;
    auto& d = dataArray.deviceDA;
    double* scal[] = {d.dev_rho, d.dev_mu, d.dev_c, d.dev_p};
    for (double* p : scal) check(cudaMemset(p, 0, n * sizeof(double)), "memset scalar");
    double* vec[] = {d.dev_vel, d.dev_dc, d.dev_normal};
    for (double* p : vec) check(cudaMemset(p, 0, n * DIM * sizeof(double)), "memset vector");
    double* pops[] = {d.dev_f, d.dev_g, d.dev_f_post, d.dev_g_post};
    for (double* p : pops) check(cudaMemset(p, 0, n * Q * sizeof(double)), "memset populations");
    check(cudaDeviceSynchronize(), "memset sync");

    clip::NSAllen nsSolver(inputData, simDomain, dataArray, boundaryConditions, geometry);
    nsSolver.initialCondition();
    dataArray.updateDevice();
    nsSolver.deviceInitializer();
    check(cudaDeviceSynchronize(), "init");

    auto dump_all = [&](long step) {
        dump(outdir, "c", (int)step, d.dev_c, n);
        dump(outdir, "p", (int)step, d.dev_p, n);
        dump(outdir, "rho", (int)step, d.dev_rho, n);
        dump(outdir, "vel", (int)step, d.dev_vel, n * DIM);
        if (full) {
            dump(outdir, "f", (int)step, d.dev_f, n * Q);
            dump(outdir, "g", (int)step, d.dev_g, n * Q);
            dump(outdir, "f_post", (int)step, d.dev_f_post, n * Q);
            dump(outdir, "g_post", (int)step, d.dev_g_post, n * Q);
            dump(outdir, "mu", (int)step, d.dev_mu, n);
            dump(outdir, "dc", (int)step, d.dev_dc, n * DIM);
            dump(outdir, "normal", (int)step, d.dev_normal, n * DIM);
        }
    };

    if (warm >= 0) {
        // Timing mode: NSAllen::solve() alone, or the stock main-loop body
        // (solve + DataArray::updateHost, as VTSwriter::writeToFile does every step).
        for (long s = 0; s < warm; ++s) {
            nsSolver.solve();
            if (mainloop) dataArray.updateHost();
        }
        check(cudaDeviceSynchronize(), "warmup");
        cudaEvent_t e0, e1;
        check(cudaEventCreate(&e0), "event");
        check(cudaEventCreate(&e1), "event");
        check(cudaEventRecord(e0, 0), "record");
        for (long s = 0; s < timed; ++s) {
            nsSolver.solve();
            if (mainloop) dataArray.updateHost();
        }
        check(cudaEventRecord(e1, 0), "record");
        check(cudaEventSynchronize(e1), "sync");
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        check(cudaGetLastError(), "solve");
        const auto& info = simDomain.info;
        double interior = 1.0;
        for (int a = 0; a < DIM; ++a) interior *= double(info.domainMaxIdx[a] - info.domainMinIdx[a] + 1);
        const double sec = ms * 1e-3;
        std::printf("{\"ref_timing\": true, \"dim\": %d, \"interior_nodes\": %.0f, \"steps\": %ld, \"warmup\": %ld, "
                    "\"ms_total\": %.6f, \"ms_per_step\": %.6f, \"mlups\": %.6f, \"mainloop\": %s}\n",
                    DIM, interior, timed, warm, (double)ms, (double)ms / double(timed > 0 ? timed : 1),
                    interior * double(timed) / sec * 1e-6, mainloop ? "true" : "false");
        return 0;
    }

    clip::TimeInfo timeInfo(inputData);
    clip::VTSwriter vtsWriter(dataArray, inputData, simDomain, timeInfo, vts_dir.empty() ? "results" : vts_dir,
                              "results");
    if (!vts_dir.empty()) vtsWriter.writeToFile();
    if (dumps.count(0)) dump_all(0);
    for (long s = 1; s <= nsteps; ++s) {
        nsSolver.solve();
        timeInfo.increment();
        if (!vts_dir.empty()) vtsWriter.writeToFile();
        if (dumps.count(s)) {
            check(cudaDeviceSynchronize(), "solve");
            dump_all(s);
        }
    }
    check(cudaDeviceSynchronize(), "final");
    check(cudaGetLastError(), "final error");
    std::printf("ref_harness: done dim=%d extent=%u,%u,%u steps=%ld\n", DIM, simDomain.info.extent[0],
                simDomain.info.extent[1], simDomain.info.extent[2], nsteps);
    return 0;
}
