// clipb_run -- host driver with the shape of the reference's main loop (src/main.cu:39-92),
// calling the lattice update only through the C ABI of libclipb.so.
//
//   clipb_run [config.txt] [--precision fp64|fp32|fp16] [--steps N] [--report K]
//             [--launch VARIANT SEG] [--vts DIR [--vts-format ascii|binary64|binary32]]
//
// Reads the config (default ./config.txt, like the reference), builds the initial state,
// then for each step calls clipb_solve and, every `report` steps (default: reportInterval
// of the config), prints the step, sum(c) and the kinetic energy; a NaN monitor stops the
// run with an error as Reporter::print does (Reporter.cu:124-144).  The step count
// defaults to the config's finalStep.  With --vts, the fields are written to
// DIR/results_t<step>.vts after the initial state and every outputInterval steps, as
// VTSwriter::writeToFile does in the reference's loop (main.cu:78-86); the writes are
// queued (clipb_write_vts_async) and overlap the following steps.  Checkpoints are not
// part of this driver.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "clipb.h"

static int die(const char* what) {
    std::fprintf(stderr, "clipb_run: %s: %s\n", what, clipb_last_error());
    return 1;
}

int main(int argc, char** argv) {
    std::string config = "config.txt";
    int precision = CLIPB_FP64;
    long steps = -1, report = -1;
    int variant = -1, seg = 0;
    std::string vts_dir;
    int vts_format = CLIPB_VTS_ASCII;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--precision" && i + 1 < argc) {
            const std::string p = argv[++i];
            precision = p == "fp32" ? CLIPB_FP32 : (p == "fp16" ? CLIPB_FP16 : CLIPB_FP64);
        } else if (a == "--steps" && i + 1 < argc) {
            steps = std::atol(argv[++i]);
        } else if (a == "--report" && i + 1 < argc) {
            report = std::atol(argv[++i]);
        } else if (a == "--launch" && i + 2 < argc) {
            variant = std::atoi(argv[++i]);
            seg = std::atoi(argv[++i]);
        } else if (a == "--vts" && i + 1 < argc) {
            vts_dir = argv[++i];
        } else if (a == "--vts-format" && i + 1 < argc) {
            const std::string f = argv[++i];
            vts_format = f == "binary64" ? CLIPB_VTS_BINARY64 : (f == "binary32" ? CLIPB_VTS_BINARY32 : CLIPB_VTS_ASCII);
        } else {
            config = a;
        }
    }
    clipb_solver* s = nullptr;
    if (clipb_create(config.c_str(), precision, &s)) return die("create");
    double params[16];
    clipb_get_params(s, params);
    clipb_info info;
    clipb_get_info(s, &info);
    long long intervals[4] = {0, 0, 0, 0};  // finalStep, outputInterval, reportInterval, checkpointInterval
    if (clipb_get_intervals(s, intervals)) return die("get_intervals");
    if (steps < 0) steps = intervals[0] > 0 ? (long)intervals[0] : 1000;
    if (report <= 0) report = intervals[2] > 0 ? (long)intervals[2] : steps;
    const long output = (long)intervals[1];
    std::printf("clipb_run: %s  dim=%d  interior=%dx%dx%d  precision=%d  sigma=%.6g tauH=%.6g tauL=%.6g\n",
                config.c_str(), info.dim, info.interior[0], info.interior[1], info.interior[2], precision, params[2],
                params[5], params[6]);
    if (variant >= 0 && clipb_set_launch(s, variant, seg)) return die("set_launch");
    if (clipb_init(s)) return die("init");
    const bool vts = !vts_dir.empty() && output > 0;
    if (vts && clipb_write_vts_async(s, vts_dir.c_str(), "results", vts_format)) return die("write_vts");
    const double nodes = (double)info.interior[0] * info.interior[1] * info.interior[2];
    const auto t0 = std::chrono::steady_clock::now();
    for (long step = 1; step <= steps; ++step) {
        if (clipb_solve(s, 1)) return die("solve");
        if (vts && step % output == 0 && clipb_write_vts_async(s, vts_dir.c_str(), "results", vts_format))
            return die("write_vts");
        if (step % report == 0 || step == steps) {
            double mass = 0, ke = 0;
            const int rc = clipb_monitors(s, &mass, &ke);
            std::printf("step %ld  sum(c) %.15g  kinetic %.6e\n", step, mass, ke);
            if (rc) return die("monitors");
        }
    }
    if (vts && clipb_vts_wait(s)) return die("vts");
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("clipb_run: %ld steps in %.3f s, %.1f MLUPS (wall clock, including monitor reads and output)\n", steps, sec,
                nodes * steps / sec * 1e-6);
    clipb_destroy(s);
    return 0;
}
