// clipb_run -- host driver with the shape of the reference's main loop (src/main.cu:39-92),
// calling the lattice update only through the C ABI of libclipb.so.
//
//   clipb_run [config.txt] [--precision fp64|fp32|fp16] [--steps N] [--report K]
//             [--launch VARIANT SEG]
//
// Reads the config (default ./config.txt, like the reference), builds the initial state,
// then for each step calls clipb_solve and, every `report` steps (default: reportInterval
// of the config), prints the step, sum(c) and the kinetic energy; a NaN monitor stops the
// run with an error as Reporter::print does (Reporter.cu:124-144).  Field output (VTS) and
// checkpoints are not part of this driver.
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
    if (steps < 0) {
        // finalStep of the config is not exposed through the ABI: default to 1000 steps
        steps = 1000;
    }
    if (report <= 0) report = steps;
    std::printf("clipb_run: %s  dim=%d  interior=%dx%dx%d  precision=%d  sigma=%.6g tauH=%.6g tauL=%.6g\n",
                config.c_str(), info.dim, info.interior[0], info.interior[1], info.interior[2], precision, params[2],
                params[5], params[6]);
    if (variant >= 0 && clipb_set_launch(s, variant, seg)) return die("set_launch");
    if (clipb_init(s)) return die("init");
    const double nodes = (double)info.interior[0] * info.interior[1] * info.interior[2];
    const auto t0 = std::chrono::steady_clock::now();
    for (long step = 1; step <= steps; ++step) {
        if (clipb_solve(s, 1)) return die("solve");
        if (step % report == 0 || step == steps) {
            double mass = 0, ke = 0;
            const int rc = clipb_monitors(s, &mass, &ke);
            std::printf("step %ld  sum(c) %.15g  kinetic %.6e\n", step, mass, ke);
            if (rc) return die("monitors");
        }
    }
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("clipb_run: %ld steps in %.3f s, %.1f MLUPS (wall clock, including monitor reads)\n", steps, sec,
                nodes * steps / sec * 1e-6);
    clipb_destroy(s);
    return 0;
}
