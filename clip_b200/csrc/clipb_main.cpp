// clipb_run -- host driver with the shape of the reference's main loop (src/main.cu:39-92),
// calling the lattice update only through the C ABI of libclipb.so.
//
//   clipb_run [config.txt] [-resume] [--precision fp64|fp32|fp16] [--steps N] [--report K]
//             [--launch VARIANT SEG] [--vts DIR [--vts-format ascii|binary64|binary32]]
//             [--checkpoint-dir DIR] [--device-init]
//
// Reads the config (default ./config.txt, like the reference) and builds the initial state
// (the initial field on the host like the reference, or with --device-init on the GPU,
// clipb_init_device), or with -resume loads the checkpoint folder (default ./Checkpoint, CheckPointer::load,
// CheckPointer.cu:84-102) and continues from its step.  Then, while the step count is
// below the final step (the config's finalStep, or --steps), it calls clipb_solve and, as
// the reference's loop does after each solve (main.cu:81-89):
//   * every outputInterval steps, with --vts, writes DIR/results_t<step>.vts (queued:
//     clipb_write_vts_async, overlapping the following steps; VTSwriter::writeToFile);
//   * every reportInterval steps (or --report), prints the step, sum(c) and the kinetic
//     energy (that step sums them as it stores the state, clipb_solve_monitored); a NaN
//     monitor stops the run with an error as Reporter::print does (Reporter.cu:124-144);
//   * every checkpointInterval steps, when checkpointCopy is not 0, rotates the checkpoint
//     folders (DIR -> DIR_1 -> ... -> DIR_checkpointCopy, CheckPointer::rotateFolders,
//     CheckPointer.cu:108-138) and saves the state into DIR (clipb_save: the reference's
//     files plus this library's exact state, so a resume continues bit for bit).
// With --vts the fields are also written after the initial state (main.cu:78).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <string>
#include <system_error>

#include "clipb.h"

namespace fs = std::filesystem;

static int die(const char* what) {
    std::fprintf(stderr, "clipb_run: %s: %s\n", what, clipb_last_error());
    return 1;
}

// CheckPointer::rotateFolders: DIR_i -> DIR_{i+1} for i = copies-1 .. 1 (replacing what is
// there), then DIR -> DIR_1, so that the newest checkpoint can be written into DIR.
static bool rotate_folders(const std::string& dir, long long copies) {
    std::error_code ec;
    if (!fs::exists(dir, ec)) return true;
    for (long long i = copies - 1; i >= 1; --i) {
        const std::string from = dir + "_" + std::to_string(i), to = dir + "_" + std::to_string(i + 1);
        if (fs::exists(from, ec)) {
            if (fs::exists(to, ec)) fs::remove_all(to, ec);
            fs::rename(from, to, ec);
            if (ec) return false;
        }
    }
    const std::string first = dir + "_1";
    if (fs::exists(first, ec)) fs::remove_all(first, ec);
    fs::rename(dir, first, ec);
    return !ec;
}

int main(int argc, char** argv) {
    std::string config = "config.txt";
    int precision = CLIPB_FP64;
    long steps = -1, report = -1;
    int variant = -1, seg = 0;
    bool resume = false, device_init = false;
    std::string vts_dir, ck_dir = "Checkpoint";
    int vts_format = CLIPB_VTS_ASCII;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "-resume") {
            resume = true;
        } else if (a == "--device-init") {
            device_init = true;
        } else if (a == "--precision" && i + 1 < argc) {
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
        } else if (a == "--checkpoint-dir" && i + 1 < argc) {
            ck_dir = argv[++i];
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
    long long copies = 0;
    if (clipb_get_checkpoint_copies(s, &copies)) return die("get_checkpoint_copies");
    if (steps < 0) steps = intervals[0] > 0 ? (long)intervals[0] : 1000;
    if (report <= 0) report = intervals[2] > 0 ? (long)intervals[2] : steps;
    const long output = (long)intervals[1], ck_every = (long)intervals[3];
    std::printf("clipb_run: %s  dim=%d  interior=%dx%dx%d  precision=%d  sigma=%.6g tauH=%.6g tauL=%.6g\n",
                config.c_str(), info.dim, info.interior[0], info.interior[1], info.interior[2], precision, params[2],
                params[5], params[6]);
    if (variant >= 0 && clipb_set_launch(s, variant, seg)) return die("set_launch");
    long start = 0;
    if (resume) {
        if (clipb_load(s, ck_dir.c_str())) return die("resume");
        clipb_get_info(s, &info);
        start = (long)info.steps;
        std::printf("clipb_run: resumed from %s at step %ld\n", ck_dir.c_str(), start);
    } else if (device_init ? clipb_init_device(s) : clipb_init(s)) {
        return die("init");
    }
    const bool vts = !vts_dir.empty() && output > 0;
    if (vts && clipb_write_vts_async(s, vts_dir.c_str(), "results", vts_format)) return die("write_vts");
    const double nodes = (double)info.interior[0] * info.interior[1] * info.interior[2];
    const auto t0 = std::chrono::steady_clock::now();
    for (long step = start + 1; step <= steps; ++step) {
        const bool reported = step % report == 0 || step == steps;
        double mass = 0, ke = 0;
        // a reported step sums its monitors as it stores the state (clipb_solve_monitored)
        const int rc = reported ? clipb_solve_monitored(s, 1, &mass, &ke) : clipb_solve(s, 1);
        if (rc && rc != CLIPB_E_DIVERGED) return die("solve");
        if (vts && step % output == 0 && clipb_write_vts_async(s, vts_dir.c_str(), "results", vts_format))
            return die("write_vts");
        if (reported) {
            std::printf("step %ld  sum(c) %.17g  kinetic %.17g\n", step, mass, ke);
            if (rc) return die("monitors");
        }
        if (copies != 0 && ck_every > 0 && step % ck_every == 0) {
            if (!rotate_folders(ck_dir, copies)) {
                std::fprintf(stderr, "clipb_run: cannot rotate the checkpoint folders of %s\n", ck_dir.c_str());
                return 1;
            }
            if (clipb_save(s, ck_dir.c_str())) return die("checkpoint");
            std::printf("clipb_run: checkpoint of step %ld saved in %s\n", step, ck_dir.c_str());
        }
    }
    if (vts && clipb_vts_wait(s)) return die("vts");
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const long ran = steps > start ? steps - start : 0;
    std::printf("clipb_run: %ld steps in %.3f s, %.1f MLUPS (wall clock, including monitor reads and output)\n", ran,
                sec, sec > 0 ? nodes * ran / sec * 1e-6 : 0.0);
    clipb_destroy(s);
    return 0;
}
