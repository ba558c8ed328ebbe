// Test program: for every x-row that row_distance_sign (clip_b200/csrc/config.hpp) reports as
// saturated, every node of the row has the value the per-node initial field gives
// (NSAllen::initialCondition, NsAllen.cu:768-824: c = 1/2 +- 1/2 tanh(2 sd / W), with tanh
// taken as +-1 where |2 sd / W| >= 22, as clipb_init evaluates it).  Prints one line per
// config and exits non-zero if any reported row holds another value.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "config.hpp"

using namespace clipb;

static double profile(const CaseConfig& c, double t) {
    const int ct = c.phys.caseType;
    if (ct == kBubble) return 0.50 + 0.50 * t;
    if (ct == kDrop || ct == kJet) return 0.50 - 0.50 * t;
    if (ct == kRTI) return 0.5 + 0.5 * t;
    return 0.0;
}

static double node_value(const CaseConfig& c, int i, int j, int k) {
    const double z = c.dim == 3 ? (double)(k + c.zoff) : 0.0;
    const double sd = signed_distance(c.geo, 0, (double)i, (double)j, z, c.dim);
    const double a = 2.0 * sd / c.phys.interfaceWidth;
    return profile(c, a >= 22.0 ? 1.0 : (a <= -22.0 ? -1.0 : std::tanh(a)));
}

int main(int argc, char** argv) {
    int bad_total = 0;
    for (int f = 1; f < argc; ++f) {
        const CaseConfig c = load_config(argv[f]);
        const double d = 11.0 * c.phys.interfaceWidth * (1.0 + 1e-9) + 1e-9;
        long long rows = 0, reported = 0, bad = 0;
        for (int k = 0; k < c.extent[2]; ++k)
            for (int j = 0; j < c.extent[1]; ++j) {
                ++rows;
                const double z = c.dim == 3 ? (double)(k + c.zoff) : 0.0;
                const int sgn = row_distance_sign(c.geo, 0, 0.0, c.extent[0] - 1.0, (double)j, z, c.dim, d);
                if (!sgn) continue;
                ++reported;
                const double v = profile(c, sgn > 0 ? 1.0 : -1.0);
                for (int i = 0; i < c.extent[0]; ++i) {
                    const double w = node_value(c, i, j, k);
                    if (std::memcmp(&w, &v, sizeof(double))) {
                        ++bad;
                        break;
                    }
                }
            }
        std::printf("%s rows %lld reported %lld wrong %lld\n", argv[f], rows, reported, bad);
        bad_total += (int)bad;
    }
    return bad_total ? 1 : 0;
}
