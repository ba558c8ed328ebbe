// Host-side case description: config.txt -> parameters, boundary map, geometry table.
//
// Keeps the reference's config.txt format and parse rules so existing CLIP inputs run
// unchanged:
//   * scalar keys: first "key = value" line anywhere in the file (InputData.cu:284-320)
//   * arrays "[a, b, c]" (InputData.cu:144-210), case names lower-cased (InputData.cu:412-426)
//   * boundary = [ {side, type, value} ... ] blocks (Boundary.cu:146-279)
//   * geometry = [ {type, center, length, radius, amplitude, id} ... ] (Geometry.cu:72-182)
//   * derived physics: sigma, mu, tau, kappa, beta per case (InputData.cu:76-114)
#pragma once

#include <math.h>
#include <cmath>

#include <string>
#include <vector>

#ifdef __CUDACC__
#define CLIPB_HD __host__ __device__
#else
#define CLIPB_HD
#endif

namespace clipb {

enum CaseType { kBubble = 0, kDrop = 1, kRTI = 2, kJet = 3, kUnknownCase = 4 };
enum BCType { kWall = 0, kSlipWall = 1, kFreeConvect = 2, kPeriodic = 3, kNeumann = 4, kVelocity = 5,
              kDoNothing = 6, kUnknownBC = 7,
              kExchange = 8,    // a z face of a slab inside the case (not a config type)
              kWrap = 9 };      // a z face of a slab on a periodic z boundary (not a config type)
enum SideId { kXMinus = 0, kXPlus = 1, kYMinus = 2, kYPlus = 3, kZMinus = 4, kZPlus = 5, kUnknownSide = 6 };
enum GeoType { kCircle = 0, kSphere = 1, kSquare = 2, kCube = 3, kPerturbation = 4, kUnknownGeo = 5 };

constexpr int kMaxGeometries = 16;  // MAX_GEOMETRIES, Geometry.cuh:27

struct Physics {
    double N[3] = {0, 0, 0};
    double referenceLength = 0, referenceVelocity = 0;
    double Re = 0, We = 0, Pe = 0, Ca = 0;
    double rhoRatio = 0, muRatio = 0;
    double gravity[3] = {0, 0, 0};
    double interfaceWidth = 0, mobility = 0;
    int caseType = kUnknownCase;
    double RhoH = 0, RhoL = 0, sigma = 0, betaConstant = 0, kConstant = 0;
    double tauL = 0, tauH = 0, muL = 0, muH = 0, amplitude = 0;
    long finalStep = 0, reportInterval = 0, outputInterval = 0, checkpointInterval = 0, checkpointCopy = 0;
};

struct Boundaries {
    int type[7] = {kUnknownBC, kUnknownBC, kUnknownBC, kUnknownBC, kUnknownBC, kUnknownBC, kUnknownBC};
    double value[7][3] = {};
    bool isPeriodic = false, isWall = false, isSlipWall = false, isFreeConvect = false, isNeumann = false,
         isVelocity = false;
};

// Geometry pool, layout-compatible in meaning with Geometry::GeometryDevice (Geometry.cuh:81-90).
struct GeometryTable {
    int n = 0;
    int type[kMaxGeometries] = {};
    double center[kMaxGeometries][3] = {};
    double length[kMaxGeometries][3] = {};
    double radius[kMaxGeometries] = {};
    double amplitude[kMaxGeometries] = {};
    int id[kMaxGeometries] = {};
};

struct CaseConfig {
    std::string path;
    int dim = 2;
    int extent[3] = {1, 1, 1};    // ghosted extent, reference convention (Domain.cu:26-81)
    int interior[3] = {1, 1, 1};  // interior node counts
    Physics phys;
    Boundaries bc;
    GeometryTable geo;
    // z slab of a larger 3D case (clipb_slab_create): local plane z is global plane z + zoff
    // of the zglobal interior planes; planes zlo .. zhi are updated, the others are filled
    // from the neighbouring slabs.  zglobal = 0: the whole case (zlo = 1, zhi = interior[2]).
    int zoff = 0, zglobal = 0, zlo = 1, zhi = 0;
};

// Parse and validate; throws std::runtime_error with a message on failure.
CaseConfig load_config(const std::string& path);
// The same from the text of a config file (`name` labels messages).
CaseConfig load_config_text(const std::string& text, const std::string& name);

// Signed distance to geometry `id` (Geometry.cuh:102-161); 1e10 if no geometry has that
// id.  Positive outside, negative inside.  Used on the host for the initial phase field
// and on the device for the velocity-inlet mask, as in the reference.
CLIPB_HD inline double signed_distance(const GeometryTable& g, int id, double x, double y, double z, int dim) {
    for (int i = 0; i < g.n; ++i) {
        if (g.id[i] != id) continue;
        switch (g.type[i]) {
            case kCircle: {
                const double dx = x - g.center[i][0], dy = y - g.center[i][1];
                return sqrt(dx * dx + dy * dy) - g.radius[i];
            }
            case kSphere: {
                const double dx = x - g.center[i][0], dy = y - g.center[i][1], dz = z - g.center[i][2];
                return sqrt(dx * dx + dy * dy + dz * dz) - g.radius[i];
            }
            case kSquare: {
                const double dx = fabs(x - g.center[i][0]) - g.length[i][0] * 0.5;
                const double dy = fabs(y - g.center[i][1]) - g.length[i][1] * 0.5;
                const double ax = dx < 0.0 ? 0.0 : dx, ay = dy < 0.0 ? 0.0 : dy;
                const double m = dx < dy ? dy : dx;
                return sqrt(ax * ax + ay * ay) + (m < 0.0 ? m : 0.0);
            }
            case kCube: {
                const double dx = fabs(x - g.center[i][0]) - g.length[i][0] * 0.5;
                const double dy = fabs(y - g.center[i][1]) - g.length[i][1] * 0.5;
                const double dz = fabs(z - g.center[i][2]) - g.length[i][2] * 0.5;
                const double ax = dx < 0.0 ? 0.0 : dx, ay = dy < 0.0 ? 0.0 : dy, az = dz < 0.0 ? 0.0 : dz;
                const double mxy = dx < dy ? dy : dx;
                const double m = mxy < dz ? dz : mxy;
                return sqrt(ax * ax + ay * ay + az * az) + (m < 0.0 ? m : 0.0);
            }
            case kPerturbation: {
                const double L = g.length[i][0];
                const double wave = dim == 2 ? cos(2.0 * M_PI * x / L) : (cos(2.0 * M_PI * x / L) + cos(2.0 * M_PI * z / L));
                return y - (g.amplitude[i] * L * wave + g.center[i][1]);
            }
            default:
                break;
        }
    }
    return 1e10;
}

// Bound of signed_distance to geometry `id` over the x-row x in [x_lo, x_hi] at (y, z):
// +1 if every point of the row is at least `d` outside, -1 if every point is at least `d`
// inside, 0 if the bounds cannot tell.  Conservative: a row reported +1 or -1 has
// |signed_distance| >= d at each of its points.
inline int row_distance_sign(const GeometryTable& g, int id, double x_lo, double x_hi, double y, double z, int dim,
                             double d) {
    for (int i = 0; i < g.n; ++i) {
        if (g.id[i] != id) continue;
        const double fx = std::fmax(std::fabs(x_lo - g.center[i][0]), std::fabs(x_hi - g.center[i][0]));
        switch (g.type[i]) {
            case kCircle:
            case kSphere: {
                const double dy = y - g.center[i][1], dz = g.type[i] == kSphere ? z - g.center[i][2] : 0.0;
                const double D = std::sqrt(dy * dy + dz * dz);  // distance of the row from the centre
                if (D - g.radius[i] >= d) return 1;
                if (std::sqrt(fx * fx + D * D) - g.radius[i] <= -d) return -1;
                return 0;
            }
            case kSquare:
            case kCube: {
                const double dy = std::fabs(y - g.center[i][1]) - g.length[i][1] * 0.5;
                const double dz = g.type[i] == kCube ? std::fabs(z - g.center[i][2]) - g.length[i][2] * 0.5 : -1e300;
                if (std::fmax(dy, dz) >= d) return 1;
                if (fx - g.length[i][0] * 0.5 <= -d && dy <= -d && (g.type[i] == kSquare || dz <= -d)) return -1;
                return 0;
            }
            case kPerturbation: {
                const double reach = std::fabs(g.amplitude[i] * g.length[i][0]) * (dim == 2 ? 1.0 : 2.0);
                if (y - g.center[i][1] - reach >= d) return 1;
                if (y - g.center[i][1] + reach <= -d) return -1;
                return 0;
            }
            default:
                return 0;
        }
    }
    return 1;  // no geometry: signed_distance is 1e10 everywhere
}

}  // namespace clipb
