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

#include <string>
#include <vector>

namespace clipb {

enum CaseType { kBubble = 0, kDrop = 1, kRTI = 2, kJet = 3, kUnknownCase = 4 };
enum BCType { kWall = 0, kSlipWall = 1, kFreeConvect = 2, kPeriodic = 3, kNeumann = 4, kVelocity = 5,
              kDoNothing = 6, kUnknownBC = 7 };
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
    long finalStep = 0, reportInterval = 0, outputInterval = 0;
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
};

// Parse and validate; throws std::runtime_error with a message on failure.
CaseConfig load_config(const std::string& path);

// Signed distance to geometry `id` (Geometry.cuh:102-161); 1e10 if absent.
double signed_distance(const GeometryTable& g, int id, double x, double y, double z, int dim);

}  // namespace clipb
