// CPU oracle for the CLIP per-timestep lattice update -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++17 FP64 restatement (host threads via std::thread) of the reference (mshadkhah/CLIP) two-phase
// Allen-Cahn + weighted-MRT lattice Boltzmann step.  It keeps the reference's own data
// layout (ghosted extent, AoS, x slowest, component fastest: include/domain/Domain.cuh:63-68)
// and its kernel sequence (src/equation/NsAllen.cu:881-892), one loop nest per reference
// kernel, with the same expression trees.  It is built with -ffp-contract=off so that
// every product and sum is rounded separately.
//
// Only tests/, the smoke check and bench.py's CPU-baseline leg use it.  The product
// (clip_b200/) never links or calls it.
//
// Parity pin: tests/golden/*.npz hold dumps of the reference's own FP64 CUDA build
// (oracle/ref_harness.cu, run on a B200); tests/test_oracle_golden.py checks this
// restatement against them.
//
// Deliberate, documented deviations from the reference:
//  * the periodic ghost copy (Solver.cu:75-141) runs as three sequential passes (x, then
//    y, then z), so the edge/corner ghosts of a doubly periodic box hold the true periodic
//    image; in the reference those cells are written concurrently by different threads;
//  * buffers start at zero (the reference reads uninitialised dev_p in
//    NsAllen.cu:159,163; its harness zeroes every buffer the same way);
//  * the boundary types "free convect" and "slip wall" are reachable: the reference's
//    parser strips every space from a block line (Boundary.cu:282-288) and then matches
//    the spaced names (Boundary.cu:57-75), so it can never produce them; here the
//    unspaced forms "freeconvect" / "slipwall" match too;
//  * the free-convect and Neumann passes read the populations of the neighbour node as
//    they were before the pass (a snapshot); the reference reads them in place, which is
//    the same wherever no two sides of one of these types meet;
//  * do-nothing and unknown sides, a slip wall without a wall side (the reference then
//    skips the bounce-back of every slip wall, Solver.cu:1000-1004), two adjacent
//    free-convect or two adjacent Neumann sides (its threads race on the edge nodes) are
//    rejected at create time;
//  * case 'jet' has no body force (the reference leaves its force array uninitialised,
//    NsAllen.cu:460-474).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

// Host threads used by every loop nest: CLIP_ORACLE_THREADS, else all hardware threads.
int n_threads() {
    static int n = [] {
        const char* e = std::getenv("CLIP_ORACLE_THREADS");
        int v = e ? std::atoi(e) : (int)std::thread::hardware_concurrency();
        return v > 0 ? v : 1;
    }();
    return n;
}

// Static block partition of [0, n) over the host threads.
template <class F>
void parallel_for(long n, F&& fn) {
    const int T = (int)std::min<long>(n_threads(), std::max<long>(n, 1));
    if (T <= 1) {
        for (long i = 0; i < n; ++i) fn(i);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(T);
    for (int t = 0; t < T; ++t) {
        const long a = n * t / T, b = n * (t + 1) / T;
        pool.emplace_back([a, b, &fn] {
            for (long i = a; i < b; ++i) fn(i);
        });
    }
    for (auto& th : pool) th.join();
}

enum CaseType { Bubble = 0, Drop = 1, RTI = 2, Jet = 3, UnknownCase = 4 };
enum BCType { Wall = 0, SlipWall = 1, FreeConvect = 2, Periodic = 3, Neumann = 4, Velocity = 5, DoNothing = 6, UnknownBC = 7 };
enum Side { XMinus = 0, XPlus = 1, YMinus = 2, YPlus = 3, ZMinus = 4, ZPlus = 5, UnknownSide = 6 };
enum GeoType { Circle = 0, Sphere = 1, Square = 2, Cube = 3, Perturbation = 4, UnknownGeo = 5 };

// ---------------------------------------------------------------- config parsing
// Restates src/input/InputData.cu:57-115,144-210,284-338 (scalar/array readers and
// the case-dependent derivation of sigma, mu, tau, kappa, beta).
struct Params {
    double N[3] = {0, 0, 0};
    double referenceLength = 0, referenceVelocity = 0, Re = 0, We = 0, Pe = 0, Ca = 0;
    double rhoRatio = 0, muRatio = 0, gravity[3] = {0, 0, 0}, interfaceWidth = 0, mobility = 0;
    int caseType = UnknownCase;
    double RhoH = 0, RhoL = 0, sigma = 0, betaConstant = 0, kConstant = 0, tauL = 0, tauH = 0, muL = 0, muH = 0,
           amplitude = 0;
};

void trim_ends(std::string& s) {  // InputData::trim (InputData.cu:326-338)
    size_t a = s.find_first_not_of(" \t"), b = s.find_last_not_of(" \t");
    if (a == std::string::npos) s.clear();
    else s = s.substr(a, b - a + 1);
}

void strip_all(std::string& s) {  // Boundary::trim / Geometry::trim (Boundary.cu:282-288)
    s.erase(std::remove_if(s.begin(), s.end(), [](unsigned char c) { return c == ' ' || c == '\t' || c == '\r'; }),
            s.end());
}

std::string lower(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    return s;
}

bool find_value(const std::string& file, const std::string& key, std::string& out) {
    std::ifstream in(file);
    if (!in.is_open()) throw std::runtime_error("cannot open config file: " + file);
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        size_t pos = line.find('=');
        if (pos == std::string::npos) continue;
        std::string k = line.substr(0, pos), v = line.substr(pos + 1);
        trim_ends(k);
        trim_ends(v);
        if (k == key) {
            out = v;
            return true;
        }
    }
    return false;
}

void read_real(const std::string& file, const char* key, double& var) {
    std::string v;
    if (find_value(file, key, v)) {
        std::istringstream iss(v);
        iss >> var;
    }
}

void read_array3(const std::string& file, const char* key, double (&arr)[3]) {
    std::string v;
    if (!find_value(file, key, v)) return;
    arr[0] = arr[1] = arr[2] = 0.0;
    v.erase(std::remove(v.begin(), v.end(), '['), v.end());
    v.erase(std::remove(v.begin(), v.end(), ']'), v.end());
    std::stringstream ss(v);
    std::string tok;
    int n = 0;
    while (std::getline(ss, tok, ',') && n < 3) {
        trim_ends(tok);
        arr[n++] = std::stod(tok);
    }
}

Params read_params(const std::string& file) {
    Params p;
    std::string cs;
    if (find_value(file, "case", cs)) {
        std::istringstream iss(cs);
        std::string w;
        iss >> w;
        w = lower(w);
        if (w == "drop") p.caseType = Drop;
        else if (w == "bubble") p.caseType = Bubble;
        else if (w == "jet") p.caseType = Jet;
        else if (w == "rti") p.caseType = RTI;
        else throw std::runtime_error("Unknown case type: " + w);
    }
    read_array3(file, "N", p.N);
    read_real(file, "referenceLength", p.referenceLength);
    read_real(file, "interfaceWidth", p.interfaceWidth);
    read_array3(file, "gravity", p.gravity);
    read_real(file, "mobility", p.mobility);
    read_real(file, "muRatio", p.muRatio);
    read_real(file, "rhoRatio", p.rhoRatio);
    read_real(file, "amplitude", p.amplitude);
    p.RhoH = 1.0;
    p.RhoL = p.RhoH / p.rhoRatio;
    const double gy = std::fabs(p.gravity[1]);
    if (p.caseType == Bubble || p.caseType == Drop) {
        read_real(file, "We", p.We);
        read_real(file, "Re", p.Re);
        p.sigma = (p.RhoH * gy * p.referenceLength * p.referenceLength) / p.We;
        p.muH = std::sqrt(gy * p.RhoH * (p.RhoH - p.RhoL) * p.referenceLength * p.referenceLength * p.referenceLength) / p.Re;
    } else if (p.caseType == RTI) {
        read_real(file, "Ca", p.Ca);
        read_real(file, "Pe", p.Pe);
        read_real(file, "Re", p.Re);
        p.muH = (p.RhoH * std::sqrt(gy * p.referenceLength) * p.referenceLength) / p.Re;
        p.sigma = (p.muH * std::sqrt(gy * p.referenceLength)) / p.Ca;
        p.mobility = (std::sqrt(gy * p.referenceLength) * p.referenceLength) / p.Pe;
    } else if (p.caseType == Jet) {
        read_real(file, "We", p.We);
        read_real(file, "Re", p.Re);
        read_real(file, "referenceVelocity", p.referenceVelocity);
        p.sigma = (p.RhoH * p.referenceVelocity * p.referenceVelocity * p.referenceLength) / p.We;
        p.muH = (p.RhoH * p.referenceVelocity * p.referenceLength) / p.Re;
    }
    p.muL = p.muH / p.muRatio;
    p.tauH = 3.0 * (p.muH / p.RhoH);
    p.tauL = 3.0 * (p.muL / p.RhoL);
    p.kConstant = 1.50 * p.sigma * p.interfaceWidth;
    p.betaConstant = 8.0 * p.sigma / p.interfaceWidth;
    return p;
}

// Boundary list, restating src/boundary/Boundary.cu:146-279,291-319.
struct BCMap {
    int types[7] = {UnknownBC, UnknownBC, UnknownBC, UnknownBC, UnknownBC, UnknownBC, UnknownBC};
    double val[7][3] = {};
    bool isPeriodic = false, isWall = false, isSlipWall = false, isFreeConvect = false, isNeumann = false,
         isVelocity = false;
};

int side_from(const std::string& s) {
    std::string l = lower(s);
    if (l == "x-") return XMinus;
    if (l == "x+") return XPlus;
    if (l == "y-") return YMinus;
    if (l == "y+") return YPlus;
    if (l == "z-") return ZMinus;
    if (l == "z+") return ZPlus;
    return UnknownSide;
}

int bctype_from(const std::string& s) {
    std::string l = lower(s);
    if (l == "wall") return Wall;
    if (l == "slip wall") return SlipWall;
    if (l == "free convect") return FreeConvect;
    if (l == "periodic") return Periodic;
    if (l == "neumann") return Neumann;
    if (l == "velocity") return Velocity;
    if (l == "do nothing") return DoNothing;
    // reachable forms of the names that the reference's space stripping hides
    if (l == "slipwall") return SlipWall;
    if (l == "freeconvect") return FreeConvect;
    return UnknownBC;
}

void parse_list(std::string v, double* out, int maxn) {
    if (!v.empty() && v.front() == '[') v.erase(0, 1);
    if (!v.empty() && v.back() == ']') v.pop_back();
    std::stringstream ss(v);
    std::string tok;
    int n = 0;
    while (std::getline(ss, tok, ',') && n < maxn) {
        strip_all(tok);
        out[n++] = std::stod(tok);
    }
}

BCMap read_boundaries(const std::string& file, int dim) {
    BCMap m;
    struct Entry {
        int side = UnknownSide, type = UnknownBC;
    };
    std::vector<Entry> entries(20);
    int count = 0;
    std::ifstream in(file);
    if (!in.is_open()) throw std::runtime_error("cannot open config file: " + file);
    std::string line;
    bool inList = false, inBlock = false;
    Entry cur;
    while (std::getline(in, line)) {
        strip_all(line);
        if (line.empty() || line[0] == '#') continue;
        if (!inList && line.find("boundary") != std::string::npos && line.find('=') != std::string::npos) {
            inList = true;
            continue;
        }
        if (!inList) continue;
        if (line == "[") continue;
        if (line == "{") {
            inBlock = true;
            cur = Entry{};
            continue;
        }
        if (line == "}" || line == "},") {
            inBlock = false;
            entries[(size_t)cur.side] = cur;
            count++;
            continue;
        }
        if (!inBlock) continue;
        size_t pos = line.find('=');
        if (pos == std::string::npos) continue;
        std::string k = line.substr(0, pos), v = line.substr(pos + 1);
        v.erase(std::remove(v.begin(), v.end(), '"'), v.end());
        if (k == "side") cur.side = side_from(v);
        else if (k == "type") {
            cur.type = bctype_from(v);
            m.types[cur.side] = cur.type;
        } else if (k == "value") {
            double tmp[3] = {0, 0, 0};
            int before = 0;
            (void)before;
            std::string vv = v;
            if (!vv.empty() && vv.front() == '[') vv.erase(0, 1);
            if (!vv.empty() && vv.back() == ']') vv.pop_back();
            std::stringstream ss(vv);
            std::string tok;
            int n = 0;
            while (std::getline(ss, tok, ',') && n < 3) {
                tmp[n] = std::stod(tok);
                m.val[cur.side][n] = tmp[n];
                n++;
            }
        }
    }
    std::set<int> found;
    for (auto& e : entries) found.insert(e.side);
    std::string missing;
    const int nsides = dim == 3 ? 6 : 4;
    static const char* names[] = {"x-", "x+", "y-", "y+", "z-", "z+"};
    for (int s = 0; s < nsides; ++s)
        if (!found.count(s)) missing += std::string(missing.empty() ? "" : ", ") + names[s];
    if (!missing.empty()) throw std::runtime_error("Missing boundary conditions for sides: " + missing);
    for (int i = 0; i < count && i < 20; ++i) {
        switch (entries[i].type) {
            case Wall: m.isWall = true; break;
            case SlipWall: m.isSlipWall = true; break;
            case FreeConvect: m.isFreeConvect = true; break;
            case Neumann: m.isNeumann = true; break;
            case Periodic: m.isPeriodic = true; break;
            case Velocity: m.isVelocity = true; break;
            default: break;
        }
    }
    return m;
}

// Geometry list and signed distance, restating src/geometry/Geometry.cu:72-203 and
// include/geometry/Geometry.cuh:102-161.
struct Geometry {
    int n = 0;
    int type[16];
    double center[16][3], length[16][3], radius[16], amplitude[16];
    int id[16];
};

Geometry read_geometry(const std::string& file) {
    Geometry g;
    std::ifstream in(file);
    if (!in.is_open()) throw std::runtime_error("cannot open config file: " + file);
    std::string line;
    bool inList = false, inBlock = false;
    int ctype = UnknownGeo, cid = -1;
    double cc[3] = {0, 0, 0}, cl[3] = {0, 0, 0}, cr = 0, ca = 0;
    while (std::getline(in, line)) {
        strip_all(line);
        if (line.empty() || line[0] == '#') continue;
        if (!inList && line.find("geometry") != std::string::npos && line.find('=') != std::string::npos) {
            inList = true;
            continue;
        }
        if (inList && line == "]") break;
        if (!inList) continue;
        if (line == "[") continue;
        if (line == "{") {
            inBlock = true;
            ctype = UnknownGeo;
            cid = -1;
            cc[0] = cc[1] = cc[2] = cl[0] = cl[1] = cl[2] = cr = ca = 0;
            continue;
        }
        if (line == "}" || line == "},") {
            inBlock = false;
            if (ctype == UnknownGeo) throw std::runtime_error("Encountered a geometry with unknown type during parsing.");
            if (g.n >= 16) throw std::runtime_error("more than 16 geometries");
            g.type[g.n] = ctype;
            for (int d = 0; d < 3; ++d) g.center[g.n][d] = cc[d], g.length[g.n][d] = cl[d];
            g.radius[g.n] = cr;
            g.amplitude[g.n] = ca;
            g.id[g.n] = cid;
            g.n++;
            continue;
        }
        if (!inBlock) continue;
        size_t pos = line.find('=');
        if (pos == std::string::npos) continue;
        std::string k = line.substr(0, pos), v = line.substr(pos + 1);
        v.erase(std::remove(v.begin(), v.end(), '"'), v.end());
        if (k == "type") {
            std::string l = lower(v);
            ctype = l == "circle" ? Circle : l == "sphere" ? Sphere : l == "square" ? Square : l == "cube" ? Cube
                  : l == "perturbation" ? Perturbation : UnknownGeo;
        } else if (k == "center") parse_list(v, cc, 3);
        else if (k == "length") parse_list(v, cl, 3);
        else if (k == "radius") cr = std::stod(v);
        else if (k == "amplitude") ca = std::stod(v);
        else if (k == "id") cid = std::stoi(v);
    }
    return g;
}

double sdf(const Geometry& geo, int id, double x, double y, double z, int dim) {
    for (int i = 0; i < geo.n; ++i) {
        if (geo.id[i] != id) continue;
        switch (geo.type[i]) {
            case Circle: {
                double dx = x - geo.center[i][0], dy = y - geo.center[i][1];
                return std::sqrt(dx * dx + dy * dy) - geo.radius[i];
            }
            case Sphere: {
                double dx = x - geo.center[i][0], dy = y - geo.center[i][1], dz = z - geo.center[i][2];
                return std::sqrt(dx * dx + dy * dy + dz * dz) - geo.radius[i];
            }
            case Square: {
                double dx = std::fabs(x - geo.center[i][0]) - geo.length[i][0] * 0.5;
                double dy = std::fabs(y - geo.center[i][1]) - geo.length[i][1] * 0.5;
                double ax = std::max(dx, 0.0), ay = std::max(dy, 0.0);
                double outside = std::sqrt(ax * ax + ay * ay);
                double inside = std::min(std::max(dx, dy), 0.0);
                return outside + inside;
            }
            case Cube: {
                double dx = std::fabs(x - geo.center[i][0]) - geo.length[i][0] * 0.5;
                double dy = std::fabs(y - geo.center[i][1]) - geo.length[i][1] * 0.5;
                double dz = std::fabs(z - geo.center[i][2]) - geo.length[i][2] * 0.5;
                double ax = std::max(dx, 0.0), ay = std::max(dy, 0.0), az = std::max(dz, 0.0);
                double outside = std::sqrt(ax * ax + ay * ay + az * az);
                double inside = std::min(std::max(std::max(dx, dy), dz), 0.0);
                return outside + inside;
            }
            case Perturbation: {
                double pert;
                if (dim == 2) pert = geo.amplitude[i] * geo.length[i][0] * std::cos(2.0 * M_PI * x / geo.length[i][0]);
                else
                    pert = geo.amplitude[i] * geo.length[i][0] *
                           (std::cos(2.0 * M_PI * x / geo.length[i][0]) + std::cos(2.0 * M_PI * z / geo.length[i][0]));
                const double yShift = pert + geo.center[i][1];
                return y - yShift;
            }
            default: break;
        }
    }
    return 1e10;
}

// ---------------------------------------------------------------- lattice
// Velocity sets and boundary maps: include/solver/WMRT.cuh:189-237.
template <int DIM> struct Lat;
template <> struct Lat<2> {
    static constexpr int Q = 9, A = 3, weight = 2;
    static constexpr int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    static constexpr int ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    static constexpr int ez[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    static constexpr double wa[9] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                                     1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
    static constexpr int wall[6][3] = {{1, 5, 8}, {3, 7, 6}, {2, 5, 6}, {4, 7, 8}, {0, 0, 0}, {0, 0, 0}};
};
template <> struct Lat<3> {
    static constexpr int Q = 19, A = 5, weight = 4;
    static constexpr int ex[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    static constexpr int ey[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
    static constexpr int ez[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
    static constexpr double wa[19] = {1.0 / 3.0,  1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
                                      1.0 / 18.0, 1.0 / 18.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                                      1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                                      1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
    static constexpr int wall[6][5] = {{1, 9, 7, 13, 11},  {2, 10, 8, 14, 12}, {3, 10, 7, 17, 15},
                                       {4, 9, 8, 18, 16},  {5, 14, 11, 18, 15}, {6, 13, 12, 17, 16}};
};

// Weighted-MRT transforms: include/solver/WMRT.cuh:54-184 (same statements).
void convert9(const double* in, double* out) {
    const double in0 = in[0], in1 = in[1], in2 = in[2], in3 = in[3], in4 = in[4], in5 = in[5], in6 = in[6],
                 in7 = in[7], in8 = in[8];
    out[0] = in0 + in1 + in2 + in3 + in4 + in5 + in6 + in7 + in8;
    out[1] = -4.0 * in0 - in1 - in2 - in3 - in4 + 2.0 * in5 + 2.0 * in6 + 2.0 * in7 + 2.0 * in8;
    out[2] = 4.0 * in0 - 2.0 * in1 - 2.0 * in2 - 2.0 * in3 - 2.0 * in4 + in5 + in6 + in7 + in8;
    out[3] = in1 - in3 + in5 - in6 - in7 + in8;
    out[4] = -2.0 * in1 + 2.0 * in3 + in5 - in6 - in7 + in8;
    out[5] = in2 - in4 + in5 + in6 - in7 - in8;
    out[6] = -2.0 * in2 + 2.0 * in4 + in5 + in6 - in7 - in8;
    out[7] = in1 - in2 + in3 - in4;
    out[8] = in5 - in6 + in7 - in8;
}
void reconvert9(const double* in, double* out) {
    const double in0 = in[0], in1 = in[1], in2 = in[2], in3 = in[3], in4 = in[4], in5 = in[5], in6 = in[6],
                 in7 = in[7], in8 = in[8];
    out[0] = (4.0 * in0 - 4.0 * in1 + 4.0 * in2) / 36.0;
    out[1] = (4.0 * in0 - in1 - 2.0 * in2 + 6.0 * in3 - 6.0 * in4 + 9.0 * in7) / 36.0;
    out[2] = (4.0 * in0 - in1 - 2.0 * in2 + 6.0 * in5 - 6.0 * in6 - 9.0 * in7) / 36.0;
    out[3] = (4.0 * in0 - in1 - 2.0 * in2 - 6.0 * in3 + 6.0 * in4 + 9.0 * in7) / 36.0;
    out[4] = (4.0 * in0 - in1 - 2.0 * in2 - 6.0 * in5 + 6.0 * in6 - 9.0 * in7) / 36.0;
    out[5] = (4.0 * in0 + 2.0 * in1 + in2 + 6.0 * in3 + 3.0 * in4 + 6.0 * in5 + 3.0 * in6 + 9.0 * in8) / 36.0;
    out[6] = (4.0 * in0 + 2.0 * in1 + in2 - 6.0 * in3 - 3.0 * in4 + 6.0 * in5 + 3.0 * in6 - 9.0 * in8) / 36.0;
    out[7] = (4.0 * in0 + 2.0 * in1 + in2 - 6.0 * in3 - 3.0 * in4 - 6.0 * in5 - 3.0 * in6 + 9.0 * in8) / 36.0;
    out[8] = (4.0 * in0 + 2.0 * in1 + in2 + 6.0 * in3 + 3.0 * in4 - 6.0 * in5 - 3.0 * in6 - 9.0 * in8) / 36.0;
}
void convert19(const double* in, double* out) {
    const double in0 = in[0], in1 = in[1], in2 = in[2], in3 = in[3], in4 = in[4], in5 = in[5], in6 = in[6],
                 in7 = in[7], in8 = in[8], in9 = in[9], in10 = in[10], in11 = in[11], in12 = in[12],
                 in13 = in[13], in14 = in[14], in15 = in[15], in16 = in[16], in17 = in[17], in18 = in[18];
    out[0] = in0 + in1 + in2 + in3 + in4 + in5 + in6 + in7 + in8 + in9 + in10 + in11 + in12 + in13 + in14 + in15 + in16 + in17 + in18;
    out[1] = in1 - in2 + in7 - in8 + in9 - in10 + in11 - in12 + in13 - in14;
    out[2] = in3 - in4 + in7 - in8 - in9 + in10 + in15 - in16 + in17 - in18;
    out[3] = in5 - in6 + in11 - in12 - in13 + in14 + in15 - in16 - in17 + in18;
    out[4] = in7 + in8 - in9 - in10;
    out[5] = in15 + in16 - in17 - in18;
    out[6] = in11 + in12 - in13 - in14;
    out[7] = 2.0 * in1 + 2.0 * in2 - in3 - in4 - in5 - in6 + in7 + in8 + in9 + in10 + in11 + in12 + in13 + in14 - 2.0 * in15 - 2.0 * in16 - 2.0 * in17 - 2.0 * in18;
    out[8] = in3 + in4 - in5 - in6 + in7 + in8 + in9 + in10 - in11 - in12 - in13 - in14;
    out[9] = -in0 + in7 + in8 + in9 + in10 + in11 + in12 + in13 + in14 + in15 + in16 + in17 + in18;
    out[10] = -2.0 * in1 + 2.0 * in2 + in7 - in8 + in9 - in10 + in11 - in12 + in13 - in14;
    out[11] = -2.0 * in3 + 2.0 * in4 + in7 - in8 - in9 + in10 + in15 - in16 + in17 - in18;
    out[12] = -2.0 * in5 + 2.0 * in6 + in11 - in12 - in13 + in14 + in15 - in16 - in17 + in18;
    out[13] = in7 - in8 + in9 - in10 - in11 + in12 - in13 + in14;
    out[14] = -in7 + in8 + in9 - in10 + in15 - in16 + in17 - in18;
    out[15] = in11 - in12 - in13 + in14 - in15 + in16 + in17 - in18;
    out[16] = in0 - 2.0 * in1 - 2.0 * in2 - 2.0 * in3 - 2.0 * in4 - 2.0 * in5 - 2.0 * in6 + in7 + in8 + in9 + in10 + in11 + in12 + in13 + in14 + in15 + in16 + in17 + in18;
    out[17] = -2.0 * in1 - 2.0 * in2 + in3 + in4 + in5 + in6 + in7 + in8 + in9 + in10 + in11 + in12 + in13 + in14 - 2.0 * in15 - 2.0 * in16 - 2.0 * in17 - 2.0 * in18;
    out[18] = -in3 - in4 + in5 + in6 + in7 + in8 + in9 + in10 - in11 - in12 - in13 - in14;
}
void reconvert19(const double* in, double* out) {
    const double in0 = in[0], in1 = in[1], in2 = in[2], in3 = in[3], in4 = in[4], in5 = in[5], in6 = in[6],
                 in7 = in[7], in8 = in[8], in9 = in[9], in10 = in[10], in11 = in[11], in12 = in[12],
                 in13 = in[13], in14 = in[14], in15 = in[15], in16 = in[16], in17 = in[17], in18 = in[18];
    out[0] = (2.0 * in0 - 3.0 * in9 + in16) / 6.0;
    out[1] = (2.0 * in0 + 6.0 * in1 + 3.0 * in7 - 6.0 * in10 - 2.0 * in16 - 3.0 * in17) / 36.0;
    out[2] = (2.0 * in0 - 6.0 * in1 + 3.0 * in7 + 6.0 * in10 - 2.0 * in16 - 3.0 * in17) / 36.0;
    out[3] = (4.0 * in0 + 12.0 * in2 - 3.0 * in7 + 9.0 * in8 - 12.0 * in11 - 4.0 * in16 + 3.0 * in17 - 9.0 * in18) / 72.0;
    out[4] = (4.0 * in0 - 12.0 * in2 - 3.0 * in7 + 9.0 * in8 + 12.0 * in11 - 4.0 * in16 + 3.0 * in17 - 9.0 * in18) / 72.0;
    out[5] = (4.0 * in0 + 12.0 * in3 - 3.0 * in7 - 9.0 * in8 - 12.0 * in12 - 4.0 * in16 + 3.0 * in17 + 9.0 * in18) / 72.0;
    out[6] = (4.0 * in0 - 12.0 * in3 - 3.0 * in7 - 9.0 * in8 + 12.0 * in12 - 4.0 * in16 + 3.0 * in17 + 9.0 * in18) / 72.0;
    out[7] = (4.0 * in0 + 12.0 * in1 + 12.0 * in2 + 36.0 * in4 + 3.0 * in7 + 9.0 * in8 + 6.0 * in9 + 6.0 * in10 + 6.0 * in11 + 18.0 * in13 - 18.0 * in14 + 2.0 * in16 + 3.0 * in17 + 9.0 * in18) / 144.0;
    out[8] = (4.0 * in0 - 12.0 * in1 - 12.0 * in2 + 36.0 * in4 + 3.0 * in7 + 9.0 * in8 + 6.0 * in9 - 6.0 * in10 - 6.0 * in11 - 18.0 * in13 + 18.0 * in14 + 2.0 * in16 + 3.0 * in17 + 9.0 * in18) / 144.0;
    out[9] = (4.0 * in0 + 12.0 * in1 - 12.0 * in2 - 36.0 * in4 + 3.0 * in7 + 9.0 * in8 + 6.0 * in9 + 6.0 * in10 - 6.0 * in11 + 18.0 * in13 + 18.0 * in14 + 2.0 * in16 + 3.0 * in17 + 9.0 * in18) / 144.0;
    out[10] = (4.0 * in0 - 12.0 * in1 + 12.0 * in2 - 36.0 * in4 + 3.0 * in7 + 9.0 * in8 + 6.0 * in9 - 6.0 * in10 + 6.0 * in11 - 18.0 * in13 - 18.0 * in14 + 2.0 * in16 + 3.0 * in17 + 9.0 * in18) / 144.0;
    out[11] = (4.0 * in0 + 12.0 * in1 + 12.0 * in3 + 36.0 * in6 + 3.0 * in7 - 9.0 * in8 + 6.0 * in9 + 6.0 * in10 + 6.0 * in12 - 18.0 * in13 + 18.0 * in15 + 2.0 * in16 + 3.0 * in17 - 9.0 * in18) / 144.0;
    out[12] = (4.0 * in0 - 12.0 * in1 - 12.0 * in3 + 36.0 * in6 + 3.0 * in7 - 9.0 * in8 + 6.0 * in9 - 6.0 * in10 - 6.0 * in12 + 18.0 * in13 - 18.0 * in15 + 2.0 * in16 + 3.0 * in17 - 9.0 * in18) / 144.0;
    out[13] = (4.0 * in0 + 12.0 * in1 - 12.0 * in3 - 36.0 * in6 + 3.0 * in7 - 9.0 * in8 + 6.0 * in9 + 6.0 * in10 - 6.0 * in12 - 18.0 * in13 - 18.0 * in15 + 2.0 * in16 + 3.0 * in17 - 9.0 * in18) / 144.0;
    out[14] = (4.0 * in0 - 12.0 * in1 + 12.0 * in3 - 36.0 * in6 + 3.0 * in7 - 9.0 * in8 + 6.0 * in9 - 6.0 * in10 + 6.0 * in12 + 18.0 * in13 + 18.0 * in15 + 2.0 * in16 + 3.0 * in17 - 9.0 * in18) / 144.0;
    out[15] = (4.0 * in0 + 12.0 * in2 + 12.0 * in3 + 36.0 * in5 - 6.0 * in7 + 6.0 * in9 + 6.0 * in11 + 6.0 * in12 + 18.0 * in14 - 18.0 * in15 + 2.0 * in16 - 6.0 * in17) / 144.0;
    out[16] = (4.0 * in0 - 12.0 * in2 - 12.0 * in3 + 36.0 * in5 - 6.0 * in7 + 6.0 * in9 - 6.0 * in11 - 6.0 * in12 - 18.0 * in14 + 18.0 * in15 + 2.0 * in16 - 6.0 * in17) / 144.0;
    out[17] = (4.0 * in0 + 12.0 * in2 - 12.0 * in3 - 36.0 * in5 - 6.0 * in7 + 6.0 * in9 + 6.0 * in11 - 6.0 * in12 + 18.0 * in14 + 18.0 * in15 + 2.0 * in16 - 6.0 * in17) / 144.0;
    out[18] = (4.0 * in0 - 12.0 * in2 + 12.0 * in3 - 36.0 * in5 - 6.0 * in7 + 6.0 * in9 - 6.0 * in11 + 6.0 * in12 - 18.0 * in14 - 18.0 * in15 + 2.0 * in16 - 6.0 * in17) / 144.0;
}

// ---------------------------------------------------------------- solver state
struct Oracle {
    std::string config;
    Params P;
    BCMap bc;
    Geometry geo;
    int dim = 2;
    unsigned ext[3] = {1, 1, 1};
    unsigned dmin[3] = {0, 0, 0}, dmax[3] = {0, 0, 0}, gmin[3] = {0, 0, 0}, gmax[3] = {0, 0, 0};
    size_t nodes = 0;
    int Q = 9;
    std::vector<double> f, g, f_post, g_post, rho, p, c, dc, vel, mu, normal;
    std::vector<double> f_prev, g_prev;  // free convect: last step's f_post, g_post (dev_f_prev, dev_g_prev)
    long steps = 0;

    size_t idx(unsigned i, unsigned j, unsigned k) const { return ((size_t)i * ext[1] + j) * ext[2] + k; }
};

template <int DIM>
inline double equilibrium(int q, double Ux, double Uy, double Uz) {  // NsAllen.cu:77-94
    using L = Lat<DIM>;
    const int exq = L::ex[q], eyq = L::ey[q];
    const double waq = L::wa[q];
    double eU, U2;
    if (DIM == 2) {
        eU = exq * Ux + eyq * Uy;
        U2 = Ux * Ux + Uy * Uy;
    } else {
        const int ezq = L::ez[q];
        eU = exq * Ux + eyq * Uy + ezq * Uz;
        U2 = Ux * Ux + Uy * Uy + Uz * Uz;
    }
    return waq * (3.0 * eU + 4.5 * eU * eU - 1.5 * U2);
}

template <int DIM>
inline void calculate_vf(const Params& P, const double* gneq, double* fv, double tau, double dcdx, double dcdy,
                         double dcdz) {  // NsAllen.cu:102-132
    using L = Lat<DIM>;
    double sxx = 0, sxy = 0, syy = 0, szy = 0, szx = 0, szz = 0;
    const double rhoDiff = P.RhoH - P.RhoL;
    for (int i = 0; i < L::Q; ++i) {
        sxx += L::ex[i] * L::ex[i] * gneq[i];
        sxy += L::ex[i] * L::ey[i] * gneq[i];
        syy += L::ey[i] * L::ey[i] * gneq[i];
        if (DIM == 3) {
            szy += L::ez[i] * L::ey[i] * gneq[i];
            szx += L::ez[i] * L::ex[i] * gneq[i];
            szz += L::ez[i] * L::ez[i] * gneq[i];
        }
    }
    fv[0] = -tau * (sxx * dcdx + sxy * dcdy + szx * dcdz) * rhoDiff;
    fv[1] = -tau * (sxy * dcdx + syy * dcdy + szy * dcdz) * rhoDiff;
    if (DIM == 3) fv[2] = -tau * (szz * dcdz + szx * dcdx + szy * dcdy) * rhoDiff;
}

template <int DIM>
inline double tau_of(const Params& P, double c) {
    if (c < 0.0) return P.tauL;
    if (c > 1.0) return P.tauH;
    return P.tauL + c * (P.tauH - P.tauL);
}

template <int DIM>
inline void wmrt_relax(double* gneq, double s9) {
    double tmp[19];
    if (DIM == 2) {
        convert9(gneq, tmp);
        tmp[7] = tmp[7] * s9;
        tmp[8] = tmp[8] * s9;
        reconvert9(tmp, gneq);
    } else {
        convert19(gneq, tmp);
        for (int m = 4; m <= 8; ++m) tmp[m] = tmp[m] * s9;
        reconvert19(tmp, gneq);
    }
}

// Loop over the (i,j,k) nodes of [lo, hi] per axis in parallel.
template <class F>
void for_nodes(const Oracle& o, const unsigned* lo, const unsigned* hi, F&& fn) {
    const long ni = (long)hi[0] - lo[0] + 1;
    parallel_for(ni, [&](long ii) {
        const unsigned i = lo[0] + (unsigned)ii;
        for (unsigned j = lo[1]; j <= hi[1]; ++j)
            for (unsigned k = lo[2]; k <= hi[2]; ++k) fn(i, j, k);
    });
    (void)o;
}

// --- per-kernel restatements ---------------------------------------------------
template <int DIM>
void chemical_potential(Oracle& o) {  // NsAllen.cu:207-236
    const double* c = o.c.data();
    for_nodes(o, o.dmin, o.dmax, [&](unsigned i, unsigned j, unsigned k) {
        double D2C;
        if (DIM == 2) {
            D2C = (c[o.idx(i - 1, j - 1, 0)] + c[o.idx(i + 1, j - 1, 0)] + c[o.idx(i - 1, j + 1, 0)] +
                   c[o.idx(i + 1, j + 1, 0)] +
                   4.0 * (c[o.idx(i, j - 1, 0)] + c[o.idx(i - 1, j, 0)] + c[o.idx(i + 1, j, 0)] + c[o.idx(i, j + 1, 0)]) -
                   20 * c[o.idx(i, j, 0)]) /
                  6.0;
        } else {
            D2C = (20.0 * (c[o.idx(i + 1, j, k)] + c[o.idx(i - 1, j, k)] + c[o.idx(i, j + 1, k)] + c[o.idx(i, j - 1, k)] +
                           c[o.idx(i, j, k + 1)] + c[o.idx(i, j, k - 1)]) +
                   6.0 * (c[o.idx(i + 1, j + 1, k)] + c[o.idx(i, j + 1, k - 1)] + c[o.idx(i - 1, j + 1, k)] +
                          c[o.idx(i, j + 1, k + 1)] + c[o.idx(i + 1, j, k + 1)] + c[o.idx(i + 1, j, k - 1)] +
                          c[o.idx(i - 1, j, k - 1)] + c[o.idx(i - 1, j, k + 1)] + c[o.idx(i, j - 1, k + 1)] +
                          c[o.idx(i + 1, j - 1, k)] + c[o.idx(i, j - 1, k - 1)] + c[o.idx(i - 1, j - 1, k)]) +
                   (c[o.idx(i + 1, j + 1, k + 1)] + c[o.idx(i + 1, j + 1, k - 1)] + c[o.idx(i - 1, j + 1, k - 1)] +
                    c[o.idx(i - 1, j + 1, k + 1)] + c[o.idx(i + 1, j - 1, k + 1)] + c[o.idx(i + 1, j - 1, k - 1)] +
                    c[o.idx(i - 1, j - 1, k - 1)] + c[o.idx(i - 1, j - 1, k + 1)]) -
                   200.0 * c[o.idx(i, j, k)]) /
                  48.0;
        }
        const size_t s = o.idx(i, j, k);
        o.mu[s] = 4.0 * o.P.betaConstant * c[s] * (c[s] - 1.0) * (c[s] - 0.50) - o.P.kConstant * D2C;
    });
}

template <int DIM>
void isotropic_gradient(Oracle& o) {  // NsAllen.cu:280-322
    const double* c = o.c.data();
    for_nodes(o, o.dmin, o.dmax, [&](unsigned i, unsigned j, unsigned k) {
        const size_t s = o.idx(i, j, k);
        double* d = &o.dc[s * DIM];
        if (DIM == 2) {
            d[0] = (c[o.idx(i + 1, j, k)] - c[o.idx(i - 1, j, k)]) / 3.0 +
                   (c[o.idx(i + 1, j - 1, k)] + c[o.idx(i + 1, j + 1, k)] - c[o.idx(i - 1, j - 1, k)] - c[o.idx(i - 1, j + 1, k)]) / 12.0;
            d[1] = (c[o.idx(i, j + 1, k)] - c[o.idx(i, j - 1, k)]) / 3.0 +
                   (c[o.idx(i - 1, j + 1, k)] + c[o.idx(i + 1, j + 1, k)] - c[o.idx(i - 1, j - 1, k)] - c[o.idx(i + 1, j - 1, k)]) / 12.0;
        } else {
            d[0] = (0.50) * ((4.0 / 9.0) * (c[o.idx(i + 1, j, k)] - c[o.idx(i - 1, j, k)]) +
                             (1.0 / 9.0) * ((c[o.idx(i + 1, j, k + 1)] + c[o.idx(i + 1, j, k - 1)] + c[o.idx(i + 1, j + 1, k)] + c[o.idx(i + 1, j - 1, k)]) -
                                            (c[o.idx(i - 1, j, k + 1)] + c[o.idx(i - 1, j, k - 1)] + c[o.idx(i - 1, j + 1, k)] + c[o.idx(i - 1, j - 1, k)])) +
                             (1.0 / 36.0) * ((c[o.idx(i + 1, j + 1, k + 1)] + c[o.idx(i + 1, j - 1, k + 1)] + c[o.idx(i + 1, j + 1, k - 1)] + c[o.idx(i + 1, j - 1, k - 1)]) -
                                             (c[o.idx(i - 1, j + 1, k + 1)] + c[o.idx(i - 1, j - 1, k + 1)] + c[o.idx(i - 1, j + 1, k - 1)] + c[o.idx(i - 1, j - 1, k - 1)])));
            d[1] = (0.50) * ((4.0 / 9.0) * (c[o.idx(i, j + 1, k)] - c[o.idx(i, j - 1, k)]) +
                             (1.0 / 9.0) * ((c[o.idx(i + 1, j + 1, k)] + c[o.idx(i - 1, j + 1, k)] + c[o.idx(i, j + 1, k + 1)] + c[o.idx(i, j + 1, k - 1)]) -
                                            (c[o.idx(i, j - 1, k + 1)] + c[o.idx(i, j - 1, k - 1)] + c[o.idx(i + 1, j - 1, k)] + c[o.idx(i - 1, j - 1, k)])) +
                             (1.0 / 36.0) * ((c[o.idx(i + 1, j + 1, k + 1)] + c[o.idx(i - 1, j + 1, k + 1)] + c[o.idx(i + 1, j + 1, k - 1)] + c[o.idx(i - 1, j + 1, k - 1)]) -
                                             (c[o.idx(i + 1, j - 1, k + 1)] + c[o.idx(i - 1, j - 1, k + 1)] + c[o.idx(i + 1, j - 1, k - 1)] + c[o.idx(i - 1, j - 1, k - 1)])));
            d[2] = (0.50) * ((4.0 / 9.0) * (c[o.idx(i, j, k + 1)] - c[o.idx(i, j, k - 1)]) +
                             (1.0 / 9.0) * ((c[o.idx(i + 1, j, k + 1)] + c[o.idx(i - 1, j, k + 1)] + c[o.idx(i, j + 1, k + 1)] + c[o.idx(i, j - 1, k + 1)]) -
                                            (c[o.idx(i + 1, j, k - 1)] + c[o.idx(i - 1, j, k - 1)] + c[o.idx(i, j + 1, k - 1)] + c[o.idx(i, j - 1, k - 1)])) +
                             (1.0 / 36.0) * ((c[o.idx(i + 1, j + 1, k + 1)] + c[o.idx(i + 1, j - 1, k + 1)] + c[o.idx(i - 1, j + 1, k + 1)] + c[o.idx(i - 1, j - 1, k + 1)]) -
                                             (c[o.idx(i + 1, j + 1, k - 1)] + c[o.idx(i - 1, j + 1, k - 1)] + c[o.idx(i + 1, j - 1, k - 1)] + c[o.idx(i - 1, j - 1, k - 1)])));
        }
    });
}

template <int DIM>
void normal_fd(Oracle& o) {  // NsAllen.cu:241-275
    for_nodes(o, o.dmin, o.dmax, [&](unsigned i, unsigned j, unsigned k) {
        const size_t s = o.idx(i, j, k);
        const double* d = &o.dc[s * DIM];
        double* n = &o.normal[s * DIM];
        if (DIM == 2) {
            const double tmp = std::sqrt((d[0] * d[0]) + (d[1] * d[1])) + 1e-32;
            n[0] = d[0] / tmp;
            n[1] = d[1] / tmp;
        } else {
            const double tmp = std::sqrt((d[0] * d[0]) + (d[1] * d[1]) + (d[2] * d[2])) + 1e-32;
            n[0] = d[0] / tmp;
            n[1] = d[1] / tmp;
            n[2] = d[2] / tmp;
        }
    });
}

template <int DIM>
void initialize_distributions(Oracle& o) {  // NsAllen.cu:137-202 (every node, ghosts included)
    using L = Lat<DIM>;
    const Params& P = o.P;
    for_nodes(o, o.gmin, o.gmax, [&](unsigned i, unsigned j, unsigned k) {
        const size_t s = o.idx(i, j, k);
        o.rho[s] = (P.RhoL) + o.c[s] * ((P.RhoH) - (P.RhoL));
        if (P.caseType == Bubble) o.p[s] = o.p[s] - o.c[s] * P.sigma / (P.referenceLength / 2.0) / (o.rho[s] / 3.0);
        else if (P.caseType == Drop) o.p[s] = o.p[s] + o.c[s] * P.sigma / (P.referenceLength / 2.0) / (o.rho[s] / 3.0);
        else o.p[s] = 0;
        double* u = &o.vel[s * DIM];
        for (int d = 0; d < DIM; ++d) u[d] = 0;
        const double* n = &o.normal[s * DIM];
        for (int q = 0; q < L::Q; ++q) {
            double ga_wa, hlp;
            if (DIM == 2) {
                ga_wa = equilibrium<DIM>(q, u[0], u[1], 0.0);
                hlp = L::wa[q] * ((1.0 - 4.0 * ((o.c[s] - 0.50) * (o.c[s] - 0.50))) / P.interfaceWidth *
                                  (L::ex[q] * n[0] + L::ey[q] * n[1]));
            } else {
                ga_wa = equilibrium<DIM>(q, u[0], u[1], u[2]);
                hlp = L::wa[q] * ((1.0 - 4.0 * ((o.c[s] - 0.50) * (o.c[s] - 0.50))) / P.interfaceWidth *
                                  (L::ex[q] * n[0] + L::ey[q] * n[1] + L::ez[q] * n[2]));
            }
            const double Gamma = ga_wa + L::wa[q];
            o.g_post[s * L::Q + q] = o.c[s] * Gamma - 0.50 * hlp;
            o.g[s * L::Q + q] = o.c[s] * Gamma - 0.50 * hlp;
            o.f_post[s * L::Q + q] = o.p[s] * L::wa[q] + ga_wa;
            o.f[s * L::Q + q] = o.p[s] * L::wa[q] + ga_wa;
        }
    });
}

template <int DIM>
void collision_g(Oracle& o) {  // NsAllen.cu:545-584
    using L = Lat<DIM>;
    const Params& P = o.P;
    const double wc = 1.0 / (0.50 + 3.0 * P.mobility);
    for_nodes(o, o.dmin, o.dmax, [&](unsigned i, unsigned j, unsigned k) {
        const size_t s = o.idx(i, j, k);
        const double* u = &o.vel[s * DIM];
        const double* n = &o.normal[s * DIM];
        const double cs = o.c[s];
        for (int q = 0; q < L::Q; ++q) {
            double ga_wa, e_normal;
            if (DIM == 2) {
                ga_wa = equilibrium<DIM>(q, u[0], u[1], 0.0);
                e_normal = (L::ex[q] * n[0] + L::ey[q] * n[1]);
            } else {
                ga_wa = equilibrium<DIM>(q, u[0], u[1], u[2]);
                e_normal = (L::ex[q] * n[0] + L::ey[q] * n[1] + L::ez[q] * n[2]);
            }
            const double eF = ((3.0 * (P.mobility) * (1.0 - 4.0 * ((cs - 0.50) * (cs - 0.50)))) / (P.interfaceWidth)) * e_normal;
            const double hlp = L::wa[q] * eF;
            const double heq = cs * (ga_wa + L::wa[q]) + hlp;
            o.g[s * L::Q + q] = o.g_post[s * L::Q + q] * (1.0 - (wc)) + heq * (wc);
        }
    });
}

template <int DIM>
void gravity_force(const Params& P, double rho, double* fg) {  // NsAllen.cu:460-474
    for (int d = 0; d < DIM; ++d) {
        if (P.caseType == RTI) fg[d] = (rho) * P.gravity[d];
        else if (P.caseType == Bubble) fg[d] = (rho - P.RhoH) * P.gravity[d];
        else if (P.caseType == Drop) fg[d] = (rho - P.RhoL) * P.gravity[d];
        else fg[d] = 0.0;  // Jet: the reference leaves fg uninitialised; no body force here
    }
}

template <int DIM>
void collision_f(Oracle& o) {  // NsAllen.cu:589-763
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    const Params& P = o.P;
    const double drho3 = (P.RhoH - P.RhoL) / 3.0;
    for_nodes(o, o.dmin, o.dmax, [&](unsigned i, unsigned j, unsigned k) {
        const size_t s = o.idx(i, j, k);
        const double* u = &o.vel[s * DIM];
        const double* d = &o.dc[s * DIM];
        const double* fp = &o.f_post[s * Q];
        double gneq[Q], ga_wa[Q], hlp[Q], fv[3] = {0, 0, 0}, fg[3] = {0, 0, 0};
        for (int q = 0; q < Q; ++q) {
            ga_wa[q] = equilibrium<DIM>(q, u[0], u[1], DIM == 3 ? u[2] : 0.0);
            const double geq = o.p[s] * L::wa[q] + ga_wa[q];
            gneq[q] = fp[q] - geq;
        }
        double tau = tau_of<DIM>(P, o.c[s]);
        double s9 = 1.0 / (tau + 0.50);
        wmrt_relax<DIM>(gneq, s9);
        calculate_vf<DIM>(P, gneq, fv, tau, d[0], d[1], DIM == 3 ? d[2] : 0.0);
        gravity_force<DIM>(P, o.rho[s], fg);
        const double Fpx = -o.p[s] * drho3 * d[0];
        const double Fpy = -o.p[s] * drho3 * d[1];
        const double Fx = o.mu[s] * d[0] + Fpx + fv[0] + fg[0];
        const double Fy = o.mu[s] * d[1] + Fpy + fv[1] + fg[1];
        double Fz = 0.0;
        if (DIM == 3) {
            const double Fpz = -o.p[s] * drho3 * d[2];
            Fz = o.mu[s] * d[2] + Fpz + fv[2] + fg[2];
        }
        for (int q = 0; q < Q; ++q) {
            double eF;
            if (DIM == 2) eF = L::ex[q] * Fx + L::ey[q] * Fy;
            else eF = L::ex[q] * Fx + L::ey[q] * Fy + L::ez[q] * Fz;
            hlp[q] = 3.0 * L::wa[q] * eF / o.rho[s];
            const double feq = o.p[s] * L::wa[q] + ga_wa[q] - 0.50 * hlp[q];
            gneq[q] = fp[q] - feq;
        }
        tau = tau_of<DIM>(P, o.c[s]);
        s9 = 1.0 / (tau + 0.50);
        wmrt_relax<DIM>(gneq, s9);
        for (int q = 0; q < Q; ++q) o.f[s * Q + q] = fp[q] - gneq[q] + hlp[q];
    });
}

// Periodic ghost copy (Solver.cu:75-141), as sequential x, y, z passes.
void periodic_copy(Oracle& o, std::vector<double>& a, int dof) {
    const int nd = o.dim;
    for (int ax = 0; ax < nd; ++ax) {
        const int sm = 2 * ax, sp = 2 * ax + 1;
        if (!(o.bc.types[sm] == Periodic || o.bc.types[sp] == Periodic)) continue;
        unsigned lo[3] = {o.gmin[0], o.gmin[1], o.gmin[2]}, hi[3] = {o.gmax[0], o.gmax[1], o.gmax[2]};
        lo[ax] = hi[ax] = 0;  // iterate the plane orthogonal to ax
        const long n0 = (long)hi[0] - lo[0] + 1;
        parallel_for(n0, [&](long ii) {
            for (unsigned j = lo[1]; j <= hi[1]; ++j)
                for (unsigned k = lo[2]; k <= hi[2]; ++k) {
                    unsigned a0[3] = {lo[0] + (unsigned)ii, j, k};
                    unsigned gm[3] = {a0[0], a0[1], a0[2]}, gp[3] = {a0[0], a0[1], a0[2]};
                    unsigned im[3] = {a0[0], a0[1], a0[2]}, ip[3] = {a0[0], a0[1], a0[2]};
                    gm[ax] = o.gmin[ax];
                    gp[ax] = o.gmax[ax];
                    im[ax] = o.dmin[ax];
                    ip[ax] = o.dmax[ax];
                    const size_t sgm = o.idx(gm[0], gm[1], gm[2]), sgp = o.idx(gp[0], gp[1], gp[2]);
                    const size_t sim = o.idx(im[0], im[1], im[2]), sip = o.idx(ip[0], ip[1], ip[2]);
                    for (int q = 0; q < dof; ++q) {
                        a[sgm * dof + q] = a[sip * dof + q];
                        a[sgp * dof + q] = a[sim * dof + q];
                    }
                }
        });
    }
}

// Velocity inlet on ghost planes (Solver.cu:550-921).
template <int DIM>
void jet_boundary(Oracle& o) {
    using L = Lat<DIM>;
    constexpr int Q = L::Q, A = L::A;
    const double weight = L::weight;
    const double* V = o.bc.val[YPlus];  // the reference reads the y+ entry for every inlet side
    for (int side = 0; side < 2 * DIM; ++side) {
        if (o.bc.types[side] != Velocity) continue;
        const int ax = side / 2;
        const bool plus = side & 1;
        const int* inDirs = L::wall[side];
        const int* oppDirs = L::wall[side ^ 1];
        unsigned lo[3] = {o.gmin[0], o.gmin[1], o.gmin[2]}, hi[3] = {o.gmax[0], o.gmax[1], o.gmax[2]};
        lo[ax] = hi[ax] = plus ? o.gmax[ax] : o.gmin[ax];
        for_nodes(o, lo, hi, [&](unsigned i, unsigned j, unsigned k) {
            const size_t s = o.idx(i, j, k);
            const double x = i, y = j, z = DIM == 3 ? (double)k : 0.0;
            double* fs = &o.f[s * Q];
            double* gs = &o.g[s * Q];
            if (sdf(o.geo, 0, x, y, z, DIM) <= 0) {
                double feq[Q], geq[Q];
                double M1 = 0, M2 = 0, N = 0;  // tangential momenta (in axis order) and phase defect
                const int* e_ax = ax == 0 ? L::ex : ax == 1 ? L::ey : L::ez;
                for (int q = 1; q < Q; ++q) {
                    const double fa_wa = equilibrium<DIM>(q, V[0], V[1], V[2]);
                    feq[q] = 0.0 * L::wa[q] + fa_wa;
                    geq[q] = o.c[s] * (fa_wa + L::wa[q]);
                    if (e_ax[q] == 0) {
                        if (ax == 0) {
                            M1 += L::ey[q] * (fs[q] - feq[q]);
                            if (DIM == 3) M2 += L::ez[q] * (fs[q] - feq[q]);
                        } else if (ax == 1) {
                            M1 += L::ex[q] * (fs[q] - feq[q]);
                            if (DIM == 3) M2 += L::ez[q] * (fs[q] - feq[q]);
                        } else {
                            M1 += L::ex[q] * (fs[q] - feq[q]);
                            M2 += L::ey[q] * (fs[q] - feq[q]);
                        }
                        N += (gs[q] - geq[q]);
                    }
                }
                for (int a = 0; a < A; ++a) {
                    const int id = inDirs[a], od = oppDirs[a];
                    double corr;
                    if (ax == 0) corr = DIM == 2 ? (L::ey[id] * M1) : (L::ey[id] * M1 + L::ez[id] * M2);
                    else if (ax == 1) corr = DIM == 2 ? (L::ex[id] * M1) : (L::ex[id] * M1 + L::ez[id] * M2);
                    else corr = (L::ex[id] * M1 + L::ey[id] * M2);
                    fs[id] = fs[od] + feq[id] - feq[od] - (1.0 / weight) * corr;
                    if (a == 0) gs[id] = geq[id] - (gs[od] - geq[od]);
                    else gs[id] = geq[id] - (gs[od] - geq[od]) - N / weight;
                }
            } else {
                unsigned ii[3] = {i, j, k};
                ii[ax] = plus ? o.dmax[ax] : o.dmin[ax];
                const size_t t = o.idx(ii[0], ii[1], ii[2]);
                for (int a = 0; a < A; ++a) {
                    gs[inDirs[a]] = o.g[t * Q + oppDirs[a]];
                    fs[inDirs[a]] = o.f[t * Q + oppDirs[a]];
                    o.c[s] = o.c[t];
                }
            }
        });
    }
}

template <int DIM>
void streaming(Oracle& o, const std::vector<double>& a, std::vector<double>& post) {  // NsAllen.cu:327-364
    using L = Lat<DIM>;
    for_nodes(o, o.dmin, o.dmax, [&](unsigned i, unsigned j, unsigned k) {
        const size_t s = o.idx(i, j, k);
        for (int q = 0; q < L::Q; ++q) {
            const unsigned id = i - L::ex[q], jd = j - L::ey[q], kd = DIM == 3 ? k - L::ez[q] : 0;
            post[s * L::Q + q] = a[o.idx(id, jd, kd) * L::Q + q];
        }
    });
}

template <int DIM>
void half_bounce_back(Oracle& o) {  // Solver.cu:248-333 with wallBCMap
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    for_nodes(o, o.gmin, o.gmax, [&](unsigned i, unsigned j, unsigned k) {
        const unsigned ijk[3] = {i, j, k};
        const size_t s = o.idx(i, j, k);
        for (int a = 0; a < L::A; ++a) {
            for (int side = 0; side < 2 * DIM; ++side) {
                const int ax = side / 2;
                const bool plus = side & 1;
                if (o.bc.types[side] != Wall && o.bc.types[side] != SlipWall) continue;
                if (ijk[ax] != (plus ? o.dmax[ax] : o.dmin[ax])) continue;
                const int id = L::wall[side][a], od = L::wall[side ^ 1][a];
                o.f_post[s * Q + id] = o.f[s * Q + od];
                o.g_post[s * Q + id] = o.g[s * Q + od];
            }
        }
    });
}

// Convective outflow on free-convect sides (kernelFreeConvect, Solver.cu:342-451): on the
// first interior layer, each direction entering across the side becomes
// (f_prev + U f_post(neighbour)) / (1 + U), U = |u| of the inner neighbour along the
// side's axis (the previous step's velocity: macroscopic has not run yet).  Sides in the
// order x-, x+, y-, y+, z-, z+, directions in wallBCMap order; neighbour values from the
// snapshot taken before the pass.
template <int DIM>
void free_convect(Oracle& o) {
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    const std::vector<double> fs = o.f_post, gs = o.g_post;
    for_nodes(o, o.dmin, o.dmax, [&](unsigned i, unsigned j, unsigned k) {
        const unsigned ijk[3] = {i, j, k};
        const size_t s = o.idx(i, j, k);
        for (int side = 0; side < 2 * DIM; ++side) {
            const int ax = side / 2;
            const bool plus = side & 1;
            if (o.bc.types[side] != FreeConvect) continue;
            if (ijk[ax] != (plus ? o.dmax[ax] : o.dmin[ax])) continue;
            unsigned nb[3] = {i, j, k};
            nb[ax] = plus ? nb[ax] - 1 : nb[ax] + 1;
            const size_t sn = o.idx(nb[0], nb[1], nb[2]);
            const double U = std::fabs(o.vel[sn * DIM + ax]);
            for (int a = 0; a < L::A; ++a) {
                const int d = L::wall[side][a];
                o.f_post[s * Q + d] = (o.f_prev[s * Q + d] + U * fs[sn * Q + d]) / (1.0 + U);
                o.g_post[s * Q + d] = (o.g_prev[s * Q + d] + U * gs[sn * Q + d]) / (1.0 + U);
            }
        }
    });
}

// Zero-gradient sides (kernelNeumann, Solver.cu:456-542): on the first interior layer,
// each direction entering across the side takes the inner neighbour's population.
// Directions in wallBCMap order outside, sides inside (the reference's loop nest);
// neighbour values from the snapshot taken before the pass.
template <int DIM>
void neumann(Oracle& o) {
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    const std::vector<double> fs = o.f_post, gs = o.g_post;
    for_nodes(o, o.dmin, o.dmax, [&](unsigned i, unsigned j, unsigned k) {
        const unsigned ijk[3] = {i, j, k};
        const size_t s = o.idx(i, j, k);
        for (int a = 0; a < L::A; ++a) {
            for (int side = 0; side < 2 * DIM; ++side) {
                const int ax = side / 2;
                const bool plus = side & 1;
                if (o.bc.types[side] != Neumann) continue;
                if (ijk[ax] != (plus ? o.dmax[ax] : o.dmin[ax])) continue;
                unsigned nb[3] = {i, j, k};
                nb[ax] = plus ? nb[ax] - 1 : nb[ax] + 1;
                const size_t sn = o.idx(nb[0], nb[1], nb[2]);
                const int d = L::wall[side][a];
                o.f_post[s * Q + d] = fs[sn * Q + d];
                o.g_post[s * Q + d] = gs[sn * Q + d];
            }
        }
    });
}

inline bool mirror_type(int t) {
    return t == Wall || t == FreeConvect || t == Neumann || t == SlipWall || t == DoNothing;
}

// Mirror copy of c into the ghost layer (Solver.cu:927-978).  The reference launches it
// three times per step when a wall exists (NsAllen.cu:931,943,955); inside one launch
// the edge/corner ghosts of two mirror sides are written concurrently, but after the
// second launch every such cell holds the value of the nearest interior node, so three
// Jacobi passes (each reading the previous pass) reproduce the reference's result.
void mirror_c(Oracle& o, int passes) {
    std::vector<double> snap;
    for (int pass = 0; pass < passes; ++pass) {
        snap = o.c;
        for_nodes(o, o.gmin, o.gmax, [&](unsigned i, unsigned j, unsigned k) {
            const unsigned ijk[3] = {i, j, k};
            const size_t s = o.idx(i, j, k);
            for (int side = 0; side < 2 * o.dim; ++side) {
                const int ax = side / 2;
                const bool plus = side & 1;
                if (!mirror_type(o.bc.types[side])) continue;
                if (ijk[ax] != (plus ? o.dmax[ax] : o.dmin[ax])) continue;
                unsigned gh[3] = {i, j, k};
                gh[ax] = plus ? o.gmax[ax] : o.gmin[ax];
                o.c[o.idx(gh[0], gh[1], gh[2])] = snap[s];
            }
        });
    }
}

template <int DIM>
void macroscopic_g(Oracle& o) {  // NsAllen.cu:516-540
    using L = Lat<DIM>;
    for_nodes(o, o.dmin, o.dmax, [&](unsigned i, unsigned j, unsigned k) {
        const size_t s = o.idx(i, j, k);
        double c = 0;
        for (int q = 0; q < L::Q; ++q) c += o.g_post[s * L::Q + q];
        o.c[s] = c;
        o.rho[s] = (o.P.RhoL + (c * (o.P.RhoH - o.P.RhoL)));
    });
}

template <int DIM>
void macroscopic_f(Oracle& o) {  // NsAllen.cu:369-511
    using L = Lat<DIM>;
    constexpr int Q = L::Q;
    const Params& P = o.P;
    const double drho3 = (P.RhoH - P.RhoL) / 3.0;
    for_nodes(o, o.dmin, o.dmax, [&](unsigned i, unsigned j, unsigned k) {
        const size_t s = o.idx(i, j, k);
        const double* fp = &o.f_post[s * Q];
        double* u = &o.vel[s * DIM];
        const double* d = &o.dc[s * DIM];
        double p = 0;
        for (int q = 0; q < Q; ++q) p += fp[q];
        o.p[s] = p;
        double gneq[Q], fv[3] = {0, 0, 0}, fg[3] = {0, 0, 0};
        for (int q = 0; q < Q; ++q) {
            const double ga_wa = equilibrium<DIM>(q, u[0], u[1], DIM == 3 ? u[2] : 0.0);
            const double geq = p * L::wa[q] + ga_wa;
            gneq[q] = fp[q] - geq;
        }
        const double tau = tau_of<DIM>(P, o.c[s]);
        const double s9 = 1.0 / (tau + 0.50);
        wmrt_relax<DIM>(gneq, s9);
        calculate_vf<DIM>(P, gneq, fv, tau, d[0], d[1], DIM == 3 ? d[2] : 0.0);
        gravity_force<DIM>(P, o.rho[s], fg);
        const double Fpx = -p * drho3 * d[0];
        const double Fpy = -p * drho3 * d[1];
        const double Fx = o.mu[s] * d[0] + Fpx + fv[0] + fg[0];
        const double Fy = o.mu[s] * d[1] + Fpy + fv[1] + fg[1];
        double Fz = 0;
        if (DIM == 3) {
            const double Fpz = -p * drho3 * d[2];
            Fz = o.mu[s] * d[2] + Fpz + fv[2] + fg[2];
        }
        double ux = 0, uy = 0, uz = 0;
        for (int q = 0; q < Q; ++q) {
            ux += L::ex[q] * fp[q];
            uy += L::ey[q] * fp[q];
            if (DIM == 3) uz += L::ez[q] * fp[q];
        }
        u[0] = ux + 0.50 * Fx / o.rho[s];
        u[1] = uy + 0.50 * Fy / o.rho[s];
        if (DIM == 3) u[2] = uz + 0.50 * Fz / o.rho[s];
    });
}

template <int DIM>
void initial_condition(Oracle& o) {  // NsAllen.cu:768-824
    for_nodes(o, o.gmin, o.gmax, [&](unsigned i, unsigned j, unsigned k) {
        const double x = i, y = j, z = DIM == 3 ? (double)k : 0.0;
        const size_t s = o.idx(i, j, k);
        switch (o.P.caseType) {
            case Bubble: o.c[s] = 0.50 + 0.50 * std::tanh(2.0 * sdf(o.geo, 0, x, y, z, DIM) / o.P.interfaceWidth); break;
            case Drop:
            case Jet: o.c[s] = 0.50 - 0.50 * std::tanh(2.0 * sdf(o.geo, 0, x, y, z, DIM) / o.P.interfaceWidth); break;
            case RTI: o.c[s] = 0.5 + 0.5 * std::tanh(2.0 * sdf(o.geo, 0, x, y, z, DIM) / o.P.interfaceWidth); break;
            default: o.c[s] = 0.0; break;
        }
    });
}

template <int DIM>
void device_initializer(Oracle& o) {  // NsAllen.cu:897-908
    chemical_potential<DIM>(o);
    isotropic_gradient<DIM>(o);
    normal_fd<DIM>(o);
    initialize_distributions<DIM>(o);
}

template <int DIM>
void solve(Oracle& o) {  // NsAllen.cu:881-892
    // collision()
    normal_fd<DIM>(o);
    collision_g<DIM>(o);
    collision_f<DIM>(o);
    // applyPeriodicBoundary()
    if (o.bc.isPeriodic) {
        periodic_copy(o, o.f, Lat<DIM>::Q);
        periodic_copy(o, o.g, Lat<DIM>::Q);
        periodic_copy(o, o.c, 1);
    }
    // velocityBoundary()
    if (o.bc.isVelocity) jet_boundary<DIM>(o);
    // streaming(): free convect keeps the last step's post-streaming populations first
    if (o.bc.isFreeConvect) {
        o.f_prev = o.f_post;
        o.g_prev = o.g_post;
    }
    streaming<DIM>(o, o.f, o.f_post);
    streaming<DIM>(o, o.g, o.g_post);
    // applyWallBoundary(), applyFreeConvectBoundary(), applyNeumannBoundary(): each ends
    // with the c mirror, which runs whenever any mirror-type side exists (c does not
    // change in between, so the three launches are the three passes below)
    if (o.bc.isWall) half_bounce_back<DIM>(o);
    if (o.bc.isFreeConvect) free_convect<DIM>(o);
    if (o.bc.isNeumann) neumann<DIM>(o);
    if (o.bc.isWall || o.bc.isSlipWall || o.bc.isFreeConvect || o.bc.isNeumann) mirror_c(o, 3);
    // macroscopic()
    macroscopic_g<DIM>(o);
    chemical_potential<DIM>(o);
    isotropic_gradient<DIM>(o);
    macroscopic_f<DIM>(o);
    o.steps++;
}

thread_local std::string g_err;

}  // namespace

// ---------------------------------------------------------------- C interface
extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void* orc_create(const char* config_path) {
    try {
        auto* o = new Oracle();
        o->config = config_path;
        o->P = read_params(o->config);
        o->geo = read_geometry(o->config);
        if (o->P.caseType == UnknownCase) throw std::runtime_error("case type missing");
        const bool three = o->P.N[2] > 1.0;
        o->dim = three ? 3 : 2;
        o->bc = read_boundaries(o->config, o->dim);
        for (int s = 0; s < 2 * o->dim; ++s) {
            const int t = o->bc.types[s];
            if (t != Wall && t != Periodic && t != Velocity && t != SlipWall && t != FreeConvect && t != Neumann)
                throw std::runtime_error("unsupported boundary type on side " + std::to_string(s));
        }
        for (int s1 = 0; s1 < 2 * o->dim; ++s1)
            for (int s2 = 0; s2 < 2 * o->dim; ++s2) {
                const int t = o->bc.types[s1];
                if (s1 / 2 != s2 / 2 && t == o->bc.types[s2] && (t == FreeConvect || t == Neumann))
                    throw std::runtime_error("two adjacent free-convect or Neumann sides: the reference's threads race on their edge nodes (Solver.cu:342-542); not supported");
            }
        if (o->bc.isSlipWall && !o->bc.isWall)
            throw std::runtime_error("a slip wall without a wall side gets no bounce-back in the reference (Solver.cu:1000-1004); not supported");
        if (o->dim == 2) {
            o->ext[0] = (unsigned)(o->P.N[0] + 2);
            o->ext[1] = (unsigned)(o->P.N[1] + 2);
            o->ext[2] = 1;
            o->dmin[0] = o->dmin[1] = 1;
            o->dmin[2] = 0;
            o->dmax[0] = o->ext[0] - 2;
            o->dmax[1] = o->ext[1] - 2;
            o->dmax[2] = 0;
            o->gmax[0] = o->ext[0] - 1;
            o->gmax[1] = o->ext[1] - 1;
            o->gmax[2] = 0;
        } else {
            for (int a = 0; a < 3; ++a) {
                o->ext[a] = (unsigned)o->P.N[a];
                o->dmin[a] = 1;
                o->dmax[a] = o->ext[a] - 2;
                o->gmax[a] = o->ext[a] - 1;
            }
        }
        o->Q = o->dim == 3 ? 19 : 9;
        o->nodes = (size_t)o->ext[0] * o->ext[1] * o->ext[2];
        const size_t n = o->nodes, Q = o->Q, D = o->dim;
        o->f.assign(n * Q, 0.0);
        o->g.assign(n * Q, 0.0);
        o->f_post.assign(n * Q, 0.0);
        o->g_post.assign(n * Q, 0.0);
        o->f_prev.assign(n * Q, 0.0);
        o->g_prev.assign(n * Q, 0.0);
        o->rho.assign(n, 0.0);
        o->p.assign(n, 0.0);
        o->c.assign(n, 0.0);
        o->mu.assign(n, 0.0);
        o->dc.assign(n * D, 0.0);
        o->vel.assign(n * D, 0.0);
        o->normal.assign(n * D, 0.0);
        return o;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }

int orc_dim(void* h) { return static_cast<Oracle*>(h)->dim; }
int orc_q(void* h) { return static_cast<Oracle*>(h)->Q; }
void orc_extent(void* h, int* e) {
    auto* o = static_cast<Oracle*>(h);
    for (int a = 0; a < 3; ++a) e[a] = (int)o->ext[a];
}
long orc_steps(void* h) { return static_cast<Oracle*>(h)->steps; }

// Derived parameters, for checking the product's config parser.
// Order: RhoL RhoH sigma muH muL tauH tauL kConstant betaConstant mobility interfaceWidth
//        referenceLength gravity[0..2] caseType
void orc_params(void* h, double* out) {
    const Params& P = static_cast<Oracle*>(h)->P;
    const double v[] = {P.RhoL, P.RhoH, P.sigma, P.muH, P.muL, P.tauH, P.tauL, P.kConstant, P.betaConstant,
                        P.mobility, P.interfaceWidth, P.referenceLength, P.gravity[0], P.gravity[1], P.gravity[2],
                        (double)P.caseType};
    std::memcpy(out, v, sizeof(v));
}
void orc_bc(void* h, int* types, double* vals) {
    auto* o = static_cast<Oracle*>(h);
    for (int s = 0; s < 6; ++s) {
        types[s] = o->bc.types[s];
        for (int d = 0; d < 3; ++d) vals[s * 3 + d] = o->bc.val[s][d];
    }
}
double orc_sdf(void* h, double x, double y, double z) {
    auto* o = static_cast<Oracle*>(h);
    return sdf(o->geo, 0, x, y, z, o->dim);
}

static std::vector<double>* field(Oracle* o, const char* name) {
    const std::string n = name;
    if (n == "f") return &o->f;
    if (n == "g") return &o->g;
    if (n == "f_post") return &o->f_post;
    if (n == "g_post") return &o->g_post;
    if (n == "f_prev") return &o->f_prev;
    if (n == "g_prev") return &o->g_prev;
    if (n == "rho") return &o->rho;
    if (n == "p") return &o->p;
    if (n == "c") return &o->c;
    if (n == "mu") return &o->mu;
    if (n == "dc") return &o->dc;
    if (n == "vel") return &o->vel;
    if (n == "normal") return &o->normal;
    return nullptr;
}

long orc_field_size(void* h, const char* name) {
    auto* v = field(static_cast<Oracle*>(h), name);
    return v ? (long)v->size() : -1;
}
int orc_get(void* h, const char* name, double* out) {
    auto* v = field(static_cast<Oracle*>(h), name);
    if (!v) return -1;
    std::memcpy(out, v->data(), v->size() * sizeof(double));
    return 0;
}
int orc_set(void* h, const char* name, const double* in) {
    auto* v = field(static_cast<Oracle*>(h), name);
    if (!v) return -1;
    std::memcpy(v->data(), in, v->size() * sizeof(double));
    return 0;
}

void orc_initial_condition(void* h) {
    auto* o = static_cast<Oracle*>(h);
    if (o->dim == 2) initial_condition<2>(*o);
    else initial_condition<3>(*o);
}
void orc_device_initializer(void* h) {
    auto* o = static_cast<Oracle*>(h);
    if (o->dim == 2) device_initializer<2>(*o);
    else device_initializer<3>(*o);
}
void orc_solve(void* h, long nsteps) {
    auto* o = static_cast<Oracle*>(h);
    for (long s = 0; s < nsteps; ++s) {
        if (o->dim == 2) solve<2>(*o);
        else solve<3>(*o);
    }
}
// Sum of c over the interior (the mass monitor, Reporter.cu:50-114 without its
// double counting of the tail block), summed in x-slowest order.
double orc_mass(void* h) {
    auto* o = static_cast<Oracle*>(h);
    double s = 0;
    for (unsigned i = o->dmin[0]; i <= o->dmax[0]; ++i)
        for (unsigned j = o->dmin[1]; j <= o->dmax[1]; ++j)
            for (unsigned k = o->dmin[2]; k <= o->dmax[2]; ++k) s += o->c[o->idx(i, j, k)];
    return s;
}
int orc_threads() { return n_threads(); }
}
