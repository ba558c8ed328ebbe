// config.txt reader with the reference's parse rules; see config.hpp for the citations.
#include "config.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace clipb {
namespace {

std::string trim_blanks(const std::string& s) {  // spaces/tabs at both ends (InputData.cu:326-338)
    const size_t a = s.find_first_not_of(" \t");
    if (a == std::string::npos) return std::string();
    const size_t b = s.find_last_not_of(" \t");
    return s.substr(a, b - a + 1);
}

std::string squeeze(std::string s) {  // every space/tab/CR removed (Boundary.cu:282-288)
    s.erase(std::remove_if(s.begin(), s.end(), [](unsigned char ch) { return ch == ' ' || ch == '\t' || ch == '\r'; }),
            s.end());
    return s;
}

std::string to_lower(std::string s) {
    for (auto& ch : s) ch = (char)std::tolower((unsigned char)ch);
    return s;
}

std::string unquote(std::string s) {
    s.erase(std::remove(s.begin(), s.end(), '"'), s.end());
    return s;
}

// The file is read once; every query below scans the stored lines the way the
// reference's readers rescan the file.
class ConfigFile {
public:
    explicit ConfigFile(std::istream& in) {
        std::string line;
        while (std::getline(in, line)) lines_.push_back(line);
    }

    // First non-comment "key = value" whose trimmed key matches.
    bool scalar(const std::string& key, std::string& value) const {
        for (const auto& line : lines_) {
            if (line.empty() || line[0] == '#') continue;
            const size_t eq = line.find('=');
            if (eq == std::string::npos) continue;
            if (trim_blanks(line.substr(0, eq)) == key) {
                value = trim_blanks(line.substr(eq + 1));
                return true;
            }
        }
        return false;
    }

    void real(const std::string& key, double& out) const {
        std::string v;
        if (scalar(key, v)) {
            std::istringstream is(v);
            is >> out;
        }
    }

    void integer(const std::string& key, long& out) const {
        std::string v;
        if (scalar(key, v)) {
            std::istringstream is(v);
            is >> out;
        }
    }

    void triple(const std::string& key, double (&out)[3]) const {
        std::string v;
        if (!scalar(key, v)) return;
        out[0] = out[1] = out[2] = 0.0;
        v.erase(std::remove(v.begin(), v.end(), '['), v.end());
        v.erase(std::remove(v.begin(), v.end(), ']'), v.end());
        std::stringstream ss(v);
        std::string tok;
        for (int n = 0; n < 3 && std::getline(ss, tok, ','); ++n) out[n] = std::stod(trim_blanks(tok));
    }

    // Lines of a "name = [ {..} {..} ]" block list, whitespace removed, after the first
    // line that mentions `name` and '='.  Geometry lists stop at "]"; the reference's
    // boundary reader runs to the end of the file (Boundary.cu:162-236).
    std::vector<std::string> block_list(const std::string& name, bool stop_at_bracket) const {
        std::vector<std::string> out;
        bool in_list = false;
        for (const auto& raw : lines_) {
            const std::string line = squeeze(raw);
            if (line.empty() || line[0] == '#') continue;
            if (!in_list) {
                if (line.find(name) != std::string::npos && line.find('=') != std::string::npos) in_list = true;
                continue;
            }
            if (stop_at_bracket && line == "]") break;
            out.push_back(line);
        }
        return out;
    }

private:
    std::vector<std::string> lines_;
};

void parse_numbers(std::string v, double* out, int maxn) {
    if (!v.empty() && v.front() == '[') v.erase(0, 1);
    if (!v.empty() && v.back() == ']') v.pop_back();
    std::stringstream ss(v);
    std::string tok;
    for (int n = 0; n < maxn && std::getline(ss, tok, ','); ++n) out[n] = std::stod(tok);
}

int side_of(const std::string& s) {
    static const char* names[] = {"x-", "x+", "y-", "y+", "z-", "z+"};
    const std::string l = to_lower(s);
    for (int i = 0; i < 6; ++i)
        if (l == names[i]) return i;
    return kUnknownSide;
}

int bc_of(const std::string& s) {
    // The reference removes all whitespace from a block line before it matches the type
    // names (Boundary.cu:57-75, 282-288), so its spaced names "slip wall", "free convect"
    // and "do nothing" can never match there.  Here the unspaced forms match as well, which
    // makes those sides reachable.
    const std::string l = to_lower(s);
    if (l == "wall") return kWall;
    if (l == "slip wall" || l == "slipwall") return kSlipWall;
    if (l == "free convect" || l == "freeconvect") return kFreeConvect;
    if (l == "periodic") return kPeriodic;
    if (l == "neumann") return kNeumann;
    if (l == "velocity") return kVelocity;
    if (l == "do nothing" || l == "donothing") return kDoNothing;
    return kUnknownBC;
}

int geo_of(const std::string& s) {
    const std::string l = to_lower(s);
    if (l == "circle") return kCircle;
    if (l == "sphere") return kSphere;
    if (l == "square") return kSquare;
    if (l == "cube") return kCube;
    if (l == "perturbation") return kPerturbation;
    return kUnknownGeo;
}

Physics read_physics(const ConfigFile& cf) {
    Physics p;
    std::string cs;
    if (cf.scalar("case", cs)) {
        std::istringstream is(cs);
        std::string word;
        is >> word;
        word = to_lower(word);
        if (word == "drop") p.caseType = kDrop;
        else if (word == "bubble") p.caseType = kBubble;
        else if (word == "jet") p.caseType = kJet;
        else if (word == "rti") p.caseType = kRTI;
        else throw std::runtime_error("Unknown case type: " + word);
    }
    cf.integer("finalStep", p.finalStep);
    cf.integer("outputInterval", p.outputInterval);
    cf.integer("reportInterval", p.reportInterval);
    cf.integer("checkpointInterval", p.checkpointInterval);
    cf.integer("checkpointCopy", p.checkpointCopy);
    cf.triple("N", p.N);
    cf.real("referenceLength", p.referenceLength);
    cf.real("interfaceWidth", p.interfaceWidth);
    cf.triple("gravity", p.gravity);
    cf.real("mobility", p.mobility);
    cf.real("muRatio", p.muRatio);
    cf.real("rhoRatio", p.rhoRatio);
    cf.real("amplitude", p.amplitude);

    // Derived physics (InputData.cu:76-114); every expression keeps the reference's
    // operation order so the FP64 values are identical.
    p.RhoH = 1.0;
    p.RhoL = p.RhoH / p.rhoRatio;
    const double g = std::fabs(p.gravity[1]);
    const double L = p.referenceLength;
    switch (p.caseType) {
        case kBubble:
        case kDrop:
            cf.real("We", p.We);
            cf.real("Re", p.Re);
            p.sigma = (p.RhoH * g * L * L) / p.We;
            p.muH = std::sqrt(g * p.RhoH * (p.RhoH - p.RhoL) * L * L * L) / p.Re;
            break;
        case kRTI:
            cf.real("Ca", p.Ca);
            cf.real("Pe", p.Pe);
            cf.real("Re", p.Re);
            p.muH = (p.RhoH * std::sqrt(g * L) * L) / p.Re;
            p.sigma = (p.muH * std::sqrt(g * L)) / p.Ca;
            p.mobility = (std::sqrt(g * L) * L) / p.Pe;
            break;
        case kJet:
            cf.real("We", p.We);
            cf.real("Re", p.Re);
            cf.real("referenceVelocity", p.referenceVelocity);
            p.sigma = (p.RhoH * p.referenceVelocity * p.referenceVelocity * L) / p.We;
            p.muH = (p.RhoH * p.referenceVelocity * L) / p.Re;
            break;
        default:
            break;
    }
    p.muL = p.muH / p.muRatio;
    p.tauH = 3.0 * (p.muH / p.RhoH);
    p.tauL = 3.0 * (p.muL / p.RhoL);
    p.kConstant = 1.50 * p.sigma * p.interfaceWidth;
    p.betaConstant = 8.0 * p.sigma / p.interfaceWidth;
    return p;
}

Boundaries read_boundaries(const ConfigFile& cf, int dim) {
    Boundaries b;
    struct Block {
        int side = kUnknownSide, type = kUnknownBC;
    };
    Block by_side[7];
    bool seen[7] = {false, false, false, false, false, false, false};
    int count = 0;
    bool in_block = false;
    Block cur;
    for (const std::string& line : cf.block_list("boundary", false)) {
        if (line == "[") continue;
        if (line == "{") {
            in_block = true;
            cur = Block{};
            continue;
        }
        if (line == "}" || line == "},") {
            in_block = false;
            by_side[cur.side] = cur;
            seen[cur.side] = true;
            ++count;
            continue;
        }
        if (!in_block) continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        const std::string key = line.substr(0, eq);
        const std::string val = unquote(line.substr(eq + 1));
        if (key == "side") {
            cur.side = side_of(val);
        } else if (key == "type") {
            cur.type = bc_of(val);
            b.type[cur.side] = cur.type;  // indexed by the side known so far, as in Boundary.cu:207-212
        } else if (key == "value") {
            double v[3] = {b.value[cur.side][0], b.value[cur.side][1], b.value[cur.side][2]};
            std::string s = val;
            if (!s.empty() && s.front() == '[') s.erase(0, 1);
            if (!s.empty() && s.back() == ']') s.pop_back();
            std::stringstream ss(s);
            std::string tok;
            for (int n = 0; n < 3 && std::getline(ss, tok, ','); ++n) v[n] = std::stod(tok);
            for (int n = 0; n < 3; ++n) b.value[cur.side][n] = v[n];
        }
    }
    std::string missing;
    static const char* names[] = {"x-", "x+", "y-", "y+", "z-", "z+"};
    for (int s = 0; s < 2 * dim; ++s)
        if (!seen[s]) missing += (missing.empty() ? "" : ", ") + std::string(names[s]);
    if (!missing.empty()) throw std::runtime_error("Missing boundary conditions for sides: " + missing);
    // Flags come from the first `count` entries of the side-indexed table (Boundary.cu:291-319).
    for (int i = 0; i < count && i < 7; ++i) {
        switch (by_side[i].type) {
            case kWall: b.isWall = true; break;
            case kSlipWall: b.isSlipWall = true; break;
            case kFreeConvect: b.isFreeConvect = true; break;
            case kNeumann: b.isNeumann = true; break;
            case kPeriodic: b.isPeriodic = true; break;
            case kVelocity: b.isVelocity = true; break;
            default: break;
        }
    }
    return b;
}

GeometryTable read_geometry(const ConfigFile& cf) {
    GeometryTable g;
    bool in_block = false;
    int type = kUnknownGeo, id = -1;
    double center[3] = {0, 0, 0}, length[3] = {0, 0, 0}, radius = 0, amplitude = 0;
    for (const std::string& line : cf.block_list("geometry", true)) {
        if (line == "[") continue;
        if (line == "{") {
            in_block = true;
            type = kUnknownGeo;
            id = -1;
            radius = amplitude = 0;
            for (int d = 0; d < 3; ++d) center[d] = length[d] = 0;
            continue;
        }
        if (line == "}" || line == "},") {
            in_block = false;
            if (type == kUnknownGeo) throw std::runtime_error("Encountered a geometry with unknown type during parsing.");
            if (g.n >= kMaxGeometries) throw std::runtime_error("more than 16 geometries in config");
            g.type[g.n] = type;
            for (int d = 0; d < 3; ++d) {
                g.center[g.n][d] = center[d];
                g.length[g.n][d] = length[d];
            }
            g.radius[g.n] = radius;
            g.amplitude[g.n] = amplitude;
            g.id[g.n] = id;
            ++g.n;
            continue;
        }
        if (!in_block) continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        const std::string key = line.substr(0, eq);
        const std::string val = unquote(line.substr(eq + 1));
        if (key == "type") type = geo_of(val);
        else if (key == "center") parse_numbers(val, center, 3);
        else if (key == "length") parse_numbers(val, length, 3);
        else if (key == "radius") radius = std::stod(val);
        else if (key == "amplitude") amplitude = std::stod(val);
        else if (key == "id") id = std::stoi(val);
    }
    return g;
}

}  // namespace

namespace {

CaseConfig parse_config(const ConfigFile& cf, const std::string& name) {
    CaseConfig c;
    c.path = name;
    c.phys = read_physics(cf);
    if (c.phys.caseType == kUnknownCase) throw std::runtime_error("config has no 'case'");
    c.dim = c.phys.N[2] > 1.0 ? 3 : 2;
    for (int a = 0; a < 3; ++a) {
        if (c.dim == 2) {
            c.extent[a] = a < 2 ? (int)(unsigned)(c.phys.N[a] + 2) : 1;
            c.interior[a] = a < 2 ? c.extent[a] - 2 : 1;
        } else {
            c.extent[a] = (int)(unsigned)c.phys.N[a];
            c.interior[a] = c.extent[a] - 2;
        }
    }
    for (int a = 0; a < c.dim; ++a)
        if (c.interior[a] < 2) throw std::runtime_error("grid too small: need at least 2 interior nodes per axis");
    c.bc = read_boundaries(cf, c.dim);
    for (int s = 0; s < 2 * c.dim; ++s) {
        const int t = c.bc.type[s];
        if (t != kWall && t != kPeriodic && t != kVelocity && t != kSlipWall && t != kFreeConvect && t != kNeumann)
            throw std::runtime_error("side " + std::to_string(s) +
                                     ": supported boundaries are wall, slip wall, periodic, velocity, free convect "
                                     "and neumann");
        // The free-convect and Neumann kernels update the edge nodes of two adjacent sides of
        // their type from several threads that read each other's writes (Solver.cu:342-542).
        for (int s2 = 0; s2 < 2 * c.dim; ++s2)
            if (s / 2 != s2 / 2 && t == c.bc.type[s2] && (t == kFreeConvect || t == kNeumann))
                throw std::runtime_error("two adjacent free-convect or two adjacent neumann sides are not supported: "
                                         "the reference's result there depends on thread timing");
    }
    // NSAllen::applyWallBoundary launches the bounce-back, which covers slip walls too, only
    // when a wall side exists (Solver.cu:997-1004); slip walls alone get none.
    if (c.bc.isSlipWall && !c.bc.isWall)
        throw std::runtime_error("a slip wall needs a wall side in the same case: the reference applies no "
                                 "bounce-back to slip walls otherwise");
    for (int a = 0; a < c.dim; ++a) {
        const bool pm = c.bc.type[2 * a] == kPeriodic, pp = c.bc.type[2 * a + 1] == kPeriodic;
        if (pm != pp) throw std::runtime_error("an axis must be periodic on both sides or on neither");
    }
    c.geo = read_geometry(cf);
    return c;
}

}  // namespace

CaseConfig load_config(const std::string& path) {
    std::ifstream in(path);
    if (!in.is_open()) throw std::runtime_error("cannot open config file: " + path);
    return parse_config(ConfigFile(in), path);
}

CaseConfig load_config_text(const std::string& text, const std::string& name) {
    std::istringstream in(text);
    return parse_config(ConfigFile(in), name);
}

}  // namespace clipb
