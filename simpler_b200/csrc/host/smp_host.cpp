// smp_host.cpp -- file formats, front-end parsing and scene assembly (see smp_host.h).
#include "smp_host.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <functional>
#include <iomanip>
#include <set>
#include <sstream>

namespace smp_host {

// ================================================================================================
// files
// ================================================================================================

// Image2::readPFM (image.h:183-245): header tokens "Pf", x, y, endianness; the texels are the
// file's last x*y doubles, stored bottom-to-top and flipped on read.
bool read_pfm_texture(const std::string &path, Texture &out, std::string &err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "Cannot open file " + path + ", or it does not exist"; return false; }
    std::string magic;
    f >> magic;
    if (magic != "Pf") { err = "Invalid magic number in " + path + ": no Pf (grayscale pfm)"; return false; }
    long x = 0, y = 0;
    std::string scale;
    f >> x >> y >> scale;
    if (!f || x <= 0 || y <= 0) { err = "bad PFM header in " + path; return false; }
    f.seekg(0, std::ios::end);
    long size = long(f.tellg());
    long need = x * y * long(sizeof(double));
    if (size < need) { err = "PFM " + path + " shorter than its header says"; return false; }
    f.seekg(size - need, std::ios::beg);
    std::vector<double> raw(size_t(x) * y);
    f.read(reinterpret_cast<char *>(raw.data()), need);
    if (!f) { err = "short read in " + path; return false; }
    out.x = int(x);
    out.y = int(y);
    out.texels.assign(size_t(x) * y, 0.0);
    for (long i = 0; i < y; ++i)
        std::memcpy(&out.texels[size_t(y - i - 1) * x], &raw[size_t(i) * x], size_t(x) * sizeof(double));
    return true;
}

// Image3::writePFM3D (image.cpp:161-206): "Pf\n" X " " Y " " Z "\n" -1 "\n", then X*Y*Z doubles,
// z-major slices, rows in y order, no flip.
bool write_pfm3d(const std::string &path, int X, int Y, int Z, const double *film, std::string &err) {
    std::ofstream f(path, std::ios::binary);
    if (!f) { err = "Problem writing output file " + path; return false; }
    f << "Pf" << '\n' << X << ' ' << Y << ' ' << Z << '\n' << static_cast<float>(-1.0) << '\n';
    f.write(reinterpret_cast<const char *>(film), std::streamsize(size_t(X) * Y * Z * sizeof(double)));
    if (!f) { err = "Problem writing output file " + path; return false; }
    return true;
}

// Image3::readPFM3D (image.h:374-436)
bool read_pfm3d(const std::string &path, int &X, int &Y, int &Z, std::vector<double> &film, std::string &err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "Cannot open file " + path + ", or it does not exist"; return false; }
    std::string magic, scale;
    f >> magic;
    if (magic != "Pf") { err = "Invalid magic number in " + path; return false; }
    long x = 0, y = 0, z = 0;
    f >> x >> y >> z >> scale;
    if (!f || x <= 0 || y <= 0 || z <= 0) { err = "bad PFM3D header in " + path; return false; }
    f.seekg(0, std::ios::end);
    long size = long(f.tellg());
    long need = x * y * z * long(sizeof(double));
    if (size < need) { err = "PFM3D " + path + " shorter than its header says"; return false; }
    f.seekg(size - need, std::ios::beg);
    film.resize(size_t(x) * y * z);
    f.read(reinterpret_cast<char *>(film.data()), need);
    if (!f) { err = "short read in " + path; return false; }
    X = int(x); Y = int(y); Z = int(z);
    return true;
}

// Spline::readVolAndBuild (spline.h:115-162): "VOL" 3, int32 type 1, int32 nx ny nz, int32
// channels 1, float xmin ymin zmin xmax ymax zmax, then nx*ny*nz floats x fastest.
bool read_vol(const std::string &path, Vol &out, std::string &err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "cannot open " + path; return false; }
    char hdr[4];
    f.read(hdr, 4);
    if (!f || hdr[0] != 'V' || hdr[1] != 'O' || hdr[2] != 'L') { err = "file " + path + " is not a VOL file"; return false; }
    if (int(hdr[3]) != 3) { err = "file " + path + " is not of VOL version 3"; return false; }
    int32_t type = 0, n[3], ch = 0;
    f.read(reinterpret_cast<char *>(&type), 4);
    if (type != 1) { err = "VOL type should be 1 (float)"; return false; }
    f.read(reinterpret_cast<char *>(n), 12);
    f.read(reinterpret_cast<char *>(&ch), 4);
    if (ch != 1) { err = "VOL should have a single channel"; return false; }
    float bb[6];
    f.read(reinterpret_cast<char *>(bb), 24);
    if (!f || n[0] < 2 || n[1] < 2 || n[2] < 2) { err = "bad VOL header in " + path; return false; }
    for (int i = 0; i < 3; ++i) { out.n[i] = n[i]; out.min[i] = bb[i]; out.max[i] = bb[3 + i]; }
    out.data.resize(size_t(n[0]) * n[1] * n[2]);
    f.read(reinterpret_cast<char *>(out.data.data()), std::streamsize(out.data.size() * sizeof(float)));
    if (!f) { err = "short read in " + path; return false; }
    return true;
}

bool write_vol(const std::string &path, const Vol &v, std::string &err) {
    std::ofstream f(path, std::ios::binary);
    if (!f) { err = "cannot write " + path; return false; }
    const char hdr[4] = {'V', 'O', 'L', 3};
    int32_t type = 1, ch = 1, n[3] = {v.n[0], v.n[1], v.n[2]};
    float bb[6] = {float(v.min[0]), float(v.min[1]), float(v.min[2]), float(v.max[0]), float(v.max[1]), float(v.max[2])};
    f.write(hdr, 4);
    f.write(reinterpret_cast<const char *>(&type), 4);
    f.write(reinterpret_cast<const char *>(n), 12);
    f.write(reinterpret_cast<const char *>(&ch), 4);
    f.write(reinterpret_cast<const char *>(bb), 24);
    f.write(reinterpret_cast<const char *>(v.data.data()), std::streamsize(v.data.size() * sizeof(float)));
    return bool(f);
}

// ================================================================================================
// JSON (RFC 8259 subset: objects, arrays, numbers, strings with the common escapes, literals)
// ================================================================================================
const Json *Json::get(const std::string &key) const {
    if (kind != Object) return nullptr;
    auto it = obj.find(key);
    return it == obj.end() ? nullptr : &it->second;
}

namespace {
struct JsonParser {
    const std::string &s;
    size_t i = 0;
    std::string err;
    explicit JsonParser(const std::string &t) : s(t) {}
    void ws() { while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i; }
    bool fail(const std::string &m) { if (err.empty()) err = m + " at offset " + std::to_string(i); return false; }
    bool value(Json &v) {
        ws();
        if (i >= s.size()) return fail("unexpected end");
        char c = s[i];
        if (c == '{') return object(v);
        if (c == '[') return array(v);
        if (c == '"') { v.kind = Json::String; return string(v.str); }
        if (s.compare(i, 4, "true") == 0) { v.kind = Json::Bool; v.b = true; i += 4; return true; }
        if (s.compare(i, 5, "false") == 0) { v.kind = Json::Bool; v.b = false; i += 5; return true; }
        if (s.compare(i, 4, "null") == 0) { v.kind = Json::Null; i += 4; return true; }
        return number(v);
    }
    bool number(Json &v) {
        const char *b = s.c_str() + i;
        char *e = nullptr;
        double d = std::strtod(b, &e);
        if (e == b) return fail("bad value");
        i += size_t(e - b);
        v.kind = Json::Number;
        v.num = d;
        return true;
    }
    bool string(std::string &out) {
        ++i;
        out.clear();
        while (i < s.size() && s[i] != '"') {
            char c = s[i++];
            if (c == '\\' && i < s.size()) {
                char e = s[i++];
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u':
                        if (i + 4 > s.size()) return fail("bad escape");
                        out += char(std::strtol(s.substr(i, 4).c_str(), nullptr, 16) & 0x7f);
                        i += 4;
                        break;
                    default: out += e;
                }
            } else {
                out += c;
            }
        }
        if (i >= s.size()) return fail("unterminated string");
        ++i;
        return true;
    }
    bool array(Json &v) {
        v.kind = Json::Array;
        ++i;
        ws();
        if (i < s.size() && s[i] == ']') { ++i; return true; }
        for (;;) {
            Json e;
            if (!value(e)) return false;
            v.arr.push_back(std::move(e));
            ws();
            if (i < s.size() && s[i] == ',') { ++i; continue; }
            if (i < s.size() && s[i] == ']') { ++i; return true; }
            return fail("expected , or ]");
        }
    }
    bool object(Json &v) {
        v.kind = Json::Object;
        ++i;
        ws();
        if (i < s.size() && s[i] == '}') { ++i; return true; }
        for (;;) {
            ws();
            if (i >= s.size() || s[i] != '"') return fail("expected key");
            std::string k;
            if (!string(k)) return false;
            ws();
            if (i >= s.size() || s[i] != ':') return fail("expected :");
            ++i;
            Json e;
            if (!value(e)) return false;
            v.obj[k] = std::move(e);
            ws();
            if (i < s.size() && s[i] == ',') { ++i; continue; }
            if (i < s.size() && s[i] == '}') { ++i; return true; }
            return fail("expected , or }");
        }
    }
};
}  // namespace

bool parse_json(const std::string &text, Json &out, std::string &err) {
    JsonParser p(text);
    if (!p.value(out)) { err = p.err; return false; }
    p.ws();
    if (p.i != text.size()) { err = "trailing characters after JSON value"; return false; }
    return true;
}

// ================================================================================================
// key=value front-end (renderer/samples/renderer3d_sample.cpp)
// ================================================================================================
namespace {

// tokenize (renderer3d_sample.cpp:26-38)
std::vector<std::string> tokenize(const std::string &str, const std::string &delim) {
    std::vector<std::string> tokens;
    std::string::size_type last = str.find_first_not_of(delim, 0);
    std::string::size_type pos = str.find_first_of(delim, last);
    while (std::string::npos != pos || std::string::npos != last) {
        tokens.push_back(str.substr(last, pos - last));
        last = str.find_first_not_of(delim, pos);
        pos = str.find_first_of(delim, last);
    }
    return tokens;
}

bool parse_bool(const std::string &key, std::string v, bool &out, std::string &err) {
    std::transform(v.begin(), v.end(), v.begin(), ::tolower);
    if (v == "true") { out = true; return true; }
    if (v == "false") { out = false; return true; }
    err = key + " should be either true or false; Argument " + v + " not recognized";
    return false;
}

bool parse_triple(const std::string &key, const std::string &v, double out[3], std::string &err) {
    std::vector<std::string> parts = tokenize(v, ",");
    if (parts.size() < 3) { err = "Three input coordinates required for " + key; return false; }
    if (parts.size() > 3) { err = "More than three input coordinates entered for " + key; return false; }
    for (int i = 0; i < 3; ++i) out[i] = std::stof(parts[i]);
    return true;
}

// keys the reference requires in strict mode, per field kind (renderer3d_sample.cpp:639-719)
const char *kCommonKeys[] = {"threads", "precision", "numPhotons", "outFilePrefix", "sigmaT", "albedo", "gVal",
                             "emitter_gap", "sensor_gap", "er_stepsize", "directTol", "useInitializationHack",
                             "rr_weight", "projectorTexture", "useDirect", "useAngularSampling",
                             "use_bounce_decomposition", "maxDepth", "maxPathlength", "pathLengthMin",
                             "pathLengthMax", "pathLengthBins", "spatialX", "spatialY", "halfThetaLimit",
                             "emitter_size", "sensor_size", "mediumLx", "mediumRx", "distribution", "gOrKappa",
                             "emitter_distance", "emitter_lens_aperture", "emitter_lens_focalLength",
                             "emitter_lens_active", "sensor_distance", "sensor_lens_aperture",
                             "sensor_lens_focalLength", "sensor_lens_active", "printInputs"};
const char *kAnalyticalKeys[] = {"f_u", "speed_u", "n_o", "n_max", "n_clip", "phi_min", "phi_max", "mode"};
const char *kSourcesKeys[] = {"f_u", "speed_u", "n_o", "n_scaling", "n_coeff", "radius", "center1", "center2",
                              "active1", "active2", "phase1", "phase2", "chordlength", "theta_sources",
                              "trans_z_sources"};
const char *kInterpolatedKeys[] = {"rifgridFile"};
// B200-side keys that the reference does not have
const char *kExtensionKeys[] = {"rendering_type", "mediumLy", "mediumRy", "mediumLz", "mediumRz", "seed",
                                "renderPrecision", "sensorMarchMax", "stepCap", "device", "planeWaves"};

void set_kind_defaults(RenderConfig &c) {
    if (c.kind == FieldKind::Sources) {      // renderer3d_sample.cpp:117-136
        c.f_u = 5e6;
        c.speed_u = 1500;
        c.n_o = 1.3333;
    }
}

}  // namespace

int parse_cli(int argc, const char *const *argv, RenderConfig &c, std::string &err) {
    std::vector<std::pair<std::string, std::string>> kv;
    for (int i = 1; i < argc; ++i) {
        std::vector<std::string> p = tokenize(argv[i], "=");
        if (p.size() != 2) { err = std::string("Input argument ") + argv[i] + " should be in the format arg=value"; return -1; }
        kv.emplace_back(p[0], p[1]);
    }
    // the field kind: rendering_type if given, else inferred from the keys present
    std::string rtype;
    bool has_sources = false, has_interp = false;
    for (auto &e : kv) {
        if (e.first == "rendering_type") rtype = e.second;
        if (e.first == "n_scaling" || e.first == "center1" || e.first == "center2" || e.first == "theta_sources") has_sources = true;
        if (e.first == "rifgridFile") has_interp = true;
    }
    if (rtype.empty()) rtype = has_interp ? "rif_interpolated" : (has_sources ? "rif_sources" : "rif_analytical");
    if (rtype == "rif_analytical") c.kind = FieldKind::Analytical;
    else if (rtype == "rif_sources") c.kind = FieldKind::Sources;
    else if (rtype == "rif_interpolated") c.kind = FieldKind::Interpolated;
    else if (rtype == "plane_waves") c.kind = FieldKind::PlaneWaves;
    else { err = "Invalid rendering_type: '" + rtype + "'. Must be one of 'rif_analytical', 'rif_sources', 'rif_interpolated' or 'plane_waves'"; return -1; }
    set_kind_defaults(c);

    std::set<std::string> seen;
    std::map<std::string, std::function<bool(const std::string &)>> num;
    auto F = [&](const char *k, double &d) { num[k] = [&d](const std::string &v) { d = std::stof(v); return true; }; };
    auto I = [&](const char *k, int &d) { num[k] = [&d](const std::string &v) { d = std::stoi(v); return true; }; };
    auto B = [&](const char *k, bool &d) {
        std::string key = k;
        num[k] = [&d, key, &err](const std::string &v) { return parse_bool(key, v, d, err); };
    };
    auto S = [&](const char *k, std::string &d) { num[k] = [&d](const std::string &v) { d = v; return true; }; };
    num["threads"] = [&](const std::string &v) { c.threads = std::stoi(v); return true; };
    I("precision", c.precision);
    num["numPhotons"] = [&](const std::string &v) { c.numPhotons = std::stoi(v); return true; };
    S("outFilePrefix", c.outFilePrefix);
    F("sigmaT", c.sigmaT); F("albedo", c.albedo); F("gVal", c.gVal);
    F("f_u", c.f_u); F("speed_u", c.speed_u); F("n_o", c.n_o);
    F("n_max", c.n_max); F("n_clip", c.n_clip); F("phi_min", c.phi_min); F("phi_max", c.phi_max); I("mode", c.mode);
    F("n_scaling", c.n_scaling); I("n_coeff", c.n_coeff); F("radius", c.radius);
    num["center1"] = [&](const std::string &v) { return parse_triple("center1", v, c.center1, err); };
    num["center2"] = [&](const std::string &v) { return parse_triple("center2", v, c.center2, err); };
    B("active1", c.active1); B("active2", c.active2); F("phase1", c.phase1); F("phase2", c.phase2);
    F("chordlength", c.chordlength); I("theta_sources", c.theta_sources); I("trans_z_sources", c.trans_z_sources);
    F("emitter_gap", c.emitter_gap); F("sensor_gap", c.sensor_gap); F("er_stepsize", c.er_stepsize);
    F("directTol", c.directTol); B("useInitializationHack", c.useInitializationHack); F("rr_weight", c.rr_weight);
    S("projectorTexture", c.projectorTexture); B("useDirect", c.useDirect); B("useAngularSampling", c.useAngularSampling);
    B("use_bounce_decomposition", c.use_bounce_decomposition); I("maxDepth", c.maxDepth); F("maxPathlength", c.maxPathlength);
    F("pathLengthMin", c.pathLengthMin); F("pathLengthMax", c.pathLengthMax); I("pathLengthBins", c.pathLengthBins);
    I("spatialX", c.spatialX); I("spatialY", c.spatialY); F("halfThetaLimit", c.halfThetaLimit);
    F("emitter_size", c.emitter_size); F("sensor_size", c.sensor_size);
    F("mediumLx", c.mediumL[0]); F("mediumRx", c.mediumR[0]);
    S("distribution", c.distribution); F("gOrKappa", c.gOrKappa);
    F("emitter_distance", c.emitter_distance); F("emitter_lens_aperture", c.emitter_lens_aperture);
    F("emitter_lens_focalLength", c.emitter_lens_focalLength); B("emitter_lens_active", c.emitter_lens_active);
    F("sensor_distance", c.sensor_distance); F("sensor_lens_aperture", c.sensor_lens_aperture);
    F("sensor_lens_focalLength", c.sensor_lens_focalLength); B("sensor_lens_active", c.sensor_lens_active);
    B("printInputs", c.printInputs); S("rifgridFile", c.rifgridFile);
    num["stricts"] = [&](const std::string &v) { return parse_bool("stricts", v, c.stricts, err); };
    // extensions
    num["rendering_type"] = [](const std::string &) { return true; };
    F("mediumLy", c.mediumL[1]); F("mediumRy", c.mediumR[1]); F("mediumLz", c.mediumL[2]); F("mediumRz", c.mediumR[2]);
    num["seed"] = [&](const std::string &v) { c.seed = std::stoull(v); return true; };
    num["renderPrecision"] = [&](const std::string &v) {
        if (v == "fp32") c.renderPrecision = SMP_PREC_FP32;
        else if (v == "mixed") c.renderPrecision = SMP_PREC_MIXED;
        else { err = "renderPrecision should be fp32 or mixed; Argument " + v + " not recognized"; return false; }
        return true;
    };
    F("sensorMarchMax", c.sensorMarchMax);
    num["stepCap"] = [&](const std::string &v) { c.stepCap = std::stoll(v); return true; };
    I("device", c.device);
    num["planeWaves"] = [&](const std::string &v) {      // "a,kx,ky,kz,phase;a,kx,ky,kz,phase"
        c.planeWaves.clear();
        for (auto &w : tokenize(v, ";")) {
            std::vector<std::string> p = tokenize(w, ",");
            if (p.size() != 5) { err = "planeWaves entries are a,kx,ky,kz,phase"; return false; }
            std::vector<double> e;
            for (auto &t : p) e.push_back(std::stod(t));
            c.planeWaves.push_back(e);
        }
        if (c.planeWaves.size() > SMP_MAX_WAVES) { err = "at most " + std::to_string(SMP_MAX_WAVES) + " plane waves"; return false; }
        return true;
    };

    for (auto &e : kv) {
        auto it = num.find(e.first);
        if (it == num.end()) {
            std::ostringstream os;
            os << "Unknown variable in the input argument:" << e.first << "\nShould be one of stricts";
            for (auto &n : num) if (n.first != "stricts") os << ", " << n.first;
            err = os.str();
            return -1;
        }
        try {
            if (!it->second(e.second)) return -1;
        } catch (const std::exception &) {
            err = "could not parse " + e.first + "=" + e.second;
            return -1;
        }
        seen.insert(e.first);
    }

    if (c.stricts) {
        std::ostringstream missing;
        auto need = [&](const char *k) { if (!seen.count(k)) missing << k << " is not specified \n"; };
        for (auto k : kCommonKeys) need(k);
        if (c.kind == FieldKind::Analytical) for (auto k : kAnalyticalKeys) need(k);
        if (c.kind == FieldKind::Sources) for (auto k : kSourcesKeys) need(k);
        if (c.kind == FieldKind::Interpolated) { for (auto k : kAnalyticalKeys) need(k); for (auto k : kInterpolatedKeys) need(k); }
        if (!missing.str().empty()) {
            err = missing.str() + "crashing as one or more inputs is absent";
            return -1;
        }
    }
    (void)kExtensionKeys;
    // sanity checks (renderer3d_sample.cpp:786-798)
    double width = c.mediumR[0] - c.mediumL[0];
    std::ostringstream bad;
    if (c.emitter_distance < 0) bad << "emitter_distance = " << c.emitter_distance << " should be strictly non-zero";
    else if (c.sensor_distance < 0) bad << "sensor_distance = " << c.sensor_distance << " should be strictly non-zero";
    else if (c.emitter_lens_active && c.emitter_distance < 1e-4) bad << "lens_active and emitter_distance = " << c.emitter_distance << ". emitter_distance should be strictly positive (>1e-4) ";
    else if (c.sensor_lens_active && c.sensor_distance < 1e-4) bad << "lens_active and sensor_distance = " << c.sensor_distance << ". sensor_distance should be strictly positive (>1e-4) ";
    else if (seen.count("emitter_gap") && (c.emitter_gap < 0 || c.emitter_gap > width)) bad << "invalid gap between the emitter and the US:" << c.emitter_gap;
    else if (seen.count("sensor_gap") && (c.sensor_gap < 0 || c.sensor_gap > width)) bad << "invalid gap between the sensor and the US:" << c.sensor_gap;
    else if (seen.count("emitter_gap") && seen.count("sensor_gap") && c.sensor_gap + c.emitter_gap > width) bad << "sum of sensor and emitter gaps is more than the medium size; sum of gaps is " << (c.sensor_gap + c.emitter_gap);
    else if (c.kind != FieldKind::Sources && c.phi_max < c.phi_min) bad << "phi_max must be greater than or equal to phi min";
    if (!bad.str().empty()) { err = bad.str(); return -1; }
    c.outputFile = c.outFilePrefix + ".pfm3d";                    // renderer3d_sample.cpp:868
    return 0;
}

// ================================================================================================
// JSON settings (simplER.cpp, settings_parser.cpp)
// ================================================================================================
int parse_json_settings(const Json &root, RenderConfig &c, std::string &err) {
    std::vector<std::string> missing;
    auto path = [&](const std::string &p) -> const Json * {
        const Json *cur = &root;
        std::string seg;
        std::istringstream is(p);
        while (std::getline(is, seg, '.')) {
            cur = cur ? cur->get(seg) : nullptr;
        }
        if (!cur) missing.push_back(p);
        return cur;
    };
    auto num = [&](const std::string &p, double &d) { const Json *j = path(p); if (j && j->kind == Json::Number) d = j->num; else if (j) missing.push_back(p + " (number)"); };
    auto inum = [&](const std::string &p, int &d) { double v = d; num(p, v); d = int(v); };
    auto lnum = [&](const std::string &p, long long &d) { double v = double(d); num(p, v); d = (long long)v; };
    auto boolean = [&](const std::string &p, bool &d) { const Json *j = path(p); if (j && j->kind == Json::Bool) d = j->b; else if (j) missing.push_back(p + " (bool)"); };
    auto str = [&](const std::string &p, std::string &d) { const Json *j = path(p); if (j && j->kind == Json::String) d = j->str; else if (j) missing.push_back(p + " (string)"); };

    boolean("stricts", c.stricts);
    std::string rtype = "rif_analytical";
    str("rendering_type", rtype);
    if (rtype == "rif_analytical") c.kind = FieldKind::Analytical;
    else if (rtype == "rif_sources") c.kind = FieldKind::Sources;
    else if (rtype == "rif_interpolated") c.kind = FieldKind::Interpolated;
    else if (rtype == "plane_waves") c.kind = FieldKind::PlaneWaves;
    else { err = "Invalid rendering_type: '" + rtype + "'. Must be one of 'rif_analytical', 'rif_sources', or 'rif_interpolated'."; return -1; }
    set_kind_defaults(c);
    inum("threads", c.threads);
    num("emitter_gap", c.emitter_gap);
    num("sensor_gap", c.sensor_gap);
    boolean("use_bounce_decomposition", c.use_bounce_decomposition);
    boolean("print_inputs", c.printInputs);
    str("projector_texture", c.projectorTexture);
    num("film_parameters.path_length.min", c.pathLengthMin);
    num("film_parameters.path_length.max", c.pathLengthMax);
    inum("film_parameters.path_length.bins", c.pathLengthBins);
    inum("film_parameters.spatial.x", c.spatialX);
    inum("film_parameters.spatial.y", c.spatialY);
    num("adoc_geometry_parameters.half_theta_limit", c.halfThetaLimit);
    num("adoc_geometry_parameters.emitter_size", c.emitter_size);
    num("adoc_geometry_parameters.sensor_size", c.sensor_size);
    num("adoc_geometry_parameters.emitter_distance", c.emitter_distance);
    num("adoc_geometry_parameters.sensor_distance", c.sensor_distance);
    num("scattering_parameters.sigma_t", c.sigmaT);
    num("scattering_parameters.albedo", c.albedo);
    num("scattering_parameters.g_val", c.gVal);
    lnum("rendering_parameters.num_photons", c.numPhotons);
    boolean("rendering_parameters.use_direct", c.useDirect);
    inum("rendering_parameters.max_depth", c.maxDepth);
    num("rendering_parameters.max_pathlength", c.maxPathlength);
    boolean("rendering_parameters.use_angular_sampling", c.useAngularSampling);
    str("importance_sampling_parameters.distribution", c.distribution);
    num("importance_sampling_parameters.g_or_kappa", c.gOrKappa);
    num("scene_parameters.medium_lx", c.mediumL[0]);
    num("scene_parameters.medium_rx", c.mediumR[0]);
    num("lens_parameters.emitter_lens_aperture", c.emitter_lens_aperture);
    num("lens_parameters.emitter_lens_focal_length", c.emitter_lens_focalLength);
    boolean("lens_parameters.emitter_lens_active", c.emitter_lens_active);
    num("lens_parameters.sensor_lens_aperture", c.sensor_lens_aperture);
    num("lens_parameters.sensor_lens_focal_length", c.sensor_lens_focalLength);
    boolean("lens_parameters.sensor_lens_active", c.sensor_lens_active);
    // rif_parameters (rif_base.h:62-76 and the subclasses' AnyMap constructors)
    num("rif_parameters.f_u", c.f_u);
    num("rif_parameters.speed_u", c.speed_u);
    num("rif_parameters.n_o", c.n_o);
    num("rif_parameters.direct_to_l", c.directTol);
    num("rif_parameters.rr_weight", c.rr_weight);
    num("rif_parameters.er_stepsize", c.er_stepsize);
    inum("rif_parameters.precision", c.precision);
    boolean("rif_parameters.use_initialization_hack", c.useInitializationHack);
    if (c.kind == FieldKind::Analytical || c.kind == FieldKind::Interpolated) {
        num("rif_parameters.n_max", c.n_max);
        num("rif_parameters.n_clip", c.n_clip);
        num("rif_parameters.phi_min", c.phi_min);
        num("rif_parameters.phi_max", c.phi_max);
        inum("rif_parameters.mode", c.mode);
    }
    if (c.kind == FieldKind::Interpolated) str("rif_parameters.rif_grid_file", c.rifgridFile);
    if (c.kind == FieldKind::Sources) {
        num("rif_parameters.n_scaling", c.n_scaling);
        inum("rif_parameters.n_coeff", c.n_coeff);
        num("rif_parameters.radius", c.radius);
        for (int k = 0; k < 2; ++k) {
            const Json *a = path(k == 0 ? "rif_parameters.center1" : "rif_parameters.center2");
            double *dst = k == 0 ? c.center1 : c.center2;
            if (a && a->kind == Json::Array && a->arr.size() == 3)
                for (int i = 0; i < 3; ++i) dst[i] = a->arr[i].num;
        }
        boolean("rif_parameters.active1", c.active1);
        boolean("rif_parameters.active2", c.active2);
        num("rif_parameters.phase1", c.phase1);
        num("rif_parameters.phase2", c.phase2);
        num("rif_parameters.chordlength", c.chordlength);
        inum("rif_parameters.theta_sources", c.theta_sources);
        inum("rif_parameters.trans_z_sources", c.trans_z_sources);
    }
    if (!missing.empty()) {
        std::ostringstream os;
        os << "Error occurred while starting simplER renderer: missing or mistyped ";
        for (size_t i = 0; i < missing.size(); ++i) os << (i ? ", " : "") << missing[i];
        if (c.stricts) { err = os.str(); return -1; }
    }
    // output name <rendering_type>_<YYYY_MM_DD_HH_MM> (settings_parser.cpp:87-93)
    std::time_t t = std::time(nullptr);
    std::tm tm = *std::localtime(&t);
    char dt[32];
    std::strftime(dt, sizeof(dt), "%Y_%m_%d_%H_%M", &tm);
    c.outFilePrefix = rtype + "_" + dt;
    c.outputFile = c.outFilePrefix + ".pfm3d";
    double width = c.mediumR[0] - c.mediumL[0];
    if (c.emitter_distance < 0 || c.sensor_distance < 0 || c.emitter_gap < 0 || c.emitter_gap > width ||
        c.sensor_gap < 0 || c.sensor_gap > width || c.sensor_gap + c.emitter_gap > width) {
        err = "settings fail the sanity checks of settings_parser.cpp:156-184";
        return -1;
    }
    return 0;
}

void print_inputs(const RenderConfig &c, std::ostream &os) {
    os << "numPhotons = " << c.numPhotons << "\n"
       << "outFilePrefix = " << c.outFilePrefix << "\n"
       << "sigmaT = " << c.sigmaT << "\n"
       << "albedo = " << c.albedo << "\n"
       << "gVal = " << c.gVal << "\n";
    if (c.kind == FieldKind::Sources) {
        os << "f_u = " << c.f_u << "\nspeed_u = " << c.speed_u << "\nn_o = " << c.n_o << "\nn_scaling = " << c.n_scaling
           << "\nn_coeff = " << c.n_coeff << "\nradius = " << c.radius << "\ncenter1 = (" << c.center1[0] << ", "
           << c.center1[1] << ", " << c.center1[2] << ")\ncenter2 = (" << c.center2[0] << ", " << c.center2[1] << ", "
           << c.center2[2] << ")\nactive1 = " << c.active1 << "\nactive2 = " << c.active2 << "\nphase1 = " << c.phase1
           << "\nphase2 = " << c.phase2 << "\nchordlength = " << c.chordlength << "\ntheta_sources = "
           << c.theta_sources << "\ntrans_z_sources = " << c.trans_z_sources << "\n";
    } else {
        os << "f_u = " << c.f_u << "\nspeed_u = " << c.speed_u << "\nn_o = " << c.n_o << "\nn_max = " << c.n_max
           << "\nn_clip = " << c.n_clip << "\nphi_min = " << c.phi_min << "\nphi_max = " << c.phi_max
           << "\nmode = " << c.mode << "\n";
    }
    os << "emitter_gap = " << c.emitter_gap << "\nsensor_gap = " << c.sensor_gap << "\nprojectorTexture = "
       << c.projectorTexture << "\nuseDirect = " << c.useDirect << "\nuseAngularSampling= " << c.useAngularSampling
       << "\nuse_bounce_decomposition= " << c.use_bounce_decomposition << "\nmaxDepth = " << c.maxDepth
       << "\nmaxPathlength = " << c.maxPathlength << "\nTotal medium length = " << (c.mediumR[0] - c.mediumL[0])
       << "\npathLengthMin = " << c.pathLengthMin << "\npathLengthMax = " << c.pathLengthMax
       << "\npathLengthBins = " << c.pathLengthBins << "\nspatialX = " << c.spatialX << "\nspatialY = " << c.spatialY
       << "\nhalfThetaLimit = " << c.halfThetaLimit << "\nemitter_size = " << c.emitter_size
       << "\nsensor_size = " << c.sensor_size << "\ndistribution = " << c.distribution << "\ngOrKappa = "
       << c.gOrKappa << "\nemitter_distance = " << c.emitter_distance << "\nemitter_lens_aperture = "
       << c.emitter_lens_aperture << "\nemitter_lens_focalLength = " << c.emitter_lens_focalLength
       << "\nemitter_lens_active = " << c.emitter_lens_active << "\nsensor_distance = " << c.sensor_distance
       << "\nsensor_lens_aperture = " << c.sensor_lens_aperture << "\nsensor_lens_focalLength = "
       << c.sensor_lens_focalLength << "\nsensor_lens_active = " << c.sensor_lens_active << "\n";
    if (c.kind == FieldKind::Interpolated) os << "rifgridFile = " << c.rifgridFile << "\n";
    os << "printInputs = " << c.printInputs << "\n";
}

// ================================================================================================
// scene assembly (renderer3d_sample.cpp:801-866)
// ================================================================================================
int build_descs(const RenderConfig &c, Built &b, std::string &err) {
    std::memset(&b.scene, 0, sizeof(b.scene));
    std::memset(&b.field, 0, sizeof(b.field));
    std::memset(&b.opts, 0, sizeof(b.opts));
    if (!read_pfm_texture(c.projectorTexture, b.texture, err)) return SMP_ERR_BAD_ARG;
    smp_scene_desc &s = b.scene;
    s.ior = c.ior;
    for (int i = 0; i < 3; ++i) { s.medium_l[i] = c.mediumL[i]; s.medium_r[i] = c.mediumR[i]; }
    s.light_origin[0] = c.mediumR[0] + c.emitter_distance;
    const float light_angle = float(3.14159265358979323846);         // lightAngle = M_PI (Float)
    s.light_dir[0] = std::cos(light_angle);
    s.light_dir[1] = std::sin(light_angle);
    s.half_theta_limit = c.halfThetaLimit;
    s.light_plane[0] = s.light_plane[1] = c.emitter_size;
    s.Li = 75000.0;
    s.tex_x = b.texture.x;
    s.tex_y = b.texture.y;
    s.texture = b.texture.texels.data();
    s.emitter_lens_origin[0] = c.mediumR[0];
    s.emitter_lens_aperture = c.emitter_lens_aperture;
    s.emitter_lens_focal_length = c.emitter_lens_focalLength;
    s.emitter_lens_active = c.emitter_lens_active;
    s.use_bounce_decomposition = c.use_bounce_decomposition;
    s.view_origin[0] = c.mediumL[0] - c.sensor_distance;
    s.view_dir[0] = -1.0;
    s.view_horizontal[1] = -1.0;
    s.view_plane[0] = s.view_plane[1] = c.sensor_size;
    s.pathlength_range[0] = c.pathLengthMin;
    s.pathlength_range[1] = c.pathLengthMax;
    s.sensor_lens_origin[0] = c.mediumL[0];
    s.sensor_lens_aperture = c.sensor_lens_aperture;
    s.sensor_lens_focal_length = c.sensor_lens_focalLength;
    s.sensor_lens_active = c.sensor_lens_active;
    s.x_res = c.spatialX;
    s.y_res = c.spatialY;
    s.z_res = c.pathLengthBins;
    b.medium.sigma_t = c.sigmaT;
    b.medium.albedo = c.albedo;
    b.medium.g = c.gVal;

    smp_field_desc &f = b.field;
    f.precision = c.precision;
    f.f_u = c.f_u;
    f.speed_u = c.speed_u;
    f.n_o = c.n_o;
    f.er_stepsize = c.er_stepsize;
    f.egap_end_x = double(float(c.mediumR[0]) - float(c.emitter_gap));   // egap_end_loc_x in Float
    f.sgap_begin_x = double(float(c.mediumL[0]) + float(c.sensor_gap));
    f.direct_tol = c.directTol;
    f.rr_weight = c.rr_weight;
    f.use_initialization_hack = c.useInitializationHack;
    f.mode = c.mode;
    f.n_max = c.n_max;
    f.n_clip = c.n_clip;
    f.phi_min = c.phi_min;
    f.phi_max = c.phi_max;
    f.n_coeff = c.n_coeff;
    f.theta_sources = c.theta_sources;
    f.trans_z_sources = c.trans_z_sources;
    f.active1 = c.active1;
    f.active2 = c.active2;
    f.n_scaling = c.n_scaling;
    f.radius = c.radius;
    f.chordlength = c.chordlength;
    f.phase1 = c.phase1;
    f.phase2 = c.phase2;
    for (int i = 0; i < 3; ++i) { f.center1[i] = c.center1[i]; f.center2[i] = c.center2[i]; }
    switch (c.kind) {
        case FieldKind::Analytical: f.type = SMP_FIELD_BESSEL; break;
        case FieldKind::Sources: f.type = SMP_FIELD_SOURCES; break;
        case FieldKind::PlaneWaves:
            f.type = SMP_FIELD_PLANEWAVE;
            f.n_waves = int(c.planeWaves.size());
            for (size_t i = 0; i < c.planeWaves.size(); ++i) {
                f.wave_amp[i] = c.planeWaves[i][0];
                for (int j = 0; j < 3; ++j) f.wave_k[i][j] = c.planeWaves[i][1 + j];
                f.wave_phase[i] = c.planeWaves[i][4];
            }
            break;
        case FieldKind::Interpolated: {
            f.type = SMP_FIELD_SPLINE;
            Vol v;
            if (!read_vol(c.rifgridFile, v, err)) return SMP_ERR_BAD_ARG;
            b.coeff.resize(v.data.size());
            int32_t n[3] = {v.n[0], v.n[1], v.n[2]};
            int rc = smp_spline_prefilter(v.data.data(), n, b.coeff.data());
            if (rc) { err = smp_last_error(); return rc; }
            for (int i = 0; i < 3; ++i) { f.grid_n[i] = v.n[i]; f.grid_min[i] = v.min[i]; f.grid_max[i] = v.max[i]; }
            f.grid_coeff = b.coeff.data();
            break;
        }
    }
    smp_render_opts &o = b.opts;
    o.max_depth = c.maxDepth;
    o.use_direct = c.useDirect;
    o.use_angular_sampling = c.useAngularSampling;
    o.rng = SMP_RNG_PHILOX;
    o.precision = c.renderPrecision;
    o.device = c.device;
    o.max_pathlength = c.maxPathlength;
    o.seed = c.seed;
    o.step_cap = c.stepCap;
    o.sensor_march_max = c.sensorMarchMax;
    return SMP_OK;
}

void print_descs(const Built &b, std::ostream &os) {
    const smp_scene_desc &s = b.scene;
    const smp_field_desc &f = b.field;
    os << std::setprecision(9);
    os << "scene.medium_l = " << s.medium_l[0] << " " << s.medium_l[1] << " " << s.medium_l[2] << "\n";
    os << "scene.medium_r = " << s.medium_r[0] << " " << s.medium_r[1] << " " << s.medium_r[2] << "\n";
    os << "scene.light_origin = " << s.light_origin[0] << " " << s.light_origin[1] << " " << s.light_origin[2] << "\n";
    os << "scene.view_origin = " << s.view_origin[0] << " " << s.view_origin[1] << " " << s.view_origin[2] << "\n";
    os << "scene.texture = " << s.tex_x << " x " << s.tex_y << "\n";
    os << "scene.film = " << s.x_res << " " << s.y_res << " " << s.z_res << "\n";
    os << "scene.pathlength_range = " << s.pathlength_range[0] << " " << s.pathlength_range[1] << "\n";
    os << "medium = " << b.medium.sigma_t << " " << b.medium.albedo << " " << b.medium.g << "\n";
    os << "field.type = " << f.type << "\nfield.mode = " << f.mode << "\nfield.f_u = " << f.f_u
       << "\nfield.n_max = " << f.n_max << "\nfield.egap_end_x = " << f.egap_end_x << "\nfield.sgap_begin_x = "
       << f.sgap_begin_x << "\nfield.er_stepsize = " << f.er_stepsize << "\nfield.precision = " << f.precision << "\n";
    os << "opts.use_direct = " << b.opts.use_direct << "\nopts.use_angular_sampling = " << b.opts.use_angular_sampling
       << "\nopts.max_depth = " << b.opts.max_depth << "\nopts.precision = " << b.opts.precision << "\n";
}

int run(const RenderConfig &c, std::ostream &log, std::string &err) {
    Built b;
    int rc = build_descs(c, b, err);
    if (rc) return rc;
    std::vector<double> film(size_t(c.spatialX) * c.spatialY * c.pathLengthBins, 0.0);
    smp_stats st;
    std::memset(&st, 0, sizeof(st));
    rc = smp_render(&b.scene, &b.medium, &b.field, &b.opts, c.numPhotons, film.data(), &st);
    if (rc) { err = smp_last_error(); return rc; }
    log << "numphotons = " << c.numPhotons << "\nphotons traced = " << st.photons << ", ER steps = " << st.er_steps
        << ", kernel " << st.kernel_ms << " ms\n";
    if (!write_pfm3d(c.outputFile, c.spatialX, c.spatialY, c.pathLengthBins, film.data(), err)) return SMP_ERR_BAD_ARG;
    return SMP_OK;
}

// ================================================================================================
// merging (helperScripts/mergeMultipleRenderings.cpp:207-231, with photon weights)
// ================================================================================================
bool merge_films(const std::vector<const std::vector<double> *> &films, const std::vector<double> &photons,
                 std::vector<double> &out, std::string &err) {
    if (films.empty() || films.size() != photons.size()) { err = "one photon count per film"; return false; }
    double total = 0.0;
    for (double n : photons) {
        if (!(n >= 0.0)) { err = "photon counts must be non-negative"; return false; }
        total += n;
    }
    if (!(total > 0.0)) { err = "photon counts sum to zero"; return false; }
    const size_t n = films[0]->size();
    out.assign(n, 0.0);
    for (size_t i = 0; i < films.size(); ++i) {
        if (films[i]->size() != n) { err = "film sizes differ"; return false; }
        const double w = photons[i] / total;
        for (size_t k = 0; k < n; ++k) out[k] += w * (*films[i])[k];
    }
    return true;
}

// Image2::writePFM's layout (rows bottom first), the inverse of read_pfm_texture
bool write_pfm_texture(const std::string &path, const Texture &t, std::string &err) {
    std::ofstream f(path, std::ios::binary);
    if (!f) { err = "Problem writing output file " + path; return false; }
    f << "Pf" << '\n' << t.x << ' ' << t.y << '\n' << static_cast<float>(-1.0) << '\n';
    for (int i = 0; i < t.y; ++i)
        f.write(reinterpret_cast<const char *>(&t.texels[size_t(t.y - i - 1) * t.x]), std::streamsize(size_t(t.x) * sizeof(double)));
    if (!f) { err = "Problem writing output file " + path; return false; }
    return true;
}

bool merge_reference_bins(const std::string &prefix, int renderings, int bins, const std::vector<double> &photons,
                          std::string &err) {
    if (renderings < 1 || bins < 1) { err = "renderings and pathLengthBins must be positive"; return false; }
    std::vector<double> w = photons;
    if (w.empty()) w.assign(size_t(renderings), 1.0);
    if (int(w.size()) != renderings) { err = "photons= needs one count per rendering"; return false; }
    for (int j = 0; j < bins; ++j) {
        std::vector<Texture> tex(static_cast<size_t>(renderings));
        std::vector<const std::vector<double> *> films;
        for (int i = 0; i < renderings; ++i) {
            if (!read_pfm_texture(prefix + "_" + std::to_string(i) + "_" + std::to_string(j) + ".pfm", tex[i], err)) return false;
            if (tex[i].x != tex[0].x || tex[i].y != tex[0].y) { err = "image sizes differ in bin " + std::to_string(j); return false; }
            films.push_back(&tex[i].texels);
        }
        Texture out;
        out.x = tex[0].x;
        out.y = tex[0].y;
        if (!merge_films(films, w, out.texels, err)) return false;
        if (!write_pfm_texture(prefix + "_mean_" + std::to_string(j) + ".pfm", out, err)) return false;
    }
    return true;
}

}  // namespace smp_host
