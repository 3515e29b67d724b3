// smp_host.h -- the C++ host side of the reference's front-ends, over the C ABI.
//
//   * file formats: the PFM texture reader (renderer/include/image.h:183-245), the PFM3D writer and
//     reader (renderer/src/image.cpp:161-206, renderer/include/image.h:374-436) and the .vol grid
//     reader (renderer/include/spline.h:115-162);
//   * the key=value front-end of renderer/samples/renderer3d_sample.cpp (same keys, defaults,
//     strict mode, sanity checks and scene geometry) and the JSON settings of simplER.cpp /
//     renderer/src/settings_parser.cpp;
//   * build_descs: a RenderConfig to the smp_* descriptors of include/simpler_b200.h.
#pragma once
#include <map>
#include <ostream>
#include <string>
#include <vector>

#include "../../../include/simpler_b200.h"

namespace smp_host {

// ---- files ------------------------------------------------------------------------------------------
struct Texture {
    int x = 0, y = 0;
    std::vector<double> texels;   // y * x + x, rows bottom-to-top flipped as the reference stores them
};
bool read_pfm_texture(const std::string &path, Texture &out, std::string &err);
bool write_pfm3d(const std::string &path, int X, int Y, int Z, const double *film, std::string &err);
bool read_pfm3d(const std::string &path, int &X, int &Y, int &Z, std::vector<double> &film, std::string &err);

struct Vol {
    int n[3] = {0, 0, 0};
    double min[3] = {0, 0, 0}, max[3] = {0, 0, 0};
    std::vector<float> data;      // x + n0 * (y + n1 * z)
};
bool read_vol(const std::string &path, Vol &out, std::string &err);
bool write_vol(const std::string &path, const Vol &v, std::string &err);

// ---- JSON ---------------------------------------------------------------------------------------------
struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::map<std::string, Json> obj;
    const Json *get(const std::string &key) const;
};
bool parse_json(const std::string &text, Json &out, std::string &err);

// ---- configuration -------------------------------------------------------------------------------
enum class FieldKind { Analytical, Sources, Interpolated, PlaneWaves };

struct RenderConfig {
    FieldKind kind = FieldKind::Analytical;
    bool stricts = false;
    int threads = -1;
    int precision = 8;
    long long numPhotons = 500;
    std::string outFilePrefix = "USOCTRendering";
    double sigmaT = 0.0, albedo = 1.0, gVal = 0.0;
    double ior = 1.3333;
    // field (analytical)
    double f_u = 848e3, speed_u = 1500.0, n_o = 1.3333, n_max = 1e-3, n_clip = 1e-3;
    double phi_min = 1.5707963267948966, phi_max = 1.5707963267948966;
    int mode = 0;
    // field (sources)
    double n_scaling = 0.05e-3, radius = 2 * 25.4e-3, phase1 = 0.0, phase2 = 0.0, chordlength = 0.5 * 25.4e-3;
    int n_coeff = 1, theta_sources = 100, trans_z_sources = 501;
    double center1[3] = {-2 * 25.4e-3, 0, 0}, center2[3] = {-2 * 25.4e-3, 0, 0};
    bool active1 = true, active2 = true;
    // field (interpolated)
    std::string rifgridFile = "us";
    // plane waves (extension): a, kx, ky, kz, phase per wave
    std::vector<std::vector<double>> planeWaves;
    // march
    double emitter_gap = 0.0, sensor_gap = 0.0, er_stepsize = 1e-3, directTol = 1e-5, rr_weight = 1e-2;
    bool useInitializationHack = true;
    std::string projectorTexture = "White.pfm";
    bool useDirect = false, useAngularSampling = true, use_bounce_decomposition = true;
    int maxDepth = -1;
    double maxPathlength = -1.0;
    // film
    double pathLengthMin = 0.0, pathLengthMax = 64.0;
    int pathLengthBins = 128, spatialX = 128, spatialY = 128;
    // geometry
    double halfThetaLimit = 12.8e-3, emitter_size = 0.002, sensor_size = 0.002;
    double mediumL[3] = {-0.015, -5.0, -5.0}, mediumR[3] = {0.015, 5.0, 5.0};
    std::string distribution = "vmf";
    double gOrKappa = 4.0;
    double emitter_distance = 0.0, emitter_lens_aperture = 0.015, emitter_lens_focalLength = 0.015;
    bool emitter_lens_active = false;
    double sensor_distance = 0.0, sensor_lens_aperture = 0.015, sensor_lens_focalLength = 0.015;
    bool sensor_lens_active = false;
    bool printInputs = true;
    // B200 extensions
    unsigned long long seed = 0;
    int renderPrecision = SMP_PREC_FP32;
    double sensorMarchMax = 0.0;
    long long stepCap = 0;
    int device = 0;
    std::string outputFile;            // resolved output path (.pfm3d)
};

// renderer3d_sample.cpp:250-798: returns 0, or -1 with err filled (the reference returns -1 / exits)
int parse_cli(int argc, const char *const *argv, RenderConfig &cfg, std::string &err);
// simplER.cpp:21-60 + settings_parser.cpp:3-153
int parse_json_settings(const Json &root, RenderConfig &cfg, std::string &err);
// renderer3d_sample.cpp:721-784
void print_inputs(const RenderConfig &cfg, std::ostream &os);

// scene geometry of renderer3d_sample.cpp:801-866; the texture / grid files are read here
struct Built {
    smp_scene_desc scene;
    smp_medium_desc medium;
    smp_field_desc field;
    smp_render_opts opts;
    Texture texture;
    std::vector<float> coeff;
};
int build_descs(const RenderConfig &cfg, Built &out, std::string &err);
void print_descs(const Built &b, std::ostream &os);

// whole run: build, render (smp_render), write <outputFile>; returns 0 or a negative smp_status
int run(const RenderConfig &cfg, std::ostream &log, std::string &err);

// ---- merging renders (helperScripts/mergeMultipleRenderings.cpp) ----------------------------------
// Photon-weighted mean sum_i N_i film_i / sum_i N_i of equally shaped films, in place into out.
// The reference helper's running mean (mean (i+1) + x_i) / (i+2) over-weights its first rendering;
// with equal N_i this is the plain mean.
bool merge_films(const std::vector<const std::vector<double> *> &films, const std::vector<double> &photons,
                 std::vector<double> &out, std::string &err);
// the helper's file set <prefix>_<i>_<j>.pfm (rendering i, path-length bin j) -> <prefix>_mean_<j>.pfm
bool merge_reference_bins(const std::string &prefix, int renderings, int bins, const std::vector<double> &photons,
                          std::string &err);
bool write_pfm_texture(const std::string &path, const Texture &t, std::string &err);

}  // namespace smp_host
