// oracle/oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker). A scalar CPU restatement of the
// reference's photon march, used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
// leg. It is never linked into, loaded by or called from the product library.
//
// Every function cites the reference file:line it restates (paths relative to the simplEr root).
// Templated on R: R = float reproduces the reference's single-precision CPU build (Float = float,
// CMakeLists.txt USE_DOUBLE_PRECISION 0) including its double-precision Bessel/RIF arithmetic;
// R = double is the FP64 oracle.
//
// Deliberate, documented deviations from the reference (all unreachable in the reference's
// well-formed runs, or undefined behaviour there):
//   * a per-photon cap on er_step calls (the reference has none) ends a photon with END_STEP_CAP;
//   * a non-finite position ends a photon with END_NAN (the reference indexes out of bounds);
//   * float->integer conversion of an out-of-range or infinite step count yields INT64_MIN, the
//     value x86-64 (cvttss2si) produces for the reference's own conversion;
//   * the 3-D spline mirrors out-of-range taps like the 1-D/2-D evaluators (spline.h:611-657)
//     where the reference's 3-D evaluator reads outside its coefficient array (spline.h:308-356).
#include "../include/simpler_b200.h"
#include "rng_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#include <omp.h>

namespace orc {

// ---- constants (renderer/include/constants.h:16-69, float build) ---------------------------------
static const float kEpsF = 1.19209290e-07f;     // M_EPSILON
static const float kMaxF = 3.40282347e+38f;     // M_MAX

template <typename R> struct K;
template <> struct K<float> {
    static float pi() { return 3.14159265358979323846f; }
    static float half() { return 0.5f; }
};
template <> struct K<double> {
    static double pi() { return 3.14159265358979323846; }
    static double half() { return 0.5; }
};

// x86-64 semantics of (long) for the reference's step counts (traceTillBlock :391).
static inline int64_t to_i64_x86(double v) {
    if (!(v >= -9.2233720368547758e18 && v < 9.2233720368547758e18)) return INT64_MIN;
    return static_cast<int64_t>(v);
}

// ---- small vector with tvector.h semantics (renderer/include/tvector.h:220-420) ------------------
template <typename R> struct V3 {
    R x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    R &operator[](int i) { return (&x)[i]; }
    R operator[](int i) const { return (&x)[i]; }
    V3 operator+(const V3 &v) const { return V3(x + v.x, y + v.y, z + v.z); }
    V3 operator-(const V3 &v) const { return V3(x - v.x, y - v.y, z - v.z); }
    V3 operator-() const { return V3(-x, -y, -z); }
    V3 &operator+=(const V3 &v) { x += v.x; y += v.y; z += v.z; return *this; }
    V3 operator*(R f) const { return V3(x * f, y * f, z * f); }
    V3 &operator*=(R f) { x *= f; y *= f; z *= f; return *this; }
    V3 operator/(R f) const { R r = R(1) / f; return V3(x * r, y * r, z * r); }   // :292-297
    R lengthSquared() const { return x * x + y * y + z * z; }
    R length() const { return std::sqrt(lengthSquared()); }
    void normalize() {                                                            // :351-358
        if (!(x == 0 && y == 0 && z == 0)) { R t = length(); x = x / t; y = y / t; z = z / t; }
    }
    bool finite() const { return std::isfinite(x) && std::isfinite(y) && std::isfinite(z); }
};
template <typename R> inline V3<R> operator*(R f, const V3<R> &v) { return v * f; }
template <typename R> inline R dot(const V3<R> &a, const V3<R> &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename R> inline R absDot(const V3<R> &a, const V3<R> &b) { return std::abs(dot(a, b)); }
template <typename R> inline V3<R> cross(const V3<R> &a, const V3<R> &b) {
    return V3<R>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename R> inline V3<R> mk(const double *v) { return V3<R>(R(v[0]), R(v[1]), R(v[2])); }

// ---- uniform source ------------------------------------------------------------------------------
struct Uniforms {
    int mode = SMP_RNG_SFMT;
    Sfmt19937 sfmt;
    PhiloxStream philox;
    const float *stream = nullptr;
    int64_t pos = 0, end = 0;
    int32_t draws = 0;
    bool exhausted = false;
    float operator()() {
        ++draws;
        if (mode == SMP_RNG_SFMT) return sfmt.next_float();
        if (mode == SMP_RNG_PHILOX) return philox.next_float();
        if (pos < end) return stream[pos++];
        exhausted = true;
        return 0.5f;
    }
};

// ---- refractive-index fields ---------------------------------------------------------------------
template <typename R> struct Field {
    int type = SMP_FIELD_BESSEL;
    R n_o, egap, sgap, k_r, n_max;
    int mode = 0;
    // FUS sources (rif_sources.h)
    int n_coeff = 1, nsources = 0;
    bool active1 = false, active2 = false;
    R n_scaling = 0, phase1 = 0, phase2 = 0;
    std::vector<V3<R>> centers1, centers2;
    // plane waves
    int n_waves = 0;
    R amp[SMP_MAX_WAVES], phase[SMP_MAX_WAVES];
    V3<R> kvec[SMP_MAX_WAVES];
    // spline
    int N[3] = {0, 0, 0};
    R xmin[3], xres[3];
    const float *coeff = nullptr;
    // Conditioning deviation: the coefficients (~n) are summed as offsets from their mean, as the
    // B-spline weights sum to 1 and their derivatives to 0. The reference sums the raw values in
    // Float and loses about four digits of a 1e-3 gradient to cancellation (spline.h:324-356).
    std::vector<R> delta;
    R base = 0;
    // fixed axes of rif_base.h:144-154
    V3<R> axis_uz = V3<R>(R(-1), R(0), R(0)), axis_ux = V3<R>(R(0), R(0), R(1)), p_u;

    void init(const smp_field_desc &f) {
        type = f.type;
        n_o = R(f.n_o);
        egap = R(f.egap_end_x);
        sgap = R(f.sgap_begin_x);
        // rif_base.h:149-153: lambda = c/f; k = 2*pi/lambda, in Float
        R lambda = R(f.speed_u) / R(f.f_u);
        k_r = (R(2) * K<R>::pi()) / lambda;
        n_max = R(f.n_max);
        mode = f.mode;
        if (type == SMP_FIELD_SOURCES) init_sources(f);
        if (type == SMP_FIELD_PLANEWAVE) {
            n_waves = f.n_waves;
            for (int i = 0; i < n_waves; ++i) {
                amp[i] = R(f.wave_amp[i]);
                phase[i] = R(f.wave_phase[i]);
                kvec[i] = mk<R>(f.wave_k[i]);
            }
        }
        if (type == SMP_FIELD_SPLINE) {
            for (int i = 0; i < 3; ++i) {
                N[i] = f.grid_n[i];
                xmin[i] = R(f.grid_min[i]);
                xres[i] = R(N[i] - 1) / (R(f.grid_max[i]) - R(f.grid_min[i]));   // spline.h:146
            }
            coeff = f.grid_coeff;
            size_t n = size_t(N[0]) * N[1] * N[2];
            double mean = 0.0;
            for (size_t i = 0; i < n; ++i) mean += coeff[i];
            mean /= double(n);
            base = R(float(f.grid_offset + mean));
            delta.resize(n);
            for (size_t i = 0; i < n; ++i) delta[i] = R(double(coeff[i]) + f.grid_offset - double(float(f.grid_offset + mean)));
        }
    }

    // source placement, rif_sources.h:156-198
    void init_sources(const smp_field_desc &f) {
        n_coeff = f.n_coeff;
        active1 = f.active1 != 0;
        active2 = f.active2 != 0;
        n_scaling = R(f.n_scaling);
        phase1 = R(f.phase1);
        phase2 = R(f.phase2);
        R radius = R(f.radius), chord = R(f.chordlength);
        R theta_min = -std::asin(chord / (R(2) * radius));
        R theta_max = std::asin(chord / (R(2) * radius));
        R zmin = -chord / R(2), zmax = chord / R(2);
        if (f.theta_max > f.theta_min) {      // explicit arcs (scene.h:78-95 constructor form)
            theta_min = R(f.theta_min); theta_max = R(f.theta_max);
            zmin = R(f.trans_z_min); zmax = R(f.trans_z_max);
        }
        int nt = f.theta_sources, nz = f.trans_z_sources;
        nsources = nt * nz;
        R theta_diff = (theta_max - theta_min) / R(nt - 1);
        R z_diff = (zmax - zmin) / R(nz - 1);
        centers1.assign(nsources, V3<R>());
        centers2.assign(nsources, V3<R>());
        V3<R> c1 = mk<R>(f.center1), c2 = mk<R>(f.center2);
        for (int i = 0; i < nt; ++i) {
            R theta = theta_min + theta_diff * R(i);
            R xval = radius * (R(1) - std::cos(theta));
            R yval = radius * std::sin(theta);
            for (int j = 0; j < nz; ++j) {
                int index = i + j * nt;
                centers1[index] = V3<R>(zmin + z_diff * R(j) + c1.x, yval + c1.y, xval + c1.z);
                centers2[index] = V3<R>(zmin + z_diff * R(j) + c2.x, xval + c2.y, yval + c2.z);
            }
        }
    }

    bool outside_gap(const V3<R> &p) const { return (p.x > egap) || (p.x < sgap); }   // rif_base.h:134-137

    // US::RIF (cuda_scene.cuh:463-471; CPU math scene.cpp:141-160, 206-215)
    double RIF(const V3<R> &p, R scaling) const {
        if (outside_gap(p)) return double(n_o);
        switch (type) {
            case SMP_FIELD_BESSEL: return bessel_RIF(p, scaling);
            case SMP_FIELD_SOURCES: return fus_RIF(p);
            case SMP_FIELD_PLANEWAVE: return wave_RIF(p, scaling);
            default: return double(spline_value(p));
        }
    }
    // US::dRIF (cuda_scene.cuh:473-481; CPU math scene.cpp:163-195, 218-257)
    V3<R> dRIF(const V3<R> &p, R scaling) const {
        if (outside_gap(p)) return V3<R>(R(0), R(0), R(0));
        switch (type) {
            case SMP_FIELD_BESSEL: return bessel_dRIF(p, scaling);
            case SMP_FIELD_SOURCES: return fus_dRIF(p);
            case SMP_FIELD_PLANEWAVE: return wave_dRIF(p, scaling);
            default: return spline_gradient(p);
        }
    }

    // scene.cpp:206-215
    double bessel_RIF(const V3<R> &p, R scaling) const {
        V3<R> p_axis = p_u + dot(p - p_u, axis_uz) * axis_uz;
        R r = (p - p_axis).length();
        R dotp = dot(p - p_axis, axis_ux);
        R detp = dot(cross(axis_ux, p - p_axis), axis_uz);
        R phi = std::atan2(detp, dotp);
        return double(n_o) + double(n_max * scaling) * jn(mode, double(k_r * r)) *
                                 double(std::cos(R(mode) * phi));
    }
    // scene.cpp:218-257
    V3<R> bessel_dRIF(const V3<R> &q, R scaling) const {
        V3<R> p_axis = p_u + dot(q - p_u, axis_uz) * axis_uz;
        V3<R> p = q - p_axis;
        R r = p.length();
        R dotp = dot(p, axis_ux);
        R detp = dot(cross(axis_ux, p), axis_uz);
        R phi = std::atan2(detp, dotp);
        if (r < R(kEpsF)) { p.y = R(kEpsF); p.z = R(kEpsF); r = R(kEpsF); }
        R krr = k_r * r;
        R besselj = R(jn(mode, double(krr)));
        R dbesselj = R(double(R(mode) / krr * besselj) - jn(mode + 1, double(krr)));
        R invr = R(1.0 / double(r));
        R invr2 = invr * invr;
        R cosmp = std::cos(R(mode) * phi);
        R sinmp = std::sin(R(mode) * phi);
        R a = n_max * scaling;
        return V3<R>(R(0),
                     a * (dbesselj * k_r * p.y * invr * cosmp - besselj * R(mode) * sinmp * p.z * invr2),
                     a * (dbesselj * k_r * p.z * invr * cosmp + besselj * R(mode) * sinmp * p.y * invr2));
    }

    // scene.cpp:141-160 (the CPU order: harmonic outer, source inner, both arcs per source)
    double fus_RIF(const V3<R> &p) const {
        R rif = 0;
        for (int c = 1; c <= n_coeff; ++c) {
            R sf = R(4 * std::pow(-1.0, c + 1) / (std::pow(double(c) * double(K<R>::pi()), 2) * nsources));
            R trif = 0;
            for (int n = 0; n < nsources; ++n) {
                if (active1) { R r = (p - centers1[n]).length(); trif += std::cos(k_r * r * R(c) + phase1) / r; }
                if (active2) { R r = (p - centers2[n]).length(); trif += std::cos(k_r * r * R(c) + phase2) / r; }
            }
            rif += trif * sf;
        }
        return double(n_o + n_scaling * rif);
    }
    // scene.cpp:163-195
    V3<R> fus_dRIF(const V3<R> &p) const {
        V3<R> dn(R(0), R(0), R(0));
        for (int c = 1; c <= n_coeff; ++c) {
            R sf = R(4 * std::pow(-1.0, c + 1) / (std::pow(double(c) * double(K<R>::pi()), 2) * nsources));
            V3<R> tdn(R(0), R(0), R(0));
            if (active1)
                for (int n = 0; n < nsources; ++n) {
                    V3<R> dv = p - centers1[n];
                    R r = dv.length(), krrc = k_r * r * R(c);
                    R ct = -(std::cos(krrc + phase1) + krrc * std::sin(krrc + phase1)) / (r * r * r);
                    tdn += ct * dv;
                }
            if (active2)
                for (int n = 0; n < nsources; ++n) {
                    V3<R> dv = p - centers2[n];
                    R r = dv.length(), krrc = k_r * r * R(c);
                    R ct = -(std::cos(krrc + phase2) + krrc * std::sin(krrc + phase2)) / (r * r * r);
                    tdn += ct * dv;
                }
            dn += tdn * sf;
        }
        return dn * n_scaling;
    }

    // plane waves: n = n_o + sum a_i sin(k_i.p - tau + phase_i); tau is the per-photon draw
    double wave_RIF(const V3<R> &p, R tau) const {
        R s = 0;
        for (int i = 0; i < n_waves; ++i) s += amp[i] * std::sin(dot(kvec[i], p) - tau + phase[i]);
        return double(n_o + s);
    }
    V3<R> wave_dRIF(const V3<R> &p, R tau) const {
        V3<R> g(R(0), R(0), R(0));
        for (int i = 0; i < n_waves; ++i) g += (amp[i] * std::cos(dot(kvec[i], p) - tau + phase[i])) * kvec[i];
        return g;
    }

    // cubic B-spline kernels, spline.h:33-62
    static R k0(R x) {
        x = std::abs(x);
        if (x > R(2)) return R(0);
        if (x > R(1)) return R(1.0 / 6.0) * (R(2) - x) * (R(2) - x) * (R(2) - x);
        return R(2.0 / 3.0) - x * x + K<R>::half() * x * x * x;
    }
    static R k1(R x) {
        R s = R((R(0) < x) - (x < R(0)));
        x = std::abs(x);
        if (x > R(2)) return R(0);
        if (x > R(1)) return s * (-K<R>::half() * (R(2) - x) * (R(2) - x));
        return s * R((1.5 * double(x) - 2) * double(x));
    }
    static int wrap(int i, int n) {                       // spline.h:18-21, :611-617
        int m = 2 * n - 2;
        int w = i % m;
        if (w < 0) w += m;
        if (w >= n) w = m - w;
        return w;
    }
    void to_grid(const V3<R> &p, R g[3]) const {         // convertToX, spline.h:599-602
        for (int i = 0; i < 3; ++i) g[i] = (p[i] - xmin[i]) * xres[i];
    }
    // spline.h:308-321 with the mirror rule
    R spline_value(const V3<R> &p) const {
        R x[3];
        to_grid(p, x);
        R v = 0;
        for (int i1 = int(std::ceil(x[0] - 2)); i1 <= int(std::floor(x[0] + 2)); ++i1)
            for (int i2 = int(std::ceil(x[1] - 2)); i2 <= int(std::floor(x[1] + 2)); ++i2)
                for (int i3 = int(std::ceil(x[2] - 2)); i3 <= int(std::floor(x[2] + 2)); ++i3) {
                    R c = delta[wrap(i1, N[0]) + wrap(i2, N[1]) * N[0] + wrap(i3, N[2]) * N[0] * N[1]];
                    v += c * k0(x[0] - R(i1)) * k0(x[1] - R(i2)) * k0(x[2] - R(i3));
                }
        return base + v;
    }
    // spline.h:324-356 with the mirror rule
    V3<R> spline_gradient(const V3<R> &p) const {
        R x[3];
        to_grid(p, x);
        V3<R> v(R(0), R(0), R(0));
        for (int i1 = int(std::ceil(x[0] - 2)); i1 <= int(std::floor(x[0] + 2)); ++i1)
            for (int i2 = int(std::ceil(x[1] - 2)); i2 <= int(std::floor(x[1] + 2)); ++i2)
                for (int i3 = int(std::ceil(x[2] - 2)); i3 <= int(std::floor(x[2] + 2)); ++i3) {
                    R c = delta[wrap(i1, N[0]) + wrap(i2, N[1]) * N[0] + wrap(i3, N[2]) * N[0] * N[1]];
                    R kx = k0(x[0] - R(i1)), ky = k0(x[1] - R(i2)), kz = k0(x[2] - R(i3));
                    v.x += c * k1(x[0] - R(i1)) * ky * kz;
                    v.y += c * kx * k1(x[1] - R(i2)) * kz;
                    v.z += c * kx * ky * k1(x[2] - R(i3));
                }
        v.x *= xres[0];
        v.y *= xres[1];
        v.z *= xres[2];
        return v;
    }
};

// ---- scene pieces ----------------------------------------------------------------------------------
template <typename R> struct Lens {                          // lens.cpp:20-97
    V3<R> origin;
    R sq_aperture = 0, focal = 0;
    bool active = false;
    void init(const double *o, double aperture, double f, int act) {
        origin = mk<R>(o);
        sq_aperture = R(aperture) * R(aperture);
        focal = R(f);
        active = act != 0;
    }
    template <typename T> bool deflect(const V3<R> &pos, V3<R> &dir, T &total) const {
        R sq = 0;
        for (int i = 1; i < 3; ++i) sq += pos[i] * pos[i];
        if (sq > sq_aperture) return false;
        R invd = -R(1) / dir[0];
        dir[0] = -focal;
        dir[1] = dir[1] * invd * focal - pos[1];
        dir[2] = dir[2] * invd * focal - pos[2];
        total += T(focal * invd - dir.length());
        dir.normalize();
        return true;
    }
    template <typename T> bool propagate_till_lens(V3<R> &pos, V3<R> &dir, T &total) const {
        R dist = -(pos[0] - origin[0]) / dir[0];
        pos += dist * dir;
        total += T(dist);
        if (active) return deflect(pos, dir, total);
        return true;
    }
};

template <typename R> struct Scene {
    // block (block.cpp:12-23)
    V3<R> L, Rr;
    // source (area_textured_source.cpp:6-46; sample_ray scene.cpp:107-137)
    V3<R> src_origin, src_dir;
    R ct = 1, plane[2], pixsize[2], Li = 0;
    int tex_x = 1, tex_y = 1;
    std::vector<float> cdf;
    Lens<R> src_lens;
    // camera (camera.cpp:11-29)
    V3<R> cam_origin, cam_dir, cam_h, cam_v;
    R cam_plane[2], pl_min, pl_max;
    bool bounce = false;
    Lens<R> cam_lens;
    int X = 1, Y = 1, Z = 1;
    // BSDF (bsdf.cpp) ior1 = 1, ior2 = ior
    R ior1 = 1, ior2 = 1;
    R fresnel_trans = 1;

    void init(const smp_scene_desc &s);
    bool inside(const V3<R> &p) const {
        for (int i = 0; i < 3; ++i)
            if (!((p[i] - L[i] > -R(kEpsF)) && (Rr[i] - p[i] > -R(kEpsF)))) return false;
        return true;
    }
};

// pmf.h:41-99 (append then normalise, in Float)
static void build_cdf(const double *tex, int n, std::vector<float> &cdf) {
    cdf.assign(1, 0.0f);
    cdf.reserve(n + 1);
    for (int i = 0; i < n; ++i) cdf.push_back(cdf.back() + static_cast<float>(tex[i]));
    float sum = cdf.back();
    if (sum > 0) {
        float norm = 1.0f / sum;
        for (size_t i = 1; i < cdf.size(); ++i) cdf[i] *= norm;
        cdf.back() = 1.0f;
    }
}
// pmf.h:109-121
static int sample_cdf(const std::vector<float> &cdf, float u) {
    size_t pos = std::lower_bound(cdf.begin(), cdf.end(), u) - cdf.begin();
    size_t n = cdf.size();
    size_t idx = std::min(n - 2, static_cast<size_t>(std::max<ptrdiff_t>(0, ptrdiff_t(pos) - 1)));
    while (idx < n - 1 && cdf[idx + 1] - cdf[idx] == 0) ++idx;
    if (idx > n - 2) idx = n - 2;
    return static_cast<int>(idx);
}

// util.h:42-57
template <typename R> static R fresnel(R cosI, R cosT, R eta) {
    if (std::abs(eta - R(1)) < R(kEpsF) * std::max(R(1), std::abs(eta))) return R(0);
    R Rs = (cosI - eta * cosT) / (cosI + eta * cosT);
    R Rp = (cosT - eta * cosI) / (cosT + eta * cosI);
    return R(0.5) * (Rs * Rs + Rp * Rp);
}
// util.h:64-88
template <typename R> static void reflect(const V3<R> &a, const V3<R> &n, V3<R> &b) {
    b = -R(2) * dot(a, n) * n + a;
}
template <typename R> static bool refract(const V3<R> &a, const V3<R> &n, R eta, V3<R> &b) {
    V3<R> q = dot(a, n) * n;
    V3<R> p = (a - q) / eta;
    if (p.length() > R(1)) { reflect(a, n, b); return false; }
    q.normalize();
    R t = R(1) - p.lengthSquared();
    q *= (t > R(0) ? std::sqrt(t) : R(0));
    b = p + q;
    return true;
}
// util.h:17-27
template <typename R> static void coordinate_system(const V3<R> &a, V3<R> &b, V3<R> &c) {
    if (std::abs(a.x) > std::abs(a.y)) {
        R inv = R(1) / std::sqrt(a.x * a.x + a.z * a.z);
        c = V3<R>(a.z * inv, R(0), -a.x * inv);
    } else {
        R inv = R(1) / std::sqrt(a.y * a.y + a.z * a.z);
        c = V3<R>(R(0), a.z * inv, -a.y * inv);
    }
    b = cross(c, a);
}

template <typename R> void Scene<R>::init(const smp_scene_desc &s) {
    L = mk<R>(s.medium_l);
    Rr = mk<R>(s.medium_r);
    src_origin = mk<R>(s.light_origin);
    src_dir = mk<R>(s.light_dir);
    plane[0] = R(s.light_plane[0]);
    plane[1] = R(s.light_plane[1]);
    tex_x = s.tex_x;
    tex_y = s.tex_y;
    pixsize[0] = plane[0] / R(tex_x);
    pixsize[1] = plane[1] / R(tex_y);
    ct = std::cos(R(s.half_theta_limit));
    Li = R(s.Li);
    build_cdf(s.texture, tex_x * tex_y, cdf);
    src_lens.init(s.emitter_lens_origin, s.emitter_lens_aperture, s.emitter_lens_focal_length,
                  s.emitter_lens_active);
    cam_origin = mk<R>(s.view_origin);
    cam_dir = mk<R>(s.view_dir);
    cam_dir.normalize();
    cam_h = mk<R>(s.view_horizontal);
    cam_h.normalize();
    cam_v = cross(cam_dir, cam_h);
    cam_plane[0] = R(s.view_plane[0]);
    cam_plane[1] = R(s.view_plane[1]);
    pl_min = R(s.pathlength_range[0]);
    pl_max = R(s.pathlength_range[1]);
    bounce = s.use_bounce_decomposition != 0;
    cam_lens.init(s.sensor_lens_origin, s.sensor_lens_aperture, s.sensor_lens_focal_length,
                  s.sensor_lens_active);
    X = s.x_res; Y = s.y_res; Z = s.z_res;
    ior1 = R(1);
    ior2 = R(s.ior);
    // scene.h:144-164
    R ior = R(s.ior);
    fresnel_trans = R(1);
    if (ior > R(1)) {
        V3<R> refr;
        R sum = 0;
        for (int i = 1; i < 3; ++i) { refr[i] = src_dir[i] / ior; sum += refr[i] * refr[i]; }
        refr.x = std::sqrt(R(1) - sum);
        if (src_dir.x < R(0)) refr.x *= -R(1);
        fresnel_trans = ior * ior * (R(1) - fresnel(src_dir.x, refr.x, ior));
    }
}

// ---- the photon march ------------------------------------------------------------------------------
// R: arithmetic of the march; A: the optical path-length accumulator and film (float in the
// reference; double for the FP32-march / FP64-accumulation form).
template <typename R, typename A> struct Tracer {
    const Scene<R> *sc;
    const Field<R> *fd;
    R sigma_t, albedo, mfp, g;
    int max_depth;
    R max_pathlength;
    bool use_direct, use_angular;
    R h0;          // er_stepsize
    R large_dist;  // LargeDist of movePhotonTillSensor
    long precision0;
    int64_t step_cap;
    R weight;
    // per photon
    Uniforms *u;
    int64_t steps = 0;
    bool abort_cap = false, abort_nan = false;
    smp_photon_record *rec = nullptr;
    int n_splats = 0;
    A *img = nullptr;                // thread-local film (X*Y*Z)

    bool aborted() const { return abort_cap || abort_nan || u->exhausted; }

    // Scene::er_step, scene.cpp:323-330
    void er_step(V3<R> &p, V3<R> &d, R h, R s) {
        d += K<R>::half() * h * fd->dRIF(p, s);
        p += h * d / R(fd->RIF(p, s));
        d += K<R>::half() * h * fd->dRIF(p, s);
        ++steps;
        if (!p.finite() || !d.finite()) abort_nan = true;
        if (steps >= step_cap) abort_cap = true;
    }

    // Scene::traceTillBlock, scene.cpp:385-425
    R trace_till_block(V3<R> &p, V3<R> &d, R dist, A &total, R s) {
        V3<R> oldp, oldd;
        R distance = 0;
        int64_t maxsteps = to_i64_x86(double(dist / h0 + R(1)));
        long prec = precision0;
        R cur = h0;
        for (int64_t i = 0; i < maxsteps; ++i) {
            oldp = p;
            oldd = d;
            er_step(p, d, cur, s);
            if (aborted()) break;
            if (!sc->inside(p) || (distance + cur) > dist) {
                --prec;
                if (prec < 0) break;
                p = oldp;
                d = oldd;
                cur = cur / R(10);
                i = 0;
                maxsteps = 11;
            } else {
                distance += cur;
                total = A(double(total) + double(cur) * fd->RIF(p, s));
            }
        }
        return distance;
    }

    // nearest-face normal, scene.cpp:655-676 / :736-757
    V3<R> face_normal(const V3<R> &p) const {
        R minDiff = R(kMaxF), minDir = 0;
        int chosen = 3;
        for (int i = 0; i < 3; ++i) {
            R diff = std::abs(sc->L[i] - p[i]);
            if (diff < minDiff) { minDiff = diff; chosen = i; minDir = -R(1); }
            diff = std::abs(sc->Rr[i] - p[i]);
            if (diff < minDiff) { minDiff = diff; chosen = i; minDir = R(1); }
        }
        V3<R> n(R(0), R(0), R(0));
        if (chosen < 3) n[chosen] = minDir;
        return n;
    }

    // SmoothDielectric::sample, bsdf.cpp:26-58
    void bsdf_sample(const V3<R> &in, const V3<R> &n, V3<R> &out) {
        if (std::abs(sc->ior1 - sc->ior2) < R(kEpsF)) { out = in; return; }
        R eta = (dot(in, n) < -R(kEpsF)) ? sc->ior2 / sc->ior1 : sc->ior1 / sc->ior2;
        V3<R> outT;
        if (!refract(in, n, eta, outT)) { out = outT; return; }
        V3<R> outR;
        reflect(in, n, outR);
        R cosI = absDot(n, in), cosT = absDot(n, outT);
        R F = fresnel(cosI, cosT, eta);
        out = ((*u)() < F) ? outR : outT;
    }

    // Scene::movePhotonTillSensor, scene.cpp:622-703
    bool move_till_sensor(V3<R> &p, V3<R> &d, R &distToSensor, A &total, R s) {
        R large = large_dist;                       // LargeDist (scene.cpp:627); see smp_render_opts
        distToSensor = trace_till_block(p, d, large, total, s);
        if (aborted()) return false;
        large -= distToSensor;
        for (;;) {
            if (large < R(0)) return false;
            V3<R> n = face_normal(p);
            if (std::abs(sc->cam_dir.x - n.x) < R(kEpsF) && std::abs(sc->cam_dir.y - n.y) < R(kEpsF) &&
                std::abs(sc->cam_dir.z - n.z) < R(kEpsF))
                return true;
            V3<R> d1;
            bsdf_sample(d, n, d1);
            if (dot(d1, n) < R(0)) d = d1; else return false;
            R disy = trace_till_block(p, d, large, total, s);
            if (aborted()) return false;
            distToSensor += disy;
            large -= disy;
        }
    }

    // Scene::movePhoton, scene.cpp:706-780
    bool move_photon(V3<R> &p, V3<R> &d, R dist, A &total, R s) {
        R disy = trace_till_block(p, d, dist, total, s);
        if (aborted()) return false;
        dist -= disy;
        while (dist > R(kEpsF)) {
            V3<R> n = face_normal(p);
            R mag = d.length();
            V3<R> d1;
            bsdf_sample(d / mag, n, d1);
            if (dot(d1, n) < R(0)) d = d1 * mag; else return false;
            disy = trace_till_block(p, d, dist, total, s);
            if (aborted()) return false;
            dist -= disy;
        }
        return true;
    }

    // Camera::propagate_till_sensor, camera.cpp:54-75
    bool propagate_till_sensor(V3<R> &pos, V3<R> &dir, R &total) const {
        if (sc->cam_lens.active && !sc->cam_lens.deflect(pos, dir, total)) return false;
        R dist = (sc->cam_origin[0] - pos[0]) / dir[0];
        pos += dist * dir;
        total += dist;
        return true;
    }

    void add_pixel(int x, int y, int z, A val) {              // scene.h:305-312, image.h:320-324
        if (img && x >= 0 && x < sc->X && y >= 0 && y < sc->Y && z >= 0 && z < sc->Z)
            img[size_t(z) * sc->X * sc->Y + size_t(y) * sc->X + x] += val;
    }

    // Scene::addEnergyToImage, scene.cpp:782-829
    void add_energy(const V3<R> &p, A pathlength, int depth, R val) {
        if (rec) {
            if (n_splats < SMP_TRACE_MAX_SPLATS) {
                smp_splat_record &sr = rec->splats[n_splats];
                sr.p[0] = float(p.x); sr.p[1] = float(p.y); sr.p[2] = float(p.z);
                sr.depth = depth;
                sr.pathlength = double(pathlength);
                sr.value = double(val);
            }
        }
        ++n_splats;
        R x = dot(sc->cam_h, p) - sc->cam_origin.y;
        R y = dot(sc->cam_v, p) - sc->cam_origin.z;
        bool nobin = (sc->pl_min == R(-1)) && (sc->pl_max == R(-1));
        if (nobin || ((pathlength > A(sc->pl_min)) && (pathlength < A(sc->pl_max)))) {
            x = (x / sc->cam_plane[0] + K<R>::half()) * R(sc->X);
            y = (y / sc->cam_plane[1] + K<R>::half()) * R(sc->Y);
            int ix = int(std::floor(x)), iy = int(std::floor(y));
            int iz;
            if (sc->bounce) iz = depth;
            else if (nobin) iz = 0;
            else {
                A z = pathlength - A(sc->pl_min);
                A range = A(sc->pl_max) - A(sc->pl_min);
                z = (z / range) * A(sc->Z);
                iz = int(std::floor(z));
            }
            R fx = x - std::floor(x), fy = y - std::floor(y);
            add_pixel(ix, iy, iz, A(val * (R(1) - fx) * (R(1) - fy)));
            add_pixel(ix + 1, iy, iz, A(val * fx * (R(1) - fy)));
            add_pixel(ix, iy + 1, iz, A(val * (R(1) - fx) * fy));
            add_pixel(ix + 1, iy + 1, iz, A(val * fx * fy));
        }
    }

    // HG f, phase.cpp:17-21
    R hg_f(const V3<R> &in, const V3<R> &out) const {
        R c = dot(in, out);
        return R(1.0 / (4.0 * double(K<R>::pi()))) * (R(1) - g * g) /
               std::pow(R(1) + g * g - R(2) * g * c, R(1.5));
    }
    // HG sample, phase.cpp:40-76
    void hg_sample(const V3<R> &in, V3<R> &out) {
        R sx = (*u)();
        R sy = (*u)();
        R cosT;
        if (std::abs(g) < R(kEpsF)) cosT = R(1) - R(2) * sx;
        else {
            R sq = (R(1) - g * g) / (R(1) - g + R(2) * g * sx);
            cosT = (R(1) + g * g - sq * sq) / (R(2) * g);
        }
        R sinT = std::sqrt(std::max(R(0), R(1) - cosT * cosT));
        R phi = R(2.0 * double(K<R>::pi())) * sy;
        R sinP = std::sin(phi), cosP = std::cos(phi);
        V3<R> ax, ay;
        coordinate_system(in, ax, ay);
        out = (sinT * cosP) * ax + (sinT * sinP) * ay + cosT * in;
    }

    // scene.cpp:26-39 + warp.cpp:22-34. The reference evaluates Vec2f(sampler(), sampler())
    // right to left under GCC x86-64: the first draw lands in sample.y (azimuth), the second in
    // sample.x (z).
    // warp::squareToUniformHemisphere (warp.cpp:22-34): z = sample.x, azimuth 2 pi sample.y
    static V3<R> uniform_hemisphere(R sx, R sy) {
        R z = sx;
        R tmp = std::sqrt(R(1) - z * z);
        R a = R(2.0 * double(K<R>::pi())) * sy;
        return V3<R>(std::cos(a) * tmp, std::sin(a) * tmp, z);
    }
    V3<R> sample_random_direction() {
        R uy = (*u)();
        R ux = (*u)();
        V3<R> v = uniform_hemisphere(ux, uy);
        R t = v.x;
        v.x = -v.z;
        v.z = v.y;
        v.y = t;
        return v;
    }

    // Scene::addEnergyInParticle, scene.cpp:866-946
    void add_energy_in_particle(const V3<R> &p, const V3<R> &d, A distTravelled, int depth, R val, R s) {
        V3<R> p1 = p;
        if ((p.x - sc->cam_origin.x) < R(1e-4)) return;
        V3<R> dirToSensor = sample_random_direction();
        dirToSensor *= R(fd->RIF(p1, s));
        R distToSensor;
        if (!move_till_sensor(p1, dirToSensor, distToSensor, distTravelled, s)) return;
        dirToSensor.normalize();
        V3<R> refr = dirToSensor;
        R fw = R(1);
        R ior = R(fd->RIF(p1, s));
        if (ior > R(1)) {
            refr.x = refr.x / ior;
            refr.normalize();
            fw = (R(1) - fresnel(dirToSensor.x, refr.x, R(1) / ior)) / ior / ior;
        }
        R foreshortening = dot(refr, sc->cam_dir) / dot(dirToSensor, sc->cam_dir);
        A tot = distTravelled;
        R dts = 0;
        if (!propagate_till_sensor(p1, refr, dts)) return;
        tot += A(dts);
        R value = val * R(2.0 * double(K<R>::pi())) * std::exp(-sigma_t * distToSensor) *
                  hg_f(d / d.length(), dirToSensor) * foreshortening * fw;
        add_energy(p1, tot, depth, value);
    }

    // Renderer::directTracing, photon.cpp:41-87 (total is the photon's own, by reference)
    void direct_tracing(const V3<R> &p, const V3<R> &d, R s, A &total) {
        V3<R> p1 = p, d1 = d;
        R distToSensor;
        if (!move_till_sensor(p1, d1, distToSensor, total, s)) return;
        R fw = R(1);
        d1.normalize();
        R ior = R(fd->RIF(p1, s));
        V3<R> refr = d1;
        if (ior > R(1)) {
            refr.x = refr.x / ior;
            refr.normalize();
            fw = (R(1) - fresnel(d1.x, refr.x, R(1) / ior)) / ior / ior;
        }
        R dts = 0;
        if (!propagate_till_sensor(p1, refr, dts)) return;
        total += A(dts);
        R value = weight * std::exp(-sigma_t * distToSensor) * fw;
        add_energy(p1, total, 0, value);
    }

    R move_step() { return -mfp * std::log((*u)()); }        // photon.h:72-74

    bool roulette() {                                          // photon.cpp:24, :97
        return (albedo > R(0)) && ((albedo >= R(1)) || ((*u)() < albedo));
    }

    // Renderer::scatterOnce, photon.cpp:20-38
    bool scatter_once(V3<R> &p, V3<R> &d, R &dist, A &total, R s, int &end) {
        if (roulette()) {
            R mag = d.length();
            V3<R> d1;
            hg_sample(d / mag, d1);
            d = mag * d1;
            dist = move_step();
            bool ok = move_photon(p, d, dist, total, s);
            if (!ok) end = SMP_END_ESCAPED;
            return ok;
        }
        dist = 0;
        end = SMP_END_ABSORBED;
        return false;
    }

    // Renderer::scatter, photon.cpp:91-136
    void scatter(V3<R> &pos, V3<R> &dir, R s, A &total, int &depth_out, int &end) {
        depth_out = 0;
        if (!roulette()) { end = SMP_END_NO_SCATTER; return; }
        R dist = move_step();
        if (!move_photon(pos, dir, dist, total, s)) { end = SMP_END_ESCAPED; return; }
        int depth = 1;
        R totalDist = dist;
        end = SMP_END_MAX_DEPTH;
        while ((max_depth < 0 || depth <= max_depth) && (max_pathlength < R(0) || totalDist <= max_pathlength)) {
            depth_out = depth;
            if (use_angular) add_energy_in_particle(pos, dir, total, depth, weight, s);
            if (aborted()) return;
            if (!scatter_once(pos, dir, dist, total, s, end)) return;
            ++depth;
        }
        depth_out = depth;
        end = SMP_END_MAX_DEPTH;
    }

    // area_textured_source::sample_ray, scene.cpp:107-137
    bool gen_ray(V3<R> &pos, V3<R> &dir, A &total) {
        pos = sc->src_origin;
        int pixel = sample_cdf(sc->cdf, (*u)());
        int py = pixel / sc->tex_x;
        int px = pixel - py * sc->tex_x;
        int pp[2] = {px, py};
        for (int it = 1; it < 3; ++it)
            pos[it] += -sc->plane[it - 1] / R(2) + R(pp[it - 1]) * sc->pixsize[it - 1] + (*u)() * sc->pixsize[it - 1];
        R z = (*u)() * (R(1) - sc->ct) + sc->ct;
        R zt = std::sqrt(R(1) - z * z);
        R phi = (*u)() * R(2) * K<R>::pi();
        dir = V3<R>(-z, zt * std::cos(phi), zt * std::sin(phi));
        return sc->src_lens.propagate_till_lens(pos, dir, total);
    }

    // one photon of Renderer::renderImage, photon.cpp:313-333
    void photon(const smp_field_desc &fdesc) {
        steps = 0;
        abort_cap = abort_nan = false;
        n_splats = 0;
        V3<R> pos, dir;
        A total = 0;
        int end = SMP_END_GENRAY_FAIL, depth = 0;
        if (gen_ray(pos, dir, total)) {
            R uu = (*u)();
            R s;
            if (fd->type == SMP_FIELD_PLANEWAVE) {
                s = R(fdesc.phi_min) + (R(fdesc.phi_max) - R(fdesc.phi_min)) * uu;
            } else if (fd->type == SMP_FIELD_SOURCES) {
                s = std::max(std::min(std::sin(R(0) + R(0) * uu), R(0)), -R(0));   // scene.h:185-198
            } else {
                R pmin = R(fdesc.phi_min), range = R(fdesc.phi_max) - R(fdesc.phi_min);
                R maxs = R(fdesc.n_clip) / R(fdesc.n_max);                           // rif_analytical.h:222
                s = std::max(std::min(std::sin(pmin + range * uu), maxs), -maxs);
            }
            dir *= R(fd->RIF(pos, s));
            if (use_direct) direct_tracing(pos, dir, s, total);
            if (!aborted()) scatter(pos, dir, s, total, depth, end);
        }
        if (abort_cap) end = SMP_END_STEP_CAP;
        if (abort_nan) end = SMP_END_NAN;
        if (u->exhausted) end = SMP_END_STREAM;
        if (rec) {
            rec->end = end;
            rec->draws = u->draws;
            rec->depth = depth;
            rec->n_splats = n_splats;
            rec->pos[0] = float(pos.x); rec->pos[1] = float(pos.y); rec->pos[2] = float(pos.z);
            rec->dir[0] = float(dir.x); rec->dir[1] = float(dir.y); rec->dir[2] = float(dir.z);
            rec->total_optical = double(total);
            rec->er_steps = steps;
        }
    }
};

template <typename R, typename A>
static int render_impl(const smp_scene_desc *sd, const smp_medium_desc *md, const smp_field_desc *fdesc,
                       const smp_render_opts *opts, int threads, int64_t first, int64_t n,
                       int64_t weight_photons, const float *uniforms, const int64_t *offsets,
                       smp_photon_record *records, double *image_out, A *thread_films = nullptr) {
    Scene<R> sc;
    sc.init(*sd);
    Field<R> fd;
    fd.init(*fdesc);
    // medium.h:24-38
    R sigma_t = R(md->sigma_t), albedo = R(md->albedo), mfp = R(1) / R(md->sigma_t);
    if (sigma_t <= R(kEpsF)) { sigma_t = 0; mfp = 1; albedo = 0; }
    R weight = sc.Li * sc.fresnel_trans / R(weight_photons);   // photon.h:76-80
    const size_t npix = size_t(sc.X) * sc.Y * sc.Z;
    int nt = threads > 0 ? threads : omp_get_max_threads();
    // per-thread films merged at the end (renderImage, photon.cpp:290-291, 337), or the caller's
    std::vector<std::vector<A>> imgs(nt, std::vector<A>(image_out && !thread_films ? npix : 0, A(0)));
    int64_t cap = opts->step_cap > 0 ? opts->step_cap : int64_t(10000000);
#pragma omp parallel num_threads(nt)
    {
        int tid = omp_get_thread_num();
        Tracer<R, A> tr;
        tr.sc = &sc;
        tr.fd = &fd;
        tr.sigma_t = sigma_t;
        tr.albedo = albedo;
        tr.mfp = mfp;
        tr.g = R(md->g);
        tr.max_depth = opts->max_depth;
        tr.max_pathlength = R(opts->max_pathlength);
        tr.use_direct = opts->use_direct != 0;
        tr.use_angular = opts->use_angular_sampling != 0;
        tr.h0 = R(fdesc->er_stepsize);
        {
            float st = float(sigma_t);
            float d = opts->sensor_march_max > 0.0 ? float(opts->sensor_march_max) : 10000.0f;
            if (!(opts->sensor_march_max > 0.0) && st > 0.0f) d = std::min(d, 110.0f / st);
            tr.large_dist = R(d);
        }
        tr.precision0 = fdesc->precision;
        tr.step_cap = cap;
        tr.weight = weight;
        tr.img = thread_films ? thread_films + size_t(tid) * npix : (image_out ? imgs[tid].data() : nullptr);
        Uniforms un;
#pragma omp for schedule(dynamic, 64)
        for (int64_t k = 0; k < n; ++k) {
            int64_t i = first + k;
            un = Uniforms();
            if (uniforms) {
                un.mode = SMP_RNG_STREAM;
                un.stream = uniforms;
                un.pos = offsets[k];
                un.end = offsets[k + 1];
            } else if (opts->rng == SMP_RNG_PHILOX) {
                un.mode = SMP_RNG_PHILOX;
                un.philox.seed(opts->seed, uint64_t(i));
            } else {
                un.mode = SMP_RNG_SFMT;
                un.sfmt.seed(opts->seed + uint64_t(i));
            }
            tr.u = &un;
            smp_photon_record *r = records ? &records[k] : nullptr;
            if (r) { std::memset(r, 0, sizeof(*r)); r->photon = i; }
            tr.rec = r;
            tr.photon(*fdesc);
        }
    }
    if (image_out && !thread_films) {
        for (size_t j = 0; j < npix; ++j) {
            A v = 0;
            for (int t = 0; t < nt; ++t) v += imgs[t][j];
            image_out[j] = double(v);
        }
    }
    return 0;
}

}  // namespace orc

namespace orc {
// ---- B-spline prefilter and 1-D / 3-D evaluation (spline.h) ----------------------------------------
// build1d, spline.h:686-714; data read with (offset, stride), written to out[0..size)
template <typename R>
static void build1d(const R *data, long offset, long stride, int size, R *out) {
    const R z1 = R(-2) + std::sqrt(R(3));
    std::vector<R> cp(size), cn(size);
    cp[0] = 0;
    for (int i = 0; i < size; ++i) cp[0] += data[offset + i * stride] * R(std::pow(double(z1), i));
    for (int i = size - 2; i > 0; --i) cp[0] += data[offset + i * stride] * R(std::pow(double(z1), 2 * size - 2 - i));
    cp[0] /= R(1 - std::pow(double(z1), 2 * size - 2));
    for (int i = 1; i < size; ++i) cp[i] = data[offset + i * stride] + z1 * cp[i - 1];
    cn[size - 1] = z1 / (z1 * z1 - R(1)) * (cp[size - 1] + z1 * cp[size - 2]);
    for (int i = size - 2; i >= 0; --i) cn[i] = z1 * (cn[i + 1] - cp[i]);
    for (int i = 0; i < size; ++i) out[i] = R(6) * cn[i];
}

// build3d, spline.h:739-764
template <typename R>
static void build3d(const R *data, const int N[3], R *coeff) {
    std::vector<R> tmp(std::max(std::max(N[0], N[1]), N[2]));
    long s01 = long(N[0]) * N[1];
    for (int k = 0; k < N[2]; ++k)
        for (int i = 0; i < N[0]; ++i) {
            build1d(data, k * s01 + i, N[0], N[1], tmp.data());
            for (int t = 0; t < N[1]; ++t) coeff[i + t * N[0] + k * s01] = tmp[t];
        }
    for (int k = 0; k < N[2]; ++k)
        for (int j = 0; j < N[1]; ++j) {
            build1d(coeff, k * s01 + long(j) * N[0], 1, N[0], tmp.data());
            for (int t = 0; t < N[0]; ++t) coeff[t + j * N[0] + k * s01] = tmp[t];
        }
    for (int i = 0; i < N[0]; ++i)
        for (int j = 0; j < N[1]; ++j) {
            build1d(coeff, long(j) * N[0] + i, s01, N[2], tmp.data());
            for (int t = 0; t < N[2]; ++t) coeff[i + j * N[0] + t * s01] = tmp[t];
        }
}

}  // namespace orc

extern "C" {

// Full render / trace through the restatement. real_bits: 32 = reference single precision,
// 64 = FP64 oracle. threads <= 0: all OpenMP threads.
int orc_render(const smp_scene_desc *scene, const smp_medium_desc *medium, const smp_field_desc *field,
               const smp_render_opts *opts, int real_bits, int threads, int64_t first, int64_t n,
               int64_t weight_photons, const float *uniforms, const int64_t *offsets,
               smp_photon_record *records, double *image_out) {
    if (!scene || !medium || !field || !opts || n < 0 || weight_photons <= 0) return SMP_ERR_BAD_ARG;
    if (uniforms && !offsets) return SMP_ERR_BAD_ARG;
    if (real_bits == 64)
        return orc::render_impl<double, double>(scene, medium, field, opts, threads, first, n, weight_photons,
                                                uniforms, offsets, records, image_out);
    if (opts->precision == SMP_PREC_MIXED)      // FP32 march, FP64 path length and film
        return orc::render_impl<float, double>(scene, medium, field, opts, threads, first, n, weight_photons,
                                               uniforms, offsets, records, image_out);
    return orc::render_impl<float, float>(scene, medium, field, opts, threads, first, n, weight_photons,
                                          uniforms, offsets, records, image_out);
}

// The same trace with the film accumulated into caller-owned per-thread films: `threads` films of
// X*Y*Z elements (double for real_bits 64 or SMP_PREC_MIXED, float otherwise), zeroed and merged by
// the caller, so that a long render timed in steps keeps its thread films across the steps as the
// reference's renderImage keeps its per-thread images across its photon loop. Philox or SFMT
// streams (no injected uniforms, no records).
int orc_render_films(const smp_scene_desc *scene, const smp_medium_desc *medium, const smp_field_desc *field,
                     const smp_render_opts *opts, int real_bits, int threads, int64_t first, int64_t n,
                     int64_t weight_photons, void *thread_films) {
    if (!scene || !medium || !field || !opts || n < 0 || weight_photons <= 0 || threads <= 0 || !thread_films)
        return SMP_ERR_BAD_ARG;
    if (real_bits == 64)
        return orc::render_impl<double, double>(scene, medium, field, opts, threads, first, n, weight_photons, nullptr,
                                                nullptr, nullptr, nullptr, static_cast<double *>(thread_films));
    if (opts->precision == SMP_PREC_MIXED)
        return orc::render_impl<float, double>(scene, medium, field, opts, threads, first, n, weight_photons, nullptr,
                                               nullptr, nullptr, nullptr, static_cast<double *>(thread_films));
    return orc::render_impl<float, float>(scene, medium, field, opts, threads, first, n, weight_photons, nullptr,
                                          nullptr, nullptr, nullptr, static_cast<float *>(thread_films));
}

// ---- single primitives (float, the reference's build), for pinning against its compiled code -------
int orc_hg_sample(float g, const float *in, uint64_t seed, int skip, float *out) {
    orc::Uniforms un;
    un.mode = SMP_RNG_SFMT;
    un.sfmt.seed(seed);
    for (int i = 0; i < skip; ++i) (void)un();
    orc::Tracer<float, float> tr;
    tr.g = g;
    tr.u = &un;
    orc::V3<float> o;
    tr.hg_sample(orc::V3<float>(in[0], in[1], in[2]), o);
    out[0] = o.x; out[1] = o.y; out[2] = o.z;
    return 0;
}

float orc_hg_f(float g, const float *in, const float *out) {
    orc::Tracer<float, float> tr;
    tr.g = g;
    return tr.hg_f(orc::V3<float>(in[0], in[1], in[2]), orc::V3<float>(out[0], out[1], out[2]));
}

void orc_hemisphere(float sx, float sy, float *out) {
    orc::V3<float> v = orc::Tracer<float, float>::uniform_hemisphere(sx, sy);
    out[0] = v.x; out[1] = v.y; out[2] = v.z;
}

float orc_fresnel(float ci, float ct, float eta) { return orc::fresnel<float>(ci, ct, eta); }

int orc_refract(const float *a, const float *n, float eta, float *b) {
    orc::V3<float> o;
    bool ok = orc::refract<float>(orc::V3<float>(a[0], a[1], a[2]), orc::V3<float>(n[0], n[1], n[2]), eta, o);
    b[0] = o.x; b[1] = o.y; b[2] = o.z;
    return ok ? 1 : 0;
}

void orc_coordinate_system(const float *a, float *b, float *c) {
    orc::V3<float> vb, vc;
    orc::coordinate_system<float>(orc::V3<float>(a[0], a[1], a[2]), vb, vc);
    b[0] = vb.x; b[1] = vb.y; b[2] = vb.z;
    c[0] = vc.x; c[1] = vc.y; c[2] = vc.z;
}

void orc_bsdf_sample(float ior1, float ior2, const float *in, const float *n, uint64_t seed, int skip, float *out) {
    orc::Uniforms un;
    un.mode = SMP_RNG_SFMT;
    un.sfmt.seed(seed);
    for (int i = 0; i < skip; ++i) (void)un();
    orc::Scene<float> sc;
    sc.ior1 = ior1;
    sc.ior2 = ior2;
    orc::Tracer<float, float> tr;
    tr.sc = &sc;
    tr.u = &un;
    orc::V3<float> o;
    tr.bsdf_sample(orc::V3<float>(in[0], in[1], in[2]), orc::V3<float>(n[0], n[1], n[2]), o);
    out[0] = o.x; out[1] = o.y; out[2] = o.z;
}

int orc_lens_propagate(const float *origin, float aperture, float focal, int active, float *pos, float *dir, float *total) {
    orc::Lens<float> lens;
    double o[3] = {origin[0], origin[1], origin[2]};
    lens.init(o, aperture, focal, active);
    orc::V3<float> p(pos[0], pos[1], pos[2]), d(dir[0], dir[1], dir[2]);
    float t = *total;
    bool ok = lens.propagate_till_lens(p, d, t);
    pos[0] = p.x; pos[1] = p.y; pos[2] = p.z;
    dir[0] = d.x; dir[1] = d.y; dir[2] = d.z;
    *total = t;
    return ok ? 1 : 0;
}

// cubic B-spline kernels k0, k1, k2 (spline.h:33-62), double
int orc_bspline_kernel(int d, int n, const double *x, double *out) {
    for (int i = 0; i < n; ++i) {
        if (d == 0) out[i] = orc::Field<double>::k0(x[i]);
        else if (d == 1) out[i] = orc::Field<double>::k1(x[i]);
        else {
            double a = std::abs(x[i]);
            out[i] = a > 2 ? 0.0 : (a > 1 ? 2 - a : 3 * a - 2);
        }
    }
    return 0;
}

int orc_sfmt_floats(uint64_t seed, int n, float *out) {
    orc::Sfmt19937 s;
    s.seed(seed);
    for (int i = 0; i < n; ++i) out[i] = s.next_float();
    return 0;
}

int orc_sfmt_u64(uint64_t seed, int n, uint64_t *out) {
    orc::Sfmt19937 s;
    s.seed(seed);
    for (int i = 0; i < n; ++i) out[i] = s.next_u64();
    return 0;
}

int orc_philox_floats(uint64_t seed, uint64_t photon, int n, float *out) {
    orc::PhiloxStream p;
    p.seed(seed, photon);
    for (int i = 0; i < n; ++i) out[i] = p.next_float();
    return 0;
}

// n and grad n at points, through the restated field code
int orc_field_eval(const smp_field_desc *field, double scaling, int real_bits, int64_t n,
                   const double *pts, double *n_out, double *grad_out) {
    if (real_bits == 64) {
        orc::Field<double> f;
        f.init(*field);
        for (int64_t i = 0; i < n; ++i) {
            orc::V3<double> p(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
            n_out[i] = f.RIF(p, scaling);
            orc::V3<double> g = f.dRIF(p, scaling);
            grad_out[3 * i] = g.x; grad_out[3 * i + 1] = g.y; grad_out[3 * i + 2] = g.z;
        }
    } else {
        orc::Field<float> f;
        f.init(*field);
        for (int64_t i = 0; i < n; ++i) {
            orc::V3<float> p(float(pts[3 * i]), float(pts[3 * i + 1]), float(pts[3 * i + 2]));
            n_out[i] = f.RIF(p, float(scaling));
            orc::V3<float> g = f.dRIF(p, float(scaling));
            grad_out[3 * i] = g.x; grad_out[3 * i + 1] = g.y; grad_out[3 * i + 2] = g.z;
        }
    }
    return 0;
}

int orc_texture_cdf(const double *tex, int n, float *cdf_out, int n_u, const float *u, int32_t *idx_out) {
    std::vector<float> cdf;
    orc::build_cdf(tex, n, cdf);
    std::memcpy(cdf_out, cdf.data(), sizeof(float) * cdf.size());
    for (int i = 0; i < n_u; ++i) idx_out[i] = orc::sample_cdf(cdf, u[i]);
    return 0;
}

int orc_spline_prefilter3d(const double *samples, const int32_t *n, int real_bits, double *coeff_out) {
    int N[3] = {n[0], n[1], n[2]};
    size_t tot = size_t(N[0]) * N[1] * N[2];
    if (real_bits == 64) {
        orc::build3d<double>(samples, N, coeff_out);
    } else {
        std::vector<float> s(tot), c(tot);
        for (size_t i = 0; i < tot; ++i) s[i] = float(samples[i]);
        orc::build3d<float>(s.data(), N, c.data());
        for (size_t i = 0; i < tot; ++i) coeff_out[i] = c[i];
    }
    return 0;
}

// 1-D spline of spline.h:120-126 (constructor), build1d, value1d<DX> (:604-621) in double
int orc_spline1d(const double *data, int n, double xmin, double xmax, int deriv, int npts,
                 const double *t, double *out) {
    std::vector<double> c(n);
    orc::build1d<double>(data, 0, 1, n, c.data());
    double xres = (n - 1) / (xmax - xmin);
    for (int k = 0; k < npts; ++k) {
        double x = (t[k] - xmin) * xres;
        double v = 0;
        for (int idx = int(std::ceil(x - 2)); idx <= int(std::floor(x + 2)); ++idx) {
            int w = orc::Field<double>::wrap(idx, n);
            double kv;
            double a = x - idx;
            if (deriv == 0) kv = orc::Field<double>::k0(a);
            else if (deriv == 1) kv = orc::Field<double>::k1(a);
            else {
                double ax = std::abs(a);
                kv = ax > 2 ? 0 : (ax > 1 ? 2 - ax : 3 * ax - 2);
            }
            v += c[w] * kv;
        }
        if (deriv == 1) v *= xres;
        if (deriv == 2) v *= xres * xres;
        out[k] = v;
    }
    return 0;
}

// 3-D value with derivative orders (dx,dy,dz) in {0,1,2}, mirror rule, double (spline.h:658-684)
int orc_spline3d_value(const double *coeff, const int32_t *n, const double *xmin, const double *xmax,
                       int dx, int dy, int dz, int npts, const double *pts, double *out) {
    int N[3] = {n[0], n[1], n[2]};
    double xres[3];
    for (int i = 0; i < 3; ++i) xres[i] = (N[i] - 1) / (xmax[i] - xmin[i]);
    auto kern = [](int d, double a) {
        if (d == 0) return orc::Field<double>::k0(a);
        if (d == 1) return orc::Field<double>::k1(a);
        double ax = std::abs(a);
        return ax > 2 ? 0.0 : (ax > 1 ? 2 - ax : 3 * ax - 2);
    };
    int D[3] = {dx, dy, dz};
    for (int k = 0; k < npts; ++k) {
        double x[3];
        for (int i = 0; i < 3; ++i) x[i] = (pts[3 * k + i] - xmin[i]) * xres[i];
        double v = 0;
        for (int i1 = int(std::ceil(x[0] - 2)); i1 <= int(std::floor(x[0] + 2)); ++i1)
            for (int i2 = int(std::ceil(x[1] - 2)); i2 <= int(std::floor(x[1] + 2)); ++i2)
                for (int i3 = int(std::ceil(x[2] - 2)); i3 <= int(std::floor(x[2] + 2)); ++i3) {
                    int w = orc::Field<double>::wrap(i1, N[0]) + orc::Field<double>::wrap(i2, N[1]) * N[0] +
                            orc::Field<double>::wrap(i3, N[2]) * N[0] * N[1];
                    v += coeff[w] * kern(D[0], x[0] - i1) * kern(D[1], x[1] - i2) * kern(D[2], x[2] - i3);
                }
        for (int i = 0; i < 3; ++i) {
            if (D[i] == 1) v *= xres[i];
            if (D[i] == 2) v *= xres[i] * xres[i];
        }
        out[k] = v;
    }
    return 0;
}

}  // extern "C"
