// capi.cu -- the extern "C" boundary of libsimpler_b200.so (declared in include/simpler_b200.h).
//
// The reference's GPU seam, cuda::CudaRenderer::renderImage (renderer/src/cuda_renderer.cu:710-742),
// deep-copies the scene with ~30 small cudaMalloc/cudaMemcpy calls per render, runs one thread per
// photon, and copies a float film back. Here a plan uploads the scene once (texture CDF, source
// table, spline coefficients, film) and each render runs asynchronously on the caller's stream (the
// slot-pool march of wavefront.cuh by default), so renders of one plan can be queued back to back.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "kparams.h"
#include "dispatch.h"
#include "wavefront.cuh"
#include "plain.cuh"
#include "adjoint.cuh"

using namespace smp;

// ---- errors ------------------------------------------------------------------------------------
static thread_local std::string g_last_error;

static int set_error(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define SMP_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return set_error(e_ == cudaErrorMemoryAllocation ? SMP_ERR_OOM : SMP_ERR_CUDA, \
                             "%s failed: %s", #call, cudaGetErrorString(e_));              \
    } while (0)

// ---- host helpers shared with the CLI / pybind layers ------------------------------------------

// DiscreteDistribution append + normalize (renderer/include/pmf.h:41-99), in float
static void texture_cdf(const double *tex, int n, std::vector<float> &cdf) {
    cdf.assign(size_t(n) + 1, 0.0f);
    for (int i = 0; i < n; ++i) cdf[i + 1] = cdf[i] + static_cast<float>(tex[i]);
    float sum = cdf[n];
    if (sum > 0.0f) {
        float norm = 1.0f / sum;
        for (int i = 1; i <= n; ++i) cdf[i] *= norm;
        cdf[n] = 1.0f;
    }
}

// Guide table of a texture CDF (KParams::cdf_guide): 2^bits buckets in u, at least 256 and about one
// per CDF entry (at most 2^20); entry b is the lower bound of b / 2^bits (exact in float), the last
// is the end. Returns 0 (no guide) when the CDF is not non-decreasing (a negative texel, or the last
// entry set to 1 below its predecessor's rounding): a binary search over unsorted entries depends on
// the order of its probes, and a narrowed search could then differ from the full one.
static int cdf_guide(const std::vector<float> &cdf, std::vector<int> &guide) {
    const int n1 = int(cdf.size());
    for (int i = 1; i < n1; ++i)
        if (!(cdf[i] >= cdf[i - 1])) return 0;
    int bits = 8;
    while ((1 << bits) < n1 - 1 && bits < 20) ++bits;
    const int G = 1 << bits;
    guide.assign(size_t(G) + 2, 0);
    int i = 0;
    for (int b = 0; b <= G; ++b) {
        const float t = float(b) / float(G);
        while (i < n1 && cdf[i] < t) ++i;
        guide[b] = i;
    }
    guide[size_t(G) + 1] = n1;
    return bits;
}

// Spline<3>::build1d (renderer/include/spline.h:686-714): causal + anticausal recursive filter,
// pole z1 = sqrt(3) - 2, mirror boundary.
static void prefilter_1d(const float *data, long off, long stride, int size, float *out) {
    const float z1 = -2.0f + std::sqrt(3.0f);
    std::vector<float> cp(size), cn(size);
    float c0 = 0.0f;
    for (int i = 0; i < size; ++i) c0 += data[off + i * stride] * float(std::pow(double(z1), i));
    for (int i = size - 2; i > 0; --i) c0 += data[off + i * stride] * float(std::pow(double(z1), 2 * size - 2 - i));
    c0 /= float(1.0 - std::pow(double(z1), 2 * size - 2));
    cp[0] = c0;
    for (int i = 1; i < size; ++i) cp[i] = data[off + i * stride] + z1 * cp[i - 1];
    cn[size - 1] = z1 / (z1 * z1 - 1.0f) * (cp[size - 1] + z1 * cp[size - 2]);
    for (int i = size - 2; i >= 0; --i) cn[i] = z1 * (cn[i + 1] - cp[i]);
    for (int i = 0; i < size; ++i) out[i] = 6.0f * cn[i];
}

// Spline<3>::build3d (spline.h:739-764): y, then x, then z passes
static void prefilter_3d(const float *samples, const int N[3], float *coeff) {
    const long s01 = long(N[0]) * N[1];
    std::vector<float> tmp(std::max(std::max(N[0], N[1]), N[2]));
    for (int k = 0; k < N[2]; ++k)
        for (int i = 0; i < N[0]; ++i) {
            prefilter_1d(samples, k * s01 + i, N[0], N[1], tmp.data());
            for (int t = 0; t < N[1]; ++t) coeff[i + t * N[0] + k * s01] = tmp[t];
        }
    for (int k = 0; k < N[2]; ++k)
        for (int j = 0; j < N[1]; ++j) {
            prefilter_1d(coeff, k * s01 + long(j) * N[0], 1, N[0], tmp.data());
            for (int t = 0; t < N[0]; ++t) coeff[t + j * N[0] + k * s01] = tmp[t];
        }
    for (int i = 0; i < N[0]; ++i)
        for (int j = 0; j < N[1]; ++j) {
            prefilter_1d(coeff, long(j) * N[0] + i, s01, N[2], tmp.data());
            for (int t = 0; t < N[2]; ++t) coeff[i + j * N[0] + t * s01] = tmp[t];
        }
}

// rif_sources::recompute_derived_ (renderer/include/rif_sources.h:156-198): centres of the
// point sources on the two arcs, arc 1 block then arc 2 block.
static void source_centres(const smp_field_desc &f, std::vector<float4> &out) {
    const float radius = float(f.radius), chord = float(f.chordlength);
    float tmin = -std::asin(chord / (2.0f * radius)), tmax = std::asin(chord / (2.0f * radius));
    float zmin = -chord / 2.0f, zmax = chord / 2.0f;
    if (f.theta_max > f.theta_min) {
        tmin = float(f.theta_min); tmax = float(f.theta_max);
        zmin = float(f.trans_z_min); zmax = float(f.trans_z_max);
    }
    const int nt = f.theta_sources, nz = f.trans_z_sources, ns = nt * nz;
    const float tdiff = (tmax - tmin) / float(nt - 1), zdiff = (zmax - zmin) / float(nz - 1);
    out.assign(size_t(2) * ns, make_float4(0, 0, 0, 0));
    for (int i = 0; i < nt; ++i) {
        float th = tmin + tdiff * float(i);
        float xv = radius * (1.0f - std::cos(th)), yv = radius * std::sin(th);
        for (int j = 0; j < nz; ++j) {
            int k = i + j * nt;
            float zx = zmin + zdiff * float(j);
            out[k] = make_float4(zx + float(f.center1[0]), yv + float(f.center1[1]), xv + float(f.center1[2]), 0.0f);
            out[ns + k] = make_float4(zx + float(f.center2[0]), xv + float(f.center2[1]), yv + float(f.center2[2]), 0.0f);
        }
    }
}

// The offsets as x-tap quads (FieldParams.coeff4): entry row * N0 + x holds the offsets at the
// mirrored x - 1, x, x + 1, x + 2 of that row, the four taps of a point with floor(t_x) = x.
static int spline_mirror(int i, int n) {
    int m = 2 * n - 2, w = i % m;
    if (w < 0) w += m;
    return w >= n ? m - w : w;
}
static void spline_quads(const int N[3], const std::vector<float> &delta, std::vector<float4> &quads) {
    const size_t rows = size_t(N[1]) * N[2];
    quads.resize(rows * N[0]);
    for (size_t r = 0; r < rows; ++r)
        for (int x = 0; x < N[0]; ++x) {
            const float *row = delta.data() + r * N[0];
            quads[r * N[0] + x] = make_float4(row[spline_mirror(x - 1, N[0])], row[x], row[spline_mirror(x + 1, N[0])],
                                              row[spline_mirror(x + 2, N[0])]);
        }
}

// The quads again with their rows padded for the brick march kernel (dev_field.cuh kSplineBrick): row
// (y', z') of the padded array is grid row (y' - 1, z' - 1) under the mirror rule, y' in [0, N1 + 3),
// z' in [0, N2 + 3) -- every row a tap of an on-grid point can need.
static void spline_quads_padded(const int N[3], const std::vector<float> &delta, std::vector<float4> &quads) {
    const int ny = N[1] + 3, nz = N[2] + 3;
    quads.resize(size_t(N[0]) * ny * nz);
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y) {
            const float *row = delta.data() + (size_t(spline_mirror(z - 1, N[2])) * N[1] + spline_mirror(y - 1, N[1])) * N[0];
            float4 *out = quads.data() + (size_t(z) * ny + y) * N[0];
            for (int x = 0; x < N[0]; ++x)
                out[x] = make_float4(row[spline_mirror(x - 1, N[0])], row[x], row[spline_mirror(x + 1, N[0])],
                                     row[spline_mirror(x + 2, N[0])]);
        }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }
    return fn;
}

// Spline coefficients as float offsets from their mean (see spline_field in dev_field.cuh).
static float spline_offsets(const smp_field_desc &f, std::vector<float> &delta) {
    size_t n = size_t(f.grid_n[0]) * f.grid_n[1] * f.grid_n[2];
    double mean = 0.0;
    for (size_t i = 0; i < n; ++i) mean += f.grid_coeff[i];
    mean /= double(n);
    float base = float(f.grid_offset + mean);
    delta.resize(n);
    for (size_t i = 0; i < n; ++i) delta[i] = float(double(f.grid_coeff[i]) + f.grid_offset - double(base));
    return base;
}

// Bessel table for the march: intervals of width h = 1/16 in x = k r up to x_max (<= 128). For
// each interval, the cubic Hermite interpolant of J_m and of J_m+1 from their values and
// derivatives at both ends (libstdc++'s std::cyl_bessel_j in double; J_n' = (J_{n-1} - J_{n+1})/2,
// J_{-1} = -J_1), written in powers of f = x/h - i and rounded to float:
//   p(f) = J_0 + h J_0' f + (3 (J_1 - J_0) - h (2 J_0' + J_1')) f^2 + (2 (J_0 - J_1) + h (J_0' + J_1')) f^3
static const double kBesselH = 1.0 / 16.0;
static const double kBesselMaxX = 128.0;
// Orders above 2 read J_m and J_m+1 from the table alone (no closed form beyond it), so their plans
// need the box's largest k r within kBesselMaxX; cos(m phi) takes m - 1 complex products.
static const int kBesselMaxOrder = 64;
static int bessel_intervals(double x_max) {
    x_max = std::min(std::max(x_max, 1.0), kBesselMaxX);
    return int(std::ceil(x_max / kBesselH)) + 1;
}
static void bessel_table_fill(int m, int intervals, float4 *tab) {
    auto J = [](int n, double x) -> double {
        if (n < 0) return (n % 2 ? -1.0 : 1.0) * std::cyl_bessel_j(double(-n), x);
        return std::cyl_bessel_j(double(n), x);
    };
    auto cubic = [](double j0, double d0, double j1, double d1, double h) {
        return make_float4(float(j0), float(h * d0), float(3.0 * (j1 - j0) - h * (2.0 * d0 + d1)),
                           float(2.0 * (j0 - j1) + h * (d0 + d1)));
    };
    double a0 = J(m, 0.0), a1 = J(m + 1, 0.0);
    double da0 = 0.5 * (J(m - 1, 0.0) - a1), da1 = 0.5 * (a0 - J(m + 2, 0.0));
    for (int i = 0; i < intervals; ++i) {
        const double x = (i + 1) * kBesselH;
        const double b0 = J(m, x), b1 = J(m + 1, x);
        const double db0 = 0.5 * (J(m - 1, x) - b1), db1 = 0.5 * (b0 - J(m + 2, x));
        tab[2 * i] = cubic(a0, da0, b0, db0, kBesselH);
        tab[2 * i + 1] = cubic(a1, da1, b1, db1, kBesselH);
        a0 = b0; a1 = b1; da0 = db0; da1 = db1;
    }
}
static void bessel_table(int m, double x_max, std::vector<float4> &tab) {
    const int intervals = bessel_intervals(x_max);
    tab.resize(2 * size_t(intervals));
    bessel_table_fill(m, intervals, tab.data());
}

// largest k*r the march can meet: the box's extent about the -x axis
static double box_max_kr(const smp_scene_desc &s, float k_r) {
    double ry = std::max(std::fabs(s.medium_l[1]), std::fabs(s.medium_r[1]));
    double rz = std::max(std::fabs(s.medium_l[2]), std::fabs(s.medium_r[2]));
    return double(k_r) * std::sqrt(ry * ry + rz * rz) * 1.01 + 1.0;
}

// util.h:42-57 in float, for the entry Fresnel transmission (scene.h:144-164)
static float fresnel_host(float cosI, float cosT, float eta) {
    if (std::fabs(eta - 1.0f) < 1.19209290e-07f * std::max(1.0f, std::fabs(eta))) return 0.0f;
    float Rs = (cosI - eta * cosT) / (cosI + eta * cosT);
    float Rp = (cosT - eta * cosI) / (cosT + eta * cosI);
    return 0.5f * (Rs * Rs + Rp * Rp);
}

static int field_kind(const smp_field_desc &f, int *fk) {
    switch (f.type) {
        case SMP_FIELD_BESSEL:
            if (f.mode < 0 || f.mode > kBesselMaxOrder)
                return set_error(SMP_ERR_UNSUPPORTED, "Bessel mode %d: orders 0..%d are built", f.mode, kBesselMaxOrder);
            *fk = f.mode <= 2 ? FK_BESSEL0 + f.mode : FK_BESSELN;
            return SMP_OK;
        case SMP_FIELD_PLANEWAVE:
            if (f.n_waves < 0 || f.n_waves > SMP_MAX_WAVES) return set_error(SMP_ERR_BAD_ARG, "n_waves out of range");
            *fk = FK_PLANEWAVE;
            return SMP_OK;
        case SMP_FIELD_SOURCES:
            if (f.theta_sources < 2 || f.trans_z_sources < 2 || f.n_coeff < 1)
                return set_error(SMP_ERR_BAD_ARG, "sources field needs theta_sources, trans_z_sources >= 2 and n_coeff >= 1");
            *fk = FK_SOURCES;
            return SMP_OK;
        case SMP_FIELD_SPLINE:
            for (int i = 0; i < 3; ++i)
                if (f.grid_n[i] < 2 || !(f.grid_max[i] > f.grid_min[i]))
                    return set_error(SMP_ERR_BAD_ARG, "spline grid axis %d invalid", i);
            if (!f.grid_coeff) return set_error(SMP_ERR_BAD_ARG, "spline grid_coeff is NULL");
            *fk = FK_SPLINE;
            return SMP_OK;
        default:
            return set_error(SMP_ERR_BAD_ARG, "unknown field type %d", f.type);
    }
}

// float field parameters shared by plans and probes (device pointers filled by the caller)
static void fill_field_params(const smp_field_desc &f, int fk, FieldParams &F) {
    std::memset(&F, 0, sizeof(F));
    F.kind = fk;
    F.mode = f.mode;
    F.n_o = float(f.n_o);
    F.egap = float(f.egap_end_x);
    F.sgap = float(f.sgap_begin_x);
    // rif_base.h:149-153 in Float: lambda = c/f, k = 2*pi/lambda
    float lambda = float(f.speed_u) / float(f.f_u);
    F.k_r = (2.0f * 3.14159265358979f) / lambda;
    F.inv_k = 1.0f / F.k_r;
    F.amp = float(f.n_max);
    F.max_scaling = float(f.n_clip) / float(f.n_max);       // rif_analytical.h:222
    F.phi_min = float(f.phi_min);
    F.phi_range = float(f.phi_max) - float(f.phi_min);
    F.n_waves = f.n_waves;
    for (int i = 0; i < SMP_MAX_WAVES && i < f.n_waves; ++i) {
        F.wamp[i] = float(f.wave_amp[i]);
        F.wphase[i] = float(f.wave_phase[i]);
        for (int j = 0; j < 3; ++j) F.wk[i][j] = float(f.wave_k[i][j]);
    }
    F.n_coeff = f.n_coeff;
    F.nsources = f.theta_sources * f.trans_z_sources;
    F.active1 = f.active1;
    F.active2 = f.active2;
    F.n_scaling = float(f.n_scaling);
    F.phase1 = float(f.phase1);
    F.phase2 = float(f.phase2);
    for (int i = 0; i < 3; ++i) {
        F.N[i] = f.grid_n[i];
        F.xmin[i] = float(f.grid_min[i]);
        F.xres[i] = float(f.grid_n[i] - 1) / (float(f.grid_max[i]) - float(f.grid_min[i]));
    }
    F.bh = float(kBesselH);
    F.binv_h = float(1.0 / kBesselH);
    F.kb = F.k_r * F.binv_h;
    // |grad n|_1 bounds for the march's checked windows. Bessel: |dn/dr| <= A k |J_m'| <= A k and
    // |dn/(r dphi)| = A k m |J_m(x)|/x <= A k (J_{m-1} + J_{m+1} = 2m J_m / x), so |grad n|_1 <= 2 A k;
    // the factor 4 leaves room for the table's interpolation error. Plane waves: sum |a_i| |k_i|_1.
    F.grad_bound = 0.0f;
    if (fk <= FK_BESSEL2) F.grad_bound = 4.0f * std::fabs(F.amp) * F.k_r;
    if (fk == FK_PLANEWAVE) {
        float G = 0.0f;
        for (int i = 0; i < F.n_waves; ++i)
            G += std::fabs(F.wamp[i]) * (std::fabs(F.wk[i][0]) + std::fabs(F.wk[i][1]) + std::fabs(F.wk[i][2]));
        F.grad_bound = 2.0f * G;
    }
}

// The box test of traceTillBlock, p - L > -eps and R - p > -eps in float, as thresholds:
// near a face p - L is exact (Sterbenz), so the test is p > L - eps in real arithmetic, i.e.
// p >= the smallest float above L - eps; likewise p <= the largest float below R + eps.
static float float_above(double x) {
    float f = float(x);
    if (double(f) <= x) f = std::nextafter(f, HUGE_VALF);
    while (double(std::nextafter(f, -HUGE_VALF)) > x) f = std::nextafter(f, -HUGE_VALF);
    return f;
}
static float float_below(double x) {
    float f = float(x);
    if (double(f) >= x) f = std::nextafter(f, -HUGE_VALF);
    while (double(std::nextafter(f, HUGE_VALF)) < x) f = std::nextafter(f, HUGE_VALF);
    return f;
}
// traceTillBlock's step sizes: h0 and each refinement's current_stepsize / 10 in float
static void step_table(double er_stepsize, float *tab) {
    tab[0] = float(er_stepsize);
    for (int i = 1; i <= SMP_MAX_REFINE; ++i) {
        volatile float q = tab[i - 1] / 10.0f;           // one IEEE float division per level
        tab[i] = q;
    }
}
static void set_step_sizes(KParams &k, const smp_field_desc &f) {
    k.h0 = float(f.er_stepsize);
    k.precision = std::max(0, std::min(int(f.precision), SMP_MAX_REFINE));
    step_table(f.er_stepsize, k.cur_tab);
}

// Runs f(begin, end) over [0, n) on up to 16 host threads.
template <class F>
static void host_parallel(size_t n, F f) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t per = (n + hw - 1) / hw;
    std::vector<std::thread> ts;
    for (unsigned t = 0; t < hw; ++t) {
        const size_t a = std::min(n, t * per), b = std::min(n, a + per);
        if (a < b) ts.emplace_back([&f, a, b] { f(a, b); });
    }
    for (auto &t : ts) t.join();
}

static void set_box_thresholds(KParams &k) {
    const double eps = double(1.19209290e-07f);
    for (int i = 0; i < 3; ++i) {
        k.box_lo[i] = float_above(double(k.L[i]) - eps);
        k.box_hi[i] = float_below(double(k.R[i]) + eps);
    }
}

// LargeDist of movePhotonTillSensor (scene.cpp:627): 1e4 m in the reference; by default capped
// where weight*exp(-sigma_t*d) underflows to 0 in FP32 (sigma_t*d > 110).
static float sensor_march_budget(const smp_render_opts &o, float sigma_t) {
    if (o.sensor_march_max > 0.0) return float(o.sensor_march_max);
    float d = 10000.0f;
    if (sigma_t > 0.0f) d = std::min(d, 110.0f / sigma_t);
    return d;
}

static int check_device(int dev) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return set_error(SMP_ERR_NO_DEVICE, "no CUDA device");
    if (dev < 0 || dev >= n) return set_error(SMP_ERR_BAD_ARG, "device %d out of range (%d devices)", dev, n);
    cudaDeviceProp prop;
    SMP_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10) return set_error(SMP_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a", dev, prop.major, prop.minor);
    SMP_CUDA(cudaSetDevice(dev));
    return SMP_OK;
}

// ---- kernel dispatch ---------------------------------------------------------------------------
static const int kBlock = 128;

// Kernels that stage the Bessel table take it as dynamic shared memory; above the default 48 KB
// window (a table for k r beyond about 96) a kernel must be opted in to the larger size first.
static int allow_dynamic_smem(const void *fn, size_t bytes) {
    if (bytes <= 48u * 1024u) return SMP_OK;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    if (e != cudaSuccess)
        return set_error(SMP_ERR_CUDA, "shared memory of %zu bytes for the Bessel table: %s", bytes, cudaGetErrorString(e));
    return SMP_OK;
}

static int grid_for(int fk, int dev, int blocks_per_sm, size_t smem, int *grid) {
    MarchFn fn = march_fn(fk);
    int rc = allow_dynamic_smem(reinterpret_cast<const void *>(fn), smem);
    if (rc) return rc;
    int per_sm = blocks_per_sm;
    if (per_sm <= 0) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, smem);
        if (e != cudaSuccess) return set_error(SMP_ERR_CUDA, "occupancy query: %s", cudaGetErrorString(e));
        if (per_sm < 1) per_sm = 1;
    }
    int sms = 0;
    SMP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    *grid = sms * per_sm;
    return SMP_OK;
}

// ---- plans -------------------------------------------------------------------------------------
struct smp_plan {
    int device = 0;
    int fk = 0;
    int grid = 0;
    smp_scene_desc scene;
    smp_medium_desc medium;
    smp_field_desc field;
    smp_render_opts opts;
    KParams kp;                 // filled except weight / work range / counters
    float *d_cdf = nullptr;
    float4 *d_centers = nullptr;
    float *d_coeff = nullptr;
    float4 *d_coeff4 = nullptr;
    float4 *d_btab = nullptr;
    size_t smem_bytes = 0;
    // spline bricks (wavefront.cuh wf_march_spline_kernel): padded quads, their TMA map, brick counts
    bool bricks = false;        // smp_render_opts.spline_bricks (spline fields)
    float4 *d_bquads = nullptr;
    CUtensorMap bmap;
    int nb = 0, nbx = 0, nby = 0, nbz = 0, bdim[3] = {0, 0, 0};
    void *d_blist = nullptr;    // two parities of nb brick lists (wave_setup) and their counts
    size_t blist_cap = 0;       // slots per brick list
    size_t march_smem = 0;      // dynamic shared memory of the pool's march kernel
    int event_batch = 8;
    void *d_film = nullptr;
    size_t film_elems = 0;
    unsigned long long *d_counters = nullptr;
    smp_stats stats;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> launches;   // since the last clear
    // the slot pool of the two-kernel march (wavefront.cuh); allocated at the first trace
    int kernel = SMP_KERNEL_POOL;   // smp_kernel (opts.kernel, or SMP_KERNEL=pool|persistent|plain)
    int wave_chunk = 96;
    int wave_slots_per_lane = 6;
    int march_block = 128;      // threads per march-kernel block (128 or 256)
    bool tuned = false;         // the schedule came from smp_plan_tune
    size_t wave_cap = 0;        // slots the pool allocation holds
    int wave_batch = 16;        // march/event launch pairs between live-slot checks
    int wave_split = 1;         // march lists and event queues by march class (WaveParams.split)
    void *d_wave = nullptr;
    size_t wave_bytes = 0;
    WaveParams wp;
    int grid_march = 0, grid_event = 0, grid_finish = 0;
    unsigned long long *h_live = nullptr;   // pinned: [live slots, march-kernel steps] x 2 batches
    cudaEvent_t live_ev[2] = {nullptr, nullptr};
    cudaEvent_t batch_ev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    // online chunk tuning: steady-state batches (pool full) cycle through the candidates, two
    // each, and the plan keeps the fastest for the rest of its life (no extra work is traced)
    bool tune_chunk = true;
    int tuned_chunk = 0;
    // SMP_WF_GRAPH=1: once the chunk is fixed, each batch of march/event pairs is one CUDA graph
    // launch (captured once per trace); march launches inside graphs are not timed individually
    bool use_graph = false;
    cudaStream_t cap_stream = nullptr;
    long long graph_march_launches = 0;
    double tune_rate[4] = {0, 0, 0, 0};
    int tune_n[4] = {0, 0, 0, 0};
    // adjoint buffers (smp_plan_adjoint), kept for the plan's life and grown on demand
    void *adj_buf = nullptr;
    size_t adj_bytes = 0;
    long long adj_batch = 0, adj_traj_mb = 0;   // adjoint batch and trajectory buffer, fixed at the first adjoint
    std::vector<cudaEvent_t> march_ev;   // event pairs around march-kernel launches (a reused pool)
    size_t march_ev_used = 0;            // since the last clear
    long long n_launched = 0;            // kernels launched since the last clear
};

static void drop_launch_events(smp_plan *p) {
    for (auto &e : p->launches) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    p->launches.clear();
}

static void plan_free(smp_plan *p) {
    if (!p) return;
    cudaFree(p->d_cdf);
    cudaFree(p->d_centers);
    cudaFree(p->d_coeff);
    cudaFree(p->d_coeff4);
    cudaFree(p->d_bquads);
    cudaFree(p->d_blist);
    cudaFree(p->d_btab);
    cudaFree(p->d_film);
    cudaFree(p->d_counters);
    cudaFree(p->d_wave);
    cudaFree(p->adj_buf);
    if (p->h_live) cudaFreeHost(p->h_live);
    for (int i = 0; i < 2; ++i) {
        if (p->live_ev[i]) cudaEventDestroy(p->live_ev[i]);
        for (int j = 0; j < 2; ++j) if (p->batch_ev[i][j]) cudaEventDestroy(p->batch_ev[i][j]);
    }
    for (cudaEvent_t e : p->march_ev) cudaEventDestroy(e);
    if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
    drop_launch_events(p);
    delete p;
}

static int check_descs(const smp_scene_desc *s, const smp_medium_desc *m, const smp_field_desc *f,
                       const smp_render_opts *o) {
    if (!s || !m || !f || !o) return set_error(SMP_ERR_BAD_ARG, "NULL descriptor");
    if (s->x_res <= 0 || s->y_res <= 0 || s->z_res <= 0) return set_error(SMP_ERR_BAD_ARG, "film resolution must be positive");
    if (s->tex_x <= 0 || s->tex_y <= 0 || !s->texture) return set_error(SMP_ERR_BAD_ARG, "texture missing");
    if (!(f->er_stepsize > 0.0)) return set_error(SMP_ERR_BAD_ARG, "er_stepsize must be positive");
    if (f->precision > SMP_MAX_REFINE)
        return set_error(SMP_ERR_UNSUPPORTED, "precision %d: at most %d refinement levels", f->precision, SMP_MAX_REFINE);
    if (!(f->f_u > 0.0) || !(f->speed_u > 0.0)) return set_error(SMP_ERR_BAD_ARG, "f_u and speed_u must be positive");
    if (o->precision != SMP_PREC_FP32 && o->precision != SMP_PREC_MIXED) return set_error(SMP_ERR_BAD_ARG, "bad precision");
    if (o->rng != SMP_RNG_PHILOX && o->rng != SMP_RNG_STREAM)
        return set_error(SMP_ERR_UNSUPPORTED, "rng %d: the march kernel draws from Philox or an injected stream", o->rng);
    if (m->albedo > 1.0 || m->albedo < 0.0) return set_error(SMP_ERR_BAD_ARG, "albedo outside [0,1]");
    return SMP_OK;
}

static int plan_setup_field(smp_plan *p, const smp_field_desc &f) {
    int rc = field_kind(f, &p->fk);
    if (rc) return rc;
    fill_field_params(f, p->fk, p->kp.field);
    if (p->fk == FK_SOURCES) {
        std::vector<float4> c;
        source_centres(f, c);
        cudaFree(p->d_centers);
        p->d_centers = nullptr;
        SMP_CUDA(cudaMalloc(&p->d_centers, c.size() * sizeof(float4)));
        SMP_CUDA(cudaMemcpy(p->d_centers, c.data(), c.size() * sizeof(float4), cudaMemcpyHostToDevice));
        p->kp.field.centers = p->d_centers;
    }
    if (p->fk == FK_SPLINE) {
        std::vector<float> delta;
        p->kp.field.spline_base = spline_offsets(f, delta);
        cudaFree(p->d_coeff);
        p->d_coeff = nullptr;
        SMP_CUDA(cudaMalloc(&p->d_coeff, delta.size() * sizeof(float)));
        SMP_CUDA(cudaMemcpy(p->d_coeff, delta.data(), delta.size() * sizeof(float), cudaMemcpyHostToDevice));
        p->kp.field.coeff = p->d_coeff;
        std::vector<float4> quads;
        spline_quads(f.grid_n, delta, quads);
        cudaFree(p->d_coeff4);
        p->d_coeff4 = nullptr;
        SMP_CUDA(cudaMalloc(&p->d_coeff4, quads.size() * sizeof(float4)));
        SMP_CUDA(cudaMemcpy(p->d_coeff4, quads.data(), quads.size() * sizeof(float4), cudaMemcpyHostToDevice));
        p->kp.field.coeff4 = p->d_coeff4;
        // bricks for the slot pool's march kernel (opts.spline_bricks): the padded quads and a tiled
        // TMA map over them
        const int nbx = (f.grid_n[0] + kSplineBrick - 1) / kSplineBrick, nby = (f.grid_n[1] + kSplineBrick - 1) / kSplineBrick,
                  nbz = (f.grid_n[2] + kSplineBrick - 1) / kSplineBrick;
        p->bricks = p->opts.spline_bricks != 0;
        if (p->bricks && nbx * nby * nbz > kMaxBricks)
            return set_error(SMP_ERR_UNSUPPORTED, "spline bricks: the grid has %d bricks of %d^3 cells, at most %d are built",
                             nbx * nby * nbz, kSplineBrick, kMaxBricks);
        if (p->bricks && tensor_map_encoder() == nullptr)
            return set_error(SMP_ERR_CUDA, "spline bricks: cuTensorMapEncodeTiled is not available from the driver");
        cudaFree(p->d_bquads);
        p->d_bquads = nullptr;
        if (p->bricks) {
            std::vector<float4> pq;
            spline_quads_padded(f.grid_n, delta, pq);
            SMP_CUDA(cudaMalloc(&p->d_bquads, pq.size() * sizeof(float4)));
            SMP_CUDA(cudaMemcpy(p->d_bquads, pq.data(), pq.size() * sizeof(float4), cudaMemcpyHostToDevice));
            p->nbx = nbx; p->nby = nby; p->nbz = nbz; p->nb = nbx * nby * nbz;
            p->bdim[0] = f.grid_n[0]; p->bdim[1] = f.grid_n[1] + 3; p->bdim[2] = f.grid_n[2] + 3;
            const cuuint64_t dims[4] = {4, cuuint64_t(p->bdim[0]), cuuint64_t(p->bdim[1]), cuuint64_t(p->bdim[2])};
            const cuuint64_t strides[3] = {16, 16ull * p->bdim[0], 16ull * p->bdim[0] * p->bdim[1]};
            const cuuint32_t box[4] = {4, cuuint32_t(kSplineBrick), cuuint32_t(kSplineBrickRows), cuuint32_t(kSplineBrickRows)};
            const cuuint32_t estr[4] = {1, 1, 1, 1};
            CUresult r = tensor_map_encoder()(&p->bmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, p->d_bquads, dims, strides, box,
                                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return set_error(SMP_ERR_CUDA, "cuTensorMapEncodeTiled (spline bricks) failed: %d", int(r));
        }
    } else {
        p->bricks = false;
    }
    p->smem_bytes = 0;
    if (p->fk <= FK_BESSELN) {
        const double xmax = box_max_kr(p->scene, p->kp.field.k_r);
        if (p->fk == FK_BESSELN && xmax > kBesselMaxX)
            return set_error(SMP_ERR_UNSUPPORTED, "Bessel mode %d: k r reaches %.1f over the box; orders above 2 "
                             "are built for k r <= %.0f", f.mode, xmax, kBesselMaxX);
        std::vector<float4> tab;
        bessel_table(f.mode, xmax, tab);
        cudaFree(p->d_btab);
        p->d_btab = nullptr;
        SMP_CUDA(cudaMalloc(&p->d_btab, tab.size() * sizeof(float4)));
        SMP_CUDA(cudaMemcpy(p->d_btab, tab.data(), tab.size() * sizeof(float4), cudaMemcpyHostToDevice));
        p->kp.field.btab = p->d_btab;
        p->kp.field.bnodes = int(tab.size());
        p->kp.field.bint = int(tab.size() / 2);
        p->smem_bytes = tab.size() * sizeof(float4);
    }
    set_step_sizes(p->kp, f);
    p->field = f;
    return grid_for(p->fk, p->device, p->opts.blocks_per_sm, p->smem_bytes, &p->grid);
}

extern "C" {

int smp_version(void) { return SMP_ABI_VERSION; }
const char *smp_last_error(void) { return g_last_error.c_str(); }
int smp_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

size_t smp_sizeof(const char *t) {
    if (!t) return 0;
    if (!std::strcmp(t, "smp_field_desc")) return sizeof(smp_field_desc);
    if (!std::strcmp(t, "smp_scene_desc")) return sizeof(smp_scene_desc);
    if (!std::strcmp(t, "smp_medium_desc")) return sizeof(smp_medium_desc);
    if (!std::strcmp(t, "smp_render_opts")) return sizeof(smp_render_opts);
    if (!std::strcmp(t, "smp_stats")) return sizeof(smp_stats);
    if (!std::strcmp(t, "smp_photon_record")) return sizeof(smp_photon_record);
    if (!std::strcmp(t, "smp_splat_record")) return sizeof(smp_splat_record);
    if (!std::strcmp(t, "smp_instance_desc")) return sizeof(smp_instance_desc);
    if (!std::strcmp(t, "smp_adjoint_stats")) return sizeof(smp_adjoint_stats);
    if (!std::strcmp(t, "smp_tuning")) return sizeof(smp_tuning);
    return 0;
}

int smp_texture_cdf(const double *texture, int32_t tex_x, int32_t tex_y, float *cdf_out) {
    if (!texture || !cdf_out || tex_x <= 0 || tex_y <= 0) return set_error(SMP_ERR_BAD_ARG, "bad texture");
    std::vector<float> cdf;
    texture_cdf(texture, tex_x * tex_y, cdf);
    std::memcpy(cdf_out, cdf.data(), cdf.size() * sizeof(float));
    return SMP_OK;
}

int smp_spline_prefilter(const float *samples, const int32_t n[3], float *coeff_out) {
    if (!samples || !n || !coeff_out) return set_error(SMP_ERR_BAD_ARG, "NULL argument");
    int N[3] = {n[0], n[1], n[2]};
    for (int i = 0; i < 3; ++i)
        if (N[i] < 2) return set_error(SMP_ERR_BAD_ARG, "spline axis %d needs >= 2 samples", i);
    prefilter_3d(samples, N, coeff_out);
    return SMP_OK;
}

int smp_plan_create(const smp_scene_desc *scene, const smp_medium_desc *medium, const smp_field_desc *field,
                    const smp_render_opts *opts, smp_plan **plan_out) {
    if (!plan_out) return set_error(SMP_ERR_BAD_ARG, "plan_out is NULL");
    *plan_out = nullptr;
    int rc = check_descs(scene, medium, field, opts);
    if (rc) return rc;
    rc = check_device(opts->device);
    if (rc) return rc;
    smp_plan *p = new smp_plan();
    p->device = opts->device;
    if (const char *eb = std::getenv("SMP_EVENT_BATCH")) p->event_batch = std::max(1, std::min(32, std::atoi(eb)));
    if (opts->kernel < SMP_KERNEL_POOL || opts->kernel > SMP_KERNEL_PLAIN) {
        delete p;
        return set_error(SMP_ERR_BAD_ARG, "kernel %d: not an smp_kernel", opts->kernel);
    }
    p->kernel = opts->kernel;
    if (const char *kn = std::getenv("SMP_KERNEL")) {
        if (!std::strcmp(kn, "persistent")) p->kernel = SMP_KERNEL_PERSISTENT;
        else if (!std::strcmp(kn, "plain")) p->kernel = SMP_KERNEL_PLAIN;
        else if (!std::strcmp(kn, "pool")) p->kernel = SMP_KERNEL_POOL;
    }
    if (const char *c = std::getenv("SMP_WF_CHUNK")) {
        p->wave_chunk = std::max(2, std::min(4096, std::atoi(c)));
        p->tune_chunk = false;
    }
    if (const char *c = std::getenv("SMP_WF_TUNE")) p->tune_chunk = p->tune_chunk && std::atoi(c) != 0;
    if (const char *c = std::getenv("SMP_WF_GRAPH")) p->use_graph = std::atoi(c) != 0;
    if (const char *c = std::getenv("SMP_WF_SLOTS")) p->wave_slots_per_lane = std::max(1, std::min(16, std::atoi(c)));
    if (const char *c = std::getenv("SMP_WF_BLOCK")) p->march_block = std::atoi(c) == 256 ? 256 : 128;
    if (const char *c = std::getenv("SMP_WF_BATCH")) p->wave_batch = std::max(1, std::min(256, std::atoi(c)));
    if (const char *c = std::getenv("SMP_WF_SPLIT")) p->wave_split = std::atoi(c) != 0;
    p->scene = *scene;
    p->medium = *medium;
    p->opts = *opts;
    std::memset(&p->stats, 0, sizeof(p->stats));
    KParams &k = p->kp;
    std::memset(&k, 0, sizeof(k));
    for (int i = 0; i < 3; ++i) {
        k.L[i] = float(scene->medium_l[i]);
        k.R[i] = float(scene->medium_r[i]);
        k.src_origin[i] = float(scene->light_origin[i]);
        k.src_lens_origin[i] = float(scene->emitter_lens_origin[i]);
        k.cam_origin[i] = float(scene->view_origin[i]);
        k.cam_lens_origin[i] = float(scene->sensor_lens_origin[i]);
    }
    set_box_thresholds(k);
    k.plane[0] = float(scene->light_plane[0]);
    k.plane[1] = float(scene->light_plane[1]);
    k.pixsize[0] = k.plane[0] / float(scene->tex_x);
    k.pixsize[1] = k.plane[1] / float(scene->tex_y);
    k.ct = std::cos(float(scene->half_theta_limit));
    k.tex_x = scene->tex_x;
    k.n_tex = scene->tex_x * scene->tex_y;
    k.src_lens_active = scene->emitter_lens_active;
    k.src_lens_sqap = float(scene->emitter_lens_aperture) * float(scene->emitter_lens_aperture);
    k.src_lens_focal = float(scene->emitter_lens_focal_length);
    // camera (camera.cpp:11-29): normalised dir and horizontal, vertical = dir x horizontal
    float cd[3], ch[3];
    for (int i = 0; i < 3; ++i) { cd[i] = float(scene->view_dir[i]); ch[i] = float(scene->view_horizontal[i]); }
    float ld = std::sqrt(cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
    float lh = std::sqrt(ch[0] * ch[0] + ch[1] * ch[1] + ch[2] * ch[2]);
    for (int i = 0; i < 3; ++i) { cd[i] = cd[i] / ld; ch[i] = ch[i] / lh; }
    for (int i = 0; i < 3; ++i) { k.cam_dir[i] = cd[i]; k.cam_h[i] = ch[i]; }
    k.cam_v[0] = cd[1] * ch[2] - cd[2] * ch[1];
    k.cam_v[1] = cd[2] * ch[0] - cd[0] * ch[2];
    k.cam_v[2] = cd[0] * ch[1] - cd[1] * ch[0];
    k.cam_plane[0] = float(scene->view_plane[0]);
    k.cam_plane[1] = float(scene->view_plane[1]);
    k.pl_min = float(scene->pathlength_range[0]);
    k.pl_max = float(scene->pathlength_range[1]);
    k.bounce = scene->use_bounce_decomposition;
    k.cam_lens_active = scene->sensor_lens_active;
    k.cam_lens_sqap = float(scene->sensor_lens_aperture) * float(scene->sensor_lens_aperture);
    k.cam_lens_focal = float(scene->sensor_lens_focal_length);
    k.ior1 = 1.0f;
    k.ior2 = float(scene->ior);
    // medium (medium.h:24-38)
    k.sigma_t = float(medium->sigma_t);
    k.albedo = float(medium->albedo);
    k.mfp = 1.0f / float(medium->sigma_t);
    if (k.sigma_t <= 1.19209290e-07f) { k.sigma_t = 0.0f; k.mfp = 1.0f; k.albedo = 0.0f; }
    k.g = float(medium->g);
    k.max_depth = opts->max_depth;
    k.max_pathlength = float(opts->max_pathlength);
    k.use_direct = opts->use_direct;
    k.use_angular = opts->use_angular_sampling;
    k.step_cap = opts->step_cap > 0 ? opts->step_cap : 10000000LL;
    k.large_dist = sensor_march_budget(*opts, k.sigma_t);
    if (k.step_cap > 2000000000LL) k.step_cap = 2000000000LL;
    k.X = scene->x_res; k.Y = scene->y_res; k.Z = scene->z_res;
    k.fp64 = opts->precision == SMP_PREC_MIXED;
    k.rng = opts->rng;
    k.seed = opts->seed;

    // texture CDF, and its guide table in the same allocation
    std::vector<float> cdf;
    texture_cdf(scene->texture, k.n_tex, cdf);
    std::vector<int> guide;
    const int gbits = cdf_guide(cdf, guide);
    const size_t cdf_bytes = (cdf.size() * sizeof(float) + 15) & ~size_t(15);
    cudaError_t e = cudaMalloc(&p->d_cdf, cdf_bytes + guide.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(p->d_cdf, cdf.data(), cdf.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && gbits)
        e = cudaMemcpy(reinterpret_cast<char *>(p->d_cdf) + cdf_bytes, guide.data(), guide.size() * sizeof(int),
                       cudaMemcpyHostToDevice);
    p->film_elems = size_t(k.X) * k.Y * k.Z;
    if (e == cudaSuccess) e = cudaMalloc(&p->d_film, p->film_elems * (k.fp64 ? 8 : 4));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_counters, CNT_COUNT * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(p->d_film, 0, p->film_elems * (k.fp64 ? 8 : 4));
    if (e == cudaSuccess) e = cudaMemset(p->d_counters, 0, CNT_COUNT * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        plan_free(p);
        return set_error(e == cudaErrorMemoryAllocation ? SMP_ERR_OOM : SMP_ERR_CUDA, "plan allocation: %s", cudaGetErrorString(e));
    }
    k.cdf = p->d_cdf;
    k.cdf_guide = gbits ? reinterpret_cast<const int *>(reinterpret_cast<const char *>(p->d_cdf) + cdf_bytes) : nullptr;
    k.guide_bits = gbits;
    k.film = p->d_film;
    k.counters = p->d_counters;
    rc = plan_setup_field(p, *field);
    if (rc) { plan_free(p); return rc; }
    *plan_out = p;
    return SMP_OK;
}

int smp_plan_destroy(smp_plan *plan) {
    if (!plan) return SMP_OK;
    cudaSetDevice(plan->device);
    plan_free(plan);
    return SMP_OK;
}

int smp_plan_set_field(smp_plan *plan, const smp_field_desc *field) {
    if (!plan || !field) return set_error(SMP_ERR_BAD_ARG, "NULL argument");
    SMP_CUDA(cudaSetDevice(plan->device));
    return plan_setup_field(plan, *field);
}

int smp_plan_clear(smp_plan *plan, void *stream) {
    if (!plan) return set_error(SMP_ERR_BAD_ARG, "NULL plan");
    SMP_CUDA(cudaSetDevice(plan->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    SMP_CUDA(cudaMemsetAsync(plan->d_film, 0, plan->film_elems * (plan->kp.fp64 ? 8 : 4), s));
    SMP_CUDA(cudaMemsetAsync(plan->d_counters, 0, CNT_COUNT * sizeof(unsigned long long), s));
    SMP_CUDA(cudaStreamSynchronize(s));
    drop_launch_events(plan);
    plan->march_ev_used = 0;
    plan->graph_march_launches = 0;
    plan->n_launched = 0;
    std::memset(&plan->stats, 0, sizeof(plan->stats));
    return SMP_OK;
}

// weight = Li * T_fresnel / N (photon.h:76-80) with T from scene.h:144-164, in float
static float photon_weight(const smp_scene_desc &s, int64_t n) {
    float ior = float(s.ior), T = 1.0f;
    if (ior > 1.0f) {
        float refr[3] = {0, 0, 0}, sum = 0.0f;
        for (int i = 1; i < 3; ++i) { refr[i] = float(s.light_dir[i]) / ior; sum += refr[i] * refr[i]; }
        refr[0] = std::sqrt(1.0f - sum);
        if (float(s.light_dir[0]) < 0.0f) refr[0] *= -1.0f;
        T = ior * ior * (1.0f - fresnel_host(float(s.light_dir[0]), refr[0], ior));
    }
    return float(s.Li) * T / float(n);
}

// Grid sizes from occupancy for the plan's current field kind, and the slot pool (slots = lanes of
// the march grid x wave_slots_per_lane), allocated at the first trace and grown if a new field
// kind needs more.
static int wave_bricks(smp_plan *p);

static int wave_setup(smp_plan *p) {
    const bool bricks = p->fk == FK_SPLINE && p->bricks;
    WaveFn fm = wf_march_fn(p->fk, p->kp.fp64 != 0, p->march_block, bricks), fe = wf_event_fn(p->fk),
           ff = wf_finish_fn(p->fk);
    if (!fm || !fe || !ff) return set_error(SMP_ERR_BAD_ARG, "bad field kind");
    p->march_smem = bricks ? size_t(kBrickSmemBytes) : p->smem_bytes;
    int sms = 0, pm = 0, pe = 0, pf = 0;
    int rc = allow_dynamic_smem(reinterpret_cast<const void *>(fm), p->march_smem);
    if (!rc) rc = allow_dynamic_smem(reinterpret_cast<const void *>(ff), p->smem_bytes);
    if (rc) return rc;
    SMP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device));
    SMP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pm, fm, p->march_block, p->march_smem));
    SMP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pe, fe, kBlock, 0));
    SMP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pf, ff, kBlock, p->smem_bytes));
    p->grid_march = sms * std::max(pm, 1);
    p->grid_event = sms * std::max(pe, 1);
    p->grid_finish = sms * std::max(pf, 1);
    const size_t n = size_t(p->grid_march) * size_t(p->march_block) * size_t(p->wave_slots_per_lane);
    p->wp.chunk = p->wave_chunk;
    if (p->d_wave && p->wave_cap >= n) {            // the allocation holds this many slots
        p->wp.n_slots = int(n);
        return wave_bricks(p);
    }
    cudaFree(p->d_wave);
    p->d_wave = nullptr;
    p->wave_cap = 0;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t b4 = al(n * sizeof(float4)), bi = al(n * sizeof(int4)), bd = al(n * sizeof(double)),
                 be = al(n * sizeof(EventPart)), bl = al(n * sizeof(int));
    const size_t bytes = 4 * b4 + bi + bd + be + 4 * bl + 256;
    cudaError_t e = cudaMalloc(&p->d_wave, bytes);
    if (e != cudaSuccess) {
        p->d_wave = nullptr;
        return set_error(e == cudaErrorMemoryAllocation ? SMP_ERR_OOM : SMP_ERR_CUDA, "slot pool (%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    p->wave_bytes = bytes;
    p->wave_cap = n;
    char *b = static_cast<char *>(p->d_wave);
    WaveParams &W = p->wp;
    W.ma = reinterpret_cast<float4 *>(b); b += b4;
    W.mb = reinterpret_cast<float4 *>(b); b += b4;
    W.mc = reinterpret_cast<float4 *>(b); b += b4;
    W.mdd = reinterpret_cast<float4 *>(b); b += b4;
    W.mi = reinterpret_cast<int4 *>(b); b += bi;
    W.mt = reinterpret_cast<double *>(b); b += bd;
    W.ev = reinterpret_cast<EventPart *>(b); b += be;
    W.list[0] = reinterpret_cast<int *>(b); b += bl;
    W.list[1] = reinterpret_cast<int *>(b); b += bl;
    W.queue[0] = reinterpret_cast<int *>(b); b += bl;
    W.queue[1] = reinterpret_cast<int *>(b); b += bl;
    W.cnt = reinterpret_cast<unsigned *>(b);
    W.n_slots = int(n);
    if (!p->h_live) SMP_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&p->h_live), 4 * sizeof(unsigned long long), cudaHostAllocDefault));
    for (int i = 0; i < 2; ++i) {
        if (!p->live_ev[i]) SMP_CUDA(cudaEventCreateWithFlags(&p->live_ev[i], cudaEventDisableTiming));
        for (int j = 0; j < 2; ++j) if (!p->batch_ev[i][j]) SMP_CUDA(cudaEventCreate(&p->batch_ev[i][j]));
    }
    return wave_bricks(p);
}

// The brick lists of a spline plan (two parities of nb lists of up to n_slots slot indices, and
// their counts), grown with the pool; the brick fields of the WaveParams.
static int wave_bricks(smp_plan *p) {
    WaveParams &W = p->wp;
    W.nb = 0;
    W.split = p->wave_split;
    if (!(p->bricks && p->fk == FK_SPLINE)) return SMP_OK;
    W.split = 0;                                    // the brick lists hold one class
    const size_t n = size_t(W.n_slots), nb = size_t(p->nb);
    if (!p->d_blist || p->blist_cap < n) {
        cudaFree(p->d_blist);
        p->d_blist = nullptr;
        p->blist_cap = 0;
        const size_t bytes = 2 * nb * n * sizeof(int) + 2 * nb * sizeof(unsigned) + 256;
        cudaError_t e = cudaMalloc(&p->d_blist, bytes);
        if (e != cudaSuccess) {
            p->d_blist = nullptr;
            return set_error(e == cudaErrorMemoryAllocation ? SMP_ERR_OOM : SMP_ERR_CUDA, "spline brick lists (%zu bytes): %s",
                             bytes, cudaGetErrorString(e));
        }
        p->blist_cap = n;
    }
    int *lists = static_cast<int *>(p->d_blist);
    W.blist[0] = lists;
    W.blist[1] = lists + nb * p->blist_cap;
    W.bcnt[0] = reinterpret_cast<unsigned *>(lists + 2 * nb * p->blist_cap);
    W.bcnt[1] = W.bcnt[0] + nb;
    W.bstride = int(p->blist_cap);
    W.nb = p->nb; W.nbx = p->nbx; W.nby = p->nby; W.nbz = p->nbz;
    W.bquads = p->d_bquads;
    for (int i = 0; i < 3; ++i) W.bdim[i] = p->bdim[i];
    W.bmap = p->bmap;
    return SMP_OK;
}

// Live slots from a readback of the two march-list counts of one parity (two unsigned in one word).
static unsigned long long live_of(unsigned long long word) {
    unsigned c[2];
    std::memcpy(c, &word, sizeof(c));
    return (unsigned long long)c[0] + c[1];
}

// The two-kernel march: fill the slots, then alternate march and event launches in batches of
// wave_batch pairs until no slot is live. The live count after each batch is read back while the
// next batch is already queued, so the device does not idle during the check.
static int wave_run(smp_plan *p, const KParams &k, cudaStream_t s) {
    int rc = wave_setup(p);
    if (rc) return rc;
    WaveFn fm = wf_march_fn(p->fk, p->kp.fp64 != 0, p->march_block, p->wp.nb > 0), fe = wf_event_fn(p->fk),
           ff = wf_finish_fn(p->fk);
    WaveParams W = p->wp;
    const int mb = p->march_block;
    if (W.nb > 0) SMP_CUDA(cudaMemsetAsync(W.bcnt[0], 0, 2 * size_t(W.nb) * sizeof(unsigned), s));
    // once the live slots fit in one persistent grid, the finisher runs them to the end
    const unsigned finish_at = unsigned(p->grid_finish) * unsigned(kBlock);
    SMP_CUDA(cudaMemsetAsync(W.cnt, 0, 8 * sizeof(unsigned), s));
    fe<<<p->grid_event, kBlock, 0, s>>>(k, W, -1);
    SMP_CUDA(cudaGetLastError());
    p->n_launched += 1;
    // every live photon advances at least one ER step per march launch, and no photon takes more
    // than step_cap steps, so the loop ends; the cap below only guards the host against a defect
    const long long max_iter = (long long)k.step_cap * 4 + (1LL << 20);
    long long it = 0;
    bool pending = false;
    int par = 0;                                     // ring slot of this batch's events and readback
    int cand_of[2] = {-1, -1};                       // tuning candidate a batch ran, -1: none
    unsigned long long prev_live = 0, prev_steps = 0;
    bool have_prev = false;
    static const int kChunkCand[4] = {64, 96, 128, 160};
    cudaGraphExec_t gexec = nullptr;                 // this trace's batch graph (graph mode)
    struct GraphGuard {
        cudaGraphExec_t *g;
        ~GraphGuard() { if (*g) cudaGraphExecDestroy(*g); }
    } gguard{&gexec};
    for (;;) {
        while (p->march_ev.size() < p->march_ev_used + 2 * size_t(p->wave_batch)) {
            cudaEvent_t e;
            SMP_CUDA(cudaEventCreate(&e));
            p->march_ev.push_back(e);
        }
        // chunk of this batch: the tuned value, or the next tuning candidate
        cand_of[par] = -1;
        W.chunk = p->tuned_chunk > 0 ? p->tuned_chunk : p->wave_chunk;
        if (p->tune_chunk && p->tuned_chunk == 0 && have_prev && prev_live == (unsigned long long)W.n_slots) {
            int c = 0;
            while (c < 3 && p->tune_n[c] >= 2) ++c;
            if (p->tune_n[c] < 2) { cand_of[par] = c; W.chunk = kChunkCand[c]; }
        }
        SMP_CUDA(cudaEventRecord(p->batch_ev[par][0], s));
        const bool graphed = p->use_graph && cand_of[par] < 0 && (p->tuned_chunk > 0 || !p->tune_chunk);
        if (graphed) {
            // batches start at even iterations, so one capture with it = 0 .. batch-1 serves all
            if (!gexec) {
                if (!p->cap_stream) SMP_CUDA(cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking));
                cudaGraph_t g = nullptr;
                SMP_CUDA(cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal));
                for (int j = 0; j < p->wave_batch; ++j) {
                    fm<<<p->grid_march, mb, p->march_smem, p->cap_stream>>>(k, W, j);
                    fe<<<p->grid_event, kBlock, 0, p->cap_stream>>>(k, W, j);
                }
                SMP_CUDA(cudaStreamEndCapture(p->cap_stream, &g));
                cudaError_t e = cudaGraphInstantiate(&gexec, g, 0ULL);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return set_error(SMP_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
            }
            SMP_CUDA(cudaGraphLaunch(gexec, s));
            it += p->wave_batch;
            p->graph_march_launches += p->wave_batch;
        } else {
            for (int j = 0; j < p->wave_batch; ++j, ++it) {
                SMP_CUDA(cudaEventRecord(p->march_ev[p->march_ev_used], s));
                fm<<<p->grid_march, mb, p->march_smem, s>>>(k, W, int(it & 0x3fffffff));
                SMP_CUDA(cudaEventRecord(p->march_ev[p->march_ev_used + 1], s));
                p->march_ev_used += 2;
                fe<<<p->grid_event, kBlock, 0, s>>>(k, W, int(it & 0x3fffffff));
            }
        }
        SMP_CUDA(cudaEventRecord(p->batch_ev[par][1], s));
        p->n_launched += 2 * p->wave_batch;
        SMP_CUDA(cudaGetLastError());
        if (pending) {                              // the previous batch's readback
            const int q = par ^ 1;
            SMP_CUDA(cudaEventSynchronize(p->live_ev[q]));
            const unsigned long long live = live_of(p->h_live[2 * q]), steps = p->h_live[2 * q + 1];
            if (cand_of[q] >= 0 && have_prev && live == (unsigned long long)W.n_slots && steps > prev_steps) {
                float ms = 0.0f;
                SMP_CUDA(cudaEventElapsedTime(&ms, p->batch_ev[q][0], p->batch_ev[q][1]));
                if (ms > 0.0f) {
                    p->tune_rate[cand_of[q]] += double(steps - prev_steps) / double(ms);
                    p->tune_n[cand_of[q]] += 1;
                    bool all = true;
                    for (int c = 0; c < 4; ++c) all = all && p->tune_n[c] >= 2;
                    if (all) {
                        int best = 0;
                        for (int c = 1; c < 4; ++c)
                            if (p->tune_rate[c] / p->tune_n[c] > p->tune_rate[best] / p->tune_n[best]) best = c;
                        p->tuned_chunk = kChunkCand[best];
                    }
                }
            }
            prev_live = live;
            prev_steps = steps;
            have_prev = true;
            if (live == 0u) break;
            // Fewer live slots than the slot pool means the photon counter is exhausted, and from
            // then on the count only falls, so the batch queued since holds at most `live`.
            if (live <= finish_at && live < (unsigned long long)W.n_slots) {
                ff<<<p->grid_finish, kBlock, p->smem_bytes, s>>>(k, W, int(it & 0x3fffffff));
                SMP_CUDA(cudaGetLastError());
                p->n_launched += 1;
                break;
            }
        }
        // live slots after this batch = the march list the next march launch reads; the march
        // kernel's step counter for the tuner
        p->h_live[2 * par] = 0;                       // free: its last readback was consumed above
        SMP_CUDA(cudaMemcpyAsync(p->h_live + 2 * par, W.cnt + 2 * (it & 1), 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        SMP_CUDA(cudaMemcpyAsync(p->h_live + 2 * par + 1, k.counters + CNT_MARCH_STEPS, sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, s));
        SMP_CUDA(cudaEventRecord(p->live_ev[par], s));
        pending = true;
        par ^= 1;
        if (it > max_iter) return set_error(SMP_ERR_CUDA, "march loop did not drain after %lld launches", it);
    }
    return SMP_OK;
}

static int launch(smp_plan *plan, int64_t first, int64_t n, int64_t weight_photons, cudaStream_t s,
                  const float *d_stream, const long long *d_offsets, smp_photon_record *d_records) {
    if (n <= 0) return SMP_OK;
    if (weight_photons <= 0) return set_error(SMP_ERR_BAD_ARG, "weight_photons must be positive");
    KParams k = plan->kp;
    k.weight = photon_weight(plan->scene, weight_photons);
    k.first_photon = first;
    k.n_photons = n;
    k.stream = d_stream;
    k.offsets = d_offsets;
    k.records = d_records;
    k.event_batch = plan->event_batch;
    if (d_stream) k.rng = SMP_RNG_STREAM;
    else if (k.rng == SMP_RNG_STREAM) return set_error(SMP_ERR_BAD_ARG, "rng STREAM needs uniforms");
    // the work counter restarts per launch; the statistics accumulate until smp_plan_clear
    SMP_CUDA(cudaMemsetAsync(plan->d_counters + CNT_NEXT_PHOTON, 0, sizeof(unsigned long long), s));
    cudaEvent_t e0, e1;
    SMP_CUDA(cudaEventCreate(&e0));
    SMP_CUDA(cudaEventCreate(&e1));
    plan->launches.emplace_back(e0, e1);
    SMP_CUDA(cudaEventRecord(e0, s));
    if (plan->kernel == SMP_KERNEL_PERSISTENT) {
        march_fn(plan->fk)<<<plan->grid, kBlock, plan->smem_bytes, s>>>(k);
        SMP_CUDA(cudaGetLastError());
        plan->n_launched += 1;
    } else if (plan->kernel == SMP_KERNEL_PLAIN) {
        MarchFn fp = plain_fn(plan->fk);
        if (!fp) return set_error(SMP_ERR_UNSUPPORTED, "no plain kernel for field kind %d", plan->fk);
        const long long blocks = (n + kPlainBlock - 1) / kPlainBlock;
        if (blocks > 0x7fffffffLL) return set_error(SMP_ERR_BAD_ARG, "too many photons for one plain launch");
        fp<<<unsigned(blocks), kPlainBlock, 0, s>>>(k);
        SMP_CUDA(cudaGetLastError());
        plan->n_launched += 1;
    } else {
        int rc = wave_run(plan, k, s);
        if (rc) return rc;
    }
    SMP_CUDA(cudaEventRecord(e1, s));
    return SMP_OK;
}

// Statistics since the last clear: device counters plus the summed launch times. Synchronises the
// device.
static int collect_stats(smp_plan *plan) {
    unsigned long long c[CNT_COUNT];
    SMP_CUDA(cudaDeviceSynchronize());
    SMP_CUDA(cudaMemcpy(c, plan->d_counters, sizeof(c), cudaMemcpyDeviceToHost));
    double ms_total = 0.0;
    for (auto &e : plan->launches) {
        float ms = 0.0f;
        SMP_CUDA(cudaEventElapsedTime(&ms, e.first, e.second));
        ms_total += ms;
    }
    plan->stats.photons = (int64_t)c[CNT_PHOTONS];
    plan->stats.er_steps = (int64_t)c[CNT_STEPS];
    plan->stats.splats = (int64_t)c[CNT_SPLATS];
    plan->stats.step_cap_hits = (int64_t)c[CNT_STEP_CAP];
    plan->stats.nan_photons = (int64_t)c[CNT_NAN];
    plan->stats.stream_exhausted = (int64_t)c[CNT_STREAM];
    plan->stats.kernel_ms = ms_total;
    double march_ms = 0.0;
    for (size_t i = 0; i + 1 < plan->march_ev_used; i += 2) {
        float ms = 0.0f;
        SMP_CUDA(cudaEventElapsedTime(&ms, plan->march_ev[i], plan->march_ev[i + 1]));
        march_ms += ms;
    }
    const bool one_kernel = plan->kernel != SMP_KERNEL_POOL;      // march and events in one kernel
    plan->stats.march_ms = one_kernel ? ms_total : march_ms;
    plan->stats.march_steps = one_kernel ? (int64_t)c[CNT_STEPS] : (int64_t)c[CNT_MARCH_STEPS];
    plan->stats.launches = plan->n_launched;
    plan->stats.march_block = plan->march_block;
    plan->stats.slots_per_lane = plan->wave_slots_per_lane;
    plan->stats.chunk = plan->tuned_chunk > 0 ? plan->tuned_chunk : (plan->tune_chunk ? 0 : plan->wave_chunk);
    plan->stats.tuned = plan->tuned ? 1 : 0;
    plan->stats.march_launches = one_kernel ? plan->n_launched
                                            : (int64_t)(plan->march_ev_used / 2) + plan->graph_march_launches;
    if (c[CNT_STAGE_TIMEOUT]) return set_error(SMP_ERR_CUDA, "%llu block(s) timed out staging the field table", c[CNT_STAGE_TIMEOUT]);
    if (c[CNT_LOST]) return set_error(SMP_ERR_CUDA, "internal: %llu live slot(s) had no lane in the tail kernel", c[CNT_LOST]);
    if (c[CNT_STEP_CAP]) return set_error(SMP_ERR_STEP_CAP, "%llu photon(s) hit the per-photon step cap", c[CNT_STEP_CAP]);
    if (c[CNT_NAN]) return set_error(SMP_ERR_NAN, "%llu photon(s) produced a non-finite state", c[CNT_NAN]);
    if (c[CNT_STREAM]) return set_error(SMP_ERR_STREAM, "%llu photon(s) ran out of injected uniforms", c[CNT_STREAM]);
    return SMP_OK;
}

int smp_plan_trace(smp_plan *plan, int64_t first_photon, int64_t n_photons, int64_t weight_photons, void *stream) {
    if (!plan || n_photons < 0 || first_photon < 0) return set_error(SMP_ERR_BAD_ARG, "bad plan / range");
    SMP_CUDA(cudaSetDevice(plan->device));
    return launch(plan, first_photon, n_photons, weight_photons, static_cast<cudaStream_t>(stream), nullptr,
                  nullptr, nullptr);
}

int smp_plan_stats(smp_plan *plan, smp_stats *stats_out) {
    if (!plan || !stats_out) return set_error(SMP_ERR_BAD_ARG, "NULL argument");
    SMP_CUDA(cudaSetDevice(plan->device));
    int rc = collect_stats(plan);
    *stats_out = plan->stats;
    return rc;
}

__global__ void film_to_double(const float *src, double *dst, size_t n) {
    size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (; i < n; i += stride) dst[i] = double(src[i]);
}

int smp_plan_read_image(smp_plan *plan, double *dst, int dst_is_device, void *stream) {
    if (!plan || !dst) return set_error(SMP_ERR_BAD_ARG, "NULL argument");
    SMP_CUDA(cudaSetDevice(plan->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t n = plan->film_elems;
    if (plan->kp.fp64) {
        SMP_CUDA(cudaMemcpyAsync(dst, plan->d_film, n * 8, dst_is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    } else if (dst_is_device) {
        film_to_double<<<592, 256, 0, s>>>(static_cast<const float *>(plan->d_film), dst, n);
        SMP_CUDA(cudaGetLastError());
    } else {
        std::vector<float> h(n);
        SMP_CUDA(cudaMemcpyAsync(h.data(), plan->d_film, n * 4, cudaMemcpyDeviceToHost, s));
        SMP_CUDA(cudaStreamSynchronize(s));
        for (size_t i = 0; i < n; ++i) dst[i] = double(h[i]);
    }
    SMP_CUDA(cudaStreamSynchronize(s));
    return SMP_OK;
}

int smp_plan_film(smp_plan *plan, void **dev_ptr, int32_t *bytes_per_pixel) {
    if (!plan || !dev_ptr || !bytes_per_pixel) return set_error(SMP_ERR_BAD_ARG, "NULL argument");
    *dev_ptr = plan->d_film;
    *bytes_per_pixel = plan->kp.fp64 ? 8 : 4;
    return SMP_OK;
}

int smp_plan_render(smp_plan *plan, int64_t n_photons, double *image_out, smp_stats *stats_out) {
    if (!plan || n_photons < 0) return set_error(SMP_ERR_BAD_ARG, "bad plan / photon count");
    int rc = smp_plan_clear(plan, nullptr);
    if (rc) return rc;
    if (n_photons > 0) {
        rc = smp_plan_trace(plan, 0, n_photons, n_photons, nullptr);
        if (rc) return rc;
    }
    int rs = n_photons > 0 ? collect_stats(plan) : SMP_OK;
    if (image_out) {
        rc = smp_plan_read_image(plan, image_out, 0, nullptr);
        if (rc) return rc;
    }
    if (stats_out) *stats_out = plan->stats;
    return rs;
}

}  // extern "C"

// ---- autotuner ------------------------------------------------------------------------------------
// Trial traces over march-kernel block size x slots per lane x chunk; the winner is kept by the plan
// and cached per process under a key of everything that changes the march's cost. A batched sweep's
// key is its scene, film and first instance's medium (not the instance list), so a smaller sweep of
// the same scene run first tunes the larger one.
namespace {
std::mutex g_tune_mutex;
std::map<std::string, smp_tuning> g_tune_cache;

std::string tune_key(const smp_plan *p, int64_t n_sample) {
    const KParams &k = p->kp;
    const FieldParams &F = k.field;
    cudaDeviceProp prop;
    std::string dev = cudaGetDeviceProperties(&prop, p->device) == cudaSuccess ? prop.name : "?";
    char buf[768];
    std::snprintf(buf, sizeof(buf),
                  "%s|%d|fk%d|fp%d|%dx%dx%d|tex%d|st%.9g|al%.9g|g%.9g|h%.9g|pr%d|amp%.9g|k%.9g|m%d|w%d|N%d,%d,%d|"
                  "dir%d|ang%d|md%d|L%.9g,%.9g,%.9g|R%.9g,%.9g,%.9g|ni%d|n%lld",
                  dev.c_str(), p->device, p->fk, k.fp64, k.X, k.Y, k.Z, k.n_tex, k.sigma_t, k.albedo, k.g, k.h0,
                  k.precision, F.amp, F.k_r, F.mode, F.n_waves, F.N[0], F.N[1], F.N[2], k.use_direct, k.use_angular,
                  k.max_depth, k.L[0], k.L[1], k.L[2], k.R[0], k.R[1], k.R[2], k.n_inst > 0 ? 1 : 0,
                  (long long)n_sample);
    return buf;
}

void tune_apply(smp_plan *p, const smp_tuning &t) {
    p->tuned = true;
    p->march_block = t.march_block;
    p->wave_slots_per_lane = t.slots_per_lane;
    p->wave_chunk = t.chunk;
    p->tuned_chunk = t.chunk;
    p->tune_chunk = false;
}

// one timed trial trace of photons [0, n) into the (cleared) film
int tune_trial(smp_plan *p, int64_t n, int64_t weight, double *ms) {
    int rc = smp_plan_clear(p, nullptr);
    if (rc) return rc;
    cudaEvent_t a, b;
    SMP_CUDA(cudaEventCreate(&a));
    SMP_CUDA(cudaEventCreate(&b));
    cudaEventRecord(a, nullptr);
    rc = launch(p, 0, n, weight, nullptr, nullptr, nullptr, nullptr);
    cudaEventRecord(b, nullptr);
    cudaError_t e = cudaEventSynchronize(b);
    float f = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&f, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    if (e != cudaSuccess) return set_error(SMP_ERR_CUDA, "tuning trial: %s", cudaGetErrorString(e));
    rc = collect_stats(p);
    *ms = f;
    return rc;
}
}  // namespace

// The tuner. n_grow > n_sample (a batched sweep, whose whole render is cheap per photon): the trial
// size is chosen from two warm-up traces instead, which separate a trace's fixed cost (the fill,
// and the tail: one photon trapped by total internal reflection marching alone, tens of ms) from its
// cost per photon, so that every trial holds about 250 ms of work per photon -- up to n_grow
// photons -- and the tails do not decide between schedules. The cache key keeps n_sample.
static int plan_tune(smp_plan *plan, int64_t n_sample, int64_t n_grow, smp_tuning *out);

extern "C" int smp_plan_tune(smp_plan *plan, int64_t n_sample, smp_tuning *out) {
    return plan_tune(plan, n_sample, n_sample, out);
}

static int plan_tune(smp_plan *plan, int64_t n_sample, int64_t n_grow, smp_tuning *out) {
    if (!plan || n_sample <= 0) return set_error(SMP_ERR_BAD_ARG, "bad plan / sample size");
    if (plan->kernel != SMP_KERNEL_POOL)
        return set_error(SMP_ERR_UNSUPPORTED, "the tuner chooses the slot pool's parameters (kernel SMP_KERNEL_POOL)");
    SMP_CUDA(cudaSetDevice(plan->device));
    const std::string key = tune_key(plan, n_sample);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            smp_tuning t = it->second;
            t.trials = 0;
            tune_apply(plan, t);
            if (out) *out = t;
            return smp_plan_clear(plan, nullptr);
        }
    }
    // n_inst > 0 (a batched sweep): each instance carries its own weight, the argument is unused
    const int64_t weight = n_sample;
    static const int kSlots[4] = {8, 6, 4, 2};      // largest first: the pool is allocated once
    static const int kChunks[4] = {64, 96, 128, 192};
    smp_tuning best;
    std::memset(&best, 0, sizeof(best));
    best.ms = 1e300;
    int trials = 0;
    double ms = 0.0;
    smp_tuning t;
    std::memset(&t, 0, sizeof(t));
    t.march_block = 128; t.slots_per_lane = kSlots[0]; t.chunk = kChunks[1];
    tune_apply(plan, t);
    // warm-up (allocations, module load) on at most 2e5 photons, which also measures the rate
    const int64_t n_warm = std::min<int64_t>(n_sample, 200000);
    int rc = tune_trial(plan, n_warm, weight, &ms);
    if (rc) return rc;
    if (n_grow > n_sample) {
        // cost per photon from a second warm-up of 8x the photons: ms = fixed + per_photon * n
        const int64_t n2 = std::min<int64_t>(n_grow, 8 * n_warm);
        double ms2 = 0.0;
        rc = tune_trial(plan, n2, weight, &ms2);
        if (rc) return rc;
        const double per = n2 > n_warm ? std::max(ms2 - ms, 1e-3) / double(n2 - n_warm) : ms2 / double(n2);
        n_sample = std::min<int64_t>(n_grow, std::max<int64_t>(n_warm, int64_t(250.0 / per)));
    } else {
        // keep each trial near 400 ms, long enough that the full pool's steady state and not the fill
        // and drain decides: a sample that takes longer is scaled down (not below 1e5 photons)
        const double est = ms * double(n_sample) / double(n_warm);
        if (est > 400.0) n_sample = std::max<int64_t>(std::min<int64_t>(n_sample, 100000), int64_t(double(n_sample) * 400.0 / est));
    }
    smp_tuning second = best;
    auto consider = [&](const smp_tuning &c, double m) {
        if (m < best.ms) { second = best; best = c; best.ms = m; }
        else if (m < second.ms) { second = c; second.ms = m; }
    };
    for (int si = 0; si < 4; ++si)
        for (int ci = 0; ci < 4; ++ci) {
            t.slots_per_lane = kSlots[si];
            t.chunk = kChunks[ci];
            tune_apply(plan, t);
            rc = tune_trial(plan, n_sample, weight, &ms);
            if (rc) return rc;
            ++trials;
            consider(t, ms);
        }
    t = best;
    t.march_block = 256;
    tune_apply(plan, t);
    rc = tune_trial(plan, n_sample, weight, &ms);
    if (rc) return rc;
    ++trials;
    consider(t, ms);
    // the two best once more each, decided on the mean of their two trials
    if (second.march_block) {
        double again[2] = {0.0, 0.0};
        smp_tuning *c2[2] = {&best, &second};
        for (int i = 0; i < 2; ++i) {
            tune_apply(plan, *c2[i]);
            rc = tune_trial(plan, n_sample, weight, &again[i]);
            if (rc) return rc;
            ++trials;
        }
        const double mb = 0.5 * (best.ms + again[0]), m2 = 0.5 * (second.ms + again[1]);
        if (m2 < mb) { best = second; best.ms = m2; }
        else best.ms = mb;
    }
    best.trials = trials;
    best.paths_per_s = double(n_sample) / (best.ms * 1e-3);
    tune_apply(plan, best);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tune_cache[key] = best;
    }
    if (out) *out = best;
    return smp_plan_clear(plan, nullptr);
}

extern "C" {

int smp_render(const smp_scene_desc *scene, const smp_medium_desc *medium, const smp_field_desc *field,
               const smp_render_opts *opts, int64_t n_photons, double *image_out, smp_stats *stats_out) {
    smp_plan *p = nullptr;
    int rc = smp_plan_create(scene, medium, field, opts, &p);
    if (rc) return rc;
    rc = smp_plan_render(p, n_photons, image_out, stats_out);
    std::string err = g_last_error;
    smp_plan_destroy(p);
    g_last_error = err;
    return rc;
}

int smp_trace_photons(const smp_scene_desc *scene, const smp_medium_desc *medium, const smp_field_desc *field,
                      const smp_render_opts *opts, int64_t first_photon, int64_t n_photons, int64_t weight_photons,
                      const float *uniforms, const int64_t *offsets, smp_photon_record *records_out,
                      double *image_out) {
    if (n_photons <= 0 || !records_out) return set_error(SMP_ERR_BAD_ARG, "need n_photons > 0 and records_out");
    if (uniforms && !offsets) return set_error(SMP_ERR_BAD_ARG, "uniforms without offsets");
    smp_render_opts o = *opts;
    if (uniforms) o.rng = SMP_RNG_STREAM;
    else if (o.rng == SMP_RNG_STREAM) return set_error(SMP_ERR_BAD_ARG, "rng STREAM needs uniforms");
    smp_plan *p = nullptr;
    int rc = smp_plan_create(scene, medium, field, &o, &p);
    if (rc) return rc;
    float *d_u = nullptr;
    long long *d_off = nullptr;
    smp_photon_record *d_rec = nullptr;
    cudaError_t e = cudaSuccess;
    if (uniforms) {
        int64_t total = offsets[n_photons];
        e = cudaMalloc(&d_u, size_t(std::max<int64_t>(total, 1)) * sizeof(float));
        if (e == cudaSuccess && total > 0) e = cudaMemcpy(d_u, uniforms, size_t(total) * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMalloc(&d_off, size_t(n_photons + 1) * sizeof(long long));
        if (e == cudaSuccess) e = cudaMemcpy(d_off, offsets, size_t(n_photons + 1) * sizeof(long long), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMalloc(&d_rec, size_t(n_photons) * sizeof(smp_photon_record));
    if (e == cudaSuccess) e = cudaMemset(d_rec, 0, size_t(n_photons) * sizeof(smp_photon_record));
    if (e != cudaSuccess) {
        rc = set_error(SMP_ERR_CUDA, "trace buffers: %s", cudaGetErrorString(e));
    } else {
        rc = launch(p, first_photon, n_photons, weight_photons, 0, d_u, d_off, d_rec);
        int rs = rc ? rc : collect_stats(p);
        if (!rc) {
            e = cudaMemcpy(records_out, d_rec, size_t(n_photons) * sizeof(smp_photon_record), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) rc = set_error(SMP_ERR_CUDA, "records copy: %s", cudaGetErrorString(e));
        }
        if (!rc && image_out) rc = smp_plan_read_image(p, image_out, 0, nullptr);
        if (!rc) rc = rs;
    }
    std::string err = g_last_error;
    cudaFree(d_u);
    cudaFree(d_off);
    cudaFree(d_rec);
    smp_plan_destroy(p);
    g_last_error = err;
    return rc;
}

int smp_field_eval(const smp_field_desc *field, double scaling, int64_t n_points, const double *points,
                   double *n_out, double *grad_out) {
    if (!field || n_points < 0 || (n_points > 0 && (!points || !n_out || !grad_out)))
        return set_error(SMP_ERR_BAD_ARG, "bad arguments");
    int fk;
    int rc = field_kind(*field, &fk);
    if (rc) return rc;
    rc = check_device(0);
    if (rc) return rc;
    if (n_points == 0) return SMP_OK;
    FieldParams F;
    fill_field_params(*field, fk, F);
    float4 *d_cen = nullptr;
    float *d_coeff = nullptr;
    double *d_pts = nullptr, *d_n = nullptr, *d_g = nullptr;
    cudaError_t e = cudaSuccess;
    if (fk == FK_SOURCES) {
        std::vector<float4> c;
        source_centres(*field, c);
        e = cudaMalloc(&d_cen, c.size() * sizeof(float4));
        if (e == cudaSuccess) e = cudaMemcpy(d_cen, c.data(), c.size() * sizeof(float4), cudaMemcpyHostToDevice);
        F.centers = d_cen;
    }
    if (fk == FK_SPLINE && e == cudaSuccess) {
        std::vector<float> delta;
        F.spline_base = spline_offsets(*field, delta);
        e = cudaMalloc(&d_coeff, delta.size() * sizeof(float));
        if (e == cudaSuccess) e = cudaMemcpy(d_coeff, delta.data(), delta.size() * sizeof(float), cudaMemcpyHostToDevice);
        F.coeff = d_coeff;
    }
    float4 *d_tab = nullptr;
    if (fk <= FK_BESSELN && e == cudaSuccess) {
        std::vector<float4> tab;
        bessel_table(field->mode, kBesselMaxX, tab);
        e = cudaMalloc(&d_tab, tab.size() * sizeof(float4));
        if (e == cudaSuccess) e = cudaMemcpy(d_tab, tab.data(), tab.size() * sizeof(float4), cudaMemcpyHostToDevice);
        F.btab = d_tab;
        F.bnodes = int(tab.size());
        F.bint = int(tab.size() / 2);
    }
    size_t np = size_t(n_points);
    if (e == cudaSuccess) e = cudaMalloc(&d_pts, np * 3 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_n, np * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_g, np * 3 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(d_pts, points, np * 3 * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        int blocks = int((np + 255) / 256);
        float s = float(scaling);
        field_probe_fn(fk)<<<blocks, 256>>>(F, s, n_points, d_pts, d_n, d_g);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(n_out, d_n, np * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(grad_out, d_g, np * 3 * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d_cen);
    cudaFree(d_coeff);
    cudaFree(d_tab);
    cudaFree(d_pts);
    cudaFree(d_n);
    cudaFree(d_g);
    if (e != cudaSuccess) return set_error(SMP_ERR_CUDA, "field probe: %s", cudaGetErrorString(e));
    return SMP_OK;
}

// FP32 FMA throughput probe: every thread runs eight independent FMA chains.
__global__ void fp32_peak_kernel(float *out, int iters) {
    float a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = float(threadIdx.x + j) * 1e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = fmaf(a[j], 0.99990f, 1.0e-4f);
    }
    float s = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += a[j];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

int smp_fp32_peak(int device, double *tflops_out) {
    if (!tflops_out) return set_error(SMP_ERR_BAD_ARG, "NULL argument");
    int rc = check_device(device);
    if (rc) return rc;
    int sms = 0;
    SMP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int blocks = sms * 8, threads = 256, iters = 1 << 16;
    float *d = nullptr;
    SMP_CUDA(cudaMalloc(&d, size_t(blocks) * threads * sizeof(float)));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    fp32_peak_kernel<<<blocks, threads>>>(d, 1024);
    cudaEventRecord(a);
    fp32_peak_kernel<<<blocks, threads>>>(d, iters);
    cudaEventRecord(b);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    if (e != cudaSuccess) return set_error(SMP_ERR_CUDA, "fp32 probe: %s", cudaGetErrorString(e));
    *tflops_out = 2.0 * 8.0 * double(iters) * blocks * threads / (double(ms) * 1e-3) / 1e12;
    return SMP_OK;
}

// The batched sweep: every instance's photons are one index range of a single photon stream, so
// the slot pool mixes instances as it refills and the whole sweep has one tail. Each instance's
// field, ER step, medium, weight, seed and film travel with its photons (Inst records); the scene,
// the film shape and the number of refinement levels are shared. Photon j of instance i draws the
// Philox stream (seed_i, j), so each instance's film is the one a single-instance render with that
// seed produces.
//
// A sweep's device state (BatchRun): its plan (field kind FK_BATCH), the instance records, the
// prefix sums of the photon budgets, the Bessel tables and n_inst consecutive films (float, or
// double in the mixed form; film_bytes each). batch_open builds it; batch_set writes the instance
// records and budgets (again for a sweep of the same fields with other steps or budgets, as the
// step tuner's rounds are); batch_trace clears the films and renders.
namespace {
struct BatchRun {
    smp_plan *p = nullptr;
    Inst *d_insts = nullptr;
    long long *d_first = nullptr;
    float4 *d_tabs = nullptr;
    void *d_films = nullptr;
    size_t film_bytes = 0;
    int n_inst = 0;
    long long total = 0;
    std::vector<int> fks;
    size_t tab_off[3] = {0, 0, 0};
    int tab_int[3] = {0, 0, 0};
    smp_scene_desc scene;
    smp_render_opts opts;
    BatchRun() = default;
    BatchRun(const BatchRun &) = delete;
    BatchRun &operator=(const BatchRun &) = delete;
    ~BatchRun() {
        const std::string err = g_last_error;
        cudaFree(d_insts);
        cudaFree(d_first);
        cudaFree(d_tabs);
        cudaFree(d_films);
        if (p) smp_plan_destroy(p);
        g_last_error = err;
    }
};
}  // namespace

static int batch_set(BatchRun &b, const smp_instance_desc *instances);

static int batch_open(const smp_scene_desc *scene, const smp_instance_desc *instances, int32_t n_inst,
                      const smp_render_opts *opts, BatchRun &b) {
    if (!scene || !instances || !opts || n_inst <= 0) return set_error(SMP_ERR_BAD_ARG, "bad batch arguments");
    if (opts->rng != SMP_RNG_PHILOX) return set_error(SMP_ERR_UNSUPPORTED, "a batched sweep draws from Philox");
    b.fks.assign(n_inst, 0);
    for (int i = 0; i < n_inst; ++i) {
        int rc = check_descs(scene, &instances[i].medium, &instances[i].field, opts);
        if (rc) return rc;
        rc = field_kind(instances[i].field, &b.fks[i]);
        if (rc) return rc;
        if (b.fks[i] > FK_BESSEL2)
            return set_error(SMP_ERR_UNSUPPORTED, "instance %d: a batched sweep renders Bessel fields of order 0-2", i);
        if (instances[i].n_photons < 0) return set_error(SMP_ERR_BAD_ARG, "instance %d: negative photon budget", i);
        if (instances[i].field.precision != instances[0].field.precision)
            return set_error(SMP_ERR_BAD_ARG, "instance %d: a batched sweep shares one number of refinement levels "
                             "(%d, instance 0 has %d)", i, instances[i].field.precision, instances[0].field.precision);
    }
    b.n_inst = n_inst;
    b.scene = *scene;
    b.opts = *opts;
    int rc = smp_plan_create(scene, &instances[0].medium, &instances[0].field, opts, &b.p);
    if (rc) return rc;
    smp_plan *p = b.p;
    const size_t px = p->film_elems, bpp = p->kp.fp64 ? 8 : 4;
    b.film_bytes = px * bpp;
    // the tables depend on the order and the largest k r only: one per order, as long as the
    // largest k r any instance of that order meets
    double xmax[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < n_inst; ++i) {
        FieldParams F;
        fill_field_params(instances[i].field, b.fks[i], F);
        xmax[b.fks[i]] = std::max(xmax[b.fks[i]], box_max_kr(*scene, F.k_r));
    }
    std::vector<float4> tabs;
    for (int m = 0; m < 3; ++m) {
        if (xmax[m] <= 0.0) continue;
        std::vector<float4> t;
        bessel_table(m, xmax[m], t);
        b.tab_off[m] = tabs.size();
        b.tab_int[m] = int(t.size() / 2);
        tabs.insert(tabs.end(), t.begin(), t.end());
    }
    cudaError_t e = cudaMalloc(&b.d_insts, sizeof(Inst) * size_t(n_inst));
    if (e == cudaSuccess) e = cudaMalloc(&b.d_first, sizeof(long long) * size_t(n_inst + 1));
    if (e == cudaSuccess) e = cudaMalloc(&b.d_tabs, sizeof(float4) * tabs.size());
    if (e == cudaSuccess) e = cudaMalloc(&b.d_films, b.film_bytes * size_t(n_inst));
    if (e == cudaSuccess) e = cudaMemcpy(b.d_tabs, tabs.data(), sizeof(float4) * tabs.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess)
        return set_error(e == cudaErrorMemoryAllocation ? SMP_ERR_OOM : SMP_ERR_CUDA, "batch buffers: %s", cudaGetErrorString(e));
    p->kp.insts = b.d_insts;
    p->kp.inst_first = b.d_first;
    p->kp.n_inst = n_inst;
    p->fk = FK_BATCH;
    p->smem_bytes = 0;
    rc = grid_for(FK_BATCH, p->device, p->opts.blocks_per_sm, 0, &p->grid);
    if (rc) return rc;
    const char *graph_env = std::getenv("SMP_WF_GRAPH");
    p->use_graph = !(graph_env && std::atoi(graph_env) == 0);
    return batch_set(b, instances);
}

// Instance records and budgets of a sweep whose fields (orders, largest k r) are those it was opened
// with; steps, media, seeds and budgets may differ.
static int batch_set(BatchRun &b, const smp_instance_desc *instances) {
    std::vector<Inst> hi(b.n_inst);
    std::vector<long long> first(size_t(b.n_inst) + 1, 0);
    const size_t px = b.p->film_elems, bpp = b.p->kp.fp64 ? 8 : 4;
    for (int i = 0; i < b.n_inst; ++i) {
        const smp_instance_desc &d = instances[i];
        Inst &I = hi[i];
        std::memset(&I, 0, sizeof(I));
        const int fk = b.fks[i];
        fill_field_params(d.field, fk, I.field);
        I.field.bnodes = 2 * b.tab_int[fk];
        I.field.bint = b.tab_int[fk];
        I.field.btab = b.d_tabs + b.tab_off[fk];
        I.film = static_cast<char *>(b.d_films) + px * bpp * size_t(i);
        I.sigma_t = float(d.medium.sigma_t);                      // medium.h:24-38
        I.albedo = float(d.medium.albedo);
        I.mfp = 1.0f / float(d.medium.sigma_t);
        if (I.sigma_t <= 1.19209290e-07f) { I.sigma_t = 0.0f; I.mfp = 1.0f; I.albedo = 0.0f; }
        I.g = float(d.medium.g);
        I.weight = d.n_photons > 0 ? photon_weight(b.scene, d.n_photons) : 0.0f;
        I.large_dist = sensor_march_budget(b.opts, I.sigma_t);
        I.seed = d.seed;
        I.h0 = float(d.field.er_stepsize);                      // each instance marches with its own step
        step_table(d.field.er_stepsize, I.cur_tab);
        first[i + 1] = first[i] + d.n_photons;
    }
    b.total = first[b.n_inst];
    cudaError_t e = cudaMemcpy(b.d_insts, hi.data(), sizeof(Inst) * size_t(b.n_inst), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b.d_first, first.data(), sizeof(long long) * size_t(b.n_inst + 1), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_error(SMP_ERR_CUDA, "batch records: %s", cudaGetErrorString(e));
    return SMP_OK;
}

// Clears the films and renders every instance's budget. schedule_tune: run the slot pool's autotuner
// first (trials on the sweep's own photons, cached per process).
static int batch_trace(BatchRun &b, bool schedule_tune, smp_stats *stats_out) {
    smp_plan *p = b.p;
    int rc = SMP_OK;
    const char *tune_env = std::getenv("SMP_TUNE");
    if (schedule_tune && b.total > 0 && p->kernel == SMP_KERNEL_POOL && !(tune_env && std::atoi(tune_env) == 0)) {
        smp_tuning tt;
        rc = plan_tune(p, std::min<long long>(b.total, 2000000LL), b.total, &tt);
        if (rc) return rc;
    }
    cudaError_t e = cudaMemset(b.d_films, 0, b.film_bytes * size_t(b.n_inst));
    if (e != cudaSuccess) return set_error(SMP_ERR_CUDA, "batch films: %s", cudaGetErrorString(e));
    rc = smp_plan_clear(p, nullptr);
    // the weight argument is unused: each instance carries its own Li T / N
    if (!rc && b.total > 0) rc = launch(p, 0, b.total, 1, nullptr, nullptr, nullptr, nullptr);
    const int rs = rc ? rc : collect_stats(p);
    if (stats_out) *stats_out = p->stats;
    return rc ? rc : rs;
}

int smp_render_batch(const smp_scene_desc *scene, const smp_instance_desc *instances, int32_t n_inst,
                     const smp_render_opts *opts, double *images_out, smp_stats *stats_out) {
    BatchRun b;
    int rc = batch_open(scene, instances, n_inst, opts, b);
    if (!rc) rc = batch_trace(b, true, stats_out);
    if (rc) return rc;
    const size_t fb = b.film_bytes;
    const void *d_films = b.d_films;
    if (images_out) {
        // The films reach host memory that is usually fresh (a new array per call): its pages are
        // first written on several threads, so that the copy, whose page faults one thread would
        // take, finds them mapped.
        cudaError_t e;
        if (opts->precision == SMP_PREC_MIXED) {
            const size_t cnt = fb / 8 * size_t(n_inst);
            host_parallel(cnt, [images_out](size_t a, size_t b) { std::memset(images_out + a, 0, (b - a) * 8); });
            e = cudaMemcpy(images_out, d_films, cnt * 8, cudaMemcpyDeviceToHost);
        } else {
            // FP32 films through a staging buffer, widened on the host by several threads
            const size_t cnt = fb / 4 * size_t(n_inst);
            std::unique_ptr<float[]> h(new float[cnt]);
            float *hp = h.get();
            host_parallel(cnt, [hp](size_t a, size_t b) { std::memset(hp + a, 0, (b - a) * 4); });
            e = cudaMemcpy(hp, d_films, cnt * 4, cudaMemcpyDeviceToHost);
            if (e == cudaSuccess)
                host_parallel(cnt, [hp, images_out](size_t a, size_t b) {
                    for (size_t j = a; j < b; ++j) images_out[j] = double(hp[j]);
                });
        }
        if (e != cudaSuccess) rc = set_error(SMP_ERR_CUDA, "batch films: %s", cudaGetErrorString(e));
    }
    return rc;
}

// Per instance i (blockIdx.y): sum (a - r)^2 and sum r^2 over its film of px pixels (each film float,
// or double when its flag is set), accumulated in double into acc[2i], acc[2i + 1].
__global__ void film_diff_kernel(const void *a, int a64, const void *r, int r64, size_t px, double *acc) {
    __shared__ double sd[32], sr[32];
    const size_t base = size_t(blockIdx.y) * px;
    double d2 = 0.0, r2 = 0.0;
    for (size_t j = size_t(blockIdx.x) * blockDim.x + threadIdx.x; j < px; j += size_t(gridDim.x) * blockDim.x) {
        const double av = a64 ? static_cast<const double *>(a)[base + j] : double(static_cast<const float *>(a)[base + j]);
        const double rv = r64 ? static_cast<const double *>(r)[base + j] : double(static_cast<const float *>(r)[base + j]);
        d2 += (av - rv) * (av - rv);
        r2 += rv * rv;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        d2 += __shfl_down_sync(0xffffffffu, d2, o);
        r2 += __shfl_down_sync(0xffffffffu, r2, o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { sd[w] = d2; sr[w] = r2; }
    __syncthreads();
    if (w == 0) {
        d2 = lane < int(blockDim.x >> 5) ? sd[lane] : 0.0;
        r2 = lane < int(blockDim.x >> 5) ? sr[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            d2 += __shfl_down_sync(0xffffffffu, d2, o);
            r2 += __shfl_down_sync(0xffffffffu, r2, o);
        }
        if (lane == 0) {
            atomicAdd(acc + 2 * blockIdx.y, d2);
            atomicAdd(acc + 2 * blockIdx.y + 1, r2);
        }
    }
}

// Step-size autotuner of a batched sweep. Photons [0, min(n_photons_i, n_sample)) of every
// instance are rendered at the instance's own er_stepsize (its reference film), and then at
// multiples of it from kStepMults, at most an eighth of the instance's ultrasound wavelength: first
// the largest allowed one, and, when that misses the budget, by bisection between the largest
// multiple known to pass and the smallest known to miss (the error grows with the step). Every
// round is one batched render of the instances still searching; an instance keeps the largest
// multiple whose film stayed within rmse_budget relative RMSE of its reference film on the same
// photons, or its own step when its reference film is empty. The search holds two films per
// instance (reference and trial), so instances are tuned in groups whose films fit in 40 % of the
// free device memory.
namespace {
const int kStepMults[] = {2, 3, 4, 6, 8, 12, 16, 24, 32};
const int kNumStepMults = int(sizeof(kStepMults) / sizeof(kStepMults[0]));

// the search over instances [0, n) of `inst`; pass/rmse per instance out; *rounds accumulates
int tune_steps_group(const smp_scene_desc *scene, const smp_instance_desc *inst, int n, const smp_render_opts *opts,
                     int64_t n_sample, double rmse_budget, int *pass, double *rmse, int *rounds) {
    std::vector<smp_instance_desc> trial(inst, inst + n);
    // The trial renders stop a sensor march at 30 mean free paths of the thinnest medium (unless the
    // caller set a budget): the reference and trial films are cut alike, a cut photon's remaining
    // contribution is below e^-30 of its weight, and the photons trapped by total internal
    // reflection, which set every round's tail, stop sooner than at the default 110.
    smp_render_opts topts = *opts;
    if (!(topts.sensor_march_max > 0.0)) {
        double st_min = HUGE_VAL;
        for (int i = 0; i < n; ++i) st_min = std::min(st_min, inst[i].medium.sigma_t);
        if (st_min > 1e-3) topts.sensor_march_max = 30.0 / st_min;
    }
    opts = &topts;
    // per instance: the allowed multiples are kStepMults[0 .. lim); index pass[i] passes (-1: the
    // instance's own step), index miss[i] misses (lim: none known), tr[i] is this round's
    std::vector<int> miss(n, 0), tr(n, -1);
    for (int i = 0; i < n; ++i) {
        const smp_field_desc &f = inst[i].field;
        const double lambda = f.speed_u / f.f_u;
        int lim = 0;
        while (lim < kNumStepMults && f.er_stepsize * kStepMults[lim] <= lambda / 8.0) ++lim;
        pass[i] = -1;
        rmse[i] = 0.0;
        miss[i] = inst[i].n_photons > 0 ? lim : 0;                 // nothing to search without photons
        trial[i].n_photons = std::min<int64_t>(inst[i].n_photons, n_sample);
    }
    // Every render of the search is in the mixed form (FP64 path length and film), whatever the
    // sweep's own form. In the FP32 form the path length is accumulated in float and a different
    // number of steps rounds it differently, which moves photons near a path-length bin edge to the
    // next bin -- at any step, the own one included, and for a few large splats (connections in the
    // Henyey-Greenstein peak) by more than the budget. In the mixed form the films differ by the
    // step's own effect on the march, which is what the step decides; the FP32 render then carries
    // the same kind of float rounding at the chosen step as at its own.
    topts.precision = SMP_PREC_MIXED;
    BatchRun b;
    int rc = batch_open(scene, trial.data(), n, opts, b);
    if (!rc) rc = batch_trace(b, false, nullptr);
    ++*rounds;
    void *d_ref = nullptr;
    double *d_acc = nullptr;
    const size_t px = b.film_bytes / 8;
    std::vector<double> acc(2 * size_t(n));
    if (!rc) {
        cudaError_t e = cudaMalloc(&d_ref, b.film_bytes * size_t(n));
        if (e == cudaSuccess) e = cudaMalloc(&d_acc, acc.size() * sizeof(double));
        if (e == cudaSuccess) e = cudaMemcpy(d_ref, b.d_films, b.film_bytes * size_t(n), cudaMemcpyDeviceToDevice);
        if (e != cudaSuccess)
            rc = set_error(e == cudaErrorMemoryAllocation ? SMP_ERR_OOM : SMP_ERR_CUDA, "tuner buffers: %s", cudaGetErrorString(e));
    }
    for (bool first = true; !rc; first = false) {
        bool any = false;
        for (int i = 0; i < n; ++i) {
            tr[i] = -1;
            if (miss[i] - pass[i] > 1) tr[i] = first ? miss[i] - 1 : (pass[i] + miss[i]) / 2;
            trial[i].field.er_stepsize = inst[i].field.er_stepsize * (tr[i] >= 0 ? kStepMults[tr[i]] : 1);
            trial[i].n_photons = tr[i] >= 0 ? std::min<int64_t>(inst[i].n_photons, n_sample) : 0;
            any = any || tr[i] >= 0;
        }
        if (!any) break;
        rc = batch_set(b, trial.data());
        if (!rc) rc = batch_trace(b, false, nullptr);
        ++*rounds;
        if (rc) break;
        cudaError_t e = cudaMemset(d_acc, 0, acc.size() * sizeof(double));
        if (e == cudaSuccess) {
            film_diff_kernel<<<dim3(64, unsigned(n)), 256>>>(b.d_films, 1, d_ref, 1, px, d_acc);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpy(acc.data(), d_acc, acc.size() * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { rc = set_error(SMP_ERR_CUDA, "tuner films: %s", cudaGetErrorString(e)); break; }
        for (int i = 0; i < n; ++i) {
            if (tr[i] < 0) continue;
            if (!(acc[2 * i + 1] > 0.0)) { miss[i] = pass[i] + 1; continue; }   // empty reference film: keep its step
            const double r = std::sqrt(acc[2 * i] / acc[2 * i + 1]);
            if (r <= rmse_budget) { pass[i] = tr[i]; rmse[i] = r; }
            else miss[i] = tr[i];
        }
    }
    std::string err = g_last_error;
    cudaFree(d_ref);
    cudaFree(d_acc);
    g_last_error = err;
    return rc;
}
}  // namespace

int smp_batch_tune_steps(const smp_scene_desc *scene, const smp_instance_desc *instances, int32_t n_inst,
                         const smp_render_opts *opts, int64_t n_sample, double rmse_budget, double *steps_out,
                         double *rmse_out, int32_t *rounds_out) {
    if (!scene || !instances || !opts || n_inst <= 0 || !steps_out) return set_error(SMP_ERR_BAD_ARG, "bad batch arguments");
    if (n_sample <= 0) return set_error(SMP_ERR_BAD_ARG, "n_sample must be positive");
    if (!(rmse_budget > 0.0)) return set_error(SMP_ERR_BAD_ARG, "rmse_budget must be positive");
    int rc = check_device(opts->device);
    if (rc) return rc;
    // instances per group: within 40 % of the free memory, 16 bytes per pixel each (the FP64
    // reference film and an FP64 trial film), at most 65535 (the difference kernel's grid height)
    size_t free_b = 0, total_b = 0;
    SMP_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t film = size_t(scene->x_res) * size_t(scene->y_res) * size_t(scene->z_res) * 16;
    const size_t fit = film ? size_t(double(free_b) * 0.4) / film : size_t(n_inst);
    if (fit == 0) return set_error(SMP_ERR_OOM, "the step tuner needs %zu bytes per instance; %zu bytes are free", film, free_b);
    const int group = int(std::min<size_t>({size_t(n_inst), fit, size_t(65535)}));
    std::vector<int> pass(n_inst, -1);
    std::vector<double> rmse(n_inst, 0.0);
    int rounds = 0;
    for (int g0 = 0; g0 < n_inst && !rc; g0 += group) {
        const int gn = std::min(group, n_inst - g0);
        rc = tune_steps_group(scene, instances + g0, gn, opts, n_sample, rmse_budget, pass.data() + g0,
                              rmse.data() + g0, &rounds);
    }
    if (rc) return rc;
    // A film of n_sample photons can be led by a few large splats (connections in the
    // Henyey-Greenstein peak), and any change of step moves some of them: then every multiple misses
    // by about the same amount, which the step does not cause and more photons average out. The
    // instances that kept their own step although they have more photons search once more with ten
    // times the sample.
    std::vector<int> again;
    for (int i = 0; i < n_inst; ++i) {
        const smp_field_desc &f = instances[i].field;
        const bool allowed = f.er_stepsize * kStepMults[0] <= f.speed_u / f.f_u / 8.0;   // any multiple at all
        if (pass[i] < 0 && allowed && instances[i].n_photons > n_sample) again.push_back(i);
    }
    if (!again.empty()) {
        std::vector<smp_instance_desc> sub(again.size());
        for (size_t j = 0; j < again.size(); ++j) sub[j] = instances[again[j]];
        std::vector<int> pass2(sub.size(), -1);
        std::vector<double> rmse2(sub.size(), 0.0);
        const int64_t n2 = n_sample * 10;
        for (int g0 = 0; g0 < int(sub.size()) && !rc; g0 += group) {
            const int gn = std::min(group, int(sub.size()) - g0);
            rc = tune_steps_group(scene, sub.data() + g0, gn, opts, n2, rmse_budget, pass2.data() + g0,
                                  rmse2.data() + g0, &rounds);
        }
        if (rc) return rc;
        for (size_t j = 0; j < again.size(); ++j) { pass[again[j]] = pass2[j]; rmse[again[j]] = rmse2[j]; }
    }
    for (int i = 0; i < n_inst; ++i) {
        steps_out[i] = instances[i].field.er_stepsize * (pass[i] >= 0 ? kStepMults[pass[i]] : 1);
        if (rmse_out) rmse_out[i] = rmse[i];
    }
    if (rounds_out) *rounds_out = rounds;
    return SMP_OK;
}

// Step-size autotuner of a plan: the batched tuner's search (multiples from kStepMults, the largest
// allowed first, then bisection) on photons [0, n_sample) of the plan's own render, against the
// film at the plan's own step on the same photons. The cap on the step is the field's shortest
// length scale: an eighth of the shortest wavelength of a Bessel, point-source (its highest
// harmonic) or plane-wave field, a quarter of a spline grid's finest spacing.
static double field_step_cap(const smp_plan *p) {
    const FieldParams &F = p->kp.field;
    const double two_pi = 6.283185307179586;
    switch (p->fk) {
        case FK_PLANEWAVE: {
            double kmax = 0.0;
            for (int i = 0; i < F.n_waves; ++i)
                kmax = std::max(kmax, std::sqrt(double(F.wk[i][0]) * F.wk[i][0] + double(F.wk[i][1]) * F.wk[i][1] +
                                                double(F.wk[i][2]) * F.wk[i][2]));
            return kmax > 0.0 ? two_pi / kmax / 8.0 : HUGE_VAL;
        }
        case FK_SPLINE: {
            double res = 0.0;
            for (int a = 0; a < 3; ++a) res = std::max(res, double(F.xres[a]));
            return res > 0.0 ? 0.25 / res : HUGE_VAL;
        }
        case FK_SOURCES:
            return F.k_r > 0.0f ? two_pi / (double(F.k_r) * std::max(1, F.n_coeff)) / 8.0 : HUGE_VAL;
        default:                                                   // Bessel, any order
            return F.k_r > 0.0f ? two_pi / double(F.k_r) / 8.0 : HUGE_VAL;
    }
}

static void plan_set_step(smp_plan *p, double h) {
    p->kp.h0 = float(h);
    step_table(h, p->kp.cur_tab);
}

extern "C" int smp_plan_tune_step(smp_plan *plan, int64_t n_sample, double rmse_budget, double *step_out,
                                  double *rmse_out) {
    if (!plan || !step_out) return set_error(SMP_ERR_BAD_ARG, "NULL argument");
    if (n_sample <= 0) return set_error(SMP_ERR_BAD_ARG, "n_sample must be positive");
    if (!(rmse_budget > 0.0)) return set_error(SMP_ERR_BAD_ARG, "rmse_budget must be positive");
    if (plan->kp.n_inst) return set_error(SMP_ERR_UNSUPPORTED, "a batched sweep tunes its steps with smp_batch_tune_steps");
    SMP_CUDA(cudaSetDevice(plan->device));
    // multiples of the field's own step (a plan tuned before starts again from it)
    const double h0 = double(float(plan->field.er_stepsize)), cap = field_step_cap(plan);
    plan_set_step(plan, h0);
    int lim = 0;
    while (lim < kNumStepMults && h0 * kStepMults[lim] <= cap) ++lim;
    // The trial renders stop a sensor march at 30 mean free paths (as the batched tuner's do): the
    // reference and trial films are cut alike and the rounds' tails are shorter.
    const float large0 = plan->kp.large_dist;
    if (plan->opts.sensor_march_max <= 0.0 && plan->kp.sigma_t > 1e-3f)
        plan->kp.large_dist = std::min(large0, 30.0f / plan->kp.sigma_t);
    // The search renders in the mixed form (FP64 path length and film), as smp_batch_tune_steps'
    // does: a plan of the FP32 form whose field is held by value searches on a mixed-form twin and
    // takes the chosen step back. (A spline's coefficients are the caller's host memory, so an FP32
    // spline plan searches in its own form, where the float path length's rounding, different at
    // every step, counts against the budget too.)
    const bool twin = plan->kp.fp64 == 0 && plan->field.type != SMP_FIELD_SPLINE;
    smp_plan *q = plan;                                        // the plan the search renders with
    int rc = SMP_OK;
    if (twin) {
        smp_render_opts ro = plan->opts;
        ro.precision = SMP_PREC_MIXED;
        if (ro.sensor_march_max <= 0.0 && plan->kp.sigma_t > 1e-3f) ro.sensor_march_max = 30.0 / double(plan->kp.sigma_t);
        q = nullptr;
        rc = smp_plan_create(&plan->scene, &plan->medium, &plan->field, &ro, &q);
    }
    const size_t px = plan->film_elems;
    const int q64 = q ? q->kp.fp64 : 0;
    const size_t fb = px * (q64 ? 8 : 4);
    void *d_ref = nullptr;
    double *d_acc = nullptr;
    cudaError_t e = cudaSuccess;
    if (!rc) {
        e = cudaMalloc(&d_acc, 2 * sizeof(double));
        if (e == cudaSuccess) e = cudaMalloc(&d_ref, fb);
        if (e != cudaSuccess) rc = set_error(SMP_ERR_OOM, "tuner buffers: %s", cudaGetErrorString(e));
    }
    // the reference film: the own step
    if (!rc) rc = smp_plan_clear(q, nullptr);
    if (!rc) rc = smp_plan_trace(q, 0, n_sample, n_sample, nullptr);
    if (!rc) {
        e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaMemcpy(d_ref, q->d_film, fb, cudaMemcpyDeviceToDevice);
        if (e != cudaSuccess) rc = set_error(SMP_ERR_CUDA, "tuner films: %s", cudaGetErrorString(e));
    }
    int pass = -1, miss = lim;
    double best_rmse = 0.0;
    for (bool first = true; !rc && miss - pass > 1; first = false) {
        const int t = first ? miss - 1 : (pass + miss) / 2;
        plan_set_step(q, h0 * kStepMults[t]);
        rc = smp_plan_clear(q, nullptr);
        if (!rc) rc = smp_plan_trace(q, 0, n_sample, n_sample, nullptr);
        if (rc) break;
        double acc[2] = {0.0, 0.0};
        e = cudaMemset(d_acc, 0, sizeof(acc));
        if (e == cudaSuccess) {
            film_diff_kernel<<<dim3(148, 1), 256>>>(q->d_film, q64, d_ref, q64, px, d_acc);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpy(acc, d_acc, sizeof(acc), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { rc = set_error(SMP_ERR_CUDA, "tuner films: %s", cudaGetErrorString(e)); break; }
        if (!(acc[1] > 0.0)) break;                            // empty reference film: keep the step
        const double r = std::sqrt(acc[0] / acc[1]);
        if (r <= rmse_budget) { pass = t; best_rmse = r; }
        else miss = t;
    }
    if (twin && q) {
        const std::string err = g_last_error;
        smp_plan_destroy(q);
        g_last_error = err;
        e = cudaSetDevice(plan->device);
        if (!rc && e != cudaSuccess) rc = set_error(SMP_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    }
    std::string err = g_last_error;
    cudaFree(d_ref);
    cudaFree(d_acc);
    g_last_error = err;
    plan->kp.large_dist = large0;
    plan_set_step(plan, pass >= 0 ? h0 * kStepMults[pass] : h0);
    const int rc2 = smp_plan_clear(plan, nullptr);
    if (rc) return rc;
    if (rc2) return rc2;
    *step_out = double(plan->kp.h0);
    if (rmse_out) *rmse_out = best_rmse;
    return SMP_OK;
}

// ---- adjoint ------------------------------------------------------------------------------------
int64_t smp_adjoint_param_count(const smp_field_desc *f) {
    if (!f) return set_error(SMP_ERR_BAD_ARG, "NULL field");
    if (f->type == SMP_FIELD_PLANEWAVE) {
        if (f->n_waves < 1 || f->n_waves > SMP_MAX_WAVES) return set_error(SMP_ERR_BAD_ARG, "n_waves %d", f->n_waves);
        return 2 * int64_t(f->n_waves);
    }
    if (f->type == SMP_FIELD_SPLINE) {
        if (f->grid_n[0] < 2 || f->grid_n[1] < 2 || f->grid_n[2] < 2) return set_error(SMP_ERR_BAD_ARG, "bad spline grid");
        return int64_t(f->grid_n[0]) * f->grid_n[1] * f->grid_n[2];
    }
    if (f->type == SMP_FIELD_BESSEL) {
        if (f->mode < 0 || f->mode > 2) return set_error(SMP_ERR_UNSUPPORTED, "the Bessel adjoint is built for modes 0-2");
        return 3;
    }
    return set_error(SMP_ERR_UNSUPPORTED, "the adjoint is built for Bessel (modes 0-2), plane-wave and spline fields");
}

static int env_int(const char *name, int def, int lo, int hi) {
    const char *v = std::getenv(name);
    if (!v) return def;
    return std::max(lo, std::min(hi, std::atoi(v)));
}

static int grid_of(const void *fn, int dev) {
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, 0) != cudaSuccess) return 0;
    return sms * std::max(per_sm, 1);
}

// The adjoint's checkpointing trace on the slot pool: the render's march kernel (no hook: the
// accepted ER steps of a march follow from its step count and refinement level) alternating with
// the checkpointing event kernel, whose per-slot state (checkpoints, flags, trajectory entries)
// stays in AdjParams.tverts/tstate between launches; the live slots' tail runs on the persistent
// lane loop once they fit in one grid. Spline plans march without coefficient bricks here.
static cudaError_t adjoint_trace_pool(smp_plan *p, const KParams &k, const AdjParams &a, AdjWaveFn fe, AdjWaveFn ff,
                                      int grid_f, long long *launches) {
    WaveParams W = p->wp;
    W.nb = 0;
    WaveFn fm = wf_march_fn(p->fk, p->kp.fp64 != 0, p->march_block, false);
    if (!fm) return cudaErrorInvalidDeviceFunction;
    if (p->smem_bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void *>(fm), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(p->smem_bytes));
        if (e != cudaSuccess) return e;
    }
    const unsigned finish_at = unsigned(grid_f) * unsigned(kBlock);
    const long long max_iter = (long long)k.step_cap * 4 + (1LL << 20);
    cudaError_t e = cudaMemsetAsync(W.cnt, 0, 8 * sizeof(unsigned), 0);
    if (e != cudaSuccess) return e;
    fe<<<p->grid_event, kBlock>>>(k, W, a, -1);
    *launches += 1;
    long long it = 0;
    bool pending = false;
    int par = 0;
    for (;;) {
        for (int j = 0; j < p->wave_batch; ++j, ++it) {
            fm<<<p->grid_march, p->march_block, p->smem_bytes>>>(k, W, int(it & 0x3fffffff));
            fe<<<p->grid_event, kBlock>>>(k, W, a, int(it & 0x3fffffff));
        }
        *launches += 2 * p->wave_batch;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (pending) {                              // the previous batch's live count
            const int q = par ^ 1;
            if ((e = cudaEventSynchronize(p->live_ev[q])) != cudaSuccess) return e;
            const unsigned long long live = live_of(p->h_live[2 * q]);
            if (live == 0u) break;
            if (live <= finish_at && live < (unsigned long long)W.n_slots) {
                ff<<<grid_f, kBlock>>>(k, W, a, int(it & 0x3fffffff));
                *launches += 1;
                return cudaGetLastError();
            }
        }
        p->h_live[2 * par] = 0;
        if ((e = cudaMemcpyAsync(p->h_live + 2 * par, W.cnt + 2 * (it & 1), 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, 0)) !=
            cudaSuccess)
            return e;
        if ((e = cudaEventRecord(p->live_ev[par], 0)) != cudaSuccess) return e;
        pending = true;
        par ^= 1;
        if (it > max_iter) return cudaErrorLaunchFailure;
    }
    return cudaSuccess;
}

// Photons are differentiated in batches. Per batch: the checkpointing trace (one checkpoint per
// scatter vertex into the batch pool), then rounds of replay (every segment the sweep needs,
// written to the trajectory buffer, as many photons as fit) and sweep (the backward pass over
// them). Buffers, one allocation kept in the plan: dJ/dfilm, gradient, counters; per trace thread
// vcap checkpoints; the pool (batch x pool_per_photon checkpoints), two segment records per
// checkpoint, one AdjPhoton per photon of the batch; the trajectory buffer.
int smp_plan_adjoint(smp_plan *plan, int64_t first_photon, int64_t n_photons, int64_t weight_photons,
                     const double *dJ_dfilm, double *grad_out, smp_adjoint_stats *stats_out) {
    if (!plan || !dJ_dfilm || !grad_out || n_photons < 0 || first_photon < 0)
        return set_error(SMP_ERR_BAD_ARG, "bad adjoint arguments");
    if (weight_photons <= 0) return set_error(SMP_ERR_BAD_ARG, "weight_photons must be positive");
    const int64_t np = smp_adjoint_param_count(&plan->field);
    if (np < 0) return int(np);
    AdjFn fa = adjoint_trace_fn(plan->fk);
    AdjWaveFn fte = adjoint_trace_event_fn(plan->fk), ftf = adjoint_trace_finish_fn(plan->fk);
    AdjRoundFn fr = adjoint_replay_fn(plan->fk), fs = adjoint_sweep_fn(plan->fk, plan->kp.field.n_waves);
    if (!fa || !fte || !ftf || !fr || !fs) return set_error(SMP_ERR_UNSUPPORTED, "no adjoint for field kind %d", plan->fk);
    if (plan->kp.rng != SMP_RNG_PHILOX) return set_error(SMP_ERR_UNSUPPORTED, "the adjoint replays Philox streams only");
    if (plan->kp.src_lens_active || plan->kp.cam_lens_active)
        return set_error(SMP_ERR_UNSUPPORTED, "the adjoint is built for scenes without lenses");
    SMP_CUDA(cudaSetDevice(plan->device));
    // the trace runs on the slot pool (march kernel + a checkpointing event kernel), or, with
    // SMP_ADJ_TRACE=lanes, as one persistent lane-loop launch
    const char *trace_env = std::getenv("SMP_ADJ_TRACE");
    const bool trace_lanes = trace_env && std::strcmp(trace_env, "lanes") == 0;
    int rc0 = wave_setup(plan);
    if (rc0) return rc0;
    const int grid_a = grid_of(reinterpret_cast<const void *>(fa), plan->device);
    const int grid_tf = grid_of(reinterpret_cast<const void *>(ftf), plan->device);
    const int grid_r = grid_of(reinterpret_cast<const void *>(fr), plan->device);
    const int grid_s = grid_of(reinterpret_cast<const void *>(fs), plan->device);
    if (!grid_a || !grid_tf || !grid_r || !grid_s) return set_error(SMP_ERR_CUDA, "adjoint occupancy query failed");
    const size_t trace_threads = trace_lanes ? size_t(grid_a) * kBlock : size_t(plan->wp.n_slots);
    AdjParams a;
    std::memset(&a, 0, sizeof(a));
    a.X = plan->kp.X; a.Y = plan->kp.Y; a.Z = plan->kp.Z;
    a.vcap = env_int("SMP_ADJ_VCAP", 256, 2, 1 << 20);
    a.idle_replay = env_int("SMP_ADJ_IDLE_REPLAY", 16, 1, 32);   // half of the live lanes
    a.idle_sweep = env_int("SMP_ADJ_IDLE_SWEEP", 4, 1, 32);     // an eighth
    if (!plan->adj_batch) {
        // from the memory free before the first adjoint, so that later calls keep the same sizes
        size_t fr = 0, tot = 0;
        SMP_CUDA(cudaMemGetInfo(&fr, &tot));
        const long long gib = 1LL << 30;
        plan->adj_batch = env_int("SMP_ADJ_BATCH", (long long)fr >= 64 * gib ? 1 << 22 : 1 << 21, 1024, 1 << 30);
        plan->adj_traj_mb = env_int("SMP_ADJ_TRAJ_MB", int(std::min<long long>(40960, std::max<long long>(1024, (long long)(fr / 4) >> 20))),
                                    16, 1 << 20);
    }
    const long long batch = plan->adj_batch;
    const long long per_photon = env_int("SMP_ADJ_POOL_PER_PHOTON", 16, 1, 4096);
    a.pool_cap = batch * per_photon;
    a.traj_cap = plan->adj_traj_mb * (1LL << 20) / (long long)sizeof(float4);
    const size_t film = size_t(a.X) * a.Y * a.Z;
    const int ncnt = ADJ_COUNT + CNT_COUNT + 4;          // + pool_next, traj_next, pending, n_order
    auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t bG = up(film * sizeof(double)), bgrad = up(size_t(np) * sizeof(double));
    const size_t bcnt = up(ncnt * sizeof(unsigned long long));
    const size_t btv = up(size_t(a.vcap) * trace_threads * sizeof(AdjVertex)) + up(trace_threads * sizeof(int4));
    const size_t bpool = up(size_t(a.pool_cap) * sizeof(AdjVertex));
    const size_t bsegs = up(2 * size_t(a.pool_cap) * sizeof(AdjSeg));
    const size_t bph = up(size_t(batch) * sizeof(AdjPhoton)) + up(size_t(batch) * sizeof(int)) + up(1024 * sizeof(unsigned));
    const size_t btraj = size_t(a.traj_cap) * sizeof(float4);
    const size_t need = bG + bgrad + bcnt + btv + bpool + bsegs + bph + btraj;
    if (plan->adj_bytes < need) {
        cudaFree(plan->adj_buf);
        plan->adj_buf = nullptr;
        plan->adj_bytes = 0;
        cudaError_t ea = cudaMalloc(&plan->adj_buf, need);
        if (ea != cudaSuccess)
            return set_error(ea == cudaErrorMemoryAllocation ? SMP_ERR_OOM : SMP_ERR_CUDA, "adjoint buffers (%zu bytes): %s",
                             need, cudaGetErrorString(ea));
        plan->adj_bytes = need;
    }
    char *base = static_cast<char *>(plan->adj_buf);
    double *d_G = reinterpret_cast<double *>(base); base += bG;
    double *d_grad = reinterpret_cast<double *>(base); base += bgrad;
    unsigned long long *d_cnt = reinterpret_cast<unsigned long long *>(base); base += bcnt;
    a.tverts = reinterpret_cast<AdjVertex *>(base);
    a.tstate = reinterpret_cast<int4 *>(base + up(size_t(a.vcap) * trace_threads * sizeof(AdjVertex)));
    base += btv;
    a.pool = reinterpret_cast<AdjVertex *>(base); base += bpool;
    a.segs = reinterpret_cast<AdjSeg *>(base); base += bsegs;
    a.photons = reinterpret_cast<AdjPhoton *>(base);
    a.order = reinterpret_cast<int *>(base + up(size_t(batch) * sizeof(AdjPhoton)));
    a.obucket = reinterpret_cast<unsigned *>(base + up(size_t(batch) * sizeof(AdjPhoton)) + up(size_t(batch) * sizeof(int)));
    base += bph;
    a.traj = reinterpret_cast<float4 *>(base);
    a.G = d_G; a.grad = d_grad; a.cnt = d_cnt;
    unsigned long long *d_kcnt = d_cnt + ADJ_COUNT;
    a.pool_next = d_kcnt + CNT_COUNT;
    a.traj_next = a.pool_next + 1;
    a.pending = reinterpret_cast<int *>(a.pool_next + 2);
    a.n_order = a.pool_next + 3;
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    int rc = SMP_OK;
    cudaError_t e = cudaMemcpy(d_G, dJ_dfilm, film * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_grad, 0, size_t(np) * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(d_cnt, 0, ncnt * sizeof(unsigned long long));
    for (int i = 0; i < 6 && e == cudaSuccess; ++i) e = cudaEventCreate(&ev[i]);
    unsigned long long c[ADJ_COUNT] = {0};
    unsigned long long fwd_steps = 0;
    long long launches = 0;
    float ms = 0.0f;
    double trace_ms = 0.0, replay_ms = 0.0, sweep_ms = 0.0;
    if (e != cudaSuccess) {
        rc = set_error(SMP_ERR_CUDA, "adjoint setup: %s", cudaGetErrorString(e));
    } else if (n_photons > 0) {
        KParams k = plan->kp;
        k.weight = photon_weight(plan->scene, weight_photons);
        k.records = nullptr;
        k.stream = nullptr;
        k.offsets = nullptr;
        k.counters = d_kcnt;
        k.event_batch = plan->event_batch;
        k.X = 0;                          // replays add nothing to any film
        cudaEventRecord(ev[0], 0);
        for (long long done = 0; done < n_photons && e == cudaSuccess; done += batch) {
            k.first_photon = first_photon + done;
            k.n_photons = std::min<long long>(batch, n_photons - done);
            e = cudaMemsetAsync(d_kcnt, 0, (CNT_COUNT + 1) * sizeof(unsigned long long), 0);
            cudaEventRecord(ev[2], 0);
            if (e == cudaSuccess) {
                if (trace_lanes) { fa<<<grid_a, kBlock>>>(k, a); ++launches; }
                else {
                    long long nl = 0;
                    e = adjoint_trace_pool(plan, k, a, fte, ftf, grid_tf, &nl);
                    launches += nl;
                }
            }
            if (e == cudaSuccess) { e = adjoint_order(a, k.n_photons, grid_r, 0); launches += 3; }
            cudaEventRecord(ev[3], 0);
            float tms = 0.0f;
            if (e == cudaSuccess) e = cudaEventSynchronize(ev[3]);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&tms, ev[2], ev[3]);
            trace_ms += tms;
            for (int round = 1; e == cudaSuccess; ++round) {
                e = cudaMemsetAsync(a.traj_next, 0, 2 * sizeof(unsigned long long), 0);
                if (e == cudaSuccess) e = cudaMemsetAsync(d_cnt + ADJ_NEXT, 0, sizeof(unsigned long long), 0);
                cudaEventRecord(ev[2], 0);
                if (e == cudaSuccess) { fr<<<grid_r, kBlock>>>(k, a, round); ++launches; }
                cudaEventRecord(ev[4], 0);
                if (e == cudaSuccess) e = cudaMemsetAsync(d_cnt + ADJ_NEXT, 0, sizeof(unsigned long long), 0);
                cudaEventRecord(ev[5], 0);
                if (e == cudaSuccess) { fs<<<grid_s, kBlock>>>(k, a, round); ++launches; }
                cudaEventRecord(ev[3], 0);
                if (e == cudaSuccess) e = cudaGetLastError();
                int pending = 0;
                if (e == cudaSuccess) e = cudaMemcpy(&pending, a.pending, sizeof(int), cudaMemcpyDeviceToHost);
                float rms = 0.0f, sms = 0.0f;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&rms, ev[2], ev[4]);
                if (e == cudaSuccess) e = cudaEventElapsedTime(&sms, ev[5], ev[3]);
                replay_ms += rms;
                sweep_ms += sms;
                if (!pending) break;
            }
            unsigned long long steps = 0;
            if (e == cudaSuccess) e = cudaMemcpy(&steps, d_kcnt + CNT_STEPS, sizeof(steps), cudaMemcpyDeviceToHost);
            fwd_steps += steps;
        }
        cudaEventRecord(ev[1], 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
        if (e == cudaSuccess) e = cudaMemcpy(grad_out, d_grad, size_t(np) * sizeof(double), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(c, d_cnt, sizeof(c), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = set_error(SMP_ERR_CUDA, "adjoint: %s", cudaGetErrorString(e));
    } else {
        std::memset(grad_out, 0, size_t(np) * sizeof(double));
    }
    if (stats_out) {
        stats_out->photons = (int64_t)c[ADJ_PHOTONS];
        stats_out->dropped = (int64_t)c[ADJ_DROPPED];
        stats_out->skipped = (int64_t)c[ADJ_SKIPPED];
        stats_out->aborted = (int64_t)c[ADJ_ABORTED];
        stats_out->replay_mismatch = (int64_t)c[ADJ_MISMATCH];
        stats_out->er_steps_forward = (int64_t)fwd_steps;
        stats_out->er_steps_replay = (int64_t)c[ADJ_STEPS_REPLAY];
        stats_out->points = (int64_t)c[ADJ_POINTS];
        stats_out->splats = (int64_t)c[ADJ_SPLATS];
        stats_out->kernel_ms = ms;
        stats_out->trace_ms = trace_ms;
        stats_out->launches = launches;
        stats_out->replay_ms = replay_ms;
        stats_out->sweep_ms = sweep_ms;
    }
    for (int i = 0; i < 6; ++i) if (ev[i]) cudaEventDestroy(ev[i]);
    if (!rc && c[ADJ_MISMATCH])
        rc = set_error(SMP_ERR_CUDA, "internal: %llu segment replay(s) diverged from their checkpoint", c[ADJ_MISMATCH]);
    return rc;
}

int smp_render_adjoint(const smp_scene_desc *scene, const smp_medium_desc *medium, const smp_field_desc *field,
                       const smp_render_opts *opts, int64_t n_photons, const double *dJ_dfilm, double *grad_out,
                       smp_adjoint_stats *stats_out) {
    smp_plan *p = nullptr;
    int rc = smp_plan_create(scene, medium, field, opts, &p);
    if (rc) return rc;
    rc = smp_plan_adjoint(p, 0, n_photons, n_photons > 0 ? n_photons : 1, dJ_dfilm, grad_out, stats_out);
    std::string err = g_last_error;
    smp_plan_destroy(p);
    g_last_error = err;
    return rc;
}

}  // extern "C"

// ==== Rendering without allocation ================================================================
// Some callers cannot call cudaMalloc: a host application whose device memory is owned by its own
// allocator or budget, code that must not hit cudaMalloc/cudaFree's implicit device-wide
// synchronisation in the middle of a frame, or a plugin host that hands the renderer only the
// buffers it may touch. smp_render_noalloc serves them: the caller passes the descriptors and an
// already-allocated device film; the work counter, statistics, Bessel table and texture CDF live
// in the fixed device array below, and host staging uses fixed static buffers.
//
// Limits: 1 MiB of device scratch per GPU that loads this library (held until the process exits);
// the texture CDF and the Bessel table share the scratch: 4 (texels + 1) + 32 x (table intervals)
// <= 1 MiB - 256 bytes (a 501 x 501 texture fits beside any table for k r up to 98; at most 262079
// texels); Bessel fields (orders 0-2) and plane-wave fields only.
// Every call on a device shares the scratch and overwrites what the previous call left there (the
// call clears the counters itself). Calls whose GPU work overlapped would race on it; this entry
// point prevents that within a process: it holds a process-wide lock from its first write to the
// scratch until its own GPU work has finished (it synchronises the stream before returning), so
// calls from several host threads, or on several streams, run one after another. The first call on
// each device looks up the array's device address (cudaGetSymbolAddress); make that first call
// before any stream capture. The caller's current device is restored on return.

#define SMP_NOALLOC_SCRATCH_BYTES (1u << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[SMP_NOALLOC_SCRATCH_BYTES];

namespace {
const size_t kNoAllocCountersBytes = 256;
const size_t kNoAllocShared = SMP_NOALLOC_SCRATCH_BYTES - kNoAllocCountersBytes;   // table, then CDF
const int kNoAllocTabMax = 2 * 2049;                                 // float4 entries for k r <= 128
const size_t kNoAllocCdfFloats = kNoAllocShared / sizeof(float);
const int kNoAllocMaxDevices = 64;

unsigned char *g_noalloc_dev[kNoAllocMaxDevices];                  // device address per device
std::mutex g_noalloc_mutex;                                          // guards the host staging below
float g_noalloc_cdf_host[kNoAllocCdfFloats];
float4 g_noalloc_tab_host[kNoAllocTabMax];
}  // namespace

// The array's device address on the current device, looked up once per device.
static int noalloc_scratch(int dev, unsigned char **out) {
    if (dev < 0 || dev >= kNoAllocMaxDevices) return set_error(SMP_ERR_BAD_ARG, "device %d beyond %d", dev, kNoAllocMaxDevices);
    if (!g_noalloc_dev[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return set_error(SMP_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
        g_noalloc_dev[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_noalloc_dev[dev];
    return SMP_OK;
}

extern "C" int smp_render_noalloc(const smp_scene_desc *scene, const smp_medium_desc *medium,
                                  const smp_field_desc *field, const smp_render_opts *opts,
                                  int64_t first_photon, int64_t n_photons, int64_t weight_photons,
                                  void *d_film, void *stream, smp_stats *stats_out) {
    int rc = check_descs(scene, medium, field, opts);
    if (rc) return rc;
    if (!d_film) return set_error(SMP_ERR_BAD_ARG, "d_film is NULL");
    if (opts->rng != SMP_RNG_PHILOX) return set_error(SMP_ERR_BAD_ARG, "smp_render_noalloc draws from Philox");
    if (n_photons < 0 || first_photon < 0 || weight_photons <= 0) return set_error(SMP_ERR_BAD_ARG, "bad photon range");
    int fk;
    rc = field_kind(*field, &fk);
    if (rc) return rc;
    if (!(fk <= FK_BESSEL2 || fk == FK_PLANEWAVE))
        return set_error(SMP_ERR_UNSUPPORTED, "smp_render_noalloc renders Bessel (orders 0-2) and plane-wave fields");
    const long long n_tex = (long long)scene->tex_x * scene->tex_y;
    int tab_entries = 0;
    if (fk <= FK_BESSEL2) {
        const float k_r = (2.0f * 3.14159265358979f) / (float(field->speed_u) / float(field->f_u));
        tab_entries = 2 * bessel_intervals(box_max_kr(*scene, k_r));
    }
    const size_t tab_bytes = size_t(tab_entries) * sizeof(float4);
    if (tab_bytes + (size_t(n_tex) + 1) * sizeof(float) > kNoAllocShared)
        return set_error(SMP_ERR_BAD_ARG, "texture has %lld texels; beside this field's Bessel table "
                         "smp_render_noalloc holds at most %zu", n_tex, (kNoAllocShared - tab_bytes) / sizeof(float) - 1);
    // the caller's current device is put back on every return path
    struct DeviceRestore {
        int dev = -1;
        ~DeviceRestore() { if (dev >= 0) cudaSetDevice(dev); }
    } restore;
    if (cudaGetDevice(&restore.dev) != cudaSuccess) restore.dev = -1;
    rc = check_device(opts->device);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    unsigned char *scratch = nullptr;
    rc = noalloc_scratch(opts->device, &scratch);
    if (rc) return rc;
    unsigned long long *d_counters = reinterpret_cast<unsigned long long *>(scratch);
    float4 *d_tab = reinterpret_cast<float4 *>(scratch + kNoAllocCountersBytes);
    float *d_cdf = reinterpret_cast<float *>(scratch + kNoAllocCountersBytes + tab_bytes);

    KParams k;
    std::memset(&k, 0, sizeof(k));
    for (int i = 0; i < 3; ++i) {
        k.L[i] = float(scene->medium_l[i]);
        k.R[i] = float(scene->medium_r[i]);
        k.src_origin[i] = float(scene->light_origin[i]);
        k.src_lens_origin[i] = float(scene->emitter_lens_origin[i]);
        k.cam_origin[i] = float(scene->view_origin[i]);
        k.cam_lens_origin[i] = float(scene->sensor_lens_origin[i]);
    }
    set_box_thresholds(k);
    k.plane[0] = float(scene->light_plane[0]);
    k.plane[1] = float(scene->light_plane[1]);
    k.pixsize[0] = k.plane[0] / float(scene->tex_x);
    k.pixsize[1] = k.plane[1] / float(scene->tex_y);
    k.ct = std::cos(float(scene->half_theta_limit));
    k.tex_x = scene->tex_x;
    k.n_tex = int(n_tex);
    k.src_lens_active = scene->emitter_lens_active;
    k.src_lens_sqap = float(scene->emitter_lens_aperture) * float(scene->emitter_lens_aperture);
    k.src_lens_focal = float(scene->emitter_lens_focal_length);
    float cd[3], ch[3];
    for (int i = 0; i < 3; ++i) { cd[i] = float(scene->view_dir[i]); ch[i] = float(scene->view_horizontal[i]); }
    float ld = std::sqrt(cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
    float lh = std::sqrt(ch[0] * ch[0] + ch[1] * ch[1] + ch[2] * ch[2]);
    for (int i = 0; i < 3; ++i) { k.cam_dir[i] = cd[i] / ld; k.cam_h[i] = ch[i] / lh; }
    k.cam_v[0] = k.cam_dir[1] * k.cam_h[2] - k.cam_dir[2] * k.cam_h[1];
    k.cam_v[1] = k.cam_dir[2] * k.cam_h[0] - k.cam_dir[0] * k.cam_h[2];
    k.cam_v[2] = k.cam_dir[0] * k.cam_h[1] - k.cam_dir[1] * k.cam_h[0];
    k.cam_plane[0] = float(scene->view_plane[0]);
    k.cam_plane[1] = float(scene->view_plane[1]);
    k.pl_min = float(scene->pathlength_range[0]);
    k.pl_max = float(scene->pathlength_range[1]);
    k.bounce = scene->use_bounce_decomposition;
    k.cam_lens_active = scene->sensor_lens_active;
    k.cam_lens_sqap = float(scene->sensor_lens_aperture) * float(scene->sensor_lens_aperture);
    k.cam_lens_focal = float(scene->sensor_lens_focal_length);
    k.ior1 = 1.0f;
    k.ior2 = float(scene->ior);
    k.sigma_t = float(medium->sigma_t);
    k.albedo = float(medium->albedo);
    k.mfp = 1.0f / float(medium->sigma_t);
    if (k.sigma_t <= 1.19209290e-07f) { k.sigma_t = 0.0f; k.mfp = 1.0f; k.albedo = 0.0f; }
    k.g = float(medium->g);
    k.max_depth = opts->max_depth;
    k.max_pathlength = float(opts->max_pathlength);
    k.use_direct = opts->use_direct;
    k.use_angular = opts->use_angular_sampling;
    k.step_cap = int(std::min<int64_t>(opts->step_cap > 0 ? opts->step_cap : 10000000LL, 2000000000LL));
    k.large_dist = sensor_march_budget(*opts, k.sigma_t);
    k.X = scene->x_res; k.Y = scene->y_res; k.Z = scene->z_res;
    k.fp64 = opts->precision == SMP_PREC_MIXED;
    k.rng = SMP_RNG_PHILOX;
    k.seed = opts->seed;
    k.weight = photon_weight(*scene, weight_photons);
    k.first_photon = first_photon;
    k.n_photons = n_photons;
    k.event_batch = 8;
    k.film = d_film;
    k.counters = d_counters;
    k.cdf = d_cdf;
    fill_field_params(*field, fk, k.field);
    set_step_sizes(k, *field);

    // texture CDF (pmf.h:41-99, float) into the static host buffer, then into the scratch
    float *cdf = g_noalloc_cdf_host;
    cdf[0] = 0.0f;
    for (long long i = 0; i < n_tex; ++i) cdf[i + 1] = cdf[i] + static_cast<float>(scene->texture[i]);
    if (cdf[n_tex] > 0.0f) {
        float norm = 1.0f / cdf[n_tex];
        for (long long i = 1; i <= n_tex; ++i) cdf[i] *= norm;
        cdf[n_tex] = 1.0f;
    }
    SMP_CUDA(cudaMemcpyAsync(d_cdf, cdf, size_t(n_tex + 1) * sizeof(float), cudaMemcpyHostToDevice, s));
    size_t smem = 0;
    if (fk <= FK_BESSEL2) {
        bessel_table_fill(field->mode, tab_entries / 2, g_noalloc_tab_host);
        SMP_CUDA(cudaMemcpyAsync(d_tab, g_noalloc_tab_host, tab_bytes, cudaMemcpyHostToDevice, s));
        k.field.btab = d_tab;
        k.field.bnodes = tab_entries;
        k.field.bint = tab_entries / 2;
        smem = tab_bytes;
    }
    SMP_CUDA(cudaMemsetAsync(d_counters, 0, CNT_COUNT * sizeof(unsigned long long), s));
    int grid = 0;
    rc = grid_for(fk, opts->device, opts->blocks_per_sm, smem, &grid);
    if (rc) return rc;
    if (n_photons > 0) {
        march_fn(fk)<<<grid, kBlock, smem, s>>>(k);
        SMP_CUDA(cudaGetLastError());
    }
    unsigned long long c[CNT_COUNT];
    SMP_CUDA(cudaMemcpyAsync(c, d_counters, sizeof(c), cudaMemcpyDeviceToHost, s));
    SMP_CUDA(cudaStreamSynchronize(s));
    if (stats_out) {
        std::memset(stats_out, 0, sizeof(*stats_out));
        stats_out->photons = (int64_t)c[CNT_PHOTONS];
        stats_out->er_steps = (int64_t)c[CNT_STEPS];
        stats_out->splats = (int64_t)c[CNT_SPLATS];
        stats_out->step_cap_hits = (int64_t)c[CNT_STEP_CAP];
        stats_out->nan_photons = (int64_t)c[CNT_NAN];
        stats_out->march_steps = (int64_t)c[CNT_STEPS];
        stats_out->launches = n_photons > 0 ? 1 : 0;
        stats_out->march_launches = stats_out->launches;
    }
    if (c[CNT_STAGE_TIMEOUT]) return set_error(SMP_ERR_CUDA, "%llu block(s) timed out staging the field table", c[CNT_STAGE_TIMEOUT]);
    if (c[CNT_STEP_CAP]) return set_error(SMP_ERR_STEP_CAP, "%llu photon(s) hit the per-photon step cap", c[CNT_STEP_CAP]);
    if (c[CNT_NAN]) return set_error(SMP_ERR_NAN, "%llu photon(s) produced a non-finite state", c[CNT_NAN]);
    return SMP_OK;
}
