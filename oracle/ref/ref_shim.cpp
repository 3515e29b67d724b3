// oracle/ref/ref_shim.cpp -- TEST INFRASTRUCTURE. C entry points over the reference's own
// compiled primitives (built by oracle/ref/build_ref.sh from the reference sources in place),
// used only to pin the oracle's restatements. Never part of the product.
#include <cstdint>
#include "rng_sse.h"
#include "phase.h"
#include "warp.h"
#include "util.h"
#include "bsdf.h"
#include "lens.h"
#include "pmf.h"

extern "C" {

int ref_sfmt_float(uint64_t seed, int n, float *out) {
    rng::SSEEngine e;
    e.seed(seed);
    for (int i = 0; i < n; ++i) out[i] = e();
    return 0;
}

float ref_hg_sample(float g, const float *in, uint64_t seed, int skip, float *out) {
    rng::SSEEngine e;
    e.seed(seed);
    for (int i = 0; i < skip; ++i) (void)e();
    pfunc::henyey_greenstein hg(g);
    tvec::Vec3f o;
    float c = hg.sample(tvec::Vec3f(in[0], in[1], in[2]), e, o);
    out[0] = o.x; out[1] = o.y; out[2] = o.z;
    return c;
}

float ref_hg_f(float g, const float *in, const float *out) {
    pfunc::henyey_greenstein hg(g);
    return hg.f(tvec::Vec3f(in[0], in[1], in[2]), tvec::Vec3f(out[0], out[1], out[2]));
}

void ref_hemisphere(float u0, float u1, float *out) {
    tvec::Vec3f v = warp::squareToUniformHemisphere(tvec::Vec2f(u0, u1));
    out[0] = v.x; out[1] = v.y; out[2] = v.z;
}

float ref_fresnel(float cosI, float cosT, float eta) {
    return util::fresnelDielectric(cosI, cosT, eta);
}

int ref_refract(const float *a, const float *n, float eta, float *b) {
    tvec::Vec3f out;
    bool ok = util::refract(tvec::Vec3f(a[0], a[1], a[2]), tvec::Vec3f(n[0], n[1], n[2]), eta, out);
    b[0] = out.x; b[1] = out.y; b[2] = out.z;
    return ok ? 1 : 0;
}

void ref_coordinate_system(const float *a, float *b, float *c) {
    tvec::Vec3f vb, vc;
    util::coordinateSystem(tvec::Vec3f(a[0], a[1], a[2]), vb, vc);
    b[0] = vb.x; b[1] = vb.y; b[2] = vb.z;
    c[0] = vc.x; c[1] = vc.y; c[2] = vc.z;
}

void ref_bsdf_sample(float ior1, float ior2, const float *in, const float *n, uint64_t seed,
                     int skip, float *out) {
    rng::SSEEngine e;
    e.seed(seed);
    for (int i = 0; i < skip; ++i) (void)e();
    bsdf::SmoothDielectric<tvec::TVector3> b(ior1, ior2);
    tvec::Vec3f o;
    b.sample(tvec::Vec3f(in[0], in[1], in[2]), tvec::Vec3f(n[0], n[1], n[2]), e, o);
    out[0] = o.x; out[1] = o.y; out[2] = o.z;
}

long ref_pmf_sample(const double *pdf, int n, int n_u, const float *u, long *idx_out, float *cdf_out) {
    DiscreteDistribution d;
    d.reserve(n);
    for (int i = 0; i < n; ++i) d.append(static_cast<Float>(pdf[i]));
    d.normalize();
    const std::vector<Float> &c = d.get_cdf();
    for (size_t i = 0; i < c.size(); ++i) cdf_out[i] = c[i];
    for (int i = 0; i < n_u; ++i) idx_out[i] = static_cast<long>(d.sample(u[i]));
    return static_cast<long>(c.size());
}

int ref_lens_propagate(const float *origin, float aperture, float focal, int active,
                       float *pos, float *dir, float *total) {
    scn::Lens<tvec::TVector3> lens(tvec::Vec3f(origin[0], origin[1], origin[2]), aperture, focal,
                                   active != 0);
    tvec::Vec3f p(pos[0], pos[1], pos[2]), d(dir[0], dir[1], dir[2]);
    Float t = *total;
    bool ok = lens.propagate_till_lens(p, d, t);
    pos[0] = p.x; pos[1] = p.y; pos[2] = p.z;
    dir[0] = d.x; dir[1] = d.y; dir[2] = d.z;
    *total = t;
    return ok ? 1 : 0;
}

int ref_lens_deflect(const float *origin, float aperture, float focal, const float *pos,
                     float *dir, float *total) {
    scn::Lens<tvec::TVector3> lens(tvec::Vec3f(origin[0], origin[1], origin[2]), aperture, focal, true);
    tvec::Vec3f d(dir[0], dir[1], dir[2]);
    Float t = *total;
    bool ok = lens.deflect(tvec::Vec3f(pos[0], pos[1], pos[2]), d, t);
    dir[0] = d.x; dir[1] = d.y; dir[2] = d.z;
    *total = t;
    return ok ? 1 : 0;
}

}  // extern "C"
