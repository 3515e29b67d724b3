// march.cuh -- the persistent photon-march kernel for sm_100a.
//
// One lane owns one photon at a time and runs the reference's per-photon algorithm
// (renderer/src/photon.cpp:302-335: genRay, scaling draw, directTracing, scatter with a sensor
// connection at every vertex) as a state machine. The expensive part -- traceTillBlock, the
// kick-drift-kick ER march with 10x refinement at faces and at the sampled distance
// (scene.cpp:385-425, :323-330) -- is one "step" that every marching lane of the warp executes
// together. When a lane's march ends it runs the discrete logic that follows (face normal,
// Fresnel BSDF, splat, Henyey-Greenstein scattering, roulette) until its next march starts; when
// its photon ends it takes a new photon index from a global counter (one atomic per warp), so
// warps stay full until the work runs out. Grid = resident CTAs over all SMs.
//
// Discrete decisions follow the reference CPU build exactly; the tests compare every photon's
// splats and end state with the CPU restatement on injected uniform streams.
#pragma once
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include "dev_field.cuh"
#include "kparams.h"

namespace smp {

namespace cg = cooperative_groups;

static constexpr unsigned kFull = 0xffffffffu;

// Resident 128-thread blocks per SM the march kernel is compiled for (register budget 65536 /
// (128 * blocks)).
#ifndef SMP_MIN_BLOCKS
#define SMP_MIN_BLOCKS 4
#endif

enum LaneState : int { ST_FETCH = 0, ST_EVENT = 1, ST_MARCH = 2, ST_DONE = 3, ST_HOOK = 4 };
enum Event : int {
    EV_NEW = 0,          // photon fetched: genRay, scaling, direct or scatter
    EV_MARCH_END = 1,    // a traceTillBlock call finished
    EV_SCATTER = 2,      // Renderer::scatter entry (photon.cpp:97)
    EV_VERTEX = 3,       // head of the scatter loop (photon.cpp:113)
    EV_SCATTER_ONCE = 4, // Renderer::scatterOnce (photon.cpp:20)
    EV_FINISH = 5
};
enum Ctx : int { CTX_DIRECT = 0, CTX_CONNECT = 1, CTX_MOVE_FIRST = 2, CTX_MOVE_VERTEX = 3 };

struct Lane {
    // photon
    long long idx;
    float3 pos, dir;          // scatter()'s pos/dir (photon.cpp:98)
    float s;                  // temporal scaling (Bessel) / phase tau (plane waves)
    double total;             // running optical path length
    float totalDist;          // first sampled distance (photon.cpp:112)
    int depth, nspl, draws, steps, end;
    // uniforms
    unsigned r0, r1, r2, r3, rblk;
    int rhave;
    long long spos, send;
    // current march (traceTillBlock) and its caller (movePhoton / movePhotonTillSensor)
    float3 mp, md, mg;        // position, optical direction v, grad n at mp
    float mn;                 // n at mp
    double mtot;              // optical length accumulated by this march (FP64 form)
    float mtotf;              // the same in the FP32 form
    float dist_acc, dlimit, cur, hh;   // hh = cur / 2
    double cur_d;             // cur in double for the FP64 accumulator
    int stop;                 // step count at which traceTillBlock's loop count runs out (<= step cap)
    int prec, ctx, first;
    float large, d2s, rem, sampled;
    const float4 *tab;        // Bessel table in this block's shared memory
    const Inst *inst;         // batched sweep: the photon's instance
};

// Per-photon medium, weight, film and seed: the instance's in a batched sweep (n_inst is uniform
// over the grid, so these are uniform branches), else the plan's.
__device__ __forceinline__ float med_g(const Lane &L, const KParams &P) { return P.n_inst ? L.inst->g : P.g; }
__device__ __forceinline__ float med_albedo(const Lane &L, const KParams &P) { return P.n_inst ? L.inst->albedo : P.albedo; }
__device__ __forceinline__ float med_sigma_t(const Lane &L, const KParams &P) { return P.n_inst ? L.inst->sigma_t : P.sigma_t; }
__device__ __forceinline__ float med_mfp(const Lane &L, const KParams &P) { return P.n_inst ? L.inst->mfp : P.mfp; }
__device__ __forceinline__ float med_weight(const Lane &L, const KParams &P) { return P.n_inst ? L.inst->weight : P.weight; }
__device__ __forceinline__ float med_large(const Lane &L, const KParams &P) { return P.n_inst ? L.inst->large_dist : P.large_dist; }
__device__ __forceinline__ void *med_film(const Lane &L, const KParams &P) { return P.n_inst ? L.inst->film : P.film; }
__device__ __forceinline__ unsigned long long med_seed(const Lane &L, const KParams &P) { return P.n_inst ? L.inst->seed : P.seed; }
// the field the photon marches through
template <int FK, class S>
__device__ __forceinline__ const FieldParams &field_of(const S &L, const KParams &P) {
    return FK == FK_BATCH ? L.inst->field : P.field;
}

// ---- uniforms -----------------------------------------------------------------------------
__device__ __forceinline__ void philox_block(unsigned &c0, unsigned &c1, unsigned &c2, unsigned &c3,
                                             unsigned k0, unsigned k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        unsigned hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        unsigned hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

// one Philox block, kept out of line: draw() is called from many places in the event code
static __device__ __noinline__ uint4 philox_refill(unsigned blk, unsigned ph_lo, unsigned ph_hi, unsigned k0, unsigned k1) {
    unsigned c0 = blk, c1 = 0u, c2 = ph_lo, c3 = ph_hi;
    philox_block(c0, c1, c2, c3, k0, k1);
    return make_uint4(c0, c1, c2, c3);
}

__device__ __forceinline__ float draw(Lane &L, const KParams &P) {
    ++L.draws;
    if (P.rng == SMP_RNG_STREAM) {
        if (L.spos < L.send) return __ldg(P.stream + (L.spos++));
        L.end = SMP_END_STREAM;
        return 0.5f;
    }
    if (L.rhave == 0) {
        const unsigned long long seed = med_seed(L, P);
        uint4 b = philox_refill(L.rblk++, unsigned(L.idx), unsigned(L.idx >> 32), unsigned(seed), unsigned(seed >> 32));
        L.r0 = b.x; L.r1 = b.y; L.r2 = b.z; L.r3 = b.w;
        L.rhave = 4;
    }
    unsigned x = L.r0;
    L.r0 = L.r1; L.r1 = L.r2; L.r2 = L.r3;
    --L.rhave;
    return float(x >> 8) * (1.0f / 16777216.0f);
}

// ---- small pieces of the scene -------------------------------------------------------------
__device__ __forceinline__ int steps_for(float dlimit, float h0) {
    // (long)(dist/h + 1) as the reference's x86-64 build converts it (scene.cpp:391): out-of-range
    // values become INT64_MIN (no steps). Counts above 2^31 - 1 are clamped: the per-photon step
    // cap (<= 2e9) ends the photon first.
    float v = dlimit / h0 + 1.0f;
    if (!(v >= -9.2233720e18f && v < 9.2233720e18f)) return 0;
    if (v >= 2147483647.0f) return 2147483647;
    return int(v);
}


// nearest face of the medium box (scene.cpp:655-676 / :736-757)
__device__ __forceinline__ float3 face_normal(const KParams &P, float3 p) {
    float best = 3.40282347e+38f, dirv = 0.0f;
    int chosen = 3;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float pi = comp(p, i);
        float d = fabsf(P.L[i] - pi);
        if (d < best) { best = d; chosen = i; dirv = -1.0f; }
        d = fabsf(P.R[i] - pi);
        if (d < best) { best = d; chosen = i; dirv = 1.0f; }
    }
    return f3(chosen == 0 ? dirv : 0.0f, chosen == 1 ? dirv : 0.0f, chosen == 2 ? dirv : 0.0f);
}

// util.h:42-57
__device__ __forceinline__ float fresnel(float cosI, float cosT, float eta) {
    if (fabsf(eta - 1.0f) < kEps * fmaxf(1.0f, fabsf(eta))) return 0.0f;
    float Rs = (cosI - eta * cosT) / (cosI + eta * cosT);
    float Rp = (cosT - eta * cosI) / (cosT + eta * cosI);
    return 0.5f * (Rs * Rs + Rp * Rp);
}

// SmoothDielectric::sample (bsdf.cpp:26-58, util.h:64-88)
__device__ __forceinline__ float3 bsdf_sample(Lane &L, const KParams &P, float3 in, float3 n) {
    if (fabsf(P.ior1 - P.ior2) < kEps) return in;
    float eta = (dot3(in, n) < -kEps) ? P.ior2 / P.ior1 : P.ior1 / P.ior2;
    float an = dot3(in, n);
    float3 q = mul(n, an);
    float3 pp = divs(sub(in, q), eta);
    float3 refl = add(mul(n, -2.0f * an), in);
    if (len3(pp) > 1.0f) return refl;                       // total internal reflection
    q = normalized(q);
    float t = 1.0f - dot3(pp, pp);
    float3 outT = add(pp, mul(q, t > 0.0f ? sqrtf(t) : 0.0f));
    float cosI = fabsf(dot3(n, in)), cosT = fabsf(dot3(n, outT));
    float F = fresnel(cosI, cosT, eta);
    return (draw(L, P) < F) ? refl : outT;
}

// thin lens deflection (lens.cpp:70-97); returns the path-length change in add_len
__device__ __forceinline__ bool lens_deflect(float sqap, float focal, float3 pos, float3 &dir, float &add_len) {
    float sq = pos.y * pos.y + pos.z * pos.z;
    if (sq > sqap) return false;
    float invd = -1.0f / dir.x;
    dir = f3(-focal, dir.y * invd * focal - pos.y, dir.z * invd * focal - pos.z);
    add_len = focal * invd - len3(dir);
    dir = normalized(dir);
    return true;
}

__device__ __forceinline__ void acc_total(double &t, float v, bool fp64) {
    t = fp64 ? t + double(v) : double(float(t) + v);
}

// Camera::propagate_till_sensor (camera.cpp:54-75): the distance goes into the caller's local
// distanceToSensor, which the caller then adds to its path length.
__device__ __forceinline__ bool propagate_till_sensor(const KParams &P, float3 &pos, float3 &dir, float &dts) {
    if (P.cam_lens_active) {
        float a = 0.0f;
        if (!lens_deflect(P.cam_lens_sqap, P.cam_lens_focal, pos, dir, a)) return false;
        dts += a;
    }
    float dist = (P.cam_origin[0] - pos.x) / dir.x;
    pos = add(pos, mul(dir, dist));
    dts += dist;
    return true;
}

// Scene::addEnergyToImage (scene.cpp:782-829) with bilinear sharing (USE_PIXEL_SHARING): one tap,
// Image3::addEnergy (image.h:320-324) with the bounds check of addPixel (scene.h:305-312).
// Warp-aggregated: the lanes that reach this call together are grouped by the film address they
// add to (__match_any_sync through cooperative groups), each group sums its values (in double for
// the FP64 film) and one lane issues the atomic. A narrow beam's direct light lands on a handful of
// pixels, where one atomic per lane would serialise on the same address.
__device__ __forceinline__ void add_pixel(const KParams &P, void *film, int x, int y, int z, float v) {
    const bool in = x >= 0 && x < P.X && y >= 0 && y < P.Y && z >= 0 && z < P.Z;
    const size_t i = in ? (size_t(z) * P.Y + y) * P.X + x : 0;
    const unsigned long long key =
        in ? reinterpret_cast<unsigned long long>(film) + (unsigned long long)i * (P.fp64 ? 8ull : 4ull) : 0ull;
    const cg::coalesced_group active = cg::coalesced_threads();
    const cg::coalesced_group same = cg::labeled_partition(active, key);
    if (P.fp64) {
        const double s = cg::reduce(same, double(v), cg::plus<double>());
        if (in && same.thread_rank() == 0) atomicAdd(reinterpret_cast<double *>(film) + i, s);
    } else {
        const float s = cg::reduce(same, v, cg::plus<float>());
        if (in && same.thread_rank() == 0) atomicAdd(reinterpret_cast<float *>(film) + i, s);
    }
}

// Film cell of a splat at sensor point p with path length pl (scene.cpp:782-829) on a film X
// pixels wide: the bilinear base pixel (ix, iy), its fractions (fx, fy) and the bin iz; false when
// pl is outside the binned range.
__device__ __forceinline__ bool splat_bin(const KParams &P, int X, float3 p, double pl, int depth,
                                          int &ix, int &iy, int &iz, float &fx, float &fy) {
    float x = dot3(ld3(P.cam_h), p) - P.cam_origin[1];
    float y = dot3(ld3(P.cam_v), p) - P.cam_origin[2];
    bool nobin = (P.pl_min == -1.0f) && (P.pl_max == -1.0f);
    bool inrange = P.fp64 ? (pl > double(P.pl_min) && pl < double(P.pl_max))
                          : (float(pl) > P.pl_min && float(pl) < P.pl_max);
    if (!(nobin || inrange)) return false;
    x = (x / P.cam_plane[0] + 0.5f) * float(X);
    y = (y / P.cam_plane[1] + 0.5f) * float(P.Y);
    float flx = floorf(x), fly = floorf(y);
    ix = int(flx); iy = int(fly);
    if (P.bounce) iz = depth;
    else if (nobin) iz = 0;
    else if (P.fp64) iz = int(floor((pl - double(P.pl_min)) / (double(P.pl_max) - double(P.pl_min)) * double(P.Z)));
    else iz = int(floorf(((float(pl) - P.pl_min) / (P.pl_max - P.pl_min)) * float(P.Z)));
    fx = x - flx; fy = y - fly;
    return true;
}

__device__ __forceinline__ void splat(Lane &L, const KParams &P, float3 p, double pl, int depth, float val) {
    if (P.records) {
        smp_photon_record *rec = P.records + (L.idx - P.first_photon);
        if (L.nspl < SMP_TRACE_MAX_SPLATS) {
            smp_splat_record &sr = rec->splats[L.nspl];
            sr.p[0] = p.x; sr.p[1] = p.y; sr.p[2] = p.z;
            sr.depth = depth;
            sr.pathlength = pl;
            sr.value = double(val);
        }
    }
    ++L.nspl;
    int ix, iy, iz;
    float fx, fy;
    if (!splat_bin(P, P.X, p, pl, depth, ix, iy, iz, fx, fy)) return;
    void *film = med_film(L, P);
    add_pixel(P, film, ix, iy, iz, val * (1.0f - fx) * (1.0f - fy));
    add_pixel(P, film, ix + 1, iy, iz, val * fx * (1.0f - fy));
    add_pixel(P, film, ix, iy + 1, iz, val * (1.0f - fx) * fy);
    add_pixel(P, film, ix + 1, iy + 1, iz, val * fx * fy);
}

// Henyey-Greenstein (phase.cpp:17-21, :40-76; util.h:17-27)
__device__ __forceinline__ float hg_f(float g, float3 in, float3 out) {
    float c = dot3(in, out);
    float b = 1.0f + g * g - 2.0f * g * c;
    return (1.0f / (4.0f * 3.14159265358979f)) * (1.0f - g * g) / (b * sqrtf(b));
}
__device__ __forceinline__ float3 hg_sample(Lane &L, const KParams &P, float3 in) {
    float sx = draw(L, P);
    float sy = draw(L, P);
    float g = med_g(L, P), cosT;
    if (fabsf(g) < kEps) cosT = 1.0f - 2.0f * sx;
    else {
        float sq = (1.0f - g * g) / (1.0f - g + 2.0f * g * sx);
        cosT = (1.0f + g * g - sq * sq) / (2.0f * g);
    }
    float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
    float phi = 6.28318548202514648f * sy;
    float sP, cP;
    sincos_red(phi, sP, cP);
    float3 ax, ay;
    if (fabsf(in.x) > fabsf(in.y)) {
        float inv = 1.0f / sqrtf(in.x * in.x + in.z * in.z);
        ay = f3(in.z * inv, 0.0f, -in.x * inv);
    } else {
        float inv = 1.0f / sqrtf(in.y * in.y + in.z * in.z);
        ay = f3(0.0f, in.z * inv, -in.y * inv);
    }
    ax = cross3(ay, in);
    return add(add(mul(ax, sinT * cP), mul(ay, sinT * sP)), mul(in, cosT));
}

// sampleRandomDirection (scene.cpp:26-39, warp.cpp:22-34): first draw -> azimuth, second -> z,
// the order the reference's GCC build evaluates Vec2f(sampler(), sampler()).
__device__ __forceinline__ float3 random_direction(Lane &L, const KParams &P) {
    float uy = draw(L, P);
    float ux = draw(L, P);
    float tmp = sqrtf(1.0f - ux * ux);
    float sP, cP;
    sincos_red(6.28318548202514648f * uy, sP, cP);
    return f3(-ux, cP * tmp, sP * tmp);
}

__device__ __forceinline__ bool roulette(Lane &L, const KParams &P) {
    const float albedo = med_albedo(L, P);
    return (albedo > 0.0f) && ((albedo >= 1.0f) || (draw(L, P) < albedo));
}

// area_textured_source::sample_ray (scene.cpp:107-137) + DiscreteDistribution::sample (pmf.h:109-121)
__device__ __forceinline__ bool gen_ray(Lane &L, const KParams &P, float3 &pos, float3 &dir, double &total) {
    float u = draw(L, P);
    int lo = 0, hi = P.n_tex + 1;                 // lower_bound over n_tex + 1 cdf entries
    if (P.cdf_guide) {
        // u's bucket of the guide table narrows the search to a few entries; the CDF is monotone
        // (the host builds no guide otherwise), so the lower bound found is the same
        const int G = 1 << P.guide_bits;
        const int b = min(int(u * float(G)), G);
        lo = __ldg(P.cdf_guide + b);
        hi = __ldg(P.cdf_guide + b + 1);
    }
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(P.cdf + mid) < u) lo = mid + 1; else hi = mid;
    }
    int idx = min(P.n_tex - 1, max(0, lo - 1));
    while (idx < P.n_tex && __ldg(P.cdf + idx + 1) - __ldg(P.cdf + idx) == 0.0f) ++idx;
    if (idx > P.n_tex - 1) idx = P.n_tex - 1;
    int py = idx / P.tex_x;
    int px = idx - py * P.tex_x;
    pos = ld3(P.src_origin);
    float uy = draw(L, P);
    pos.y += -P.plane[0] / 2.0f + float(px) * P.pixsize[0] + uy * P.pixsize[0];
    float uz = draw(L, P);
    pos.z += -P.plane[1] / 2.0f + float(py) * P.pixsize[1] + uz * P.pixsize[1];
    float z = draw(L, P) * (1.0f - P.ct) + P.ct;
    float zt = sqrtf(1.0f - z * z);
    float phi = draw(L, P) * 2.0f * 3.14159265358979f;
    float sP, cP;
    sincos_red(phi, sP, cP);
    dir = f3(-z, zt * cP, zt * sP);
    // Lens::propagate_till_lens (lens.cpp:20-33)
    float dist = -(pos.x - P.src_lens_origin[0]) / dir.x;
    pos = add(pos, mul(dir, dist));
    acc_total(total, dist, P.fp64);
    if (P.src_lens_active) {
        float a = 0.0f;
        if (!lens_deflect(P.src_lens_sqap, P.src_lens_focal, pos, dir, a)) return false;
        acc_total(total, a, P.fp64);
    }
    return true;
}

// ---- the traceTillBlock step ----------------------------------------------------------------
// the photon's ER step and refinement steps: its instance's in a batched sweep, else the plan's
template <int FK, class S>
__device__ __forceinline__ float step_h0(const S &L, const KParams &P) { return FK == FK_BATCH ? L.inst->h0 : P.h0; }
template <int FK, class S>
__device__ __forceinline__ const float *step_tab(const S &L, const KParams &P) {
    return FK == FK_BATCH ? L.inst->cur_tab : P.cur_tab;
}

template <int FK>
__device__ __forceinline__ void begin_march(Lane &L, const KParams &P, float dlimit, bool eval) {
    if (eval) Field<FK>::eval(field_of<FK>(L, P), L.tab, L.mp, L.s, L.mn, L.mg);
    const float h0 = step_h0<FK>(L, P);
    L.dist_acc = 0.0f;
    L.dlimit = dlimit;
    L.cur = h0;
    L.hh = 0.5f * h0;
    L.cur_d = double(h0);
    L.prec = P.precision;
    L.stop = int(min((long long)L.steps + (long long)steps_for(dlimit, h0), (long long)P.step_cap));
    L.mtotf = float(L.mtot);
}
// a march with no steps ends at once (traceTillBlock's maxsteps <= 0)
__device__ __forceinline__ bool march_has_steps(const Lane &L) { return L.stop > L.steps; }

// One iteration of the traceTillBlock loop (scene.cpp:395-419): kick, drift, one fused field
// evaluation, kick, then the loop's tests. Returns true when the march has ended (loop count or
// refinement exhausted, or the photon aborted). S is a Lane or any state with the same march
// members.
//
// The tests are arranged for the common case, an accepted step with steps to go: the box test
// (thresholds box_lo/box_hi, exact) and the distance test (dist_acc + cur <= dlimit) are one chain
// of predicate comparisons, and the loop count and the step cap share one counter (`stop` is the
// loop's end clamped to the cap; the cap is told apart on the rare path).
template <int FK, int FP = -1, class S>
__device__ __forceinline__ bool march_step(S &L, const KParams &P) {
    const bool f64 = FP < 0 ? P.fp64 != 0 : FP != 0;     // FP: the path-length form, if fixed at compile time
    const float3 d = f3(fmaf(L.hh, L.mg.x, L.md.x), fmaf(L.hh, L.mg.y, L.md.y), fmaf(L.hh, L.mg.z, L.md.z));
    const float hinv = L.cur * rcp_fast(L.mn);
    const float3 p = f3(fmaf(d.x, hinv, L.mp.x), fmaf(d.y, hinv, L.mp.y), fmaf(d.z, hinv, L.mp.z));
    float n2;
    float3 g2;
    Field<FK>::eval(field_of<FK>(L, P), L.tab, p, L.s, n2, g2);
    const float3 d2 = f3(fmaf(L.hh, g2.x, d.x), fmaf(L.hh, g2.y, d.y), fmaf(L.hh, g2.z, d.z));
    ++L.steps;
    const float sacc = L.dist_acc + L.cur;
    // p - L > -eps and R - p > -eps per axis (as thresholds) and dist + h <= dlimit, as one chain of
    // predicate comparisons; a NaN coordinate fails it, as it fails the reference's test
    const bool ok = (p.x >= P.box_lo[0]) & (p.x <= P.box_hi[0]) & (p.y >= P.box_lo[1]) & (p.y <= P.box_hi[1]) &
                    (p.z >= P.box_lo[2]) & (p.z <= P.box_hi[2]) & (sacc <= L.dlimit);
    if (ok && L.steps < L.stop) {
        L.mp = p; L.md = d2; L.mn = n2; L.mg = g2;
        L.dist_acc = sacc;
        if (f64) L.mtot = fma(L.cur_d, double(n2), L.mtot);
        else L.mtotf = fmaf(L.cur, n2, L.mtotf);
        return false;
    }
    // A non-finite position fails the box test, so refinement ends the march within
    // `precision` steps; run_events checks finiteness when the march ends.
    if (L.steps >= P.step_cap) { L.end = SMP_END_STEP_CAP; return true; }
    if (ok) {                                     // accepted, and the loop count is exhausted
        L.mp = p; L.md = d2; L.mn = n2; L.mg = g2;
        L.dist_acc = sacc;
        if (f64) L.mtot = fma(L.cur_d, double(n2), L.mtot);
        else L.mtotf = fmaf(L.cur, n2, L.mtotf);
        return true;
    }
    if (--L.prec < 0) {                           // refinement exhausted: keep the failed step
        L.mp = p; L.md = d2; L.mn = n2; L.mg = g2;
        return true;
    }
    L.cur = step_tab<FK>(L, P)[P.precision - L.prec];   // restore (mp, md unchanged) and refine: cur / 10
    L.hh = 0.5f * L.cur;
    L.cur_d = double(L.cur);
    L.stop = min(L.steps + 10, P.step_cap);       // maxsteps = 11 from i = 0: ten more steps
    return false;
}

// ---- discrete logic between marches ---------------------------------------------------------
// Observation points for path replay (adjoint.cuh). The render kernels use NoHook, for which every
// hook call below is compiled out.
struct NoHook {
    static constexpr bool on = false;
    __device__ bool at(Lane &, int) { return false; }
    __device__ void splatted(const Lane &, float3, double, int, float) {}
    __device__ void photon_begin(const Lane &) {}
    __device__ void photon_end(const Lane &) {}
    __device__ void march_begin() {}
    __device__ void accepted() {}
};

// Runs the lane's events until it starts a march (returns ST_MARCH) or its photon ends
// (returns ST_FETCH). With a hook, h->at(L, ev) is asked at the entry of EV_SCATTER and
// EV_SCATTER_ONCE and at EV_VERTEX once the depth test has passed; true stops here with ST_HOOK
// (the lane state is that of the event's entry). h->splatted sees every splat.
template <int FK, class H = NoHook>
__device__ __forceinline__ int run_events(Lane &L, const KParams &P, int ev, H *h = nullptr) {
    for (;;) {
        if (ev == EV_MARCH_END) {
            if (!P.fp64) L.mtot = double(L.mtotf);
            if (L.end == 0 && !isfinite((L.mp.x + L.mp.y) + (L.mp.z + L.md.x) + (L.md.y + L.md.z) + L.mn))
                L.end = SMP_END_NAN;
        }
        if (ev != EV_FINISH && L.end != 0) {                    // aborted (cap, NaN, stream)
            if (ev == EV_MARCH_END) {
                if (L.ctx == CTX_MOVE_FIRST || L.ctx == CTX_MOVE_VERTEX) { L.pos = L.mp; L.dir = L.md; L.total = L.mtot; }
                else if (L.ctx == CTX_DIRECT) L.total = L.mtot;
            }
            ev = EV_FINISH;
        }
        switch (ev) {
        case EV_NEW: {
            L.total = 0.0;
            L.depth = 0; L.nspl = 0; L.draws = 0; L.steps = 0; L.end = 0;
            L.rblk = 0; L.rhave = 0;
            if (P.rng == SMP_RNG_STREAM) {
                long long k = L.idx - P.first_photon;
                L.spos = P.offsets[k];
                L.send = P.offsets[k + 1];
            }
            if (FK == FK_BATCH) {
                // sweep photon index -> (instance, the instance's photon index)
                int lo = 0, hi = P.n_inst;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (P.inst_first[mid] <= L.idx) lo = mid; else hi = mid;
                }
                L.inst = P.insts + lo;
                L.idx -= P.inst_first[lo];
                L.tab = L.inst->field.btab;
            }
            if (!gen_ray(L, P, L.pos, L.dir, L.total)) { L.end = SMP_END_GENRAY_FAIL; ev = EV_FINISH; break; }
            float u = draw(L, P);
            const FieldParams &F = field_of<FK>(L, P);
            if (FK == FK_PLANEWAVE) L.s = fmaf(F.phi_range, u, F.phi_min);
            else if (FK == FK_SOURCES) L.s = 0.0f;
            else {
                float sn, cs;
                sincos_red(F.phi_min + F.phi_range * u, sn, cs);
                L.s = fmaxf(fminf(sn, F.max_scaling), -F.max_scaling);
            }
            L.mp = L.pos;
            Field<FK>::eval(F, L.tab, L.mp, L.s, L.mn, L.mg);
            L.dir = mul(L.dir, L.mn);                     // photon.cpp:329
            if (P.use_direct) {
                L.ctx = CTX_DIRECT;
                L.md = L.dir;
                L.mtot = L.total;
                L.first = 1;
                L.large = med_large(L, P);
                begin_march<FK>(L, P, L.large, false);
                if (march_has_steps(L)) return ST_MARCH;
                ev = EV_MARCH_END;
            } else {
                ev = EV_SCATTER;
            }
            break;
        }
        case EV_MARCH_END: {
            const float disy = L.dist_acc;
            if (L.ctx == CTX_DIRECT || L.ctx == CTX_CONNECT) {
                // movePhotonTillSensor (scene.cpp:622-703)
                if (L.first) { L.d2s = disy; L.first = 0; } else { L.d2s += disy; }
                L.large -= disy;
                bool done = false, ok = false;
                if (L.large < 0.0f) { done = true; ok = false; }
                else {
                    float3 n = face_normal(P, L.mp);
                    if (fabsf(P.cam_dir[0] - n.x) < kEps && fabsf(P.cam_dir[1] - n.y) < kEps &&
                        fabsf(P.cam_dir[2] - n.z) < kEps) { done = true; ok = true; }
                    else {
                        float3 d1 = bsdf_sample(L, P, L.md, n);
                        if (dot3(d1, n) < 0.0f) {
                            L.md = d1;
                            begin_march<FK>(L, P, L.large, false);
                            if (march_has_steps(L)) return ST_MARCH;
                            ev = EV_MARCH_END;
                            break;
                        }
                        done = true; ok = false;
                    }
                }
                if (!done) break;
                if (L.ctx == CTX_DIRECT) {
                    // directTracing (photon.cpp:41-87); total is the photon's own
                    L.total = L.mtot;
                    if (ok) {
                        float3 d1 = normalized(L.md);
                        float ior = L.mn;
                        float3 refr = d1;
                        float fw = 1.0f;
                        if (ior > 1.0f) {
                            refr.x = refr.x / ior;
                            refr = normalized(refr);
                            fw = (1.0f - fresnel(d1.x, refr.x, 1.0f / ior)) / ior / ior;
                        }
                        float3 p1 = L.mp;
                        float dts = 0.0f;
                        if (propagate_till_sensor(P, p1, refr, dts)) {
                            acc_total(L.total, dts, P.fp64);
                            float val = med_weight(L, P) * expf(-med_sigma_t(L, P) * L.d2s) * fw;
                            splat(L, P, p1, L.total, 0, val);
                            if (H::on) h->splatted(L, p1, L.total, 0, val);
                        }
                    }
                    ev = EV_SCATTER;
                } else {
                    // addEnergyInParticle (scene.cpp:866-946); its path length is a copy
                    if (ok) {
                        float3 dsen = normalized(L.md);
                        float ior = L.mn;
                        float3 refr = dsen;
                        float fw = 1.0f;
                        if (ior > 1.0f) {
                            refr.x = refr.x / ior;
                            refr = normalized(refr);
                            fw = (1.0f - fresnel(dsen.x, refr.x, 1.0f / ior)) / ior / ior;
                        }
                        float fore = dot3(refr, ld3(P.cam_dir)) / dot3(dsen, ld3(P.cam_dir));
                        double tot = L.mtot;
                        float3 p1 = L.mp;
                        float dts = 0.0f;
                        if (propagate_till_sensor(P, p1, refr, dts)) {
                            acc_total(tot, dts, P.fp64);
                            float val = med_weight(L, P) * 6.28318548202514648f * expf(-med_sigma_t(L, P) * L.d2s) *
                                        hg_f(med_g(L, P), divs(L.dir, len3(L.dir)), dsen) * fore * fw;
                            splat(L, P, p1, tot, L.depth, val);
                            if (H::on) h->splatted(L, p1, tot, L.depth, val);
                        }
                    }
                    ev = EV_SCATTER_ONCE;
                }
            } else {
                // movePhoton (scene.cpp:706-780)
                L.rem -= disy;
                bool ok = true;
                if (L.rem > kEps) {
                    float3 n = face_normal(P, L.mp);
                    float mag = len3(L.md);
                    float3 d1 = bsdf_sample(L, P, divs(L.md, mag), n);
                    if (dot3(d1, n) < 0.0f) {
                        L.md = mul(d1, mag);
                        begin_march<FK>(L, P, L.rem, false);
                        if (march_has_steps(L)) return ST_MARCH;
                        ev = EV_MARCH_END;
                        break;
                    }
                    ok = false;
                }
                L.total = L.mtot;
                L.pos = L.mp;
                L.dir = L.md;
                if (!ok) { L.end = SMP_END_ESCAPED; ev = EV_FINISH; break; }
                if (L.ctx == CTX_MOVE_FIRST) { L.depth = 1; L.totalDist = L.sampled; }
                else ++L.depth;
                ev = EV_VERTEX;
            }
            break;
        }
        case EV_SCATTER: {
            if (H::on && h->at(L, EV_SCATTER)) return ST_HOOK;
            if (!roulette(L, P)) { L.end = SMP_END_NO_SCATTER; ev = EV_FINISH; break; }
            float dist = -med_mfp(L, P) * logf(draw(L, P));
            L.ctx = CTX_MOVE_FIRST;
            L.sampled = dist;
            L.rem = dist;
            L.mp = L.pos;
            L.md = L.dir;
            L.mtot = L.total;
            begin_march<FK>(L, P, dist, true);
            if (march_has_steps(L)) return ST_MARCH;
            ev = EV_MARCH_END;
            break;
        }
        case EV_VERTEX: {
            if (!((P.max_depth < 0 || L.depth <= P.max_depth) &&
                  (P.max_pathlength < 0.0f || L.totalDist <= P.max_pathlength))) {
                L.end = SMP_END_MAX_DEPTH; ev = EV_FINISH; break;
            }
            if (H::on && h->at(L, EV_VERTEX)) return ST_HOOK;
            if (P.use_angular && !(double(L.pos.x - P.cam_origin[0]) < 1e-4)) {
                float3 dts = random_direction(L, P);
                // mp == pos and (mn, mg) are the field at pos: the move march ended there
                L.md = mul(dts, L.mn);
                L.ctx = CTX_CONNECT;
                L.mtot = L.total;
                L.first = 1;
                L.large = med_large(L, P);
                begin_march<FK>(L, P, L.large, false);
                if (march_has_steps(L)) return ST_MARCH;
                ev = EV_MARCH_END;
                break;
            }
            ev = EV_SCATTER_ONCE;
            break;
        }
        case EV_SCATTER_ONCE: {
            if (H::on && h->at(L, EV_SCATTER_ONCE)) return ST_HOOK;
            if (!roulette(L, P)) { L.end = SMP_END_ABSORBED; ev = EV_FINISH; break; }
            float mag = len3(L.dir);
            float3 d1 = hg_sample(L, P, divs(L.dir, mag));
            L.dir = mul(d1, mag);
            float dist = -med_mfp(L, P) * logf(draw(L, P));
            L.ctx = CTX_MOVE_VERTEX;
            L.rem = dist;
            L.mp = L.pos;
            L.md = L.dir;
            L.mtot = L.total;
            begin_march<FK>(L, P, dist, true);
            if (march_has_steps(L)) return ST_MARCH;
            ev = EV_MARCH_END;
            break;
        }
        default: {   // EV_FINISH
            if (P.records) {
                smp_photon_record *rec = P.records + (L.idx - P.first_photon);
                rec->photon = L.idx;
                rec->end = L.end;
                rec->draws = L.draws;
                rec->depth = L.depth;
                rec->n_splats = L.nspl;
                rec->pos[0] = L.pos.x; rec->pos[1] = L.pos.y; rec->pos[2] = L.pos.z;
                rec->dir[0] = L.dir.x; rec->dir[1] = L.dir.y; rec->dir[2] = L.dir.z;
                rec->total_optical = L.total;
                rec->er_steps = L.steps;
            }
            return ST_FETCH;
        }
        }
    }
}

struct LaneStats {
    unsigned long long steps = 0, splats = 0, photons = 0, cap = 0, nan = 0, stream = 0;
};

template <int FK>
__device__ __forceinline__ void finish_photon_stats(const Lane &L, LaneStats &S) {
    S.steps += (unsigned long long)L.steps;
    S.splats += (unsigned long long)L.nspl;
    S.photons += 1;
    if (L.end == SMP_END_STEP_CAP) S.cap += 1;
    if (L.end == SMP_END_NAN) S.nan += 1;
    if (L.end == SMP_END_STREAM) S.stream += 1;
}

// ---- shared-memory staging with the Tensor Memory Accelerator ---------------------------------
// One elected thread issues a 1-D bulk copy (cp.async.bulk, no multicast) of `bytes` (a multiple of
// 16, both addresses 16-byte aligned) into this block's shared memory and the block waits on an
// mbarrier. Every wait is bounded: on timeout the block records the failure, waits (bounded) once
// more so no copy is left writing into its shared memory, and reports false.
__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity, int limit) {
    for (int it = 0; it < limit; ++it) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
static __device__ __noinline__ bool stage_to_shared(void *dst, const void *src, unsigned bytes, unsigned long long *err) {
    __shared__ __align__(8) unsigned long long bar;
    const unsigned b = smem_u32(&bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(b), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
            ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(b)
            : "memory");
    }
    bool ok = mbar_wait_bounded(b, 0, 1 << 22);
    if (!ok) {
        mbar_wait_bounded(b, 0, 1 << 22);
        if (threadIdx.x == 0) atomicAdd(err, 1ull);
    }
    __syncthreads();
    return __syncthreads_and(ok ? 1 : 0) != 0;
}

// The lane loop of the persistent kernel: event phase (lanes whose march ended, or that need a
// photon, run their discrete logic together until every live lane marches again; photons come
// from the global counter, one atomic per warp) alternating with the march phase (two ER steps per
// vote until event_batch lanes, scaled by the live lanes, wait for events). A lane enters with
// `st` = ST_FETCH (no photon) or ST_MARCH (a photon loaded mid-march). All 32 lanes call it.
// A hook (adjoint.cuh's checkpointing trace) also sees each photon's start and end; the render
// kernels use NoHook.
template <int FK, class H = NoHook>
__device__ __forceinline__ void lane_loop(Lane &L, int st, const KParams &P, LaneStats &S, int lane, H *h = nullptr) {
    int pending_ev = EV_NEW;
    for (;;) {
        for (;;) {
            unsigned need = __ballot_sync(kFull, st == ST_FETCH);
            if (need) {
                int leader = __ffs(need) - 1;
                unsigned long long base = 0;
                if (lane == leader) base = atomicAdd(P.counters + CNT_NEXT_PHOTON, (unsigned long long)__popc(need));
                base = __shfl_sync(kFull, base, leader);
                if (st == ST_FETCH) {
                    unsigned long long k = base + __popc(need & ((1u << lane) - 1u));
                    if (k < (unsigned long long)P.n_photons) {
                        L.idx = P.first_photon + (long long)k;
                        L.end = 0;                       // the previous photon's end code
                        st = ST_EVENT;
                        pending_ev = EV_NEW;
                        if (H::on) h->photon_begin(L);
                    } else {
                        st = ST_DONE;
                    }
                }
            }
            if (st == ST_EVENT) {
                st = run_events<FK, H>(L, P, pending_ev, h);
                if (st == ST_FETCH) {
                    finish_photon_stats<FK>(L, S);
                    if (H::on) h->photon_end(L);
                }
                if (H::on && st == ST_MARCH) h->march_begin();
            }
            if (!__any_sync(kFull, st == ST_FETCH)) break;
        }
        const unsigned alive = __ballot_sync(kFull, st != ST_DONE);
        if (alive == 0) break;
        const int thr = max(1, (P.event_batch * __popc(alive) + 16) >> 5);
        for (;;) {
            // two steps per vote; a lane whose march ends on the first skips the second
            if (!H::on) {
                if (st == ST_MARCH && (march_step<FK>(L, P) || march_step<FK>(L, P))) {
                    st = ST_EVENT;
                    pending_ev = EV_MARCH_END;
                }
            } else if (st == ST_MARCH) {
                // the same two steps, telling the hook which ones were accepted
                for (int t = 0; t < 2; ++t) {
                    const float3 q = L.mp;
                    const bool end = march_step<FK>(L, P);
                    if (q.x != L.mp.x || q.y != L.mp.y || q.z != L.mp.z) h->accepted();
                    if (end) { st = ST_EVENT; pending_ev = EV_MARCH_END; break; }
                }
            }
            const unsigned waiting = __ballot_sync(kFull, st == ST_EVENT);
            if (__popc(waiting) >= thr || !__any_sync(kFull, st == ST_MARCH)) break;
        }
    }
}

// warp-reduces the statistics, one atomic per warp per counter
__device__ __forceinline__ void flush_stats(LaneStats &S, const KParams &P, int lane) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        S.steps += __shfl_down_sync(kFull, S.steps, o);
        S.splats += __shfl_down_sync(kFull, S.splats, o);
        S.photons += __shfl_down_sync(kFull, S.photons, o);
        S.cap += __shfl_down_sync(kFull, S.cap, o);
        S.nan += __shfl_down_sync(kFull, S.nan, o);
        S.stream += __shfl_down_sync(kFull, S.stream, o);
    }
    if (lane == 0 && S.photons) {
        atomicAdd(P.counters + CNT_STEPS, S.steps);
        atomicAdd(P.counters + CNT_SPLATS, S.splats);
        atomicAdd(P.counters + CNT_PHOTONS, S.photons);
        if (S.cap) atomicAdd(P.counters + CNT_STEP_CAP, S.cap);
        if (S.nan) atomicAdd(P.counters + CNT_NAN, S.nan);
        if (S.stream) atomicAdd(P.counters + CNT_STREAM, S.stream);
    }
}

template <int FK>
__global__ void __launch_bounds__(128, SMP_MIN_BLOCKS) march_kernel(const __grid_constant__ KParams P) {
    extern __shared__ __align__(16) float4 smem_tab[];
    const int lane = threadIdx.x & 31;
    Lane L;
    L.end = 0;
    L.idx = 0;
    L.tab = P.field.btab;
    if (FK <= FK_BESSELN && P.field.btab != nullptr) {
        if (!stage_to_shared(smem_tab, P.field.btab, unsigned(P.field.bnodes) * 16u, P.counters + CNT_STAGE_TIMEOUT))
            return;                                  // whole block: other blocks take the photons
        L.tab = smem_tab;
    }
    LaneStats S;
    lane_loop<FK>(L, ST_FETCH, P, S, lane);
    flush_stats(S, P, lane);
}

// n(p), grad n(p) at host-given points with the march's own field code
template <int FK>
__global__ void field_probe_kernel(const __grid_constant__ FieldParams F, float s, long long n,
                                   const double *pts, double *n_out, double *g_out) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 p = f3(float(pts[3 * i]), float(pts[3 * i + 1]), float(pts[3 * i + 2]));
    float nn;
    float3 g;
    Field<FK>::eval(F, F.btab, p, s, nn, g);
    n_out[i] = nn;
    g_out[3 * i] = g.x; g_out[3 * i + 1] = g.y; g_out[3 * i + 2] = g.z;
}

}  // namespace smp
