// dev_field.cuh -- fused refractive-index evaluation: n(p) and grad n(p) in one call.
//
// The reference evaluates RIF and dRIF separately, twice per leapfrog step
// (renderer/src/scene.cpp:323-330) plus once more for the optical length (scene.cpp:416).
// All three evaluations after a step are at the same point p', and the next step starts at that
// point again, so the march keeps (n, grad n) of its current position and a step costs one
// fused evaluation.
//
// Gap gating (renderer/include/rif_base.h:104-137, cuda_scene.cuh:463-481): outside
// sgap <= x <= egap the index is n_o and the gradient zero.
#pragma once
#include "dev_math.cuh"
#include "kparams.h"

namespace smp {

static constexpr float kEps = 1.19209290e-07f;    // M_EPSILON (constants.h)

// Cylindrical Bessel mode about the -x axis (scene.cpp:206-257, fixed axes rif_base.h:146-148):
//   n = n_o + n_max*s*J_m(k r) cos(m phi),  phi = atan2(y, z), r = |(y, z)|
//   dn/dy = n_max*s*(J_m' k y/r cos(m phi) - J_m m sin(m phi) z/r^2)
//   dn/dz = n_max*s*(J_m' k z/r cos(m phi) + J_m m sin(m phi) y/r^2),  J_m' = (m/kr) J_m - J_{m+1}
// cos(m phi), sin(m phi) come from (z/r + i y/r)^m instead of atan2 + sincos.
// Below r = M_EPSILON the gradient uses y = z = r = M_EPSILON as the reference does.
template <int M>
__device__ __forceinline__ void bessel_field_ng(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) {
    float y = p.y, z = p.z;
    const float r2 = fmaf(y, y, z * z);
    float rs = rsqrt_fast(r2);                 // +inf at r2 = 0
    const float A = F.amp * s;
    float jm, jm1;
    if (r2 * rs >= kEps) {                     // off the axis (false for r2 = 0: 0 * inf is NaN)
        const float r = r2 * rs;
        bessel_pair_table_t<M>(tab, F.bint, F.kb * r, F.k_r * r, jm, jm1);
        if (M == 0) {
            // grad = A k J_0'(kr) (0, y, z)/r = -A k J_1(kr) (0, y, z)/r
            n = fmaf(A, jm, F.n_o);
            const float w = -(A * F.k_r) * jm1 * rs;
            g = f3(0.0f, w * y, w * z);
        } else if (M == 1) {
            // n = n_o + A J_1(kr) z/r; with J_1' = J_1/(kr) - J_2 the gradient reduces to
            // dn/dy = -A k J_2(kr) y z/r^2,  dn/dz = A J_1(kr)/r - A k J_2(kr) z^2/r^2
            const float aj = A * jm * rs;
            n = fmaf(aj, z, F.n_o);
            const float wz = (A * F.k_r) * jm1 * (rs * rs) * z;
            g = f3(0.0f, -wz * y, fmaf(-wz, z, aj));
        } else {
            const float c = z * rs, sn = y * rs;
            const float cm = fmaf(c, c, -sn * sn), sm = 2.0f * c * sn;
            n = fmaf(A * jm, cm, F.n_o);
            const float djm = fmaf(float(M) * F.inv_k * rs, jm, -jm1);
            const float a1 = A * djm * F.k_r * rs * cm;
            const float a2 = A * jm * float(M) * sm * rs * rs;
            g = f3(0.0f, fmaf(a1, y, -a2 * z), fmaf(a1, z, a2 * y));
        }
        return;
    }
    // on or next to the axis: the value at r, the gradient from y = z = r = M_EPSILON
    // (scene.cpp:229-234); at r = 0, phi = atan2(0, 0) = 0
    float r = r2 > 0.0f ? r2 * rs : 0.0f;
    float cm = 1.0f, sm = 0.0f;
    if (M > 0 && r2 > 0.0f) {
        const float c = z * rs, sn = y * rs;
        if (M == 1) { cm = c; sm = sn; }
        else { cm = fmaf(c, c, -sn * sn); sm = 2.0f * c * sn; }
    }
    bessel_pair_table<M>(tab, F.bint, F.binv_h, F.k_r * r, jm, jm1);
    n = fmaf(A * jm, cm, F.n_o);
    y = kEps; z = kEps; r = kEps; rs = 1.0f / kEps;
    bessel_pair_table<M>(tab, F.bint, F.binv_h, F.k_r * kEps, jm, jm1);
    // J_m'(kr) = (m/kr) J_m - J_{m+1}, with 1/(kr) = rs/k
    const float djm = (M == 0) ? -jm1 : fmaf(float(M) * F.inv_k * rs, jm, -jm1);
    const float a1 = A * djm * F.k_r * rs * cm;            // radial part / r
    const float a2 = (M == 0) ? 0.0f : A * jm * float(M) * sm * rs * rs;
    g = f3(0.0f, fmaf(a1, y, -a2 * z), fmaf(a1, z, a2 * y));
}

// gap gating (rif_base.h:104-137): n_o and no gradient outside sgap <= x <= egap
__device__ __forceinline__ bool in_gap(const FieldParams &F, float3 p) { return p.x > F.egap || p.x < F.sgap; }

// In the gaps the amplitude is zeroed instead of branching: n = n_o + 0 and grad n = 0 exactly,
// and every lane runs the same instructions.
template <int M>
__device__ __forceinline__ void bessel_field(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) {
    bessel_field_ng<M>(F, tab, p, in_gap(F, p) ? 0.0f : s, n, g);
}

// Plane waves (not in the reference): n = n_o + sum_i a_i sin(k_i.p - tau + phase_i)
__device__ __forceinline__ void wave_field_ng(const FieldParams &F, float3 p, float tau, float &n, float3 &g) {
    float acc = 0.0f;
    float3 gg = f3(0.0f, 0.0f, 0.0f);
    for (int i = 0; i < F.n_waves; ++i) {
        float ph = F.wk[i][0] * p.x + F.wk[i][1] * p.y + F.wk[i][2] * p.z - tau + F.wphase[i];
        float sn, cs;
        sincos_red(ph, sn, cs);
        acc = fmaf(F.wamp[i], sn, acc);
        float ac = F.wamp[i] * cs;
        gg.x = fmaf(ac, F.wk[i][0], gg.x);
        gg.y = fmaf(ac, F.wk[i][1], gg.y);
        gg.z = fmaf(ac, F.wk[i][2], gg.z);
    }
    n = F.n_o + acc;
    g = gg;
}

__device__ __forceinline__ void wave_field(const FieldParams &F, float3 p, float tau, float &n, float3 &g) {
    if (in_gap(F, p)) {
        n = F.n_o;
        g = f3(0.0f, 0.0f, 0.0f);
        return;
    }
    wave_field_ng(F, p, tau, n, g);
}

// Spherical point sources on two arcs (scene.cpp:139-195, rif_sources.h:156-198):
//   n = n_o + n_scaling * sum_c w_c sum_src cos(k r c + phase)/r,  w_c = 4(-1)^(c+1)/((c pi)^2 nsrc)
//   grad = n_scaling * sum_c w_c sum_src -(cos(k r c + ph) + k r c sin(k r c + ph))/r^3 (p - centre)
// All lanes of a warp read the same centre each iteration (broadcast loads through L1).
__device__ __forceinline__ void sources_field(const FieldParams &F, float3 p, float &n, float3 &g) {
    if (p.x > F.egap || p.x < F.sgap) {
        n = F.n_o;
        g = f3(0.0f, 0.0f, 0.0f);
        return;
    }
    float rif = 0.0f;
    float3 dn = f3(0.0f, 0.0f, 0.0f);
    const float pi = 3.14159265358979f;
    for (int c = 1; c <= F.n_coeff; ++c) {
        float sf = ((c & 1) ? 4.0f : -4.0f) / (float(c) * pi * float(c) * pi * float(F.nsources));
        float trif = 0.0f;
        float3 tdn = f3(0.0f, 0.0f, 0.0f);
        for (int arc = 0; arc < 2; ++arc) {
            if (!(arc == 0 ? F.active1 : F.active2)) continue;
            const float ph = arc == 0 ? F.phase1 : F.phase2;
            const float4 *cen = F.centers + arc * F.nsources;
            for (int k = 0; k < F.nsources; ++k) {
                float4 q = __ldg(cen + k);
                float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
                float rr2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                float ir = rsqrtf(rr2);
                float r = rr2 * ir;
                float krc = F.k_r * r * float(c);
                float sn, cs;
                sincos_red(krc + ph, sn, cs);
                trif = fmaf(cs, ir, trif);
                float ct = -fmaf(krc, sn, cs) * ir * ir * ir;
                tdn.x = fmaf(ct, dx, tdn.x);
                tdn.y = fmaf(ct, dy, tdn.y);
                tdn.z = fmaf(ct, dz, tdn.z);
            }
        }
        rif = fmaf(trif, sf, rif);
        dn = add(dn, mul(tdn, sf));
    }
    n = fmaf(F.n_scaling, rif, F.n_o);
    g = mul(dn, F.n_scaling);
}

// Tricubic B-spline (spline.h:33-62 kernels, :308-356 value/gradient) with the mirror rule of the
// reference's 1-D/2-D evaluators for taps outside the grid. The B-spline weights sum to 1 and
// their derivatives to 0, so the coefficients are stored as offsets from their mean:
// n = base + sum(delta w), grad n = sum(delta w'). Summing the raw coefficients (~1.33) in FP32,
// as the reference does, cancels about four digits of a 1e-3 gradient signal.
__device__ __forceinline__ int spline_wrap(int i, int n) {
    if (unsigned(i) < unsigned(n)) return i;     // inside the grid: the common case
    int m = 2 * n - 2;
    int w = i % m;
    if (w < 0) w += m;
    return w >= n ? m - w : w;
}
__device__ __forceinline__ void bspline_weights(float t, float w[4], float dw[4]) {
    // taps at floor(t)-1 .. floor(t)+2, offsets d = t - i in (1,2], (0,1], (-1,0], (-2,-1]
    float f = t - floorf(t);
    float f2 = f * f, f3v = f2 * f;
    float g = 1.0f - f;
    w[0] = g * g * g * (1.0f / 6.0f);
    w[1] = (2.0f / 3.0f) - f2 + 0.5f * f3v;
    w[2] = (2.0f / 3.0f) - g * g + 0.5f * g * g * g;
    w[3] = f3v * (1.0f / 6.0f);
    dw[0] = -0.5f * g * g;
    dw[1] = (1.5f * f - 2.0f) * f;
    dw[2] = -(1.5f * g - 2.0f) * g;
    dw[3] = 0.5f * f2;
}
// The march kernel of the slot pool stages one brick of the coefficient grid in shared memory (the
// x-tap quads of kSplineBrick^3 cells and their rows' one-cell apron below and two-cell apron above
// in y and z: kSplineBrick x (kSplineBrick + 3)^2 quads) and passes it as `brick`: entry 0 holds the
// brick's first cell (x, y, z) as ints and a valid flag, the quads follow, x fastest. A point whose
// 4x4x4 taps lie in the brick reads them there; any other point (and every kernel without a brick,
// brick == nullptr) reads the global quads. The values and sums are the same either way.
static constexpr int kSplineBrick = 16;
static constexpr int kSplineBrickRows = kSplineBrick + 3;
static constexpr int kSplineBrickQuads = kSplineBrick * kSplineBrickRows * kSplineBrickRows;

__device__ __forceinline__ void spline_field(const FieldParams &F, const float4 *brick, float3 p, float &n, float3 &g) {
    if (p.x > F.egap || p.x < F.sgap) {
        n = F.n_o;
        g = f3(0.0f, 0.0f, 0.0f);
        return;
    }
    float t[3] = {(p.x - F.xmin[0]) * F.xres[0], (p.y - F.xmin[1]) * F.xres[1], (p.z - F.xmin[2]) * F.xres[2]};
    float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
    bspline_weights(t[0], wx, dx);
    bspline_weights(t[1], wy, dy);
    bspline_weights(t[2], wz, dz);
    int ix[4], iy[4], iz[4];
    int bx = int(floorf(t[0])) - 1, by = int(floorf(t[1])) - 1, bz = int(floorf(t[2])) - 1;
    const int N0 = F.N[0], N1 = F.N[1], N2 = F.N[2];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        ix[a] = spline_wrap(bx + a, N0);
        iy[a] = spline_wrap(by + a, N1) * N0;
        iz[a] = spline_wrap(bz + a, N2) * N0 * N1;
    }
    float v = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
    // x-tap quads: one 16-byte load per row when floor(t_x) lies on the grid (same values, same
    // sums as the four single loads)
    const bool quad = F.coeff4 != nullptr && unsigned(bx + 1) < unsigned(N0);
    // the staged brick holds every tap when floor(t) lies in its cells on all three axes (and on
    // the grid)
    const float4 *bq = nullptr;
    if (brick != nullptr) {
        const int4 h = *reinterpret_cast<const int4 *>(brick);
        const int ox = bx + 1 - h.x, oy = by + 1 - h.y, oz = bz + 1 - h.z;
        if (h.w != 0 && unsigned(ox) < unsigned(kSplineBrick) && unsigned(oy) < unsigned(kSplineBrick) &&
            unsigned(oz) < unsigned(kSplineBrick) && unsigned(bx + 1) < unsigned(N0) && unsigned(by + 1) < unsigned(N1) &&
            unsigned(bz + 1) < unsigned(N2))
            bq = brick + 1 + (oz * kSplineBrickRows + oy) * kSplineBrick + ox;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            float r0, r1, r2, r3;
            if (bq != nullptr) {
                const float4 q = bq[(c * kSplineBrickRows + b) * kSplineBrick];
                r0 = q.x; r1 = q.y; r2 = q.z; r3 = q.w;
            } else if (quad) {
                const float4 q = __ldg(F.coeff4 + (iz[c] + iy[b] + bx + 1));
                r0 = q.x; r1 = q.y; r2 = q.z; r3 = q.w;
            } else {
                const float *row = F.coeff + iz[c] + iy[b];
                r0 = __ldg(row + ix[0]); r1 = __ldg(row + ix[1]); r2 = __ldg(row + ix[2]); r3 = __ldg(row + ix[3]);
            }
            float sv = r0 * wx[0] + r1 * wx[1] + r2 * wx[2] + r3 * wx[3];
            float sd = r0 * dx[0] + r1 * dx[1] + r2 * dx[2] + r3 * dx[3];
            float wyz = wy[b] * wz[c];
            v = fmaf(sv, wyz, v);
            gx = fmaf(sd, wyz, gx);
            gy = fmaf(sv, dy[b] * wz[c], gy);
            gz = fmaf(sv, wy[b] * dz[c], gz);
        }
    }
    n = F.spline_base + v;
    g = f3(gx * F.xres[0], gy * F.xres[1], gz * F.xres[2]);
}

// Field<FK>::eval(F, tab, p, s, n, g): tab is the Bessel table (shared memory in the march
// kernel), unused by the other kinds.
template <int FK> struct Field;
template <> struct Field<FK_BESSEL0> {
    static __device__ __forceinline__ void eval(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) { bessel_field<0>(F, tab, p, s, n, g); }
    static __device__ __forceinline__ void eval_ng(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) { bessel_field_ng<0>(F, tab, p, s, n, g); }
};
template <> struct Field<FK_BESSEL1> {
    static __device__ __forceinline__ void eval(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) { bessel_field<1>(F, tab, p, s, n, g); }
    static __device__ __forceinline__ void eval_ng(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) { bessel_field_ng<1>(F, tab, p, s, n, g); }
};
template <> struct Field<FK_BESSEL2> {
    static __device__ __forceinline__ void eval(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) { bessel_field<2>(F, tab, p, s, n, g); }
    static __device__ __forceinline__ void eval_ng(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) { bessel_field_ng<2>(F, tab, p, s, n, g); }
};
// Bessel mode m in 0..2 chosen at run time, one branch-free path for all orders (lanes of a warp
// may hold photons of different instances and orders): cos/sin(m phi) by selects from
// (z + iy)/r, J_m' = (m/kr) J_m - J_{m+1}; beyond the table the order-specific formulas.
__device__ __forceinline__ void bessel_field_rt(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) {
    const int M = F.mode;
    const float A = F.amp * (in_gap(F, p) ? 0.0f : s);
    float y = p.y, z = p.z;
    const float r2 = fmaf(y, y, z * z);
    float rs = rsqrt_fast(r2);                 // +inf at r2 = 0
    float r = r2 > 0.0f ? r2 * rs : 0.0f;
    float cm = 1.0f, sm = 0.0f;
    if (r2 > 0.0f) {
        const float c = z * rs, sn = y * rs;
        cm = M == 0 ? 1.0f : (M == 1 ? c : fmaf(c, c, -sn * sn));
        sm = M == 0 ? 0.0f : (M == 1 ? sn : 2.0f * c * sn);
    }
    float jm, jm1;
    const float t = F.kb * r;
    if (t < float(F.bint)) {
        const float tb = __fadd_rd(t, 8388608.0f);
        const int i = __float_as_int(tb) - 0x4B000000;
        const float f = t - (tb - 8388608.0f);
        const float4 a = tab[2 * i], b = tab[2 * i + 1];
        jm = fmaf(fmaf(fmaf(a.w, f, a.z), f, a.y), f, a.x);
        jm1 = fmaf(fmaf(fmaf(b.w, f, b.z), f, b.y), f, b.x);
    } else if (M == 0) {
        bessel_pair<0>(F.k_r * r, jm, jm1);
    } else if (M == 1) {
        bessel_pair<1>(F.k_r * r, jm, jm1);
    } else {
        bessel_pair<2>(F.k_r * r, jm, jm1);
    }
    n = fmaf(A * jm, cm, F.n_o);
    if (!(r >= kEps)) {                        // the gradient's near-axis substitution (scene.cpp:229-234)
        y = kEps; z = kEps; r = kEps; rs = 1.0f / kEps;
        if (M == 0) bessel_pair_table<0>(tab, F.bint, F.binv_h, F.k_r * kEps, jm, jm1);
        else if (M == 1) bessel_pair_table<1>(tab, F.bint, F.binv_h, F.k_r * kEps, jm, jm1);
        else bessel_pair_table<2>(tab, F.bint, F.binv_h, F.k_r * kEps, jm, jm1);
    }
    const float fm = float(M);
    const float djm = fmaf(fm * F.inv_k * rs, jm, -jm1);
    const float a1 = A * djm * F.k_r * rs * cm;
    const float a2 = A * jm * fm * sm * rs * rs;
    g = f3(0.0f, fmaf(a1, y, -a2 * z), fmaf(a1, z, a2 * y));
}

// Bessel mode m >= 3 (scene.cpp:206-257 take any integer order through jn(mode, .)): J_m and J_m+1
// from the per-plan table, which the host sizes to cover the whole box (k r <= 128, checked when the
// plan is made; a point beyond it reads the table's last interval); cos(m phi), sin(m phi) as
// ((z + i y)/r)^m by m - 1 complex products.
__device__ __forceinline__ void bessel_field_n(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) {
    const int M = F.mode;
    const float A = F.amp * (in_gap(F, p) ? 0.0f : s);
    float y = p.y, z = p.z;
    const float r2 = fmaf(y, y, z * z);
    float rs = rsqrt_fast(r2);                 // +inf at r2 = 0
    float r = r2 > 0.0f ? r2 * rs : 0.0f;
    float cm = 1.0f, sm = 0.0f;
    if (r2 > 0.0f) {
        const float c = z * rs, sn = y * rs;
        cm = c; sm = sn;
        for (int k = 1; k < M; ++k) {
            const float t = fmaf(cm, c, -sm * sn);
            sm = fmaf(cm, sn, sm * c);
            cm = t;
        }
    }
    auto lookup = [&](float x, float &jm, float &jm1) {
        float t = fminf(x * F.binv_h, float(F.bint) - 1.0f / 64.0f);
        const float tb = __fadd_rd(t, 8388608.0f);
        const int i = __float_as_int(tb) - 0x4B000000;
        const float f = t - (tb - 8388608.0f);
        const float4 a = tab[2 * i], b = tab[2 * i + 1];
        jm = fmaf(fmaf(fmaf(a.w, f, a.z), f, a.y), f, a.x);
        jm1 = fmaf(fmaf(fmaf(b.w, f, b.z), f, b.y), f, b.x);
    };
    float jm, jm1;
    lookup(F.k_r * r, jm, jm1);
    n = fmaf(A * jm, cm, F.n_o);
    if (!(r >= kEps)) {                        // the gradient's near-axis substitution (scene.cpp:229-234)
        y = kEps; z = kEps; r = kEps; rs = 1.0f / kEps;
        lookup(F.k_r * kEps, jm, jm1);
    }
    const float fm = float(M);
    const float djm = fmaf(fm * F.inv_k * rs, jm, -jm1);
    const float a1 = A * djm * F.k_r * rs * cm;
    const float a2 = A * jm * fm * sm * rs * rs;
    g = f3(0.0f, fmaf(a1, y, -a2 * z), fmaf(a1, z, a2 * y));
}
template <> struct Field<FK_BESSELN> {
    static __device__ __forceinline__ void eval(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) {
        bessel_field_n(F, tab, p, s, n, g);
    }
    static __device__ __forceinline__ void eval_ng(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) {
        bessel_field_n(F, tab, p, s, n, g);
    }
};

// batched sweep: the instance's Bessel field
template <> struct Field<FK_BATCH> {
    static __device__ __forceinline__ void eval(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) {
        bessel_field_rt(F, tab, p, s, n, g);
    }
    static __device__ __forceinline__ void eval_ng(const FieldParams &F, const float4 *tab, float3 p, float s, float &n, float3 &g) {
        bessel_field_rt(F, tab, p, s, n, g);
    }
};
template <> struct Field<FK_PLANEWAVE> {
    static __device__ __forceinline__ void eval(const FieldParams &F, const float4 *, float3 p, float s, float &n, float3 &g) { wave_field(F, p, s, n, g); }
    static __device__ __forceinline__ void eval_ng(const FieldParams &F, const float4 *, float3 p, float s, float &n, float3 &g) { wave_field_ng(F, p, s, n, g); }
};
template <> struct Field<FK_SOURCES> {
    static __device__ __forceinline__ void eval(const FieldParams &F, const float4 *, float3 p, float, float &n, float3 &g) { sources_field(F, p, n, g); }
    static __device__ __forceinline__ void eval_ng(const FieldParams &F, const float4 *, float3 p, float, float &n, float3 &g) { sources_field(F, p, n, g); }
};
// the spline's `tab` argument is the staged brick of the slot pool's march kernel (or nullptr)
template <> struct Field<FK_SPLINE> {
    static __device__ __forceinline__ void eval(const FieldParams &F, const float4 *brick, float3 p, float, float &n, float3 &g) { spline_field(F, brick, p, n, g); }
    static __device__ __forceinline__ void eval_ng(const FieldParams &F, const float4 *brick, float3 p, float, float &n, float3 &g) { spline_field(F, brick, p, n, g); }
};

}  // namespace smp
