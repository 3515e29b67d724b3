// dev_math.cuh -- device math for the photon march: float3 helpers with the reference vector
// semantics (renderer/include/tvector.h), a Cody-Waite 2*pi reduction, and FP32 Bessel J_m.
//
// Bessel functions J_m(x), m = 0..3, in single precision:
//   x <  3 : the power series J_m(x) = (x/2)^m sum_k (-(x/2)^2)^k / (k! (k+m)!), ten terms
//            (truncation < 1e-9 for x < 3);
//   x >= 3 : Abramowitz & Stegun, Handbook of Mathematical Functions, 9.4.3 and 9.4.6:
//            J_0 = x^-1/2 f_0 cos(theta_0), J_1 = x^-1/2 f_1 cos(theta_1) with the published
//            degree-6 polynomials in 3/x (|eps| <= 1.6e-8 / 7e-8 / 4e-8 / 9e-8), and the
//            upward three-term recurrence J_{n+1} = (2n/x) J_n - J_{n-1} for n + 1 <= 3 <= x.
//   theta_1 is evaluated as theta_0 - pi/2 + (P_1 - P_0), so one sincos serves both orders.
// The march itself reads J_m and J_{m+1} from a per-plan table (bessel_pair_table): for each
// interval [i h, (i+1) h) the cubic Hermite interpolant of (J, J') at its two nodes, as power-basis
// coefficients in f = x/h - i (computed on the host in double); two 16-byte shared-memory loads
// and six FMAs (Horner); the formulas above serve arguments beyond the table.
// The reference evaluates J_m with the double-precision libm jn (scene.cpp:214, :238-240);
// tests bound the absolute error of this code against it.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace smp {

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 mul(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len3(float3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// v / f as the reference divides vectors: one reciprocal, three products (tvector.h:292-297)
__device__ __forceinline__ float3 divs(float3 a, float f) { float r = 1.0f / f; return mul(a, r); }
// normalize() divides each component by the length (tvector.h:351-358)
__device__ __forceinline__ float3 normalized(float3 a) {
    if (a.x == 0.0f && a.y == 0.0f && a.z == 0.0f) return a;
    float l = len3(a);
    return f3(a.x / l, a.y / l, a.z / l);
}
__device__ __forceinline__ bool finite3(float3 a) {
    return isfinite(a.x) && isfinite(a.y) && isfinite(a.z);
}
// single hardware approximations (PTX rcp.approx.ftz / rsqrt.approx.ftz: <= 1 ulp / 2^-22.9
// relative error) for the inner march; the discrete logic keeps IEEE division
__device__ __forceinline__ float rcp_fast(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rsqrt_fast(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
// floor(t) and t - floor(t) for 0 <= t < 2^22 without integer conversions: adding 2^23 rounds t to
// an integer held in the low mantissa bits
__device__ __forceinline__ int floor_frac(float t, float &frac) {
    const float big = 8388608.0f;
    float tb = t + big;
    int i = __float_as_int(tb) - 0x4B000000;
    float fr = t - (tb - big);
    if (fr < 0.0f) { fr += 1.0f; i -= 1; }
    frac = fr;
    return i;
}
__device__ __forceinline__ float comp(float3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__device__ __forceinline__ float3 ld3(const float *v) { return f3(v[0], v[1], v[2]); }

// sin and cos of an argument of moderate size (|t| < 1e4): Cody-Waite reduction by 2*pi with a
// two-term split of 2*pi, then the hardware approximations on [-pi, pi].
__device__ __forceinline__ void sincos_red(float t, float &s, float &c) {
    const float kInv2Pi = 0.159154943091895335768f;
    const float k2PiHi = 6.28318548202514648438f;     // float(2*pi)
    const float k2PiLo = -1.74845553146951609e-07f;   // 2*pi - float(2*pi)
    float q = rintf(t * kInv2Pi);
    float r = fmaf(-q, k2PiHi, t);
    r = fmaf(-q, k2PiLo, r);
    __sincosf(r, &s, &c);
}

template <int M> struct BesselSeries;
template <> struct BesselSeries<0> {
    static __device__ __forceinline__ float sum(float q) {
        // c_k = 1/(k! k!)
        float s = 7.594058428e-12f;
        s = fmaf(s, q, 6.151187327e-10f); s = fmaf(s, q, 3.936759889e-08f);
        s = fmaf(s, q, 1.929012346e-06f); s = fmaf(s, q, 6.944444444e-05f);
        s = fmaf(s, q, 1.736111111e-03f); s = fmaf(s, q, 2.777777778e-02f);
        s = fmaf(s, q, 2.500000000e-01f); s = fmaf(s, q, 1.0f);
        return fmaf(s, q, 1.0f);
    }
};
template <> struct BesselSeries<1> {
    static __device__ __forceinline__ float sum(float q) {
        float s = 7.594058428e-13f;
        s = fmaf(s, q, 6.834652585e-11f); s = fmaf(s, q, 4.920949861e-09f);
        s = fmaf(s, q, 2.755731922e-07f); s = fmaf(s, q, 1.157407407e-05f);
        s = fmaf(s, q, 3.472222222e-04f); s = fmaf(s, q, 6.944444444e-03f);
        s = fmaf(s, q, 8.333333333e-02f); s = fmaf(s, q, 5.000000000e-01f);
        return fmaf(s, q, 1.0f);
    }
};
template <> struct BesselSeries<2> {
    static __device__ __forceinline__ float sum(float q) {
        float s = 6.903689480e-14f;
        s = fmaf(s, q, 6.834652585e-12f); s = fmaf(s, q, 5.467722068e-10f);
        s = fmaf(s, q, 3.444664903e-08f); s = fmaf(s, q, 1.653439153e-06f);
        s = fmaf(s, q, 5.787037037e-05f); s = fmaf(s, q, 1.388888889e-03f);
        s = fmaf(s, q, 2.083333333e-02f); s = fmaf(s, q, 1.666666667e-01f);
        return fmaf(s, q, 5.000000000e-01f);
    }
};
template <> struct BesselSeries<3> {
    static __device__ __forceinline__ float sum(float q) {
        float s = 5.753074567e-15f;
        s = fmaf(s, q, 6.213320532e-13f); s = fmaf(s, q, 5.467722068e-11f);
        s = fmaf(s, q, 3.827405448e-09f); s = fmaf(s, q, 2.066798942e-07f);
        s = fmaf(s, q, 8.267195767e-06f); s = fmaf(s, q, 2.314814815e-04f);
        s = fmaf(s, q, 4.166666667e-03f); s = fmaf(s, q, 4.166666667e-02f);
        return fmaf(s, q, 1.666666667e-01f);
    }
};

// J_m(x) for x < 3 from the series; q = -(x/2)^2, h = x/2
template <int M> __device__ __forceinline__ float bessel_small(float h, float q) {
    float hm = (M == 0) ? 1.0f : (M == 1 ? h : (M == 2 ? h * h : h * h * h));
    return hm * BesselSeries<M>::sum(q);
}

// J_0 and J_1 for x >= 3 (A&S 9.4.3, 9.4.6)
__device__ __forceinline__ void bessel01_large(float x, float &j0, float &j1) {
    float y = 3.0f * rcp_fast(x);
    float f0 = 0.00014476f;
    f0 = fmaf(f0, y, -0.00072805f); f0 = fmaf(f0, y, 0.00137237f); f0 = fmaf(f0, y, -0.00009512f);
    f0 = fmaf(f0, y, -0.00552740f); f0 = fmaf(f0, y, -0.00000077f); f0 = fmaf(f0, y, 0.79788456f);
    float p0 = 0.00013558f;
    p0 = fmaf(p0, y, -0.00029333f); p0 = fmaf(p0, y, -0.00054125f); p0 = fmaf(p0, y, 0.00262573f);
    p0 = fmaf(p0, y, -0.00003954f); p0 = fmaf(p0, y, -0.04166397f);
    p0 = p0 * y;                                   // theta_0 = x - 0.78539816 + p0
    float f1 = -0.00020033f;
    f1 = fmaf(f1, y, 0.00113653f); f1 = fmaf(f1, y, -0.00249511f); f1 = fmaf(f1, y, 0.00017105f);
    f1 = fmaf(f1, y, 0.01659667f); f1 = fmaf(f1, y, 0.00000156f); f1 = fmaf(f1, y, 0.79788456f);
    float p1 = -0.00029166f;
    p1 = fmaf(p1, y, 0.00079824f); p1 = fmaf(p1, y, 0.00074348f); p1 = fmaf(p1, y, -0.00637879f);
    p1 = fmaf(p1, y, 0.00005650f); p1 = fmaf(p1, y, 0.12499612f);
    p1 = p1 * y;                                   // theta_1 = x - 2.35619449 + p1
    float th0 = (x - 0.78539816f) + p0;
    float s0, c0;
    sincos_red(th0, s0, c0);
    // theta_1 = theta_0 - pi/2 + e, e = p1 - p0 (|e| < 0.17): cos(theta_1) = sin(theta_0 + e)
    float e = p1 - p0;
    float e2 = e * e;
    float ce = fmaf(e2, fmaf(e2, fmaf(e2, -1.0f / 720.0f, 1.0f / 24.0f), -0.5f), 1.0f);
    float se = e * fmaf(e2, fmaf(e2, fmaf(e2, -1.0f / 5040.0f, 1.0f / 120.0f), -1.0f / 6.0f), 1.0f);
    float c1 = fmaf(s0, ce, c0 * se);
    float rs = rsqrtf(x);
    j0 = rs * f0 * c0;
    j1 = rs * f1 * c1;
}

// (J_M(x), J_{M+1}(x)) for M in 0..2
template <int M> __device__ __forceinline__ void bessel_pair(float x, float &jm, float &jm1) {
    if (x < 3.0f) {
        float h = 0.5f * x;
        float q = -(h * h);
        jm = bessel_small<M>(h, q);
        jm1 = bessel_small<M + 1>(h, q);
    } else {
        float j0, j1;
        bessel01_large(x, j0, j1);
        if (M == 0) { jm = j0; jm1 = j1; return; }
        float ix = rcp_fast(x);
        float j2 = fmaf(2.0f * ix, j1, -j0);
        if (M == 1) { jm = j1; jm1 = j2; return; }
        float j3 = fmaf(4.0f * ix, j2, -j1);
        jm = j2; jm1 = j3;
    }
}

// (J_M, J_{M+1}) at x = t h from the per-plan table: entry 2i = the cubic of J_M on interval i,
// entry 2i+1 that of J_{M+1} (coefficients of 1, f, f^2, f^3); `intervals` intervals. floor(t) by a
// round-down add of 2^23, which leaves t - floor(t) exact. Beyond the table, A&S + recurrence.
template <int M>
__device__ __forceinline__ void bessel_pair_table_t(const float4 *tab, int intervals, float t, float x,
                                                    float &jm, float &jm1) {
    if (t < float(intervals)) {
        const float tb = __fadd_rd(t, 8388608.0f);
        const int i = __float_as_int(tb) - 0x4B000000;
        const float f = t - (tb - 8388608.0f);
        const float4 a = tab[2 * i], b = tab[2 * i + 1];
        jm = fmaf(fmaf(fmaf(a.w, f, a.z), f, a.y), f, a.x);
        jm1 = fmaf(fmaf(fmaf(b.w, f, b.z), f, b.y), f, b.x);
    } else {
        bessel_pair<M>(x, jm, jm1);
    }
}
template <int M>
__device__ __forceinline__ void bessel_pair_table(const float4 *tab, int intervals, float inv_h, float x,
                                                  float &jm, float &jm1) {
    bessel_pair_table_t<M>(tab, intervals, x * inv_h, x, jm, jm1);
}

}  // namespace smp
