// adjoint.cuh -- reverse-mode derivative of a render's sensor objective with respect to the
// refractive-index field's parameters (Bessel amplitude and phase window, plane-wave amplitudes and phases,
// spline coefficients).
//
// Objective: J = sum_pixels G[pixel] * film[pixel] for a caller-given weight image G (dJ/dfilm;
// a region-of-interest mask gives ROI throughput). The film is the render's own estimator
// (Philox streams keyed by photon index), so J and its gradient are per-photon sums and the
// gradient is the pathwise derivative of exactly the estimator the forward render evaluates on
// the same seed: random numbers, discrete choices (roulette, Fresnel reflect/refract, texel,
// z bin) and the ER step sequence of every march are held fixed, and the continuous chain
//
//   source -> n(p0) omega0 -> [march] -> vertex 1 -> [connection march] -> sensor splat
//                                     \-> HG rotation -> [march] -> vertex 2 -> ...
//
// is differentiated. Marches that end on a face are differentiated as ending ON the face: the
// end point moves along the ray to the face plane (the implicit crossing of the continuous
// path), which shifts the arc length (exp(-sigma_t d) of connections; the remaining distance of
// a move after a reflection).
//
// Path replay with checkpointed scatter vertices, in batches of photons, three kernels per batch:
//   adjoint_trace_kernel   traces every photon with the render's own lane loop (march.cuh) and a
//            hook that records a checkpoint at the source and at every scatter vertex: position,
//            optical direction, path length, step count and the Philox draw index (draw k of
//            photon i is a pure function of (seed, i, k), so any segment can be replayed from its
//            checkpoint); it marks the splats that reach dJ/dfilm and counts the trajectory
//            entries of every segment the backward pass will need;
//   adjoint_replay_kernel  replays those segments forward from their checkpoints, writing each
//            accepted ER step's position and step size to the trajectory buffer (rounds: photons
//            that do not fit wait for the next one);
//   adjoint_sweep_kernel   (adjoint_sweep.cu) walks each photon's vertices backwards and sweeps
//            every recorded segment with the adjoint of kick-drift-kick (scene.cpp:323-330)
//              dh = d + h/2 g(p),  p' = p + dh h/n(p),  d' = dh + h/2 g(p')
//            which needs n, grad n and the Hessian of n at every point, and accumulates dJ/dtheta
//            through dn/dtheta and dgrad n/dtheta at every point.
// The splat's value (Fresnel exit, foreshortening, Henyey-Greenstein, exp(-sigma_t d), bilinear
// weights) and the HG frame rotation at a vertex are differentiated with forward-mode dual numbers.
#pragma once
#include "dispatch.h"
#include "march.cuh"
#include "wavefront.cuh"

namespace smp {

// ---- forward-mode dual numbers (event-level functions of a few inputs) -----------------------
template <int N> struct Dual {
    float v;
    float d[N];
};
template <int N> __device__ __forceinline__ Dual<N> dc(float v) {
    Dual<N> r; r.v = v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = 0.0f;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> dvar(float v, int i) { Dual<N> r = dc<N>(v); r.d[i] = 1.0f; return r; }
template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r; r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r; r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r; r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(const Dual<N> &a, float s) {
    Dual<N> r; r.v = a.v * s;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * s;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(float s, const Dual<N> &a) { return a * s; }
template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N> &a, float s) { Dual<N> r = a; r.v += s; return r; }
template <int N> __device__ __forceinline__ Dual<N> operator+(float s, const Dual<N> &a) { return a + s; }
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N> &a, float s) { Dual<N> r = a; r.v -= s; return r; }
template <int N> __device__ __forceinline__ Dual<N> operator-(float s, const Dual<N> &a) {
    Dual<N> r; r.v = s - a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r; r.v = a.v / b.v;
    const float ib = 1.0f / b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N> &a, float s) {
    Dual<N> r; r.v = a.v / s;
    const float is = 1.0f / s;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * is;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator/(float s, const Dual<N> &b) {
    Dual<N> r; r.v = s / b.v;
    const float k = -r.v / b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = b.d[i] * k;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> dsqrt(const Dual<N> &a) {
    Dual<N> r; r.v = sqrtf(a.v);
    const float h = 0.5f / r.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * h;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> dexp(const Dual<N> &a) {
    Dual<N> r; r.v = expf(a.v);
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * r.v;
    return r;
}

// ---- device-side parameters of an adjoint launch -----------------------------------------------
struct AdjVertex {             // a checkpoint (source: index 0, scatter vertex k: index k)
    float pos[3], dir[3];      // photon position and optical direction v = n omega
    float total_dist;          // first sampled distance (maxPathlength test)
    int depth;
    int draws_v, steps_v;      // Philox draw index and ER-step count at EV_VERTEX (after its depth test)
    int draws_so, steps_so;    // the same at EV_SCATTER_ONCE (source: at EV_SCATTER)
    int hits;                  // the splat that follows lands where dJ/dfilm is nonzero: bit 0 the
                               // connection from this vertex, bit 1 (source) the direct splat
    int len_in;                // trajectory entries of the move into this vertex (source: the direct march)
    int len_conn;              // trajectory entries of the connection from this vertex
    int pad;
    double total;              // optical path length
};

enum AdjCounter : int {
    ADJ_NEXT = 0,          // work distribution
    ADJ_PHOTONS = 1,       // photons differentiated
    ADJ_DROPPED = 2,       // photons left out: more vertices than checkpoints, pool or trajectory buffer full
    ADJ_ABORTED = 3,       // photons left out: step cap or non-finite state in the forward trace
    ADJ_MISMATCH = 4,      // replays whose end state differed from the checkpoint (a defect)
    ADJ_RESERVED = 5,      // (the trace counts its ER steps in KParams.counters)
    ADJ_STEPS_REPLAY = 6,  // er_step evaluations of the replays
    ADJ_POINTS = 7,        // trajectory points swept backwards
    ADJ_SPLATS = 8,        // splats differentiated
    ADJ_SKIPPED = 9,       // segments left out of the sweep: a malformed or truncated record
    ADJ_COUNT = 10
};

// One photon's result of the checkpointing trace, and where its replayed segments go.
enum AdjStatus : int { PH_OK = 0, PH_ABORTED = 1, PH_DROPPED = 2 };
struct AdjPhoton {
    int off, nv;               // its checkpoints: pool[off .. off + nv), source first
    int status;                // AdjStatus
    int hits;                  // bit 0: some connection splat reaches dJ/dfilm, bit 1: the direct one
    float s;                   // its temporal scaling / phase draw
    int tlen;                  // trajectory entries its needed segments can take (an upper bound)
    int round;                 // replay round that took it (0: not yet)
    int last;                  // the last vertex whose connection reaches dJ/dfilm (0: none)
    long long toff;            // its trajectory entries: traj[toff .. toff + tlen)
    long long pad;
};

// A replayed segment. Segment c of a photon (c = 0 the direct march, 2k - 1 the move into vertex k,
// 2k the connection from vertex k) is segs[2 * off + c].
struct AdjSeg {
    long long off;             // trajectory entries traj[off .. off + len)
    int len;
    int ok;                    // the replay reproduced its checkpoint and, for a sensor march, splatted
    float mp[3], md[3];        // end position and direction
    float mn, d2s;             // n at the end, the marched distance (sensor marches)
    float dir[3];              // the photon direction at the end (the vertex direction of a connection)
    float md0[3];              // start direction
    float sp[3];               // splat point, path length and depth (sensor marches)
    int sdepth;
    double spl;
};

struct AdjParams {
    int X, Y, Z;               // film shape (KParams.X is 0 in an adjoint launch: replays splat nothing)
    const double *G;           // dJ/dfilm, X*Y*Z, Image3 layout
    float4 *traj;              // replayed trajectories, segment after segment: (position, step size);
                               // step size 0 = segment start, -1 = a face reflection between marches
    long long traj_cap;
    unsigned long long *traj_next;
    AdjSeg *segs;              // 2 * pool_cap entries
    int *pending;              // a replay round left photons for the next round
    AdjVertex *tverts;         // checkpointing trace: [slots][vcap] checkpoints of each slot's photon
    int4 *tstate;              // per slot: checkpoints so far, flags (bit 0 overflow, bit 1 the direct
                               // splat reaches dJ/dfilm), trajectory entries of the current segment,
                               // the ER-step count at the start of the slot's current march
    int vcap;
    AdjVertex *pool;           // the batch's checkpoints, photon after photon
    long long pool_cap;
    unsigned long long *pool_next;
    AdjPhoton *photons;        // per photon of the batch
    int *order;                // the photons the replays and sweeps take, longest trajectory first
                               // (adjoint_order_*), so that a warp's lanes carry similar lengths
    unsigned *obucket;         // kOrderBuckets counters of the ordering
    unsigned long long *n_order;   // entries of `order`
    int idle_replay, idle_sweep;   // a warp leaves its march / sweep loop for discrete work once this
                                   // many 32nds of its live lanes wait
    double *grad;              // dJ/dtheta (layout per field kind, see FieldAdj)
    unsigned long long *cnt;   // AdjCounter
};

// Position the lane's Philox stream at draw index d (draw k uses word k % 4 of block k / 4).
__device__ __forceinline__ void rng_seek(Lane &L, const KParams &P, int d) {
    L.rblk = unsigned(d >> 2);
    L.rhave = 0;
    L.draws = d & ~3;
    for (int i = 0; i < (d & 3); ++i) (void)draw(L, P);
}

// ---- field: n, grad n, Hessian, and the parameter vector-Jacobian product -------------------------
// H = (xx, yy, zz, xy, xz, yz).
__device__ __forceinline__ float3 hmul(const float H[6], float3 b) {
    return f3(H[0] * b.x + H[3] * b.y + H[4] * b.z,
              H[3] * b.x + H[1] * b.y + H[5] * b.z,
              H[4] * b.x + H[5] * b.y + H[2] * b.z);
}

template <int FK> struct FieldAdj;

// Plane waves n = n_o + sum_i a_i sin(k_i.p - tau + phase_i):
//   grad n = sum_i a_i cos(.) k_i,  H = -sum_i a_i sin(.) k_i k_i^T,
//   dJ/da_i += a sin + cos (k_i.b),  dJ/dphase_i += a a_i cos - a_i sin (k_i.b)
// for the cotangent (a, b) of (n, grad n). Gradient layout: a_0..a_{W-1}, phase_0..phase_{W-1}.
// NW: the largest wave count the instance handles (its accumulators and caches live in registers)
template <int NW> struct FieldAdjPW {
    struct Acc { float ga[NW], gp[NW]; };
    struct Cache { float sn[NW], cs[NW]; int gap; };   // eval_h -> theta_c at one point
    static __device__ __forceinline__ void begin(Acc &, Lane &, const KParams &, float) {}
    static __device__ __forceinline__ void clear(Acc &c) {
#pragma unroll
        for (int i = 0; i < NW; ++i) { c.ga[i] = 0.0f; c.gp[i] = 0.0f; }
    }
    static __device__ __forceinline__ void eval_h(const FieldParams &F, float3 p, float tau, float &n, float3 &g, float H[6]) {
#pragma unroll
        for (int j = 0; j < 6; ++j) H[j] = 0.0f;
        n = F.n_o;
        g = f3(0.0f, 0.0f, 0.0f);
        if (in_gap(F, p)) return;
#pragma unroll
        for (int i = 0; i < NW; ++i) {
            if (i < F.n_waves) {
                const float kx = F.wk[i][0], ky = F.wk[i][1], kz = F.wk[i][2];
                float sn, cs;
                sincos_red(kx * p.x + ky * p.y + kz * p.z - tau + F.wphase[i], sn, cs);
                n += F.wamp[i] * sn;
                const float ac = F.wamp[i] * cs, as = -F.wamp[i] * sn;
                g.x += ac * kx; g.y += ac * ky; g.z += ac * kz;
                H[0] += as * kx * kx; H[1] += as * ky * ky; H[2] += as * kz * kz;
                H[3] += as * kx * ky; H[4] += as * kx * kz; H[5] += as * ky * kz;
            }
        }
    }
    static __device__ __forceinline__ void theta(const FieldParams &F, float3 p, float tau, float a, float3 b, Acc &c, const AdjParams &) {
        if (in_gap(F, p)) return;
#pragma unroll
        for (int i = 0; i < NW; ++i) {
            if (i < F.n_waves) {
                const float kx = F.wk[i][0], ky = F.wk[i][1], kz = F.wk[i][2];
                float sn, cs;
                sincos_red(kx * p.x + ky * p.y + kz * p.z - tau + F.wphase[i], sn, cs);
                const float kb = kx * b.x + ky * b.y + kz * b.z;
                c.ga[i] += a * sn + cs * kb;
                c.gp[i] += F.wamp[i] * (a * cs - sn * kb);
            }
        }
    }
    // the same pair with the sines and cosines computed once
    static __device__ __forceinline__ void eval_h(const FieldParams &F, float3 p, float tau, float &n, float3 &g, float H[6],
                                                  Cache &k) {
#pragma unroll
        for (int j = 0; j < 6; ++j) H[j] = 0.0f;
        n = F.n_o;
        g = f3(0.0f, 0.0f, 0.0f);
        k.gap = in_gap(F, p);
        if (k.gap) return;
#pragma unroll
        for (int i = 0; i < NW; ++i) {
            if (i < F.n_waves) {
                const float kx = F.wk[i][0], ky = F.wk[i][1], kz = F.wk[i][2];
                float sn, cs;
                sincos_red(kx * p.x + ky * p.y + kz * p.z - tau + F.wphase[i], sn, cs);
                k.sn[i] = sn; k.cs[i] = cs;
                n += F.wamp[i] * sn;
                const float ac = F.wamp[i] * cs, as = -F.wamp[i] * sn;
                g.x += ac * kx; g.y += ac * ky; g.z += ac * kz;
                H[0] += as * kx * kx; H[1] += as * ky * ky; H[2] += as * kz * kz;
                H[3] += as * kx * ky; H[4] += as * kx * kz; H[5] += as * ky * kz;
            }
        }
    }
    static __device__ __forceinline__ void theta_c(const FieldParams &F, float3, float, float a, float3 b, Acc &c,
                                                   const AdjParams &, const Cache &k) {
        if (k.gap) return;
#pragma unroll
        for (int i = 0; i < NW; ++i) {
            if (i < F.n_waves) {
                const float kb = F.wk[i][0] * b.x + F.wk[i][1] * b.y + F.wk[i][2] * b.z;
                c.ga[i] += a * k.sn[i] + k.cs[i] * kb;
                c.gp[i] += F.wamp[i] * (a * k.cs[i] - k.sn[i] * kb);
            }
        }
    }
    static __device__ __forceinline__ void flush(const Acc &c, const FieldParams &F, const AdjParams &A) {
#pragma unroll
        for (int i = 0; i < NW; ++i) {
            if (i < F.n_waves) {
                atomicAdd(A.grad + i, double(c.ga[i]));
                atomicAdd(A.grad + F.n_waves + i, double(c.gp[i]));
            }
        }
    }
};

template <> struct FieldAdj<FK_PLANEWAVE> : FieldAdjPW<SMP_MAX_WAVES> {};

// Tricubic B-spline n = sum_taps c w_x w_y w_z (the coefficient mean is stored apart, which is the
// same function because the weights sum to 1). dJ/dc for each of the 64 taps is
// a W + b . grad W, scattered with double atomics into the N0 x N1 x N2 gradient grid (taps outside
// the grid land on their mirrored coefficient, as they are read). B-spline second-derivative
// weights: (1 - f, 3f - 2, 1 - 3f, f).
__device__ __forceinline__ void bspline_dd(float t, float dd[4]) {
    float f = t - floorf(t);
    dd[0] = 1.0f - f;
    dd[1] = 3.0f * f - 2.0f;
    dd[2] = 1.0f - 3.0f * f;
    dd[3] = f;
}
template <> struct FieldAdj<FK_SPLINE> {
    struct Acc {};
    struct Cache {};
    static __device__ __forceinline__ void begin(Acc &, Lane &, const KParams &, float) {}
    static __device__ __forceinline__ void clear(Acc &) {}
    static __device__ __forceinline__ void taps(const FieldParams &F, float3 p, float wx[4], float wy[4], float wz[4],
                                                float dx[4], float dy[4], float dz[4], float ddx[4], float ddy[4],
                                                float ddz[4], int ix[4], int iy[4], int iz[4]) {
        const float t0 = (p.x - F.xmin[0]) * F.xres[0], t1 = (p.y - F.xmin[1]) * F.xres[1], t2 = (p.z - F.xmin[2]) * F.xres[2];
        bspline_weights(t0, wx, dx);
        bspline_weights(t1, wy, dy);
        bspline_weights(t2, wz, dz);
        bspline_dd(t0, ddx);
        bspline_dd(t1, ddy);
        bspline_dd(t2, ddz);
        const int bx = int(floorf(t0)) - 1, by = int(floorf(t1)) - 1, bz = int(floorf(t2)) - 1;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            ix[q] = spline_wrap(bx + q, F.N[0]);
            iy[q] = spline_wrap(by + q, F.N[1]) * F.N[0];
            iz[q] = spline_wrap(bz + q, F.N[2]) * F.N[0] * F.N[1];
        }
    }
    static __device__ __forceinline__ void eval_h(const FieldParams &F, float3 p, float, float &n, float3 &g, float H[6]) {
#pragma unroll
        for (int j = 0; j < 6; ++j) H[j] = 0.0f;
        if (in_gap(F, p)) { n = F.n_o; g = f3(0.0f, 0.0f, 0.0f); return; }
        float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4], ddx[4], ddy[4], ddz[4];
        int ix[4], iy[4], iz[4];
        taps(F, p, wx, wy, wz, dx, dy, dz, ddx, ddy, ddz, ix, iy, iz);
        float v = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
        float hxx = 0.0f, hyy = 0.0f, hzz = 0.0f, hxy = 0.0f, hxz = 0.0f, hyz = 0.0f;
        const int fx = int(floorf((p.x - F.xmin[0]) * F.xres[0]));
        const bool quad = F.coeff4 != nullptr && unsigned(fx) < unsigned(F.N[0]);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                float r0, r1, r2, r3;
                if (quad) {
                    const float4 q = __ldg(F.coeff4 + (iz[c] + iy[b] + fx));
                    r0 = q.x; r1 = q.y; r2 = q.z; r3 = q.w;
                } else {
                    const float *row = F.coeff + iz[c] + iy[b];
                    r0 = __ldg(row + ix[0]); r1 = __ldg(row + ix[1]); r2 = __ldg(row + ix[2]); r3 = __ldg(row + ix[3]);
                }
                const float sv = r0 * wx[0] + r1 * wx[1] + r2 * wx[2] + r3 * wx[3];
                const float sd = r0 * dx[0] + r1 * dx[1] + r2 * dx[2] + r3 * dx[3];
                const float sdd = r0 * ddx[0] + r1 * ddx[1] + r2 * ddx[2] + r3 * ddx[3];
                const float yz = wy[b] * wz[c], dyz = dy[b] * wz[c], ydz = wy[b] * dz[c];
                v += sv * yz;
                gx += sd * yz; gy += sv * dyz; gz += sv * ydz;
                hxx += sdd * yz; hyy += sv * ddy[b] * wz[c]; hzz += sv * wy[b] * ddz[c];
                hxy += sd * dyz; hxz += sd * ydz; hyz += sv * dy[b] * dz[c];
            }
        }
        const float r0 = F.xres[0], r1 = F.xres[1], r2 = F.xres[2];
        n = F.spline_base + v;
        g = f3(gx * r0, gy * r1, gz * r2);
        H[0] = hxx * r0 * r0; H[1] = hyy * r1 * r1; H[2] = hzz * r2 * r2;
        H[3] = hxy * r0 * r1; H[4] = hxz * r0 * r2; H[5] = hyz * r1 * r2;
    }
    static __device__ __forceinline__ void theta(const FieldParams &F, float3 p, float, float a, float3 b, Acc &, const AdjParams &A) {
        if (in_gap(F, p)) return;
        float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4], ddx[4], ddy[4], ddz[4];
        int ix[4], iy[4], iz[4];
        taps(F, p, wx, wy, wz, dx, dy, dz, ddx, ddy, ddz, ix, iy, iz);
        const float bx = b.x * F.xres[0], by = b.y * F.xres[1], bz = b.z * F.xres[2];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float ar = a * wy[q] * wz[c] + by * dy[q] * wz[c] + bz * wy[q] * dz[c];
                const float br = bx * wy[q] * wz[c];
                double *row = A.grad + iz[c] + iy[q];
#pragma unroll
                for (int i = 0; i < 4; ++i) atomicAdd(row + ix[i], double(ar * wx[i] + br * dx[i]));
            }
        }
    }
    static __device__ __forceinline__ void eval_h(const FieldParams &F, float3 p, float s, float &n, float3 &g, float H[6],
                                                  Cache &) {
        eval_h(F, p, s, n, g, H);
    }
    static __device__ __forceinline__ void theta_c(const FieldParams &F, float3 p, float s, float a, float3 b, Acc &c,
                                                   const AdjParams &A, const Cache &) {
        theta(F, p, s, a, b, c, A);
    }
    static __device__ __forceinline__ void flush(const Acc &, const FieldParams &, const AdjParams &) {}
};

// ---- replay hook: checkpoints (phase A), stop at a segment's end (phase B), splat capture ----------
// Cylindrical Bessel mode m = 0, 1, 2 (scene.cpp:205-257): n = n_o + A f, A = n_max s, f = J_m(k r)
// cos(m phi), phi = atan2(y, z). In polar form, with e_r = (y, z)/r, e_phi = (z, -y)/r and
// J'' = -J'/x - (1 - m^2/x^2) J (Bessel's equation):
//   grad f = f_r e_r + f_phi/r e_phi,
//   H = f_rr e_r e_r^T + (f_r/r + f_phiphi/r^2) e_phi e_phi^T + (f_rphi/r - f_phi/r^2)(e_r e_phi^T + e_phi e_r^T),
// with f_r = k J' cos, f_phi = -m J sin, f_rr = k^2 J'' cos, f_rphi = -m k J' sin, f_phiphi = -m^2 J cos.
// Parameters: n_max, phi_min, phi_max. Per photon the sum dJ/dA = sum (a f + b . grad f) is taken;
// with the scaling s = sin(psi), psi = phi_min + (phi_max - phi_min) u, unclamped, dJ/dn_max = s dJ/dA
// and dJ/dpsi = n_max cos(psi) dJ/dA; a clamped s (|sin psi| >= n_clip/n_max) makes A = +-n_clip,
// which depends on neither. Within M_EPSILON of the axis the Hessian is taken as zero.
template <int M> struct FieldAdjBessel {
    struct Acc { float dA, s, u; };
    struct Cache { float f; float3 gf; int gap; };
    static __device__ __forceinline__ void clear(Acc &c) { c.dA = 0.0f; c.s = 0.0f; c.u = 0.0f; }
    static __device__ __forceinline__ void parts(const FieldParams &F, float3 p, float &f, float3 &gf, float H[6]) {
#pragma unroll
        for (int j = 0; j < 6; ++j) H[j] = 0.0f;
        const float y = p.y, z = p.z;
        const float r2 = y * y + z * z;
        const float r = sqrtf(r2);
        const float rr = fmaxf(r, kEps);
        float jm, jm1;
        bessel_pair_table_t<M>(F.btab, F.bint, F.kb * rr, F.k_r * rr, jm, jm1);
        const float c = r > 0.0f ? z / r : 1.0f, sn = r > 0.0f ? y / r : 0.0f;
        float cm = 1.0f, sm = 0.0f;
        if (M == 1) { cm = c; sm = sn; }
        else if (M == 2) { cm = c * c - sn * sn; sm = 2.0f * c * sn; }
        const float x = F.k_r * rr, k = F.k_r, m = float(M);
        const float dj = m / x * jm - jm1;
        const float ddj = -dj / x - (1.0f - m * m / (x * x)) * jm;
        f = jm * cm;
        const float fr = k * dj * cm, fp = -m * jm * sm;
        // e_r = (sn, c), e_phi = (c, -sn) in (y, z)
        gf = f3(0.0f, fr * sn + fp / rr * c, fr * c - fp / rr * sn);
        if (r < kEps) return;
        const float frr = k * k * ddj * cm, frp = -m * k * dj * sm, fpp = -m * m * jm * cm;
        const float app = fr / r + fpp / r2, arp = frp / r - fp / r2;
        // H in (y, z): frr er er^T + app ep ep^T + arp (er ep^T + ep er^T)
        H[1] = frr * sn * sn + app * c * c + 2.0f * arp * sn * c;                 // yy
        H[2] = frr * c * c + app * sn * sn - 2.0f * arp * c * sn;                 // zz
        H[5] = frr * sn * c - app * c * sn + arp * (c * c - sn * sn);             // yz
    }
    static __device__ __forceinline__ void eval_h(const FieldParams &F, float3 p, float s, float &n, float3 &g, float H[6],
                                                  Cache &k) {
        k.gap = in_gap(F, p);
        if (k.gap) {
#pragma unroll
            for (int j = 0; j < 6; ++j) H[j] = 0.0f;
            n = F.n_o; g = f3(0.0f, 0.0f, 0.0f); k.f = 0.0f; k.gf = g;
            return;
        }
        parts(F, p, k.f, k.gf, H);
        const float A = F.amp * s;
        n = fmaf(A, k.f, F.n_o);
        g = mul(k.gf, A);
#pragma unroll
        for (int j = 0; j < 6; ++j) H[j] *= A;
    }
    static __device__ __forceinline__ void eval_h(const FieldParams &F, float3 p, float s, float &n, float3 &g, float H[6]) {
        Cache k;
        eval_h(F, p, s, n, g, H, k);
    }
    static __device__ __forceinline__ void theta_c(const FieldParams &, float3, float, float a, float3 b, Acc &c,
                                                   const AdjParams &, const Cache &k) {
        if (k.gap) return;
        c.dA += a * k.f + dot3(b, k.gf);
    }
    static __device__ __forceinline__ void theta(const FieldParams &F, float3 p, float s, float a, float3 b, Acc &c,
                                                 const AdjParams &A) {
        float n, H[6];
        float3 g;
        Cache k;
        eval_h(F, p, s, n, g, H, k);
        theta_c(F, p, s, a, b, c, A, k);
    }
    // the photon's scaling draw (the sixth uniform: five for genRay, scene.cpp:107-137)
    static __device__ __forceinline__ void begin(Acc &c, Lane &L, const KParams &P, float s) {
        rng_seek(L, P, 5);
        c.u = draw(L, P);
        c.s = s;
    }
    static __device__ __forceinline__ void flush(const Acc &c, const FieldParams &F, const AdjParams &A) {
        float sn, cs;
        sincos_red(F.phi_min + F.phi_range * c.u, sn, cs);
        if (!(sn < F.max_scaling && sn > -F.max_scaling)) return;      // clamped: A = +-n_clip
        atomicAdd(A.grad + 0, double(c.s * c.dA));
        const float dpsi = F.amp * cs * c.dA;
        atomicAdd(A.grad + 1, double(dpsi * (1.0f - c.u)));
        atomicAdd(A.grad + 2, double(dpsi * c.u));
    }
};
template <> struct FieldAdj<FK_BESSEL0> : FieldAdjBessel<0> {};
template <> struct FieldAdj<FK_BESSEL1> : FieldAdjBessel<1> {};
template <> struct FieldAdj<FK_BESSEL2> : FieldAdjBessel<2> {};

__device__ __forceinline__ float g_at(const AdjParams &A, int x, int y, int z) {
    if (x < 0 || x >= A.X || y < 0 || y >= A.Y || z < 0 || z >= A.Z) return 0.0f;
    return float(__ldg(A.G + (size_t(z) * A.Y + y) * A.X + x));
}

// dJ/dfilm at the four pixels a splat at sensor point p (path length pl) would touch; false when
// the splat leaves the film's binned range or all four weights are zero.
__device__ __forceinline__ bool splat_taps(const KParams &P, const AdjParams &A, float3 p, double pl, int depth,
                                           int &ix, int &iy, float G[4]) {
    int iz;
    float fx, fy;
    if (!splat_bin(P, A.X, p, pl, depth, ix, iy, iz, fx, fy)) return false;
    G[0] = g_at(A, ix, iy, iz); G[1] = g_at(A, ix + 1, iy, iz);
    G[2] = g_at(A, ix, iy + 1, iz); G[3] = g_at(A, ix + 1, iy + 1, iz);
    return G[0] != 0.0f || G[1] != 0.0f || G[2] != 0.0f || G[3] != 0.0f;
}

// Checkpointing trace (first kernel): records the source and every scatter vertex of the photon in
// this thread's buffer, marks which of them are followed by a splat that reaches the objective,
// bounds the length of every move, and at the photon's end copies its checkpoints into the batch
// pool. Never stops the events.
struct AdjTraceHook {
    static constexpr bool on = true;
    const KParams *P;
    const AdjParams *A;
    AdjVertex *v;              // this thread's checkpoints
    int nv, vcap, overflow;
    int direct_hit;
    int seg_entries;           // trajectory entries of the current segment: its start, one marker per
                               // later march, one per accepted step
    unsigned long long nok, ndrop, nabort;
    __device__ void put(int k, const Lane &L) {
        AdjVertex &c = v[k];
        c.pos[0] = L.pos.x; c.pos[1] = L.pos.y; c.pos[2] = L.pos.z;
        c.dir[0] = L.dir.x; c.dir[1] = L.dir.y; c.dir[2] = L.dir.z;
        c.total_dist = L.totalDist;
        c.depth = L.depth;
        c.total = L.total;
        c.draws_v = L.draws; c.steps_v = L.steps;
        c.draws_so = L.draws; c.steps_so = L.steps;
        c.hits = 0;
        c.len_in = seg_entries;
        c.len_conn = 0;
    }
    __device__ void photon_begin(const Lane &) { nv = 0; overflow = 0; direct_hit = 0; seg_entries = 0; }
    __device__ void march_begin() { ++seg_entries; }
    __device__ void accepted() { ++seg_entries; }
    // each hook ends a segment: the direct march at EV_SCATTER, a move at EV_VERTEX, a connection
    // at EV_SCATTER_ONCE
    __device__ bool at(Lane &L, int ev) {
        if (ev == EV_SCATTER) {
            put(0, L);
            v[0].hits = direct_hit ? 2 : 0;
            nv = 1;
        } else if (ev == EV_VERTEX) {
            if (nv < vcap) put(nv, L);
            else overflow = 1;
            ++nv;
        } else if (ev == EV_SCATTER_ONCE && nv - 1 < vcap && nv >= 1) {
            v[nv - 1].draws_so = L.draws;
            v[nv - 1].steps_so = L.steps;
            v[nv - 1].len_conn = seg_entries;
        }
        seg_entries = 0;
        return false;
    }
    __device__ void splatted(const Lane &, float3 p, double pl, int depth, float) {
        int ix, iy;
        float G[4];
        if (splat_taps(*P, *A, p, pl, depth, ix, iy, G)) {
            if (nv == 0) direct_hit = 1;                      // before EV_SCATTER: the direct splat
            else if (nv - 1 < vcap) v[nv - 1].hits |= 1;      // the connection from the last vertex
        }
    }
    __device__ void photon_end(const Lane &L) {
        AdjPhoton r;
        r.off = 0; r.nv = 0; r.hits = 0; r.s = L.s; r.tlen = 0; r.round = 0; r.last = 0; r.toff = 0; r.pad = 0;
        if (L.end == SMP_END_STEP_CAP || L.end == SMP_END_NAN) { r.status = PH_ABORTED; ++nabort; }
        else if (overflow) { r.status = PH_DROPPED; ++ndrop; }
        else {
            r.status = PH_OK;
            // the segments the sweep needs, with their exact trajectory entries: connections that
            // reach dJ/dfilm, every move up to the last of them, the direct march if it does
            int hits = 0, last = 0;
            long long tlen = 0;
            for (int k = 0; k < nv; ++k) {
                hits |= v[k].hits;
                if (k >= 1 && (v[k].hits & 1)) last = k;
            }
            if (v[0].hits & 2) tlen += v[0].len_in;
            for (int k = 1; k < nv; ++k) {
                if (k <= last) tlen += v[k].len_in;
                if (v[k].hits & 1) tlen += v[k].len_conn;
            }
            r.hits = hits;
            r.last = last;
            r.tlen = int(min(tlen, 2147483647LL));
            if (tlen > A->traj_cap) { r.status = PH_DROPPED; ++ndrop; hits = 0; r.hits = 0; }
            if (hits && nv > 0) {
                const unsigned long long off = atomicAdd(A->pool_next, (unsigned long long)nv);
                if ((long long)(off + nv) > A->pool_cap) { r.status = PH_DROPPED; ++ndrop; }
                else {
                    r.off = int(off);
                    r.nv = nv;
                    for (int k = 0; k < nv; ++k) A->pool[off + k] = v[k];
                }
            }
            if (r.status == PH_OK) ++nok;
        }
        A->photons[L.idx - P->first_photon] = r;
    }
};

// Segment replay (sweep kernel): stops at the entry of the event that ends the segment and keeps
// the segment's splat.
struct AdjReplayHook {
    static constexpr bool on = true;
    int stop_ev;
    int seg_len;               // trajectory entries of the current segment
    int splat;                 // a splat happened in this segment
    float3 sp;                 // its sensor point, path length, depth
    double spl;
    int sdepth;
    __device__ bool at(Lane &, int ev) { return ev == stop_ev; }
    __device__ void splatted(const Lane &, float3 p, double pl, int depth, float) {
        splat = 1; sp = p; spl = pl; sdepth = depth;
    }
    __device__ void photon_begin(const Lane &) {}
    __device__ void photon_end(const Lane &) {}
};

__device__ __forceinline__ float4 traj_get(const AdjParams &A, long long base, int i) {
    return A.traj[base + i];
}

__device__ __forceinline__ int face_axis(float3 nf) { return nf.x != 0.0f ? 0 : (nf.y != 0.0f ? 1 : 2); }
__device__ __forceinline__ float3 reflect_n(float3 v, float3 nf) { return sub(v, mul(nf, 2.0f * dot3(v, nf))); }
__device__ __forceinline__ void add_axis(float3 &v, int ax, float x) {
    if (ax == 0) v.x += x; else if (ax == 1) v.y += x; else v.z += x;
}

// Backward sweep over one recorded segment (entries [0, nent) of this thread's buffer), one step
// per sweep_point call so that a warp's sweeping lanes advance together.
// sweep_begin takes (Pa, Da), the adjoints of the segment's end position and optical direction,
// a_end the adjoint of n at the end point, T the adjoint of each face crossing's arc-length shift
// and face_end: the last march ends on a face (connections, direct) or at its sampled distance
// (moves; T is then derived here from the end adjoints). When sweep_point returns 1 the state
// holds the adjoints of the start position (Pa, field terms included) and start direction (Da),
// the start point's parameter cotangent (a0, b0) left to the caller, and n, grad n there (n0, gk).
struct Sweep {
    int i;                     // entry whose step is undone next
    float4 e;
    float4 pn;                 // entry i - 1, loaded one step ahead (its latency overlaps a step)
    float3 d, gk, Pa, Da, b0;
    float T, a0, n0;
};

template <int FK, class FA>
__device__ __forceinline__ void sweep_begin(Sweep &w, const KParams &P, const AdjParams &A, long long base, int nent,
                                            float3 md_end, float3 Pa, float3 Da, float a_end, float T, bool face_end,
                                            float s, typename FA::Acc &acc) {
    const FieldParams &F = P.field;
    w.i = nent - 1;
    w.e = traj_get(A, base, w.i);
    w.pn = traj_get(A, base, w.i - 1);          // nent >= 2
    const float3 pk = f3(w.e.x, w.e.y, w.e.z);
    float n_k, H[6];
    float3 g_k;
    typename FA::Cache kc;
    FA::eval_h(F, pk, s, n_k, g_k, H, kc);
    const float3 u = divs(md_end, n_k);
    const float At = dot3(u, Pa) + dot3(g_k, Da) + dot3(g_k, u) * a_end;
    if (face_end) {
        const int ax = face_axis(face_normal(P, pk));
        add_axis(Pa, ax, -(At + T) / comp(u, ax));
    } else {
        T = -At;        // each earlier face crossing delays the sampled end by its own shift
    }
    // second kick of the last step, and the end point's own use of n
    const float3 b = mul(Da, 0.5f * w.e.w);
    Pa = add(Pa, add(mul(g_k, a_end), hmul(H, b)));
    FA::theta_c(F, pk, s, a_end, b, acc, A, kc);
    w.d = md_end; w.gk = g_k; w.Pa = Pa; w.Da = Da; w.T = T;
}

// Undo one step. 0: more to go; 1: the start point is reached (outputs in w); 2: malformed.
template <int FK, class FA>
__device__ __forceinline__ int sweep_point(Sweep &w, const KParams &P, const AdjParams &A, long long base, float s,
                                           typename FA::Acc &acc) {
    const FieldParams &F = P.field;
    const float c = w.e.w, hh = 0.5f * c;
    int j = w.i - 1;
    if (j < 0) return 2;
    float4 pe = w.pn;
    const bool junction = pe.w < 0.0f;
    if (junction) {
        j -= 1;
        if (j < 0) return 2;
        pe = traj_get(A, base, j);
    }
    // the next call's entry, in flight while this step is undone
    const float4 nx = (j >= 1 && pe.w != 0.0f) ? traj_get(A, base, j - 1) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float3 pp = f3(pe.x, pe.y, pe.z);
    float n1, H[6];
    float3 g1;
    typename FA::Cache kc;
    FA::eval_h(F, pp, s, n1, g1, H, kc);
    const float3 dh = sub(w.d, mul(w.gk, hh));
    const float3 dprev = sub(dh, mul(g1, hh));
    const float q = c / n1;
    const float3 Dh = add(w.Da, mul(w.Pa, q));
    const float a1 = -(q / n1) * dot3(dh, w.Pa);
    float3 b1 = mul(Dh, hh);
    float3 Pa = add(w.Pa, add(mul(g1, a1), hmul(H, b1)));
    float3 Da = Dh;
    float3 d = dprev;
    if (junction) {
        // the previous march ended on a face and reflected: undo the reflection, then the crossing
        const float3 nf = face_normal(P, pp);
        Da = reflect_n(Da, nf);
        d = reflect_n(d, nf);
        const float3 u = divs(d, n1);
        const int ax = face_axis(nf);
        const float At = dot3(u, Pa) + dot3(g1, Da) + w.T;
        add_axis(Pa, ax, -At / comp(u, ax));
    }
    w.gk = g1;
    w.d = d;
    if (pe.w == 0.0f) {                // the segment's start point
        w.Pa = Pa; w.Da = Da; w.a0 = a1; w.b0 = b1; w.n0 = n1;
        return 1;
    }
    // second kick of the previous step
    const float3 b2 = mul(Da, 0.5f * pe.w);
    Pa = add(Pa, hmul(H, b2));
    b1 = add(b1, b2);
    FA::theta_c(F, pp, s, a1, b1, acc, A, kc);
    w.Pa = Pa; w.Da = Da;
    w.i = j;
    w.e = pe;
    w.pn = nx;
    return 0;
}

// ---- the splat's value as a function of the march's end state --------------------------------------
// Inputs (the order of the derivative components): end position p (0-2), end direction md (3-5),
// n at the end (6), the connection's marched distance d2s (7), the vertex direction dv (8-10, used
// by the Henyey-Greenstein factor of a connection). Follows run_events' exit at the sensor face
// (directTracing photon.cpp:41-87; addEnergyInParticle scene.cpp:866-946; propagate_till_sensor
// camera.cpp:54-75 without a lens) and the bilinear split of addEnergyToImage with the base
// pixel (ix, iy) held fixed. Returns dJ/d(inputs) for J = value * sum_taps G w.
static __device__ __noinline__ void sensor_grad(const KParams &P, int X, float weight, float sigma_t, float g, bool connect,
                                         float3 p, float3 md, float n, float d2s, float3 dv, int ix, int iy,
                                         float G00, float G10, float G01, float G11, float *out) {
    typedef Dual<11> D;
    D px = dvar<11>(p.x, 0), py = dvar<11>(p.y, 1), pz = dvar<11>(p.z, 2);
    D mx = dvar<11>(md.x, 3), my = dvar<11>(md.y, 4), mz = dvar<11>(md.z, 5);
    D nn = dvar<11>(n, 6), dd = dvar<11>(d2s, 7);
    D l = dsqrt(mx * mx + my * my + mz * mz);
    D sx = mx / l, sy = my / l, sz = mz / l;
    D rx = sx, ry = sy, rz = sz;
    D fw = dc<11>(1.0f);
    if (n > 1.0f) {
        rx = rx / nn;
        D lr = dsqrt(rx * rx + ry * ry + rz * rz);
        rx = rx / lr; ry = ry / lr; rz = rz / lr;
        D eta = 1.0f / nn;
        D F = dc<11>(0.0f);
        if (!(fabsf(eta.v - 1.0f) < kEps * fmaxf(1.0f, fabsf(eta.v)))) {
            D Rs = (sx - eta * rx) / (sx + eta * rx);
            D Rp = (rx - eta * sx) / (rx + eta * sx);
            F = 0.5f * (Rs * Rs + Rp * Rp);
        }
        fw = (1.0f - F) / nn / nn;
    }
    D val = weight * dexp(dd * (-sigma_t)) * fw;
    if (connect) {
        const float cx = P.cam_dir[0], cy = P.cam_dir[1], cz = P.cam_dir[2];
        D fore = (rx * cx + ry * cy + rz * cz) / (sx * cx + sy * cy + sz * cz);
        D vx = dvar<11>(dv.x, 8), vy = dvar<11>(dv.y, 9), vz = dvar<11>(dv.z, 10);
        D il = 1.0f / dsqrt(vx * vx + vy * vy + vz * vz);
        D c = (vx * il) * sx + (vy * il) * sy + (vz * il) * sz;
        D b = (1.0f + g * g) - (2.0f * g) * c;
        D hg = ((1.0f / (4.0f * 3.14159265358979f)) * (1.0f - g * g)) / (b * dsqrt(b));
        val = val * 6.28318548202514648f * hg * fore;
    }
    D dist = (P.cam_origin[0] - px) / rx;
    D qx = px + rx * dist, qy = py + ry * dist, qz = pz + rz * dist;
    D x = ((qx * P.cam_h[0] + qy * P.cam_h[1] + qz * P.cam_h[2]) - P.cam_origin[1]) / P.cam_plane[0];
    D y = ((qx * P.cam_v[0] + qy * P.cam_v[1] + qz * P.cam_v[2]) - P.cam_origin[2]) / P.cam_plane[1];
    D fx = (x + 0.5f) * float(X) - float(ix);
    D fy = (y + 0.5f) * float(P.Y) - float(iy);
    D gx = 1.0f - fx, gy = 1.0f - fy;
    D w = gx * gy * G00 + fx * gy * G10 + gx * fy * G01 + fx * fy * G11;
    D J = val * w;
#pragma unroll
    for (int i = 0; i < 11; ++i) out[i] = J.d[i];
}

// Jacobian^T of the scatterOnce direction update (photon.cpp:20-38: v' = |v| HG(v/|v|), the HG
// sample drawn in the frame of util::coordinateSystem, util.h:17-27) applied to D.
static __device__ __noinline__ float3 hg_vjp(float3 v, float cosT, float sinT, float cP, float sP, float3 Dout) {
    typedef Dual<3> D;
    D x = dvar<3>(v.x, 0), y = dvar<3>(v.y, 1), z = dvar<3>(v.z, 2);
    D mag = dsqrt(x * x + y * y + z * z);
    D r = 1.0f / mag;
    D ix = x * r, iy = y * r, iz = z * r;
    D ax, ay, az, bx, by, bz;     // ay-axis (b) of the frame, then ax = ay x in
    if (fabsf(ix.v) > fabsf(iy.v)) {
        D inv = 1.0f / dsqrt(ix * ix + iz * iz);
        bx = iz * inv; by = dc<3>(0.0f); bz = dc<3>(0.0f) - ix * inv;
    } else {
        D inv = 1.0f / dsqrt(iy * iy + iz * iz);
        bx = dc<3>(0.0f); by = iz * inv; bz = dc<3>(0.0f) - iy * inv;
    }
    ax = by * iz - bz * iy; ay = bz * ix - bx * iz; az = bx * iy - by * ix;
    const float u = sinT * cP, w = sinT * sP;
    D ox = (ax * u + bx * w + ix * cosT) * mag;
    D oy = (ay * u + by * w + iy * cosT) * mag;
    D oz = (az * u + bz * w + iz * cosT) * mag;
    return f3(Dout.x * ox.d[0] + Dout.y * oy.d[0] + Dout.z * oz.d[0],
              Dout.x * ox.d[1] + Dout.y * oy.d[1] + Dout.z * oz.d[1],
              Dout.x * ox.d[2] + Dout.y * oy.d[2] + Dout.z * oz.d[2]);
}

__device__ __forceinline__ void restore(Lane &L, const KParams &P, const AdjVertex &c, bool at_vertex) {
    L.pos = f3(c.pos[0], c.pos[1], c.pos[2]);
    L.dir = f3(c.dir[0], c.dir[1], c.dir[2]);
    L.total = c.total;
    L.totalDist = c.total_dist;
    L.depth = c.depth;
    L.end = 0;
    L.steps = at_vertex ? c.steps_v : c.steps_so;
    rng_seek(L, P, at_vertex ? c.draws_v : c.draws_so);
}


// Checkpointing trace: the render's persistent lane loop over the batch's photons with the
// recording hook (no film is written: P.X = 0).
template <int FK>
__global__ void __launch_bounds__(128, 4) adjoint_trace_kernel(const __grid_constant__ KParams P,
                                                               const __grid_constant__ AdjParams A) {
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    Lane L;
    L.end = 0;
    L.idx = 0;
    L.tab = P.field.btab;                       // Bessel table (global memory); NULL for other fields
    L.inst = nullptr;
    L.s = 0.0f;
    AdjTraceHook h;
    h.P = &P;
    h.A = &A;
    h.v = A.tverts + size_t(t) * A.vcap;
    h.vcap = A.vcap;
    h.nok = h.ndrop = h.nabort = 0;
    h.photon_begin(L);
    LaneStats S;
    lane_loop<FK, AdjTraceHook>(L, ST_FETCH, P, S, lane, &h);
    flush_stats(S, P, lane);
    atomicAdd(A.cnt + ADJ_PHOTONS, h.nok);
    atomicAdd(A.cnt + ADJ_DROPPED, h.ndrop);
    atomicAdd(A.cnt + ADJ_ABORTED, h.nabort);
}

// ---- the checkpointing trace on the slot pool ------------------------------------------------------
// The render's two-kernel march (wavefront.cuh) with the recording hook in the event and tail kernels:
// wf_march_kernel marches the slots unchanged, and each slot carries its photon's checkpoints
// (A.tverts) and hook state (A.tstate) between launches. The hook counts a segment's trajectory
// entries as its march-start markers plus the accepted ER steps; the march kernel does not count:
// a march's accepted steps are its steps less its refinements (a refinement restores the position,
// every other step moves it), and the refinements are the precision levels it used,
// precision - max(prec, 0) at its end.
__device__ __forceinline__ void trace_hook_load(AdjTraceHook &h, const KParams &P, const AdjParams &A, int slot,
                                                const Lane &L) {
    const int4 hs = A.tstate[slot];
    h.v = A.tverts + size_t(slot) * size_t(A.vcap);
    h.nv = hs.x;
    h.overflow = hs.y & 1;
    h.direct_hit = (hs.y >> 1) & 1;
    h.seg_entries = hs.z + (L.steps - hs.w) - (P.precision - max(L.prec, 0));
}

template <int FK>
__global__ void __launch_bounds__(128, 4)
adjoint_trace_event_kernel(const __grid_constant__ KParams P, const __grid_constant__ WaveParams W,
                           const __grid_constant__ AdjParams A, int it) {
    const int lane = threadIdx.x & 31;
    const bool init = it < 0;
    const int cur = init ? 1 : (it & 1), nxt = cur ^ 1;
    const unsigned q0 = init ? unsigned(W.n_slots) : queue_cnt(W, cur)[0];
    const unsigned n = init ? q0 : q0 + queue_cnt(W, cur)[1];
    if (!init && blockIdx.x == 0 && threadIdx.x < 2) {
        list_cnt(W, cur)[threadIdx.x] = 0u;     // consumed by march launch `it`
        queue_cnt(W, nxt)[threadIdx.x] = 0u;    // filled by march launch `it + 1`
    }
    LaneStats S;
    AdjTraceHook h;
    h.P = &P;
    h.A = &A;
    h.vcap = A.vcap;
    h.nok = h.ndrop = h.nabort = 0;
    const unsigned lanes = gridDim.x * blockDim.x, nwarps = lanes >> 5;
    for (unsigned base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; base < n; base += nwarps * 32u) {
        const unsigned i = base + unsigned(lane);
        const bool valid = i < n;
        int st = ST_DONE, slot = 0;
        bool cls1 = false;
        if (valid) {
            slot = init ? int(i) : two_class_at(W.queue[cur], q0, W.n_slots, i);
            Lane L;
            L.inst = nullptr;
            if (init) {
                L.end = 0;
                L.idx = 0;
                st = ST_FETCH;
                h.v = A.tverts + size_t(slot) * size_t(A.vcap);
            } else {
                wf_load_lane(W, P, slot, L);
                L.tab = P.field.btab;
                trace_hook_load(h, P, A, slot, L);
                st = run_events<FK, AdjTraceHook>(L, P, EV_MARCH_END, &h);
                if (st == ST_FETCH) {
                    finish_photon_stats<FK>(L, S);
                    h.photon_end(L);
                }
            }
            L.tab = P.field.btab;
            while (st == ST_FETCH) {
                const cg::coalesced_group g = cg::coalesced_threads();
                unsigned long long k = 0;
                if (g.thread_rank() == 0) k = atomicAdd(P.counters + CNT_NEXT_PHOTON, (unsigned long long)g.size());
                k = g.shfl(k, 0) + g.thread_rank();
                if (k < (unsigned long long)P.n_photons) {
                    L.idx = P.first_photon + (long long)k;
                    L.end = 0;
                    h.photon_begin(L);
                    st = run_events<FK, AdjTraceHook>(L, P, EV_NEW, &h);
                    if (st == ST_FETCH) {
                        finish_photon_stats<FK>(L, S);
                        h.photon_end(L);
                    }
                } else {
                    st = ST_DONE;
                }
            }
            if (st == ST_MARCH) {
                wf_store_lane(W, P, slot, L);
                // + 1: the march's start marker
                A.tstate[slot] = make_int4(h.nv, h.overflow | (h.direct_hit << 1), h.seg_entries + 1, L.steps);
                cls1 = move_class(W, L.ctx);
            }
        }
        const unsigned mm = __ballot_sync(kFull, valid && st == ST_MARCH);
        warp_append2(W.list[nxt], list_cnt(W, nxt), W.n_slots, mm, cls1, slot, lane);
    }
    flush_stats(S, P, lane);
    if (h.nok) atomicAdd(A.cnt + ADJ_PHOTONS, h.nok);
    if (h.ndrop) atomicAdd(A.cnt + ADJ_DROPPED, h.ndrop);
    if (h.nabort) atomicAdd(A.cnt + ADJ_ABORTED, h.nabort);
}

// the trace's tail: the live slots, with their checkpoints and hook state, on the persistent lane loop
template <int FK>
__global__ void __launch_bounds__(128, 4)
adjoint_trace_finish_kernel(const __grid_constant__ KParams P, const __grid_constant__ WaveParams W,
                            const __grid_constant__ AdjParams A, int it) {
    const int lane = threadIdx.x & 31, cur = it & 1;
    const unsigned n0 = list_cnt(W, cur)[0], n = n0 + list_cnt(W, cur)[1];
    const unsigned gid = blockIdx.x * blockDim.x + threadIdx.x, lanes = gridDim.x * blockDim.x;
    if (gid == 0 && n > lanes) atomicAdd(P.counters + CNT_LOST, (unsigned long long)(n - lanes));
    Lane L;
    L.end = 0;
    L.idx = 0;
    L.inst = nullptr;
    L.tab = P.field.btab;
    AdjTraceHook h;
    h.P = &P;
    h.A = &A;
    h.vcap = A.vcap;
    h.nok = h.ndrop = h.nabort = 0;
    h.v = A.tverts;
    h.nv = 0; h.overflow = 0; h.direct_hit = 0; h.seg_entries = 0;
    int st = ST_FETCH;
    if (gid < n) {
        const int slot = two_class_at(W.list[cur], n0, W.n_slots, gid);
        wf_load_lane(W, P, slot, L);
        L.tab = P.field.btab;
        trace_hook_load(h, P, A, slot, L);
        st = ST_MARCH;
    }
    LaneStats S;
    lane_loop<FK, AdjTraceHook>(L, st, P, S, lane, &h);
    flush_stats(S, P, lane);
    if (h.nok) atomicAdd(A.cnt + ADJ_PHOTONS, h.nok);
    if (h.ndrop) atomicAdd(A.cnt + ADJ_DROPPED, h.ndrop);
    if (h.nabort) atomicAdd(A.cnt + ADJ_ABORTED, h.nabort);
}

// Segment c of a photon is needed by the sweep: the direct march if its splat reaches dJ/dfilm,
// a connection if its splat does, a move if a later connection does.
__device__ __forceinline__ bool seg_needed(const AdjPhoton &r, const AdjVertex *V, int c) {
    if (c == 0) return (V[0].hits & 2) != 0;
    const int k = (c + 1) >> 1;
    return (c & 1) ? k <= r.last : (V[k].hits & 1) != 0;
}

// Discrete work, marching and sweeping lanes (see the two kernels below).
enum AdjMode : int { M_DISC = 0, M_MARCH = 1, M_SWEEP = 2, M_EXIT = 3 };

// Replay kernel: for each photon of this round, every segment the sweep needs, replayed forward from
// its checkpoint with the trajectory written to traj[toff ..] and the end state to its AdjSeg.
// Lanes run their discrete work (photon fetch, restore, events) one by one and then march together
// until a quarter of the live lanes wait, as the render's lane loop does. A photon whose entries
// no longer fit this round's trajectory buffer waits for the next round.
template <int FK>
__global__ void __launch_bounds__(128, 3) adjoint_replay_kernel(const __grid_constant__ KParams P,
                                                                const __grid_constant__ AdjParams A, int round) {
    const FieldParams &F = P.field;
    AdjReplayHook h;
    Lane L;
    L.tab = P.field.btab;                       // Bessel table (global memory); NULL for other fields
    L.inst = nullptr;
    L.s = 0.0f;
    long long rsteps = 0;
    unsigned long long nmis = 0;
    const AdjVertex *V = A.pool;
    AdjSeg *segs = A.segs;
    AdjPhoton r;
    r.last = 0; r.nv = 0;
    const long long n_order = (long long)*A.n_order;
    int mode = M_DISC, c = 0, K = -1, ev = EV_NEW;
    bool in_seg = false, first = true, trunc = false;
    long long base = 0, pos = 0, pend = 0;          // pend: end of the photon's reserved entries
    float3 md0 = f3(0.0f, 0.0f, 0.0f);

    for (;;) {
        while (mode == M_DISC) {
            if (!in_seg) {
                // the photon's next needed segment, or the next photon
                ++c;
                while (c <= 2 * K && !seg_needed(r, V, c)) ++c;
                if (c > 2 * K) {
                    const long long q = (long long)atomicAdd(A.cnt + ADJ_NEXT, 1ull);
                    if (q >= n_order) { mode = M_EXIT; break; }
                    const long long k = A.order[q];
                    r = A.photons[k];
                    K = -1;
                    if (r.status != PH_OK || !r.hits || r.round != 0) continue;
                    const unsigned long long off = atomicAdd(A.traj_next, (unsigned long long)r.tlen);
                    if ((long long)(off + r.tlen) > A.traj_cap) { atomicExch(A.pending, 1); continue; }
                    A.photons[k].round = round;
                    A.photons[k].toff = (long long)off;
                    L.idx = P.first_photon + k;         // keys the photon's Philox stream
                    L.s = r.s;
                    V = A.pool + r.off;
                    segs = A.segs + 2LL * r.off;
                    K = r.nv - 1;
                    pos = (long long)off;
                    pend = (long long)off + r.tlen;
                    c = -1;
                    continue;
                }
                const int k = (c + 1) >> 1;
                h.seg_len = 0;
                h.splat = 0;
                if (c == 0) {                           // the direct march, from the photon's start
                    L.end = 0;                          // run_events tests the end code before EV_NEW
                    ev = EV_NEW;
                    h.stop_ev = EV_SCATTER;
                } else if (c & 1) {                     // the move into vertex k
                    restore(L, P, V[k - 1], false);
                    ev = k == 1 ? EV_SCATTER : EV_SCATTER_ONCE;
                    h.stop_ev = EV_VERTEX;
                } else {                                // the connection from vertex k
                    restore(L, P, V[k], true);
                    L.mp = L.pos;
                    Field<FK>::eval(F, L.tab, L.mp, L.s, L.mn, L.mg);
                    ev = EV_VERTEX;
                    h.stop_ev = EV_SCATTER_ONCE;
                }
                base = pos;
                first = true;
                trunc = false;
                in_seg = true;
            }
            const int st = run_events<FK, AdjReplayHook>(L, P, ev, &h);
            if (st == ST_MARCH) {
                if (base + h.seg_len < pend)
                    A.traj[base + h.seg_len] = first ? make_float4(L.mp.x, L.mp.y, L.mp.z, 0.0f)
                                                     : make_float4(0.0f, 0.0f, 0.0f, -1.0f);
                else trunc = true;
                if (first) md0 = L.md;
                first = false;
                ++h.seg_len;
                mode = M_MARCH;
                break;
            }
            // the segment has ended: check it against the checkpoint it leads to, record its end
            const int k = (c + 1) >> 1;
            bool ok = st == ST_HOOK && !trunc;
            if (ok && (c & 1)) {
                const AdjVertex &cv = V[k];
                ok = L.pos.x == cv.pos[0] && L.pos.y == cv.pos[1] && L.pos.z == cv.pos[2] &&
                     L.dir.x == cv.dir[0] && L.dir.y == cv.dir[1] && L.dir.z == cv.dir[2];
            }
            if (!ok) ++nmis;
            AdjSeg &g = segs[c];
            g.off = base;
            g.len = int(min((long long)h.seg_len, pend - base));
            g.ok = ok && ((c & 1) || h.splat);
            g.mp[0] = L.mp.x; g.mp[1] = L.mp.y; g.mp[2] = L.mp.z;
            g.md[0] = L.md.x; g.md[1] = L.md.y; g.md[2] = L.md.z;
            g.mn = L.mn;
            g.d2s = L.d2s;
            g.dir[0] = L.dir.x; g.dir[1] = L.dir.y; g.dir[2] = L.dir.z;
            g.md0[0] = md0.x; g.md0[1] = md0.y; g.md0[2] = md0.z;
            g.sp[0] = h.sp.x; g.sp[1] = h.sp.y; g.sp[2] = h.sp.z;
            g.sdepth = h.sdepth;
            g.spl = h.spl;
            pos = min(base + h.seg_len, pend);
            in_seg = false;
        }

        const unsigned live = __ballot_sync(kFull, mode != M_EXIT);
        if (live == 0) break;
        const int thr = max(1, (__popc(live) * A.idle_replay + 16) >> 5);
        if (__any_sync(kFull, mode == M_MARCH)) {
            for (;;) {
                if (mode == M_MARCH) {
                    for (int t = 0; t < 2; ++t) {
                        const float3 q = L.mp;
                        const bool end = march_step<FK>(L, P);
                        ++rsteps;
                        if (q.x != L.mp.x || q.y != L.mp.y || q.z != L.mp.z) {
                            if (base + h.seg_len < pend) A.traj[base + h.seg_len] = make_float4(L.mp.x, L.mp.y, L.mp.z, L.cur);
                            else trunc = true;
                            ++h.seg_len;
                        }
                        if (end) { mode = M_DISC; ev = EV_MARCH_END; break; }
                    }
                }
                const unsigned waiting = __ballot_sync(kFull, mode == M_DISC);
                if (__popc(waiting) >= thr || !__any_sync(kFull, mode == M_MARCH)) break;
            }
        }
    }
    atomicAdd(A.cnt + ADJ_STEPS_REPLAY, (unsigned long long)rsteps);
    if (nmis) atomicAdd(A.cnt + ADJ_MISMATCH, nmis);
}

// Sweep kernel: for each photon of this round, the jobs of its backward pass over the recorded
// segments -- the connection from vertex K, the move into vertex K, ..., the move into vertex 1,
// the direct march, the source direction n(p0) omega0 -- each a backward sweep (sweep_begin, then
// sweep_point per recorded step). Lanes run their discrete work one by one and then sweep together
// until few lanes are left sweeping.
enum AdjJob : int { JOB_CONN = 1, JOB_MOVE = 2, JOB_DIRECT = 3, JOB_SOURCE = 4 };



// The sweep kernel per field kind; NW bounds the plane-wave count (a plane-wave field of at most two
// waves runs the NW = 2 instance, whose accumulators take fewer registers); MINB resident blocks.
template <int FK, int NW> struct FieldAdjSel { typedef FieldAdj<FK> T; };
template <int NW> struct FieldAdjSel<FK_PLANEWAVE, NW> { typedef FieldAdjPW<NW> T; };

template <int FK, int NW, int MINB>
__global__ void __launch_bounds__(128, MINB) adjoint_sweep_kernel(const __grid_constant__ KParams P,
                                                            const __grid_constant__ AdjParams A, int round) {
    typedef typename FieldAdjSel<FK, NW>::T FA;
    const FieldParams &F = P.field;
    Lane L;                                     // Philox draws of the HG rotation
    L.tab = P.field.btab;                       // Bessel table (global memory); NULL for other fields
    L.inst = nullptr;
    long long pts = 0;
    unsigned long long nspl = 0, nskip = 0;
    const float albedo = P.albedo;
    const int rr_draw = (albedo > 0.0f && albedo < 1.0f) ? 1 : 0;
    const AdjVertex *V = A.pool;
    const AdjSeg *segs = A.segs;
    const long long n_order = (long long)*A.n_order;
    int mode = M_DISC, job = 0, kv = 0;
    bool busy = false;                          // a photon is in progress
    float s = 0.0f;
    float3 lp = f3(0.0f, 0.0f, 0.0f), ld = lp, Ddir = lp;
    long long sbase = 0;
    typename FA::Acc acc;
    FA::clear(acc);
    Sweep w;
    bool after = false;                         // a sweep just finished: its job's start handling is due

    for (;;) {
        while (mode == M_DISC) {
            if (after) {
                after = false;
                const float4 e0 = traj_get(A, sbase, 0);
                const float3 p0 = f3(e0.x, e0.y, e0.z);
                const AdjSeg &g = segs[job == JOB_DIRECT ? 0 : (job == JOB_MOVE ? 2 * kv - 1 : 2 * kv)];
                if (job == JOB_CONN) {
                    // md0 = omega n(pos): the start direction's dependence on n at the vertex
                    const float as = (g.md0[0] * w.Da.x + g.md0[1] * w.Da.y + g.md0[2] * w.Da.z) / w.n0;
                    lp = add(lp, add(w.Pa, mul(w.gk, as)));
                    ld = add(ld, Ddir);
                    FA::theta(F, p0, s, w.a0 + as, w.b0, acc, A);
                } else if (job == JOB_MOVE) {
                    FA::theta(F, p0, s, w.a0, w.b0, acc, A);
                    lp = w.Pa;
                    if (kv >= 2) {
                        // the move began with v' = |v| HG(v / |v|) at vertex kv - 1
                        const AdjVertex &c = V[kv - 1];
                        rng_seek(L, P, c.draws_so + rr_draw);
                        const float u1 = draw(L, P), u2 = draw(L, P);
                        const float gg = P.g;
                        float cosT;
                        if (fabsf(gg) < kEps) cosT = 1.0f - 2.0f * u1;
                        else {
                            const float sq = (1.0f - gg * gg) / (1.0f - gg + 2.0f * gg * u1);
                            cosT = (1.0f + gg * gg - sq * sq) / (2.0f * gg);
                        }
                        const float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
                        float sP, cP;
                        sincos_red(6.28318548202514648f * u2, sP, cP);
                        ld = hg_vjp(f3(c.dir[0], c.dir[1], c.dir[2]), cosT, sinT, cP, sP, w.Da);
                    } else {
                        ld = w.Da;
                    }
                } else {                            // JOB_DIRECT: starts from the source state
                    lp = add(lp, w.Pa);
                    ld = add(ld, w.Da);
                    FA::theta(F, p0, s, w.a0, w.b0, acc, A);
                }
                // the next job
                if (job == JOB_CONN) job = JOB_MOVE;
                else if (job == JOB_MOVE) {
                    if (kv == 1) job = JOB_DIRECT;
                    else { --kv; job = JOB_CONN; }
                } else job = JOB_SOURCE;
            }
            if (!busy) {
                const long long q = (long long)atomicAdd(A.cnt + ADJ_NEXT, 1ull);
                if (q >= n_order) { mode = M_EXIT; break; }
                const long long k = A.order[q];
                const AdjPhoton r = A.photons[k];
                if (r.round != round) continue;
                L.idx = P.first_photon + k;
                s = r.s;
                V = A.pool + r.off;
                segs = A.segs + 2LL * r.off;
                FA::clear(acc);
                FA::begin(acc, L, P, s);
                lp = f3(0.0f, 0.0f, 0.0f); ld = lp;
                kv = r.nv - 1;
                job = kv >= 1 ? JOB_CONN : JOB_DIRECT;
                busy = true;
            }
            // set up the current job's sweep, skipping jobs with nothing to carry
            if (job == JOB_SOURCE) {
                // dir0 = n(p0) omega0 (photon.cpp:329)
                if (ld.x != 0.0f || ld.y != 0.0f || ld.z != 0.0f) {
                    const AdjVertex &c = V[0];
                    const float3 p0 = f3(c.pos[0], c.pos[1], c.pos[2]);
                    float n0, H[6];
                    float3 g0;
                    FA::eval_h(F, p0, s, n0, g0, H);
                    const float as = (c.dir[0] * ld.x + c.dir[1] * ld.y + c.dir[2] * ld.z) / n0;
                    FA::theta(F, p0, s, as, f3(0.0f, 0.0f, 0.0f), acc, A);
                }
                FA::flush(acc, F, A);
                busy = false;
                continue;
            }
            const int c = job == JOB_DIRECT ? 0 : (job == JOB_MOVE ? 2 * kv - 1 : 2 * kv);
            bool run = false, face_end = true;
            float3 Pa = f3(0.0f, 0.0f, 0.0f), Da = Pa;
            float a_end = 0.0f, T = 0.0f;
            Ddir = Pa;
            if (job == JOB_MOVE) {
                run = !(lp.x == 0.0f && lp.y == 0.0f && lp.z == 0.0f && ld.x == 0.0f && ld.y == 0.0f && ld.z == 0.0f);
                Pa = lp; Da = ld;
                face_end = false;
            } else if (job == JOB_CONN ? (V[kv].hits & 1) : (V[0].hits & 2)) {
                const AdjSeg &g = segs[c];
                int ix, iy;
                float Gt[4];
                if (g.ok && splat_taps(P, A, f3(g.sp[0], g.sp[1], g.sp[2]), g.spl, g.sdepth, ix, iy, Gt)) {
                    float gr[11];
                    sensor_grad(P, A.X, P.weight, P.sigma_t, P.g, job == JOB_CONN, f3(g.mp[0], g.mp[1], g.mp[2]),
                                f3(g.md[0], g.md[1], g.md[2]), g.mn, g.d2s, f3(g.dir[0], g.dir[1], g.dir[2]),
                                ix, iy, Gt[0], Gt[1], Gt[2], Gt[3], gr);
                    Pa = f3(gr[0], gr[1], gr[2]);
                    Da = f3(gr[3], gr[4], gr[5]);
                    a_end = gr[6];
                    T = gr[7];
                    Ddir = f3(gr[8], gr[9], gr[10]);
                    run = true;
                    ++nspl;
                }
            }
            if (run && segs[c].len >= 2 && (job != JOB_MOVE || segs[c].ok)) {
                const AdjSeg &g = segs[c];
                sbase = g.off;
                sweep_begin<FK, FA>(w, P, A, sbase, g.len, f3(g.md[0], g.md[1], g.md[2]), Pa, Da, a_end, T, face_end, s, acc);
                mode = M_SWEEP;
                break;
            }
            if (run) ++nskip;
            // nothing to sweep: the next job, with the adjoint carried as it is
            if (job == JOB_CONN) job = JOB_MOVE;
            else if (job == JOB_MOVE) {
                if (kv == 1) job = JOB_DIRECT;
                else { --kv; job = JOB_CONN; }
            } else job = JOB_SOURCE;
        }

        const unsigned live = __ballot_sync(kFull, mode != M_EXIT);
        if (live == 0) break;
        const int thr = max(1, (__popc(live) * A.idle_sweep + 16) >> 5);
        if (__any_sync(kFull, mode == M_SWEEP)) {
            for (;;) {
                if (mode == M_SWEEP) {
                    const int rr = sweep_point<FK, FA>(w, P, A, sbase, s, acc);
                    ++pts;
                    if (rr == 1) { mode = M_DISC; after = true; }
                    else if (rr == 2) {
                        mode = M_DISC;
                        ++nskip;
                        if (job == JOB_CONN) job = JOB_MOVE;
                        else if (job == JOB_MOVE) {
                            if (kv == 1) job = JOB_DIRECT;
                            else { --kv; job = JOB_CONN; }
                        } else job = JOB_SOURCE;
                    }
                }
                const unsigned idle = __ballot_sync(kFull, mode == M_DISC);
                if (__popc(idle) >= thr || !__any_sync(kFull, mode == M_SWEEP)) break;
            }
        }
    }
    atomicAdd(A.cnt + ADJ_POINTS, (unsigned long long)pts);
    atomicAdd(A.cnt + ADJ_SPLATS, nspl);
    atomicAdd(A.cnt + ADJ_SKIPPED, nskip);
}

}  // namespace smp
