// kparams.h -- the parameter block every march launch receives by value (__grid_constant__):
// scene, medium, film, field and work range, already converted to the device's float layout.
// Shared by the host (capi.cu) and the device code (march.cuh).
#pragma once
#include <stdint.h>
#include "../../include/simpler_b200.h"

namespace smp {

// Field kernels are compiled per kind; the Bessel order is a compile-time constant for m <= 2.
enum FieldKind : int {
    FK_BESSEL0 = 0,
    FK_BESSEL1 = 1,
    FK_BESSEL2 = 2,
    FK_BESSELN = 3,
    FK_PLANEWAVE = 4,
    FK_SOURCES = 5,
    FK_SPLINE = 6,
    FK_BATCH = 7,           // Bessel modes 0-2 with per-instance parameters (batched sweep)
    FK_COUNT = 8
};

struct FieldParams {
    int kind;
    int mode;               // Bessel order
    float n_o;
    float egap, sgap;       // field is n_o outside sgap <= x <= egap
    float k_r;              // 2*pi*f/c
    float inv_k;            // 1/k_r
    float amp;              // Bessel n_max
    float max_scaling;      // n_clip / n_max
    float phi_min, phi_range;
    // plane waves
    int n_waves;
    float wamp[SMP_MAX_WAVES];
    float wk[SMP_MAX_WAVES][3];
    float wphase[SMP_MAX_WAVES];
    // FUS point sources: centres as float4 (xyz, unused), arc 1 then arc 2
    int n_coeff, nsources, active1, active2;
    float n_scaling, phase1, phase2;
    const float4 *centers;  // 2*nsources entries (arc 1 block, arc 2 block)
    // spline
    int N[3];
    float xmin[3], xres[3];
    float spline_base;      // coefficients are stored as offsets from this value
    const float *coeff;
    const float4 *coeff4;   // the same offsets as x-tap quads: coeff4[row * N0 + x] holds the
                            // coefficients at mirrored x-1, x, x+1, x+2 of that (y, z) row (NULL:
                            // read coeff tap by tap)
    // Bessel table: for interval i of width bh, btab[2i] / btab[2i+1] hold the cubics of J_m /
    // J_m+1 in f = x/bh - i; bint intervals, bnodes = 2 * bint float4 entries
    const float4 *btab;
    int bnodes, bint;
    float bh, binv_h;
    float kb;               // k_r / bh: table coordinate per metre of r
    float grad_bound;       // bound on |grad n|_1 anywhere (0: unknown)
};

#define SMP_MAX_REFINE 39

// One instance of a batched sweep: its field, ER step, medium, photon weight, film and seed. The
// scene (box, source, camera, film shape) and the number of refinement levels are shared by all
// instances.
struct Inst {
    FieldParams field;
    float sigma_t, albedo, mfp, g;
    float weight;           // Li T / N of this instance
    float large_dist;       // movePhotonTillSensor budget for this sigma_t
    void *film;             // this instance's film (X*Y*Z, float or double)
    unsigned long long seed;
    float h0;               // this instance's ER step
    float cur_tab[SMP_MAX_REFINE + 1];   // its refinement steps, as KParams::cur_tab
};

struct KParams {
    // medium box (block.cpp)
    float L[3], R[3];
    // the same box as exact float thresholds: p - L > -eps  <=>  p >= box_lo, R - p > -eps  <=>  p <= box_hi
    float box_lo[3], box_hi[3];
    // textured source (area_textured_source)
    float src_origin[3];
    float plane[2], pixsize[2];
    float ct;
    int tex_x, n_tex;
    const float *cdf;       // n_tex + 1 entries
    // Guide table of the CDF (NULL: none): for bucket b of 2^guide_bits in u, cdf_guide[b] is the
    // lower bound of b / 2^guide_bits in the CDF (b = 0 .. 2^guide_bits), cdf_guide[2^guide_bits + 1]
    // = n_tex + 1; the lower bound of any u in the bucket lies in [cdf_guide[b], cdf_guide[b + 1]].
    const int *cdf_guide;
    int guide_bits;
    int src_lens_active;
    float src_lens_origin[3], src_lens_sqap, src_lens_focal;
    // camera
    float cam_origin[3], cam_dir[3], cam_h[3], cam_v[3];
    float cam_plane[2];
    float pl_min, pl_max;
    int bounce;
    int cam_lens_active;
    float cam_lens_origin[3], cam_lens_sqap, cam_lens_focal;
    // smooth dielectric (ior1 = 1, ior2 = scene ior)
    float ior1, ior2;
    // medium
    float sigma_t, albedo, mfp, g;
    // renderer
    int max_depth;
    float max_pathlength;
    int use_direct, use_angular;
    float weight;
    float h0;
    float large_dist;       // movePhotonTillSensor path budget (LargeDist)
    int precision;          // refinement levels, <= SMP_MAX_REFINE
    float cur_tab[SMP_MAX_REFINE + 1];   // h0, h0/10, (h0/10)/10, ... as traceTillBlock divides in float
    int step_cap;
    // film
    void *film;
    int X, Y, Z;
    int fp64;               // SMP_PREC_MIXED: FP64 path length + FP64 film
    // uniforms
    int rng;
    unsigned long long seed;
    const float *stream;
    const long long *offsets;
    // work: photons [first_photon, first_photon + n_photons)
    long long first_photon, n_photons;
    unsigned long long *counters;     // device scratch, see Counter
    smp_photon_record *records;       // trace mode only (indexed by photon - first_photon)
    int event_batch;                  // lanes that must finish a march before the warp runs events
    FieldParams field;
    // batched sweep (FK_BATCH): photon k of the sweep belongs to instance i with
    // inst_first[i] <= k < inst_first[i+1] and is that instance's photon k - inst_first[i]
    const Inst *insts;
    const long long *inst_first;
    int n_inst;                       // 0 outside a batched sweep
};

enum Counter : int {
    CNT_NEXT_PHOTON = 0,   // work distribution (relative to first_photon)
    CNT_STEPS = 1,
    CNT_SPLATS = 2,
    CNT_STEP_CAP = 3,
    CNT_NAN = 4,
    CNT_STREAM = 5,
    CNT_PHOTONS = 6,
    CNT_STAGE_TIMEOUT = 7,   // a block gave up waiting for its shared-memory staging copy
    CNT_LOST = 8,            // live slots the tail kernel had no lane for (a host defect)
    CNT_MARCH_STEPS = 9,     // ER steps executed by the march kernel of the two-kernel path
    CNT_COUNT = 10
};

}  // namespace smp
