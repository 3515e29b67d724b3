/*
 * simpler_b200.h -- C ABI of libsimpler_b200.so, the B200 (sm_100a) photon march of
 * simplEr's refractive radiative transfer renderer.
 *
 * Everything crossing this boundary is plain C: POD descriptors of doubles/ints, host
 * pointers and sizes, no C++ or torch types. Every entry point returns SMP_OK (0) or a
 * negative smp_status; the text of the last error of the calling thread is returned by
 * smp_last_error(). No entry point exits, asserts or prints.
 *
 * Units are the reference's: metres, Hz, m/s, radians.
 *
 * Reference interfaces replaced (paths relative to the simplEr project root):
 *   smp_render / smp_plan_render   <- cuda::CudaRenderer::renderImage      renderer/include/cuda_renderer.h:28-40
 *                                   <- photon::Renderer::renderImage        renderer/include/photon.h:82-84,
 *                                                                           renderer/src/photon.cpp:267-340
 *   smp_plan_create                <- cuda::CudaRenderer::setup             renderer/src/cuda_renderer.cu:745-786
 *   smp_plan_destroy               <- cuda::CudaRenderer::cleanup           renderer/src/cuda_renderer.cu:788-793
 *   smp_trace_photons              <- the per-photon body of renderImage    renderer/src/photon.cpp:302-335
 *                                     (directTracing :41-87, scatter :91-136) with the uniform stream
 *                                     injected instead of smp::Sampler (renderer/include/sampler.h:19-20)
 *   smp_field_eval                 <- US::RIF / US::dRIF                    renderer/include/cuda_scene.cuh:463-481
 *   smp_texture_cdf                <- area_textured_source texture CDF      renderer/src/area_textured_source.cpp:41-45
 *   smp_render_batch               <- the serial per-configuration loops    renderer/pybindFiles/tests/FUS_configurations.ipynb
 *                                     (one renderImage per configuration)   (cells at lines 591-603, 713-725)
 *   smp_batch_tune_steps /         <- no counterpart: the reference's ER step is a fixed setting
 *   smp_plan_tune_step
 *   smp_render_adjoint /           <- no counterpart: the reference has forward-mode tangents of
 *   smp_plan_adjoint                  single leapfrog steps only (er_derivativestep scene.cpp:351-359,
 *                                     bessel_HessianRIF :259-320, Spline::hessian spline.h:359-413),
 *                                     used by no render path
 */
#ifndef SIMPLER_B200_H_
#define SIMPLER_B200_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SMP_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------------------------- */
typedef enum smp_status {
    SMP_OK              =  0,
    SMP_ERR_BAD_ARG     = -1,   /* invalid descriptor / size / pointer                      */
    SMP_ERR_CUDA        = -2,   /* a CUDA runtime call failed (text in smp_last_error)       */
    SMP_ERR_STEP_CAP    = -3,   /* at least one photon hit the per-photon ER-step cap         */
    SMP_ERR_NAN         = -4,   /* a non-finite position / direction was produced             */
    SMP_ERR_STREAM      = -5,   /* an injected uniform stream ran out for some photon         */
    SMP_ERR_NO_DEVICE   = -6,   /* no CUDA device, or not an sm_100 device                    */
    SMP_ERR_OOM         = -7,   /* device allocation failed                                   */
    SMP_ERR_UNSUPPORTED = -8    /* option combination not built                               */
} smp_status;

/* ---- refractive-index field ---------------------------------------------------------------- */
typedef enum smp_field_type {
    SMP_FIELD_BESSEL    = 0,  /* rif_analytical: n_o + n_max*s*J_m(k r) cos(m phi)   scene.cpp:205-257   */
    SMP_FIELD_SOURCES   = 1,  /* rif_sources: spherical point sources on two arcs    scene.cpp:139-195   */
    SMP_FIELD_PLANEWAVE = 2,  /* n_o + sum_i a_i sin(k_i.x - tau + phase_i) (not in the reference)        */
    SMP_FIELD_SPLINE    = 3   /* rif_interpolated: tricubic B-spline              spline.h:308-448    */
} smp_field_type;

#define SMP_MAX_WAVES 8

typedef struct smp_field_desc {
    int32_t type;                 /* smp_field_type */
    int32_t precision;            /* refinement levels of traceTillBlock (rif_base.h:28)            */
    /* common (rif_base.h:10-32, recompute_derived_ :144-154) */
    double  f_u;                  /* ultrasound frequency (Hz)                                      */
    double  speed_u;              /* ultrasound speed (m/s); k = 2*pi*f_u/speed_u                   */
    double  n_o;                  /* baseline refractive index                                      */
    double  er_stepsize;          /* ER step (m)                                                    */
    double  egap_end_x;           /* field is n_o, grad 0 for x > egap_end_x   (rif_base.h:134-137) */
    double  sgap_begin_x;         /*                      or  x < sgap_begin_x                      */
    double  direct_tol;           /* carried for the settings round trip; unused on the path        */
    double  rr_weight;            /* carried; unused on the path                                    */
    int32_t use_initialization_hack; /* carried; unused on the path                                 */
    /* Bessel (rif_analytical.h:168-175) */
    int32_t mode;                 /* Bessel order 0 <= m <= 64 (orders above 2 need k r <= 128 over
                                     the medium box)                                                */
    double  n_max, n_clip, phi_min, phi_max;
    /* FUS point sources (rif_sources.h:18-45) */
    int32_t n_coeff;              /* triangle-wave harmonics                                        */
    int32_t theta_sources, trans_z_sources;
    int32_t active1, active2;
    int32_t _pad0;
    double  n_scaling, radius, chordlength, phase1, phase2;
    double  center1[3], center2[3];
    /* plane waves (new field type): n = n_o + sum_i a_i sin(k_i . x - tau + phase_i),
       tau = phi_min + (phi_max - phi_min) * u is the per-photon temporal phase drawn where the
       reference draws its Bessel 'scaling' (photon.cpp:324) */
    int32_t n_waves;
    int32_t _pad1;
    double  wave_amp[SMP_MAX_WAVES];
    double  wave_k[SMP_MAX_WAVES][3];
    double  wave_phase[SMP_MAX_WAVES];
    /* tricubic B-spline over a regular grid (spline.h); coefficients are already prefiltered
       (smp_spline_prefilter), x fastest: c[x + Nx*(y + Ny*z)]; host pointer, float */
    int32_t grid_n[3];
    int32_t _pad2;
    double  grid_min[3], grid_max[3];
    const float *grid_coeff;
    /* FUS source arcs given explicitly, as the Scene constructor takes them (scene.h:78-95):
       used when theta_max > theta_min, else derived from chordlength as
       renderer3d_sample.cpp:136-140 does (theta = -+asin(chord/2r), trans_z = -+chord/2) */
    double  theta_min, theta_max, trans_z_min, trans_z_max;
    /* spline: a value added to every grid_coeff entry (in double), so that a grid of a small
       field on a large background (n_o + dn, dn ~ 1e-5) keeps dn's full float precision; 0 for the
       reference's absolute grids */
    double  grid_offset;
} smp_field_desc;

/* ---- scene: medium box, textured collimated source, sensor --------------------------------- */
typedef struct smp_scene_desc {
    double  ior;                  /* medium ior for the boundary BSDF and entry Fresnel (scene.h:47)*/
    double  medium_l[3], medium_r[3];
    /* source (area_textured_source.h:20-30) */
    double  light_origin[3], light_dir[3];
    double  half_theta_limit;
    double  light_plane[2];
    double  Li;
    int32_t tex_x, tex_y;         /* texture resolution                                             */
    const double *texture;        /* tex_x*tex_y texels, index y*tex_x + x, rows as stored after the
                                     PFM bottom-to-top flip (image.h:183-245); host pointer         */
    double  emitter_lens_origin[3];
    double  emitter_lens_aperture, emitter_lens_focal_length;
    int32_t emitter_lens_active;
    /* camera (camera.cpp:11-29) */
    int32_t use_bounce_decomposition;
    double  view_origin[3], view_dir[3], view_horizontal[3];
    double  view_plane[2];
    double  pathlength_range[2];  /* (-1,-1) = no binning                                           */
    double  sensor_lens_origin[3];
    double  sensor_lens_aperture, sensor_lens_focal_length;
    int32_t sensor_lens_active;
    /* film (image.h Image3 x_res, y_res, z_res) */
    int32_t x_res, y_res, z_res;
    int32_t _pad0;
} smp_scene_desc;

/* ---- medium (medium.h:24-38) + Henyey-Greenstein g (phase.cpp) ----------------------------- */
typedef struct smp_medium_desc {
    double sigma_t, albedo, g;
} smp_medium_desc;

/* ---- renderer options (photon.h:27-32 plus the B200 choices) ------------------------------- */
typedef enum smp_rng {
    SMP_RNG_SFMT   = 0,   /* SFMT-19937 seeded per photon with (seed + photon index), as
                             photon.cpp:313: the reference CPU's own stream                      */
    SMP_RNG_PHILOX = 1,   /* Philox-4x32-10 keyed by (seed, photon index): no state in memory     */
    SMP_RNG_STREAM = 2    /* injected per-photon uniforms (smp_trace_photons only)                */
} smp_rng;

typedef enum smp_precision {
    SMP_PREC_FP32  = 0,   /* FP32 march, FP32 path length, FP32 image atomics (the reference GPU)  */
    SMP_PREC_MIXED = 1    /* FP32 march, FP64 path-length accumulator, FP64 image atomics         */
} smp_precision;

typedef struct smp_render_opts {
    int32_t  max_depth;           /* -1 = unlimited (photon.h:111)                                  */
    int32_t  use_direct;          /* photon.h:113                                                   */
    int32_t  use_angular_sampling;/* photon.h:114                                                   */
    int32_t  rng;                 /* smp_rng                                                        */
    int32_t  precision;           /* smp_precision                                                  */
    int32_t  device;              /* CUDA ordinal                                                   */
    double   max_pathlength;      /* -1 = unlimited (photon.h:112)                                  */
    uint64_t seed;                /* photon i uses stream (seed + i); seed 0 == the reference       */
    int64_t  step_cap;            /* per-photon ER-step cap (0 = default 1e7); the reference has none */
    int32_t  block_size;          /* 0 = autotuned / default                                        */
    int32_t  blocks_per_sm;       /* 0 = default                                                    */
    /* Path budget of one sensor march (movePhotonTillSensor's LargeDist, scene.cpp:627, fixed at
       1e4 m in the reference). > 0: that many metres. 0: min(1e4, 110/sigma_t), beyond which the
       march's contribution weight*exp(-sigma_t*d) is exactly 0 in FP32, so a photon trapped by
       total internal reflection stops there instead of marching 1e4 m. */
    double   sensor_march_max;
    int32_t  kernel;              /* smp_kernel: which kernel traces the photons (0 = the default)   */
    /* Spline fields on the slot pool: 1 stages the coefficient grid in bricks of 16^3 cells in
       shared memory with the Tensor Memory Accelerator and bins the march lists by brick; 0 (the
       default) reads the taps through the L1 cache. Both give the same photons. The march is bound
       by the L1/shared-memory data path either way (16 random 16-byte gathers per evaluation), and
       the staged bricks' shared-memory gathers conflict in banks and halve the resident warps, so the
       default is measurably faster on B200. */
    int32_t  spline_bricks;
} smp_render_opts;

/* Kernels that trace a plan's photons. All three run the same per-photon arithmetic, so their
   photons are identical; they differ in scheduling. */
typedef enum smp_kernel {
    SMP_KERNEL_POOL       = 0,    /* the default: march and event kernels alternating over a
                                     resident pool of photon slots, with a persistent tail kernel  */
    SMP_KERNEL_PERSISTENT = 1,    /* one persistent launch; each lane runs its photons to the end
                                     and takes the next index from a global counter                */
    SMP_KERNEL_PLAIN      = 2     /* one thread per photon in one launch, no regeneration: the
                                     reference GPU renderer's structure (cuda_renderer.cu:681-725) */
} smp_kernel;

typedef struct smp_stats {
    int64_t photons;              /* photons traced                                                 */
    int64_t er_steps;             /* accepted + rejected er_step evaluations                        */
    int64_t splats;               /* addEnergyToImage calls that reached the film                   */
    int64_t step_cap_hits;        /* photons stopped by step_cap                                    */
    int64_t nan_photons;          /* photons stopped by a non-finite state                          */
    int64_t stream_exhausted;     /* photons whose injected stream ran out                          */
    double  kernel_ms;            /* device time of the trace(s): every kernel, first to last       */
    double  march_ms;             /* device time inside the ER-march kernel alone                   */
    int64_t march_steps;          /* er_step evaluations executed by that kernel                    */
    int64_t launches;             /* kernels launched                                               */
    int64_t march_launches;       /* of which ER-march kernel launches                              */
    /* the slot pool's schedule of the last trace (smp_plan_tune): march-kernel block size, slots
       per march lane, chunk (ER steps per slot per march launch; 0 while it was still being tuned
       online), and 1 when the plan was tuned */
    int32_t march_block, slots_per_lane, chunk, tuned;
} smp_stats;

/* ---- parity records (smp_trace_photons) ---------------------------------------------------- */
#define SMP_TRACE_MAX_SPLATS 8

typedef enum smp_photon_end {
    SMP_END_GENRAY_FAIL = 1,      /* source ray missed the emitter lens aperture                    */
    SMP_END_NO_SCATTER  = 2,      /* first albedo roulette failed (or albedo 0)                     */
    SMP_END_ESCAPED     = 3,      /* refracted out through a face in movePhoton                     */
    SMP_END_ABSORBED    = 4,      /* albedo roulette killed the photon at a vertex                  */
    SMP_END_MAX_DEPTH   = 5,      /* maxDepth / maxPathlength reached                               */
    SMP_END_STEP_CAP    = 6,
    SMP_END_NAN         = 7,
    SMP_END_STREAM      = 8
} smp_photon_end;

typedef struct smp_splat_record {
    float   p[3];                 /* position handed to addEnergyToImage (sensor plane)             */
    int32_t depth;                /* 0 = direct                                                     */
    double  pathlength;           /* optical path length used for the z bin                         */
    double  value;                /* totalPhotonValue before the bilinear split                     */
} smp_splat_record;

typedef struct smp_photon_record {
    int64_t photon;
    int32_t end;                  /* smp_photon_end                                                 */
    int32_t draws;                /* uniforms consumed                                              */
    int32_t depth;                /* depth when the photon ended                                    */
    int32_t n_splats;             /* splat events (may exceed SMP_TRACE_MAX_SPLATS)                 */
    float   pos[3];               /* photon position at termination                                 */
    float   dir[3];               /* photon optical direction v = n*omega at termination            */
    double  total_optical;        /* the photon's running optical path length at termination        */
    int64_t er_steps;
    smp_splat_record splats[SMP_TRACE_MAX_SPLATS];
} smp_photon_record;

/* ---- batched sweep: many field / medium configurations in one launch --------------------- */
typedef struct smp_instance_desc {
    smp_field_desc  field;        /* per-instance field (Bessel / plane wave)                       */
    smp_medium_desc medium;
    int64_t         n_photons;    /* this instance's budget                                         */
    uint64_t        seed;
} smp_instance_desc;

/* ---- opaque plan ---------------------------------------------------------------------------- */
typedef struct smp_plan smp_plan;

/* library */
int         smp_version(void);
const char *smp_last_error(void);
int         smp_device_count(void);
/* sizes of the descriptor structs, so foreign-language mirrors can check their layout */
size_t      smp_sizeof(const char *type_name);

/* One-shot render (the reference's CudaRenderer::renderImage): uploads the scene, traces
   n_photons, writes the x*y*z image (index z*X*Y + y*X + x) to the caller-owned host buffer
   image_out (overwritten, as cuda_renderer.cu:732-739 does), frees everything. */
int smp_render(const smp_scene_desc *scene, const smp_medium_desc *medium,
               const smp_field_desc *field, const smp_render_opts *opts,
               int64_t n_photons, double *image_out, smp_stats *stats_out);

/* Plans keep the scene, texture CDF, field data and film resident on the device so repeated
   renders pay no setup. */
int smp_plan_create(const smp_scene_desc *scene, const smp_medium_desc *medium,
                    const smp_field_desc *field, const smp_render_opts *opts, smp_plan **plan_out);
int smp_plan_destroy(smp_plan *plan);
/* change per-render scalars, as the pybind setters set_f_u / set_n_max / set_n_scaling /
   set_phase1 / set_phase2 do (renderer/include/scene.h:179-219) */
int smp_plan_set_field(smp_plan *plan, const smp_field_desc *field);
/* Render photons [first_photon, first_photon + n_photons) into the plan's device film
   (accumulating; the film is zeroed by smp_plan_clear). Asynchronous on 'stream'
   (a cudaStream_t, NULL = legacy default stream). weight_photons is the N of Li*T/N
   (photon.h:76-80); pass the total photon count of the render. */
int smp_plan_clear(smp_plan *plan, void *stream);
int smp_plan_trace(smp_plan *plan, int64_t first_photon, int64_t n_photons,
                   int64_t weight_photons, void *stream);
/* Copy the film out as doubles (host or device destination). Synchronises 'stream'. */
int smp_plan_read_image(smp_plan *plan, double *dst, int dst_is_device, void *stream);
/* Device pointer of the film (float or double per smp_render_opts.precision) and its dtype
   (4 or 8 bytes per pixel), for zero-copy torch views. */
int smp_plan_film(smp_plan *plan, void **dev_ptr, int32_t *bytes_per_pixel);
int smp_plan_stats(smp_plan *plan, smp_stats *stats_out);
/* Whole render through a plan: clear, trace [0,n), read back to host. */
int smp_plan_render(smp_plan *plan, int64_t n_photons, double *image_out, smp_stats *stats_out);

/* Autotuner (no counterpart in the reference): times trial traces of n_sample photons (photons
   [0, n_sample) of this plan's render) over the slot pool's march-kernel block size (128, 256),
   resident slots per march lane (2-8) and chunk (ER steps per slot per march launch, 64-192; a sample
   slower than about 400 ms per trial is scaled down), keeps the fastest (the two best timed twice)
   for the plan and caches it per process under the device, field kind, precision, film,
   medium, field, scene and sample size, so a later plan of the same configuration takes it without
   trials. The trials render into the plan's film, which is cleared on return: tune before tracing.
   Plans that are not tuned keep their defaults and tune the chunk alone, online, while they trace. */
typedef struct smp_tuning {
    int32_t march_block;          /* threads per march-kernel block                                 */
    int32_t slots_per_lane;       /* resident photon slots per march lane                           */
    int32_t chunk;                /* ER steps per slot per march launch                             */
    int32_t trials;               /* configurations timed (0: taken from the cache)                 */
    double  ms;                   /* device time of the chosen configuration's trial trace          */
    double  paths_per_s;          /* its photon paths/s                                             */
} smp_tuning;
int smp_plan_tune(smp_plan *plan, int64_t n_sample, smp_tuning *out);

/* Step-size autotuner for a plan (no counterpart in the reference, whose ER step is a fixed
   setting): renders photons [0, n_sample) of the plan's render at its field's own ER step (the
   reference film) and at multiples of it (2, 3, 4, 6, 8, 12, 16, 24 or 32), on the same photons, and
   sets the plan's step to the largest multiple whose film stays within rmse_budget relative RMSE
   (sqrt(sum (film - ref)^2 / sum ref^2)) of the reference film -- the largest allowed multiple
   first, then bisection, as smp_batch_tune_steps. The search renders in the mixed form, as there: a
   plan of the FP32 form searches on a mixed-form copy of itself, except a spline plan (its
   coefficients are the caller's host memory), which searches in its own form, where the float path
   length's rounding counts against the budget too. The step stays at most an eighth of the field's
   shortest wavelength (Bessel, plane waves, point sources at their highest harmonic) or a quarter
   of a spline grid's finest spacing. Unless opts.sensor_march_max is set, the tuner's renders stop a
   sensor march at 30 mean free paths (all films alike). *step_out receives the plan's new step,
   rmse_out (may be NULL) the error measured at it. The film is cleared on return; a second call
   starts again from the field's own step; smp_plan_set_field restores that step. Not for batched
   sweeps. */
int smp_plan_tune_step(smp_plan *plan, int64_t n_sample, double rmse_budget, double *step_out, double *rmse_out);

/* Parity mode: traces n_photons with per-photon injected uniforms
   (photon i consumes uniforms[offsets[i] .. offsets[i+1]) ), or with the opts->rng stream when
   uniforms == NULL, and returns one record per photon. Also accumulates the image into image_out
   (host, may be NULL). weight_photons as in smp_plan_trace. */
int smp_trace_photons(const smp_scene_desc *scene, const smp_medium_desc *medium,
                      const smp_field_desc *field, const smp_render_opts *opts,
                      int64_t first_photon, int64_t n_photons, int64_t weight_photons,
                      const float *uniforms, const int64_t *offsets,
                      smp_photon_record *records_out, double *image_out);

/* Field probe: n(p) and grad n(p) at n_points host points (xyz interleaved) for a given
   temporal scaling, with the kernel's own device code. */
int smp_field_eval(const smp_field_desc *field, double scaling, int64_t n_points,
                   const double *points, double *n_out, double *grad_out);

/* Texture CDF exactly as area_textured_source builds it (float accumulate + normalise),
   tex_x*tex_y+1 entries. */
int smp_texture_cdf(const double *texture, int32_t tex_x, int32_t tex_y, float *cdf_out);

/* B-spline prefilter (spline.h:686-764, mirror boundary) of samples -> coefficients, float. */
int smp_spline_prefilter(const float *samples, const int32_t n[3], float *coeff_out);

/* Batched sweep: n_inst instances sharing one scene/film shape, traced in one persistent
   launch; images_out holds n_inst consecutive films (host). */
int smp_render_batch(const smp_scene_desc *scene, const smp_instance_desc *instances,
                     int32_t n_inst, const smp_render_opts *opts,
                     double *images_out, smp_stats *stats_out);

/* Step-size autotuner for a batched sweep (no counterpart in the reference, whose ER step is a fixed
   setting). For each instance it renders photons [0, min(n_photons, n_sample)) at the instance's own
   field.er_stepsize (the reference film) and at multiples of that step (2, 3, 4, 6, 8, 12, 16, 24 or
   32, none above an eighth of the instance's ultrasound wavelength speed_u / f_u), on the same
   Philox photons, and keeps the largest multiple whose film stays within rmse_budget relative RMSE
   (sqrt(sum (film - ref)^2 / sum ref^2)) of the reference film. These renders are all in the mixed
   form (FP64 path length and film), whatever opts->precision says: in the FP32 form the float path
   length rounds differently at every step, the own one included, and moves photons across
   path-length bins, which the step does not cause and the FP32 render keeps at any step. It tries
   the largest allowed multiple first and, where that misses, bisects between the multiples known to
   pass and to miss (the error grows with the step); each round is one batched render of the
   instances still searching. An instance that misses at every multiple and has more than n_sample
   photons searches once more with 10 n_sample photons (a small film led by a few large splats moves
   by about the same amount at any step change, which more photons average out). An instance with
   no photons or an empty reference film keeps its own step. Unless opts->sensor_march_max is set,
   the tuner's renders stop a sensor march at 30 mean free
   paths of the thinnest medium, which cuts the compared films alike by less than e^-30 of a photon's
   weight and shortens the rounds' tails. steps_out[i] receives instance i's chosen er_stepsize;
   rmse_out[i] (may be NULL) the relative RMSE measured at that step (0 where the instance kept its
   own); rounds_out (may be NULL) the number of batched renders. Set
   instances[i].field.er_stepsize = steps_out[i] and call smp_render_batch. Instances are tuned in
   groups that fit in 40 % of the free device memory at 16 bytes per film pixel each (SMP_ERR_OOM
   when not even one fits). */
int smp_batch_tune_steps(const smp_scene_desc *scene, const smp_instance_desc *instances,
                         int32_t n_inst, const smp_render_opts *opts, int64_t n_sample,
                         double rmse_budget, double *steps_out, double *rmse_out, int32_t *rounds_out);

/* Rendering without allocation -- no counterpart in the reference. For callers that cannot call
   cudaMalloc (device memory owned by the host application's allocator or budget, code that must not
   hit cudaMalloc/cudaFree's device-wide synchronisation mid-frame, plugin hosts that hand over only
   the buffers the renderer may touch). Traces photons [first_photon, first_photon + n_photons)
   with Philox streams into the caller's device film d_film (float per pixel for SMP_PREC_FP32,
   double for SMP_PREC_MIXED, Image3 layout, accumulated -- zero it first for a fresh render) on
   'stream', and returns after the trace has finished. It allocates nothing: the work counter,
   statistics, Bessel table and texture CDF live in a fixed 1 MiB device array that every GPU
   loading this library holds until the process exits. Limits: texture CDF + Bessel table within the 1 MiB (a 501x501 texture fits);
   Bessel fields of order 0-2 and plane-wave fields; larger inputs are rejected with
   SMP_ERR_BAD_ARG / SMP_ERR_UNSUPPORTED. All calls on a device share that array and each call
   overwrites what the last one left there. Calls whose GPU work overlapped would race on it, so
   each call holds a process-wide lock until its own GPU work has finished: calls from several
   threads or streams run one after another. The first call on each device looks up the array's
   device address, so make it before any stream capture. The caller's current device is restored
   on return. stats_out (may be NULL) receives photon, step and splat counts; kernel_ms is not
   measured. */
int smp_render_noalloc(const smp_scene_desc *scene, const smp_medium_desc *medium,
                       const smp_field_desc *field, const smp_render_opts *opts,
                       int64_t first_photon, int64_t n_photons, int64_t weight_photons,
                       void *d_film, void *stream, smp_stats *stats_out);

/* ---- adjoint: gradient of a sensor objective with respect to the field's parameters ---------- */
typedef struct smp_adjoint_stats {
    int64_t photons;              /* photons differentiated                                         */
    int64_t dropped;              /* photons left out: more scatter vertices than the checkpoint
                                     buffer holds, or a move longer than the trajectory buffer      */
    int64_t skipped;              /* sensor marches (direct, connections) left out: longer than the
                                     trajectory buffer (SMP_ADJ_TCAP accepted steps, default 8192);
                                     their value carries exp(-sigma_t d) of that length            */
    int64_t aborted;              /* photons left out: step cap or non-finite state                 */
    int64_t replay_mismatch;      /* segment replays that did not reproduce their checkpoint (0)    */
    int64_t er_steps_forward;     /* er_step evaluations of the checkpointing trace                 */
    int64_t er_steps_replay;      /* er_step evaluations of the segment replays                     */
    int64_t points;               /* trajectory points swept backwards                              */
    int64_t splats;               /* splats whose value entered the objective                       */
    double  kernel_ms;            /* device time of the adjoint, both kernels, all batches          */
    double  trace_ms;             /* of which the checkpointing trace                               */
    int64_t launches;             /* kernels launched (the trace's per batch, a replay and a sweep
                                     per round)                                                     */
    double  replay_ms;            /* of kernel_ms: the segment replays                              */
    double  sweep_ms;             /* of kernel_ms: the backward sweeps                              */
} smp_adjoint_stats;
/* Number of parameters smp_render_adjoint returns for this field, or a negative smp_status:
   Bessel modes 0-2: 3 (n_max, phi_min, phi_max); plane waves 2*n_waves (amplitudes
   a_0..a_{W-1}, then phases phase_0..phase_{W-1}); spline grid_n[0]*grid_n[1]*grid_n[2]
   coefficients in grid_coeff's order. */
int64_t smp_adjoint_param_count(const smp_field_desc *field);
/* Gradient of J = sum_pixels dJ_dfilm[pixel] * film[pixel] with respect to the field parameters,
   where film is the image smp_render would produce for photons [first_photon, first_photon +
   n_photons) with the same opts (Philox streams, same seed; weight_photons as in smp_plan_trace).
   It is the pathwise derivative of that estimator: per photon, random numbers, discrete events
   and ER step sequences are held fixed, and marches ending on a face end on the face plane.
   dJ_dfilm: host, X*Y*Z doubles (Image3 layout); grad_out: host, smp_adjoint_param_count doubles,
   overwritten. Bessel (modes 0-2), plane-wave and spline fields, Philox streams, no lenses; others
   return SMP_ERR_UNSUPPORTED. Synchronous. Device memory, sized at the plan's first adjoint and
   kept by the plan: photons are differentiated in batches of 2^22 (2^21 when less than 64 GiB is
   free), each with 16 checkpoints per photon in its pool, and the replayed trajectories go through
   a buffer of a quarter of the free memory, 1-40 GiB (environment: SMP_ADJ_BATCH photons,
   SMP_ADJ_TRAJ_MB MiB, SMP_ADJ_POOL_PER_PHOTON); a smaller buffer only means more replay rounds. */
int smp_plan_adjoint(smp_plan *plan, int64_t first_photon, int64_t n_photons, int64_t weight_photons,
                     const double *dJ_dfilm, double *grad_out, smp_adjoint_stats *stats_out);
int smp_render_adjoint(const smp_scene_desc *scene, const smp_medium_desc *medium,
                       const smp_field_desc *field, const smp_render_opts *opts, int64_t n_photons,
                       const double *dJ_dfilm, double *grad_out, smp_adjoint_stats *stats_out);
/* Measurement utility with no counterpart in the reference: the device's FP32 FMA throughput
   (TFLOP/s, 2 FLOP per FMA) measured with independent FMA chains on every SM; the roofline
   denominator for the march, which is bound by the FP32 and issue pipes. */
int smp_fp32_peak(int device, double *tflops_out);

#ifdef __cplusplus
}
#endif

#endif /* SIMPLER_B200_H_ */
