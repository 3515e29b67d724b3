"""ctypes mirror of include/simpler_b200.h and loader for libsimpler_b200.so.

The structs here must match the C header byte for byte; ``check_layout()`` compares every
``sizeof`` with the library's own ``smp_sizeof``.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsimpler_b200.so")

SMP_MAX_WAVES = 8
SMP_TRACE_MAX_SPLATS = 8

# status codes
SMP_OK = 0
SMP_ERR_BAD_ARG = -1
SMP_ERR_CUDA = -2
SMP_ERR_STEP_CAP = -3
SMP_ERR_NAN = -4
SMP_ERR_STREAM = -5
SMP_ERR_NO_DEVICE = -6
SMP_ERR_OOM = -7
SMP_ERR_UNSUPPORTED = -8

FIELD_BESSEL, FIELD_SOURCES, FIELD_PLANEWAVE, FIELD_SPLINE = 0, 1, 2, 3
RNG_SFMT, RNG_PHILOX, RNG_STREAM = 0, 1, 2
PREC_FP32, PREC_MIXED = 0, 1
KERNEL_POOL, KERNEL_PERSISTENT, KERNEL_PLAIN = 0, 1, 2

END_NAMES = {1: "GENRAY_FAIL", 2: "NO_SCATTER", 3: "ESCAPED", 4: "ABSORBED", 5: "MAX_DEPTH",
             6: "STEP_CAP", 7: "NAN", 8: "STREAM"}

D3 = C.c_double * 3
D2 = C.c_double * 2


class FieldDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("precision", C.c_int32),
        ("f_u", C.c_double), ("speed_u", C.c_double), ("n_o", C.c_double), ("er_stepsize", C.c_double),
        ("egap_end_x", C.c_double), ("sgap_begin_x", C.c_double),
        ("direct_tol", C.c_double), ("rr_weight", C.c_double),
        ("use_initialization_hack", C.c_int32),
        ("mode", C.c_int32),
        ("n_max", C.c_double), ("n_clip", C.c_double), ("phi_min", C.c_double), ("phi_max", C.c_double),
        ("n_coeff", C.c_int32), ("theta_sources", C.c_int32), ("trans_z_sources", C.c_int32),
        ("active1", C.c_int32), ("active2", C.c_int32), ("_pad0", C.c_int32),
        ("n_scaling", C.c_double), ("radius", C.c_double), ("chordlength", C.c_double),
        ("phase1", C.c_double), ("phase2", C.c_double),
        ("center1", D3), ("center2", D3),
        ("n_waves", C.c_int32), ("_pad1", C.c_int32),
        ("wave_amp", C.c_double * SMP_MAX_WAVES),
        ("wave_k", (C.c_double * 3) * SMP_MAX_WAVES),
        ("wave_phase", C.c_double * SMP_MAX_WAVES),
        ("grid_n", C.c_int32 * 3), ("_pad2", C.c_int32),
        ("grid_min", D3), ("grid_max", D3),
        ("grid_coeff", C.POINTER(C.c_float)),
        ("theta_min", C.c_double), ("theta_max", C.c_double),
        ("trans_z_min", C.c_double), ("trans_z_max", C.c_double),
        ("grid_offset", C.c_double),
    ]


class SceneDesc(C.Structure):
    _fields_ = [
        ("ior", C.c_double),
        ("medium_l", D3), ("medium_r", D3),
        ("light_origin", D3), ("light_dir", D3),
        ("half_theta_limit", C.c_double),
        ("light_plane", D2),
        ("Li", C.c_double),
        ("tex_x", C.c_int32), ("tex_y", C.c_int32),
        ("texture", C.POINTER(C.c_double)),
        ("emitter_lens_origin", D3),
        ("emitter_lens_aperture", C.c_double), ("emitter_lens_focal_length", C.c_double),
        ("emitter_lens_active", C.c_int32),
        ("use_bounce_decomposition", C.c_int32),
        ("view_origin", D3), ("view_dir", D3), ("view_horizontal", D3),
        ("view_plane", D2),
        ("pathlength_range", D2),
        ("sensor_lens_origin", D3),
        ("sensor_lens_aperture", C.c_double), ("sensor_lens_focal_length", C.c_double),
        ("sensor_lens_active", C.c_int32),
        ("x_res", C.c_int32), ("y_res", C.c_int32), ("z_res", C.c_int32),
        ("_pad0", C.c_int32),
    ]


class MediumDesc(C.Structure):
    _fields_ = [("sigma_t", C.c_double), ("albedo", C.c_double), ("g", C.c_double)]


class RenderOpts(C.Structure):
    _fields_ = [
        ("max_depth", C.c_int32), ("use_direct", C.c_int32), ("use_angular_sampling", C.c_int32),
        ("rng", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32),
        ("max_pathlength", C.c_double),
        ("seed", C.c_uint64),
        ("step_cap", C.c_int64),
        ("block_size", C.c_int32), ("blocks_per_sm", C.c_int32),
        ("sensor_march_max", C.c_double),
        ("kernel", C.c_int32), ("spline_bricks", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("photons", C.c_int64), ("er_steps", C.c_int64), ("splats", C.c_int64),
        ("step_cap_hits", C.c_int64), ("nan_photons", C.c_int64), ("stream_exhausted", C.c_int64),
        ("kernel_ms", C.c_double), ("march_ms", C.c_double), ("march_steps", C.c_int64),
        ("launches", C.c_int64), ("march_launches", C.c_int64),
        ("march_block", C.c_int32), ("slots_per_lane", C.c_int32), ("chunk", C.c_int32), ("tuned", C.c_int32),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("march_block", C.c_int32), ("slots_per_lane", C.c_int32), ("chunk", C.c_int32), ("trials", C.c_int32),
        ("ms", C.c_double), ("paths_per_s", C.c_double),
    ]


class SplatRecord(C.Structure):
    _fields_ = [("p", C.c_float * 3), ("depth", C.c_int32), ("pathlength", C.c_double), ("value", C.c_double)]


class PhotonRecord(C.Structure):
    _fields_ = [
        ("photon", C.c_int64), ("end", C.c_int32), ("draws", C.c_int32), ("depth", C.c_int32),
        ("n_splats", C.c_int32),
        ("pos", C.c_float * 3), ("dir", C.c_float * 3),
        ("total_optical", C.c_double),
        ("er_steps", C.c_int64),
        ("splats", SplatRecord * SMP_TRACE_MAX_SPLATS),
    ]


class InstanceDesc(C.Structure):
    _fields_ = [("field", FieldDesc), ("medium", MediumDesc), ("n_photons", C.c_int64), ("seed", C.c_uint64)]


class AdjointStats(C.Structure):
    _fields_ = [
        ("photons", C.c_int64), ("dropped", C.c_int64), ("skipped", C.c_int64), ("aborted", C.c_int64),
        ("replay_mismatch", C.c_int64), ("er_steps_forward", C.c_int64), ("er_steps_replay", C.c_int64),
        ("points", C.c_int64), ("splats", C.c_int64), ("kernel_ms", C.c_double), ("trace_ms", C.c_double),
        ("launches", C.c_int64), ("replay_ms", C.c_double), ("sweep_ms", C.c_double),
    ]


STRUCTS = {
    "smp_field_desc": FieldDesc, "smp_scene_desc": SceneDesc, "smp_medium_desc": MediumDesc,
    "smp_render_opts": RenderOpts, "smp_stats": Stats, "smp_photon_record": PhotonRecord,
    "smp_splat_record": SplatRecord, "smp_instance_desc": InstanceDesc,
    "smp_adjoint_stats": AdjointStats, "smp_tuning": Tuning,
}

# every entry point declared in include/simpler_b200.h
EXPORTS = [
    "smp_version", "smp_last_error", "smp_device_count", "smp_sizeof", "smp_render",
    "smp_plan_create", "smp_plan_destroy", "smp_plan_set_field", "smp_plan_clear", "smp_plan_trace",
    "smp_plan_read_image", "smp_plan_film", "smp_plan_stats", "smp_plan_render", "smp_trace_photons",
    "smp_field_eval", "smp_texture_cdf", "smp_spline_prefilter", "smp_render_batch", "smp_fp32_peak",
    "smp_render_noalloc", "smp_adjoint_param_count", "smp_plan_adjoint", "smp_render_adjoint", "smp_plan_tune",
    "smp_batch_tune_steps", "smp_plan_tune_step",
]

_lib = None


class SmpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"simpler_b200 error {code}: {msg}")
        self.code = code


def load() -> C.CDLL:
    """Load libsimpler_b200.so. Raises if it has not been built: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m simpler_b200.build`")
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER
    vp = C.c_void_p
    lib.smp_version.restype = C.c_int
    lib.smp_last_error.restype = C.c_char_p
    lib.smp_device_count.restype = C.c_int
    lib.smp_sizeof.restype = C.c_size_t
    lib.smp_sizeof.argtypes = [C.c_char_p]
    lib.smp_render.argtypes = [P(SceneDesc), P(MediumDesc), P(FieldDesc), P(RenderOpts), C.c_int64, vp, P(Stats)]
    lib.smp_plan_create.argtypes = [P(SceneDesc), P(MediumDesc), P(FieldDesc), P(RenderOpts), P(vp)]
    lib.smp_plan_destroy.argtypes = [vp]
    lib.smp_plan_set_field.argtypes = [vp, P(FieldDesc)]
    lib.smp_plan_clear.argtypes = [vp, vp]
    lib.smp_plan_trace.argtypes = [vp, C.c_int64, C.c_int64, C.c_int64, vp]
    lib.smp_plan_read_image.argtypes = [vp, vp, C.c_int, vp]
    lib.smp_plan_film.argtypes = [vp, P(vp), P(C.c_int32)]
    lib.smp_plan_stats.argtypes = [vp, P(Stats)]
    lib.smp_plan_render.argtypes = [vp, C.c_int64, vp, P(Stats)]
    lib.smp_trace_photons.argtypes = [P(SceneDesc), P(MediumDesc), P(FieldDesc), P(RenderOpts), C.c_int64,
                                      C.c_int64, C.c_int64, vp, vp, P(PhotonRecord), vp]
    lib.smp_field_eval.argtypes = [P(FieldDesc), C.c_double, C.c_int64, vp, vp, vp]
    lib.smp_texture_cdf.argtypes = [vp, C.c_int32, C.c_int32, vp]
    lib.smp_spline_prefilter.argtypes = [vp, vp, vp]
    lib.smp_render_batch.argtypes = [P(SceneDesc), P(InstanceDesc), C.c_int32, P(RenderOpts), vp, P(Stats)]
    lib.smp_plan_tune_step.argtypes = [vp, C.c_int64, C.c_double, P(C.c_double), P(C.c_double)]
    lib.smp_batch_tune_steps.argtypes = [P(SceneDesc), P(InstanceDesc), C.c_int32, P(RenderOpts), C.c_int64,
                                         C.c_double, vp, vp, P(C.c_int32)]
    lib.smp_fp32_peak.argtypes = [C.c_int, P(C.c_double)]
    lib.smp_render_noalloc.argtypes = [P(SceneDesc), P(MediumDesc), P(FieldDesc), P(RenderOpts), C.c_int64, C.c_int64,
                                       C.c_int64, vp, vp, P(Stats)]
    lib.smp_plan_tune.argtypes = [vp, C.c_int64, P(Tuning)]
    lib.smp_adjoint_param_count.restype = C.c_int64
    lib.smp_adjoint_param_count.argtypes = [P(FieldDesc)]
    lib.smp_plan_adjoint.argtypes = [vp, C.c_int64, C.c_int64, C.c_int64, vp, vp, P(AdjointStats)]
    lib.smp_render_adjoint.argtypes = [P(SceneDesc), P(MediumDesc), P(FieldDesc), P(RenderOpts), C.c_int64, vp, vp,
                                       P(AdjointStats)]
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != SMP_OK:
        raise SmpError(rc, load().smp_last_error().decode())


def check_layout() -> dict:
    """Return {struct: (python sizeof, library sizeof)} and raise on mismatch."""
    lib = load()
    out = {}
    for name, cls in STRUCTS.items():
        a, b = C.sizeof(cls), lib.smp_sizeof(name.encode())
        out[name] = (a, b)
        if a != b:
            raise AssertionError(f"{name}: python {a} bytes, library {b} bytes")
    return out
