"""Render setups: the scene / medium / field / options the reference's front-ends assemble,
as C-ABI descriptors, plus the synthetic workloads of the benchmark configurations.

Geometry follows the reference's key=value front-end (renderer/samples/renderer3d_sample.cpp:801-866):
the source sits at x = mediumR.x + emitter_distance shooting along -x, the emitter lens at
mediumR.x, the sensor at x = mediumL.x - sensor_distance looking along -x with horizontal -y,
and the sensor lens at mediumL.x. Units are metres.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


def disk_texture(n: int = 501, r2: int = 63000) -> np.ndarray:
    """The reference's Disk_501.pfm texture: texel (x, y) is 1 where (x-c)^2+(y-c)^2 <= r2."""
    c = (n - 1) // 2
    yy, xx = np.mgrid[0:n, 0:n]
    return (((xx - c) ** 2 + (yy - c) ** 2) <= r2).astype(np.float64)


def bernoulli_texture(n: int = 64, p: float = 0.5, seed: int = 1) -> np.ndarray:
    """n x n Bernoulli(p) mask from numpy's default_rng(seed)."""
    return (np.random.default_rng(seed).random((n, n)) < p).astype(np.float64)


@dataclass
class Setup:
    """Everything one render needs, in the reference's parameter names (metres, Hz, m/s)."""
    # scene / geometry (renderer3d_sample.cpp:60-147)
    ior: float = 1.3333
    medium_l: tuple = (-0.005, -0.005, -0.005)
    medium_r: tuple = (0.005, 0.005, 0.005)
    half_theta_limit: float = 0.0
    emitter_size: float = 0.001
    sensor_size: float = 0.01
    emitter_distance: float = 0.0
    sensor_distance: float = 0.0
    Li: float = 75000.0
    texture: np.ndarray = field(default_factory=disk_texture)
    emitter_lens_aperture: float = 0.015
    emitter_lens_focal_length: float = 0.015
    emitter_lens_active: bool = False
    sensor_lens_aperture: float = 0.015
    sensor_lens_focal_length: float = 0.015
    sensor_lens_active: bool = False
    # film
    spatial_x: int = 128
    spatial_y: int = 128
    path_length_bins: int = 32
    path_length_min: float = 0.0
    path_length_max: float = 0.05
    use_bounce_decomposition: bool = False
    # medium
    sigma_t: float = 100.0 / 0.9
    albedo: float = 0.9
    g: float = 0.9
    # field (rif parameters)
    field_type: int = L.FIELD_BESSEL
    f_u: float = 848e3
    speed_u: float = 1500.0
    n_o: float = 1.3333
    n_max: float = 1e-3
    n_clip: float = 1e-3
    phi_min: float = 0.0
    phi_max: float = 2.0 * math.pi
    mode: int = 0
    er_stepsize: float = 1e-5
    precision: int = 4
    emitter_gap: float = 0.0
    sensor_gap: float = 0.0
    direct_tol: float = 1e-5
    rr_weight: float = 1e-2
    use_initialization_hack: bool = False
    # FUS sources
    n_scaling: float = 0.05e-3
    n_coeff: int = 1
    radius: float = 2 * 25.4e-3
    center1: tuple = (-2 * 25.4e-3, 0.0, 0.0)
    center2: tuple = (-2 * 25.4e-3, 0.0, 0.0)
    active1: bool = True
    active2: bool = True
    phase1: float = 0.0
    phase2: float = 0.0
    chordlength: float = 0.5 * 25.4e-3
    theta_sources: int = 100
    trans_z_sources: int = 501
    # plane waves
    wave_amp: tuple = ()
    wave_k: tuple = ()
    wave_phase: tuple = ()
    # spline (prefiltered coefficients, x fastest)
    grid_coeff: np.ndarray | None = None
    grid_min: tuple = (0.0, 0.0, 0.0)
    grid_max: tuple = (1.0, 1.0, 1.0)
    grid_offset: float = 0.0        # added to every coefficient in double (small fields on n_o)
    # renderer
    max_depth: int = -1
    max_pathlength: float = -1.0
    use_direct: bool = True
    use_angular_sampling: bool = True
    rng: int = L.RNG_PHILOX
    precision_mode: int = L.PREC_FP32
    seed: int = 0
    step_cap: int = 0
    sensor_march_max: float = 0.0
    device: int = 0
    blocks_per_sm: int = 0
    kernel: int = L.KERNEL_POOL     # smp_kernel: slot pool (default), persistent lane loop, or plain
    spline_bricks: bool = False     # spline fields: TMA-staged coefficient bricks in shared memory

    # ---- descriptors -------------------------------------------------------------------------
    def film_shape(self) -> tuple:
        return (self.path_length_bins, self.spatial_y, self.spatial_x)

    def scene_desc(self) -> L.SceneDesc:
        """The scene as the reference's front-end assembles it (renderer3d_sample.cpp:807-830): the
        box, the source, lens and sensor origins and the film's extents are computed in its Float
        (single precision) and handed over as those float values, so the FP32 path and an FP64
        evaluation of the same descriptors place the source, the faces and the gaps identically
        (a source point on the gap boundary is then inside the field in both)."""
        f32 = np.float32
        s = L.SceneDesc()
        s.ior = self.ior
        s.medium_l[:] = tuple(float(f32(v)) for v in self.medium_l)
        s.medium_r[:] = tuple(float(f32(v)) for v in self.medium_r)
        s.light_origin[:] = (float(f32(self.medium_r[0]) + f32(self.emitter_distance)), 0.0, 0.0)
        ang = np.float32(math.pi)        # lightAngle = M_PI in Float (renderer3d_sample.cpp:815)
        s.light_dir[:] = (float(np.cos(ang)), float(np.sin(ang)), 0.0)
        s.half_theta_limit = self.half_theta_limit
        s.light_plane[:] = (float(f32(self.emitter_size)), float(f32(self.emitter_size)))
        s.Li = self.Li
        tex = np.ascontiguousarray(self.texture, dtype=np.float64)
        self._tex_keep = tex
        s.tex_y, s.tex_x = tex.shape
        s.texture = tex.ctypes.data_as(C.POINTER(C.c_double))
        s.emitter_lens_origin[:] = (float(f32(self.medium_r[0])), 0.0, 0.0)
        s.emitter_lens_aperture = self.emitter_lens_aperture
        s.emitter_lens_focal_length = self.emitter_lens_focal_length
        s.emitter_lens_active = int(self.emitter_lens_active)
        s.use_bounce_decomposition = int(self.use_bounce_decomposition)
        s.view_origin[:] = (float(f32(self.medium_l[0]) - f32(self.sensor_distance)), 0.0, 0.0)
        s.view_dir[:] = (-1.0, 0.0, 0.0)
        s.view_horizontal[:] = (0.0, -1.0, 0.0)
        s.view_plane[:] = (float(f32(self.sensor_size)), float(f32(self.sensor_size)))
        s.pathlength_range[:] = (float(f32(self.path_length_min)), float(f32(self.path_length_max)))
        s.sensor_lens_origin[:] = (float(f32(self.medium_l[0])), 0.0, 0.0)
        s.sensor_lens_aperture = self.sensor_lens_aperture
        s.sensor_lens_focal_length = self.sensor_lens_focal_length
        s.sensor_lens_active = int(self.sensor_lens_active)
        s.x_res, s.y_res, s.z_res = self.spatial_x, self.spatial_y, self.path_length_bins
        return s

    def medium_desc(self) -> L.MediumDesc:
        return L.MediumDesc(self.sigma_t, self.albedo, self.g)

    def field_desc(self) -> L.FieldDesc:
        f = L.FieldDesc()
        f.type = self.field_type
        f.precision = self.precision
        f.f_u, f.speed_u, f.n_o = self.f_u, self.speed_u, self.n_o
        f.er_stepsize = self.er_stepsize
        # gaps (renderer3d_sample.cpp:808-811): egap_end = mediumR.x - emitter_gap, sgap = mediumL.x + sensor_gap
        f.egap_end_x = float(np.float32(self.medium_r[0]) - np.float32(self.emitter_gap))
        f.sgap_begin_x = float(np.float32(self.medium_l[0]) + np.float32(self.sensor_gap))
        f.direct_tol, f.rr_weight = self.direct_tol, self.rr_weight
        f.use_initialization_hack = int(self.use_initialization_hack)
        f.mode = self.mode
        f.n_max, f.n_clip, f.phi_min, f.phi_max = self.n_max, self.n_clip, self.phi_min, self.phi_max
        f.n_coeff, f.theta_sources, f.trans_z_sources = self.n_coeff, self.theta_sources, self.trans_z_sources
        f.active1, f.active2 = int(self.active1), int(self.active2)
        f.n_scaling, f.radius, f.chordlength = self.n_scaling, self.radius, self.chordlength
        f.phase1, f.phase2 = self.phase1, self.phase2
        f.center1[:] = self.center1
        f.center2[:] = self.center2
        f.n_waves = len(self.wave_amp)
        for i, a in enumerate(self.wave_amp):
            f.wave_amp[i] = a
            f.wave_phase[i] = self.wave_phase[i]
            f.wave_k[i][:] = self.wave_k[i]
        if self.grid_coeff is not None:
            g = np.ascontiguousarray(self.grid_coeff, dtype=np.float32)
            self._coeff_keep = g
            nz, ny, nx = g.shape
            f.grid_n[:] = (nx, ny, nz)
            f.grid_min[:] = self.grid_min
            f.grid_max[:] = self.grid_max
            f.grid_coeff = g.ctypes.data_as(C.POINTER(C.c_float))
            f.grid_offset = float(self.grid_offset)
        return f

    def opts(self) -> L.RenderOpts:
        o = L.RenderOpts()
        o.max_depth = self.max_depth
        o.use_direct = int(self.use_direct)
        o.use_angular_sampling = int(self.use_angular_sampling)
        o.rng = self.rng
        o.precision = self.precision_mode
        o.device = self.device
        o.max_pathlength = self.max_pathlength
        o.seed = self.seed
        o.step_cap = self.step_cap
        o.blocks_per_sm = self.blocks_per_sm
        o.sensor_march_max = self.sensor_march_max
        o.kernel = self.kernel
        o.spline_bricks = int(self.spline_bricks)
        return o

    def descs(self):
        return self.scene_desc(), self.medium_desc(), self.field_desc(), self.opts()


# ---- the benchmark workloads (synthetic inputs; metres) ---------------------------------------

def config_plain_small(**kw) -> Setup:
    """Bessel mode 0, dn 1e-3 at 848 kHz, 10 mm cube, sigma_s 0.1/mm, albedo 0.9, g 0.9, 0.5 mm
    radius collimated beam (the Disk_501 texture on a 1 mm emitter), 100% duty cycle
    (phase uniform on [0, 2 pi)), 0.01 mm ER step, 128x128 px x 32 bins over 0-50 mm, FP32."""
    s = Setup()
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def config_precision(**kw) -> Setup:
    """Bessel mode 1, dn 2e-3, sigma_s 1/mm, albedo 0.95, g 0.85, 64x64 Bernoulli(0.5) texture
    (seed 1), 512x512 px x 128 bins over 0-100 mm, FP32 march with FP64 path length and film."""
    s = Setup(mode=1, n_max=2e-3, n_clip=2e-3, sigma_t=1000.0 / 0.95, albedo=0.95, g=0.85,
              texture=bernoulli_texture(64, 0.5, 1), spatial_x=512, spatial_y=512, path_length_bins=128,
              path_length_max=0.1, precision_mode=L.PREC_MIXED)
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def config_planewave(**kw) -> Setup:
    """Two plane waves a = 1e-3 at 1 MHz travelling along +y and +z (90 degrees apart), phases
    uniform on [0, 2 pi) (seed 3), sigma_s 0.5/mm, albedo 0.9, g 0.9."""
    k = 2.0 * math.pi * 1e6 / 1500.0
    ph = np.random.default_rng(3).random(2) * 2.0 * math.pi
    s = Setup(field_type=L.FIELD_PLANEWAVE, f_u=1e6, wave_amp=(1e-3, 1e-3), wave_k=((0.0, k, 0.0), (0.0, 0.0, k)),
              wave_phase=(float(ph[0]), float(ph[1])), phi_min=0.0, phi_max=0.0,
              sigma_t=500.0 / 0.9, albedo=0.9, g=0.9)
    for kk, v in kw.items():
        setattr(s, kk, v)
    return s


def config_sources(**kw) -> Setup:
    """The focused-ultrasound point-source field (rif_sources) with the reference's source layout:
    two arcs of radius 2 in with a 0.5 in chord, 100 x 501 point sources each, centred 2 in behind
    the medium on the -x axis, first harmonic, n_scaling 5e-5; medium, beam and film of
    config_plain_small."""
    s = Setup(field_type=L.FIELD_SOURCES)
    for kk, v in kw.items():
        setattr(s, kk, v)
    return s


def config_batch_sweep(n_inst: int = 256, seed: int = 2, scale: float = 1.0, **kw):
    """The batched sweep: n_inst cylindrical-transducer instances over the plain small scene
    (medium, optics and 128x128 x 32 film of config_plain_small), with amplitude n_max ~ U[0, 2e-3],
    frequency ~ U[0.5, 2] MHz, mode in {0, 1, 2}, duty cycle D ~ U[1, 100] % (phase range
    [0, 2 pi D)) and a photon budget log-uniform in [1e5, 1e7] (times `scale`), all drawn from
    numpy's default_rng(seed); instance i draws Philox stream seed (seed << 32) + i.
    Returns (setup, instances) for render_batch."""
    rng = np.random.default_rng(seed)
    setup = config_plain_small(**kw)
    insts = []
    for i in range(n_inst):
        n_max = float(rng.uniform(0.0, 2e-3))
        f_u = float(rng.uniform(0.5e6, 2e6))
        mode = int(rng.integers(0, 3))
        duty = float(rng.uniform(0.01, 1.0))
        n_ph = int(round(10.0 ** rng.uniform(5.0, 7.0) * scale))
        insts.append({"mode": mode, "n_max": n_max, "n_clip": n_max, "f_u": f_u, "phi_min": 0.0,
                      "phi_max": 2.0 * math.pi * duty, "n_photons": max(n_ph, 1), "seed": (seed << 32) + i})
    return setup, insts


def config_spline(n: int = 64, seed: int = 4, **kw) -> Setup:
    """The spline-field configuration: an n^3 tricubic B-spline coefficient grid over the 10 mm
    cube whose coefficients are n_o + Gaussian-filtered (sigma 4 voxels) N(0, 1) noise from
    numpy's default_rng(seed), scaled to a largest |dn| of 1e-3; sigma_s 1/mm, albedo 0.95,
    g 0.8, 256x256 px x 64 bins."""
    from scipy.ndimage import gaussian_filter
    noise = gaussian_filter(np.random.default_rng(seed).standard_normal((n, n, n)), sigma=4.0, mode="wrap")
    coeff = 1.3333 + noise * (1e-3 / np.abs(noise).max())
    s = Setup(field_type=L.FIELD_SPLINE, grid_coeff=coeff.astype(np.float32), grid_min=(-0.005,) * 3,
              grid_max=(0.005,) * 3, sigma_t=1000.0 / 0.95, albedo=0.95, g=0.8, spatial_x=256, spatial_y=256,
              path_length_bins=64, path_length_max=0.1)
    for kk, v in kw.items():
        setattr(s, kk, v)
    return s
