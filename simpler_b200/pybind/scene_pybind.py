"""scene pybind module (renderer/pybindFiles/scene_pybind.cpp): Scene with the positional
constructor of renderer/include/scene.h:47-105 and the ultrasound setters of scene.h:179-219.

The reference compiles one of three constructor forms; this Scene takes any of them and tells
them apart by argument count:

* 43 arguments: rif_analytical (f_u, speed_u, n_o, n_max, n_clip, phi_min, phi_max, mode);
* 44 arguments: rif_interpolated (the analytical block plus rifgridFile, a .vol grid);
* 53 arguments: rif_sources (f_u, speed_u, n_o, n_scaling, n_coeff, radius, center1, center2,
  active1, active2, phase1, phase2, theta_min, theta_max, theta_sources, trans_z_min,
  trans_z_max, trans_z_sources).

The film resolution is not part of a Scene; photon_pybind.Renderer.renderImage takes it from
the SmallImage it fills.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from .. import _lib as L
from .. import pfm
from .tvector_pybind import _f, as2, as3

_N_COMMON = 25
_N_TAIL = 10
_FORMS = {_N_COMMON + 8 + _N_TAIL: "rif_analytical",
          _N_COMMON + 8 + _N_TAIL + 1: "rif_interpolated",
          _N_COMMON + 18 + _N_TAIL: "rif_sources"}
# the ultrasound frame the kernel is built for (renderer3d_sample.cpp:839-841, rif_base.h:146-148)
_AXIS_UZ, _AXIS_UX, _P_U = (-1.0, 0.0, 0.0), (0.0, 0.0, 1.0), (0.0, 0.0, 0.0)


class Scene:
    def __init__(self, *args):
        form = _FORMS.get(len(args))
        if form is None:
            raise TypeError(f"Scene: expected 43, 44 or 53 positional arguments (scene.h:47-105), got {len(args)}")
        self.form = form
        a = list(args)
        s = L.SceneDesc()
        s.ior = _f(a[0])
        s.medium_l[:] = as3(a[1])
        s.medium_r[:] = as3(a[2])
        s.light_origin[:] = as3(a[3])
        s.light_dir[:] = as3(a[4])
        s.half_theta_limit = _f(a[5])
        self.texture = pfm.read_pfm(str(a[6]))
        s.light_plane[:] = as2(a[7])
        s.Li = _f(a[8])
        s.view_origin[:] = as3(a[9])
        s.view_dir[:] = as3(a[10])
        s.view_horizontal[:] = as3(a[11])
        s.view_plane[:] = as2(a[12])
        s.pathlength_range[:] = as2(a[13])
        s.use_bounce_decomposition = int(bool(a[14]))
        self.distribution, self.g_or_kappa = str(a[15]), _f(a[16])   # carried; unused by the 3-D march
        s.emitter_lens_origin[:] = as3(a[17])
        s.emitter_lens_aperture, s.emitter_lens_focal_length = _f(a[18]), _f(a[19])
        s.emitter_lens_active = int(bool(a[20]))
        s.sensor_lens_origin[:] = as3(a[21])
        s.sensor_lens_aperture, s.sensor_lens_focal_length = _f(a[22]), _f(a[23])
        s.sensor_lens_active = int(bool(a[24]))
        self._tex = np.ascontiguousarray(self.texture, dtype=np.float64)
        s.tex_y, s.tex_x = self._tex.shape
        s.texture = self._tex.ctypes.data_as(C.POINTER(C.c_double))
        self.scene_desc = s

        f = L.FieldDesc()
        us = a[_N_COMMON:]
        f.f_u, f.speed_u, f.n_o = _f(us[0]), _f(us[1]), _f(us[2])
        if form == "rif_sources":
            f.type = L.FIELD_SOURCES
            f.n_scaling, f.n_coeff, f.radius = _f(us[3]), int(us[4]), _f(us[5])
            f.center1[:] = as3(us[6])
            f.center2[:] = as3(us[7])
            f.active1, f.active2 = int(bool(us[8])), int(bool(us[9]))
            f.phase1, f.phase2 = _f(us[10]), _f(us[11])
            f.theta_min, f.theta_max, f.theta_sources = _f(us[12]), _f(us[13]), int(us[14])
            f.trans_z_min, f.trans_z_max, f.trans_z_sources = _f(us[15]), _f(us[16]), int(us[17])
            if not f.theta_max > f.theta_min:
                raise ValueError("Scene: theta_max must exceed theta_min")
            tail = us[18:]
        else:
            f.type = L.FIELD_BESSEL
            f.n_max, f.n_clip, f.phi_min, f.phi_max = _f(us[3]), _f(us[4]), _f(us[5]), _f(us[6])
            f.mode = int(us[7])
            tail = us[8:]
        axis_uz, axis_ux, p_u = as3(tail[0]), as3(tail[1]), as3(tail[2])
        if (axis_uz, axis_ux, p_u) != (_AXIS_UZ, _AXIS_UX, _P_U):
            raise L.SmpError(L.SMP_ERR_UNSUPPORTED,
                             "Scene: the ultrasound frame must be axis_uz=(-1,0,0), axis_ux=(0,0,1), p_u=(0,0,0)")
        f.er_stepsize, f.direct_tol, f.rr_weight = _f(tail[3]), _f(tail[4]), _f(tail[5])
        f.precision = int(tail[6])
        f.egap_end_x, f.sgap_begin_x = _f(tail[7]), _f(tail[8])
        f.use_initialization_hack = int(bool(tail[9]))
        if form == "rif_interpolated":
            vals, lo, hi = pfm.read_vol(str(tail[10]))
            nz, ny, nx = vals.shape
            coeff = np.zeros_like(vals)
            n = (C.c_int32 * 3)(nx, ny, nz)
            self._n = n
            lib = L.load()
            L.check(lib.smp_spline_prefilter(C.c_void_p(vals.ctypes.data), C.cast(n, C.c_void_p),
                                            C.c_void_p(coeff.ctypes.data)))
            self._coeff = coeff
            f.type = L.FIELD_SPLINE
            f.grid_n[:] = (nx, ny, nz)
            f.grid_min[:] = lo
            f.grid_max[:] = hi
            f.grid_coeff = coeff.ctypes.data_as(C.POINTER(C.c_float))
        self.field_desc = f

    # ---- setters (scene.h:179-219); k = 2 pi f_u / speed_u follows f_u as rif_base.h:144-154 derives it
    def set_f_u(self, value: float) -> None:
        self.field_desc.f_u = _f(value)

    def set_n_max(self, value: float) -> None:
        self.field_desc.n_max = _f(value)

    def set_n_scaling(self, value: float) -> None:
        self.field_desc.n_scaling = _f(value)

    def set_phase1(self, value: float) -> None:
        self.field_desc.phase1 = _f(value)

    def set_phase2(self, value: float) -> None:
        self.field_desc.phase2 = _f(value)

    def getUSFrequency(self) -> float:  # noqa: N802 -- scene.h:174-177
        return self.field_desc.f_u

    def wavelength(self) -> float:
        return self.field_desc.speed_u / self.field_desc.f_u

    def k(self) -> float:
        return 2.0 * math.pi / self.wavelength()
