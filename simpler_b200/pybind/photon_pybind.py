"""photon pybind module (renderer/pybindFiles/photon_pybind.cpp): Renderer(maxDepth,
maxPathlength, useDirect, useAngularSampling, threads).renderImage(img, medium, scene, numPhotons),
the reference's photon::Renderer::renderImage (renderer/src/photon.cpp:267-340) on the B200 kernel.

``threads`` is accepted and ignored: the render runs on one GPU. Keyword-only extensions choose
the device, the Philox seed (photon i draws stream (seed, i)) and the film precision.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _lib as L
from .image_pybind import SmallImage
from .medium_pybind import Medium
from .scene_pybind import Scene


class Renderer:
    def __init__(self, maxDepth: int, maxPathlength: float, useDirect: bool, useAngularSampling: bool,  # noqa: N803
                 threads: int, *, device: int = 0, seed: int = 0, precision: int = L.PREC_FP32):
        self.max_depth = int(maxDepth)
        self.max_pathlength = float(np.float32(maxPathlength))
        self.use_direct = bool(useDirect)
        self.use_angular_sampling = bool(useAngularSampling)
        self.threads = int(threads)
        self.device, self.seed, self.precision = int(device), int(seed), int(precision)
        self.last_stats: L.Stats | None = None

    def renderImage(self, img: SmallImage, medium: Medium, scene: Scene, numPhotons: int) -> None:  # noqa: N802,N803
        """Render numPhotons photons into img (overwriting it, as the reference's renderImage does
        after its per-thread images are merged)."""
        lib = L.load()
        s = scene.scene_desc
        s.x_res, s.y_res, s.z_res = img.get_x_res(), img.get_y_res(), img.getZRes()
        m = L.MediumDesc(medium.sigma_t, medium.albedo, medium.phase.g)
        o = L.RenderOpts()
        o.max_depth = self.max_depth
        o.max_pathlength = self.max_pathlength
        o.use_direct = int(self.use_direct)
        o.use_angular_sampling = int(self.use_angular_sampling)
        o.rng = L.RNG_PHILOX
        o.precision = self.precision
        o.device = self.device
        o.seed = self.seed
        st = L.Stats()
        film = img.pixels
        if not (film.flags.c_contiguous and film.dtype == np.float64):
            film = np.ascontiguousarray(film, dtype=np.float64)
        # written in place (the library overwrites every pixel); ctypes releases the GIL meanwhile
        L.check(lib.smp_render(C.byref(s), C.byref(m), C.byref(scene.field_desc), C.byref(o), int(numPhotons),
                               C.c_void_p(film.ctypes.data), C.byref(st)))
        if film is not img.pixels:
            img.pixels[...] = film
        self.last_stats = st
