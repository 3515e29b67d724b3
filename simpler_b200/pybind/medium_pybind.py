"""medium pybind module (renderer/pybindFiles/medium_pybind.cpp): Medium(sigma_t, albedo, phase)."""
from __future__ import annotations

import numpy as np

from .phase_pybind import henyey_greenstein


class Medium:
    def __init__(self, sigma_t: float, albedo: float, phase: henyey_greenstein):
        if not isinstance(phase, henyey_greenstein):
            raise TypeError("Medium: phase must be a phase_pybind.henyey_greenstein")
        self.sigma_t = float(np.float32(sigma_t))
        self.albedo = float(np.float32(albedo))
        self.phase = phase

    def getSigmaT(self) -> float:  # noqa: N802 -- med::Medium accessors (medium.h)
        return self.sigma_t

    def getAlbedo(self) -> float:  # noqa: N802
        return self.albedo
