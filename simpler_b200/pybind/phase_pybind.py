"""phase pybind module (renderer/pybindFiles/phase_pybind.cpp): the Henyey-Greenstein phase function."""
from __future__ import annotations

import numpy as np


class henyey_greenstein:  # noqa: N801 -- the reference's class name
    def __init__(self, g: float):
        self.g = float(np.float32(g))

    def getG(self) -> float:  # noqa: N802 -- pfunc::henyey_greenstein::getG (phase.h)
        return self.g
