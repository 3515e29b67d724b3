"""tvector pybind module (renderer/pybindFiles/tvector_pybind.cpp): Vec2f, Vec3f, Vec3i."""
from __future__ import annotations

import numpy as np


def _f(v) -> float:
    return float(np.float32(v))


class Vec2f:
    def __init__(self, x: float, y: float):
        self.x, self.y = _f(x), _f(y)

    def __iter__(self):
        return iter((self.x, self.y))

    def __repr__(self):
        return f"Vec2f({self.x}, {self.y})"


class Vec3f:
    def __init__(self, x: float, y: float, z: float):
        self.x, self.y, self.z = _f(x), _f(y), _f(z)

    def index(self, i: int) -> float:
        """Component i, as TVector3::index (tvector.h:327-329)."""
        return (self.x, self.y, self.z)[i]

    def __iter__(self):
        return iter((self.x, self.y, self.z))

    def __repr__(self):
        return f"Vec3f({self.x}, {self.y}, {self.z})"


class Vec3i:
    def __init__(self, x: int, y: int, z: int):
        self.x, self.y, self.z = int(x), int(y), int(z)

    def __iter__(self):
        return iter((self.x, self.y, self.z))

    def __repr__(self):
        return f"Vec3i({self.x}, {self.y}, {self.z})"


def as3(v) -> tuple:
    """A Vec3f or any 3-sequence as a float32-rounded tuple."""
    x, y, z = tuple(v)
    return (_f(x), _f(y), _f(z))


def as2(v) -> tuple:
    x, y = tuple(v)
    return (_f(x), _f(y))
