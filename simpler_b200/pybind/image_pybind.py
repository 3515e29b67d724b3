"""image pybind module (renderer/pybindFiles/image_pybind.cpp): SmallImage(x, y, z) over a numpy
film (Image3<double>, index z*X*Y + y*X + x) that photon_pybind.Renderer.renderImage fills."""
from __future__ import annotations

import numpy as np

from .. import pfm


class SmallImage:
    def __init__(self, x: int, y: int, z: int):
        self._x, self._y, self._z = int(x), int(y), int(z)
        self.pixels = np.zeros((self._z, self._y, self._x), dtype=np.float64)

    def get_x_res(self) -> int:
        return self._x

    def get_y_res(self) -> int:
        return self._y

    def getZRes(self) -> int:  # noqa: N802 -- the reference's method name
        return self._z

    def get_pixel(self, x: int, y: int, z: int) -> float:
        """Image3::get_pixel (image.h:309-312). The reference reads index z*X*Y + y*Y + x there,
        which is the film's (x, y, z) texel when X == Y; the same flat index is read here."""
        if not (0 <= x < self._x and 0 <= y < self._y and 0 <= z < self._z):
            raise IndexError("get_pixel: coordinate out of range")
        return float(self.pixels.reshape(-1)[z * self._x * self._y + y * self._y + x])

    def zero(self) -> None:
        self.pixels[...] = 0.0

    def writePFM3D(self, path: str) -> None:  # noqa: N802 -- Image3::writePFM3D (image.cpp:161-206)
        pfm.write_pfm3d(path, self.pixels)

    def torch(self):
        """The film as a CPU torch tensor sharing this image's memory, shape (Z, Y, X)."""
        import torch
        return torch.from_numpy(self.pixels)
