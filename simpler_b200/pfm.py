"""The reference's image files, in numpy.

* PFM texture (``Image2::readPFM``, renderer/include/image.h:183-245): header tokens ``Pf``, X, Y,
  endianness; the last X*Y doubles of the file are the texels, stored bottom row first. The
  reader returns them flipped, texel (x, y) at ``tex[y, x]``, as the projector samples them.
* PFM3D film (``Image3::writePFM3D``, renderer/src/image.cpp:161-206; reader image.h:374-436):
  ``Pf\\nX Y Z\\n-1\\n`` then X*Y*Z little-endian doubles, index z*X*Y + y*X + x, no flip.
* VOL grid (``Spline::readVolAndBuild``, renderer/include/spline.h:115-162): ``VOL`` 3, int32
  type 1, int32 nx ny nz, int32 channels 1, six float32 bounds, nx*ny*nz float32 (x fastest).
"""
from __future__ import annotations

import numpy as np


def _header_tokens(data: bytes, n: int) -> list[bytes]:
    toks, i = [], 0
    while len(toks) < n:
        while i < len(data) and data[i:i + 1].isspace():
            i += 1
        j = i
        while j < len(data) and not data[j:j + 1].isspace():
            j += 1
        if j == i:
            raise ValueError("truncated PFM header")
        toks.append(data[i:j])
        i = j
    return toks


def read_pfm(path: str) -> np.ndarray:
    """A grayscale PFM texture as a (Y, X) float64 array, rows flipped as the reference reads them."""
    data = open(path, "rb").read()
    magic, x, y, _ = _header_tokens(data, 4)
    if magic != b"Pf":
        raise ValueError(f"Invalid magic number in {path}: no Pf (grayscale pfm)")
    x, y = int(x), int(y)
    need = x * y * 8
    if len(data) < need:
        raise ValueError(f"PFM {path} shorter than its header says")
    raw = np.frombuffer(data[len(data) - need:], dtype="<f8").reshape(y, x)
    return raw[::-1].copy()


def write_pfm(path: str, tex: np.ndarray) -> None:
    """Inverse of read_pfm: writes the rows bottom first so that read_pfm returns ``tex``."""
    tex = np.ascontiguousarray(tex, dtype="<f8")
    y, x = tex.shape
    with open(path, "wb") as f:
        f.write(b"Pf\n%d %d\n-1\n" % (x, y))
        f.write(tex[::-1].tobytes())


def write_pfm3d(path: str, film: np.ndarray) -> None:
    """A (Z, Y, X) film in the reference's PFM3D layout."""
    film = np.ascontiguousarray(film, dtype="<f8")
    z, y, x = film.shape
    with open(path, "wb") as f:
        f.write(b"Pf\n%d %d %d\n-1\n" % (x, y, z))
        f.write(film.tobytes())


def read_pfm3d(path: str) -> np.ndarray:
    """A PFM3D film as a (Z, Y, X) float64 array."""
    data = open(path, "rb").read()
    magic, x, y, z, _ = _header_tokens(data, 5)
    if magic != b"Pf":
        raise ValueError(f"Invalid magic number in {path}")
    x, y, z = int(x), int(y), int(z)
    need = x * y * z * 8
    if len(data) < need:
        raise ValueError(f"PFM3D {path} shorter than its header says")
    return np.frombuffer(data[len(data) - need:], dtype="<f8").reshape(z, y, x).copy()


def read_vol(path: str) -> tuple[np.ndarray, tuple, tuple]:
    """A VOL grid as ((nz, ny, nx) float32 array, (xmin, ymin, zmin), (xmax, ymax, zmax))."""
    data = open(path, "rb").read()
    if data[:3] != b"VOL" or data[3] != 3:
        raise ValueError(f"file {path} is not a VOL version 3 file")
    typ, nx, ny, nz, ch = np.frombuffer(data[4:24], dtype="<i4")
    if typ != 1 or ch != 1:
        raise ValueError("VOL must hold one float32 channel")
    bb = np.frombuffer(data[24:48], dtype="<f4").astype(np.float64)
    vals = np.frombuffer(data[48:48 + 4 * nx * ny * nz], dtype="<f4").reshape(nz, ny, nx).copy()
    return vals, tuple(bb[:3]), tuple(bb[3:])


def write_vol(path: str, grid: np.ndarray, lo: tuple, hi: tuple) -> None:
    grid = np.ascontiguousarray(grid, dtype="<f4")
    nz, ny, nx = grid.shape
    with open(path, "wb") as f:
        f.write(b"VOL\x03")
        f.write(np.array([1, nx, ny, nz, 1], dtype="<i4").tobytes())
        f.write(np.array(list(lo) + list(hi), dtype="<f4").tobytes())
        f.write(grid.tobytes())
