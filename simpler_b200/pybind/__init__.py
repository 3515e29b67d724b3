"""The Python side of the reference's pybind users.

The reference's six pybind11 modules (renderer/pybindFiles/{tvector,phase,medium,image,scene,
photon}_pybind.cpp) are compiled under their own names from simpler_b200/csrc/pybind/ into
``module_dir()``; put that directory on sys.path and ``import scene_pybind, photon_pybind, ...``
works unchanged, rendering on the B200 kernels. ``autograd`` holds the torch.autograd.Function over
the render and its adjoint.
"""
import os


def module_dir() -> str:
    """The directory holding the compiled tvector/phase/medium/image/scene/photon_pybind modules."""
    return os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pybind_ext")
