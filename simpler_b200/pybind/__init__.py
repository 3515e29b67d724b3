"""Drop-in Python modules for the reference's pybind11 bindings (renderer/pybindFiles/*.cpp).

``from simpler_b200.pybind import scene_pybind, photon_pybind, ...`` replaces ``import
scene_pybind, photon_pybind, ...``: same module, class, constructor and method names and argument
order, with the render running on the B200 kernel through the C ABI. Scalars pass through float32
as the reference's ``Float`` arguments do.
"""
from . import image_pybind, medium_pybind, phase_pybind, photon_pybind, scene_pybind, tvector_pybind

__all__ = ["image_pybind", "medium_pybind", "phase_pybind", "photon_pybind", "scene_pybind", "tvector_pybind"]
