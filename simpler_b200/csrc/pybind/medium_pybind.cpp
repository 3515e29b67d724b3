// medium_pybind -- the reference's medium module (renderer/pybindFiles/medium_pybind.cpp):
// Medium(sigma_t, albedo, phase_pybind.henyey_greenstein).
#include "pybind_types.h"

using namespace smp_pybind;

PYBIND11_MODULE(medium_pybind, m) {
    m.doc() = "medium pybind module";
    py::module_::import("phase_pybind");
    py::class_<Medium>(m, "Medium")
        .def(py::init([](float sigma_t, float albedo, const HenyeyGreenstein *phase) {
                 if (!phase) throw py::type_error("Medium: phase must be a phase_pybind.henyey_greenstein");
                 Medium md;
                 md.sigma_t = sigma_t;
                 md.albedo = albedo;
                 md.phase = *phase;
                 return md;
             }))
        .def("getSigmaT", [](const Medium &md) { return md.sigma_t; })
        .def("getAlbedo", [](const Medium &md) { return md.albedo; })
        .def_property_readonly("phase", [](const Medium &md) { return md.phase; });
}
