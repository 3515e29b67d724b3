// phase_pybind -- the reference's phase module (renderer/pybindFiles/phase_pybind.cpp):
// henyey_greenstein(g).
#include "pybind_types.h"

using namespace smp_pybind;

PYBIND11_MODULE(phase_pybind, m) {
    m.doc() = "phase pybind module";
    py::class_<HenyeyGreenstein>(m, "henyey_greenstein")
        .def(py::init([](float g) { return HenyeyGreenstein{g}; }))
        .def("getG", [](const HenyeyGreenstein &h) { return h.g; });
}
