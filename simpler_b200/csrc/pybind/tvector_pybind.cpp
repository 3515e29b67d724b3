// tvector_pybind -- the reference's tvector module (renderer/pybindFiles/tvector_pybind.cpp):
// Vec2f(x, y), Vec3f(x, y, z) with index(i), Vec3i(x, y, z) with x, y, z. Components are Float
// (single precision) as in the reference's build.
#include "pybind_types.h"

using namespace smp_pybind;

PYBIND11_MODULE(tvector_pybind, m) {
    m.doc() = "tvector pybind module";
    py::class_<Vec2f>(m, "Vec2f")
        .def(py::init([](float x, float y) { return Vec2f{x, y}; }))
        .def_readwrite("x", &Vec2f::x)
        .def_readwrite("y", &Vec2f::y)
        .def("__repr__", [](const Vec2f &v) { return "Vec2f(" + std::to_string(v.x) + ", " + std::to_string(v.y) + ")"; });
    py::class_<Vec3f>(m, "Vec3f")
        .def(py::init([](float x, float y, float z) { return Vec3f{x, y, z}; }))
        .def("index", &Vec3f::index)
        .def_readwrite("x", &Vec3f::x)
        .def_readwrite("y", &Vec3f::y)
        .def_readwrite("z", &Vec3f::z)
        .def("__repr__", [](const Vec3f &v) {
            return "Vec3f(" + std::to_string(v.x) + ", " + std::to_string(v.y) + ", " + std::to_string(v.z) + ")";
        });
    py::class_<Vec3i>(m, "Vec3i")
        .def(py::init([](int x, int y, int z) { return Vec3i{x, y, z}; }))
        .def_readwrite("x", &Vec3i::x)
        .def_readwrite("y", &Vec3i::y)
        .def_readwrite("z", &Vec3i::z);
}
