// image_pybind -- the reference's image module (renderer/pybindFiles/image_pybind.cpp):
// SmallImage(x, y, z) with get_x_res, get_y_res, getZRes and get_pixel. The film is also exposed
// without a copy: through the buffer protocol (numpy.asarray(img), shape (z, y, x), float64) and the
// `pixels` view, so a render's film is read as one array instead of pixel by pixel.
#include "pybind_types.h"

using namespace smp_pybind;

PYBIND11_MODULE(image_pybind, m) {
    m.doc() = "image pybind module";
    py::class_<SmallImage>(m, "SmallImage", py::buffer_protocol())
        .def(py::init<int, int, int>())
        .def("get_x_res", [](const SmallImage &i) { return i.xres; })
        .def("get_y_res", [](const SmallImage &i) { return i.yres; })
        .def("getZRes", [](const SmallImage &i) { return i.zres; })
        .def("get_pixel", &SmallImage::get_pixel)
        .def("zero", [](SmallImage &i) { std::fill(i.pixels.begin(), i.pixels.end(), 0.0); })
        // Image3::writePFM3D (renderer/src/image.cpp:161-206)
        .def("writePFM3D", [](const SmallImage &i, const std::string &path) {
            std::string err;
            if (!smp_host::write_pfm3d(path, i.xres, i.yres, i.zres, i.pixels.data(), err)) throw std::runtime_error(err);
        })
        .def_buffer([](SmallImage &i) -> py::buffer_info {
            const py::ssize_t d = sizeof(double);
            return py::buffer_info(i.pixels.data(), d, py::format_descriptor<double>::format(), 3,
                                   {py::ssize_t(i.zres), py::ssize_t(i.yres), py::ssize_t(i.xres)},
                                   {d * i.xres * i.yres, d * i.xres, d});
        })
        .def_property_readonly("pixels", [](py::object self) {
            SmallImage &i = self.cast<SmallImage &>();
            const py::ssize_t d = sizeof(double);
            return py::array_t<double>({py::ssize_t(i.zres), py::ssize_t(i.yres), py::ssize_t(i.xres)},
                                       {d * i.xres * i.yres, d * i.xres, d}, i.pixels.data(), self);
        });
}
