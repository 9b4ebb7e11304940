// Shared by the compiled drop-in modules `carma` and `sutra`: the device-array
// view (the role of the reference's carma objects, python_module/carma/src/obj.hpp:32-76)
// and the error check that turns a libaob200 status into the exception the
// reference's bindings raise (std::runtime_error -> RuntimeError).
#pragma once

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "aob200.h"

namespace aobpy {

namespace py = pybind11;

inline void check(int st, const char *what) {
  if (st != AOB_OK) throw std::runtime_error(std::string(what) + ": " + aob_last_error());
}

// A view of a device buffer owned by the library.  ``owner`` keeps the object
// that owns the buffer alive for as long as the view exists.  np.array(view)
// copies it to the host, shaped like the reference's arrays (Fortran order).
struct DevArr {
  uintptr_t ptr = 0;
  int64_t n = 0;
  py::dtype dtype = py::dtype::of<float>();
  std::vector<py::ssize_t> shape;
  std::shared_ptr<void> owner;

  DevArr() = default;
  DevArr(uintptr_t p, int64_t count, py::dtype dt, std::vector<py::ssize_t> shp, std::shared_ptr<void> own)
      : ptr(p), n(count), dtype(std::move(dt)), owner(std::move(own)) {
    int64_t prod = 1;
    for (auto d : shp) prod *= d;
    shape = (!shp.empty() && prod == count) ? std::move(shp) : std::vector<py::ssize_t>{(py::ssize_t)count};
  }

  std::vector<py::ssize_t> fortran_strides() const {
    std::vector<py::ssize_t> st;
    py::ssize_t acc = dtype.itemsize();
    for (auto d : shape) {
      st.push_back(acc);
      acc *= d;
    }
    return st;
  }

  py::array host() const {
    py::array a(dtype, shape, fortran_strides());
    const size_t bytes = (size_t)n * (size_t)dtype.itemsize();
    if (ptr && n > 0)
      check(aob_memcpy_d2h(a.mutable_data(), reinterpret_cast<const void *>(ptr), bytes, nullptr), "d2h copy");
    else if (bytes)
      std::memset(a.mutable_data(), 0, bytes);
    return a;
  }

  void set(const py::object &src) {
    py::module_ np = py::module_::import("numpy");
    py::array a = np.attr("ascontiguousarray")(np.attr("asarray")(src, dtype).attr("ravel")("F"));
    if ((int64_t)a.size() != n)
      throw std::runtime_error("set: size mismatch (" + std::to_string(a.size()) + " != " + std::to_string(n) + ")");
    if (n > 0)
      check(aob_memcpy_h2d(reinterpret_cast<void *>(ptr), a.data(), (size_t)n * (size_t)dtype.itemsize(), nullptr),
            "h2d copy");
  }
};

// Registers the view type in module ``m`` (module-local, so each compiled module
// owns its copy and neither has to import the other).
inline void bind_device_array(py::module_ &m, const char *name) {
  py::class_<DevArr>(m, name, py::module_local())
      .def("host", &DevArr::host)
      .def(
          "__array__",
          [](const DevArr &d, py::object dtype, py::object copy) {
            py::array a = d.host();
            return dtype.is_none() ? py::object(a) : a.attr("astype")(dtype);
          },
          py::arg("dtype") = py::none(), py::arg("copy") = py::none())
      .def("set", &DevArr::set)
      .def("get_dims", [](const DevArr &d) { return py::tuple(py::cast(d.shape)); })
      .def_property_readonly("ptr", [](const DevArr &d) { return d.ptr; })
      .def_property_readonly("shape", [](const DevArr &d) { return py::tuple(py::cast(d.shape)); })
      .def_property_readonly("dtype", [](const DevArr &d) { return d.dtype; })
      .def_property_readonly("nbElem", [](const DevArr &d) { return d.n; })
      .def("__len__", [](const DevArr &d) { return d.shape.empty() ? (py::ssize_t)0 : d.shape[0]; })
      .def_property_readonly("__cuda_array_interface__", [](const DevArr &d) {
        py::dict r;
        r["shape"] = py::tuple(py::cast(d.shape));
        r["typestr"] = d.dtype.attr("str");
        r["data"] = py::make_tuple(d.ptr, false);
        r["strides"] = py::tuple(py::cast(d.fortran_strides()));
        r["version"] = 3;
        return r;
      });
}

// Contiguous Fortran-order host copies of array arguments, as the reference's
// bindings take them (py::array_t<T, f_style | forcecast>, sutraUtils.hpp:31-32).
template <typename T>
using farray = py::array_t<T, py::array::f_style | py::array::forcecast>;

}  // namespace aobpy
