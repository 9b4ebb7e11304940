// Compiled drop-in `carma` module: the parts of the reference's pybind11 carma
// module (python_module/carma/src/carma.cpp, context.cpp) that COMPASS's hot
// path touches, over libaob200.
//  * context: the GPUs this process drives and the active one (get_instance,
//    get_instance_1gpu, get_instance_ngpu, activate_device);
//  * obj: the device-array view that the compiled `sutra` returns for its d_*
//    buffers; np.array(obj) copies it to the host like np.array(carma_obj).

#include <algorithm>
#include <mutex>

#include "native_common.hpp"

namespace py = pybind11;
using aobpy::check;

namespace {

struct Context {
  std::vector<int> devices;
  int active = 0;
};

std::shared_ptr<Context> g_instance;
std::mutex g_mu;

std::shared_ptr<Context> make_context(std::vector<int> devs) {
  if (devs.empty()) {
    const int n = aob_device_count();
    for (int i = 0; i < std::max(n, 1); ++i) devs.push_back(i);
  }
  auto c = std::make_shared<Context>();
  c->devices = std::move(devs);
  c->active = c->devices.front();
  return c;
}

}  // namespace

PYBIND11_MODULE(carma, m) {
  m.doc() = "libaob200 drop-in for the reference's carma module (context and device arrays)";
  aobpy::bind_device_array(m, "obj");
  py::class_<Context, std::shared_ptr<Context>>(m, "context")
      .def(py::init([](py::object devices) {
             std::vector<int> d;
             if (!devices.is_none())
               for (auto v : devices) d.push_back(v.cast<int>());
             return make_context(d);
           }),
           py::arg("devices") = py::none())
      .def_static("get_instance",
                  []() {
                    std::lock_guard<std::mutex> lock(g_mu);
                    if (!g_instance) g_instance = make_context({});
                    return g_instance;
                  })
      .def_static("get_instance_1gpu",
                  [](int dev) {
                    std::lock_guard<std::mutex> lock(g_mu);
                    g_instance = make_context({dev});
                    return g_instance;
                  })
      .def_static("get_instance_ngpu",
                  [](int ngpu, py::iterable devices) {
                    std::vector<int> d;
                    for (auto v : devices) {
                      if ((int)d.size() == ngpu) break;
                      d.push_back(v.cast<int>());
                    }
                    std::lock_guard<std::mutex> lock(g_mu);
                    g_instance = make_context(d);
                    return g_instance;
                  })
      .def_property_readonly("ndevice", [](const Context &c) { return (int)c.devices.size(); })
      .def_readonly("devices", &Context::devices)
      .def_property_readonly("active_device", [](const Context &c) { return c.active; })
      .def_property_readonly("active_device_id", [](const Context &c) { return c.active; })
      .def(
          "activate_device",
          [](Context &c, int dev, bool silent) {
            for (int d : c.devices)
              if (d == dev) {
                c.active = dev;
                return;
              }
            throw std::runtime_error("device " + std::to_string(dev) + " is not in this context");
          },
          py::arg("dev"), py::arg("silent") = true)
      .def("get_device", [](const Context &, int dev) { return dev; });
}
