// Centroiders, controllers and Rtc_FFF of the compiled drop-in `sutra`
// (centroider.cpp:83-356, controller.cpp:65-330, controller_ls.cpp:69-245,
// controller_generic.cpp, rtc.cpp:100-485).  A controller reads the slopes of the
// centroiders in its idx_centro (all of them by default), one block after the
// other, as rtc.cpp stacks them.
#pragma once

#include <algorithm>
#include <tuple>

#include "sutra_dms.hpp"
#include "sutra_sensors.hpp"

namespace aobpy {

struct CentroOwner {
  aob_centro *h = nullptr;
  ~CentroOwner() {
    if (h) aob_centro_destroy(h);
  }
};
struct LsOwner {
  aob_ls *h = nullptr;
  ~LsOwner() {
    if (h) aob_ls_destroy(h);
  }
};

inline int centro_type(const std::string &t) {
  if (t == "cog") return AOB_CENTRO_COG;
  if (t == "tcog") return AOB_CENTRO_TCOG;
  if (t == "wcog") return AOB_CENTRO_WCOG;
  if (t == "pyr" || t == "pyrhr") return AOB_CENTRO_PYR;
  if (t == "maskedpix") return AOB_CENTRO_MASKEDPIX;
  if (t == "bpcog") return AOB_CENTRO_BPCOG;
  throw py::value_error("centroider type '" + t + "' is not supported (cog, tcog, wcog, bpcog, pyr, maskedpix)");
}

struct Centroider {
  std::string type;
  int device = 0, nvalid = 0, npix = 0, nmax = 0;
  float offset = 0.f, scale = 1.f, threshold = 0.f;
  std::shared_ptr<CentroOwner> c;
  std::shared_ptr<Wfs> wfs;
  std::vector<py::ssize_t> img_shape;
  bool tin_u16 = false;                            // Rtc_UFF: frames are uint16
  py::dtype raw_dtype = py::dtype::of<float>();  // type of the loaded frame

  int nslopes() const { return type == "maskedpix" ? nvalid : 2 * nvalid; }
  DevArr buffer(const char *which, py::dtype dt, std::vector<py::ssize_t> shape = {}) const {
    void *p = nullptr;
    int64_t n = 0;
    check(aob_centro_buffer(c->h, which, &p, &n), which);
    return DevArr((uintptr_t)p, n, std::move(dt), std::move(shape), c);
  }
  void get_cog_into(uintptr_t dev_slopes) {
    check(aob_centro_get_cog(c->h, reinterpret_cast<float *>(dev_slopes), nullptr), "get_cog");
  }
};

struct Controller {
  std::string type;
  int nslope = 0, nactu = 0;
  float delay = 0.f, gain = 0.f;
  std::pair<float, float> comRange{-1.0e6f, 1.0e6f};
  std::vector<int> centro_idx;
  std::vector<int> dm_idx;  // the DMs it drives (indexes into the Dms given to do_imat)
  bool dm_idx_set = false;
  std::shared_ptr<LsOwner> l;
  // perturbation voltages: name -> (voltages [N, nactu], row counter, enabled), N
  std::map<std::string, std::tuple<py::object, int, bool>> perturb;
  std::map<std::string, int> perturb_n;
  virtual ~Controller() = default;
  void advance_perturb() {
    for (auto &kv : perturb)
      if (std::get<2>(kv.second)) std::get<1>(kv.second) = (std::get<1>(kv.second) + 1) % perturb_n[kv.first];
  }
  DevArr buffer(const char *which, std::vector<py::ssize_t> shape = {}) const {
    void *p = nullptr;
    int64_t n = 0;
    check(aob_ls_buffer(l->h, which, &p, &n), which);
    return DevArr((uintptr_t)p, n, py::dtype::of<float>(), std::move(shape), l);
  }
};
struct ControllerLS : Controller {};
struct ControllerGENERIC : Controller {};

struct Rtc {
  bool u16 = false;  // Rtc_UFF
  virtual ~Rtc() = default;
  std::vector<std::shared_ptr<Centroider>> centro;
  std::vector<std::shared_ptr<Controller>> control;
  Controller &ctl(int n) { return *control.at(n); }
};

inline farray<float> checked_matrix(const py::object &o, int rows, int cols, const char *what) {
  farray<float> a = o.cast<farray<float>>();
  if (a.ndim() != 2 || a.shape(0) != rows || a.shape(1) != cols)
    throw std::runtime_error(std::string(what) + " must be (" + std::to_string(rows) + ", " + std::to_string(cols) +
                             ")");
  return a;
}

inline void bind_rtc(py::module_ &m) {
  py::class_<Centroider, std::shared_ptr<Centroider>>(m, "Centroider")
      .def_readonly("type", &Centroider::type)
      .def_readonly("nvalid", &Centroider::nvalid)
      .def_readonly("npix", &Centroider::npix)
      .def_readonly("offset", &Centroider::offset)
      .def_readonly("scale", &Centroider::scale)
      .def_readonly("threshold", &Centroider::threshold)
      .def_readonly("nmax", &Centroider::nmax)
      .def_property_readonly("nslopes", &Centroider::nslopes)
      .def_property_readonly("wfs", [](const Centroider &x) -> py::object {
        return x.wfs ? py::cast(x.wfs) : py::object(py::none());
      })
      .def_property_readonly("d_img", [](const Centroider &x) { return x.buffer("img", py::dtype::of<float>(), x.img_shape); })
      .def_property_readonly("d_dark", [](const Centroider &x) { return x.buffer("dark", py::dtype::of<float>(), x.img_shape); })
      .def_property_readonly("d_flat", [](const Centroider &x) { return x.buffer("flat", py::dtype::of<float>(), x.img_shape); })
      .def_property_readonly("d_centroids_ref",
                             [](const Centroider &x) { return x.buffer("centroids_ref", py::dtype::of<float>()); })
      .def_property_readonly("d_intensities",
                             [](const Centroider &x) { return x.buffer("intensities", py::dtype::of<float>()); })
      .def_property_readonly("d_validx", [](const Centroider &x) { return x.buffer("validx", py::dtype::of<int32_t>()); })
      .def_property_readonly("d_validy", [](const Centroider &x) { return x.buffer("validy", py::dtype::of<int32_t>()); })
      .def_property_readonly("d_weights", [](const Centroider &x) { return x.buffer("weights", py::dtype::of<float>()); })
      .def("get_cog",
           [](Centroider &x) {
             // centroids of the sensor's current image into its d_slopes (centroider.cpp:186-188)
             if (!x.wfs) throw std::runtime_error("get_cog: the centroider has no sensor (use Rtc.do_centroids)");
             x.get_cog_into(x.wfs->buffer("slopes", py::dtype::of<float>()).ptr);
             return 0;
           })
      .def("load_validpos",
           [](Centroider &x, const farray<int32_t> &vx, const farray<int32_t> &vy, int N) {
             if (vx.size() < N || vy.size() < N) throw std::runtime_error("load_validpos: fewer than N positions");
             check(aob_centro_load_validpos(x.c->h, vx.data(), vy.data(), N), "load_validpos");
           })
      .def("set_npix",
           [](Centroider &x, int n) {
             x.npix = n;
             check(aob_centro_set_npix(x.c->h, n), "set_npix");
           })
      .def("set_scale",
           [](Centroider &x, float v) {
             x.scale = v;
             check(aob_centro_set_scale(x.c->h, v), "set_scale");
           })
      .def("set_offset",
           [](Centroider &x, float v) {
             x.offset = v;
             check(aob_centro_set_offset(x.c->h, v), "set_offset");
           })
      .def("set_threshold",
           [](Centroider &x, float v) {
             x.threshold = v;
             check(aob_centro_set_threshold(x.c->h, v), "set_threshold");
           })
      .def("set_nmax",
           [](Centroider &x, int v) {
             // bpCoG (centroider_bpcog.cpp): rank of the threshold pixel
             x.nmax = v;
             check(aob_centro_set_nmax(x.c->h, v), "set_nmax");
           })
      .def("init_weights", [](Centroider &) { return 0; })  // allocated by load_weights (centroider_wcog.cpp:61-62)
      .def("set_pyr_method",
           [](Centroider &x, int method) { check(aob_centro_set_pyr_method(x.c->h, method), "set_pyr_method"); })
      .def("set_pyr_thresh",
           [](Centroider &x, float t) { check(aob_centro_set_pyr_thresh(x.c->h, t), "set_pyr_thresh"); })
      .def(
          "load_weights",
          [](Centroider &x, const farray<float> &w, int) {
            check(aob_centro_load_weights(x.c->h, w.data(), (int64_t)w.size()), "load_weights");
          },
          py::arg("weights"), py::arg("ndim") = 2)
      .def("set_centroids_ref",
           [](Centroider &x, const farray<float> &r) {
             if (r.size() < x.nslopes()) throw std::runtime_error("set_centroids_ref: too few reference slopes");
             check(aob_centro_set_centroids_ref(x.c->h, r.data()), "set_centroids_ref");
           })
      .def("load_img",
           [](Centroider &x, py::object img, py::args) {
             // a frame from the host, cast to the RTC's input type as the reference's
             // binding does, or for a uint16 RTC a uint16 device array (a sensor's d_camimg)
             if (py::isinstance<DevArr>(img) || py::hasattr(img, "__cuda_array_interface__")) {
               // a device frame: 2-D uint16 in column-major order (the layout of this
               // library's buffers), copied on the device
               py::dict cai = img.attr("__cuda_array_interface__");
               const auto shape = cai["shape"].cast<std::vector<py::ssize_t>>();
               const std::string ts = cai["typestr"].cast<std::string>();
               const bool fortran = cai.contains("strides") && !cai["strides"].is_none() && shape.size() == 2 &&
                                    cai["strides"].cast<std::vector<py::ssize_t>>() ==
                                        std::vector<py::ssize_t>{2, 2 * shape[0]};
               if (ts != "<u2" || shape.size() != 2 || !fortran)
                 throw std::runtime_error("load_img from device memory takes a 2-D column-major uint16 frame");
               const auto ptr = cai["data"].cast<py::tuple>()[0].cast<uintptr_t>();
               x.img_shape = shape;
               x.raw_dtype = py::dtype::of<uint16_t>();
               check(aob_centro_load_img_u16(x.c->h, reinterpret_cast<const uint16_t *>(ptr), (int)shape[0],
                                             (int)shape[1], 1, nullptr),
                     "load_img");
               return 0;
             }
             if (x.tin_u16) {
               farray<uint16_t> a = img.cast<farray<uint16_t>>();
               if (a.ndim() != 2) throw std::runtime_error("load_img: a 2-D image is required");
               x.img_shape = {a.shape(0), a.shape(1)};
               x.raw_dtype = py::dtype::of<uint16_t>();
               check(aob_centro_load_img_u16(x.c->h, a.data(), (int)a.shape(0), (int)a.shape(1), 0, nullptr),
                     "load_img");
               return 0;
             }
             farray<float> a = img.cast<farray<float>>();
             if (a.ndim() != 2) throw std::runtime_error("load_img: a 2-D image is required");
             x.img_shape = {a.shape(0), a.shape(1)};
             x.raw_dtype = py::dtype::of<float>();
             check(aob_centro_load_img(x.c->h, a.data(), (int)a.shape(0), (int)a.shape(1)), "load_img");
             return 0;
           })
      .def_property_readonly("d_img_raw",
                             [](const Centroider &x) { return x.buffer("img_raw", x.raw_dtype, x.img_shape); })
      .def(
          "set_lutPix",
          [](Centroider &x, const farray<int32_t> &lut, py::object) {
            check(aob_centro_set_lut_pix(x.c->h, lut.data(), (int)lut.size()), "set_lutPix");
            return 0;
          },
          py::arg("lutPix"), py::arg("n") = py::none())
      .def("calibrate_img_validPix",
           [](Centroider &x) {
             check(aob_centro_calibrate_img_validpix(x.c->h, nullptr), "calibrate_img_validPix");
             return 0;
           })
      .def("calibrate_img", [](Centroider &x) { check(aob_centro_calibrate_img(x.c->h, nullptr), "calibrate_img"); })
      .def("set_dark",
           [](Centroider &x, const farray<float> &d, int n) {
             if (x.img_shape.empty()) x.img_shape = {n, n};
             check(aob_centro_set_dark(x.c->h, d.data(), n), "set_dark");
           })
      .def("set_flat", [](Centroider &x, const farray<float> &f, int n) {
        if (x.img_shape.empty()) x.img_shape = {n, n};
        check(aob_centro_set_flat(x.c->h, f.data(), n), "set_flat");
      });
}

}  // namespace aobpy
