// Sensors of the compiled drop-in `sutra`: SutraWfsSH (python_module/sutra/src/wfs_sh.cpp:41-148),
// SutraWfs_PyrHR (wfs_pyrhr.cpp:131-163), their common Wfs properties and methods
// (wfs.cpp:54-300), the guide star a sensor sees (d_gs.d_phase.d_screen,
// add_layer) and SutraSensors (sensors.cpp:28-210).  Every method calls the C ABI
// of libaob200 directly.
#pragma once

#include <cmath>
#include <map>
#include <type_traits>

#include "native_common.hpp"

namespace aobpy {

struct ShOwner {
  aob_sh *h = nullptr;
  ~ShOwner() {
    if (h) aob_sh_destroy(h);
  }
};
struct PyrOwner {
  aob_pyr *h = nullptr;
  ~PyrOwner() {
    if (h) aob_pyr_destroy(h);
  }
};

// numpy's view of an argument: element i of np.asarray(a).ravel() (the reference
// passes per-sensor arrays; a scalar stands for every sensor), converted as
// Python's int() / float() / bool() would (a float index array counts)
template <typename T>
T elem(const py::object &a, int i) {
  py::module_ np = py::module_::import("numpy");
  py::object r = np.attr("asarray")(a).attr("ravel")();
  const int n = r.attr("size").cast<int>();
  py::object v = r[py::int_(n == 1 ? 0 : i)];
  if constexpr (std::is_same_v<T, bool>)
    return py::bool_(v).cast<bool>();
  else if constexpr (std::is_integral_v<T>)
    return py::int_(v).cast<T>();
  else
    return py::float_(v).cast<T>();
}

// The guide star's phase screen of one sensor: d_gs.d_phase.d_screen
struct PhaseView {
  std::shared_ptr<void> owner;
  aob_sh *sh = nullptr;
  aob_pyr *pyr = nullptr;
  int side = 0;
  DevArr screen() const {
    void *p = nullptr;
    int64_t n = 0;
    if (sh)
      check(aob_sh_buffer(sh, "phase", &p, &n), "d_screen");
    else
      check(aob_pyr_buffer(pyr, "phase", &p, &n), "d_screen");
    return DevArr((uintptr_t)p, n, py::dtype::of<float>(), {side, side}, owner);
  }
};

// wfs.d_gs: the phase it sees and the DM layers placed on it (SutraSource::add_layer)
struct GuideStar {
  PhaseView phase;
  float lambda_um = 0.5f;
  std::map<int, std::pair<float, float>> dm_layers;
};

struct Wfs {
  std::string type;  // "sh" or "pyrhr"
  int device = 0, nxsub = 0, nvalid = 0, npix = 0, nphase = 0, nrebin = 0, nfft = 0, ntot = 0, npup = 0;
  float pdiam = 0.f, nphot = 0.f, nphot4imat = 0.f, noise = -1.f;
  std::shared_ptr<ShOwner> sh;
  std::shared_ptr<PyrOwner> pyr;
  std::shared_ptr<GuideStar> gs;
  bool compute_focal = false;

  virtual ~Wfs() = default;
  std::shared_ptr<void> owner() const {
    return sh ? std::shared_ptr<void>(sh) : std::shared_ptr<void>(pyr);
  }
  DevArr buffer(const char *which, py::dtype dtype, std::vector<py::ssize_t> shape = {}) const {
    void *p = nullptr;
    int64_t n = 0;
    if (sh)
      check(aob_sh_buffer(sh->h, which, &p, &n), which);
    else
      check(aob_pyr_buffer(pyr->h, which, &p, &n), which);
    return DevArr((uintptr_t)p, n, std::move(dtype), std::move(shape), owner());
  }
  PhaseView phase_view() const {
    PhaseView v;
    v.owner = owner();
    v.sh = sh ? sh->h : nullptr;
    v.pyr = pyr ? pyr->h : nullptr;
    v.side = sh ? npup : ntot;
    return v;
  }
  void comp_image(bool noise) {
    if (sh)
      check(aob_sh_comp_image(sh->h, noise ? 1 : 0, nullptr), "comp_image");
    else
      check(aob_pyr_comp_image(pyr->h, noise ? 1 : 0, nullptr), "comp_image");
  }
  void set_noise(float nz, int64_t seed) {
    noise = nz;
    if (sh)
      check(aob_sh_set_noise(sh->h, nz, seed), "set_noise");
    else
      check(aob_pyr_set_noise(pyr->h, nz, seed), "set_noise");
  }
  void set_lambda(float lam) {
    if (sh)
      check(aob_sh_set_lambda(sh->h, lam), "set_lambda");
    else
      check(aob_pyr_set_lambda(pyr->h, lam), "set_lambda");
  }
  void set_nphot(float n) {
    nphot = n;
    if (sh)
      check(aob_sh_set_nphot(sh->h, n), "set_nphot");
    else
      check(aob_pyr_set_nphot(pyr->h, n), "set_nphot");
  }
  void set_pupil(const farray<float> &p) {
    const int side = sh ? npup : ntot;
    if (p.size() != (py::ssize_t)side * side)
      throw std::runtime_error("set_pupil: the pupil must be " + std::to_string(side) + " x " + std::to_string(side));
    if (sh)
      check(aob_sh_set_pupil(sh->h, p.data()), "set_pupil");
    else
      check(aob_pyr_set_pupil(pyr->h, p.data()), "set_pupil");
  }
  void set_binimg(const farray<float> &img, int64_t nelem) {
    if (img.size() != nelem) throw std::runtime_error("set_binimg: nElem does not match the array");
    if (sh)
      check(aob_sh_set_binimg(sh->h, img.data(), nelem), "set_binimg");
    else
      check(aob_pyr_set_binimg(pyr->h, img.data(), nelem), "set_binimg");
  }
  void slopes_geom(int kind) {
    if (sh)
      check(aob_sh_slopes_geom(sh->h, kind, nullptr, nullptr), "slopes_geom");
    else
      check(aob_pyr_slopes_geom(pyr->h, kind, nullptr, nullptr), "slopes_geom");
  }
  DevArr d_binimg() const {
    const int side = sh ? npix * nxsub : nfft / nrebin;
    return buffer("binimg", py::dtype::of<float>(), {side, side});
  }
};

inline void bind_wfs(py::module_ &m) {
  py::class_<PhaseView>(m, "Phase")
      .def_property_readonly("d_screen", &PhaseView::screen);
  py::class_<GuideStar, std::shared_ptr<GuideStar>>(m, "Source")
      .def_property_readonly("d_phase", [](const GuideStar &g) { return g.phase; })
      .def_readonly("Lambda", &GuideStar::lambda_um)
      .def("add_layer",
           [](GuideStar &g, const std::string &type, int idx, float xoff, float yoff) {
             if (type == "pzt" || type == "tt" || type == "kl") g.dm_layers[idx] = {xoff, yoff};
             return 0;
           })
      .def_property_readonly("dm_layers", [](const GuideStar &g) { return g.dm_layers; });

  auto w = py::class_<Wfs, std::shared_ptr<Wfs>>(m, "Wfs");
  w.def_readonly("type", &Wfs::type)
      .def_readonly("nvalid", &Wfs::nvalid)
      .def_readonly("npix", &Wfs::npix)
      .def_readonly("nfft", &Wfs::nfft)
      .def_readonly("ntot", &Wfs::ntot)
      .def_readonly("nphase", &Wfs::nphase)
      .def_readonly("nrebin", &Wfs::nrebin)
      .def_readonly("nxsub", &Wfs::nxsub)
      .def_readonly("nphot", &Wfs::nphot)
      .def_readonly("noise", &Wfs::noise)
      .def_property_readonly("d_gs", [](const Wfs &x) -> py::object {
        return x.gs ? py::cast(x.gs) : py::object(py::none());
      })
      .def_property_readonly("d_binimg", &Wfs::d_binimg)
      .def_property_readonly("d_validsubsx",
                             [](const Wfs &x) { return x.buffer("validsubsx", py::dtype::of<int32_t>()); })
      .def_property_readonly("d_validsubsy",
                             [](const Wfs &x) { return x.buffer("validsubsy", py::dtype::of<int32_t>()); })
      .def_property_readonly("d_fluxPerSub", [](const Wfs &x) { return x.buffer("fluxPerSub", py::dtype::of<float>()); })
      .def_property_readonly("d_slopes", [](const Wfs &x) { return x.buffer("slopes", py::dtype::of<float>()); })
      .def("comp_image", &Wfs::comp_image, py::arg("noise") = true)
      .def("set_noise", &Wfs::set_noise, py::arg("noise"), py::arg("seed"))
      .def("set_pupil", &Wfs::set_pupil)
      .def("set_binimg", &Wfs::set_binimg, py::arg("binimg"), py::arg("nElem"))
      .def(
          "slopes_geom",
          [](Wfs &x, py::args args, py::kwargs kw) {
            // slopes_geom(type=0) into d_slopes, or slopes_geom(slopes, type=0) into a
            // host float32 array (wfs.cpp:242-262)
            py::object slopes = py::none();
            size_t i = 0;
            if (args.size() > 0 && py::isinstance<py::array>(args[0])) slopes = args[i++];
            if (kw.contains("slopes")) slopes = kw["slopes"];
            int kind = 0;
            if (args.size() > i)
              kind = args[i].cast<int>();
            else if (kw.contains("type"))
              kind = kw["type"].cast<int>();
            x.slopes_geom(kind);
            if (!slopes.is_none()) {
              py::array h = x.buffer("slopes", py::dtype::of<float>()).host();
              slopes.attr("__setitem__")(py::ellipsis(),
                                          h.attr("reshape")(slopes.attr("shape"), py::arg("order") = "F"));
            }
            return 0;
          });
}

}  // namespace aobpy
