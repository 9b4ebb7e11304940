// Piezo-stack DMs of the compiled drop-in `sutra`: SutraDms / SutraDm
// (python_module/sutra/src/dms.cpp:120-600) as shesha's dm_init loads them
// (pzt_loadarrays with the influence functions and each actuator's corner).
#pragma once

#include <algorithm>

#include "native_common.hpp"

namespace aobpy {

struct DmOwner {
  aob_dm *h = nullptr;
  ~DmOwner() {
    if (h) aob_dm_destroy(h);
  }
};

// a device buffer allocated here and freed with its owner
struct DevAlloc {
  void *p = nullptr;
  DevAlloc(size_t bytes, int device) { check(aob_malloc(&p, bytes, device), "device allocation"); }
  ~DevAlloc() {
    if (p) aob_free(p);
  }
  DevAlloc(const DevAlloc &) = delete;
  DevAlloc &operator=(const DevAlloc &) = delete;
};

struct Dm {
  std::string type;
  float altitude = 0.f, push4imat = 0.f;
  int dim = 0, nactus = 0, influsize = 0, device = 0;
  std::shared_ptr<DmOwner> d;
  std::shared_ptr<DevAlloc> one;  // the single-actuator command of comp_oneactu

  aob_dm *need() const {
    if (!d) throw std::runtime_error("Dm: pzt_loadarrays has not been called");
    return d->h;
  }
  DevArr buffer(const char *which, std::vector<py::ssize_t> shape = {}) const {
    void *p = nullptr;
    int64_t n = 0;
    check(aob_dm_buffer(need(), which, &p, &n), which);
    return DevArr((uintptr_t)p, n, py::dtype::of<float>(), std::move(shape), d);
  }
  void comp_shape() { check(aob_dm_comp_shape(need(), nullptr, nullptr), "comp_shape"); }

  // The influence functions [influsize, influsize, nactus] and each actuator's corner
  // (xoff, yoff) on the support, as dm_init.py:186-193 passes them.  influpos /
  // npoints / istart (the reference's pixel lists) give the support's offset when it
  // is smaller than the screen: comp_dmgeom (dm_init.py:902-955) places actuator a's
  // sample (x, y) at pixel (offs + i1[a] + x) + dim (offs + j1[a] + y).
  void pzt_loadarrays(const farray<float> &influ, const py::array_t<int64_t, py::array::forcecast> &influpos,
                      const py::array_t<int64_t, py::array::forcecast> &npoints,
                      const py::array_t<int64_t, py::array::forcecast> &istart,
                      const py::array_t<int64_t, py::array::forcecast> &xoff,
                      const py::array_t<int64_t, py::array::forcecast> &yoff) {
    if (influ.ndim() != 3) throw std::runtime_error("pzt_loadarrays: influ must be [influsize, influsize, nactus]");
    const int s = (int)influ.shape(0), nact = (int)influ.shape(2);
    if (xoff.size() < nact || yoff.size() < nact) throw std::runtime_error("pzt_loadarrays: one corner per actuator");
    const int64_t *np_ = npoints.data(), *ist = istart.data(), *pos = influpos.data(), *i1 = xoff.data(),
                  *j1 = yoff.data();
    int64_t off = 0;
    const int64_t lim = std::min<int64_t>(npoints.size(), (int64_t)dim * dim);
    for (int64_t p = 0; p < lim; ++p) {
      if (!np_[p]) continue;
      if (ist[p] < 0 || ist[p] >= influpos.size()) throw std::runtime_error("pzt_loadarrays: istart out of range");
      const int64_t q = pos[ist[p]];
      const int64_t a = q / ((int64_t)s * s), y = (q / s) % s, x = q % s;
      if (a < 0 || a >= nact) throw std::runtime_error("pzt_loadarrays: influpos out of range");
      off = p % dim - x - i1[a];
      if (p / dim - y - j1[a] != off) throw std::runtime_error("pzt_loadarrays: influpos does not match xoff / yoff");
      break;
    }
    std::vector<int32_t> ii(nact), jj(nact);
    for (int a = 0; a < nact; ++a) {
      ii[a] = (int32_t)(i1[a] + off);
      jj[a] = (int32_t)(j1[a] + off);
    }
    auto o = std::make_shared<DmOwner>();
    check(aob_dm_create(&o->h, device, dim, nact, s, influ.data(), ii.data(), jj.data()), "pzt_loadarrays");
    d = o;
    nactus = nact;
    influsize = s;
  }
};

struct Dms {
  std::vector<std::shared_ptr<Dm>> dms;
};

inline void bind_dms(py::module_ &m) {
  py::class_<Dm, std::shared_ptr<Dm>>(m, "Dm")
      .def_readonly("type", &Dm::type)
      .def_readonly("altitude", &Dm::altitude)
      .def_readonly("dim", &Dm::dim)
      .def_readonly("nactus", &Dm::nactus)
      .def_readonly("influsize", &Dm::influsize)
      .def_readonly("push4imat", &Dm::push4imat)
      .def_readonly("device", &Dm::device)
      .def("pzt_loadarrays",
           [](Dm &x, const farray<float> &influ, const py::array_t<int64_t, py::array::forcecast> &influpos,
              const py::array_t<int64_t, py::array::forcecast> &npoints,
              const py::array_t<int64_t, py::array::forcecast> &istart,
              const py::array_t<int64_t, py::array::forcecast> &xoff,
              const py::array_t<int64_t, py::array::forcecast> &yoff) {
             x.pzt_loadarrays(influ, influpos, npoints, istart, xoff, yoff);
             return 0;
           })
      .def_property_readonly("d_shape", [](const Dm &x) { return x.buffer("shape", {x.dim, x.dim}); })
      .def_property_readonly("d_com", [](const Dm &x) { return x.buffer("com"); })
      .def(
          "set_com",
          [](Dm &x, py::object com, bool shape_dm) {
            x.buffer("com").set(com);
            if (shape_dm) x.comp_shape();
            return 0;
          },
          py::arg("com"), py::arg("shape_dm") = true)
      .def(
          "comp_shape",
          [](Dm &x, py::object com) {
            if (!com.is_none()) x.buffer("com").set(com);
            x.comp_shape();
            return 0;
          },
          py::arg("com") = py::none())
      .def("reset_shape",
           [](Dm &x) {
             DevArr s = x.buffer("shape", {x.dim, x.dim});
             check(aob_fill_f32(reinterpret_cast<float *>(s.ptr), (size_t)s.n, 0.f, nullptr), "reset_shape");
             return 0;
           })
      .def("comp_oneactu", [](Dm &x, int nactu, float ampli) {
        // the shape of one actuator alone at ampli volts; d_com is left as it is
        aob_dm *h = x.need();
        if (nactu < 0 || nactu >= x.nactus) throw std::runtime_error("comp_oneactu: actuator out of range");
        if (!x.one) x.one = std::make_shared<DevAlloc>(sizeof(float) * (size_t)x.nactus, x.device);
        std::vector<float> v((size_t)x.nactus, 0.f);
        v[(size_t)nactu] = ampli;
        check(aob_memcpy_h2d(x.one->p, v.data(), sizeof(float) * v.size(), nullptr), "comp_oneactu");
        check(aob_dm_comp_shape(h, static_cast<const float *>(x.one->p), nullptr), "comp_oneactu");
        return 0;
      });

  py::class_<Dms, std::shared_ptr<Dms>>(m, "Dms")
      .def(py::init([]() { return std::make_shared<Dms>(); }))
      .def_property_readonly("d_dms", [](const Dms &x) { return x.dms; })
      .def("add_dm",
           [](Dms &x, py::object context, const std::string &type, float alt, int dim, int nactus, int influsize,
              int ninflupos, int n_npoints, float push4imat, int nord, py::args rest) {
             // both reference overloads: (..., nord, device) and
             // (..., nord, dx, dy, thetaML, G, device); only dx = dy = thetaML = 0, G = 1
             int device = 0;
             if (rest.size() == 5) {
               if (rest[0].cast<double>() != 0 || rest[1].cast<double>() != 0 || rest[2].cast<double>() != 0 ||
                   rest[3].cast<double>() != 1)
                 throw py::value_error("add_dm: DM mis-registration is not supported");
               device = rest[4].cast<int>();
             } else if (rest.size() == 1) {
               device = rest[0].cast<int>();
             } else {
               throw py::type_error("add_dm: expected (..., nord, device) or (..., nord, dx, dy, thetaML, G, device)");
             }
             if (type != "pzt") throw py::value_error("add_dm: DM type '" + type + "' is not supported (pzt)");
             auto d = std::make_shared<Dm>();
             d->type = type, d->altitude = alt, d->dim = dim, d->nactus = nactus, d->influsize = influsize;
             d->push4imat = push4imat, d->device = device;
             x.dms.push_back(d);
             return 0;
           })
      .def("remove_dm", [](Dms &x, int idx) {
        x.dms.erase(x.dms.begin() + idx);
        return 0;
      });
}

}  // namespace aobpy
