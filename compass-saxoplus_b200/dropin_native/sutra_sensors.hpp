// SHWFS, PYRWFS and Sensors of the compiled drop-in `sutra` (wfs_sh.cpp:41-148,
// wfs_pyrhr.cpp:131-163, sensors.cpp:28-210).
#pragma once

#include "sutra_wfs.hpp"

namespace aobpy {

struct SHWFS : Wfs {};
struct PYRWFS : Wfs {};

// An optional array argument (None -> no pointer), kept alive by the caller's local
template <typename T>
struct Opt {
  farray<T> a;
  bool set = false;
  explicit Opt(const py::object &o) {
    if (!o.is_none()) {
      a = o.cast<farray<T>>();
      set = true;
    }
  }
  const T *ptr() const { return set ? a.data() : nullptr; }
};

inline std::shared_ptr<SHWFS> make_sh(int nxsub, int nvalid, int npix, int nphase, int nrebin, int nfft, int ntot,
                                      int npup, float pdiam, float nphot, float nphot4imat, int device) {
  auto w = std::make_shared<SHWFS>();
  w->type = "sh";
  w->device = device;
  w->nxsub = nxsub, w->nvalid = nvalid, w->npix = npix, w->nphase = nphase, w->nrebin = nrebin;
  w->nfft = nfft, w->ntot = ntot, w->npup = npup;
  w->pdiam = pdiam, w->nphot = nphot, w->nphot4imat = nphot4imat;
  w->sh = std::make_shared<ShOwner>();
  check(aob_sh_create(&w->sh->h, device, nxsub, nvalid, npix, nphase, nrebin, nfft, ntot, npup, pdiam, nphot,
                      nphot4imat),
        "SHWFS");
  return w;
}

inline std::shared_ptr<PYRWFS> make_pyr(int nxsub, int nvalid, int npix, int nphase, int nrebin, int nfft, int ntot,
                                        int npts, float pdiam, float nphot, float nphot4imat, int device) {
  auto w = std::make_shared<PYRWFS>();
  w->type = "pyrhr";
  w->device = device;
  w->nxsub = nxsub, w->nvalid = nvalid, w->npix = npix, w->nphase = nphase, w->nrebin = nrebin;
  w->nfft = nfft, w->ntot = ntot, w->npup = npts;
  w->pdiam = pdiam, w->nphot = nphot, w->nphot4imat = nphot4imat;
  w->pyr = std::make_shared<PyrOwner>();
  check(aob_pyr_create(&w->pyr->h, device, nxsub, nvalid, npix, nphase, nrebin, nfft, ntot, npts, pdiam, nphot,
                       nphot4imat),
        "PYRWFS");
  return w;
}

struct Sensors {
  int device = 0;
  std::vector<std::shared_ptr<Wfs>> wfs;
};

inline void bind_sensors(py::module_ &m) {
  py::class_<SHWFS, Wfs, std::shared_ptr<SHWFS>>(m, "SHWFS")
      .def(py::init(&make_sh), py::arg("nxsub"), py::arg("nvalid"), py::arg("npix"), py::arg("nphase"),
           py::arg("nrebin"), py::arg("nfft"), py::arg("ntot"), py::arg("npup"), py::arg("pdiam"), py::arg("nphot"),
           py::arg("nphot4imat"), py::arg("device"))
      .def(
          "load_arrays",
          [](SHWFS &w, py::object phasemap, py::object hrmap, const farray<int32_t> &binmap,
             const farray<float> &offsets, const farray<float> &flux, const farray<int32_t> &vx,
             const farray<int32_t> &vy, const farray<int32_t> &istart, const farray<int32_t> &jstart,
             py::object ttprojmat, py::object kernel) {
            // hrmap is read when the field of view is extended (ntot != nfft); phasemap
            // and ttprojmat are kept for the geometric slopes
            Opt<int32_t> pm(phasemap), hr(w.ntot != w.nfft ? hrmap : py::none());
            Opt<float> tt(ttprojmat);
            check(aob_sh_load_arrays(w.sh->h, pm.ptr(), hr.ptr(), binmap.data(), offsets.data(), flux.data(),
                                     vx.data(), vy.data(), istart.data(), jstart.data(), tt.ptr(), nullptr),
                  "load_arrays");
          },
          py::arg("phasemap"), py::arg("hrmap"), py::arg("binmap"), py::arg("offsets"), py::arg("fluxPerSub"),
          py::arg("validsubsx"), py::arg("validsubsy"), py::arg("istart"), py::arg("jstart"),
          py::arg("ttprojmat") = py::none(), py::arg("kernel") = py::none())
      .def_property_readonly("d_bincube",
                             [](const SHWFS &w) {
                               return w.buffer("bincube", py::dtype::of<float>(), {w.npix, w.npix, w.nvalid});
                             })
      .def_property_readonly("d_intensities", [](const SHWFS &w) { return w.buffer("intensities", py::dtype::of<float>()); })
      .def_property_readonly("d_binmap", [](const SHWFS &w) { return w.buffer("binmap", py::dtype::of<int32_t>()); })
      .def_property_readonly("d_validpuppixx", [](const SHWFS &w) { return w.buffer("istart", py::dtype::of<int32_t>()); })
      .def_property_readonly("d_validpuppixy", [](const SHWFS &w) { return w.buffer("jstart", py::dtype::of<int32_t>()); })
      .def_property_readonly("d_camimg",
                             [](const SHWFS &w) {
                               const int side = w.npix * w.nxsub;
                               return w.buffer("camimg", py::dtype::of<uint16_t>(), {side, side});
                             })
      .def(
          "fill_binimage", [](SHWFS &w, bool) { check(aob_sh_fill_binimage(w.sh->h, nullptr), "fill_binimage"); },
          py::arg("async") = false)
      .def(
          "comp_nphot",
          [](SHWFS &w, float ittime, float optthroughput, float diam, int nxsub, float zerop, float gsmag,
             float lgsreturnperwatt, float laserpower) {
            // photons per sub-aperture and frame (sutra_wfs_sh.cpp:645-663)
            double nphot;
            if (laserpower == 0.f) {
              const double zp = zerop == 0.f ? 1e11 : (double)zerop;
              nphot = zp * std::pow(10.0, -0.4 * (double)gsmag) * ittime * optthroughput * std::pow((double)diam / nxsub, 2);
            } else {
              nphot = (double)lgsreturnperwatt * laserpower * optthroughput * std::pow((double)diam / nxsub, 2) * 1e4 *
                      ittime;
            }
            w.set_nphot((float)nphot);
            return 0;
          },
          py::arg("ittime"), py::arg("optthroughput"), py::arg("diam"), py::arg("nxsub"), py::arg("zerop") = 0.f,
          py::arg("gsmag") = 0.f, py::arg("lgsreturnperwatt") = 0.f, py::arg("laserpower") = 0.f)
      .def("set_bincube",
           [](SHWFS &w, const farray<float> &cube, int64_t nelem) {
             if (cube.size() != nelem) throw std::runtime_error("set_bincube: nElem does not match the array");
             check(aob_sh_set_bincube(w.sh->h, cube.data(), nelem), "set_bincube");
             return 0;
           })
      .def("set_dark",
           [](SHWFS &w, const farray<float> &d, int n) { check(aob_sh_set_dark(w.sh->h, d.data(), n), "set_dark"); })
      .def("set_flat",
           [](SHWFS &w, const farray<float> &f, int n) { check(aob_sh_set_flat(w.sh->h, f.data(), n), "set_flat"); });

  py::class_<PYRWFS, Wfs, std::shared_ptr<PYRWFS>>(m, "PYRWFS")
      .def(py::init(&make_pyr), py::arg("nxsub"), py::arg("nvalid"), py::arg("npix"), py::arg("nphase"),
           py::arg("nrebin"), py::arg("nfft"), py::arg("ntot"), py::arg("npup"), py::arg("pdiam"), py::arg("nphot"),
           py::arg("nphot4imat"), py::arg("device"))
      .def(
          "load_arrays",
          [](PYRWFS &w, py::object halfxy, const farray<float> &cx, const farray<float> &cy, py::object weights,
             const farray<float> &sincar, const farray<float> &submask, const farray<int32_t> &vx,
             const farray<int32_t> &vy, py::object phasemap, py::object flux, py::object ttprojmat) {
            // the pyramid phase as exp(i halfxy), transposed, as wfs_init.py:203 passes it
            py::module_ np = py::module_::import("numpy");
            py::object j = py::module_::import("builtins").attr("complex")(0.0, 1.0);
            py::object c = np.attr("exp")(j * np.attr("asarray")(halfxy, np.attr("float64")))
                               .attr("astype")(np.attr("complex64"))
                               .attr("T");
            farray<float> hx = np.attr("asfortranarray")(c).attr("ravel")("F").attr("view")(np.attr("float32"))
                                   .attr("copy")()
                                   .cast<farray<float>>();
            farray<float> wt = weights.is_none() ? farray<float>(np.attr("ones")(cx.size(), np.attr("float32")))
                                                 : weights.cast<farray<float>>();
            Opt<int32_t> pm(phasemap);
            Opt<float> fl(flux), tt(ttprojmat);
            check(aob_pyr_load_arrays(w.pyr->h, hx.data(), cx.data(), cy.data(), wt.data(), sincar.data(),
                                      submask.data(), vx.data(), vy.data(), pm.ptr(), fl.ptr(), tt.ptr()),
                  "load_arrays");
            w.compute_focal = false;
          },
          py::arg("halfxy"), py::arg("cx"), py::arg("cy"), py::arg("weights"), py::arg("sincar"), py::arg("submask"),
          py::arg("validsubsx"), py::arg("validsubsy"), py::arg("phasemap") = py::none(),
          py::arg("fluxPerSub") = py::none(), py::arg("ttprojmat") = py::none())
      .def(
          "set_pyr_modulation_points",
          [](PYRWFS &w, const farray<float> &cx, const farray<float> &cy, py::object weights, py::object) {
            py::module_ np = py::module_::import("numpy");
            farray<float> wt = weights.is_none() ? farray<float>(np.attr("ones")(cx.size(), np.attr("float32")))
                                                 : weights.cast<farray<float>>();
            check(aob_pyr_set_modulation(w.pyr->h, cx.data(), cy.data(), wt.data(), (int)cx.size()),
                  "set_pyr_modulation_points");
            w.npup = (int)cx.size();
          },
          py::arg("cx"), py::arg("cy"), py::arg("weights") = py::none(), py::arg("npts") = py::none())
      .def_property_readonly("d_submask",
                             [](const PYRWFS &w) { return w.buffer("submask", py::dtype::of<float>(), {w.nfft, w.nfft}); })
      .def_property_readonly("d_hrimg",
                             [](const PYRWFS &w) { return w.buffer("hrimg", py::dtype::of<float>(), {w.nfft, w.nfft}); })
      .def_property_readonly(
          "d_pyrfocalplane",
          [](const PYRWFS &w) { return w.buffer("pyrfocalplane", py::dtype::of<float>(), {w.nfft, w.nfft}); })
      .def_property_readonly("d_phalfxy",
                             [](const PYRWFS &w) {
                               DevArr a = w.buffer("phalfxy", py::dtype::of<float>());
                               return DevArr(a.ptr, (int64_t)w.nfft * w.nfft, py::dtype("complex64"),
                                             {w.nfft, w.nfft}, a.owner);
                             })
      .def_property(
          "compute_pyrfocalplane", [](const PYRWFS &w) { return w.compute_focal; },
          [](PYRWFS &w, bool on) {
            // when set, every comp_image also forms d_pyrfocalplane (wfs_pyrhr.cpp:83-90)
            check(aob_pyr_set_compute_focalplane(w.pyr->h, on ? 1 : 0), "compute_pyrfocalplane");
            w.compute_focal = on;
          })
      .def("set_phalfxy",
           [](PYRWFS &w, py::object ph) {
             py::module_ np = py::module_::import("numpy");
             farray<float> a = np.attr("ascontiguousarray")(np.attr("asarray")(ph, np.attr("complex64")).attr("ravel")("F"))
                                   .attr("view")(np.attr("float32"))
                                   .cast<farray<float>>();
             check(aob_pyr_set_phalfxy(w.pyr->h, a.data(), (int64_t)(a.size() / 2)), "set_phalfxy");
             return 0;
           })
      .def("set_submask",
           [](PYRWFS &w, const farray<float> &s) {
             check(aob_pyr_set_submask(w.pyr->h, s.data(), (int64_t)s.size()), "set_submask");
             return 0;
           })
      .def("set_pyrimg",
           [](PYRWFS &w, const farray<float> &img) {
             check(aob_pyr_set_binimg(w.pyr->h, img.data(), (int64_t)img.size()), "set_pyrimg");
             return 0;
           })
      .def(
          "comp_nphot",
          [](PYRWFS &w, float ittime, float optthroughput, float diam, float cobs, float zerop, float gsmag) {
            // photons per frame over the pupil (sutra_wfs_pyr_pyrhr.cpp:722-729)
            const double nphot = (double)zerop * std::pow(10.0, -0.4 * (double)gsmag) * ittime * optthroughput *
                                 M_PI / 4.0 * (1.0 - (double)cobs * cobs) * (double)diam * diam;
            w.set_nphot((float)nphot);
            return 0;
          },
          py::arg("ittime"), py::arg("optthroughput"), py::arg("diam"), py::arg("cobs"), py::arg("zerop") = 0.f,
          py::arg("gsmag") = 0.f);

  py::class_<Sensors, std::shared_ptr<Sensors>>(m, "Sensors")
      .def(py::init([](py::object context, py::object d_tel, py::object type, int nwfs, py::object nxsub,
                       py::object nvalid, py::object npupils, py::object npix, py::object nphase, py::object nrebin,
                       py::object nfft, py::object ntot, py::object npup, py::object pdiam, py::object nphot,
                       py::object nphot4imat, py::object lgs, py::object fakecam, py::object max_flux_per_pix,
                       py::object max_pix_value, int device, py::object roket) {
             auto s = std::make_shared<Sensors>();
             s->device = device;
             for (int i = 0; i < nwfs; ++i) {
               const std::string t = py::str(type[py::int_(i)]);
               const int a0 = elem<int>(nxsub, i), a1 = elem<int>(nvalid, i), a2 = elem<int>(npix, i);
               const int a3 = elem<int>(nphase, i), a4 = elem<int>(nrebin, i), a5 = elem<int>(nfft, i);
               const int a6 = elem<int>(ntot, i), a7 = elem<int>(npup, i);
               const float f0 = elem<float>(pdiam, i), f1 = elem<float>(nphot, i), f2 = elem<float>(nphot4imat, i);
               if (t == "sh") {
                 auto w = make_sh(a0, a1, a2, a3, a4, a5, a6, a7, f0, f1, f2, device);
                 if (elem<bool>(fakecam, i))
                   check(aob_sh_set_fakecam(w->sh->h, 1, elem<int>(max_flux_per_pix, i), elem<int>(max_pix_value, i)),
                         "Sensors: fakecam");
                 s->wfs.push_back(w);
               } else if (t == "pyrhr") {
                 s->wfs.push_back(make_pyr(a0, a1, a2, a3, a4, a5, a6, a7, f0, f1, f2, device));
               } else {
                 throw py::value_error("Sensors: sensor type '" + t + "' is not supported (sh, pyrhr)");
               }
             }
             return s;
           }),
           py::arg("context"), py::arg("d_tel"), py::arg("type"), py::arg("nwfs"), py::arg("nxsub"), py::arg("nvalid"),
           py::arg("npupils"), py::arg("npix"), py::arg("nphase"), py::arg("nrebin"), py::arg("nfft"), py::arg("ntot"),
           py::arg("npup"), py::arg("pdiam"), py::arg("nphot"), py::arg("nphot4imat"), py::arg("lgs"),
           py::arg("fakecam"), py::arg("max_flux_per_pix"), py::arg("max_pix_value"), py::arg("device"),
           py::arg("roket"))
      .def_property_readonly("d_wfs", [](const Sensors &s) { return s.wfs; })
      .def_readonly("device", &Sensors::device)
      .def("set_field_stop",
           [](Sensors &s, int nwfs, py::object field_stop, int N) {
             // SutraSensors::set_field_stop (sensors.cpp:200-210): SH sensors only
             auto &w = s.wfs.at(nwfs);
             if (w->sh) {
               py::module_ np = py::module_::import("numpy");
               farray<float> a = np.attr("asarray")(field_stop, np.attr("float32"))
                                     .attr("reshape")(py::make_tuple(N, N))
                                     .cast<farray<float>>();
               check(aob_sh_set_field_stop(w->sh->h, a.data(), N), "set_field_stop");
             }
             return 0;
           })
      .def("initgs", [](Sensors &s, py::object xpos, py::object ypos, py::object lambda_um, py::object mag,
                        py::object zerop, py::object sizes, py::object noise, py::object seeds, py::object G,
                        py::object thetaML, py::object dx, py::object dy) {
        // guide stars (sensors.cpp:159-191): wavelength, noise level and noise seed per sensor
        for (size_t i = 0; i < s.wfs.size(); ++i) {
          auto &w = s.wfs[i];
          const float lam = elem<float>(lambda_um, (int)i);
          w->set_lambda(lam);
          w->set_noise(elem<float>(noise, (int)i), elem<int64_t>(seeds, (int)i));
          auto g = std::make_shared<GuideStar>();
          g->phase = w->phase_view();
          g->lambda_um = lam;
          w->gs = g;
        }
        return 0;
      });
}

}  // namespace aobpy
