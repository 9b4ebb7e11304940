// Compiled drop-in `sutra` module: the classes and methods of the reference's
// pybind11 sutra module (python_module/sutra/src/sutra.cpp:62-103) that
// COMPASS's supervisor calls on the real-time path, with their names,
// constructor arguments and method names, each calling libaob200's C ABI.
// Failures raise RuntimeError with the library's message, as the reference's
// C++ layer does (std::runtime_error).
//
// Covered: Sensors (SHWFS, PYRWFS, guide star), Dms / Dm (piezo stacks), Rtc_FFF
// and Rtc_UFF (uint16 frames) with the cog, tcog, wcog, bpcog, pyr and maskedpix
// centroiders and the ls and generic controllers (do_centroids, do_control,
// apply_control, comp_voltage, do_clipping, gains, do_imat, imat_svd, build_cmat,
// reference slopes, perturbation voltages).

#include "sutra_rtc.hpp"

namespace py = pybind11;
using namespace aobpy;

namespace {

int command_law(const std::string &law) {
  if (law == "integrator") return AOB_LAW_INTEGRATOR;
  if (law == "modal_integrator") return AOB_LAW_MODAL_INTEGRATOR;
  if (law == "2matrices") return AOB_LAW_2MATRICES;
  throw py::value_error("set_commandlaw: unknown command law '" + law + "'");
}

void bind_controllers(py::module_ &m) {
  py::class_<Controller, std::shared_ptr<Controller>>(m, "Controller")
      .def_readonly("type", &Controller::type)
      .def_readonly("nslope", &Controller::nslope)
      .def_readonly("nactu", &Controller::nactu)
      .def_readonly("delay", &Controller::delay)
      .def_readonly("gain", &Controller::gain)
      .def_readonly("comRange", &Controller::comRange)
      .def_readonly("centro_idx", &Controller::centro_idx)
      .def_property_readonly("d_centroids", [](const Controller &c) { return c.buffer("centroids"); })
      .def_property_readonly("d_com", [](const Controller &c) { return c.buffer("com"); })
      .def_property_readonly("d_com_clipped", [](const Controller &c) { return c.buffer("com_clipped"); })
      .def_property_readonly("d_voltage", [](const Controller &c) { return c.buffer("voltage"); })
      .def_property_readonly("d_err", [](const Controller &c) { return c.buffer("err"); })
      .def_property_readonly("d_cmat", [](const Controller &c) { return c.buffer("cmat", {c.nactu, c.nslope}); })
      .def_property_readonly("d_imat", [](const Controller &c) { return c.buffer("imat", {c.nslope, c.nactu}); })
      .def_property_readonly("d_gain", [](const Controller &c) { return c.buffer("gain"); })
      .def_property_readonly("d_circularComs0", [](const Controller &c) { return c.buffer("com0"); })
      .def_property_readonly("d_circularComs1", [](const Controller &c) { return c.buffer("com1"); })
      .def("set_cmat",
           [](Controller &c, py::object a) {
             farray<float> x = checked_matrix(a, c.nactu, c.nslope, "cmat");
             check(aob_ls_set_cmat(c.l->h, x.data()), "set_cmat");
           })
      .def("set_imat",
           [](Controller &c, py::object a) {
             farray<float> x = checked_matrix(a, c.nslope, c.nactu, "imat");
             check(aob_ls_set_imat(c.l->h, x.data()), "set_imat");
           })
      .def("set_gain",
           [](Controller &c, float g) {
             c.gain = g;
             check(aob_ls_set_gain(c.l->h, g), "set_gain");
           })
      .def("set_modal_gains",
           [](Controller &c, const farray<float> &g) {
             if (g.size() < c.nactu) throw std::runtime_error("set_modal_gains: nactu gains are required");
             check(aob_ls_set_modal_gains(c.l->h, g.data()), "set_modal_gains");
           })
      .def("set_delay",
           [](Controller &c, float d) {
             c.delay = d;
             check(aob_ls_set_delay(c.l->h, d), "set_delay");
           })
      .def(
          "set_com",
          [](Controller &c, const farray<float> &com, py::object) {
            check(aob_ls_set_com(c.l->h, com.data(), (int)com.size()), "set_com");
          },
          py::arg("com"), py::arg("nElem") = py::none())
      .def("set_comRange",
           [](Controller &c, float lo, float hi) {
             c.comRange = {lo, hi};
             check(aob_ls_set_com_range(c.l->h, lo, hi), "set_comRange");
           })
      .def(
          "set_open_loop",
          [](Controller &c, bool ol, bool reset) {
            check(aob_ls_set_open_loop(c.l->h, ol ? 1 : 0, reset ? 1 : 0), "set_open_loop");
          },
          py::arg("open_loop"), py::arg("reset") = true)
      .def("comp_voltage",
           [](Controller &c) {
             check(aob_ls_comp_voltage(c.l->h, nullptr), "comp_voltage");
             c.advance_perturb();
           })
      .def("clip_commands", [](Controller &c) { check(aob_ls_clip(c.l->h, nullptr), "clip_commands"); })
      .def("add_perturb",
           [](Controller &c) {
             // com_clipped += the current row of every enabled perturbation (controller.cpp add_perturb)
             check(aob_ls_apply_perturb(c.l->h, nullptr), "add_perturb");
             c.advance_perturb();
           })
      .def("add_perturb_voltage",
           [](Controller &c, const std::string &name, const farray<float> &p, int N) {
             check(aob_ls_add_perturb(c.l->h, name.c_str(), p.data(), N), "add_perturb_voltage");
             c.perturb[name] = std::make_tuple(py::object(py::array(p).attr("copy")()), 0, true);
             c.perturb_n[name] = N;
           })
      .def("remove_perturb_voltage",
           [](Controller &c, const std::string &name) {
             check(aob_ls_remove_perturb(c.l->h, name.c_str()), "remove_perturb_voltage");
             c.perturb.erase(name);
             c.perturb_n.erase(name);
           })
      .def("enable_perturb_voltage",
           [](Controller &c, const std::string &name) {
             check(aob_ls_enable_perturb(c.l->h, name.c_str(), 1), "enable_perturb_voltage");
             std::get<2>(c.perturb.at(name)) = true;
           })
      .def("disable_perturb_voltage",
           [](Controller &c, const std::string &name) {
             check(aob_ls_enable_perturb(c.l->h, name.c_str(), 0), "disable_perturb_voltage");
             std::get<2>(c.perturb.at(name)) = false;
           })
      .def("reset_perturb_voltage",
           [](Controller &c) {
             check(aob_ls_reset_perturb(c.l->h), "reset_perturb_voltage");
             c.perturb.clear();
             c.perturb_n.clear();
           })
      .def_property_readonly("d_perturb_map", [](const Controller &c) {
        // name -> (perturbation voltages [N, nactu], counter, enabled), as the reference's map
        py::dict d;
        for (auto &kv : c.perturb)
          d[py::str(kv.first)] = py::make_tuple(std::get<0>(kv.second), std::get<1>(kv.second), std::get<2>(kv.second));
        return d;
      });

  py::class_<ControllerLS, Controller, std::shared_ptr<ControllerLS>>(m, "ControllerLS")
      .def_property_readonly("d_eigenvals", [](const ControllerLS &c) { return c.buffer("eigenvals"); });

  py::class_<ControllerGENERIC, Controller, std::shared_ptr<ControllerGENERIC>>(m, "ControllerGENERIC")
      .def("set_commandlaw",
           [](ControllerGENERIC &c, const std::string &law) {
             check(aob_ls_set_commandlaw(c.l->h, command_law(law)), "set_commandlaw");
           })
      .def_property_readonly("command_law",
                             [](const ControllerGENERIC &c) {
                               int kind = 0, law = 0, polc = 0;
                               float leaky = 0.f;
                               check(aob_ls_get_kind(c.l->h, &kind, &law, &leaky, &polc), "command_law");
                               return std::string(law == AOB_LAW_MODAL_INTEGRATOR ? "modal_integrator"
                                                  : law == AOB_LAW_2MATRICES       ? "2matrices"
                                                                                   : "integrator");
                             })
      .def("set_leaky_factor",
           [](ControllerGENERIC &c, float f) { check(aob_ls_set_leaky_factor(c.l->h, f), "set_leaky_factor"); })
      .def("set_polc", [](ControllerGENERIC &c, bool on) { check(aob_ls_set_polc(c.l->h, on ? 1 : 0), "set_polc"); })
      .def("set_decayFactor",
           [](ControllerGENERIC &c, const farray<float> &d) {
             if (d.size() < c.nactu) throw std::runtime_error("set_decayFactor: nactu factors are required");
             check(aob_ls_set_decay_factor(c.l->h, d.data()), "set_decayFactor");
           })
      .def("set_matE", [](ControllerGENERIC &c, py::object a) {
        farray<float> x = checked_matrix(a, c.nactu, c.nactu, "matE");
        check(aob_ls_set_matE(c.l->h, x.data()), "set_matE");
      });
}

// The slopes a controller reads: (centroider, device address of its block)
std::vector<std::pair<std::shared_ptr<Centroider>, uintptr_t>> slopes_of(Rtc &r, int n) {
  Controller &c = r.ctl(n);
  const uintptr_t base = c.buffer("centroids").ptr;
  std::vector<std::pair<std::shared_ptr<Centroider>, uintptr_t>> out;
  int64_t off = 0;
  for (int i : c.centro_idx) {
    auto cen = r.centro.at(i);
    out.emplace_back(cen, base + 4 * (uintptr_t)off);
    off += cen->nslopes();
  }
  if (off > c.nslope) throw std::runtime_error("do_centroids: the centroiders' slopes exceed the controller's nslope");
  return out;
}

void bind_rtc_fff(py::module_ &m) {
  py::class_<Rtc, std::shared_ptr<Rtc>>(m, "Rtc_FFF")
      .def(py::init([]() { return std::make_shared<Rtc>(); }))
      .def_property_readonly("d_centro", [](const Rtc &r) { return r.centro; })
      .def_property_readonly("d_control", [](const Rtc &r) { return r.control; })
      .def(
          "add_centroider",
          [](Rtc &r, py::object context, int nvalid, float offset, float scale, bool filter_TT, int device,
             const std::string &typec, std::shared_ptr<Wfs> wfs) {
            auto c = std::make_shared<Centroider>();
            c->type = typec;
            c->device = device;
            // a masked-pixel centroider has one slope per valid pixel (maskedPix.cpp:35-36)
            c->nvalid = (typec == "maskedpix" && wfs) ? 4 * wfs->nvalid : nvalid;
            c->offset = offset;
            c->scale = scale;
            c->tin_u16 = r.u16;
            c->c = std::make_shared<CentroOwner>();
            check(aob_centro_create(&c->c->h, device, centro_type(typec), c->nvalid, offset, scale), "add_centroider");
            if (wfs) {
              if (wfs->pyr)
                check(aob_centro_attach_pyr(c->c->h, wfs->pyr->h), "add_centroider");
              else
                check(aob_centro_attach_wfs(c->c->h, wfs->sh->h), "add_centroider");
              c->wfs = wfs;
            }
            r.centro.push_back(c);
            return 0;
          },
          py::arg("context"), py::arg("nvalid"), py::arg("offset"), py::arg("scale"), py::arg("filter_TT"),
          py::arg("device"), py::arg("typec"), py::arg("wfs") = py::none())
      .def(
          "add_controller",
          [](Rtc &r, py::object context, const std::string &typec, int device, float delay, int nslope, int nactu,
             int, int, int, int, int, int, bool, bool, py::object dms, py::object idx_dms, int ndm,
             py::object idx_centro, int ncentro, int, bool) {
            std::shared_ptr<Controller> c;
            if (typec == "ls")
              c = std::make_shared<ControllerLS>();
            else if (typec == "generic")
              c = std::make_shared<ControllerGENERIC>();
            else
              throw py::value_error("add_controller: controller type '" + typec + "' is not supported (ls, generic)");
            c->type = typec;
            c->nslope = nslope, c->nactu = nactu, c->delay = delay;
            c->l = std::make_shared<LsOwner>();
            if (typec == "ls")
              check(aob_ls_create(&c->l->h, device, nslope, nactu, delay), "add_controller");
            else
              check(aob_generic_create(&c->l->h, device, nslope, nactu, delay), "add_controller");
            if (!idx_dms.is_none() && ndm > 0) {
              for (int i = 0; i < ndm; ++i) c->dm_idx.push_back(elem<int>(idx_dms, i));
              c->dm_idx_set = true;
            }
            if (!idx_centro.is_none() && ncentro > 0) {
              for (int i = 0; i < ncentro; ++i) c->centro_idx.push_back(elem<int>(idx_centro, i));
            } else {
              for (size_t i = 0; i < r.centro.size(); ++i) c->centro_idx.push_back((int)i);
            }
            r.control.push_back(c);
            return 0;
          },
          py::arg("context"), py::arg("typec"), py::arg("device"), py::arg("delay"), py::arg("nslope"),
          py::arg("nactu"), py::arg("nslope_buffers") = 0, py::arg("nstates") = 0, py::arg("nstate_buffers") = 0,
          py::arg("nmodes") = 0, py::arg("niir_in") = 0, py::arg("niir_out") = 0, py::arg("polc") = false,
          py::arg("is_modal") = false, py::arg("dms") = py::none(), py::arg("idx_dms") = py::none(),
          py::arg("ndm") = 0, py::arg("idx_centro") = py::none(), py::arg("ncentro") = 0, py::arg("Nphi") = 0,
          py::arg("wfs_direction") = false)
      .def(
          "do_imat",
          [](Rtc &r, int ncontrol, std::shared_ptr<Dms> dms, bool kernconv) {
            // push-pull interaction matrix (sutra_rtc.cpp:150-292): every actuator of every
            // DM the controller drives, pushed and pulled by its push4imat, seen by the
            // controller's SH sensors (noise-free, nphot4imat photons); the slopes
            // (s_push - s_pull) / (2 push) are the columns of d_imat.  All actuators of a
            // DM go through one batched evaluation (aob_imat_build) per sensor.
            if (kernconv) throw std::runtime_error("do_imat: the spot convolution kernel is not supported");
            Controller &c = r.ctl(ncontrol);
            if (c.type != "ls") throw std::runtime_error("do_imat: the controller must be ls");
            std::vector<std::pair<int, std::shared_ptr<Dm>>> seen;
            if (c.dm_idx_set)
              for (int i : c.dm_idx) seen.emplace_back(i, dms->dms.at(i));
            else
              for (size_t i = 0; i < dms->dms.size(); ++i) seen.emplace_back((int)i, dms->dms[i]);
            int total = 0;
            for (auto &p : seen) total += p.second->nactus;
            if (total != c.nactu)
              throw std::runtime_error("do_imat: the DMs' actuators do not add up to the controller's nactu");
            std::vector<float> imat((size_t)c.nslope * c.nactu, 0.f);  // Fortran order, nslope x nactu
            int a0 = 0;
            for (auto &p : seen) {
              Dm &dm = *p.second;
              aob_dm *dh = dm.need();
              int off = 0;
              for (int i : c.centro_idx) {
                Centroider &cen = *r.centro.at(i);
                const int ns = cen.nslopes();
                if (!cen.wfs || !cen.wfs->sh)
                  throw std::runtime_error("do_imat: only Shack-Hartmann sensors are supported");
                if (off + ns > c.nslope) throw std::runtime_error("do_imat: the slopes exceed the controller's nslope");
                Wfs &w = *cen.wfs;
                // the DM's place on the sensor's phase grid (wfs.d_gs.add_layer), else centred
                float xoff = (float)((dm.dim - w.npup) / 2.0), yoff = xoff;
                if (w.gs) {
                  auto it = w.gs->dm_layers.find(p.first);
                  if (it != w.gs->dm_layers.end()) xoff = it->second.first, yoff = it->second.second;
                }
                check(aob_centro_attach_wfs(cen.c->h, w.sh->h), "do_imat");
                DevAlloc tmp(sizeof(float) * (size_t)ns * dm.nactus, dm.device);
                check(aob_imat_build(w.sh->h, cen.c->h, dh, xoff, yoff, dm.push4imat, 0, static_cast<float *>(tmp.p),
                                     nullptr),
                      "do_imat");
                std::vector<float> h((size_t)ns * dm.nactus);
                check(aob_memcpy_d2h(h.data(), tmp.p, sizeof(float) * h.size(), nullptr), "do_imat");
                for (int a = 0; a < dm.nactus; ++a)
                  for (int k = 0; k < ns; ++k)
                    imat[(size_t)(off + k) + (size_t)(a0 + a) * c.nslope] = h[(size_t)k + (size_t)a * ns];
                off += ns;
              }
              a0 += dm.nactus;
            }
            check(aob_ls_set_imat(c.l->h, imat.data()), "do_imat");
            return 0;
          },
          py::arg("ncontrol"), py::arg("dms"), py::arg("kernconv") = false)
      .def("remove_controller", [](Rtc &r, int n) { r.control.erase(r.control.begin() + n); })
      .def("remove_centroider", [](Rtc &r, int n) { r.centro.erase(r.centro.begin() + n); })
      .def("do_centroids",
           [](Rtc &r, int n) {
             for (auto &cp : slopes_of(r, n)) cp.first->get_cog_into(cp.second);
             return 0;
           })
      .def("do_calibrate_img",
           [](Rtc &r, int n) {
             for (auto &cp : slopes_of(r, n))
               if (!cp.first->wfs) check(aob_centro_calibrate_img(cp.first->c->h, nullptr), "do_calibrate_img");
             return 0;
           })
      .def("do_control",
           [](Rtc &r, int n) {
             check(aob_ls_comp_com(r.ctl(n).l->h, nullptr), "do_control");
             return 0;
           })
      .def("comp_voltage",
           [](Rtc &r, int n) {
             check(aob_ls_comp_voltage(r.ctl(n).l->h, nullptr), "comp_voltage");
             return 0;
           })
      .def(
          "apply_control",
          [](Rtc &r, int n, bool comp) {
            // the voltages of controller n (the DM shapes they drive are the caller's)
            if (comp) check(aob_ls_comp_voltage(r.ctl(n).l->h, nullptr), "apply_control");
            return 0;
          },
          py::arg("ncontrol"), py::arg("compVoltage") = true)
      .def("do_clipping",
           [](Rtc &r, int n) {
             check(aob_ls_clip(r.ctl(n).l->h, nullptr), "do_clipping");
             return 0;
           })
      .def("set_gain",
           [](Rtc &r, int n, float g) {
             r.ctl(n).gain = g;
             check(aob_ls_set_gain(r.ctl(n).l->h, g), "set_gain");
             return 0;
           })
      .def("set_modal_gains",
           [](Rtc &r, int n, const farray<float> &g) {
             if (g.size() < r.ctl(n).nactu) throw std::runtime_error("set_modal_gains: nactu gains are required");
             check(aob_ls_set_modal_gains(r.ctl(n).l->h, g.data()), "set_modal_gains");
             return 0;
           })
      .def("imat_svd",
           [](Rtc &r, int n) {
             check(aob_ls_svdec_imat(r.ctl(n).l->h), "imat_svd");
             return 0;
           })
      .def(
          "build_cmat",
          [](Rtc &r, int n, int nfilt, bool filt_tt) {
            if (filt_tt) throw std::runtime_error("build_cmat: tip-tilt filtering is not supported");
            check(aob_ls_build_cmat(r.ctl(n).l->h, nfilt), "build_cmat");
            return 0;
          },
          py::arg("ncontrol"), py::arg("nfilt"), py::arg("filt_tt") = false)
      .def("set_centroids_ref", [](Rtc &r, const farray<float> &ref) {
        // one block per centroider, in order
        int64_t off = 0;
        for (auto &cen : r.centro) {
          if (off + cen->nslopes() > ref.size()) throw std::runtime_error("set_centroids_ref: too few slopes");
          check(aob_centro_set_centroids_ref(cen->c->h, ref.data() + off), "set_centroids_ref");
          off += cen->nslopes();
        }
        return 0;
      });
}

// SutraRtc<uint16_t, float, float>: the centroiders load uint16 frames (from the host
// or a sensor's d_camimg) and calibrate them with dark, flat and a pixel look-up table
struct RtcU : Rtc {
  RtcU() { u16 = true; }
};

}  // namespace

PYBIND11_MODULE(sutra, m) {
  m.doc() = "libaob200 drop-in for the reference's sutra module (real-time path)";
  bind_device_array(m, "obj");
  bind_wfs(m);
  bind_sensors(m);
  bind_rtc(m);
  bind_controllers(m);
  bind_dms(m);
  bind_rtc_fff(m);
  py::class_<RtcU, Rtc, std::shared_ptr<RtcU>>(m, "Rtc_UFF").def(py::init([]() { return std::make_shared<RtcU>(); }));
}
