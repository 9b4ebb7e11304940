"""The drop-in `carma` / `sutra` modules import without a GPU, carry the class and
method names shesha calls on the hot path (the reference's pybind11 bindings:
python_module/sutra/src/sutra.cpp:62-103, rtc.cpp:100-485, wfs_sh.cpp:41-148,
wfs_pyrhr.cpp:131-163, centroider.cpp:83-352, controller.cpp), and reject
unsupported sensor / centroider / controller types (correlation centroider,
minimum-variance controller, low-resolution pyramid) before any device work.

Both implementations are checked: the Python drop-in (dropin/) and the compiled
pybind11 pair (dropin_native/)."""

import pytest

from helpers import import_dropin

API = {
    "Sensors": ["initgs", "d_wfs", "set_field_stop"],
    "SHWFS": ["load_arrays", "comp_image", "set_noise", "set_pupil", "fill_binimage", "d_binimg", "d_bincube",
              "d_intensities", "d_validsubsx", "d_validsubsy", "d_fluxPerSub", "slopes_geom", "set_binimg",
              "set_dark", "set_flat", "comp_nphot", "set_bincube", "d_binmap", "d_slopes", "d_camimg",
              "d_validpuppixx", "d_validpuppixy"],
    "PYRWFS": ["load_arrays", "comp_image", "set_noise", "set_pupil", "set_pyr_modulation_points", "d_binimg",
               "slopes_geom", "set_binimg", "set_phalfxy", "set_submask", "compute_pyrfocalplane",
               "d_pyrfocalplane", "set_pyrimg", "comp_nphot", "d_submask", "d_phalfxy", "d_hrimg", "d_slopes"],
    "Dms": ["add_dm", "remove_dm", "d_dms"],
    "Dm": ["pzt_loadarrays", "set_com", "comp_shape", "comp_oneactu", "reset_shape", "d_shape", "d_com"],
    "Centroider": ["get_cog", "load_validpos", "set_npix", "set_scale", "set_offset", "set_threshold", "load_weights",
                   "set_centroids_ref", "load_img", "calibrate_img", "set_dark", "set_flat", "set_pyr_method",
                   "set_pyr_thresh", "d_centroids_ref", "d_intensities", "d_img", "d_img_raw", "d_validx", "d_validy",
                   "d_weights", "set_nmax", "init_weights", "d_dark", "d_flat", "nslopes", "set_lutPix",
                   "calibrate_img_validPix"],
    "ControllerLS": ["set_cmat", "set_imat", "set_gain", "set_modal_gains", "set_delay", "set_com", "set_comRange",
                     "set_open_loop", "comp_voltage", "clip_commands", "add_perturb_voltage",
                     "remove_perturb_voltage", "enable_perturb_voltage", "disable_perturb_voltage",
                     "reset_perturb_voltage", "d_centroids", "d_com", "d_com_clipped", "d_voltage", "d_err", "d_cmat",
                     "d_imat", "d_eigenvals", "d_gain", "add_perturb", "d_perturb_map", "d_circularComs0",
                     "d_circularComs1"],
    "ControllerGENERIC": ["set_cmat", "set_gain", "set_modal_gains", "set_commandlaw", "set_leaky_factor", "set_polc",
                          "set_decayFactor", "set_matE", "set_imat", "comp_voltage", "add_perturb", "d_com",
                          "d_com_clipped", "d_voltage", "d_cmat", "d_centroids"],
    "Rtc_UFF": ["add_centroider", "add_controller", "do_centroids", "do_control", "do_calibrate_img"],
    "Rtc_FFF": ["add_centroider", "add_controller", "remove_controller", "remove_centroider", "do_calibrate_img",
                "do_centroids", "do_control", "comp_voltage", "apply_control", "do_clipping", "set_gain",
                "set_modal_gains", "imat_svd", "build_cmat", "set_centroids_ref", "do_imat"],
}


@pytest.fixture(scope="module", params=["python", "native"])
def mods(request):
    return (request.param,) + import_dropin(request.param)


def test_names(mods):
    kind, carma, sutra = mods
    for cls, names in API.items():
        c = getattr(sutra, cls)
        missing = [n for n in names if not hasattr(c, n)]
        assert not missing, f"{cls} lacks {missing}"
    for n in ("get_instance", "get_instance_1gpu", "get_instance_ngpu", "activate_device"):
        assert hasattr(carma.context, n)


def test_rejects_before_device_work(mods):
    kind, carma, sutra = mods
    ctx = carma.context.get_instance()
    assert ctx.ndevice >= 1
    rtc = sutra.Rtc_FFF()
    with pytest.raises(ValueError):
        rtc.add_centroider(ctx, 10, 0.0, 1.0, False, 0, "corr")
    with pytest.raises(ValueError):
        rtc.add_controller(ctx, "mv", 0, 0.0, 20, 10)
    with pytest.raises(ValueError):
        sutra.Sensors(ctx, None, ["pyrlr"], 1, [8], [52], 1, [6], [8], [3], [16], [24], [64], [8.0], [100.0],
                      [0.0], [False], False, 0, 0, 0, False)
    assert rtc.d_centro == [] and rtc.d_control == []
