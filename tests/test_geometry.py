"""The project's geometry builder against fixtures produced by the reference's own
init code (geom_init.py, make_pupil.py).  Integer maps must match bit for bit."""

import numpy as np
import pytest

from aob200 import geometry as G

SH = {
    "sh16": G.ShParams(nxsub=16, npix=8, pixsize=0.3, wavelength_um=0.7, fracsub=0.5, gsmag=8.0),
    "sh40": G.ShParams(nxsub=40, npix=6, pixsize=0.36, wavelength_um=0.7, fracsub=0.5, gsmag=8.0),
    "sh8": G.ShParams(nxsub=8, npix=2, pixsize=0.3, wavelength_um=0.7, fracsub=0.5, gsmag=8.0),
    # shesha/tests/pytest/par/test_sh.py's sensor: extended field of view (ntot > nfft)
    "sh16x": G.ShParams(nxsub=16, npix=8, pixsize=0.3, wavelength_um=0.5, fracsub=0.8, gsmag=3.0),
    # field stops in the focal plane of the full pupil
    "sh16fs": G.ShParams(nxsub=16, npix=8, pixsize=0.3, wavelength_um=0.7, fracsub=0.5, gsmag=8.0, fssize=1.6,
                         fstop="round"),
    "sh16fsq": G.ShParams(nxsub=16, npix=8, pixsize=0.3, wavelength_um=0.7, fracsub=0.5, gsmag=8.0, fssize=1.2,
                          fstop="square"),
}
SH_PUP = {"sh16": 128, "sh40": 240, "sh8": 48, "sh16x": 128, "sh16fs": 128, "sh16fsq": 128}
SH_TEL = {"sh16x": dict(cobs=0.12, ittime=0.002)}


@pytest.mark.parametrize("name", sorted(SH))
def test_sh_geometry_matches_reference(name, golden):
    ref = golden("geom_" + name)
    tel = SH_TEL.get(name, dict(cobs=0.14, ittime=0.001))
    g = G.sh_geometry(SH[name], SH_PUP[name], diam=8.0, **tel)
    for k in ("pdiam", "nfft", "ntot", "nrebin", "nvalid"):
        assert getattr(g, k) == int(ref[k]), k
    assert g.tel.n == int(ref["n"])
    for k in ("spupil", "mpupil", "ipupil"):
        np.testing.assert_array_equal(getattr(g.tel, k), ref[k])
    for k in ("isvalid", "validsubsx", "validsubsy", "validpuppixx", "validpuppixy",
              "phasemap", "binmap", "hrmap"):
        a = getattr(g, k)
        assert a.dtype == ref[k].dtype, k
        np.testing.assert_array_equal(a, ref[k], err_msg=k)
    for k in ("fluxPerSub", "fluxPerSub_grid", "halfxy"):
        np.testing.assert_array_equal(getattr(g, k), ref[k], err_msg=k)
    if "submask" in ref:
        np.testing.assert_array_equal(g.submask, ref["submask"])
    else:
        assert g.submask is None
    # tip/tilt projection (not on the image-formation path): float rounding only
    np.testing.assert_allclose(g.ttprojmat, ref["ttprojmat"], rtol=1e-6, atol=1e-7)
    # the reference keeps these two through float32 parameter setters
    assert np.float32(g.pixsize) == np.float32(ref["pixsize"])
    assert np.float32(g.qpixsize) == np.float32(ref["qpixsize"])
    assert g.nphotons == pytest.approx(float(ref["nphotons"]), rel=1e-6)


PYR = {
    "pyr16": (G.PyrParams(nxsub=16, wavelength_um=0.7, ampl=3.0, npts=8, pup_sep=12, fssize=3.2), 64),
    "pyr50": (G.PyrParams(nxsub=50, wavelength_um=1.075, ampl=3.0, npts=24, pup_sep=32, fssize=3.2), 100),
}


@pytest.mark.parametrize("name", sorted(PYR))
def test_pyr_geometry_matches_reference(name, golden):
    ref = golden("geom_" + name)
    p, pup = PYR[name]
    g = G.pyr_geometry(p, pup, diam=8.0, cobs=0.14, ittime=0.001)
    for k in ("pdiam", "nfft", "ntot", "nrebin", "nvalid"):
        assert getattr(g, k) == int(ref[k]), k
    np.testing.assert_array_equal(g.tel.mpupil, ref["mpupil"])
    for k in ("validsubsx", "validsubsy", "isvalid", "phasemap"):
        np.testing.assert_array_equal(getattr(g, k), ref[k], err_msg=k)
    for k in ("halfxy", "pyr_cx", "pyr_cy", "sincar", "submask", "fluxPerSub"):
        np.testing.assert_array_equal(getattr(g, k), ref[k], err_msg=k)


@pytest.mark.parametrize("name,nact,pup,margin", [("dm17", 17, 128, None), ("dm41", 41, 240, 1.0)])
def test_dm_geometry_matches_reference(name, nact, pup, margin, golden):
    from aob200 import dm_geometry as D

    ref = golden(name)
    tel = G.telescope_geometry(pup, 8.0, 0.14)
    g = D.pzt_dm_geometry(nact, tel.pupdiam, tel.cent, tel.ssize, tel.n, 0.14, coupling=0.3, margin_out=margin)
    assert g.ntotact == int(ref["ntotact"])
    assert (g.n1, g.n2, g.dim, g.influsize) == (int(ref["n1"]), int(ref["n2"]), int(ref["dim"]), int(ref["influsize"]))
    np.testing.assert_array_equal(g.i1, ref["i1"])
    np.testing.assert_array_equal(g.j1, ref["j1"])
    np.testing.assert_array_equal(g.xpos, ref["xpos"])
    np.testing.assert_allclose(g.influ, ref["influ"], rtol=1e-6, atol=1e-7)
