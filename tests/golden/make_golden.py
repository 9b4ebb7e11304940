"""Generate golden fixtures by running the reference's own Python init code.

This script is run by hand in a container where the reference checkout is
present (default path below, override with ``AO_REFERENCE``).  It imports the
reference's ``shesha`` package with small stub modules standing in for its
compiled ``carma``/``sutra`` extensions and for optional third-party packages
(``aenum``, ``h5py``, ``astropy``) that the init functions used here never
call.  The outputs are written as ``.npz`` fixtures next to this file; the
tests compare the project's own geometry / turbulence / DM builders against
them.  Nothing at test time reads the reference checkout.

Reference functions exercised (paths within the reference project):
  shesha/shesha/init/geom_init.py  init_wfs_geom / init_wfs_size / init_sh_geom /
                                   init_pyrhr_geom / geom_init
  shesha/shesha/util/make_pupil.py make_pupil (generic aperture)
  shesha/shesha/util/iterkolmo.py  create_stencil / stencil_size / AB
  shesha/shesha/util/influ_util.py makeGaussian
  shesha/shesha/init/dm_init.py    make_pzt_dm
"""

import contextlib
import enum
import io
import os
import sys
import types

import numpy as np

REF = os.environ.get("AO_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))


def _stub(name, **attrs):
    m = types.ModuleType(name)
    m.__dict__.update(attrs)
    sys.modules[name] = m
    return m


def _install_stubs():
    _stub("carma", __version__="6.0.0")
    _stub("sutra", __version__="6.0.0")

    class MultiValueEnum(enum.Enum):
        pass

    _stub("aenum", MultiValueEnum=MultiValueEnum)
    _stub("h5py")
    a = _stub("astropy")
    io_ = _stub("astropy.io")
    fits = _stub("astropy.io.fits")
    a.io = io_
    io_.fits = fits
    sys.path.insert(0, os.path.join(REF, "shesha"))


# Workloads.  The SH ones are the plain 16x16 loop, the SAXO-scale 40x40 loop
# and a small 8x8 case whose FFT support is 16 (the others use 32).
SH_CASES = {
    "sh16": dict(nxsub=16, pupdiam=128, npix=8, pixsize=0.3, lam=0.7, fracsub=0.5,
                 cobs=0.14, gsmag=8.0, r0=0.16, ittime=0.001),
    "sh40": dict(nxsub=40, pupdiam=240, npix=6, pixsize=0.36, lam=0.7, fracsub=0.5,
                 cobs=0.14, gsmag=8.0, r0=0.14, ittime=0.001),
    "sh8": dict(nxsub=8, pupdiam=48, npix=2, pixsize=0.3, lam=0.7, fracsub=0.5,
                cobs=0.14, gsmag=8.0, r0=0.16, ittime=0.001),
}

PYR_CASES = {
    # pyramid with 50 pupil samples across; modulation radius 3 lambda/D, 24 points
    "pyr50": dict(nxsub=50, pupdiam=100, lam=1.075, fracsub=0.0001, cobs=0.14,
                  ampl=3.0, npts=24, pup_sep=32, fssize=3.2, gsmag=6.0, r0=0.14,
                  ittime=0.001),
    "pyr16": dict(nxsub=16, pupdiam=64, lam=0.7, fracsub=0.0001, cobs=0.14,
                  ampl=3.0, npts=8, pup_sep=12, fssize=3.2, gsmag=6.0, r0=0.16,
                  ittime=0.001),
}


def make_sh(conf, gi, c):
    p_geom = conf.ParamGeom()
    p_geom.set_pupdiam(c["pupdiam"])
    p_geom.set_zenithangle(0.0)
    p_tel = conf.ParamTel()
    p_tel.set_diam(8.0)
    p_tel.set_cobs(c["cobs"])
    w = conf.ParamWfs()
    w.set_type("sh")
    w.set_nxsub(c["nxsub"])
    w.set_npix(c["npix"])
    w.set_pixsize(c["pixsize"])
    w.set_fracsub(c["fracsub"])
    w.set_xpos(0.0)
    w.set_ypos(0.0)
    w.set_Lambda(c["lam"])
    w.set_gsmag(c["gsmag"])
    w.set_optthroughput(0.5)
    w.set_zerop(1e11)
    w.set_noise(0.5)
    with contextlib.redirect_stdout(io.StringIO()):
        gi.init_wfs_geom(w, c["r0"], p_tel, p_geom, c["ittime"], verbose=0)
    fluxPerSub = w._fluxPerSub.T[np.where(w._isvalid.T > 0)].copy()
    return dict(
        pdiam=w._pdiam, nfft=w._Nfft, ntot=w._Ntot, nrebin=w._nrebin,
        nvalid=w._nvalid, pixsize=np.float64(w.pixsize), qpixsize=np.float64(w._qpixsize),
        nphotons=np.float64(w._nphotons), subapd=np.float64(w._subapd),
        n=p_geom._n, pupdiam_eff=p_geom.pupdiam, ssize=p_geom.ssize,
        p1=p_geom._p1, p2=p_geom._p2, n1=p_geom._n1, n2=p_geom._n2,
        spupil=p_geom._spupil, mpupil=p_geom._mpupil, ipupil=p_geom._ipupil,
        isvalid=w._isvalid, fluxPerSub_grid=w._fluxPerSub, fluxPerSub=fluxPerSub,
        validsubsx=w._validsubsx, validsubsy=w._validsubsy,
        validpuppixx=w._validpuppixx, validpuppixy=w._validpuppixy,
        phasemap=w._phasemap, binmap=w._binmap, halfxy=w._halfxy,
        hrmap=w._hrmap, ttprojmat=w._ttprojmat,
    )


def make_pyr(conf, gi, c):
    p_geom = conf.ParamGeom()
    if c["pupdiam"]:
        p_geom.set_pupdiam(c["pupdiam"])
    p_geom.set_zenithangle(0.0)
    p_tel = conf.ParamTel()
    p_tel.set_diam(8.0)
    p_tel.set_cobs(c["cobs"])
    w = conf.ParamWfs()
    w.set_type("pyrhr")
    w.set_nxsub(c["nxsub"])
    w.set_fracsub(c["fracsub"])
    w.set_xpos(0.0)
    w.set_ypos(0.0)
    w.set_Lambda(c["lam"])
    w.set_gsmag(c["gsmag"])
    w.set_optthroughput(0.5)
    w.set_zerop(1e11)
    w.set_noise(-1.0)
    w.set_pyr_ampl(c["ampl"])
    w.set_pyr_npts(c["npts"])
    w.set_pyr_pup_sep(c["pup_sep"])
    if c["fssize"]:
        w.set_fstop("round")
        w.set_fssize(c["fssize"])
    with contextlib.redirect_stdout(io.StringIO()):
        gi.init_wfs_geom(w, c["r0"], p_tel, p_geom, c["ittime"], verbose=0)
    fluxPerSub = w._fluxPerSub.T[np.where(w._isvalid.T > 0)].copy()
    return dict(
        pdiam=w._pdiam, nfft=w._Nfft, ntot=w._Ntot, nrebin=w._nrebin,
        nvalid=w._nvalid, qpixsize=np.float64(w._qpixsize), pixsize=np.float64(w.pixsize),
        nphotons=np.float64(w._nphotons), n=p_geom._n, pupdiam_eff=p_geom.pupdiam,
        spupil=p_geom._spupil, mpupil=p_geom._mpupil,
        halfxy=w._halfxy, pyr_cx=w._pyr_cx, pyr_cy=w._pyr_cy,
        sincar=w._sincar, submask=w._submask,
        validsubsx=w._validsubsx, validsubsy=w._validsubsy,
        isvalid=w._isvalid, fluxPerSub=fluxPerSub, phasemap=w._phasemap,
        pyr_pos=w.pyr_pos if w.pyr_pos is not None else np.zeros(0),
    )


def make_kolmo(itk, n, L0, seed):
    zref = 0
    with contextlib.redirect_stdout(io.StringIO()):
        A, B, istx, isty = itk.AB(n, L0)
    return dict(A=A, B=B, istencilx=istx, istencily=isty)


def make_dm(conf, gi, dmi, sh, nact, thresh, coupling, cobs=0.14, pupdiam=240):
    p_geom = conf.ParamGeom()
    p_geom.set_pupdiam(pupdiam)
    p_geom.set_zenithangle(0.0)
    p_tel = conf.ParamTel()
    p_tel.set_diam(8.0)
    p_tel.set_cobs(cobs)
    with contextlib.redirect_stdout(io.StringIO()):
        gi.geom_init(p_geom, p_tel)
    p_dm = conf.ParamDm()
    p_dm.set_type("pzt")
    p_dm.set_nact(nact)
    p_dm.set_alt(0.0)
    p_dm.set_thresh(thresh)
    p_dm.set_coupling(coupling)
    p_dm.set_unitpervolt(1.0)
    p_dm.set_push4imat(1.0)
    p_dm.set_influ_type("gaussian")
    with contextlib.redirect_stdout(io.StringIO()):
        dmi.dim_dm_init(p_tel, p_dm, p_geom, "pzt") if hasattr(dmi, "dim_dm_init") else None
        if p_dm._n1 is None or p_dm._n1 == 0:
            # same padding the reference applies in dm_init for an altitude-0 pzt DM
            extent = p_geom.pupdiam + 2 * np.ceil(1.0 * p_geom.pupdiam / (nact - 1))
            dim = int(max(p_geom._n, extent))
            p_dm._n1 = int(np.floor(p_geom.cent - dim / 2.0))
            p_dm._n2 = p_dm._n1 + dim - 1
        dmi.make_pzt_dm(p_dm, p_geom, cobs)
    return dict(
        xpos=p_dm._xpos, ypos=p_dm._ypos, i1=p_dm._i1, j1=p_dm._j1,
        influ=p_dm._influ, ntotact=p_dm._ntotact, influsize=p_dm._influsize,
        pitch=p_dm._pitch, n1=p_dm._n1, n2=p_dm._n2, ninflu=p_dm._ninflu,
        influstart=p_dm._influstart, influpos=p_dm._influpos,
        dim_screen=p_dm._n2 - p_dm._n1 + 1,
    )


def main():
    _install_stubs()
    import warnings

    warnings.simplefilter("ignore")
    import shesha.config as conf
    import shesha.init.geom_init as gi

    for name, c in SH_CASES.items():
        out = make_sh(conf, gi, c)
        np.savez_compressed(os.path.join(HERE, f"geom_{name}.npz"), **out)
        print(name, "nvalid", out["nvalid"], "nfft", out["nfft"], "nrebin", out["nrebin"])
    for name, c in PYR_CASES.items():
        out = make_pyr(conf, gi, c)
        np.savez_compressed(os.path.join(HERE, f"geom_{name}.npz"), **out)
        print(name, "nvalid", out["nvalid"], "nfft", out["nfft"], "nrebin", out["nrebin"])


if __name__ == "__main__":
    main()
