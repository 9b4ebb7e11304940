"""Generate golden fixtures by running the reference's own Python init code.

This script is run by hand in a container where the reference checkout is
present; ``AO_REFERENCE`` names its directory (the one holding ``shesha/``).  It imports the
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

REF = os.environ.get("AO_REFERENCE")
if not REF:
    raise SystemExit("make_golden.py: set AO_REFERENCE to the reference checkout (the directory holding shesha/)")
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
    # the reference's own test sensor (shesha/tests/pytest/par/test_sh.py): at
    # 0.5 um its 8 pixels of 0.3" extend the field of view beyond the FFT support
    "sh16x": dict(nxsub=16, pupdiam=128, npix=8, pixsize=0.3, lam=0.5, fracsub=0.8,
                  cobs=0.12, gsmag=3.0, r0=0.16, ittime=0.002),
    # with a round field stop of 1.6 arcsec and a square one of 1.2 arcsec
    "sh16fs": dict(nxsub=16, pupdiam=128, npix=8, pixsize=0.3, lam=0.7, fracsub=0.5,
                   cobs=0.14, gsmag=8.0, r0=0.16, ittime=0.001, fssize=1.6, fstop="round"),
    "sh16fsq": dict(nxsub=16, pupdiam=128, npix=8, pixsize=0.3, lam=0.7, fracsub=0.5,
                    cobs=0.14, gsmag=8.0, r0=0.16, ittime=0.001, fssize=1.2, fstop="square"),
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
    if c.get("fssize"):
        import shesha.constants as scons

        w.set_fssize(c["fssize"])
        w.set_fstop(scons.FieldStopType.ROUND if c["fstop"] == "round" else scons.FieldStopType.SQUARE)
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
        **({"submask": w._submask} if c.get("fssize") else {}),
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


def make_kolmo(itk, n, L0, deltax, deltay):
    with contextlib.redirect_stdout(io.StringIO()):
        A, B, istx, isty = itk.AB(n, L0, deltax, deltay, 0)
    r2 = np.concatenate([np.linspace(0.0, 4.0, 41), np.linspace(4.0, 3.0 * n * n, 200)])
    return dict(A=A, B=B, istencilx=istx, istencily=isty, stencil_size=itk.stencil_size(n),
                struct_r2=r2, struct_L0=np.float64(L0), struct_val=itk.phase_struct(r2, L0))


class _FakeDms:
    """Records what the reference's dm_init hands to the GPU object."""

    def __init__(self):
        self.added = []
        self.d_dms = []

    def add_dm(self, *args):
        self.added.append(args)
        rec = types.SimpleNamespace()

        def pzt_loadarrays(influ, influpos, ninflu, influstart, i1, j1):
            rec.arrays = dict(influ=influ, influpos=influpos, ninflu=ninflu, influstart=influstart,
                              i1=i1, j1=j1)

        rec.pzt_loadarrays = pzt_loadarrays
        self.d_dms.append(rec)


def make_dm(conf, gi, dmi, c):
    p_geom = conf.ParamGeom()
    p_geom.set_pupdiam(c["pupdiam"])
    p_geom.set_zenithangle(0.0)
    p_tel = conf.ParamTel()
    p_tel.set_diam(8.0)
    p_tel.set_cobs(c["cobs"])
    with contextlib.redirect_stdout(io.StringIO()):
        gi.geom_init(p_geom, p_tel)
    p_dm = conf.ParamDm()
    p_dm.set_type("pzt")
    p_dm.set_nact(c["nact"])
    p_dm.set_alt(0.0)
    p_dm.set_coupling(c["coupling"])
    p_dm.set_unitpervolt(1.0)
    p_dm.set_push4imat(1.0)
    p_dm.set_influ_type("gaussian")
    if c.get("margin_out") is not None:
        p_dm.set_margin_out(c["margin_out"])
    fake = _FakeDms()
    with contextlib.redirect_stdout(io.StringIO()):
        dmi._dm_init(types.SimpleNamespace(active_device=0), fake, p_dm, [0.0], [0.0], p_geom, 8.0, c["cobs"],
                     0.0, 0)
    a = fake.d_dms[-1].arrays
    args = fake.added[-1]
    return dict(
        xpos=p_dm._xpos, ypos=p_dm._ypos, i1=a["i1"], j1=a["j1"], influ=a["influ"],
        ntotact=p_dm._ntotact, influsize=p_dm._influsize, pitch=np.float64(p_dm._pitch),
        n1=p_dm._n1, n2=p_dm._n2, dim=args[3], n_mpupil=p_geom._n, cent=np.float64(p_geom.cent),
        # the reference's per-pixel lists of influence samples (comp_dmgeom), for
        # driving its own SutraDm in the reference-run fixtures
        influpos=np.asarray(a["influpos"], np.int32), ninflu=np.asarray(a["ninflu"], np.int32),
        influstart=np.asarray(a["influstart"], np.int32),
    )


DM_CASES = {
    "dm17": dict(pupdiam=128, nact=17, coupling=0.3, cobs=0.14),
    "dm41": dict(pupdiam=240, nact=41, coupling=0.3, cobs=0.14, margin_out=1.0),
}

KOLMO_CASES = {"kolmo32": dict(n=32, L0=25.0 * 32 / 8.0, deltax=0.5, deltay=0.3),
               "kolmo64neg": dict(n=64, L0=25.0 * 64 / 8.0, deltax=-0.7, deltay=-0.2)}


def main():
    _install_stubs()
    import warnings

    warnings.simplefilter("ignore")
    import shesha.config as conf
    import shesha.init.geom_init as gi

    only = os.environ.get("AO_GOLDEN_ONLY")
    for name, c in SH_CASES.items():
        if only and only != name:
            continue
        out = make_sh(conf, gi, c)
        np.savez_compressed(os.path.join(HERE, f"geom_{name}.npz"), **out)
        print(name, "nvalid", out["nvalid"], "nfft", out["nfft"], "nrebin", out["nrebin"])
    for name, c in PYR_CASES.items():
        if only and only != name:
            continue
        out = make_pyr(conf, gi, c)
        np.savez_compressed(os.path.join(HERE, f"geom_{name}.npz"), **out)
        print(name, "nvalid", out["nvalid"], "nfft", out["nfft"], "nrebin", out["nrebin"])
    import shesha.init.dm_init as dmi
    import shesha.util.iterkolmo as itk

    for name, c in DM_CASES.items():
        if only and only != name:
            continue
        out = make_dm(conf, gi, dmi, c)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, "ntotact", out["ntotact"], "influsize", out["influsize"], "dim", out["dim"])
    for name, c in KOLMO_CASES.items():
        if only and only != name:
            continue
        out = make_kolmo(itk, c["n"], c["L0"], c["deltax"], c["deltay"])
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, "A", out["A"].shape, "B", out["B"].shape)


if __name__ == "__main__":
    main()
