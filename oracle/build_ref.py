"""Build the reference's own GPU code (libcarma, libsutra and its pybind11
modules ``carma`` / ``sutra``) into ``oracle/_ref/`` -- test infrastructure.

The reference's sutra CUDA build is the parity oracle for the noise-free
sensor, centroider and controller paths: ``tests/golden/make_ref_fixtures.py``
imports the modules built here on a GPU, feeds them this project's geometry
and seeded phase screens, and stores what they compute as fixtures.  Nothing
in the package, the benchmark's timed path or the tests imports these modules.

This is a plain compile of the reference's source files where they lie (their
own CMake project is not used): every ``.cpp`` / ``.cu`` that the reference's
CMake lists name for libcarma (libcarma/CMakeLists.txt), libsutra
(libsutra/CMakeLists.txt) and the two Python modules
(python_module/{carma,sutra}/CMakeLists.txt), with the flags those files set:
C++14, ``-use_fast_math`` for CUDA sources (libcarma/CMakeLists.txt:45),
position-independent code, the CUDA toolkit's cuFFT / cuBLAS / cuRAND /
cuSPARSE / cuSOLVER.  Objects and libraries go to ``oracle/_ref/`` only.

Usage:  python oracle/build_ref.py [--reference DIR] [--jobs N]
``--reference`` (or ``AO_REFERENCE``) names the reference checkout; when it is
absent the build is skipped (the GPU box uses the libraries built here).
"""

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "obj")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
DEFAULT_REF = "/root/reference"

# source lists of the reference's CMake files (commented-out entries stay out)
CARMA_SRC = ["src.cpp/carma_context.cpp", "src.cpp/carma_cublas.cpp", "src.cpp/carma_cusolver.cpp",
             "src.cpp/carma_cusparse.cpp", "src.cpp/carma_fft.cpp", "src.cpp/carma_host_obj.cpp",
             "src.cpp/carma_sparse_host_obj.cpp", "src.cpp/carma_sparse_obj.cpp", "src.cpp/carma_streams.cpp",
             "src.cpp/carma_utils.cpp", "src.cpp/carma_obj.cpp", "src.cu/carma_timer.cu", "src.cu/carma_rng.cu",
             "src.cu/carma_svd.cu", "src.cu/carma_utils.cu", "src.cu/carma_obj.cu", "src.cu/carma_sum.cu",
             "src.cu/carma_transpose.cu"]
SUTRA_SRC = ["src.cpp/" + f + ".cpp" for f in (
    "sutra_acquisim", "sutra_atmos", "sutra_centroider_bpcog", "sutra_centroider_cog", "sutra_centroider_corr",
    "sutra_centroider", "sutra_centroider_pyr", "sutra_centroider_maskedPix", "sutra_centroider_tcog",
    "sutra_centroider_wcog", "sutra_controller", "sutra_controller_generic", "sutra_controller_generic_linear",
    "sutra_controller_geo", "sutra_controller_ls", "sutra_controller_mv", "sutra_dm", "sutra_gamora", "sutra_groot",
    "sutra_kl", "sutra_lgs", "sutra_phase", "sutra_rtc", "sutra_source", "sutra_target", "sutra_telemetry",
    "sutra_telescope", "sutra_tscreen", "sutra_sensors", "sutra_wfs", "sutra_wfs_pyr_pyrhr", "sutra_wfs_sh",
    "sutra_coronagraph", "sutra_perfectCoronagraph", "sutra_stellarCoronagraph")] + \
    ["src.cu/" + f + ".cu" for f in (
        "sutra_acquisim", "sutra_utils", "sutra_centroider", "sutra_centroider_cog", "sutra_centroider_tcog",
        "sutra_centroider_wcog", "sutra_centroider_bpcog", "sutra_centroider_corr", "sutra_centroider_pyr",
        "sutra_centroider_maskedPix", "sutra_controller", "sutra_controller_utils", "sutra_dm", "sutra_gamora",
        "sutra_groot", "sutra_kl", "sutra_lgs", "sutra_target", "sutra_tscreen", "sutra_wfs", "sutra_coronagraph")]
PYCARMA_SRC = ["context.cpp", "timer.cpp", "host_obj.cpp", "obj.cpp", "sparse_obj.cpp", "carma.cpp"]
PYSUTRA_SRC = [f + ".cpp" for f in (
    "telescope", "tscreen", "atmos", "dms", "source", "lgs", "target", "sensors", "wfs", "wfs_sh", "wfs_pyrhr",
    "centroider", "centroider_tcog", "centroider_wcog", "centroider_bpcog", "centroider_corr", "centroider_pyr",
    "centroider_maskedPix", "controller", "controller_ls", "controller_mv", "controller_geo", "controller_generic",
    "controller_generic_linear", "rtc", "gamora", "groot", "coronagraph", "perfect_coronagraph",
    "stellar_coronagraph", "sutra")]

ARCH = ["-gencode", "arch=compute_100,code=sm_100"]
LIBS = ["-L" + os.path.join(CUDA, "lib64"), "-lcudart", "-lcufft", "-lcublas", "-lcurand", "-lcusparse",
        "-lcusolver", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]


def _pybind_includes():
    import pybind11

    return ["-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"]]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, obj, incs, extra=()):
    if not _stale(obj, [src, __file__]):
        return None
    os.makedirs(os.path.dirname(obj), exist_ok=True)
    common = ["-O3", "-std=c++14", "-DVERSION_INFO=6.0.0", "-DUSE_P2P_ACCESS"] + incs + list(extra)
    if src.endswith(".cu"):
        cmd = [NVCC] + ARCH + ["-use_fast_math", "-Xcompiler", "-fPIC", "-Wno-deprecated-gpu-targets",
                               "-Xcudafe", "--diag_suppress=esa_on_defaulted_function_ignored"] + common + \
            ["-c", src, "-o", obj]
    else:
        cmd = ["g++", "-fPIC", "-w", "-I" + os.path.join(CUDA, "include")] + common + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return "FAILED: " + " ".join(cmd) + "\n" + r.stdout[-4000:] + r.stderr[-4000:]
    return None


def build(ref=None, jobs=None, verbose=False):
    ref = ref or os.environ.get("AO_REFERENCE") or DEFAULT_REF
    if not os.path.isdir(os.path.join(ref, "libsutra")):
        if verbose:
            print(f"build_ref: no reference checkout at {ref}; skipped")
        return None
    inc = ["-I" + os.path.join(ref, p) for p in ("libcarma/include", "libcarma/include.cuh", "libsutra/include",
                                                 "libsutra/src.cu")]
    jobs = jobs or os.cpu_count() or 4
    units = [(os.path.join(ref, "libcarma", s), os.path.join(OBJ, "carma", s + ".o"), inc, ()) for s in CARMA_SRC]
    units += [(os.path.join(ref, "libsutra", s), os.path.join(OBJ, "sutra", s + ".o"), inc, ()) for s in SUTRA_SRC]
    pyinc = _pybind_includes()
    pyx = ("-fvisibility=hidden",)
    units += [(os.path.join(ref, "python_module/carma/src", s), os.path.join(OBJ, "pycarma", s + ".o"), inc + pyinc,
               pyx) for s in PYCARMA_SRC]
    units += [(os.path.join(ref, "python_module/sutra/src", s), os.path.join(OBJ, "pysutra", s + ".o"), inc + pyinc,
               pyx) for s in PYSUTRA_SRC]
    errors = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for msg in ex.map(lambda u: _compile(*u), units):
            if msg:
                errors.append(msg)
    if errors:
        raise RuntimeError("\n\n".join(errors[:3]))
    core = os.path.join(OUT, "libcompass_ref.so")
    core_objs = [u[1] for u in units if "/carma/" in u[1] or "/sutra/" in u[1]]
    if _stale(core, core_objs):
        # device link of the CUDA objects, then one shared library
        dlink = os.path.join(OBJ, "dlink.o")
        cu_objs = [o for o in core_objs if o.endswith(".cu.o")]
        subprocess.run([NVCC] + ARCH + ["-Xcompiler", "-fPIC", "-dlink"] + cu_objs + ["-o", dlink], check=True)
        r = subprocess.run(["g++", "-shared", "-o", core] + core_objs + [dlink] + LIBS, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: " + r.stderr[-4000:])
    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    for name, sub in (("carma", "pycarma"), ("sutra", "pysutra")):
        mod = os.path.join(OUT, name + suffix)
        objs = [u[1] for u in units if f"/{sub}/" in u[1]]
        if _stale(mod, objs + [core]):
            r = subprocess.run(["g++", "-shared", "-o", mod] + objs + ["-L" + OUT, "-lcompass_ref",
                                                                       "-Wl,-rpath,$ORIGIN"] + LIBS,
                               capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("link failed: " + r.stderr[-4000:])
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args()
    print(build(a.reference, a.jobs, verbose=True))
    sys.exit(0)
