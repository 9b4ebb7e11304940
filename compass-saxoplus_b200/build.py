"""Build libaob200.so in-tree for sm_100a with nvcc.

Usage:  python compass-saxoplus_b200/build.py [--force] [--jobs N]

Every ``csrc/*.cu`` file is compiled to an object under ``_build/`` (skipped
when up to date) and linked into ``aob200/libaob200.so`` next to the Python
package that loads it.  No GPU is needed to build.
"""

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "aob200")
LIB = os.path.join(OUT_DIR, "libaob200.so")
BUILD = os.path.join(HERE, "_build")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
    "-DAOB_BUILD",
]
LDFLAGS = ARCH + ["-shared", "-L" + os.path.join(CUDA, "lib64"), "-lcublas", "-lcusolver", "-lcuda",
                  "-Xlinker", "-rpath=" + os.path.join(CUDA, "lib64")]


def _deps(src):
    hdrs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return [src] + hdrs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def compile_one(src, force=False, extra=()):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and not _stale(obj, _deps(src) + [__file__]):
        return obj, None
    cmd = [NVCC] + CFLAGS + list(extra) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "FAILED: " + " ".join(cmd) + "\n" + r.stdout + r.stderr
    return obj, r.stderr.strip() or None


def build(force=False, jobs=None, verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    objs = []
    errors = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for obj, msg in ex.map(lambda s: compile_one(s, force, extra), srcs):
            objs.append(obj)
            if msg and msg.startswith("FAILED"):
                errors.append(msg)
            elif msg and verbose:
                print(msg)
    if errors:
        raise RuntimeError("\n".join(errors))
    # visibility: the C ABI functions carry default visibility via the export map below
    if force or _stale(LIB, objs):
        cmd = [NVCC] + LDFLAGS + objs + ["-o", LIB]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    build_native_dropin(force=force)
    return LIB


NATIVE = os.path.join(HERE, "dropin_native")


def build_native_dropin(force=False):
    """The compiled drop-in modules `carma` and `sutra` (pybind11, g++), linked
    against libaob200.so next to them (rpath $ORIGIN/../aob200)."""
    import sysconfig

    import pybind11

    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    hdrs = glob.glob(os.path.join(NATIVE, "*.hpp")) + [os.path.join(ROOT, "include", "aob200.h"), __file__]
    cflags = ["-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", "-I" + pybind11.get_include(),
              "-I" + sysconfig.get_paths()["include"], "-I" + os.path.join(ROOT, "include")]
    out = []
    for name in ("carma", "sutra"):
        src = os.path.join(NATIVE, name + ".cpp")
        so = os.path.join(NATIVE, name + suffix)
        if force or _stale(so, [src] + hdrs + [LIB]):
            cmd = ["g++"] + cflags + [src, "-o", so, "-L" + OUT_DIR, "-laob200", "-Wl,-rpath,$ORIGIN/../aob200"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("native drop-in build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        out.append(so)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--ptxas-v", action="store_true", help="print register / shared-memory usage")
    a = ap.parse_args()
    extra = ("-Xptxas", "-v") if a.ptxas_v else ()
    print(build(force=a.force or a.ptxas_v, jobs=a.jobs, verbose=True, extra=extra))
    sys.exit(0)
