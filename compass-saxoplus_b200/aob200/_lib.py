"""ctypes binding of libaob200.so.

The prototypes are read from the C header (include/aob200.h) so that every
declared entry point is bound with the right argument types; a missing symbol
or a missing library raises immediately -- there is no fallback path.
"""

from __future__ import annotations

import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaob200.so")
HEADER = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include", "aob200.h")

_SCALARS = {
    "int": ctypes.c_int,
    "float": ctypes.c_float,
    "double": ctypes.c_double,
    "int64_t": ctypes.c_int64,
    "uint64_t": ctypes.c_uint64,
    "int32_t": ctypes.c_int32,
    "uint32_t": ctypes.c_uint32,
    "size_t": ctypes.c_size_t,
    "void": None,
}


class AobError(RuntimeError):
    pass


def _ctype(decl: str):
    decl = decl.strip()
    if "*" in decl:
        if decl.replace(" ", "").startswith("constchar*") and decl.count("*") == 1:
            return ctypes.c_char_p
        return ctypes.c_void_p
    toks = [t for t in decl.replace("const", "").split() if t]
    # drop the parameter name
    base = toks[0] if toks else "void"
    return _SCALARS[base]


def parse_header(path: str = HEADER):
    """Return {name: (restype, [argtypes])} for every prototype in the header."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("#"))
    protos = {}
    for stmt in text.split(";"):
        stmt = " ".join(stmt.split())
        m = re.match(r"^(?:extern \"C\" \{ )?(?:\} )?(.*?)\b(aob_\w+)\s*\((.*)\)$", stmt)
        if not m or stmt.startswith("typedef"):
            continue
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3)
        restype = ctypes.c_char_p if ret.replace(" ", "") == "constchar*" else _ctype(ret + " x")
        argtypes = []
        a = args.strip()
        if a and a != "void":
            for part in a.split(","):
                argtypes.append(_ctype(part))
        protos[name] = (restype, argtypes)
    return protos


_lib = None
PROTOS = None


def lib():
    """Load the library once (raises AobError if it is not built)."""
    global _lib, PROTOS
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise AobError(f"{LIB_PATH} is missing: build it with compass-saxoplus_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        PROTOS = parse_header()
        for name, (res, args) in PROTOS.items():
            fn = getattr(L, name)  # AttributeError if the symbol is not exported
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def call(name: str, *args):
    """Call an entry point that returns a status code; raise AobError on failure."""
    st = getattr(lib(), name)(*args)
    if st != 0:
        msg = lib().aob_last_error().decode()
        raise AobError(f"{name}: {msg}")


def out_ptr():
    return ctypes.c_void_p()


def addr(x):
    """Address of a numpy array (host), a ctypes object, an int device pointer, or None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if isinstance(x, (ctypes.c_void_p,)):
        return x.value
    return ctypes.addressof(x)


def host_array(a, dtype) -> np.ndarray:
    """Contiguous Fortran-order flat copy of ``a`` with the given dtype."""
    return np.ascontiguousarray(np.asarray(a, dtype=dtype).ravel(order="F"))


def d2h(ptr: int, n: int, dtype, stream=None) -> np.ndarray:
    out = np.empty(int(n), dtype=dtype)
    if n:
        call("aob_memcpy_d2h", out.ctypes.data, ptr, out.nbytes, stream)
    return out


def h2d(ptr: int, a: np.ndarray, stream=None) -> None:
    a = np.ascontiguousarray(a)
    if a.size:
        call("aob_memcpy_h2d", ptr, a.ctypes.data, a.nbytes, stream)


def device_count() -> int:
    return int(lib().aob_device_count())
