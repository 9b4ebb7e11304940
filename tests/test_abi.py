"""CPU checks of the C ABI: the library loads, exports every symbol the header
declares, and reports errors as status codes with a message (no GPU needed)."""

import ctypes
import subprocess

import pytest

from aob200 import _lib


def test_library_exports_every_declared_symbol():
    protos = _lib.parse_header()
    assert len(protos) > 50
    L = _lib.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in protos if n not in exported]
    assert not missing, missing
    for n in protos:
        assert getattr(L, n) is not None


def test_version_and_device_count_never_fail():
    assert _lib.lib().aob_version().startswith(b"aob200")
    assert _lib.device_count() >= 0


def test_null_handles_return_error_status():
    L = _lib.lib()
    assert L.aob_sh_comp_image(None, 0, None) == 1
    assert b"null" in L.aob_last_error()
    assert L.aob_ls_comp_com(None, None) == 1
    assert L.aob_centro_get_cog(None, None, None) == 1
    with pytest.raises(_lib.AobError):
        _lib.call("aob_ls_set_gain", None, ctypes.c_float(0.1))


def test_bad_sizes_rejected_before_any_allocation():
    h = ctypes.c_void_p()
    # nfft = 24 is not a supported support size: rejected by the constructor checks
    assert _lib.lib().aob_sh_create(ctypes.addressof(h), 0, 8, 10, 4, 6, 2, 24, 24, 52, 1.0, 100.0, 0.0) == 1
    assert b"nfft" in _lib.lib().aob_last_error()
    assert h.value is None
