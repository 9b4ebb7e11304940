"""The allocation-free extrusion entry point against the atmosphere object.

aob_extrude_noalloc serves callers that may not allocate device memory once
they run: a real-time controller that reserves everything at start-up (because
cudaMalloc / cudaFree synchronise the device and take an unbounded time) or a
plugin whose host owns the device memory.  Its scratch is a fixed device array
inside the library, so this file checks that two and more calls in a row, each
reusing that array, give the same screens as aob_atmos_move on the same
operators and noise counters.  The file name sorts last so that a run stopping
at the first failure has run every other test before this one.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(screen, n, nst, A_rows, B_rows, ist, direction, amp, seed, counter, layer):
    from aob200 import _lib

    _lib.call("aob_extrude_noalloc", screen.data_ptr(), int(n), int(nst), A_rows.data_ptr(), B_rows.data_ptr(),
              ist.data_ptr(), int(direction), ctypes.c_float(amp), int(seed), int(counter), int(layer), 0, None)


def test_noalloc_extrusion_matches_atmosphere_move():
    import torch

    from aob200 import _lib
    from aob200 import turbulence as T

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    n = 48
    # one column along +x and one row along -y per move
    lp = T.LayerParams(r0_pix=2.5, alt=0.0, deltax=1.0, deltay=-1.0, dim=n, L0_pix=150.0, seed=4242)
    A, B, istx, isty = T.extrusion_operators(n, lp.L0_pix, lp.deltax, lp.deltay)
    atm = T.Atmosphere([], device=0)
    atm.add_screen(lp, A, B, istx, isty)
    atm.refresh(0)  # 2n extrusions: the layer's noise counter is now 2n
    counter = 2 * n

    dev = torch.device("cuda", 0)
    mine = torch.from_numpy(np.ascontiguousarray(atm.screen_host(0).ravel(order="F"))).to(dev)
    A_rows = torch.from_numpy(np.ascontiguousarray(A, dtype=np.float32)).to(dev)  # row i = A[i, :]
    B_rows = torch.from_numpy(np.ascontiguousarray(B, dtype=np.float32)).to(dev)
    ix = torch.from_numpy(istx.astype(np.int32)).to(dev)
    iy = torch.from_numpy(isty.astype(np.int32)).to(dev)
    amp = float(np.float32(np.float32(lp.r0_pix) ** np.float32(-5.0 / 6.0) * np.float32(0.5) /
                           np.float32(2 * np.pi)))

    for _ in range(2):  # two moves in a row: four calls reusing the same scratch
        atm.move()
        _noalloc(mine, n, istx.size, A_rows, B_rows, ix, 1, amp, lp.seed, counter, 0)
        counter += 1
        _noalloc(mine, n, isty.size, A_rows, B_rows, iy, -2, amp, lp.seed, counter, 0)
        counter += 1
        torch.cuda.synchronize()
        got = mine.cpu().numpy().reshape(n, n, order="F")
        ref = atm.screen_host(0)
        # the same two kernels on the same operands: the screens are equal bit for bit
        np.testing.assert_array_equal(got, ref)


def test_noalloc_rejects_screens_beyond_the_fixed_scratch():
    import torch

    from aob200 import _lib

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    dev = torch.device("cuda", 0)
    small = torch.zeros(16, device=dev)
    ist = torch.zeros(4, dtype=torch.int32, device=dev)
    too_big = 513  # AOB_NOALLOC_EXTRUDE_MAX_N + 1
    with pytest.raises(_lib.AobError, match="outside"):
        _noalloc(small, too_big, 4, small, small, ist, 1, 0.1, 1, 0, 0)
