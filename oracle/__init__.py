"""CPU oracle for the adaptive-optics hot path -- TEST INFRASTRUCTURE ONLY.

This package is a float64 NumPy restatement of the reference's algorithms
(Shack-Hartmann and pyramid image formation, centre-of-gravity centroiders,
least-squares control law, command delay/clip, turbulence extrusion,
raytracing, DM shape and Strehl).  Each function cites the reference file and
lines it follows.  It exists to check the GPU kernels: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it, and only as the checker or the timed CPU baseline -- never as part of the
product path, which fails loudly when its CUDA library is missing.

Pinning: the geometry inputs come from the project's geometry builder, which
is pinned bit-for-bit against fixtures produced by the reference's own Python
init code (``tests/golden/make_golden.py``).  The centroid, control-law, clip
and latency/voltage functions are pinned by the same known-answer checks the
reference's own test-suite uses (``shesha/tests/pytest/rtc/test_rtcFFF.py``:
centre of mass against ``scipy.ndimage``, ``-gain*cmat.s``, clip, latency
interpolation), restated in ``tests/test_oracle.py``.  The spot-formation FFT
path has no golden data in the reference (its FFT tests are disabled), so it is
pinned by analytic properties instead (flat wavefront -> centred diffraction
spot, tilt -> known shift, Parseval, flux normalisation).
"""
