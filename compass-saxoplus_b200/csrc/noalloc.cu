// aob_extrude_noalloc: one screen extrusion that allocates no device memory.
//
// Who needs it: a real-time controller or a host framework that owns all the
// device memory up front and may not call cudaMalloc / cudaFree once its loop is
// running -- those calls synchronise the device and take an unbounded time, and
// a caller working inside a fixed memory budget may have no headroom for them.
// The aob_atmos object allocates two screens and a column buffer per layer;
// this entry point instead works on a screen the caller owns and keeps its
// scratch (the new column and a copy of the screen, for n <= 512) in one
// file-scope device array that every GPU loading the library holds until exit.
//
// It launches the two-kernel form of the extrusion (extrude_gemv_kernel, then
// extrude_shift_kernel, in sim.cu); the atmosphere object runs the same
// arithmetic fused into extrude_fused_kernel, so the result equals
// aob_atmos_move's for the same operators, noise counter and layer index, and
// the two forms check each other.

#include <algorithm>
#include <mutex>
#include <string>

#include "aob_objects.hpp"
#include "sim.hpp"

namespace {

constexpr int NOALLOC_MAX_N = AOB_NOALLOC_EXTRUDE_MAX_N;
constexpr int NOALLOC_MAX_DEVICES = 64;

// [0, MAX_N): the new column / row; [MAX_N, MAX_N + MAX_N^2): copy of the screen.
// 512 + 512^2 floats = 1,050,624 bytes per device.  Every call writes both parts
// in full before reading them, so nothing here needs to start at zero.
static __device__ __align__(256) float g_extrude_scratch[NOALLOC_MAX_N + NOALLOC_MAX_N * NOALLOC_MAX_N];

// Device address of g_extrude_scratch per device, filled on the first call made
// for that device (host code may not use the symbol's name as a pointer).  The
// address belongs to the device's primary context: after cudaDeviceReset (or
// any teardown of that context) it is stale, and the process must not call
// this entry point on that device again.
float *g_scratch_ptr[NOALLOC_MAX_DEVICES] = {};
std::mutex g_scratch_mutex;

float *scratch_on(int device) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[device]) {
    float *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_extrude_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      throw aob::Error(std::string("aob_extrude_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
    }
    g_scratch_ptr[device] = p;
  }
  return g_scratch_ptr[device];
}

}  // namespace

extern "C" int aob_extrude_noalloc(float *dev_screen, int n, int nstencil, const float *dev_A_rows,
                                   const float *dev_B_rows, const uint32_t *dev_stencil, int direction,
                                   float amplitude, int64_t seed, uint32_t counter, int layer_index, int device,
                                   void *stream) {
  try {
    if (!dev_screen || !dev_A_rows || !dev_B_rows || !dev_stencil)
      throw aob::Error("aob_extrude_noalloc: null pointer");
    if (n < 3 || n > NOALLOC_MAX_N)
      throw aob::Error("aob_extrude_noalloc: screen size n = " + std::to_string(n) +
                       " is outside [3, " + std::to_string(NOALLOC_MAX_N) + "] (the fixed scratch holds n <= " +
                       std::to_string(NOALLOC_MAX_N) + ")");
    if (nstencil < 1 || nstencil > n * n) throw aob::Error("aob_extrude_noalloc: nstencil out of range");
    if (sizeof(float) * ((size_t)nstencil + n) > 48 * 1024)
      throw aob::Error("aob_extrude_noalloc: stencil + column exceed 48 KB of shared memory");
    if (direction != 1 && direction != -1 && direction != 2 && direction != -2)
      throw aob::Error("aob_extrude_noalloc: direction must be +-1 (x) or +-2 (y)");
    if (layer_index < 0) throw aob::Error("aob_extrude_noalloc: negative layer index");
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) throw aob::Error("aob_extrude_noalloc: device out of range");
    // the caller's current device is put back on every return path
    int prev = -1;
    AOB_CUDA(cudaGetDevice(&prev));
    struct Restore {
      int dev;
      ~Restore() {
        if (dev >= 0) cudaSetDevice(dev);
      }
    } restore{prev};
    AOB_CUDA(cudaSetDevice(device));
    float *scratch = scratch_on(device);
    float *y = scratch;
    float *copy = scratch + NOALLOC_MAX_N;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

    // same launch shape and stencil reference point as aob_atmos::Layer::extrude
    const int x0ref = (direction == 1 || direction == -2) ? n - 1 : n * (n - 1);
    const uint64_t sd = (uint64_t)seed;
    const int threads = 256;
    const int rows_per_cta = threads / 32;
    const int grid = std::max(1, std::min((n + rows_per_cta - 1) / rows_per_cta, 2 * aob::num_sms(device)));
    const size_t sm = sizeof(float) * ((size_t)nstencil + n);
    aob::extrude_gemv_kernel<<<grid, threads, sm, s>>>(dev_screen, n, nstencil, dev_A_rows, dev_B_rows, dev_stencil,
                                                       x0ref, amplitude, (uint32_t)(sd & 0xffffffffu),
                                                       (uint32_t)(sd >> 32), counter, (uint32_t)layer_index, y);
    AOB_LAUNCH_CHECK("extrude_gemv_kernel");
    const int64_t nn = (int64_t)n * n;
    AOB_CUDA(cudaMemcpyAsync(copy, dev_screen, sizeof(float) * nn, cudaMemcpyDeviceToDevice, s));
    aob::extrude_shift_kernel<<<(int)std::min<int64_t>((nn + 255) / 256, 8192), 256, 0, s>>>(dev_screen, copy, y, n,
                                                                                            direction);
    AOB_LAUNCH_CHECK("extrude_shift_kernel");
    return AOB_OK;
  } catch (const std::exception &e) {
    aob::set_last_error(e.what());
    return AOB_ERR;
  }
}
