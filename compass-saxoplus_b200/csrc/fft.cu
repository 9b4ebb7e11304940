// Batched complex 2-D FFT for power-of-two sizes (16 .. 2048), single
// precision, in place.  Used for the target PSF and the pyramid sensor.
//
// Row pass: one CTA per row, the row staged in shared memory, Stockham
// radix-8 passes with the butterflies in registers (fft.cuh), written back.
// Column pass: one CTA per group of 8 adjacent columns (64-byte row segments,
// coalesced), the same transform per column in shared memory.  Twiddles come from a table computed
// in double on the host.  Sign convention of cuFFT: forward = exp(-2 pi i k m / n),
// inverse = exp(+2 pi i k m / n), both unnormalised.

#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "aob_objects.hpp"
#include "fft.cuh"

namespace aob {

namespace {
struct TwiddleKey {
  int device, n;
  bool operator<(const TwiddleKey &o) const { return device != o.device ? device < o.device : n < o.n; }
};
std::map<TwiddleKey, DevBuf<float2> *> g_tw;
std::mutex g_tw_mu;
}  // namespace

const float2 *fft_twiddles(int device, int n) {
  std::lock_guard<std::mutex> lk(g_tw_mu);
  auto it = g_tw.find({device, n});
  if (it != g_tw.end()) return it->second->p;
  std::vector<float2> h(n / 2);
  for (int m = 0; m < n / 2; ++m) {
    const double a = 2.0 * M_PI * (double)m / (double)n;
    h[m] = make_float2((float)std::cos(a), (float)-std::sin(a));  // forward twiddles
  }
  auto *b = new DevBuf<float2>(n / 2);
  b->upload(h.data(), n / 2);
  g_tw[{device, n}] = b;  // kept for the lifetime of the process
  return b->p;
}

__global__ void fft_rows_kernel(float2 *data, int n, int logn, const float2 *tw, int inverse) {
  extern __shared__ float2 srow[];
  float2 *row = data + (size_t)blockIdx.x * n;  // blockIdx.x = row index over the whole batch
  for (int i = threadIdx.x; i < n; i += blockDim.x) srow[i] = row[i];
  __syncthreads();
  smem_fft_stockham<1>(srow, n, 1, tw, inverse != 0);
  for (int i = threadIdx.x; i < n; i += blockDim.x) row[i] = srow[i];
}

constexpr int FFT_COLS = 8;

__global__ void fft_cols_kernel(float2 *data, int n, int logn, const float2 *tw, int inverse) {
  extern __shared__ float2 scol[];
  const int groups = n / FFT_COLS;
  const int img = blockIdx.x / groups;
  const int c0 = (blockIdx.x - img * groups) * FFT_COLS;
  float2 *base = data + (size_t)img * n * n + c0;
  for (int t = threadIdx.x; t < n * FFT_COLS; t += blockDim.x) {
    const int m = t / FFT_COLS, c = t - m * FFT_COLS;
    scol[m * FFT_COLS + c] = base[(size_t)m * n + c];
  }
  __syncthreads();
  smem_fft_stockham<4>(scol, n, FFT_COLS, tw, inverse != 0);
  for (int t = threadIdx.x; t < n * FFT_COLS; t += blockDim.x) {
    const int m = t / FFT_COLS, c = t - m * FFT_COLS;
    base[(size_t)m * n + c] = scol[m * FFT_COLS + c];
  }
}

void fft2d(float2 *data, int n, int batch, bool inverse, int device, cudaStream_t s) {
  AOB_REQUIRE(n >= FFT_COLS && n <= 2048 && (n & (n - 1)) == 0, "fft2d: n must be a power of two in [8, 2048]");
  int logn = 0;
  while ((1 << logn) < n) ++logn;
  const float2 *tw = fft_twiddles(device, n);
  smem_opt_in(reinterpret_cast<const void *>(fft_cols_kernel), 2048 * FFT_COLS * 8);
  const int thr = std::min(512, std::max(32, n / 2));
  fft_rows_kernel<<<n * batch, thr, n * sizeof(float2), s>>>(data, n, logn, tw, inverse ? 1 : 0);
  AOB_LAUNCH_CHECK("fft_rows_kernel");
  fft_cols_kernel<<<(n / FFT_COLS) * batch, 512, n * FFT_COLS * sizeof(float2), s>>>(data, n, logn, tw,
                                                                                      inverse ? 1 : 0);
  AOB_LAUNCH_CHECK("fft_cols_kernel");
}

}  // namespace aob

extern "C" int aob_fft2d_c64(void *data, int n, int batch, int inverse, int device, void *stream) {
  try {
    if (!data) throw aob::Error("aob_fft2d_c64: null data");
    AOB_CUDA(cudaSetDevice(device));
    aob::fft2d(static_cast<float2 *>(data), n, batch, inverse != 0, device, reinterpret_cast<cudaStream_t>(stream));
    return AOB_OK;
  } catch (const std::exception &e) {
    aob::set_last_error(e.what());
    return AOB_ERR;
  }
}
