// High-resolution pyramid wavefront sensor with modulation.
//
// Reference: SutraWfs_PyrHR::comp_generic / comp_modulation
// (libsutra/src.cpp/sutra_wfs_pyr_pyrhr.cpp:379-627) and its kernels
// (libsutra/src.cu/sutra_wfs.cu: pyrgetpup_krnl :1191-1233, submask_krnl and
// submaskpyr_krnl :1864-1958, pyr_bimg_krnl :1580-1630, pyrfact_krnl
// :2164-2241; abs2_krnl with a factor, sutra_utils.cu:118-142).  Per
// modulation point the reference fills the padded pupil field, runs a cuFFT
// inverse transform, multiplies by the field stop and the pyramid phase mask,
// runs a forward transform and accumulates the weighted |.|^2; then the
// high-resolution image is convolved with the pixel transfer function (FFT,
// x sinc, FFT), binned by nrebin and normalised to nphot.
//
// Here the npts modulation planes (npts x nfft^2 complex, 50 MB at 512^2 x 24:
// resident in the 126 MB L2) go through three fused passes:
//   rows   inverse transform along x of the ntot pupil rows only (the other
//          rows of the padded field are zero), field and modulation tilt
//          formed on the fly;
//   cols   per 8 columns: inverse transform along y (zero rows skipped on
//          load), field stop x pyramid mask, forward transform along y, all
//          in shared memory;
//   accum  per row: forward transform along x of every modulation plane at
//          once (interleaved in shared memory) and the weighted |.|^2 summed
//          over the points in registers, in point order.
// The pixel-transfer convolution reuses the row / column pattern, the last
// pass bins nrebin rows per CTA, and one kernel normalises and adds the
// Philox photon / readout noise of the SH sensor (same sampler, same streams).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "aob_objects.hpp"
#include "fft.cuh"

namespace aob {

constexpr int PYR_COLS = 8;
constexpr int PYR_THREADS = 512;
constexpr int PYR_MAX_ACC = 4;  // nfft / PYR_THREADS <= 4 -> nfft <= 2048

struct PyrArgs {
  int n, logn, ntot, off, npts;
  const float *phase, *pupil;
  float mic2rad;
  const float *cx, *cy, *w;
  const float *submask;
  const float2 *phalfxy;
  const float *sincar;
  const float2 *tw;
  float2 *work;   // npts x n x n
  float2 *conv;   // n x n
  float *hrimg;   // n x n
  float *binimg;  // nb x nb
  float *partial; // nb row sums
  int nrebin, nb;
};

// complex multiply
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.y * b.x + a.x * b.y);
}

// 1. rows of the padded pupil field, inverse transform along x.
//    CTA (p, yb): work[p][yb][:] for pupil row yb < ntot.
__global__ void __launch_bounds__(PYR_THREADS) pyr_rows_kernel(PyrArgs A) {
  extern __shared__ float2 srow[];
  const int p = blockIdx.x / A.ntot, yb = blockIdx.x - p * A.ntot;
  const float cxp = A.cx[p], cyp = A.cy[p];
  const float yy = (float)yb - A.ntot / 2.0f;
  for (int i = threadIdx.x; i < A.n; i += blockDim.x) {
    const int x = i - A.off;
    float2 v = make_float2(0.f, 0.f);
    if (x >= 0 && x < A.ntot) {
      const int id = x + yb * A.ntot;
      const float xx = (float)x - A.ntot / 2.0f;
      float sn, cs;
      sincosf(A.phase[id] * A.mic2rad + (cxp * xx + cyp * yy), &sn, &cs);
      const float a = A.pupil[id];
      v = make_float2(cs * a, sn * a);
    }
    srow[bitrev(i, A.logn)] = v;
  }
  __syncthreads();
  smem_fft(srow, A.n, A.logn, 1, A.tw, 1);
  float2 *out = A.work + ((size_t)p * A.n + yb) * A.n;
  for (int i = threadIdx.x; i < A.n; i += blockDim.x) out[i] = srow[i];
}

// 2. per group of PYR_COLS columns of one modulation plane: inverse transform
//    along y (rows outside the pupil are zero), x field stop, x pyramid
//    phase mask, forward transform along y.  In place in work[p].
__global__ void __launch_bounds__(PYR_THREADS) pyr_cols_kernel(PyrArgs A) {
  extern __shared__ float2 scol[];
  const int groups = A.n / PYR_COLS;
  const int p = blockIdx.x / groups;
  const int c0 = (blockIdx.x - p * groups) * PYR_COLS;
  float2 *base = A.work + (size_t)p * A.n * A.n + c0;
  const int nel = A.n * PYR_COLS;
  for (int t = threadIdx.x; t < nel; t += blockDim.x) {
    const int m = t / PYR_COLS, c = t - m * PYR_COLS;
    const int yb = m - A.off;
    const float2 v = (yb >= 0 && yb < A.ntot) ? base[(size_t)yb * A.n + c] : make_float2(0.f, 0.f);
    scol[bitrev(m, A.logn) * PYR_COLS + c] = v;
  }
  __syncthreads();
  smem_fft(scol, A.n, A.logn, PYR_COLS, A.tw, 1);
  // masks, and the bit-reversal permutation for the forward transform (each
  // pair m < bitrev(m) is swapped by one thread)
  for (int t = threadIdx.x; t < nel; t += blockDim.x) {
    const int m = t / PYR_COLS, c = t - m * PYR_COLS;
    const int r = (int)bitrev(m, A.logn);
    if (m > r) continue;
    const size_t gm = (size_t)(c0 + c) + (size_t)m * A.n, gr = (size_t)(c0 + c) + (size_t)r * A.n;
    float2 a = scol[m * PYR_COLS + c];
    const float sm = A.submask[gm];
    a = cmul(make_float2(a.x * sm, a.y * sm), A.phalfxy[gm]);
    if (m == r) {
      scol[m * PYR_COLS + c] = a;
    } else {
      float2 b = scol[r * PYR_COLS + c];
      const float sr = A.submask[gr];
      b = cmul(make_float2(b.x * sr, b.y * sr), A.phalfxy[gr]);
      scol[m * PYR_COLS + c] = b;
      scol[r * PYR_COLS + c] = a;
    }
  }
  __syncthreads();
  smem_fft(scol, A.n, A.logn, PYR_COLS, A.tw, 0);
  for (int t = threadIdx.x; t < nel; t += blockDim.x) {
    const int m = t / PYR_COLS, c = t - m * PYR_COLS;
    base[(size_t)m * A.n + c] = scol[m * PYR_COLS + c];
  }
}

// 3. per row y: forward transform along x of ``pb`` modulation planes at a
//    time (interleaved), hrimg[y][x] = sum_p w_p |.|^2 in point order.
__global__ void __launch_bounds__(PYR_THREADS) pyr_accum_kernel(PyrArgs A, int pb_max) {
  extern __shared__ float2 sacc[];
  const int y = blockIdx.x;
  float acc[PYR_MAX_ACC];
#pragma unroll
  for (int j = 0; j < PYR_MAX_ACC; ++j) acc[j] = 0.f;
  for (int p0 = 0; p0 < A.npts; p0 += pb_max) {
    const int pb = min(pb_max, A.npts - p0);
    for (int t = threadIdx.x; t < A.n * pb; t += blockDim.x) {
      const int q = t / A.n, m = t - q * A.n;
      sacc[bitrev(m, A.logn) * pb + q] = A.work[((size_t)(p0 + q) * A.n + y) * A.n + m];
    }
    __syncthreads();
    smem_fft(sacc, A.n, A.logn, pb, A.tw, 0);
#pragma unroll
    for (int j = 0; j < PYR_MAX_ACC; ++j) {
      const int m = threadIdx.x + j * blockDim.x;
      if (m < A.n)
        for (int q = 0; q < pb; ++q) {
          const float2 v = sacc[m * pb + q];
          acc[j] += A.w[p0 + q] * (v.x * v.x + v.y * v.y);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < PYR_MAX_ACC; ++j) {
    const int m = threadIdx.x + j * blockDim.x;
    if (m < A.n) A.hrimg[(size_t)y * A.n + m] = acc[j];
  }
}

// 4. pixel transfer function: rows of hrimg (real), inverse transform along x.
__global__ void __launch_bounds__(PYR_THREADS) pyr_conv_rows_kernel(PyrArgs A) {
  extern __shared__ float2 srow[];
  const int y = blockIdx.x;
  for (int i = threadIdx.x; i < A.n; i += blockDim.x)
    srow[bitrev(i, A.logn)] = make_float2(A.hrimg[(size_t)y * A.n + i], 0.f);
  __syncthreads();
  smem_fft(srow, A.n, A.logn, 1, A.tw, 1);
  for (int i = threadIdx.x; i < A.n; i += blockDim.x) A.conv[(size_t)y * A.n + i] = srow[i];
}

// 5. columns: inverse transform along y, x sinc, forward transform along y.
__global__ void __launch_bounds__(PYR_THREADS) pyr_conv_cols_kernel(PyrArgs A) {
  extern __shared__ float2 scol[];
  const int c0 = blockIdx.x * PYR_COLS;
  float2 *base = A.conv + c0;
  const int nel = A.n * PYR_COLS;
  for (int t = threadIdx.x; t < nel; t += blockDim.x) {
    const int m = t / PYR_COLS, c = t - m * PYR_COLS;
    scol[bitrev(m, A.logn) * PYR_COLS + c] = base[(size_t)m * A.n + c];
  }
  __syncthreads();
  smem_fft(scol, A.n, A.logn, PYR_COLS, A.tw, 1);
  for (int t = threadIdx.x; t < nel; t += blockDim.x) {
    const int m = t / PYR_COLS, c = t - m * PYR_COLS;
    const int r = (int)bitrev(m, A.logn);
    if (m > r) continue;
    float2 a = scol[m * PYR_COLS + c];
    const float sm = A.sincar[(size_t)(c0 + c) + (size_t)m * A.n];
    a = make_float2(a.x * sm, a.y * sm);
    if (m == r) {
      scol[m * PYR_COLS + c] = a;
    } else {
      float2 b = scol[r * PYR_COLS + c];
      const float sr = A.sincar[(size_t)(c0 + c) + (size_t)r * A.n];
      scol[m * PYR_COLS + c] = make_float2(b.x * sr, b.y * sr);
      scol[r * PYR_COLS + c] = a;
    }
  }
  __syncthreads();
  smem_fft(scol, A.n, A.logn, PYR_COLS, A.tw, 0);
  for (int t = threadIdx.x; t < nel; t += blockDim.x) {
    const int m = t / PYR_COLS, c = t - m * PYR_COLS;
    base[(size_t)m * A.n + c] = scol[m * PYR_COLS + c];
  }
}

// 6. nrebin rows per CTA: forward transform along x, real part, binning
//    (pyr_bimg_krnl order: x offset outer, y offset inner, then / nrebin^2),
//    and the row sum of the binned image for the normalisation.
__global__ void __launch_bounds__(PYR_THREADS) pyr_bin_kernel(PyrArgs A) {
  extern __shared__ float2 sbin[];
  float *real = reinterpret_cast<float *>(sbin + A.n);  // nrebin x n
  const int by = blockIdx.x;
  for (int jj = 0; jj < A.nrebin; ++jj) {
    const int y = by * A.nrebin + jj;
    for (int i = threadIdx.x; i < A.n; i += blockDim.x) sbin[bitrev(i, A.logn)] = A.conv[(size_t)y * A.n + i];
    __syncthreads();
    smem_fft(sbin, A.n, A.logn, 1, A.tw, 0);
    for (int i = threadIdx.x; i < A.n; i += blockDim.x) real[jj * A.n + i] = sbin[i].x;
    __syncthreads();
  }
  const float inv = (float)(A.nrebin * A.nrebin);
  for (int bx = threadIdx.x; bx < A.nb; bx += blockDim.x) {
    float o = 0.f;
    for (int ii = 0; ii < A.nrebin; ++ii)
      for (int jj = 0; jj < A.nrebin; ++jj) o = o + real[jj * A.n + bx * A.nrebin + ii];
    A.binimg[(size_t)by * A.nb + bx] = o / inv;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int bx = 0; bx < A.nb; ++bx) s += A.binimg[(size_t)by * A.nb + bx];
    A.partial[by] = s;
  }
}

// 7. normalisation to nphot (sum of the row sums in row order) and noise.
__global__ void pyr_norm_noise_kernel(float *binimg, const float *partial, int nb, float nphot, int noise_mode,
                                      float noise, uint32_t frame, uint32_t k0, uint32_t k1) {
  __shared__ float s_fact;
  __shared__ float rk[AOB_POISSON_INV_KMAX + 1];
  if (noise_mode >= 1)
    for (int i = threadIdx.x; i <= AOB_POISSON_INV_KMAX; i += blockDim.x) rk[i] = i ? __frcp_rn((float)i) : 0.f;
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int r = 0; r < nb; ++r) s += partial[r];
    s_fact = nphot / s;
  }
  __syncthreads();
  const float fact = s_fact;
  const int n2 = nb * nb;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) {
    float v = binimg[i] * fact;
    if (noise_mode >= 1) {
      const U4 w0 = philox4x32_10(U4{(uint32_t)i, frame, TAG_POISSON, 0u}, k0, k1);
      v = v < AOB_POISSON_INV_MAX_MEAN ? poisson_inversion(v, w0, rk) : poisson_ptrs(v, w0, (uint32_t)i, frame, k0, k1);
      if (noise_mode >= 2) v = v + noise * gauss_sample(w0);
    }
    binimg[i] = v;
  }
}

}  // namespace aob

using namespace aob;

aob_pyr::aob_pyr(int device_, int nxsub_, int nvalid_, int npix_, int nphase_, int nrebin_, int nfft_, int ntot_,
                 int npts_, float pdiam_, float nphot_, float nphot4imat_)
    : device(device_), nxsub(nxsub_), nvalid(nvalid_), npix(npix_), nphase(nphase_), nrebin(nrebin_), nfft(nfft_),
      ntot(ntot_), npts(npts_), pdiam(pdiam_), nphot(nphot_), nphot4imat(nphot4imat_) {
  AOB_REQUIRE(nvalid > 0 && nrebin > 0 && ntot > 0 && npts > 0, "pyr: sizes must be > 0");
  AOB_REQUIRE(nfft >= 64 && nfft <= PYR_THREADS * PYR_MAX_ACC && (nfft & (nfft - 1)) == 0,
              "pyr: nfft must be a power of two in [64, 2048]");
  AOB_REQUIRE(ntot <= nfft, "pyr: the phase grid (ntot) must fit in nfft");
  AOB_REQUIRE(nfft % nrebin == 0, "pyr: nfft must be a multiple of nrebin");
  AOB_REQUIRE((size_t)nfft * PYR_COLS * sizeof(float2) <= 200 * 1024, "pyr: nfft too large for the column pass");
  while ((1 << logn) < nfft) ++logn;
  AOB_CUDA(cudaSetDevice(device));
  phase.alloc((int64_t)ntot * ntot);
  pupil.alloc((int64_t)ntot * ntot);
  const int64_t n2 = (int64_t)nfft * nfft;
  submask.alloc(n2);
  sincar.alloc(n2);
  phalfxy.alloc(n2);
  conv.alloc(n2);
  hrimg.alloc(n2);
  binimg.alloc((int64_t)nbin() * nbin());
  partial.alloc(nbin());
  validsubsx.alloc(4 * (int64_t)nvalid);
  validsubsy.alloc(4 * (int64_t)nvalid);
  fluxPerSub.alloc(nvalid);
}

void aob_pyr::set_modulation(const float *h_cx, const float *h_cy, const float *h_w, int n) {
  AOB_REQUIRE(h_cx && h_cy && n > 0, "pyr.set_modulation: null points");
  AOB_CUDA(cudaSetDevice(device));
  npts = n;
  cx.alloc(n);
  cy.alloc(n);
  weights.alloc(n);
  cx.upload(h_cx, n);
  cy.upload(h_cy, n);
  std::vector<float> one(n, 1.f);
  weights.upload(h_w ? h_w : one.data(), n);
  work.alloc((int64_t)npts * nfft * nfft);
}

void aob_pyr::load_arrays(const float2 *h_halfxy, const float *h_cx, const float *h_cy, const float *h_w,
                          const float *h_sincar, const float *h_submask, const int32_t *h_vsx, const int32_t *h_vsy,
                          const float *h_flux) {
  AOB_REQUIRE(h_halfxy && h_sincar && h_submask && h_vsx && h_vsy, "pyr.load_arrays: a required array is NULL");
  const int nb = nbin();
  for (int i = 0; i < 4 * nvalid; ++i)
    AOB_REQUIRE(h_vsx[i] >= 0 && h_vsx[i] < nb && h_vsy[i] >= 0 && h_vsy[i] < nb,
                "pyr.load_arrays: valid pixel outside the binned image");
  set_modulation(h_cx, h_cy, h_w, npts);
  const int64_t n2 = (int64_t)nfft * nfft;
  phalfxy.upload(h_halfxy, n2);
  sincar.upload(h_sincar, n2);
  submask.upload(h_submask, n2);
  validsubsx.upload(h_vsx, 4 * (int64_t)nvalid);
  validsubsy.upload(h_vsy, 4 * (int64_t)nvalid);
  if (h_flux) fluxPerSub.upload(h_flux, nvalid);
  loaded = true;
}

void aob_pyr::comp_image(bool with_noise, cudaStream_t s) {
  AOB_REQUIRE(loaded, "pyr.comp_image: load_arrays has not been called");
  AOB_CUDA(cudaSetDevice(device));
  PyrArgs A{};
  A.n = nfft;
  A.logn = logn;
  A.ntot = ntot;
  A.off = (int)((nfft - ntot) / 2.0f);
  A.npts = npts;
  A.phase = phase.p;
  A.pupil = pupil.p;
  A.mic2rad = 2.0f * (float)M_PI / lambda_um;
  A.cx = cx.p;
  A.cy = cy.p;
  A.w = weights.p;
  A.submask = submask.p;
  A.phalfxy = phalfxy.p;
  A.sincar = sincar.p;
  A.tw = fft_twiddles(device, nfft);
  A.work = work.p;
  A.conv = conv.p;
  A.hrimg = hrimg.p;
  A.binimg = binimg.p;
  A.partial = partial.p;
  A.nrebin = nrebin;
  A.nb = nbin();
  const size_t row_sm = sizeof(float2) * nfft;
  const size_t col_sm = sizeof(float2) * nfft * PYR_COLS;
  const int pb = std::max(1, std::min(npts, (int)((200 * 1024) / row_sm)));
  const size_t acc_sm = row_sm * pb;
  const size_t bin_sm = row_sm + sizeof(float) * nfft * nrebin;
  static size_t configured[3] = {0, 0, 0};
  auto attr = [](const void *k, size_t sm, size_t &done) {
    if (sm > done) {
      AOB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(sm, 48 * 1024)));
      done = std::max<size_t>(sm, 48 * 1024);
    }
  };
  attr((const void *)pyr_cols_kernel, col_sm, configured[0]);
  attr((const void *)pyr_accum_kernel, acc_sm, configured[1]);
  attr((const void *)pyr_conv_cols_kernel, col_sm, configured[2]);
  AOB_REQUIRE(bin_sm <= 48 * 1024, "pyr: nfft * nrebin too large for the binning pass");
  pyr_rows_kernel<<<npts * ntot, PYR_THREADS, row_sm, s>>>(A);
  AOB_LAUNCH_CHECK("pyr_rows_kernel");
  pyr_cols_kernel<<<npts * (nfft / PYR_COLS), PYR_THREADS, col_sm, s>>>(A);
  AOB_LAUNCH_CHECK("pyr_cols_kernel");
  pyr_accum_kernel<<<nfft, PYR_THREADS, acc_sm, s>>>(A, pb);
  AOB_LAUNCH_CHECK("pyr_accum_kernel");
  pyr_conv_rows_kernel<<<nfft, PYR_THREADS, row_sm, s>>>(A);
  AOB_LAUNCH_CHECK("pyr_conv_rows_kernel");
  pyr_conv_cols_kernel<<<nfft / PYR_COLS, PYR_THREADS, col_sm, s>>>(A);
  AOB_LAUNCH_CHECK("pyr_conv_cols_kernel");
  pyr_bin_kernel<<<nbin(), PYR_THREADS, bin_sm, s>>>(A);
  AOB_LAUNCH_CHECK("pyr_bin_kernel");
  const float nz = with_noise ? noise : -1.f;
  const int noise_mode = nz > 0 ? 2 : (nz > -1 ? 1 : 0);
  const int nb2 = nbin() * nbin();
  pyr_norm_noise_kernel<<<std::min((nb2 + 255) / 256, 4 * num_sms(device)), 256, 0, s>>>(
      binimg.p, partial.p, nbin(), nphot, noise_mode, nz, (uint32_t)frame, (uint32_t)((uint64_t)seed & 0xffffffffu),
      (uint32_t)((uint64_t)seed >> 32));
  AOB_LAUNCH_CHECK("pyr_norm_noise_kernel");
  if (noise_mode) ++frame;
  ++image_gen;
}
