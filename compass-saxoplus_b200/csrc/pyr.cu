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
//          rows of the padded field are zero), 8 rows per CTA, field and
//          modulation tilt formed on the fly;
//   cols   per 8 columns: inverse transform along y (zero rows skipped on
//          load), field stop x pyramid mask, forward transform along y, all
//          in shared memory;
//   accum  per row: forward transform along x of 8 modulation planes at a
//          time (interleaved in shared memory) and the weighted |.|^2 summed
//          over the points in registers, in point order.
// The transforms are Stockham radix-8 passes with the butterflies in
// registers (fft.cuh, fft_ct), compiled per nfft so that every index is a
// constant expression, in natural order, so no permutation pass is needed.
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

constexpr int PYR_SEQ = 8;        // sequences (rows or columns) per CTA
constexpr int PYR_THREADS = 512;

struct PyrArgs {
  int ntot, off, npts;
  const float *phase, *pupil;
  float mic2rad;
  const float *cx, *cy, *w;
  const float *submask;
  const float2 *phalfxy;
  const float *sincar;
  const float2 *tw;  // N/2 forward twiddles (global)
  float2 *work;      // npts x N x N
  float2 *conv;      // N x N
  float *hrimg;      // N x N
  float *binimg;     // nb x nb
  float *partial;    // nb row sums
  float *focal_work; // npts x N x N, w_p |field stop x focal field|^2 (null: not computed)
  int nrebin, nb, rows_per_bin_cta;
};

// complex multiply
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.y * b.x + a.x * b.y);
}

// shared memory of every pyramid kernel: PYR_SEQ interleaved sequences of N
// complex values, then the N/2 twiddles
template <int N>
__device__ __forceinline__ float2 *pyr_load_twiddles(float2 *sm, const float2 *tw) {
  float2 *tws = sm + N * PYR_SEQ;
  for (int i = threadIdx.x; i < N / 2; i += blockDim.x) tws[i] = tw[i];
  return tws;
}

// 1. rows of the padded pupil field, inverse transform along x; a CTA takes
//    PYR_SEQ pupil rows of one modulation point: work[p][yb][:].
template <int N>
__global__ void __launch_bounds__(PYR_THREADS) pyr_rows_kernel(PyrArgs A) {
  extern __shared__ float2 sm[];
  float2 *tws = pyr_load_twiddles<N>(sm, A.tw);
  const int groups = (A.ntot + PYR_SEQ - 1) / PYR_SEQ;
  const int p = blockIdx.x / groups;
  const int y0 = (blockIdx.x - p * groups) * PYR_SEQ;
  const float cxp = A.cx[p], cyp = A.cy[p];
  for (int t = threadIdx.x; t < N * PYR_SEQ; t += PYR_THREADS) {
    const int c = t / N, i = t - c * N;
    const int yb = y0 + c, x = i - A.off;
    float2 v = make_float2(0.f, 0.f);
    if (yb < A.ntot && x >= 0 && x < A.ntot) {
      const int id = x + yb * A.ntot;
      const float xx = (float)x - A.ntot / 2.0f, yy = (float)yb - A.ntot / 2.0f;
      float sn, cs;
      sincosf(A.phase[id] * A.mic2rad + (cxp * xx + cyp * yy), &sn, &cs);
      const float a = A.pupil[id];
      v = make_float2(cs * a, sn * a);
    }
    sm[i * PYR_SEQ + c] = v;
  }
  __syncthreads();
  fft_ct<N, PYR_SEQ, PYR_THREADS>(sm, tws, true);
  for (int t = threadIdx.x; t < N * PYR_SEQ; t += PYR_THREADS) {
    const int c = t / N, i = t - c * N;
    if (y0 + c < A.ntot) A.work[((size_t)p * N + y0 + c) * N + i] = sm[i * PYR_SEQ + c];
  }
}

// 2. per group of PYR_SEQ columns of one modulation plane: inverse transform
//    along y (rows outside the pupil are zero), x field stop, x pyramid
//    phase mask (submask_krnl, submaskpyr_krnl), forward transform along y.
//    In place in work[p].
template <int N>
__global__ void __launch_bounds__(PYR_THREADS) pyr_cols_kernel(PyrArgs A) {
  extern __shared__ float2 sm[];
  float2 *tws = pyr_load_twiddles<N>(sm, A.tw);
  constexpr int groups = N / PYR_SEQ;
  const int p = blockIdx.x / groups;
  const int c0 = (blockIdx.x - p * groups) * PYR_SEQ;
  float2 *base = A.work + (size_t)p * N * N + c0;
  for (int t = threadIdx.x; t < N * PYR_SEQ; t += PYR_THREADS) {
    const int m = t / PYR_SEQ, c = t - m * PYR_SEQ;
    const int yb = m - A.off;
    sm[t] = (yb >= 0 && yb < A.ntot) ? base[(size_t)yb * N + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_ct<N, PYR_SEQ, PYR_THREADS>(sm, tws, true);
  for (int t = threadIdx.x; t < N * PYR_SEQ; t += PYR_THREADS) {
    const int m = t / PYR_SEQ, c = t - m * PYR_SEQ;
    const size_t g = (size_t)(c0 + c) + (size_t)m * N;
    const float2 a = sm[t];
    const float msk = A.submask[g];
    const float2 f = make_float2(a.x * msk, a.y * msk);
    // the focal plane image (compute_pyrfocalplane): abs2_krnl with the point's weight
    if (A.focal_work) A.focal_work[(size_t)p * N * N + g] = A.w[p] * (f.x * f.x + f.y * f.y);
    sm[t] = cmul(f, A.phalfxy[g]);
  }
  __syncthreads();
  fft_ct<N, PYR_SEQ, PYR_THREADS>(sm, tws, false);
  for (int t = threadIdx.x; t < N * PYR_SEQ; t += PYR_THREADS) {
    const int m = t / PYR_SEQ, c = t - m * PYR_SEQ;
    base[(size_t)m * N + c] = sm[t];
  }
}

// 3. per row y: forward transform along x of PYR_SEQ modulation planes at a
//    time, hrimg[y][x] = sum_p w_p |.|^2 in point order (abs2_krnl with the
//    modulation weight).
template <int N>
__global__ void __launch_bounds__(PYR_THREADS) pyr_accum_kernel(PyrArgs A) {
  extern __shared__ float2 sm[];
  float2 *tws = pyr_load_twiddles<N>(sm, A.tw);
  constexpr int ACC = (N + PYR_THREADS - 1) / PYR_THREADS;
  const int y = blockIdx.x;
  float acc[ACC];
#pragma unroll
  for (int j = 0; j < ACC; ++j) acc[j] = 0.f;
  for (int p0 = 0; p0 < A.npts; p0 += PYR_SEQ) {
    const int pb = min(PYR_SEQ, A.npts - p0);
    for (int t = threadIdx.x; t < N * PYR_SEQ; t += PYR_THREADS) {
      const int q = t / N, m = t - q * N;
      sm[m * PYR_SEQ + q] = q < pb ? A.work[((size_t)(p0 + q) * N + y) * N + m] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_ct<N, PYR_SEQ, PYR_THREADS>(sm, tws, false);
#pragma unroll
    for (int j = 0; j < ACC; ++j) {
      const int m = threadIdx.x + j * PYR_THREADS;
      if (m < N)
        for (int q = 0; q < pb; ++q) {
          const float2 v = sm[m * PYR_SEQ + q];
          acc[j] += A.w[p0 + q] * (v.x * v.x + v.y * v.y);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < ACC; ++j) {
    const int m = threadIdx.x + j * PYR_THREADS;
    if (m < N) A.hrimg[(size_t)y * N + m] = acc[j];
  }
}

// The single-image tails below (pixel-transfer convolution and binning) take
// TSEQ sequences per CTA on TSEQ * 64 threads, so one image spreads over
// N / TSEQ CTAs (256 at N = 512, TSEQ = 2) instead of N / PYR_SEQ; each
// sequence's transform is the same whatever the CTA shape.
// 4. pixel transfer function: TSEQ rows of hrimg (real), inverse transform along x.
template <int N, int TSEQ>
__global__ void __launch_bounds__(TSEQ * 64) pyr_conv_rows_kernel(PyrArgs A) {
  constexpr int NT = TSEQ * 64;
  extern __shared__ float2 sm[];
  float2 *tws = sm + N * TSEQ;
  for (int i = threadIdx.x; i < N / 2; i += NT) tws[i] = A.tw[i];
  const int y0 = blockIdx.x * TSEQ;
  for (int t = threadIdx.x; t < N * TSEQ; t += NT) {
    const int c = t / N, i = t - c * N;
    sm[i * TSEQ + c] = make_float2(A.hrimg[(size_t)(y0 + c) * N + i], 0.f);
  }
  __syncthreads();
  fft_ct<N, TSEQ, NT>(sm, tws, true);
  for (int t = threadIdx.x; t < N * TSEQ; t += NT) {
    const int c = t / N, i = t - c * N;
    A.conv[(size_t)(y0 + c) * N + i] = sm[i * TSEQ + c];
  }
}

// 5. columns: inverse transform along y, x sinc, forward transform along y.
template <int N, int TSEQ>
__global__ void __launch_bounds__(TSEQ * 64) pyr_conv_cols_kernel(PyrArgs A) {
  constexpr int NT = TSEQ * 64;
  extern __shared__ float2 sm[];
  float2 *tws = sm + N * TSEQ;
  for (int i = threadIdx.x; i < N / 2; i += NT) tws[i] = A.tw[i];
  const int c0 = blockIdx.x * TSEQ;
  float2 *base = A.conv + c0;
  for (int t = threadIdx.x; t < N * TSEQ; t += NT) {
    const int m = t / TSEQ, c = t - m * TSEQ;
    sm[t] = base[(size_t)m * N + c];
  }
  __syncthreads();
  fft_ct<N, TSEQ, NT>(sm, tws, true);
  for (int t = threadIdx.x; t < N * TSEQ; t += NT) {
    const int m = t / TSEQ, c = t - m * TSEQ;
    const float msk = A.sincar[(size_t)(c0 + c) + (size_t)m * N];
    const float2 a = sm[t];
    sm[t] = make_float2(a.x * msk, a.y * msk);
  }
  __syncthreads();
  fft_ct<N, TSEQ, NT>(sm, tws, false);
  for (int t = threadIdx.x; t < N * TSEQ; t += NT) {
    const int m = t / TSEQ, c = t - m * TSEQ;
    base[(size_t)m * N + c] = sm[t];
  }
}

// 6. rows_per_bin_cta (a multiple of nrebin, <= TSEQ) rows per CTA: forward
//    transform along x, real part, binning (pyr_bimg_krnl order: x offset
//    outer, y offset inner, then / nrebin^2) and the row sums of the binned
//    image for the normalisation.
template <int N, int TSEQ>
__global__ void __launch_bounds__(TSEQ * 64) pyr_bin_kernel(PyrArgs A) {
  constexpr int NT = TSEQ * 64;
  extern __shared__ float2 sm[];
  float2 *tws = sm + N * TSEQ;
  for (int i = threadIdx.x; i < N / 2; i += NT) tws[i] = A.tw[i];
  float *real = reinterpret_cast<float *>(tws + N / 2);  // TSEQ x N
  const int rows = A.rows_per_bin_cta;
  const int y0 = blockIdx.x * rows;
  for (int t = threadIdx.x; t < N * TSEQ; t += NT) {
    const int c = t / N, i = t - c * N;
    sm[i * TSEQ + c] = c < rows ? A.conv[(size_t)(y0 + c) * N + i] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_ct<N, TSEQ, NT>(sm, tws, false);
  for (int t = threadIdx.x; t < N * TSEQ; t += NT) {
    const int c = t / N, i = t - c * N;
    real[c * N + i] = sm[i * TSEQ + c].x;
  }
  __syncthreads();
  const int nbr = rows / A.nrebin;
  const float div = (float)(A.nrebin * A.nrebin);
  for (int t = threadIdx.x; t < nbr * A.nb; t += NT) {
    const int br = t / A.nb, bx = t - br * A.nb;
    float o = 0.f;
    for (int ii = 0; ii < A.nrebin; ++ii)
      for (int jj = 0; jj < A.nrebin; ++jj) o = o + real[(br * A.nrebin + jj) * N + bx * A.nrebin + ii];
    A.binimg[(size_t)(blockIdx.x * nbr + br) * A.nb + bx] = o / div;
  }
  __syncthreads();
  if (threadIdx.x < nbr) {
    const int by = blockIdx.x * nbr + threadIdx.x;
    float sum = 0.f;
    for (int bx = 0; bx < A.nb; ++bx) sum += A.binimg[(size_t)by * A.nb + bx];
    A.partial[by] = sum;
  }
}

// 7. normalisation to nphot (sum of the row sums in row order) and noise.
__global__ void pyr_norm_noise_kernel(float *binimg, const float *partial, int nb, float nphot, int noise_mode,
                                      float noise, uint32_t frame, uint32_t k0, uint32_t k1) {
  __shared__ float s_fact;
  __shared__ float rk[AOB_POISSON_INV_KMAX + 1];
  if (noise_mode >= 1)
    for (int i = threadIdx.x; i <= AOB_POISSON_INV_KMAX; i += blockDim.x) rk[i] = i ? __frcp_rn((float)i) : 0.f;
  if (threadIdx.x < 32) {
    // the row sums in a fixed order: lane-strided partial sums, then a butterfly
    float s = 0.f;
    for (int r = threadIdx.x; r < nb; r += 32) s += partial[r];
    s = warp_sum(s);
    if (threadIdx.x == 0) s_fact = nphot / s;
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

// focal plane: the per-point images summed in point order from zero, as the
// reference accumulates d_pyrfocalplane (sutra_wfs_pyr_pyrhr.cpp:398-401,501-506)
__global__ void pyr_focal_sum_kernel(float *focal, const float *work, int npts, int64_t n2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n2; i += (int64_t)gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int p = 0; p < npts; ++p) acc += work[(size_t)p * n2 + i];
    focal[i] = acc;
  }
}

template <int N, int TSEQ>
static void pyr_launch_tails(const PyrArgs &A, int nbin_ctas, cudaStream_t s) {
  const size_t sm = sizeof(float2) * (N * TSEQ + N / 2);
  const size_t bin_sm = sm + sizeof(float) * N * TSEQ;
  const int lim = (int)std::max<size_t>(bin_sm, 48 * 1024);
  smem_opt_in(reinterpret_cast<const void *>(pyr_conv_rows_kernel<N, TSEQ>), lim);
  smem_opt_in(reinterpret_cast<const void *>(pyr_conv_cols_kernel<N, TSEQ>), lim);
  smem_opt_in(reinterpret_cast<const void *>(pyr_bin_kernel<N, TSEQ>), lim);
  pyr_conv_rows_kernel<N, TSEQ><<<N / TSEQ, TSEQ * 64, sm, s>>>(A);
  AOB_LAUNCH_CHECK("pyr_conv_rows_kernel");
  pyr_conv_cols_kernel<N, TSEQ><<<N / TSEQ, TSEQ * 64, sm, s>>>(A);
  AOB_LAUNCH_CHECK("pyr_conv_cols_kernel");
  pyr_bin_kernel<N, TSEQ><<<nbin_ctas, TSEQ * 64, bin_sm, s>>>(A);
  AOB_LAUNCH_CHECK("pyr_bin_kernel");
}

template <int N>
static void pyr_launch(const PyrArgs &A, int npts, int ntot, int nrebin, cudaStream_t s) {
  const size_t sm = sizeof(float2) * (N * PYR_SEQ + N / 2);
  {
    const int lim = (int)std::max<size_t>(sm, 48 * 1024);
    smem_opt_in(reinterpret_cast<const void *>(pyr_rows_kernel<N>), lim);
    smem_opt_in(reinterpret_cast<const void *>(pyr_cols_kernel<N>), lim);
    smem_opt_in(reinterpret_cast<const void *>(pyr_accum_kernel<N>), lim);
  }
  pyr_rows_kernel<N><<<npts * ((ntot + PYR_SEQ - 1) / PYR_SEQ), PYR_THREADS, sm, s>>>(A);
  AOB_LAUNCH_CHECK("pyr_rows_kernel");
  pyr_cols_kernel<N><<<npts * (N / PYR_SEQ), PYR_THREADS, sm, s>>>(A);
  AOB_LAUNCH_CHECK("pyr_cols_kernel");
  pyr_accum_kernel<N><<<N, PYR_THREADS, sm, s>>>(A);
  AOB_LAUNCH_CHECK("pyr_accum_kernel");
  // tails: as few rows per CTA as the binning allows (rows_per_bin_cta == TSEQ)
  const int nbin_ctas = N / A.rows_per_bin_cta;
  if (A.rows_per_bin_cta <= 2)
    pyr_launch_tails<N, 2>(A, nbin_ctas, s);
  else if (A.rows_per_bin_cta <= 4)
    pyr_launch_tails<N, 4>(A, nbin_ctas, s);
  else
    pyr_launch_tails<N, 8>(A, nbin_ctas, s);
}

}  // namespace aob

using namespace aob;

aob_pyr::aob_pyr(int device_, int nxsub_, int nvalid_, int npix_, int nphase_, int nrebin_, int nfft_, int ntot_,
                 int npts_, float pdiam_, float nphot_, float nphot4imat_)
    : device(device_), nxsub(nxsub_), nvalid(nvalid_), npix(npix_), nphase(nphase_), nrebin(nrebin_), nfft(nfft_),
      ntot(ntot_), npts(npts_), pdiam(pdiam_), nphot(nphot_), nphot4imat(nphot4imat_) {
  AOB_REQUIRE(nvalid > 0 && nrebin > 0 && ntot > 0 && npts > 0, "pyr: sizes must be > 0");
  AOB_REQUIRE(nfft >= 64 && nfft <= 2048 && (nfft & (nfft - 1)) == 0,
              "pyr: nfft must be a power of two in [64, 2048]");
  AOB_REQUIRE(nrebin <= PYR_SEQ && (nrebin & (nrebin - 1)) == 0,
              "pyr: nrebin must be a power of two <= 8 (the binning rows tile nfft)");
  AOB_REQUIRE(ntot <= nfft, "pyr: the phase grid (ntot) must fit in nfft");
  AOB_REQUIRE(nfft % nrebin == 0, "pyr: nfft must be a multiple of nrebin");
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
  // binning rows per CTA: nrebin, at least 2 (a power of two dividing nfft)
  A.rows_per_bin_cta = std::max(nrebin, 2);
  const int64_t n2 = (int64_t)nfft * nfft;
  A.focal_work = nullptr;
  if (compute_focalplane) {
    if (focal_work.n != npts * n2) focal_work.alloc(npts * n2);
    if (focalplane.n != n2) focalplane.alloc(n2);
    A.focal_work = focal_work.p;
  }
  switch (nfft) {
    case 64: pyr_launch<64>(A, npts, ntot, nrebin, s); break;
    case 128: pyr_launch<128>(A, npts, ntot, nrebin, s); break;
    case 256: pyr_launch<256>(A, npts, ntot, nrebin, s); break;
    case 512: pyr_launch<512>(A, npts, ntot, nrebin, s); break;
    case 1024: pyr_launch<1024>(A, npts, ntot, nrebin, s); break;
    default: pyr_launch<2048>(A, npts, ntot, nrebin, s); break;
  }
  if (compute_focalplane) {
    pyr_focal_sum_kernel<<<(int)std::min<int64_t>((n2 + 255) / 256, 8 * num_sms(device)), 256, 0, s>>>(
        focalplane.p, focal_work.p, npts, n2);
    AOB_LAUNCH_CHECK("pyr_focal_sum_kernel");
  }
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
