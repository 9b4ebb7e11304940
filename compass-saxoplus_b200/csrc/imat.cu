// Interaction matrix of a DM seen by a SH sensor, every actuator poked in one
// batch.
//
// The reference's SutraRtc::do_imat (libsutra/src.cpp/sutra_rtc.cpp:150-292)
// loops over the actuators: comp_oneactu (push), raytrace to the sensor,
// comp_image, do_centroids, then the same with the pull, and the column
// (s_push - s_pull) / (2 push).  Here the 2 nact pokes of a chunk go through
// four launches in total: the single-actuator DM shapes (the pixel-major CSR
// gather with one non-zero command), the bilinear raytrace of each onto the
// sensor's phase grid, ONE sensor launch over all pokes' sub-apertures with the
// attached centroider fused (grid.y = poke; no cube or image is written), and
// the push-pull difference into the matrix.  Every step has the arithmetic of
// the corresponding separate call, so the matrix equals the poke-by-poke one
// bit for bit.

#include <algorithm>

#include "aob_objects.hpp"
#include "sh_core.cuh"
#include "sim.hpp"

namespace aob {

// poke j of the chunk: actuator a0 + j / 2, command +push (j even) or -push (odd)
__global__ void imat_dm_kernel(float *shapes, int64_t npix, const int32_t *rowptr, const int32_t *act,
                               const float *w, int a0, float push) {
  const int j = blockIdx.y;
  const int a = a0 + j / 2;
  const float c = (j & 1) ? -push : push;
  float *out = shapes + (int64_t)j * npix;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npix; p += (int64_t)gridDim.x * blockDim.x) {
    float v = 0.f;  // (the other actuators' zero commands add nothing)
    for (int k = rowptr[p]; k < rowptr[p + 1]; ++k)
      if (act[k] == a) v += c * w[k];
    out[p] = v;
  }
}

// the raytrace of one DM shape per poke (raytrace_kernel with one source, reset)
__global__ void imat_trace_kernel(float *phases, int nx, const float *shapes, int N, float xoff, float yoff) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int j = blockIdx.z;
  if (x >= nx || y >= nx) return;
  const float *d = shapes + (int64_t)j * N * N;
  float acc = 0.f;
  const float xref = (float)x - nx / 2.0f + nx / 2.0f + xoff;
  const float yref = (float)y - nx / 2.0f + nx / 2.0f + yoff;
  const int iref = (int)xref, jref = (int)yref;
  const float xs = xref - iref, ys = yref - jref;
  const float wx1 = 1.0f - xs, wx2 = xs, wy1 = 1.0f - ys, wy2 = ys;
  if (iref + 1 < N && jref + 1 < N) {
    acc += (wx1 * wy1 * d[iref + jref * N] + wx2 * wy1 * d[iref + 1 + jref * N] +
            wx1 * wy2 * d[iref + (jref + 1) * N] + wx2 * wy2 * d[iref + 1 + (jref + 1) * N]);
  } else {
    acc += 0.0f;
  }
  phases[(int64_t)j * nx * nx + x + y * nx] = acc;
}

// The sensor over all pokes: CTA (x, y) takes sub-aperture batch x of poke y,
// with the poke's phase, slopes and intensities.
constexpr int IMAT_SH_THREADS = 256;
template <int NFFT, int PD>
__global__ void __launch_bounds__(IMAT_SH_THREADS)
    imat_sh_kernel(ShKernelArgs P, int S, int64_t phase_stride, int nslope) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ ShKernelArgs Q;
  if (threadIdx.x == 0) {
    Q = P;
    const int j = blockIdx.y;
    Q.phase = P.phase + (int64_t)j * phase_stride;
    Q.c_slopes = P.c_slopes + (int64_t)j * nslope;
    Q.intensities = P.intensities + (int64_t)j * P.nvalid;
    Q.c_intens = Q.intensities;
  }
  __syncthreads();
  const int pd = PD > 0 ? PD : Q.pdiam;
  const ShSmem L(NFFT, Q.nu, Q.nv, pd, Q.nrebin2 * Q.npix * Q.npix, Q.npix * Q.npix, S);
  sh_load_tables<NFFT>(Q, smem, threadIdx.x, blockDim.x);
  for (int base = blockIdx.x; base < Q.nvalid; base += S * gridDim.x) {
    const int Sb = min(S, (Q.nvalid - base + (int)gridDim.x - 1) / (int)gridDim.x);
    sh_batch<NFFT, PD>(Q, base, gridDim.x, Sb, smem, smem + L.hdr, L, Team{(int)threadIdx.x, (int)blockDim.x, 0});
  }
}

__global__ void imat_diff_kernel(float *imat, const float *slopes, int nslope, int a0, int count, float push) {
  const int64_t n = (int64_t)nslope * count;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t / nslope), s = (int)(t - (int64_t)i * nslope);
    const float sp = slopes[(int64_t)(2 * i) * nslope + s], sm = slopes[(int64_t)(2 * i + 1) * nslope + s];
    imat[s + (int64_t)(a0 + i) * nslope] = (sp - sm) / (2.f * push);
  }
}

template <int NFFT, int PD>
static void launch_imat_sh(const ShKernelArgs &P, int nvalid, int S, size_t sm, int npoke, int64_t stride,
                           int nslope, cudaStream_t s) {
  const int gx = std::max(1, (nvalid + S - 1) / S);
  smem_opt_in(reinterpret_cast<const void *>(imat_sh_kernel<NFFT, PD>), (int)std::max<size_t>(sm, 48 * 1024));
  imat_sh_kernel<NFFT, PD><<<dim3(gx, npoke), IMAT_SH_THREADS, sm, s>>>(P, S, stride, nslope);
}
template <int NFFT>
static void launch_imat_sh_pd(const ShKernelArgs &P, int nvalid, int S, size_t sm, int npoke, int64_t stride,
                              int nslope, cudaStream_t s) {
  switch (P.pdiam) {
    case 4: launch_imat_sh<NFFT, 4>(P, nvalid, S, sm, npoke, stride, nslope, s); break;
    case 6: launch_imat_sh<NFFT, 6>(P, nvalid, S, sm, npoke, stride, nslope, s); break;
    case 8: launch_imat_sh<NFFT, 8>(P, nvalid, S, sm, npoke, stride, nslope, s); break;
    default: launch_imat_sh<NFFT, 0>(P, nvalid, S, sm, npoke, stride, nslope, s); break;
  }
}

}  // namespace aob

using namespace aob;

extern "C" int aob_imat_build(aob_sh *w, aob_centro *c, aob_dm *dm, float xoff, float yoff, float push, int chunk,
                              float *dev_imat, void *stream) {
  try {
    if (!w || !c || !dm || !dev_imat) throw Error("aob_imat_build: null handle or pointer");
    AOB_REQUIRE(w->device == c->device && w->device == dm->device, "aob_imat_build: objects on different devices");
    AOB_REQUIRE(push != 0.f, "aob_imat_build: push must be non-zero");
    AOB_REQUIRE(!w->fs_n, "aob_imat_build: sensors with a field stop are not supported");
    AOB_CUDA(cudaSetDevice(w->device));
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    ShKernelArgs P;
    aob_centro *fc = w->make_args(false, nullptr, nullptr, P);
    AOB_REQUIRE(fc == c, "aob_imat_build: attach the CoG-family centroider to the sensor first");
    // the reference forms the calibration images with nphot4imat photons
    // (SutraRtc::comp_images_imat, sutra_rtc.cpp:380-395); 0 keeps nphot
    if (w->nphot4imat > 0.f) P.nphot = w->nphot4imat;
    const int nact = dm->nact, nslope = 2 * w->nvalid;
    const int per = chunk > 0 ? std::min(chunk, nact) : nact;
    AOB_REQUIRE(2 * (int64_t)per <= 65535, "aob_imat_build: at most 32767 actuators per chunk");
    const int64_t npix = (int64_t)dm->dim * dm->dim, nphase = (int64_t)w->npup * w->npup;
    DevBuf<float> shapes(2 * per * npix), phases(2 * per * nphase), slopes(2 * (int64_t)per * nslope),
        inten(2 * (int64_t)per * w->nvalid);
    const int S = w->pick_batch();
    const size_t sm = w->smem_bytes(S);
    P.bincube = nullptr;  // slopes only
    P.binimg = nullptr;
    P.phase = phases.p;
    P.c_slopes = slopes.p;
    P.intensities = inten.p;
    for (int a0 = 0; a0 < nact; a0 += per) {
      const int cnt = std::min(per, nact - a0), npoke = 2 * cnt;
      const int gx = (int)std::min<int64_t>((npix + 255) / 256, 1024);
      imat_dm_kernel<<<dim3(gx, npoke), 256, 0, s>>>(shapes.p, npix, dm->rowptr.p, dm->actidx.p, dm->weight.p, a0,
                                                      push);
      AOB_LAUNCH_CHECK("imat_dm_kernel");
      const dim3 tb(16, 16), tg((w->npup + 15) / 16, (w->npup + 15) / 16, npoke);
      imat_trace_kernel<<<tg, tb, 0, s>>>(phases.p, w->npup, shapes.p, dm->dim, xoff, yoff);
      AOB_LAUNCH_CHECK("imat_trace_kernel");
      if (w->nfft == 16)
        launch_imat_sh_pd<16>(P, w->nvalid, S, sm, npoke, nphase, nslope, s);
      else if (w->nfft == 32)
        launch_imat_sh_pd<32>(P, w->nvalid, S, sm, npoke, nphase, nslope, s);
      else
        launch_imat_sh_pd<64>(P, w->nvalid, S, sm, npoke, nphase, nslope, s);
      AOB_LAUNCH_CHECK("imat_sh_kernel");
      const int64_t nd = (int64_t)nslope * cnt;
      imat_diff_kernel<<<(int)std::min<int64_t>((nd + 255) / 256, 4096), 256, 0, s>>>(dev_imat, slopes.p, nslope, a0,
                                                                                      cnt, push);
      AOB_LAUNCH_CHECK("imat_diff_kernel");
    }
    // the scratch is released below: wait for the launches that read it
    AOB_CUDA(cudaStreamSynchronize(s));
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}
