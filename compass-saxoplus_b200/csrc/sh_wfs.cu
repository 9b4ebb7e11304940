// Shack-Hartmann image formation: one fused kernel per sensor image.
//
// The reference runs eight launches and two memsets per image
// (SutraWfsSH::comp_generic, libsutra/src.cpp/sutra_wfs_sh.cpp:337-589):
// fill the padded Nfft x Nfft field cube (camplipup_krnl, sutra_wfs.cu:27-53),
// batched cuFFT, |E|^2 (abs2c_krnl, sutra_utils.cu:144-168), binning through
// binmap (fillbincube_krnl, sutra_wfs.cu:369-414), per-sub-aperture sum
// (reduce2, sutra_wfs.cu:556-590), normalisation (subapnorm_krnl,
// sutra_utils.cu:170-193), cuRAND Poisson + Gaussian noise, then the image
// scatter (bimg_krnl, sutra_wfs.cu:183-229).  The padded cube (2.5 MB at 40x40)
// is written and re-read several times.
//
// Here one warp owns one sub-aperture from phase to pixels:
//  * the pdiam x pdiam field is built in shared memory (the Nfft^2 - pdiam^2
//    zero padding is never materialised);
//  * the 2-D DFT is evaluated only at the spatial frequencies that binmap
//    reads (an nu x nv subset of the Nfft x Nfft grid, found on the host from
//    binmap), as two separable passes of exact twiddle-table products -- the
//    same transform as the reference's forward cuFFT, pruned on both input
//    and output;
//  * binning, normalisation, Philox-keyed Poisson/readout noise, the bincube
//    and image writes, and (optionally) the CoG/tCoG/wCoG centroid of the
//    sub-aperture happen in registers before the warp moves on.
// HBM traffic per image is the phase and pupil samples read once, the cube,
// image and slopes written once.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "aob_objects.hpp"

namespace aob {

constexpr int SH_WARPS = 4;      // sub-apertures per CTA
constexpr int SH_MAX_PPL = 8;    // binned pixels per lane -> npix^2 <= 256

struct ShKernelArgs {
  const float *phase;
  const float *pupil;
  int npup;
  const int32_t *puppixx;
  const int32_t *puppixy;
  const float *offsets;
  float scale;
  int pdiam, nvalid, npix, nrebin2;
  int nu, nv;
  const int32_t *ulist;
  const int32_t *vlist;
  const int32_t *cbin;  // [nrebin2, npix^2] indexes into the nu x nv intensity tile
  const float *flux;
  float nphot;
  float *bincube;
  float *binimg;
  int img_size;
  const int32_t *validsubsx;
  const int32_t *validsubsy;
  float *intensities;
  int noise_mode;  // 0 none, 1 photon, 2 photon + readout
  float noise;
  uint32_t frame, k0, k1;
  const uint32_t *frame_ptr;  // when set, the frame number is read from device memory
  NoiseTables tables;
  // fused centroider (kind < 0: none)
  int ckind;
  float c_scale, c_offset, c_thresh;
  const float *c_ref;
  const float *c_weights;
  int c_wper;
  int c_order;
  float *c_slopes;
  float *c_intens;
};

// i / d for 0 <= i < 4096 and 0 < d < 256 with magic = ceil(2^20 / d)
__device__ __forceinline__ int fdiv(int i, uint32_t magic) { return (int)(((uint32_t)i * magic) >> 20); }

// Group of WPS warps working on one sub-aperture: named barrier per group
// (barrier 0 is __syncthreads).
template <int WPS>
__device__ __forceinline__ void group_sync(int group) {
  if (WPS == 1)
    __syncwarp();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(group + 1), "r"(WPS * 32) : "memory");
}

// Sum over the group; every thread of the group gets the result.
template <int WPS>
__device__ __forceinline__ float group_sum(float v, float *red, int gw, int lane, int group) {
  v = warp_sum(v);
  if (WPS == 1) return v;
  if (lane == 0) red[gw] = v;
  group_sync<WPS>(group);
  float t = 0.f;
#pragma unroll
  for (int i = 0; i < WPS; ++i) t += red[i];
  group_sync<WPS>(group);
  return t;
}

// PD > 0: phase-grid side known at compile time (the DFT loops unroll and all
// their shared-memory loads issue back to back); PD == 0: runtime side.
template <int NFFT, int WPS, int PD>
__global__ void __launch_bounds__(SH_WARPS * 32, 6) sh_image_kernel(ShKernelArgs P) {
  constexpr int GT = WPS * 32;                // threads per sub-aperture
  constexpr int GROUPS = SH_WARPS / WPS;      // sub-apertures per CTA
  constexpr int PPT = (32 * SH_MAX_PPL) / GT; // binned pixels per thread
  extern __shared__ __align__(16) unsigned char smem[];
  float2 *tw = reinterpret_cast<float2 *>(smem);
  int32_t *ul = reinterpret_cast<int32_t *>(tw + NFFT);
  int32_t *vl = ul + NFFT;
  int32_t *cb = vl + NFFT;
  const int ncb = P.nrebin2 * P.npix * P.npix;
  const int pd = PD > 0 ? PD : P.pdiam;
  const int pd2 = pd * pd;
  const size_t hdr = ((sizeof(float2) * NFFT + sizeof(int32_t) * (2 * NFFT + ncb)) + 15) & ~size_t(15);
  const size_t per_grp = ((size_t)(pd2 + P.nu * pd) * sizeof(float2) + (size_t)P.nu * P.nv * sizeof(float) +
                          4 * WPS * sizeof(float) + 15) & ~size_t(15);

  const int group = threadIdx.x / GT;
  const int gt = threadIdx.x - group * GT;
  const int lane = threadIdx.x & 31;
  const int gw = gt >> 5;  // warp index inside the group
  for (int i = threadIdx.x; i < NFFT; i += blockDim.x) {
    double sn, cs;
    sincospi(2.0 * (double)i / (double)NFFT, &sn, &cs);
    tw[i] = make_float2((float)cs, (float)-sn);  // exp(-2 pi i m / N): forward transform
  }
  for (int i = threadIdx.x; i < P.nu; i += blockDim.x) ul[i] = P.ulist[i];
  for (int i = threadIdx.x; i < P.nv; i += blockDim.x) vl[i] = P.vlist[i];
  for (int i = threadIdx.x; i < ncb; i += blockDim.x) cb[i] = P.cbin[i];
  __syncthreads();

  float2 *E = reinterpret_cast<float2 *>(smem + hdr + per_grp * group);
  float2 *Gt = E + pd2;
  float *I = reinterpret_cast<float *>(Gt + P.nu * pd);
  float *red = I + P.nu * P.nv;
  const int npix2 = P.npix * P.npix;
  const uint32_t mg_pd = (1u << 20) / pd + 1, mg_nu = (1u << 20) / P.nu + 1,
                 mg_np = (1u << 20) / P.npix + 1;

  for (int k = blockIdx.x * GROUPS + group; k < P.nvalid; k += gridDim.x * GROUPS) {
    // 1. complex field of the sub-aperture: pupil * exp(i (phase*2pi/lambda - offset))
    const int px = P.puppixx[k], py = P.puppixy[k];
    for (int i = gt; i < pd2; i += GT) {
      const int y = fdiv(i, mg_pd), x = i - y * pd;
      const int id = (x + px) + (y + py) * P.npup;
      const float ph = P.phase[id] * P.scale - P.offsets[i];
      float sn, cs;
      sincosf(ph, &sn, &cs);
      const float a = P.pupil[id];
      E[i] = make_float2(cs * a, sn * a);
    }
    group_sync<WPS>(group);
    // 2. DFT along x at the needed kx: G[a, y] = sum_x E[x, y] W^(u_a x)
    for (int i = gt; i < P.nu * pd; i += GT) {
      const int y = fdiv(i, mg_nu), a = i - y * P.nu;
      const int ua = ul[a];
      const float2 *e = E + y * pd;
      float re = 0.f, im = 0.f;
#pragma unroll
      for (int x = 0; x < (PD > 0 ? PD : 32); ++x) {
        if (PD == 0 && x >= pd) break;
        const float2 w = tw[(ua * x) & (NFFT - 1)], v = e[x];
        re = fmaf(v.x, w.x, fmaf(-v.y, w.y, re));
        im = fmaf(v.x, w.y, fmaf(v.y, w.x, im));
      }
      Gt[i] = make_float2(re, im);
    }
    group_sync<WPS>(group);
    // 3. DFT along y at the needed ky and |.|^2: I[a, b]
    for (int i = gt; i < P.nu * P.nv; i += GT) {
      const int b = fdiv(i, mg_nu), a = i - b * P.nu;
      const int vb = vl[b];
      float re = 0.f, im = 0.f;
#pragma unroll
      for (int y = 0; y < (PD > 0 ? PD : 32); ++y) {
        if (PD == 0 && y >= pd) break;
        const float2 w = tw[(vb * y) & (NFFT - 1)], v = Gt[a + y * P.nu];
        re = fmaf(v.x, w.x, fmaf(-v.y, w.y, re));
        im = fmaf(v.x, w.y, fmaf(v.y, w.x, im));
      }
      I[i] = fmaf(re, re, im * im);
    }
    group_sync<WPS>(group);
    // 4. binning and per-sub-aperture flux
    float bv[PPT];
    float part = 0.f;
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      const int p = gt + GT * j;
      float v = 0.f;
      if (p < npix2) {
        const int32_t *c = cb + p * P.nrebin2;
        for (int r = 0; r < P.nrebin2; ++r) v += I[c[r]];
      }
      bv[j] = v;
      part += v;
    }
    const float tot = group_sum<WPS>(part, red, gw, lane, group);
    if (gt == 0) P.intensities[k] = tot;
    const float fk = P.flux[k];
    const uint32_t frame = P.frame_ptr ? *P.frame_ptr : P.frame;
    // 5. normalise, noise, write cube + image, centroid partial sums
    const int vx = P.validsubsx[k], vy = P.validsubsy[k];
    float cs = 0.f, cx = 0.f, cy = 0.f;
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      const int p = gt + GT * j;
      if (p < npix2) {
        float v = bv[j];
        if (tot != 0.f) v = v * fk / tot * P.nphot;
        const uint32_t pix = (uint32_t)(p + k * npix2);
        if (P.noise_mode >= 1) v = (float)poisson_sample((double)v, pix, frame, P.k0, P.k1, P.tables);
        if (P.noise_mode >= 2) v = v + P.noise * gauss_sample(pix, frame, P.k0, P.k1);
        P.bincube[pix] = v;
        const int y = fdiv(p, mg_np), x = p - y * P.npix;
        const int idim = (x + vx) + (y + vy) * P.img_size;
        float d = v;
        if (P.ckind == 1 || P.ckind == 2) d = (v > P.c_thresh) ? v - P.c_thresh : 1.e-6f;
        // raw pixels here; the tCoG write-back of thresholded pixels happens when
        // the slopes are collected (aob_centro::get_cog), as in the reference
        P.binimg[idim] = v;
        if (P.ckind == 2) d *= P.c_weights[p + (P.c_wper ? k * npix2 : 0)];
        cs += d;
        cx = fmaf(d, (float)x, cx);
        cy = fmaf(d, (float)y, cy);
      }
    }
    if (P.ckind >= 0) {
      cs = group_sum<WPS>(cs, red + WPS, gw, lane, group);
      cx = group_sum<WPS>(cx, red + 2 * WPS, gw, lane, group);
      cy = group_sum<WPS>(cy, red + 3 * WPS, gw, lane, group);
      if (gt == 0) {
        const int ix = P.c_order ? 2 * k : k;
        const int iy = P.c_order ? 2 * k + 1 : k + P.nvalid;
        P.c_slopes[ix] = (cx / (cs + 1.e-6f) - P.c_offset) * P.c_scale - P.c_ref[ix];
        P.c_slopes[iy] = (cy / (cs + 1.e-6f) - P.c_offset) * P.c_scale - P.c_ref[iy];
        P.c_intens[k] = cs;
      }
    }
    group_sync<WPS>(group);
  }
}

__global__ void sh_fill_image_kernel(float *img, const float *cube, const int32_t *vx,
                                     const int32_t *vy, int npix, int nvalid, int size) {
  const int npix2 = npix * npix;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npix2 * nvalid; t += gridDim.x * blockDim.x) {
    const int k = t / npix2, p = t - k * npix2;
    img[(p % npix + vx[k]) + (p / npix + vy[k]) * size] = cube[t];
  }
}

}  // namespace aob

using namespace aob;

aob_sh::aob_sh(int device_, int nxsub_, int nvalid_, int npix_, int nphase_, int nrebin_, int nfft_,
               int ntot_, int npup_, float pdiam_, float nphot_, float nphot4imat_)
    : device(device_), nxsub(nxsub_), nvalid(nvalid_), npix(npix_), nphase(nphase_), nrebin(nrebin_),
      nfft(nfft_), ntot(ntot_), npup(npup_), pdiam(pdiam_), nphot(nphot_), nphot4imat(nphot4imat_) {
  AOB_REQUIRE(nvalid > 0 && npix > 0 && nphase > 0 && nrebin > 0 && npup > 0, "sh: sizes must be > 0");
  AOB_REQUIRE(nfft == 16 || nfft == 32 || nfft == 64, "sh: nfft must be 16, 32 or 64");
  AOB_REQUIRE(ntot == nfft, "sh: extended field of view (ntot != nfft) is not supported");
  AOB_REQUIRE(nphase <= nfft && nphase <= 32, "sh: nphase must be <= min(nfft, 32)");
  AOB_REQUIRE(npix * npix <= 32 * SH_MAX_PPL, "sh: npix^2 must be <= 256");
  AOB_REQUIRE(nphase * nphase < 4096 && nfft * nfft <= 4096, "sh: sizes beyond the index arithmetic range");
  AOB_REQUIRE((int64_t)nxsub * npix < (1 << 15), "sh: image too large");
  AOB_CUDA(cudaSetDevice(device));
  phase.alloc((int64_t)npup * npup);
  pupil.alloc((int64_t)npup * npup);
  istart.alloc(nvalid);
  jstart.alloc(nvalid);
  validsubsx.alloc(nvalid);
  validsubsy.alloc(nvalid);
  binmap.alloc((int64_t)nrebin * nrebin * npix * npix);
  offsets.alloc((int64_t)nphase * nphase);
  fluxPerSub.alloc(nvalid);
  bincube.alloc((int64_t)npix * npix * nvalid);
  binimg.alloc((int64_t)npix * nxsub * npix * nxsub);
  intensities.alloc(nvalid);
  slopes.alloc(2 * (int64_t)nvalid);
  // noise tables: log(k!) as cumulative sums of log(i), and 1/k (same as the CPU oracle)
  std::vector<double> lf(AOB_LOGFACT_N, 0.0), rkh(AOB_RK_N, 0.0);
  for (int k = 1; k < AOB_LOGFACT_N; ++k) lf[k] = lf[k - 1] + std::log((double)k);
  for (int k = 1; k < AOB_RK_N; ++k) rkh[k] = 1.0 / (double)k;
  logfact.alloc(AOB_LOGFACT_N);
  logfact.upload(lf.data(), AOB_LOGFACT_N);
  rk.alloc(AOB_RK_N);
  rk.upload(rkh.data(), AOB_RK_N);
}

void aob_sh::load_arrays(const int32_t *h_binmap, const float *h_offsets, const float *h_flux,
                         const int32_t *h_vx, const int32_t *h_vy, const int32_t *h_istart,
                         const int32_t *h_jstart) {
  AOB_REQUIRE(h_binmap && h_offsets && h_flux && h_vx && h_vy && h_istart && h_jstart,
              "sh.load_arrays: a required array is NULL");
  AOB_CUDA(cudaSetDevice(device));
  const int nr2 = nrebin * nrebin, np2 = npix * npix;
  const int n2 = nfft * nfft;
  const int img = npix * nxsub;
  for (int i = 0; i < nvalid; ++i) {
    AOB_REQUIRE(h_istart[i] >= 0 && h_jstart[i] >= 0 && h_istart[i] + nphase <= npup &&
                    h_jstart[i] + nphase <= npup,
                "sh.load_arrays: sub-aperture phase window outside the screen");
    AOB_REQUIRE(h_vx[i] >= 0 && h_vy[i] >= 0 && h_vx[i] + npix <= img && h_vy[i] + npix <= img,
                "sh.load_arrays: sub-aperture outside the sensor image");
  }
  // frequencies that binmap reads: kx = m % nfft, ky = m / nfft
  std::vector<int> usex(nfft, -1), usey(nfft, -1);
  for (int i = 0; i < nr2 * np2; ++i) {
    const int m = h_binmap[i];
    AOB_REQUIRE(m >= 0 && m < n2, "sh.load_arrays: binmap entry out of range");
    usex[m % nfft] = 1;
    usey[m / nfft] = 1;
  }
  std::vector<int32_t> U, V;
  for (int i = 0; i < nfft; ++i) {
    if (usex[i] > 0) { usex[i] = (int)U.size(); U.push_back(i); }
    if (usey[i] > 0) { usey[i] = (int)V.size(); V.push_back(i); }
  }
  nu = (int)U.size();
  nv = (int)V.size();
  std::vector<int32_t> C(nr2 * np2);
  for (int i = 0; i < nr2 * np2; ++i) {
    const int m = h_binmap[i];
    C[i] = usex[m % nfft] + usey[m / nfft] * nu;
  }
  ulist.alloc(nu);
  vlist.alloc(nv);
  cbin.alloc((int64_t)nr2 * np2);
  ulist.upload(U.data(), nu);
  vlist.upload(V.data(), nv);
  cbin.upload(C.data(), (int64_t)nr2 * np2);
  binmap.upload(h_binmap, (int64_t)nr2 * np2);
  offsets.upload(h_offsets, (int64_t)nphase * nphase);
  fluxPerSub.upload(h_flux, nvalid);
  validsubsx.upload(h_vx, nvalid);
  validsubsy.upload(h_vy, nvalid);
  istart.upload(h_istart, nvalid);
  jstart.upload(h_jstart, nvalid);
  AOB_REQUIRE(smem_bytes(1) <= 200 * 1024, "sh: shared-memory footprint too large for this geometry");
  loaded = true;
}

size_t aob_sh::smem_bytes(int wps) const {
  const int ncb = nrebin * nrebin * npix * npix;
  const size_t hdr = ((sizeof(float2) * nfft + sizeof(int32_t) * (2 * nfft + ncb)) + 15) & ~size_t(15);
  const size_t per_grp = ((size_t)(nphase * nphase + nu * nphase) * sizeof(float2) + (size_t)nu * nv * sizeof(float) +
                          4 * wps * sizeof(float) + 15) & ~size_t(15);
  return hdr + (SH_WARPS / wps) * per_grp;
}

// Warps per sub-aperture: the autotuner's choice if set, otherwise enough to
// give every SM at least ~24 resident warps.
int aob_sh::pick_wps() const {
  if (wps_override == 1 || wps_override == 2 || wps_override == 4) return wps_override;
  const int nsm = num_sms(device);
  if (nvalid >= 24 * nsm) return 1;
  if (nvalid >= 12 * nsm) return 2;
  return 4;
}

template <int NFFT, int WPS, int PD>
static void launch_sh(const ShKernelArgs &P, int nvalid, size_t sm, int nsm, cudaStream_t s) {
  constexpr int GROUPS = SH_WARPS / WPS;
  int grid = (nvalid + GROUPS - 1) / GROUPS;
  grid = std::max(1, std::min(grid, nsm * 32));
  // the attribute is set once per instantiation (a driver call per launch costs microseconds)
  static size_t configured = 0;
  if (sm > configured) {
    AOB_CUDA(cudaFuncSetAttribute(sh_image_kernel<NFFT, WPS, PD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)std::max<size_t>(sm, 48 * 1024)));
    configured = std::max<size_t>(sm, 48 * 1024);
  }
  sh_image_kernel<NFFT, WPS, PD><<<grid, SH_WARPS * 32, sm, s>>>(P);
}

template <int NFFT, int WPS>
static void launch_sh_pd(int pd, const ShKernelArgs &P, int nvalid, size_t sm, int nsm, cudaStream_t s) {
  switch (pd) {
    case 4: launch_sh<NFFT, WPS, 4>(P, nvalid, sm, nsm, s); break;
    case 6: launch_sh<NFFT, WPS, 6>(P, nvalid, sm, nsm, s); break;
    case 8: launch_sh<NFFT, WPS, 8>(P, nvalid, sm, nsm, s); break;
    default: launch_sh<NFFT, WPS, 0>(P, nvalid, sm, nsm, s); break;
  }
}

template <int NFFT>
static void launch_sh_n(int wps, const ShKernelArgs &P, int nvalid, size_t sm, int nsm, cudaStream_t s) {
  if (wps == 1)
    launch_sh_pd<NFFT, 1>(P.pdiam, P, nvalid, sm, nsm, s);
  else if (wps == 2)
    launch_sh_pd<NFFT, 2>(P.pdiam, P, nvalid, sm, nsm, s);
  else
    launch_sh_pd<NFFT, 4>(P.pdiam, P, nvalid, sm, nsm, s);
}

void aob_sh::comp_image(bool with_noise, cudaStream_t s) { comp_image_to(with_noise, s, nullptr, nullptr); }

void aob_sh::comp_image_to(bool with_noise, cudaStream_t s, float *slopes_dst, const uint32_t *frame_ptr) {
  AOB_REQUIRE(loaded, "sh.comp_image: load_arrays has not been called");
  AOB_CUDA(cudaSetDevice(device));
  ShKernelArgs P{};
  P.phase = phase.p;
  P.pupil = pupil.p;
  P.npup = npup;
  P.puppixx = istart.p;
  P.puppixy = jstart.p;
  P.offsets = offsets.p;
  P.scale = (float)(2.0 * M_PI / (double)lambda_um);
  P.pdiam = nphase;
  P.nvalid = nvalid;
  P.npix = npix;
  P.nrebin2 = nrebin * nrebin;
  P.nu = nu;
  P.nv = nv;
  P.ulist = ulist.p;
  P.vlist = vlist.p;
  P.cbin = cbin.p;
  P.flux = fluxPerSub.p;
  P.nphot = nphot;
  P.bincube = bincube.p;
  P.binimg = binimg.p;
  P.img_size = npix * nxsub;
  P.validsubsx = validsubsx.p;
  P.validsubsy = validsubsy.p;
  P.intensities = intensities.p;
  const float nz = with_noise ? noise : -1.f;
  P.noise_mode = nz > 0 ? 2 : (nz > -1 ? 1 : 0);
  P.noise = nz;
  P.frame = (uint32_t)frame;
  P.k0 = (uint32_t)((uint64_t)seed & 0xffffffffu);
  P.k1 = (uint32_t)((uint64_t)seed >> 32);
  P.frame_ptr = frame_ptr;
  P.tables = NoiseTables{logfact.p, rk.p};
  P.ckind = -1;
  aob_centro *c = fused;
  if (c && c->npix == npix && c->nvalid == nvalid && c->type <= 2 && c->validx.n == nvalid) {
    P.ckind = c->type;
    P.c_scale = c->scale;
    P.c_offset = c->offset;
    P.c_thresh = c->threshold;
    P.c_ref = c->ref.p;
    P.c_weights = c->weights.p;
    P.c_wper = c->weights_per_sub;
    P.c_order = c->order;
    P.c_slopes = slopes_dst ? slopes_dst : c->fused_slopes.p;
    P.c_intens = c->intensities.p;
    if (c->type == 2) AOB_REQUIRE(c->weights.p != nullptr, "wcog: weights not loaded");
  } else {
    c = nullptr;
  }
  const int nsm = num_sms(device);
  const int wps = pick_wps();
  const size_t sm = smem_bytes(wps);
  if (nfft == 16)
    launch_sh_n<16>(wps, P, nvalid, sm, nsm, s);
  else if (nfft == 32)
    launch_sh_n<32>(wps, P, nvalid, sm, nsm, s);
  else
    launch_sh_n<64>(wps, P, nvalid, sm, nsm, s);
  AOB_LAUNCH_CHECK("sh_image_kernel");
  if (P.noise_mode) ++frame;
  ++image_gen;
  if (c && !slopes_dst) {
    c->fused_gen = image_gen;
    c->fused_params_gen = c->params_gen;
  }
}

void aob_sh::fill_binimage(cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  const int n = npix * npix * nvalid;
  sh_fill_image_kernel<<<std::min((n + 255) / 256, 4096), 256, 0, s>>>(
      binimg.p, bincube.p, validsubsx.p, validsubsy.p, npix, nvalid, npix * nxsub);
  AOB_LAUNCH_CHECK("sh_fill_image_kernel");
  ++image_gen;
}
