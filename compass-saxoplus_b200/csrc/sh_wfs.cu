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
// Here one kernel forms the whole image; each CTA takes a batch of
// sub-apertures through the stages of sh_core.cuh with all its threads:
//  * the pdiam x pdiam fields are built in shared memory (the Nfft^2 - pdiam^2
//    zero padding is never materialised);
//  * the 2-D DFT is evaluated only at the spatial frequencies that binmap
//    reads (an nu x nv subset of the Nfft x Nfft grid, found on the host from
//    binmap), as two separable passes of exact twiddle-table products -- the
//    same transform as the reference's forward cuFFT, pruned on both input
//    and output;
//  * binning, normalisation, Philox-keyed Poisson/readout noise, the bincube
//    and image writes, and (optionally) the CoG/tCoG/wCoG centroids follow in
//    shared memory.
// HBM traffic per image is the phase and pupil samples read once, the cube,
// image and slopes written once.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "aob_objects.hpp"
#include "fft.cuh"
#include "sh_core.cuh"

namespace aob {

constexpr int SH_THREADS = 256;  // threads per CTA of the standalone sensor kernel
constexpr int SH_MAX_BATCH = 32;

// PD > 0: phase-grid side known at compile time (the DFT loops unroll and all
// their shared-memory loads issue back to back); PD == 0: runtime side.
// Sub-apertures k = blockIdx.x + (r * S + s) * gridDim.x, s < S, rounds r.
template <int NFFT, int PD, bool FS = false>
__global__ void __launch_bounds__(SH_THREADS) sh_image_kernel(ShKernelArgs P, int S) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int pd = PD > 0 ? PD : P.pdiam;
  const ShSmem L(NFFT, P.nu, P.nv, pd, P.nrebin2 * P.npix * P.npix, P.npix * P.npix, S);
  sh_load_tables<NFFT>(P, smem, threadIdx.x, blockDim.x);
  // (the barrier closing sh_batch's stage 1 publishes the tables: stages 0-1
  // read none of them, so their loads overlap the field's)
  for (int base = blockIdx.x; base < P.nvalid; base += S * gridDim.x) {
    const int Sb = min(S, (P.nvalid - base + (int)gridDim.x - 1) / (int)gridDim.x);
    sh_batch<NFFT, PD, TEAM_CTA, NoHook, false, FS>(P, base, gridDim.x, Sb, smem, smem + L.hdr, L,
                                                    Team{(int)threadIdx.x, (int)blockDim.x, 0});
  }
}

// Field stop (SutraWfsSH::comp_generic with a field stop, sutra_wfs_sh.cpp:366-391):
// pupil * exp(i phase scale) in the top-left npup x npup corner of the n x n
// array (fsamplipup_krnl, sutra_wfs.cu:148-166), zero elsewhere ...
__global__ void fs_fill_kernel(float2 *out, int n, const float *phase, const float *pupil, int npup, float scale) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)n * n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(t % n), y = (int)(t / n);
    float2 v = make_float2(0.f, 0.f);
    if (x < npup && y < npup) {
      const int id = x + y * npup;
      float sn, cs;
      sincosf(phase[id] * scale, &sn, &cs);
      v = make_float2(cs * pupil[id], sn * pupil[id]);
    }
    out[t] = v;
  }
}
// ... and, between the forward and inverse FFTs, the focal-plane mask (submask_krnl, :1868-1876)
__global__ void fs_mask_kernel(float2 *d, const float *mask, int64_t n2) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n2; t += (int64_t)gridDim.x * blockDim.x) {
    const float m = mask[t];
    d[t] = make_float2(d[t].x * m, d[t].y * m);
  }
}

// fakecam (SutraWfsSH::comp_image, sutra_wfs_sh.cpp:623-643, digitalize_krnl,
// libsutra/src.cu/sutra_wfs.cu:2243-2255): the image as a uint16 camera frame,
// min((img * flat + dark) / max_flux_per_pix, 1) * max_pix_value, truncated
// (the float-to-integer conversion saturates at 0 and 65535).
__global__ void digitalize_kernel(uint16_t *cam, const float *img, const float *dark, const float *flat,
                                  int max_flux, int max_pix, int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    float v = (img[t] * flat[t] + dark[t]) / (float)max_flux;
    v = v < 1.f ? v : 1.f;
    cam[t] = (uint16_t)(v * (float)max_pix);
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
  AOB_REQUIRE(ntot >= nfft && ntot <= 4096, "sh: ntot must be in [nfft, 4096]");
  AOB_REQUIRE((int64_t)nrebin * npix <= ntot, "sh: nrebin * npix exceeds the field of view ntot");
  AOB_REQUIRE(nphase <= nfft && nphase <= 32, "sh: nphase must be <= min(nfft, 32)");
  AOB_REQUIRE(npix >= 2 && nphase >= 2, "sh: npix and nphase must be >= 2");
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
  std::vector<float> tw(2 * nfft);
  for (int m = 0; m < nfft; ++m) {
    const double ang = 2.0 * M_PI * (double)m / (double)nfft;
    tw[2 * m] = (float)std::cos(ang);
    tw[2 * m + 1] = (float)-std::sin(ang);  // forward transform: exp(-2 pi i m / nfft)
  }
  twiddle.alloc(2 * nfft);
  twiddle.upload(tw.data(), 2 * nfft);
}

void aob_sh::load_arrays(const int32_t *h_binmap, const float *h_offsets, const float *h_flux,
                         const int32_t *h_vx, const int32_t *h_vy, const int32_t *h_istart,
                         const int32_t *h_jstart, const int32_t *h_hrmap) {
  AOB_REQUIRE(h_binmap && h_offsets && h_flux && h_vx && h_vy && h_istart && h_jstart,
              "sh.load_arrays: a required array is NULL");
  AOB_REQUIRE(ntot == nfft || h_hrmap, "sh.load_arrays: hrmap is required when ntot != nfft");
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
  // Binning map over the nfft x nfft spot.  With an extended field of view
  // (ntot > nfft) the reference writes the spot into an ntot x ntot image at
  // hrmap (indexfill_krnl, libsutra/src.cu/sutra_wfs.cu:462-473; zero elsewhere)
  // and bins that image through binmap (sutra_wfs_sh.cpp:409-481): composed here
  // into one map, where an entry of -1 reads a zero.
  std::vector<int32_t> bm(nr2 * np2);
  if (ntot != nfft) {
    const int64_t nt2 = (int64_t)ntot * ntot;
    std::vector<int32_t> inv(nt2, -1);
    for (int i = 0; i < n2; ++i) {
      AOB_REQUIRE(h_hrmap[i] >= 0 && h_hrmap[i] < nt2, "sh.load_arrays: hrmap entry out of range");
      inv[h_hrmap[i]] = i;
    }
    for (int i = 0; i < nr2 * np2; ++i) {
      AOB_REQUIRE(h_binmap[i] >= 0 && h_binmap[i] < nt2, "sh.load_arrays: binmap entry out of range");
      bm[i] = inv[h_binmap[i]];
    }
  } else {
    for (int i = 0; i < nr2 * np2; ++i) {
      AOB_REQUIRE(h_binmap[i] >= 0 && h_binmap[i] < n2, "sh.load_arrays: binmap entry out of range");
      bm[i] = h_binmap[i];
    }
  }
  // frequencies that the map reads: kx = m % nfft, ky = m / nfft
  std::vector<int> usex(nfft, -1), usey(nfft, -1);
  for (int i = 0; i < nr2 * np2; ++i) {
    const int m = bm[i];
    if (m < 0) continue;
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
  AOB_REQUIRE(nu >= 2 && nv >= 2, "sh.load_arrays: binmap reads fewer than 2 frequencies along an axis");
  std::vector<int32_t> C(nr2 * np2);
  for (int i = 0; i < nr2 * np2; ++i) {
    const int m = bm[i];
    C[i] = m < 0 ? -1 : usex[m % nfft] + usey[m / nfft] * nu;
  }
  // per-geometry twiddles WX[a][x] = W^(U[a] x), WY[b][y] = W^(V[b] y): the same
  // float values as the nfft-point table, gathered so the DFT loops need no index math
  std::vector<float> W(2 * (size_t)(nu + nv) * nphase);
  auto tw = [&](int m, float *out) {
    const double ang = 2.0 * M_PI * (double)(m % nfft) / (double)nfft;
    out[0] = (float)std::cos(ang);
    out[1] = (float)-std::sin(ang);
  };
  for (int a = 0; a < nu; ++a)
    for (int x = 0; x < nphase; ++x) tw(U[a] * x, &W[2 * ((size_t)a * nphase + x)]);
  for (int b = 0; b < nv; ++b)
    for (int y = 0; y < nphase; ++y) tw(V[b] * y, &W[2 * ((size_t)(nu + b) * nphase + y)]);
  wxy.alloc((int64_t)W.size());
  wxy.upload(W.data(), (int64_t)W.size());
  // the shared-memory table image [tw | ulist | vlist | cbin | wxy]
  {
    const ShSmem L(nfft, nu, nv, nphase, nr2 * np2, np2, 1);
    std::vector<unsigned char> img(L.rk, 0);
    std::vector<float> t(2 * nfft);
    for (int m = 0; m < nfft; ++m) tw(m, &t[2 * m]);
    std::memcpy(img.data(), t.data(), sizeof(float) * 2 * nfft);
    std::memcpy(img.data() + sizeof(float) * 2 * nfft, U.data(), sizeof(int32_t) * nu);
    std::memcpy(img.data() + sizeof(float) * 2 * nfft + sizeof(int32_t) * nfft, V.data(), sizeof(int32_t) * nv);
    std::memcpy(img.data() + sizeof(float) * 2 * nfft + sizeof(int32_t) * 2 * nfft, C.data(), sizeof(int32_t) * C.size());
    std::memcpy(img.data() + L.wxy, W.data(), sizeof(float) * W.size());
    tblob.alloc((int64_t)(L.rk / 16));
    AOB_CUDA(cudaMemcpy(tblob.p, img.data(), L.rk, cudaMemcpyHostToDevice));
  }
  ulist.alloc(nu);
  vlist.alloc(nv);
  cbin.alloc((int64_t)nr2 * np2);
  ulist.upload(U.data(), nu);
  vlist.upload(V.data(), nv);
  cbin.upload(C.data(), (int64_t)nr2 * np2);
  binmap.upload(h_binmap, (int64_t)nr2 * np2);
  if (ntot != nfft) {
    hrmap.alloc(n2);
    hrmap.upload(h_hrmap, n2);
  }
  offsets.upload(h_offsets, (int64_t)nphase * nphase);
  fluxPerSub.upload(h_flux, nvalid);
  validsubsx.upload(h_vx, nvalid);
  validsubsy.upload(h_vy, nvalid);
  istart.upload(h_istart, nvalid);
  jstart.upload(h_jstart, nvalid);
  AOB_REQUIRE(smem_bytes(1) <= 200 * 1024, "sh: shared-memory footprint too large for this geometry");
  loaded = true;
}

size_t aob_sh::smem_bytes(int batch) const {
  const ShSmem L(nfft, nu, nv, nphase, nrebin * nrebin * npix * npix, npix * npix, batch);
  return L.bytes();
}

// Sub-apertures per CTA: the autotuner's choice if set, otherwise enough for
// about two CTAs per SM in a single wave.
int aob_sh::pick_batch() const {
  int b = batch_override > 0 ? batch_override : (nvalid + 2 * num_sms(device) - 1) / (2 * num_sms(device));
  b = std::max(1, std::min(b, SH_MAX_BATCH));
  while (b > 1 && smem_bytes(b) > 200 * 1024) --b;
  return b;
}

template <int NFFT, int PD, bool FS>
static void launch_sh_fs(const ShKernelArgs &P, int nvalid, int S, size_t sm, cudaStream_t s) {
  const int grid = std::max(1, (nvalid + S - 1) / S);
  // opt-in per (kernel, device), only ever raised (a driver call per launch costs microseconds)
  smem_opt_in(reinterpret_cast<const void *>(sh_image_kernel<NFFT, PD, FS>), (int)std::max<size_t>(sm, 48 * 1024));
  sh_image_kernel<NFFT, PD, FS><<<grid, SH_THREADS, sm, s>>>(P, S);
}
template <int NFFT, int PD>
static void launch_sh(const ShKernelArgs &P, int nvalid, int S, size_t sm, cudaStream_t s) {
  if (P.fs_field)
    launch_sh_fs<NFFT, PD, true>(P, nvalid, S, sm, s);
  else
    launch_sh_fs<NFFT, PD, false>(P, nvalid, S, sm, s);
}

template <int NFFT>
static void launch_sh_pd(const ShKernelArgs &P, int nvalid, int S, size_t sm, cudaStream_t s) {
  switch (P.pdiam) {
    case 4: launch_sh<NFFT, 4>(P, nvalid, S, sm, s); break;
    case 6: launch_sh<NFFT, 6>(P, nvalid, S, sm, s); break;
    case 8: launch_sh<NFFT, 8>(P, nvalid, S, sm, s); break;
    default: launch_sh<NFFT, 0>(P, nvalid, S, sm, s); break;
  }
}

void aob_sh::comp_image(bool with_noise, cudaStream_t s) { comp_image_to(with_noise, s, nullptr, nullptr); }

aob_centro *aob_sh::make_args(bool with_noise, float *slopes_dst, const uint32_t *frame_ptr, ShKernelArgs &P) {
  AOB_REQUIRE(loaded, "sh.comp_image: load_arrays has not been called");
  P = ShKernelArgs{};
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
  P.twiddle = reinterpret_cast<const float2 *>(twiddle.p);
  P.tblob = tblob.p;
  P.wxy = reinterpret_cast<const float2 *>(wxy.p);
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
  P.mg_pd = udiv_magic((uint32_t)nphase);
  P.mg_pd2 = udiv_magic((uint32_t)(nphase * nphase));
  P.mg_nu = udiv_magic((uint32_t)nu);
  P.mg_nupd = udiv_magic((uint32_t)(nu * nphase));
  P.mg_nunv = udiv_magic((uint32_t)(nu * nv));
  P.mg_np = udiv_magic((uint32_t)npix);
  P.mg_np2 = udiv_magic((uint32_t)(npix * npix));
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
    return c;
  }
  return nullptr;
}

// Host-side bookkeeping after an image was launched with make_args' arguments.
void aob_sh::after_image(const ShKernelArgs &P, aob_centro *c, bool staged) {
  if (P.noise_mode) ++frame;
  ++image_gen;
  if (c && staged) {
    c->fused_gen = image_gen;
    c->fused_params_gen = c->params_gen;
  }
}

void aob_sh::set_field_stop(const float *mask, int n) {
  AOB_CUDA(cudaSetDevice(device));
  if (!mask || n == 0) {
    fs_n = 0;
    fs_mask.release();
    fs_field.release();
    return;
  }
  AOB_REQUIRE(n >= 8 && n <= 2048 && (n & (n - 1)) == 0, "sh.set_field_stop: n must be a power of two in [8, 2048]");
  AOB_REQUIRE(n >= npup, "sh.set_field_stop: the field-stop plane must hold the npup x npup screen");
  fs_mask.alloc((int64_t)n * n);
  fs_mask.upload(mask, (int64_t)n * n);
  fs_field.alloc(2 * (int64_t)n * n);
  fs_n = n;
}

// The filtered full-pupil field of the current phase (field stop).
void aob_sh::field_stop_prepare(cudaStream_t s) {
  const int64_t n2 = (int64_t)fs_n * fs_n;
  const int grid = (int)std::min<int64_t>((n2 + 255) / 256, 8192);
  float2 *f = reinterpret_cast<float2 *>(fs_field.p);
  fs_fill_kernel<<<grid, 256, 0, s>>>(f, fs_n, phase.p, pupil.p, npup, (float)(2.0 * M_PI / (double)lambda_um));
  AOB_LAUNCH_CHECK("fs_fill_kernel");
  fft2d(f, fs_n, 1, false, device, s);
  fs_mask_kernel<<<grid, 256, 0, s>>>(f, fs_mask.p, n2);
  AOB_LAUNCH_CHECK("fs_mask_kernel");
  fft2d(f, fs_n, 1, true, device, s);
}

void aob_sh::comp_image_to(bool with_noise, cudaStream_t s, float *slopes_dst, const uint32_t *frame_ptr) {
  AOB_CUDA(cudaSetDevice(device));
  ShKernelArgs P;
  aob_centro *c = make_args(with_noise, slopes_dst, frame_ptr, P);
  if (fs_n) {
    field_stop_prepare(s);
    P.fs_field = reinterpret_cast<const float2 *>(fs_field.p);
    P.fs_n = fs_n;
    P.fs_inv = 1.f / ((float)fs_n * (float)fs_n);  // exact: fs_n is a power of two
  }
  const int S = pick_batch();
  const size_t sm = smem_bytes(S);
  if (nfft == 16)
    launch_sh_pd<16>(P, nvalid, S, sm, s);
  else if (nfft == 32)
    launch_sh_pd<32>(P, nvalid, S, sm, s);
  else
    launch_sh_pd<64>(P, nvalid, S, sm, s);
  AOB_LAUNCH_CHECK("sh_image_kernel");
  after_image(P, c, slopes_dst == nullptr);
  if (fakecam) digitalize(s);
}

void aob_sh::set_fakecam(int enable, int max_flux, int max_pix) {
  AOB_REQUIRE(!enable || (max_flux > 0 && max_pix > 0 && max_pix <= 65535),
              "sh.set_fakecam: max_flux_per_pix > 0 and 0 < max_pix_value <= 65535 required");
  AOB_CUDA(cudaSetDevice(device));
  fakecam = enable ? 1 : 0;
  max_flux_per_pix = max_flux;
  max_pix_value = max_pix;
  const int64_t n = binimg.n;
  if (fakecam && camimg.n != n) {
    camimg.alloc(n);
    if (cam_dark.n != n) cam_dark.alloc(n);  // dark 0 (reset), flat 1 (sutra_wfs_sh.cpp:100-104)
    if (cam_flat.n != n) {
      cam_flat.alloc(n);
      std::vector<float> one(n, 1.f);
      cam_flat.upload(one.data(), n);
    }
  }
}

void aob_sh::digitalize(cudaStream_t s) {
  const int64_t n = binimg.n;
  digitalize_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, s>>>(
      camimg.p, binimg.p, cam_dark.p, cam_flat.p, max_flux_per_pix, max_pix_value, n);
  AOB_LAUNCH_CHECK("digitalize_kernel");
}

void aob_sh::fill_binimage(cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  const int n = npix * npix * nvalid;
  sh_fill_image_kernel<<<std::min((n + 255) / 256, 4096), 256, 0, s>>>(
      binimg.p, bincube.p, validsubsx.p, validsubsy.p, npix, nvalid, npix * nxsub);
  AOB_LAUNCH_CHECK("sh_fill_image_kernel");
  ++image_gen;
}
