// Per-sub-aperture Shack-Hartmann image formation, shared by the standalone
// sensor kernel (sh_wfs.cu) and the fused RTC kernel (rtc_fused.cu).
//
// A group of WPS warps owns one sub-aperture: field in shared memory, pruned
// separable DFT at the frequencies binmap reads, |E|^2, binning, flux
// normalisation, Philox-keyed photon/readout noise, cube/image writes and the
// CoG-family centroid.  Every global load a sub-aperture needs is issued at
// the top of the routine, before the first barrier, so that one memory round
// trip (plus the index -> phase dependency) is paid per sub-aperture instead of
// one per stage.
#pragma once

#include "aob_common.cuh"

namespace aob {

constexpr int SH_MAX_PPL = 8;  // binned pixels per warp lane -> npix^2 <= 256

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
  const float2 *twiddle;  // exp(-2 pi i m / nfft), m < nfft
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

// i / d for 0 <= i < 4096 and 0 < d < 256 with magic = floor(2^20 / d) + 1
__device__ __forceinline__ int fdiv(int i, uint32_t magic) { return (int)(((uint32_t)i * magic) >> 20); }

// Named barrier per group of WPS warps (barrier 0 is __syncthreads).
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

// Shared-memory layout: CTA-wide tables, then one scratch area per group.
struct ShSmem {
  size_t hdr, per_grp;
  __host__ __device__ static size_t align16(size_t x) { return (x + 15) & ~size_t(15); }
  __host__ __device__ ShSmem(int nfft, int nu, int nv, int pd, int ncb, int npix2, int wps) {
    hdr = align16(sizeof(float2) * nfft + sizeof(int32_t) * (2 * nfft + ncb) + sizeof(float) * npix2);
    per_grp = align16((size_t)(pd * pd + nu * pd) * sizeof(float2) + (size_t)nu * nv * sizeof(float) +
                      4 * wps * sizeof(float));
  }
  __host__ __device__ size_t bytes(int groups) const { return hdr + per_grp * groups; }
};

// CTA-cooperative load of the tables (caller synchronises afterwards).
template <int NFFT>
__device__ __forceinline__ void sh_load_tables(const ShKernelArgs &P, unsigned char *smem, int tid, int nthreads) {
  float2 *tw = reinterpret_cast<float2 *>(smem);
  int32_t *ul = reinterpret_cast<int32_t *>(tw + NFFT);
  int32_t *vl = ul + NFFT;
  int32_t *cb = vl + NFFT;
  const int npix2 = P.npix * P.npix;
  const int ncb = P.nrebin2 * npix2;
  float *wt = reinterpret_cast<float *>(cb + ncb);
  for (int i = tid; i < NFFT; i += nthreads) tw[i] = P.twiddle[i];
  for (int i = tid; i < P.nu; i += nthreads) ul[i] = P.ulist[i];
  for (int i = tid; i < P.nv; i += nthreads) vl[i] = P.vlist[i];
  for (int i = tid; i < ncb; i += nthreads) cb[i] = P.cbin[i];
  if (P.ckind == 2 && !P.c_wper)
    for (int i = tid; i < npix2; i += nthreads) wt[i] = P.c_weights[i];
}

// One sub-aperture k processed by one group (gt = thread index in the group).
template <int NFFT, int WPS, int PD>
__device__ __forceinline__ void sh_subap(const ShKernelArgs &P, int k, const unsigned char *tables,
                                         unsigned char *scratch, int group, int gt) {
  constexpr int GT = WPS * 32;
  constexpr int PPT = (32 * SH_MAX_PPL) / GT;  // binned pixels per thread
  constexpr int FPT = PD > 0 ? (PD * PD + GT - 1) / GT : 1;
  const int lane = gt & 31, gw = gt >> 5;
  const float2 *tw = reinterpret_cast<const float2 *>(tables);
  const int32_t *ul = reinterpret_cast<const int32_t *>(tw + NFFT);
  const int32_t *vl = ul + NFFT;
  const int32_t *cb = vl + NFFT;
  const int npix2 = P.npix * P.npix;
  const float *wt = reinterpret_cast<const float *>(cb + P.nrebin2 * npix2);
  const int pd = PD > 0 ? PD : P.pdiam;
  const int pd2 = pd * pd;
  float2 *E = reinterpret_cast<float2 *>(scratch);
  float2 *Gt = E + pd2;
  float *I = reinterpret_cast<float *>(Gt + P.nu * pd);
  float *red = I + P.nu * P.nv;
  const uint32_t mg_pd = (1u << 20) / pd + 1, mg_nu = (1u << 20) / P.nu + 1, mg_np = (1u << 20) / P.npix + 1;

  // ---- all per-sub-aperture global loads first ----
  const int px = P.puppixx[k], py = P.puppixy[k];
  const float fk = P.flux[k];
  const int vx = P.validsubsx[k], vy = P.validsubsy[k];
  const int ix = P.c_order ? 2 * k : k;
  const int iy = P.c_order ? 2 * k + 1 : k + P.nvalid;
  float refx = 0.f, refy = 0.f;
  if (P.ckind >= 0 && gt == 0) {
    refx = P.c_ref[ix];
    refy = P.c_ref[iy];
  }
  const uint32_t frame = P.frame_ptr ? *P.frame_ptr : P.frame;
  float wpix[PPT];
  if (P.ckind == 2) {
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      const int p = gt + GT * j;
      wpix[j] = (p < npix2) ? (P.c_wper ? P.c_weights[p + k * npix2] : wt[p]) : 0.f;
    }
  }
  // 1. complex field: pupil * exp(i (phase*2pi/lambda - offset))
  if (PD > 0) {
    float ph[FPT], am[FPT], of[FPT];
#pragma unroll
    for (int j = 0; j < FPT; ++j) {
      const int i = gt + GT * j;
      if (i < pd2) {
        const int y = fdiv(i, mg_pd), x = i - y * pd;
        const int id = (x + px) + (y + py) * P.npup;
        ph[j] = P.phase[id];
        am[j] = P.pupil[id];
        of[j] = P.offsets[i];
      }
    }
#pragma unroll
    for (int j = 0; j < FPT; ++j) {
      const int i = gt + GT * j;
      if (i < pd2) {
        float sn, cs;
        sincosf(ph[j] * P.scale - of[j], &sn, &cs);
        E[i] = make_float2(cs * am[j], sn * am[j]);
      }
    }
  } else {
    for (int i = gt; i < pd2; i += GT) {
      const int y = fdiv(i, mg_pd), x = i - y * pd;
      const int id = (x + px) + (y + py) * P.npup;
      float sn, cs;
      sincosf(P.phase[id] * P.scale - P.offsets[i], &sn, &cs);
      const float a = P.pupil[id];
      E[i] = make_float2(cs * a, sn * a);
    }
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
      float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
      int r = 0;
      for (; r + 3 < P.nrebin2; r += 4) {
        v0 += I[c[r]];
        v1 += I[c[r + 1]];
        v2 += I[c[r + 2]];
        v3 += I[c[r + 3]];
      }
      for (; r < P.nrebin2; ++r) v0 += I[c[r]];
      v = (v0 + v1) + (v2 + v3);
    }
    bv[j] = v;
    part += v;
  }
  const float tot = group_sum<WPS>(part, red, gw, lane, group);
  if (gt == 0) P.intensities[k] = tot;
  // 5. normalise, noise, write cube + image, centroid partial sums
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
      P.binimg[(x + vx) + (y + vy) * P.img_size] = v;
      float d = v;
      if (P.ckind == 1 || P.ckind == 2) d = (v > P.c_thresh) ? v - P.c_thresh : 1.e-6f;
      if (P.ckind == 2) d *= wpix[j];
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
      P.c_slopes[ix] = (cx / (cs + 1.e-6f) - P.c_offset) * P.c_scale - refx;
      P.c_slopes[iy] = (cy / (cs + 1.e-6f) - P.c_offset) * P.c_scale - refy;
      P.c_intens[k] = cs;
    }
  }
  group_sync<WPS>(group);
}

}  // namespace aob
