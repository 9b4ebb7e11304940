// Shack-Hartmann image formation for a batch of sub-apertures, shared by the
// standalone sensor kernel (sh_wfs.cu), the fused RTC kernel (rtc_fused.cu)
// and the batched Monte Carlo kernel (batch.cu).
//
// A team of threads -- the whole CTA, or a group of its warps synchronised by
// a named barrier, or one warp -- works on the whole batch at once, stage by
// stage:
//   0. per-sub-aperture metadata (phase window, flux, image position, refs)
//   1. complex field  pupil * exp(i (phase * 2 pi / lambda - offset))
//   2. DFT along x at the nu frequencies binmap reads
//   3. DFT along y at the nv frequencies binmap reads, |.|^2
//   4. binning through the compact binmap, the flux per sub-aperture (one
//      warp per sub-aperture, fixed summation order) and normalisation
//   5. Philox photon / readout noise, centroid weights
//   6. CoG-family centroid per sub-aperture (one warp each, fixed order),
//      then that sub-aperture's cube block and image window, coalesced
//      (or, for a caller that wants the slopes out first, later through
//      sh_store_images)
// so a team pays each stage's latency once for the batch instead of once per
// sub-aperture; small teams (one warp) meet only at warp barriers and run
// independently of the CTA's other teams.  The reductions run in an order
// that does not depend on the batch size or the team size: every kernel gives
// bit-identical images and slopes.
#pragma once

#include "aob_common.cuh"

namespace aob {

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
  const int4 *tblob;      // twiddles, ulist, vlist, cbin and wxy in their shared-memory layout
  const float2 *twiddle;  // exp(-2 pi i m / nfft), m < nfft
  const int32_t *ulist;
  const int32_t *vlist;
  const int32_t *cbin;  // [nrebin2, npix^2] indexes into the nu x nv intensity tile
  const float2 *wxy;    // per-geometry twiddles: WX[a][x] (nu x pdiam) then WY[b][y] (nv x pdiam)
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
  // field stop: the filtered full-pupil field (fs_n x fs_n complex) read in place
  // of the phase and pupil, scaled by fs_inv = 1 / fs_n^2 (sh_batch<..., FS = true>)
  const float2 *fs_field;
  int fs_n;
  float fs_inv;
  // magic multipliers for the runtime divisions (see udiv)
  uint32_t mg_pd, mg_pd2, mg_nu, mg_nupd, mg_nunv, mg_np, mg_np2;
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

// i / d for i * d < 2^32 with magic = floor(2^32 / d) + 1 (d >= 2).
__host__ __device__ inline uint32_t udiv_magic(uint32_t d) {
  return (uint32_t)((0x100000000ull / (uint64_t)d) + 1ull);
}
__device__ __forceinline__ int udiv(int i, uint32_t magic) { return (int)__umulhi((uint32_t)i, magic); }

// Shared-memory layout: CTA-wide tables, then the batch work area.
// Tables: [tw | ulist | vlist | cbin | wxy | 1/k | wCoG weights]; everything
// before the 1/k table is one contiguous image per sensor (ShKernelArgs::tblob).
struct ShSmem {
  size_t wxy, rk, wt, hdr;                      // table offsets, header size
  size_t meta, E, Gt, I, bins, dw, ord, per_batch;  // offsets within a team's work area
  __host__ __device__ static size_t align16(size_t x) { return (x + 15) & ~size_t(15); }
  __host__ __device__ ShSmem(int nfft, int nu, int nv, int pd, int ncb, int npix2, int S) {
    wxy = align16(sizeof(float2) * nfft + sizeof(int32_t) * (2 * nfft + ncb));
    rk = align16(wxy + sizeof(float2) * (size_t)(nu + nv) * pd);
    wt = align16(rk + sizeof(float) * (AOB_POISSON_INV_KMAX + 1));
    hdr = align16(wt + sizeof(float) * npix2);
    size_t o = 0;
    meta = o;  // 8 values per sub-aperture, then the team's two pixel counters
    o += align16(sizeof(int32_t) * (8 * (size_t)S + 2));
    E = o;
    o += align16(sizeof(float2) * (size_t)S * pd * pd);
    Gt = o;
    o += align16(sizeof(float2) * (size_t)S * nu * pd);
    I = o;
    o += align16(sizeof(float) * (size_t)S * nu * nv);
    bins = o;
    o += align16(sizeof(float) * (size_t)S * npix2);
    dw = o;
    o += align16(sizeof(float) * (size_t)S * npix2);
    ord = o;
    o += align16(sizeof(int32_t) * (size_t)S * npix2);
    per_batch = o;
  }
  __host__ __device__ size_t bytes() const { return hdr + per_batch; }
  // tables plus one work area per team
  __host__ __device__ size_t team_bytes(int nteams) const { return hdr + (size_t)nteams * per_batch; }
};

// A team of threads that runs sh_batch together: nt threads (a multiple of
// 32) with team-relative index tid, synchronised according to its kind (a
// compile-time parameter): the whole CTA (__syncthreads), one warp
// (__syncwarp, nt = 32) or named barrier ``bar`` (1..15) over nt threads.
enum : int { TEAM_CTA = 0, TEAM_WARP = 1, TEAM_NAMED = 2 };
struct Team {
  int tid, nt, bar;
};
template <int TK>
__device__ __forceinline__ void team_sync(const Team &t) {
  if constexpr (TK == TEAM_WARP)
    __syncwarp();
  else if constexpr (TK == TEAM_CTA)
    __syncthreads();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(t.bar), "r"(t.nt) : "memory");
}

// The bulk-copyable part of the tables: the table image (ShSmem::rk bytes at
// offset 0) and, when its size and address allow a bulk copy (16-byte
// multiple and alignment), the shared wCoG weights (wt_bytes at ShSmem::wt).
struct ShTableCopy {
  uint32_t image_bytes, wt_bytes;
  __device__ ShTableCopy(const ShKernelArgs &P, const ShSmem &L) {
    const int npix2 = P.npix * P.npix;
    image_bytes = (uint32_t)L.rk;
    const bool wt = P.ckind == 2 && !P.c_wper && (npix2 * 4) % 16 == 0 &&
                    (reinterpret_cast<uintptr_t>(P.c_weights) & 15) == 0;
    wt_bytes = wt ? (uint32_t)(npix2 * 4) : 0u;
  }
};

// CTA-cooperative load of the tables (caller synchronises afterwards): the
// sensor's table image with 16-byte loads (one page, one request per
// thread), the wCoG weights and the 1/k table of the Poisson sampler.
// image_done / wt_done: those parts already arrive by bulk copy.
template <int NFFT>
__device__ __forceinline__ void sh_load_tables(const ShKernelArgs &P, unsigned char *smem, int tid, int nthreads,
                                               bool image_done = false, bool wt_done = false) {
  const int npix2 = P.npix * P.npix;
  const ShSmem L(NFFT, P.nu, P.nv, P.pdiam, P.nrebin2 * npix2, npix2, 1);
  int4 *dst = reinterpret_cast<int4 *>(smem);
  if (!image_done)
    for (int i = tid; i < (int)(L.rk / 16); i += nthreads) dst[i] = __ldg(P.tblob + i);
  if (P.ckind == 2 && !P.c_wper && !wt_done) {
    float *wt = reinterpret_cast<float *>(smem + L.wt);
    for (int i = tid; i < npix2; i += nthreads) wt[i] = __ldg(P.c_weights + i);
  }
  if (P.noise_mode >= 1) {
    float *rk = reinterpret_cast<float *>(smem + L.rk);
    for (int i = tid; i <= AOB_POISSON_INV_KMAX; i += nthreads) rk[i] = i ? __frcp_rn((float)i) : 0.f;
  }
}

struct NoHook {
  __device__ void operator()() const {}
};

// Where sh_batch keeps the batch's metadata in its work area.
struct ShMeta {
  int32_t *vx, *vy;
  float *fl, *tot, *rx, *ry;
  int *n_listed;  // pixels listed for inversion / PTRS in stage 4
  __device__ ShMeta(unsigned char *work, const ShSmem &L, int S) {
    vx = reinterpret_cast<int32_t *>(work + L.meta) + 2 * S;
    vy = vx + S;
    fl = reinterpret_cast<float *>(vy + S);
    tot = fl + S;
    rx = tot + S;
    ry = rx + S;
    n_listed = reinterpret_cast<int *>(ry + S);
  }
};

// One warp writes sub-aperture k's pixels bs[0 .. npix^2): its block of the
// cube (contiguous) and its npix x npix window of the binned image.
__device__ __forceinline__ void sh_store_subap(const ShKernelArgs &P, int k, const float *bs, int vx, int vy,
                                               int lane) {
  if (!P.bincube) return;  // (slopes only: the batched interaction-matrix images keep no cube or image)
  const int npix = P.npix, npix2 = npix * npix;
  for (int p = lane; p < npix2; p += 32) {
    const float v = bs[p];
    P.bincube[p + k * npix2] = v;
    const int y = udiv(p, P.mg_np), x = p - y * npix;
    P.binimg[(x + vx) + (y + vy) * P.img_size] = v;
  }
}

// The image writes of a batch that sh_batch<..., DEFER_IMG = true> left in
// its work area (same team, same arguments); the work area must be intact.
template <int TK = TEAM_CTA>
__device__ __forceinline__ void sh_store_images(const ShKernelArgs &P, int base, int stride, int S,
                                                unsigned char *work, const ShSmem &L, const Team &T) {
  const int tid = TK == TEAM_CTA ? (int)threadIdx.x : T.tid;
  const int nt = TK == TEAM_CTA ? (int)blockDim.x : (TK == TEAM_WARP ? 32 : T.nt);
  const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const ShMeta M(work, L, S);
  const float *bins = reinterpret_cast<const float *>(work + L.bins);
  const int npix2 = P.npix * P.npix;
  for (int s = warp; s < S; s += nw) sh_store_subap(P, base + s * stride, bins + s * npix2, M.vx[s], M.vy[s], lane);
}

// Sub-apertures k = base + s * stride for s < S, processed by team T.  Must
// be called by every thread of the team (it synchronises the team
// internally); the caller guarantees base + (S - 1) * stride < nvalid.  On
// return the team's work area may be reused.  ``after_field`` runs on every
// thread of the team once the field stage is complete (its global loads have
// returned), before the DFTs.  With DEFER_IMG the cube and image writes are
// left to sh_store_images (the noisy pixels stay in the work area).
template <int NFFT, int PD, int TK = TEAM_CTA, class Hook = NoHook, bool DEFER_IMG = false, bool FS = false>
__device__ __forceinline__ void sh_batch(const ShKernelArgs &P, int base, int stride, int S,
                                         const unsigned char *tables, unsigned char *work, const ShSmem &L,
                                         const Team &T, const Hook &after_field = Hook{}) {
  const int tid = TK == TEAM_CTA ? (int)threadIdx.x : T.tid;
  const int nt = TK == TEAM_CTA ? (int)blockDim.x : (TK == TEAM_WARP ? 32 : T.nt);
  const int lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const float2 *tw = reinterpret_cast<const float2 *>(tables);
  const int32_t *ul = reinterpret_cast<const int32_t *>(tw + NFFT);
  const int32_t *vl = ul + NFFT;
  const int32_t *cb = vl + NFFT;
  const int npix = P.npix, npix2 = npix * npix, nr2 = P.nrebin2;
  const float *wt = reinterpret_cast<const float *>(tables + L.wt);
  const int nu = P.nu, nv = P.nv;
  const int pd = PD > 0 ? PD : P.pdiam;
  const int pd2 = pd * pd, nupd = nu * pd, nunv = nu * nv;

  const ShMeta M(work, L, S);
  int32_t *m_vx = M.vx, *m_vy = M.vy;
  float *m_fl = M.fl, *m_tot = M.tot, *m_rx = M.rx, *m_ry = M.ry;
  int *n_listed = M.n_listed;
  float2 *E = reinterpret_cast<float2 *>(work + L.E);
  float2 *Gt = reinterpret_cast<float2 *>(work + L.Gt);
  float *I = reinterpret_cast<float *>(work + L.I);
  float *bins = reinterpret_cast<float *>(work + L.bins);
  float *dw = reinterpret_cast<float *>(work + L.dw);
  int *order = reinterpret_cast<int *>(work + L.ord);  // stage 4-5 pixel list
  const float *rk = reinterpret_cast<const float *>(tables + L.rk);

  // ---- 0. metadata of the batch (one global round trip for all of it:
  //      global-space loads, free to overtake the shared stores) ----
  const uint32_t frame = P.frame_ptr ? __ldcg(P.frame_ptr) : P.frame;
  // (threads with no field element take the metadata when there are such:
  // the shared stores wait for their loads, which would otherwise hold back a
  // field thread's own loads by a round trip)
  const int nE = S * pd2;
  const int t0 = max(0, min(nE, nt - S));
  for (int mt = tid - t0; mt < S; mt += nt) {
    if (mt < 0) break;
    const int k = base + mt * stride;
    const int vx = __ldg(P.validsubsx + k), vy = __ldg(P.validsubsy + k);
    const float fl = __ldg(P.flux + k);
    float rx = 0.f, ry = 0.f;
    if (P.ckind >= 0) {
      rx = __ldg(P.c_ref + (P.c_order ? 2 * k : k));
      ry = __ldg(P.c_ref + (P.c_order ? 2 * k + 1 : k + P.nvalid));
    }
    m_vx[mt] = vx;
    m_vy[mt] = vy;
    m_fl[mt] = fl;
    m_rx[mt] = rx;
    m_ry[mt] = ry;
  }
  if (tid == 0) n_listed[0] = n_listed[1] = 0;
  // (no barrier here: stage 1 reads the phase-window corners itself, the
  // metadata and the counters are first used after stage 1's barrier)

  // ---- 1. complex field: loads of up to 4 elements issued before any use ----
  if constexpr (FS) {
    // field stop: the sub-aperture's window of the filtered full-pupil field times
    // exp(-i offset), normalised (camplipup_krnl, libsutra/src.cu/sutra_wfs.cu:87-117)
    for (int i0 = tid; i0 < nE; i0 += 4 * nt) {
      float2 fv[4];
      float of[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int i = i0 + j * nt;
        if (i < nE) {
          const int s = PD > 0 ? i / (PD * PD) : udiv(i, P.mg_pd2);
          const int l = i - s * pd2;
          const int y = PD > 0 ? l / PD : udiv(l, P.mg_pd);
          const int x = l - y * pd;
          const int k = base + s * stride;
          fv[j] = P.fs_field[(x + __ldg(P.puppixx + k)) + (y + __ldg(P.puppixy + k)) * P.fs_n];
          of[j] = __ldg(P.offsets + l);
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int i = i0 + j * nt;
        if (i < nE) {
          float so, co;
          sincosf(of[j], &so, &co);
          E[i] = make_float2((fv[j].x * co + fv[j].y * so) * P.fs_inv, (fv[j].y * co - fv[j].x * so) * P.fs_inv);
        }
      }
    }
  } else
  for (int i0 = tid; i0 < nE; i0 += 4 * nt) {
    float ph[4], am[4], of[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int i = i0 + j * nt;
      if (i < nE) {
        const int s = PD > 0 ? i / (PD * PD) : udiv(i, P.mg_pd2);
        const int l = i - s * pd2;
        const int y = PD > 0 ? l / PD : udiv(l, P.mg_pd);
        const int x = l - y * pd;
        const int k = base + s * stride;
        const int id = (x + __ldg(P.puppixx + k)) + (y + __ldg(P.puppixy + k)) * P.npup;
        ph[j] = __ldcg(P.phase + id);  // (L2: a resident kernel reads a new phase every step)
        am[j] = __ldg(P.pupil + id);
        of[j] = __ldg(P.offsets + l);
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int i = i0 + j * nt;
      if (i < nE) {
        float sn, cs;
        sincosf(ph[j] * P.scale - of[j], &sn, &cs);
        E[i] = make_float2(cs * am[j], sn * am[j]);
      }
    }
  }
  team_sync<TK>(T);
  after_field();

  if constexpr (PD > 0) {
    // Register-blocked DFTs: a thread keeps one input row (column) in registers
    // and produces ACH (BCH) outputs from it, with the per-geometry twiddles
    // WX / WY; lanes of a warp share the output chunk, so twiddle reads are
    // broadcasts.  Each output accumulates over the input in the same order as
    // the generic path below.
    constexpr int ACH = 3, BCH = 6;
    const float2 *WX = reinterpret_cast<const float2 *>(tables + L.wxy);
    const float2 *WY = WX + nu * PD;
    // ---- 2. DFT along x: Gt[y][s * nu + a] = sum_x E[s][y][x] WX[a][x] ----
    const int R = S * PD, Q = S * nu;
    const int nach = (nu + ACH - 1) / ACH;
    const uint32_t mgR = udiv_magic((uint32_t)R);
    for (int i = tid; i < R * nach; i += nt) {
      const int c = udiv(i, mgR), row = i - c * R;
      const int sl = row / PD, y = row - sl * PD;
      float2 ev[PD];
#pragma unroll
      for (int x = 0; x < PD; ++x) ev[x] = E[row * PD + x];
#pragma unroll
      for (int j = 0; j < ACH; ++j) {
        const int a = c * ACH + j;
        if (a < nu) {
          const float2 *w = WX + a * PD;
          float re = 0.f, im = 0.f;
#pragma unroll
          for (int x = 0; x < PD; ++x) {
            const float2 wv = w[x], v = ev[x];
            re = fmaf(v.x, wv.x, fmaf(-v.y, wv.y, re));
            im = fmaf(v.x, wv.y, fmaf(v.y, wv.x, im));
          }
          Gt[y * Q + sl * nu + a] = make_float2(re, im);
        }
      }
    }
    team_sync<TK>(T);
    // ---- 3. DFT along y and |.|^2: I[s][b][a] ----
    const int nbch = (nv + BCH - 1) / BCH;
    const uint32_t mgQ = udiv_magic((uint32_t)Q);
    for (int i = tid; i < Q * nbch; i += nt) {
      const int c = udiv(i, mgQ), q = i - c * Q;
      const int sl = udiv(q, P.mg_nu), a = q - sl * nu;
      float2 gv[PD];
#pragma unroll
      for (int y = 0; y < PD; ++y) gv[y] = Gt[y * Q + q];
#pragma unroll
      for (int j = 0; j < BCH; ++j) {
        const int b = c * BCH + j;
        if (b < nv) {
          const float2 *w = WY + b * PD;
          float re = 0.f, im = 0.f;
#pragma unroll
          for (int y = 0; y < PD; ++y) {
            const float2 wv = w[y], v = gv[y];
            re = fmaf(v.x, wv.x, fmaf(-v.y, wv.y, re));
            im = fmaf(v.x, wv.y, fmaf(v.y, wv.x, im));
          }
          I[sl * nunv + b * nu + a] = fmaf(re, re, im * im);
        }
      }
    }
    team_sync<TK>(T);
  } else {
    // ---- 2. DFT along x: Gt[s][y][a] = sum_x E[s][y][x] W^(u_a x) ----
    for (int i = tid; i < S * nupd; i += nt) {
      const int s = udiv(i, P.mg_nupd);
      const int r = i - s * nupd;
      const int y = udiv(r, P.mg_nu), a = r - y * nu;
      const int ua = ul[a];
      const float2 *e = E + s * pd2 + y * pd;
      float re = 0.f, im = 0.f;
      for (int x = 0; x < pd; ++x) {
        const float2 w = tw[(ua * x) & (NFFT - 1)], v = e[x];
        re = fmaf(v.x, w.x, fmaf(-v.y, w.y, re));
        im = fmaf(v.x, w.y, fmaf(v.y, w.x, im));
      }
      Gt[i] = make_float2(re, im);
    }
    team_sync<TK>(T);
    // ---- 3. DFT along y and |.|^2: I[s][b][a] ----
    for (int i = tid; i < S * nunv; i += nt) {
      const int s = udiv(i, P.mg_nunv);
      const int r = i - s * nunv;
      const int b = udiv(r, P.mg_nu), a = r - b * nu;
      const int vb = vl[b];
      const float2 *g = Gt + s * nupd + a;
      float re = 0.f, im = 0.f;
      for (int y = 0; y < pd; ++y) {
        const float2 w = tw[(vb * y) & (NFFT - 1)], v = g[y * nu];
        re = fmaf(v.x, w.x, fmaf(-v.y, w.y, re));
        im = fmaf(v.x, w.y, fmaf(v.y, w.x, im));
      }
      I[i] = fmaf(re, re, im * im);
    }
    team_sync<TK>(T);
  }

  const int nP = S * npix2;
  // ---- 4. binning and flux: one warp per sub-aperture; the flux is summed as
  //      lane-strided partial sums, then a butterfly ----
  for (int s = warp; s < S; s += nw) {
    const float *Is = I + s * nunv;
    float part = 0.f;
    for (int p = lane; p < npix2; p += 32) {
      const int32_t *c = cb + p * nr2;
      float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
      int r = 0;
      // (an entry of -1 lies outside the spot's nfft x nfft support: zero)
      auto at = [&](int ci) { return ci >= 0 ? Is[ci] : 0.f; };
      for (; r + 3 < nr2; r += 4) {
        v0 += at(c[r]);
        v1 += at(c[r + 1]);
        v2 += at(c[r + 2]);
        v3 += at(c[r + 3]);
      }
      for (; r < nr2; ++r) v0 += at(c[r]);
      const float v = (v0 + v1) + (v2 + v3);
      bins[s * npix2 + p] = v;
      part += v;
    }
    part = warp_sum(part);
    if (lane == 0) {
      m_tot[s] = part;
      P.intensities[base + s * stride] = part;
    }
    // normalise in place; with photon noise list the pixels by sampler
    // (inversion from the front of `order`, PTRS from the back) so that the
    // warps of stage 5 each run one sampler
    const float fl = m_fl[s];
    for (int p0 = 0; p0 < npix2; p0 += 32) {
      const int p = p0 + lane;
      const bool valid = p < npix2;
      float v = valid ? bins[s * npix2 + p] : 0.f;
      if (valid && part != 0.f) v = v * fl / part * P.nphot;
      if (valid) bins[s * npix2 + p] = v;
      if (P.noise_mode >= 1) {
        const bool inv = valid && v < AOB_POISSON_INV_MAX_MEAN;
        const bool ptr = valid && !inv;
        const unsigned mi = __ballot_sync(0xffffffffu, inv), mp = __ballot_sync(0xffffffffu, ptr);
        int bi = 0, bp = 0;
        if (lane == 0) {
          bi = atomicAdd(&n_listed[0], __popc(mi));
          bp = atomicAdd(&n_listed[1], __popc(mp));
        }
        bi = __shfl_sync(0xffffffffu, bi, 0);
        bp = __shfl_sync(0xffffffffu, bp, 0);
        const unsigned lt = (1u << lane) - 1u;
        if (inv) order[bi + __popc(mi & lt)] = s * npix2 + p;
        if (ptr) order[nP - 1 - (bp + __popc(mp & lt))] = s * npix2 + p;
      }
    }
  }
  team_sync<TK>(T);

  // ---- 5. noise (the noisy pixel replaces its mean in bins), centroid weights ----
  for (int t = tid; t < nP; t += nt) {
    const int i = P.noise_mode >= 1 ? order[t] : t;
    const int s = udiv(i, P.mg_np2), p = i - s * npix2;
    const int k = base + s * stride;
    float wgt = 1.f;
    if (P.ckind == 2) wgt = P.c_wper ? P.c_weights[p + k * npix2] : wt[p];
    float v = bins[i];
    const uint32_t pix = (uint32_t)(p + k * npix2);
    if (P.noise_mode >= 1) {
      const U4 w0 = philox4x32_10(U4{pix, frame, TAG_POISSON, 0u}, P.k0, P.k1);
      v = v < AOB_POISSON_INV_MAX_MEAN ? poisson_inversion(v, w0, rk) : poisson_ptrs(v, w0, pix, frame, P.k0, P.k1);
      if (P.noise_mode >= 2) v = v + P.noise * gauss_sample(w0);
    }
    bins[i] = v;
    float d = v;
    if (P.ckind == 1 || P.ckind == 2) d = (v > P.c_thresh) ? v - P.c_thresh : 1.e-6f;
    dw[i] = d * wgt;
  }
  team_sync<TK>(T);

  // ---- 6. centroids, then the sub-aperture's cube block and image window ----
  for (int s = warp; s < S; s += nw) {
    if (P.ckind >= 0) {
      float cs = 0.f, cx = 0.f, cy = 0.f;
      for (int p = lane; p < npix2; p += 32) {
        const float d = dw[s * npix2 + p];
        const int y = udiv(p, P.mg_np), x = p - y * npix;
        cs += d;
        cx = fmaf(d, (float)x, cx);
        cy = fmaf(d, (float)y, cy);
      }
      cs = warp_sum(cs);
      cx = warp_sum(cx);
      cy = warp_sum(cy);
      if (lane == 0) {
        const int k = base + s * stride;
        const int ix = P.c_order ? 2 * k : k;
        const int iy = P.c_order ? 2 * k + 1 : k + P.nvalid;
        P.c_slopes[ix] = (cx / (cs + 1.e-6f) - P.c_offset) * P.c_scale - m_rx[s];
        P.c_slopes[iy] = (cy / (cs + 1.e-6f) - P.c_offset) * P.c_scale - m_ry[s];
        P.c_intens[k] = cs;
      }
    }
    if constexpr (!DEFER_IMG) sh_store_subap(P, base + s * stride, bins + s * npix2, m_vx[s], m_vy[s], lane);
  }
  team_sync<TK>(T);
}

}  // namespace aob
