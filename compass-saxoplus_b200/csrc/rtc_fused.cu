// One RTC iteration in one cooperative kernel: Shack-Hartmann image + fused
// centroids -> grid barrier -> command-matrix MVM + integrator + voltage.
//
// The MVM's HBM stream does not depend on the slopes, so it is started first:
// at kernel entry one thread per CTA issues TMA bulk copies of that CTA's rows of
// the packed command matrix into shared memory (one mbarrier per row).  While
// those bytes are in flight the CTA's warps form sensor images (sh_core.cuh).
// A bounded grid barrier then publishes the slopes; every CTA stages them in
// shared memory and reduces its rows, which by then have landed, applying the
// integrator (sutra_controller_ls.cpp:251-285, sutra_utils.cu:631-639) and the
// delay/latency/clip voltage stage (sutra_controller.cpp:205-263) per actuator.
//
// Co-residency of all CTAs is guaranteed by the cooperative launch attribute;
// every wait is bounded and reports ERR_MBAR_TIMEOUT / ERR_GRID_TIMEOUT in the
// controller's status word instead of hanging.  No cluster multicast is used.

#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <algorithm>

#include "aob_objects.hpp"
#include "sh_core.cuh"

namespace aob {

enum : uint32_t { ERR_GRID_TIMEOUT = 2u };
constexpr uint32_t GRID_MAX_POLLS = 1u << 24;
constexpr uint32_t ROW_MAX_POLLS = 1u << 22;
constexpr int FUSED_THREADS = 512;

template <typename T>
struct FPack;
template <>
struct FPack<float> {
  static constexpr int N = 4;
  __device__ static float dot(const uint4 &q, const float4 *sv) {
    const float *f = reinterpret_cast<const float *>(&q);
    const float4 s = sv[0];
    return fmaf(f[3], s.w, fmaf(f[2], s.z, fmaf(f[1], s.y, f[0] * s.x)));
  }
};
template <>
struct FPack<__nv_bfloat16> {
  static constexpr int N = 8;
  __device__ static float dot(const uint4 &q, const float4 *sv) {
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
    float a = 0.f;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const float4 s = sv[32 * i];
      const float2 f0 = __bfloat1622float2(h[2 * i]), f1 = __bfloat1622float2(h[2 * i + 1]);
      a = fmaf(f1.y, s.w, fmaf(f1.x, s.z, fmaf(f0.y, s.y, fmaf(f0.x, s.x, a))));
    }
    return a;
  }
};
template <>
struct FPack<__nv_fp8_e4m3> {
  static constexpr int N = 16;
  __device__ static float dot(const uint4 &q, const float4 *sv) {
    const __nv_fp8x2_e4m3 *h = reinterpret_cast<const __nv_fp8x2_e4m3 *>(&q);
    float a = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float4 s = sv[32 * i];
      const float2 f0 = static_cast<float2>(h[2 * i]), f1 = static_cast<float2>(h[2 * i + 1]);
      a = fmaf(f1.y, s.w, fmaf(f1.x, s.z, fmaf(f0.y, s.y, fmaf(f0.x, s.x, a))));
    }
    return a;
  }
};

struct RtcFusedArgs {
  ShKernelArgs sh;     // sensor; sh.c_slopes is the controller's slope vector
  const void *mat;     // packed command matrix rows
  const float *rscale; // FP8 per-row scales or null
  int ld, nrow, ncol;
  float *err, *com;
  const float *mgain;
  float gain;
  float *oldest;        // delay ring[0] (read, then replaced by the new command)
  const float *second;  // delay ring[1]
  float a, b;
  int delayed;
  float vmin, vmax;
  int do_clip;
  float *volt;
  uint32_t *bump;     // noise frame counter (incremented once)
  uint32_t *status;   // error word
  uint32_t *gbar;     // grid barrier {arrived, generation}
  int rows_per_cta;
};

__host__ __device__ inline int fused_slope_floats(int ld, int v) { return ((ld / v + 31) / 32) * 32 * v; }

// Grid-wide barrier for a cooperative launch: {arrived, generation} in global
// memory; the last CTA to arrive resets the count and advances the generation.
// The wait is bounded; on expiry ERR_GRID_TIMEOUT is set and false returned.
__device__ __forceinline__ bool grid_barrier(uint32_t *gbar, uint32_t nblocks, uint32_t *status) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile uint32_t *vgen = gbar + 1;
    const uint32_t gen = *vgen;
    __threadfence();
    const uint32_t arrived = atomicAdd(gbar, 1u);
    if (arrived == nblocks - 1) {
      gbar[0] = 0u;
      __threadfence();
      atomicAdd(gbar + 1, 1u);
    } else {
      uint32_t i = 0;
      while (*vgen == gen && i < GRID_MAX_POLLS) {
        __nanosleep(32);
        ++i;
      }
      if (*vgen == gen) {
        ok = 0;
        atomicOr(status, (uint32_t)ERR_GRID_TIMEOUT);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <typename T, int NFFT, int WPS, int PD>
__global__ void __launch_bounds__(FUSED_THREADS, 1) rtc_fused_kernel(RtcFusedArgs A) {
  extern __shared__ __align__(128) unsigned char sm[];
  constexpr int V = FPack<T>::N;
  constexpr int Q = V / 4;
  constexpr int GT = WPS * 32;
  constexpr int GROUPS = FUSED_THREADS / GT;
  const uint32_t row_bytes = (uint32_t)(A.ld * sizeof(T));
  const int r0 = (int)(((int64_t)blockIdx.x * A.nrow) / gridDim.x);
  const int r1 = (int)(((int64_t)(blockIdx.x + 1) * A.nrow) / gridDim.x);
  const int R = r1 - r0;
  // shared memory: barriers | matrix rows | sensor tables + group scratch | slopes
  uint64_t *bars = reinterpret_cast<uint64_t *>(sm);
  unsigned char *rows = sm + 128 * ((A.rows_per_cta * 8 + 127) / 128);
  unsigned char *shm = rows + (size_t)A.rows_per_cta * row_bytes;
  const int pd = PD > 0 ? PD : A.sh.pdiam;
  const ShSmem L(NFFT, A.sh.nu, A.sh.nv, pd, A.sh.nrebin2 * A.sh.npix * A.sh.npix, A.sh.npix * A.sh.npix, WPS);
  float *s_sh = reinterpret_cast<float *>(shm + L.bytes(GROUPS));

  if (threadIdx.x == 0) {
    for (int r = 0; r < R; ++r) mbar_init(&bars[r], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned char *src = static_cast<const unsigned char *>(A.mat) + (size_t)r0 * row_bytes;
    for (int r = 0; r < R; ++r) {
      mbar_expect_tx(&bars[r], row_bytes);
      bulk_g2s(rows + (size_t)r * row_bytes, src + (size_t)r * row_bytes, row_bytes, &bars[r]);
    }
  }
  // ---- sensor images and slopes ----
  sh_load_tables<NFFT>(A.sh, shm, threadIdx.x, blockDim.x);
  __syncthreads();
  {
    const int group = threadIdx.x / GT;
    const int gt = threadIdx.x - group * GT;
    unsigned char *scratch = shm + L.hdr + L.per_grp * group;
    // round-robin over CTAs first so that every SM gets nvalid / nsm sub-apertures
    for (int k = group * gridDim.x + blockIdx.x; k < A.sh.nvalid; k += gridDim.x * GROUPS)
      sh_subap<NFFT, WPS, PD>(A.sh, k, shm, scratch, group, gt);
  }
  // ---- all slopes published ----
  const bool ok = grid_barrier(A.gbar, gridDim.x, A.status);
  if (ok) {
    if (A.bump && blockIdx.x == 0 && threadIdx.x == 0) *A.bump += 1u;
    const int nsh = fused_slope_floats(A.ld, V);
    for (int i = threadIdx.x; i < nsh; i += blockDim.x) {
      const int g = i >> 2, e = i & 3;
      const int l = g & 31, jq = g >> 5;
      const int j = jq / Q, q = jq - j * Q;
      const int src = (l + 32 * j) * V + 4 * q + e;
      s_sh[i] = (src < A.ncol) ? __ldcg(A.sh.c_slopes + src) : 0.f;
    }
    __syncthreads();
    const int nchunk = A.ld / V;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float4 *svl = reinterpret_cast<const float4 *>(s_sh) + lane;
    for (int r = warp; r < R; r += FUSED_THREADS / 32) {
      if (!mbar_wait(&bars[r], 0, ROW_MAX_POLLS)) {
        if (lane == 0) atomicOr(A.status, (uint32_t)ERR_MBAR_TIMEOUT);
        continue;
      }
      const uint4 *row = reinterpret_cast<const uint4 *>(rows + (size_t)r * row_bytes) + lane;
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      int j = 0;
      for (; 32 * (j + 3) + lane < nchunk; j += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) acc[u] += FPack<T>::dot(row[32 * (j + u)], svl + 32 * Q * (j + u));
      }
      for (; 32 * j + lane < nchunk; ++j) acc[0] += FPack<T>::dot(row[32 * j], svl + 32 * Q * j);
      float tot = warp_sum((acc[0] + acc[1]) + (acc[2] + acc[3]));
      if (lane == 0) {
        const int gr = r0 + r;
        if (A.rscale) tot *= A.rscale[gr];
        const float e = -tot;
        A.err[gr] = e;
        const float c = A.gain * (e * A.mgain[gr]) + A.com[gr];
        A.com[gr] = c;
        float v;
        if (A.delayed) {
          v = A.a * A.oldest[gr] + A.b * A.second[gr];
          A.oldest[gr] = c;
        } else {
          v = c;
        }
        if (A.do_clip) v = fminf(fmaxf(v, A.vmin), A.vmax);
        A.volt[gr] = v;
      }
    }
  }
  // no CTA may exit with a copy still landing in its shared memory
  __syncthreads();
  if (threadIdx.x == 0)
    for (int r = 0; r < R; ++r) mbar_wait(&bars[r], 0, ROW_MAX_POLLS);
}

// ---------------------------------------------------------------------------
template <typename T, int NFFT, int WPS, int PD>
static bool launch_fused_t(const RtcFusedArgs &A0, int grid, size_t sm, cudaStream_t s, bool dry) {
  auto kern = rtc_fused_kernel<T, NFFT, WPS, PD>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, FUSED_THREADS, sm) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    return false;
  }
  if (dry) return true;
  RtcFusedArgs A = A0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(FUSED_THREADS);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  AOB_CUDA(cudaLaunchKernelEx(&cfg, kern, A));
  return true;
}

template <typename T, int NFFT, int WPS>
static bool launch_fused_pd(int pd, const RtcFusedArgs &A, int grid, size_t sm, cudaStream_t s, bool dry) {
  switch (pd) {
    case 4: return launch_fused_t<T, NFFT, WPS, 4>(A, grid, sm, s, dry);
    case 6: return launch_fused_t<T, NFFT, WPS, 6>(A, grid, sm, s, dry);
    case 8: return launch_fused_t<T, NFFT, WPS, 8>(A, grid, sm, s, dry);
    default: return launch_fused_t<T, NFFT, WPS, 0>(A, grid, sm, s, dry);
  }
}

template <typename T, int NFFT>
static bool launch_fused_w(int wps, int pd, const RtcFusedArgs &A, int grid, size_t sm, cudaStream_t s, bool dry) {
  if (wps == 1) return launch_fused_pd<T, NFFT, 1>(pd, A, grid, sm, s, dry);
  if (wps == 2) return launch_fused_pd<T, NFFT, 2>(pd, A, grid, sm, s, dry);
  return launch_fused_pd<T, NFFT, 4>(pd, A, grid, sm, s, dry);
}

template <typename T>
static bool launch_fused_n(int nfft, int wps, int pd, const RtcFusedArgs &A, int grid, size_t sm, cudaStream_t s,
                           bool dry) {
  if (nfft == 16) return launch_fused_w<T, 16>(wps, pd, A, grid, sm, s, dry);
  if (nfft == 32) return launch_fused_w<T, 32>(wps, pd, A, grid, sm, s, dry);
  return launch_fused_w<T, 64>(wps, pd, A, grid, sm, s, dry);
}

}  // namespace aob

using namespace aob;

// Launch (or, with dry = true, only check that it can launch) the fused kernel
// for this loop.  Returns false when the configuration does not fit (shared
// memory, co-residency), in which case the caller runs the three-kernel path.
bool aob_loop::launch_fused(bool noise, cudaStream_t s, bool frame_on_device, bool dry) {
  aob_sh *w = wfs;
  aob_ls *c = ls;
  bool perturbed = false;
  for (auto &kv : c->perturb) perturbed |= kv.second.on;
  if (perturbed || c->open_loop || centro->type > 2) return false;
  c->ensure_packed(c->prec);
  RtcFusedArgs A{};
  aob_centro *fc = w->make_args(noise, c->centroids.p, frame_on_device ? d_frame.p : nullptr, A.sh);
  if (fc != centro) return false;
  const int esize = c->prec == AOB_PREC_F32 ? 4 : (c->prec == AOB_PREC_BF16 ? 2 : 1);
  const int V = 16 / esize;
  A.ld = (c->nslope + V - 1) / V * V;
  A.mat = c->prec == AOB_PREC_F32 ? (const void *)c->cm_f32.p
                                  : (c->prec == AOB_PREC_BF16 ? (const void *)c->cm_bf16.p : (const void *)c->cm_fp8.p);
  A.rscale = c->prec == AOB_PREC_FP8 ? c->row_scale.p : nullptr;
  A.nrow = c->nactu;
  A.ncol = c->nslope;
  A.err = c->err.p;
  A.com = c->com();
  A.mgain = c->gains.p;
  A.gain = c->gain;
  A.delayed = c->delay > 0 ? 1 : 0;
  if (A.delayed) {
    A.oldest = c->ring[0].p;
    A.second = c->ring[1].p;
  }
  A.a = c->a;
  A.b = c->b;
  A.vmin = c->volt_min;
  A.vmax = c->volt_max;
  A.do_clip = c->volt_min < c->volt_max ? 1 : 0;
  A.volt = c->com_clipped.p;
  const bool noisy = noise && w->noise > -1.f;
  A.bump = (frame_on_device && noisy) ? d_frame.p : nullptr;
  A.status = c->status.p;
  A.gbar = gbar.p;
  const int nsm = num_sms(w->device);
  const int grid = std::min(nsm, c->nactu);
  A.rows_per_cta = (c->nactu + grid - 1) / grid;
  const int wps = fused_wps > 0 ? fused_wps : 1;
  const int groups = FUSED_THREADS / (32 * wps);
  const ShSmem L(w->nfft, w->nu, w->nv, w->nphase, w->nrebin * w->nrebin * w->npix * w->npix, w->npix * w->npix, wps);
  const size_t sm = 128 * ((A.rows_per_cta * 8 + 127) / 128) + (size_t)A.rows_per_cta * A.ld * esize +
                    L.bytes(groups) + sizeof(float) * fused_slope_floats(A.ld, V);
  if (sm > 227 * 1024) return false;
  bool ok;
  if (c->prec == AOB_PREC_F32)
    ok = launch_fused_n<float>(w->nfft, wps, w->nphase, A, grid, sm, s, dry);
  else if (c->prec == AOB_PREC_BF16)
    ok = launch_fused_n<__nv_bfloat16>(w->nfft, wps, w->nphase, A, grid, sm, s, dry);
  else
    ok = launch_fused_n<__nv_fp8_e4m3>(w->nfft, wps, w->nphase, A, grid, sm, s, dry);
  if (!ok || dry) return ok;
  AOB_LAUNCH_CHECK("rtc_fused_kernel");
  w->after_image(A.sh, fc, false);
  if (A.delayed) {
    aob::DevBuf<float> t = std::move(c->ring.front());
    c->ring.pop_front();
    c->ring.push_back(std::move(t));
  }
  return true;
}
