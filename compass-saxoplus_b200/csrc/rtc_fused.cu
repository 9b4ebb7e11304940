// One RTC iteration in one cooperative kernel: Shack-Hartmann image + fused
// centroids -> grid barrier -> command-matrix MVM + integrator + voltage.
//
// At entry one thread per CTA bulk-copies the sensor tables into shared memory
// and prefetches its slice of the phase screen and pupil into L2.  The MVM's
// HBM stream does not depend on the slopes: once the first batch's complex
// field is formed (so the sensor's own first loads did not queue behind it),
// the same thread issues TMA bulk copies of the CTA's rows of the packed
// command matrix into shared memory, all completing on one mbarrier.  While
// those bytes are in flight the CTA forms the sensor images of its share of the
// sub-apertures (k = blockIdx.x + j * gridDim.x) (sh_core.cuh).  The CTA then
// arrives at a bounded grid barrier, writes its cube and image while the other
// CTAs arrive, and once all slopes are published stages them in shared memory
// and reduces its rows, which by then have landed, applying the integrator
// (sutra_controller_ls.cpp:251-285, sutra_utils.cu:631-639) and the
// delay/latency/clip voltage stage (sutra_controller.cpp:205-263) per actuator.
//
// Co-residency of all CTAs is guaranteed by the cooperative launch attribute;
// every wait is bounded and reports ERR_MBAR_TIMEOUT / ERR_GRID_TIMEOUT in the
// controller's status word instead of hanging.  No cluster multicast is used.

#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <map>
#include <mutex>

#include "aob_objects.hpp"
#include "mvm_core.cuh"
#include "sh_core.cuh"

namespace aob {

constexpr uint32_t ROW_MAX_POLLS = 1u << 22;
constexpr int FUSED_THREADS = 512;

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
  unsigned long long *gbar;  // grid-barrier arrival counter (never reset)
  int rows_per_cta;
  int batch;  // sub-apertures per CTA and round
  float *volt_host;  // caller's pinned host voltages (mapped), also written, or null
  uint32_t grid_polls;  // poll limit of the grid-barrier wait
  int absent_cta;       // test of the bounded wait: this CTA never arrives (-1: none)
  // persistent mode (ctl non-null): the kernel stays resident and runs one step
  // per doorbell.  ctl[PERSIST_DOOR]: the id of the step to run (written by the
  // host's stream), ctl[PERSIST_STOP]: non-zero to leave, ctl[PERSIST_DONE]: the
  // id of the last step every CTA finished (read by the host's stream),
  // ctl[PERSIST_FIN]: CTA completions.  Step ids count from 1.
  uint32_t *ctl;
  uint32_t door_polls;  // poll limit of one doorbell wait (each poll sleeps ~256 ns)
};

// control words of the persistent mode, one 128-byte line each
constexpr int PERSIST_DOOR = 0, PERSIST_STOP = 32, PERSIST_DONE = 64, PERSIST_FIN = 96, PERSIST_WORDS = 128;
// on the doorbell's line, written before it: the command (0 an RTC step, 1 write
// ARG bytes of zeros at ARG pointer -- the L2 flush of a benchmark, which has to
// come from the resident kernel since it holds every SM's registers)
constexpr int PERSIST_CMD = 4, PERSIST_ARG = 8;
// on the done line: the global-timer time CTA 0 saw the doorbell (64 bits) and
// the sum over steps of (done - that time) in nanoseconds (64 bits)
constexpr int PERSIST_T0 = 72, PERSIST_TSUM = 74;

__device__ __forceinline__ unsigned long long global_timer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// done value a persistent kernel leaves behind when it exits: far ahead of every
// step id a host stream may be waiting for (the waits compare cyclically)
constexpr uint32_t PERSIST_EXIT_AHEAD = 0x40000000u;

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__host__ __device__ inline size_t fused_bars_bytes(int rows) { return 128 * (((size_t)rows * 8 + 127) / 128); }
__host__ __device__ inline size_t fused_pre_bytes(int rows) { return 128 * (((size_t)rows * 20 + 127) / 128); }

template <typename T, int NFFT, int PD>
__global__ void __launch_bounds__(FUSED_THREADS, 1) rtc_fused_kernel(RtcFusedArgs A) {
  extern __shared__ __align__(128) unsigned char sm[];
  constexpr int V = RowPack<T>::N;
  constexpr int Q = V / 4;
  const uint32_t row_bytes = (uint32_t)(A.ld * sizeof(T));
  // (32-bit: nrow * gridDim < 2^32 is checked on the host)
  const int r0 = (int)((blockIdx.x * (uint32_t)A.nrow) / gridDim.x);
  const int r1 = (int)(((blockIdx.x + 1) * (uint32_t)A.nrow) / gridDim.x);
  const int R = r1 - r0;
  // shared memory: barriers | per-row epilogue inputs | matrix rows |
  //                sensor tables + batch work area | slopes
  uint64_t *bars = reinterpret_cast<uint64_t *>(sm);
  float *pre = reinterpret_cast<float *>(sm + fused_bars_bytes(A.rows_per_cta));
  unsigned char *rows = sm + fused_bars_bytes(A.rows_per_cta) + fused_pre_bytes(A.rows_per_cta);
  unsigned char *shm = rows + (size_t)A.rows_per_cta * row_bytes;
  const int pd = PD > 0 ? PD : A.sh.pdiam;
  const ShSmem L(NFFT, A.sh.nu, A.sh.nv, pd, A.sh.nrebin2 * A.sh.npix * A.sh.npix, A.sh.npix * A.sh.npix, A.batch);
  // sensor tables + work area, later the MVM's per-warp partial sums
  const size_t work_bytes = max(L.bytes(), L.hdr + sizeof(float) * (FUSED_THREADS / 32) * A.rows_per_cta);
  float *s_sh = reinterpret_cast<float *>(shm + work_bytes);

  // The last warp, which has the least sensor work in stage 1 (its threads
  // take field samples only when a CTA has more than 13 sub-apertures of
  // 6 x 6 samples), initialises the row barrier, issues the copies and fetches the
  // epilogue inputs; the other threads first wait on the barrier after
  // several __syncthreads.  The copies go out once the first batch's field
  // is formed: the sensor's own first loads (tables, pupil windows, phase)
  // then do not queue behind the matrix stream, which still has the DFT,
  // binning, noise and centroid stages to land.
  const int helper = (int)blockDim.x - 32;
  // The sensor tables arrive by bulk copy on bars[1], issued at entry: no
  // thread holds a register waiting for them before the DFTs, so the field
  // stage's loads (pupil windows, then phase) go out at once.
  const ShSmem L1(NFFT, A.sh.nu, A.sh.nv, pd, A.sh.nrebin2 * A.sh.npix * A.sh.npix, A.sh.npix * A.sh.npix, 1);
  const ShTableCopy tcopy(A.sh, L1);
  if ((int)threadIdx.x == helper) {
    // this CTA's slice of the phase screen and of the pupil into L2: the field
    // stage's loads depend on the pupil-window corners (a first round trip),
    // and the values they then fetch are in L2 by that time
    const uint32_t screen = (uint32_t)A.sh.npup * (uint32_t)A.sh.npup * 4u;
    const uint32_t slice = ((screen + gridDim.x - 1) / gridDim.x + 15u) & ~15u;
    const uint32_t off = blockIdx.x * slice;
    if (off < screen) {
      const uint32_t len = min(slice, (screen - off) & ~15u);
      if (len) {
        if ((reinterpret_cast<uintptr_t>(A.sh.phase) & 15) == 0)
          bulk_prefetch_l2(reinterpret_cast<const unsigned char *>(A.sh.phase) + off, len);
        if ((reinterpret_cast<uintptr_t>(A.sh.pupil) & 15) == 0)
          bulk_prefetch_l2(reinterpret_cast<const unsigned char *>(A.sh.pupil) + off, len);
      }
    }
    // one barrier for all the rows: a single wait later; one for the tables
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
    mbar_expect_tx(&bars[1], tcopy.image_bytes + tcopy.wt_bytes);
    bulk_g2s(shm, A.sh.tblob, tcopy.image_bytes, &bars[1]);
    if (tcopy.wt_bytes) bulk_g2s(shm + L1.wt, A.sh.c_weights, tcopy.wt_bytes, &bars[1]);
  }
  bool copies_out = false, tables_in = false;
  auto issue_rows = [&]() {
    if (!copies_out && (int)threadIdx.x == helper) {
      const unsigned char *src = static_cast<const unsigned char *>(A.mat) + (size_t)r0 * row_bytes;
      mbar_expect_tx(&bars[0], (uint32_t)R * row_bytes);
      for (int r = 0; r < R; ++r)
        bulk_g2s(rows + (size_t)r * row_bytes, src + (size_t)r * row_bytes, row_bytes, &bars[0]);
    }
    copies_out = true;
    if (!tables_in) {  // every thread, before the first stage that reads the tables
      if (!mbar_wait(&bars[1], 0, ROW_MAX_POLLS)) atomicOr(A.status, (uint32_t)ERR_MBAR_TIMEOUT);
      tables_in = true;
    }
  };
  // epilogue inputs of this CTA's rows, fetched now so the epilogue makes no
  // global round trip: [scale | modal gain | com | ring[0] | ring[1]]
  const int RP = A.rows_per_cta;
  // (global-space loads, all issued before the shared stores)
  for (int r = (int)threadIdx.x - helper; r >= 0 && r < R; r += 32) {
    const int gr = r0 + r;
    const float sc = A.rscale ? __ldg(A.rscale + gr) : 1.f;
    const float mg = __ldg(A.mgain + gr);
    const float cm = __ldcg(A.com + gr);
    float o0 = 0.f, o1 = 0.f;
    if (A.delayed) {
      o0 = __ldcg(A.oldest + gr);
      o1 = __ldcg(A.second + gr);
    }
    pre[r] = sc;
    pre[RP + r] = mg;
    pre[2 * RP + r] = cm;
    if (A.delayed) {
      pre[3 * RP + r] = o0;
      pre[4 * RP + r] = o1;
    }
  }
  sh_load_tables<NFFT>(A.sh, shm, threadIdx.x, blockDim.x, true, tcopy.wt_bytes != 0);
  const bool persist = A.ctl != nullptr;
  __shared__ uint32_t s_go, s_cmd[5];
  uint32_t step = 0;
  for (;;) {
  if (persist) {
    // the next step: its doorbell rung, and every CTA done with the previous step
    // (so no CTA overwrites slopes another one still reads)
    if (threadIdx.x == 0) {
      uint32_t go = 0;
      for (uint32_t i = 0; i < A.door_polls; ++i) {
        if (ld_acquire_u32(A.ctl + PERSIST_STOP)) break;
        if ((int32_t)(ld_acquire_u32(A.ctl + PERSIST_DOOR) - (step + 1)) >= 0 &&
            (int32_t)(ld_acquire_u32(A.ctl + PERSIST_DONE) - step) >= 0) {
          go = 1;
          break;
        }
        __nanosleep(256);
      }
      if (!go && !ld_acquire_u32(A.ctl + PERSIST_STOP)) atomicOr(A.status, (uint32_t)ERR_DOOR_TIMEOUT);
      s_go = go;
      s_cmd[0] = go ? ld_acquire_u32(A.ctl + PERSIST_CMD) : 0u;
      for (int k = 0; k < 4; ++k) s_cmd[1 + k] = go ? ld_acquire_u32(A.ctl + PERSIST_ARG + k) : 0u;
    }
    __syncthreads();
    if (!s_go) break;
    ++step;
    if (blockIdx.x == 0 && threadIdx.x == 0)
      *reinterpret_cast<unsigned long long *>(A.ctl + PERSIST_T0) = global_timer_ns();
    if (s_cmd[0] == 1u) {
      // zeros over the buffer, this CTA's slice, 16 bytes per store
      float4 *buf = reinterpret_cast<float4 *>((uint64_t)s_cmd[1] | ((uint64_t)s_cmd[2] << 32));
      const uint64_t n16 = ((uint64_t)s_cmd[3] | ((uint64_t)s_cmd[4] << 32)) / 16;
      for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n16; i += (uint64_t)gridDim.x * blockDim.x)
        buf[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  bool ok = true;
  if (!persist || s_cmd[0] == 0u) {
    if ((int)threadIdx.x == helper && step > 1) {
      // this step's phase slice into L2 (the first step's went out at entry)
      const uint32_t screen = (uint32_t)A.sh.npup * (uint32_t)A.sh.npup * 4u;
      const uint32_t slice = ((screen + gridDim.x - 1) / gridDim.x + 15u) & ~15u;
      const uint32_t off = blockIdx.x * slice;
      if (off < screen && (reinterpret_cast<uintptr_t>(A.sh.phase) & 15) == 0) {
        const uint32_t len = min(slice, (screen - off) & ~15u);
        if (len) bulk_prefetch_l2(reinterpret_cast<const unsigned char *>(A.sh.phase) + off, len);
      }
    }
  // ---- sensor images and slopes: this CTA's sub-apertures, A.batch per round ----
  // (stages 0-1 read no tables; the copied ones are waited for after stage 1,
  // the rest is published by the barrier that closes stage 1)
  // With the CTA's whole share in one round (the usual case) the cube and
  // image writes wait until the CTA has arrived at the grid barrier: the slopes
  // go out first and the barrier's release does not wait on the image stores.
  const int nvalid = A.sh.nvalid;
  const Team team{(int)threadIdx.x, (int)blockDim.x, 0};
  const bool one_round = A.batch * (int)gridDim.x >= nvalid;
  const int S1 = (int)blockIdx.x < nvalid ? min(A.batch, (nvalid - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x) : 0;
  if (one_round) {
    if (S1 > 0)
      sh_batch<NFFT, PD, TEAM_CTA, decltype(issue_rows), true>(A.sh, blockIdx.x, gridDim.x, S1, shm, shm + L.hdr, L,
                                                               team, issue_rows);
  } else {
    for (int base = blockIdx.x; base < nvalid; base += A.batch * gridDim.x) {
      const int Sb = min(A.batch, (nvalid - base + (int)gridDim.x - 1) / (int)gridDim.x);
      sh_batch<NFFT, PD>(A.sh, base, gridDim.x, Sb, shm, shm + L.hdr, L, team, issue_rows);
    }
  }
  issue_rows();  // a CTA without sub-apertures
  // ---- all slopes published ----
  // (absent: the CTA a wait-expiry test keeps from arriving; it skips the MVM)
  const bool absent = (int)blockIdx.x == A.absent_cta;
  const unsigned long long ticket = absent ? 0ull : grid_arrive(A.gbar, gridDim.x);
  if (one_round && S1 > 0) sh_store_images(A.sh, blockIdx.x, gridDim.x, S1, shm + L.hdr, L, team);
  ok = !absent && grid_wait(A.gbar, ticket, A.status, A.grid_polls);
  if (ok) {
    if (A.bump && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(A.bump, 1u);  // no round trip
    // slopes into shared memory, 16 bytes per load (L2 only: they were written by
    // other CTAs of this launch); group g of the layout holds slopes
    // [(chunk) * V + 4 q, +4) for chunk = (g & 31) + 32 j, g >> 5 = j * Q + q
    const int ngrp = swizzled_slope_floats(A.ld, V) / 4;
    constexpr int SU = 2;  // groups per thread and pass: both loads go out before either store
    for (int g0 = threadIdx.x; g0 < ngrp; g0 += SU * blockDim.x) {
      float4 v4[SU];
#pragma unroll
      for (int u = 0; u < SU; ++u) {
        const int g = g0 + u * (int)blockDim.x;
        const int l = g & 31, jq = g >> 5;
        const int j = jq / Q, q = jq - j * Q;
        const int src = (l + 32 * j) * V + 4 * q;
        if (g >= ngrp) {
          v4[u] = make_float4(0.f, 0.f, 0.f, 0.f);
        } else if (src + 3 < A.ncol) {
          v4[u] = __ldcg(reinterpret_cast<const float4 *>(A.sh.c_slopes + src));
        } else {
          v4[u].x = src < A.ncol ? __ldcg(A.sh.c_slopes + src) : 0.f;
          v4[u].y = src + 1 < A.ncol ? __ldcg(A.sh.c_slopes + src + 1) : 0.f;
          v4[u].z = src + 2 < A.ncol ? __ldcg(A.sh.c_slopes + src + 2) : 0.f;
          v4[u].w = 0.f;
        }
      }
#pragma unroll
      for (int u = 0; u < SU; ++u) {
        const int g = g0 + u * (int)blockDim.x;
        if (g < ngrp) reinterpret_cast<float4 *>(s_sh)[g] = v4[u];
      }
    }
    __syncthreads();
    // Split-K over the CTA's rows: warp w, lane l take chunks c = l + 32 (w + NW i);
    // each slope chunk is read once and applied to every row from registers
    // (up to RB rows in one pass), then the per-warp partial sums are added in
    // warp order (deterministic).
    constexpr int NW = FUSED_THREADS / 32;
    constexpr int RB = 16;  // rows per register block: two transposed butterflies of 8
    const int nchunk = A.ld / V;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    bool rows_ok = true;
    rows_ok = mbar_wait(&bars[0], 0, ROW_MAX_POLLS);
    if (!rows_ok && lane == 0) atomicOr(A.status, (uint32_t)ERR_MBAR_TIMEOUT);
    float *part = reinterpret_cast<float *>(shm + L.hdr);  // [NW][rows_per_cta], sensor work area is free now
    const float4 *sv4 = reinterpret_cast<const float4 *>(s_sh);
    for (int rb = 0; rb < R; rb += RB) {
      float acc[RB];
#pragma unroll
      for (int u = 0; u < RB; ++u) acc[u] = 0.f;
      if (rows_ok) {
        for (int jj = warp; 32 * jj + lane < nchunk; jj += NW) {
          const int c = lane + 32 * jj;
          float4 sv[Q];
#pragma unroll
          for (int q = 0; q < Q; ++q) sv[q] = sv4[(jj * Q + q) * 32 + lane];
#pragma unroll
          for (int u = 0; u < RB; ++u)
            if (rb + u < R) {
              const uint4 q4 = reinterpret_cast<const uint4 *>(rows + (size_t)(rb + u) * row_bytes)[c];
              acc[u] += RowPack<T>::dot(q4, sv);
            }
        }
      }
#pragma unroll
      for (int h = 0; h < RB / 8; ++h) {
        if (rb + 8 * h >= R) break;
        float a8[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) a8[u] = acc[8 * h + u];
        int u;
        const float t = warp_sum8(a8, lane, u);
        if ((lane & 3) == 0 && rb + 8 * h + u < R) part[warp * A.rows_per_cta + rb + 8 * h + u] = t;
      }
    }
    __syncthreads();
    // integrator and voltage per row, one thread per row
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
      float tot = 0.f;
#pragma unroll
      for (int w = 0; w < NW; ++w) tot += part[w * A.rows_per_cta + r];
      const int gr = r0 + r;
      if (A.rscale) tot *= pre[r];
      const float e = -tot;
      A.err[gr] = e;
      const float c = A.gain * (e * pre[RP + r]) + pre[2 * RP + r];
      A.com[gr] = c;
      pre[2 * RP + r] = c;  // the integrator's state for a next (persistent) step
      float v;
      if (A.delayed) {
        v = A.a * pre[3 * RP + r] + A.b * pre[4 * RP + r];
        A.oldest[gr] = c;
      } else {
        v = c;
      }
      if (A.do_clip) v = fminf(fmaxf(v, A.vmin), A.vmax);
      A.volt[gr] = v;
      if (A.volt_host) A.volt_host[gr] = v;
    }
  }
  }  // RTC step
  if (!persist) break;
  // end of a persistent step: the last CTA to finish publishes its id (the
  // voltages written to host memory are made visible to the host first)
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence_system();
    const uint32_t old = atomicAdd(A.ctl + PERSIST_FIN, 1u);
    if (old + 1u == step * gridDim.x) {
      if (s_cmd[0] == 0u) {  // busy time of an RTC step, doorbell seen by CTA 0 to done
        const unsigned long long t0 = *reinterpret_cast<volatile unsigned long long *>(A.ctl + PERSIST_T0);
        atomicAdd(reinterpret_cast<unsigned long long *>(A.ctl + PERSIST_TSUM), global_timer_ns() - t0);
      }
      __threadfence_system();
      atomicExch(A.ctl + PERSIST_DONE, step);
    }
  }
  if (!ok) break;  // a bounded wait expired: leave (the status word says which)
  }  // step loop
  if (persist && threadIdx.x == 0) {
    // release any host stream still waiting for a step that will not run
    __threadfence_system();
    atomicMax(A.ctl + PERSIST_DONE, step + PERSIST_EXIT_AHEAD);
  }
  // no CTA may exit with a copy still landing in its shared memory
  __syncthreads();
  if ((int)threadIdx.x == helper) {
    mbar_wait(&bars[0], 0, ROW_MAX_POLLS);
    mbar_wait(&bars[1], 0, ROW_MAX_POLLS);
  }
}

// ---------------------------------------------------------------------------
template <typename T, int NFFT, int PD>
static bool launch_fused_t(const RtcFusedArgs &A0, int grid, size_t sm, cudaStream_t s, bool dry) {
  auto kern = rtc_fused_kernel<T, NFFT, PD>;
  // The shared-memory opt-in (set once per device to the largest size, so no
  // configuration lowers it under another) and the occupancy answer per size
  // are kept, so a step that launches directly pays for them once.
  struct Fit {
    std::mutex mu;
    std::map<int, size_t> opted;  // dynamic bytes allowed per device (0: the opt-in failed)
    std::map<std::pair<int, size_t>, bool> ok;
  };
  static Fit fit;
  int dev = 0;
  AOB_CUDA(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lock(fit.mu);
    auto od = fit.opted.find(dev);
    if (od == fit.opted.end()) {
      int optin = 0;
      cudaFuncAttributes fa{};
      size_t allow = 0;
      if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess &&
          cudaFuncGetAttributes(&fa, kern) == cudaSuccess && (size_t)optin > fa.sharedSizeBytes) {
        allow = (size_t)optin - fa.sharedSizeBytes;  // the kernel's static shared memory counts against the opt-in
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)allow) != cudaSuccess)
          allow = 0;
      }
      if (!allow) cudaGetLastError();
      od = fit.opted.emplace(dev, allow).first;
    }
    if (sm > od->second) return false;
    auto it = fit.ok.find({dev, sm});
    if (it == fit.ok.end()) {
      int per_sm = 0;
      const bool ok =
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, FUSED_THREADS, sm) == cudaSuccess && per_sm >= 1;
      if (!ok) cudaGetLastError();
      it = fit.ok.emplace(std::make_pair(dev, sm), ok).first;
    }
    if (!it->second) return false;
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

template <typename T, int NFFT>
static bool launch_fused_pd(int pd, const RtcFusedArgs &A, int grid, size_t sm, cudaStream_t s, bool dry) {
  switch (pd) {
    case 4: return launch_fused_t<T, NFFT, 4>(A, grid, sm, s, dry);
    case 6: return launch_fused_t<T, NFFT, 6>(A, grid, sm, s, dry);
    case 8: return launch_fused_t<T, NFFT, 8>(A, grid, sm, s, dry);
    default: return launch_fused_t<T, NFFT, 0>(A, grid, sm, s, dry);
  }
}

template <typename T>
static bool launch_fused_n(int nfft, int pd, const RtcFusedArgs &A, int grid, size_t sm, cudaStream_t s, bool dry) {
  if (nfft == 16) return launch_fused_pd<T, 16>(pd, A, grid, sm, s, dry);
  if (nfft == 32) return launch_fused_pd<T, 32>(pd, A, grid, sm, s, dry);
  return launch_fused_pd<T, 64>(pd, A, grid, sm, s, dry);
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
  if (perturbed || c->open_loop || centro->type > 2 || c->kind != AOB_CTRL_LS || w->fs_n || w->fakecam) return false;
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
  A.volt_host = io_volt;
  A.grid_polls = test_grid_polls ? test_grid_polls : GRID_MAX_POLLS;
  A.absent_cta = test_absent_cta;
  A.ctl = persist_launch ? persist_ctl.p : nullptr;
  A.door_polls = persist_door_polls;
  const int nsm = num_sms(w->device);
  const int grid = std::min(nsm, c->nactu);
  AOB_REQUIRE((int64_t)c->nactu * grid < (int64_t)1 << 32, "loop: too many actuators for the fused kernel");
  A.rows_per_cta = (c->nactu + grid - 1) / grid;
  // sub-apertures per CTA and round: the CTA's whole share if shared memory allows
  const size_t fixed = fused_bars_bytes(A.rows_per_cta) + fused_pre_bytes(A.rows_per_cta) +
                       (size_t)A.rows_per_cta * A.ld * esize + sizeof(float) * swizzled_slope_floats(A.ld, V);
  const int npix2 = w->npix * w->npix;
  const int share = (w->nvalid + grid - 1) / grid;
  int batch = fused_batch > 0 ? std::min(fused_batch, share) : share;
  auto smem_for = [&](int b) {
    const ShSmem L(w->nfft, w->nu, w->nv, w->nphase, w->nrebin * w->nrebin * npix2, npix2, b);
    // the sensor work area holds the MVM's per-warp partial sums afterwards
    return fixed + std::max(L.bytes(), L.hdr + sizeof(float) * (FUSED_THREADS / 32) * A.rows_per_cta);
  };
  while (batch > 1 && smem_for(batch) > 227 * 1024) --batch;
  A.batch = std::max(batch, 1);
  const size_t sm = smem_for(A.batch);
  if (sm > 227 * 1024) return false;
  bool ok;
  if (c->prec == AOB_PREC_F32)
    ok = launch_fused_n<float>(w->nfft, w->nphase, A, grid, sm, s, dry);
  else if (c->prec == AOB_PREC_BF16)
    ok = launch_fused_n<__nv_bfloat16>(w->nfft, w->nphase, A, grid, sm, s, dry);
  else
    ok = launch_fused_n<__nv_fp8_e4m3>(w->nfft, w->nphase, A, grid, sm, s, dry);
  if (!ok || dry) return ok;
  AOB_LAUNCH_CHECK("rtc_fused_kernel");
  if (persist_launch) return true;  // the steps run, and are accounted for, one doorbell at a time
  w->after_image(A.sh, fc, false);
  if (A.delayed) {
    aob::DevBuf<float> t = std::move(c->ring.front());
    c->ring.pop_front();
    c->ring.push_back(std::move(t));
  }
  return true;
}
