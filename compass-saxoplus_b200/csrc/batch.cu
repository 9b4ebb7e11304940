// Batched Monte Carlo: many independent Shack-Hartmann RTC instances of uneven
// size (sub-aperture count, pixels, FFT size, precision) advanced by ONE
// persistent kernel launch per loop step, replayable from a CUDA graph.
//
// The reference has no batched mode: each COMPASS simulation is its own
// process driving its own sensor / centroider / controller objects
// (CompassSupervisor.next, shesha/shesha/supervisor/compassSupervisor.py:
// 175-289), so a Monte Carlo campaign is N sequential or N separate runs.
// Here one launch carries every instance's step:
//
//  * the work is a queue of items in dependency order: "sensor" items (a run
//    of consecutive valid sub-apertures of one instance: image, noise, fused
//    CoG-family slopes -- the stages of sh_core.cuh) and "MVM" items (a block
//    of command-matrix rows of one instance: integrator and voltage in the
//    epilogue).  An instance's MVM items are queued `lag` instances after its
//    sensor items, so HBM streams command matrices while SMs form images;
//  * persistent CTAs take tickets from an atomic head counter (the next ticket
//    is requested while the current item runs).  An MVM item first issues the
//    bulk copies of its rows into shared memory, then waits, bounded, until
//    the instance's sensor-item counter is complete, then stages the slopes and
//    reduces.  Every ticket below an item's was handed to a running CTA before
//    it, so the smallest unfinished ticket never waits on anything unfinished:
//    the queue cannot deadlock, with or without co-residency;
//  * the last CTA to leave resets the head, the per-instance counters and
//    advances each noisy instance's frame, so the launch is self-contained and
//    a captured graph replays it unchanged.
//
// Arithmetic per instance is the standalone one in the same order: the sensor
// stages are the same code with the same deterministic reductions, and the
// MVM reduction is the standalone bulk-copy MVM's split-K (16 warp slots,
// chunk c = lane + 32 (slot + 16 i), per-slot partials added in slot order),
// run here by 8 warps that take two slots each.  Slopes, commands and
// voltages are bit-identical to stepping each instance's own loop.
//
// Tile shapes (sub-apertures per sensor item, threads per sensor team,
// command-matrix bytes per MVM item, the lag, CTAs per SM and the instance
// order) are parameters, chosen by the autotuner in aob200/autotune.py.

#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "aob_objects.hpp"
#include "mvm_core.cuh"
#include "sh_core.cuh"

namespace aob {

constexpr int BATCH_THREADS = 256;
constexpr int BATCH_SLOTS = 16;  // warp slots of the split-K reduction
constexpr int BATCH_RB = 8;      // rows per register block
constexpr int BATCH_MAX_ROWS = 256;  // command-matrix rows per MVM item, at most
constexpr uint32_t DEP_MAX_POLLS = 1u << 22;
constexpr uint32_t BROW_MAX_POLLS = 1u << 22;
enum : uint32_t { ERR_DEP_TIMEOUT = 4u };
enum : int { BI_SENSOR = 0, BI_MVM = 1 };

struct BatchInst {
  ShKernelArgs sh;        // sensor with fused centroider; sh.c_slopes = controller input
  const void *mat;        // packed command-matrix rows
  const float *rscale;    // FP8 row scales or null
  int prec, ld, nrow, ncol;
  float *err, *com, *volt, *volt_out;
  const float *mgain;
  float gain, vmin, vmax;
  int do_clip;
  int cls;    // sensor code path: 0 (Nfft 16, 6 px), 1 (32, 6), 2 (16, any), 3 (32, any)
  int nsensor;  // sensor items of this instance
  int noisy;  // frame advances after the step
  int smax;   // sub-apertures per team and item, at most (sizes a team's work area)
};

struct BatchArgs {
  const BatchInst *inst;
  const int4 *items;  // (instance, kind, first, count)
  int nitems, ninst;
  unsigned int *ctl;   // [0] ticket head, [32] CTAs finished
  unsigned int *done;  // sensor items finished, per instance
  uint32_t *frames;    // noise frame per instance
  uint32_t *status;
  int rows_max;  // MVM rows per item, upper bound
  int team;      // threads per sensor team (32, 64, 128 or 256)
  uint32_t dep_polls;  // poll limit of an MVM item's dependency wait
  uint32_t dep_extra;  // wait-expiry test: items waited for beyond the instance's sensor items (0)
};

__host__ __device__ inline size_t batch_bars_bytes(int rows) { return 128 * (((size_t)rows * 8 + 127) / 128); }
__host__ __device__ inline size_t batch_pre_bytes(int rows) { return 128 * (((size_t)rows * 12 + 127) / 128); }

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// order earlier generic-proxy accesses of shared memory before later bulk copies into it
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Sub-apertures [first, first + count) by the CTA's teams of ``team``
// threads: team t takes first + t + j * nteams, all in one batch.
template <int NFFT, int PD>
__device__ __forceinline__ void sensor_item(const ShKernelArgs &P, int first, int count, int team, int smax,
                                            unsigned char *area, bool reload) {
  const int pd = PD > 0 ? PD : P.pdiam;
  const int nteams = blockDim.x / team, t = threadIdx.x / team;
  const ShSmem L(NFFT, P.nu, P.nv, pd, P.nrebin2 * P.npix * P.npix, P.npix * P.npix, smax);
  if (reload) {
    sh_load_tables<NFFT>(P, area, threadIdx.x, blockDim.x);
    __syncthreads();
  }
  const int S = (count - t + nteams - 1) / nteams;
  if (S > 0) {
    const Team T{(int)threadIdx.x - t * team, team, 1 + t};
    unsigned char *work = area + L.hdr + (size_t)t * L.per_batch;
    if (team == 32)
      sh_batch<NFFT, PD, TEAM_WARP>(P, first + t, nteams, S, area, work, L, T);
    else
      sh_batch<NFFT, PD, TEAM_NAMED>(P, first + t, nteams, S, area, work, L, T);
  }
  __syncthreads();  // every slope of the item written
}

// Rows [r0, r0 + R) of instance ``ii``.  All row copies complete on one
// barrier, which completes one phase per MVM item: its parity is the CTA's
// MVM-item count modulo 2.
template <typename T>
__device__ __forceinline__ void mvm_item(const BatchInst &I, int ii, int r0, int R, const BatchArgs &A,
                                         uint64_t *bars, float *pre, unsigned char *area, uint32_t parity) {
  constexpr int V = RowPack<T>::N;
  constexpr int Q = V / 4;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
  const uint32_t row_bytes = (uint32_t)(I.ld * sizeof(T));
  unsigned char *rows = area;
  float *s_sl = reinterpret_cast<float *>(area + (size_t)R * row_bytes);
  const int nsl = swizzled_slope_floats(I.ld, V);
  float *part = s_sl + nsl;
  const int RM = A.rows_max;
  if (tid == 0) {
    fence_proxy_async_smem();
    const unsigned char *src = static_cast<const unsigned char *>(I.mat) + (size_t)r0 * row_bytes;
    mbar_expect_tx(&bars[0], (uint32_t)R * row_bytes);
    for (int r = 0; r < R; ++r)
      bulk_g2s(rows + (size_t)r * row_bytes, src + (size_t)r * row_bytes, row_bytes, &bars[0]);
  }
  for (int r = tid; r < R; r += nt) {
    const int gr = r0 + r;
    const float sc = I.rscale ? __ldg(I.rscale + gr) : 1.f;
    const float mg = __ldg(I.mgain + gr);
    const float cm = __ldcg(I.com + gr);
    pre[r] = sc;
    pre[RM + r] = mg;
    pre[2 * RM + r] = cm;
  }
  // the instance's slopes are complete once all its sensor items have finished
  __shared__ int s_dep;
  if (tid == 0) {
    int ok = 1;
    uint32_t i = 0;
    const unsigned need = (unsigned)I.nsensor + A.dep_extra;
    while (ld_acquire_u32(&A.done[ii]) < need) {
      if (++i >= A.dep_polls) {
        ok = 0;
        atomicOr(A.status, (uint32_t)ERR_DEP_TIMEOUT);
        break;
      }
      __nanosleep(32);
    }
    s_dep = ok;
  }
  __syncthreads();
  const bool dep_ok = s_dep != 0;
  if (dep_ok) {
    // swizzled staging: group g holds slopes [chunk * V + 4 q, +4) for
    // chunk = (g & 31) + 32 j, g >> 5 = j * Q + q (L2 reads: other CTAs wrote them)
    const float *sl = I.sh.c_slopes;
    for (int g = tid; g < nsl / 4; g += nt) {
      const int l = g & 31, jq = g >> 5;
      const int j = jq / Q, q = jq - j * Q;
      const int src = (l + 32 * j) * V + 4 * q;
      float4 v4;
      if (src + 3 < I.ncol) {
        v4 = __ldcg(reinterpret_cast<const float4 *>(sl + src));
      } else {
        v4.x = src < I.ncol ? __ldcg(sl + src) : 0.f;
        v4.y = src + 1 < I.ncol ? __ldcg(sl + src + 1) : 0.f;
        v4.z = src + 2 < I.ncol ? __ldcg(sl + src + 2) : 0.f;
        v4.w = 0.f;
      }
      reinterpret_cast<float4 *>(s_sl)[g] = v4;
    }
  }
  bool rows_ok = true;
  rows_ok = mbar_wait(&bars[0], parity, BROW_MAX_POLLS);
  rows_ok = __syncthreads_and(rows_ok) != 0;  // also publishes the staged slopes
  if (!rows_ok && tid == 0) atomicOr(A.status, (uint32_t)ERR_MBAR_TIMEOUT);
  if (dep_ok && rows_ok) {
    const int nchunk = I.ld / V;
    const float4 *sv4 = reinterpret_cast<const float4 *>(s_sl);
    for (int rb = 0; rb < R; rb += BATCH_RB) {
      for (int slot = warp; slot < BATCH_SLOTS; slot += nw) {
        float acc[BATCH_RB];
#pragma unroll
        for (int u = 0; u < BATCH_RB; ++u) acc[u] = 0.f;
        for (int jj = slot; 32 * jj + lane < nchunk; jj += BATCH_SLOTS) {
          const int c = lane + 32 * jj;
          float4 sv[Q];
#pragma unroll
          for (int q = 0; q < Q; ++q) sv[q] = sv4[(jj * Q + q) * 32 + lane];
#pragma unroll
          for (int u = 0; u < BATCH_RB; ++u)
            if (rb + u < R) {
              const uint4 q4 = reinterpret_cast<const uint4 *>(rows + (size_t)(rb + u) * row_bytes)[c];
              acc[u] += RowPack<T>::dot(q4, sv);
            }
        }
        int u;
        const float t = warp_sum8(acc, lane, u);
        if ((lane & 3) == 0 && rb + u < R) part[slot * R + rb + u] = t;
      }
    }
    __syncthreads();
    for (int r = tid; r < R; r += nt) {
      float tot = 0.f;
#pragma unroll
      for (int w = 0; w < BATCH_SLOTS; ++w) tot += part[w * R + r];
      const int gr = r0 + r;
      if (I.rscale) tot *= pre[r];
      const float e = -tot;
      I.err[gr] = e;
      const float c = I.gain * (e * pre[RM + r]) + pre[2 * RM + r];
      I.com[gr] = c;
      float v = c;
      if (I.do_clip) v = fminf(fmaxf(v, I.vmin), I.vmax);
      I.volt[gr] = v;
      if (I.volt_out) I.volt_out[gr] = v;
    }
  } else if (!rows_ok && tid == 0) {
    // no copy may still be landing when this area is reused
    mbar_wait(&bars[0], parity, BROW_MAX_POLLS);
  }
  __syncthreads();
}

// MINB: CTAs per SM the register budget is sized for (2: up to 128
// registers per thread, 4: up to 64)
template <int MINB>
__global__ void __launch_bounds__(BATCH_THREADS, MINB) batch_step_kernel(BatchArgs A) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ __align__(16) BatchInst s_I;
  __shared__ int s_ticket;
  const int tid = threadIdx.x;
  uint64_t *bars = reinterpret_cast<uint64_t *>(sm);
  float *pre = reinterpret_cast<float *>(sm + batch_bars_bytes(A.rows_max));
  unsigned char *area = sm + batch_bars_bytes(A.rows_max) + batch_pre_bytes(A.rows_max);
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    fence_mbar_init();
    s_ticket = (int)atomicAdd(&A.ctl[0], 1u);
  }
  __syncthreads();
  int t = s_ticket;
  int cur = -1;     // instance held in s_I
  int tables = -1;  // instance whose sensor tables are in the area
  uint32_t parity = 0;
  while (t < A.nitems) {
    unsigned nxt = 0;
    if (tid == 0) nxt = atomicAdd(&A.ctl[0], 1u);  // consumed after this item
    const int4 it = A.items[t];
    if (it.x != cur) {
      const uint32_t *src = reinterpret_cast<const uint32_t *>(A.inst + it.x);
      uint32_t *dst = reinterpret_cast<uint32_t *>(&s_I);
      for (int w = tid; w < (int)(sizeof(BatchInst) / 4); w += blockDim.x) dst[w] = __ldg(src + w);
      cur = it.x;
      __syncthreads();
    }
    if (it.y == BI_SENSOR) {
      const bool reload = tables != it.x;
      switch (s_I.cls) {
        case 0: sensor_item<16, 6>(s_I.sh, it.z, it.w, A.team, s_I.smax, area, reload); break;
        case 1: sensor_item<32, 6>(s_I.sh, it.z, it.w, A.team, s_I.smax, area, reload); break;
        case 2: sensor_item<16, 0>(s_I.sh, it.z, it.w, A.team, s_I.smax, area, reload); break;
        default: sensor_item<32, 0>(s_I.sh, it.z, it.w, A.team, s_I.smax, area, reload); break;
      }
      tables = it.x;
      if (tid == 0) {
        __threadfence();
        atomicAdd(&A.done[it.x], 1u);
      }
    } else {
      if (s_I.prec == AOB_PREC_F32)
        mvm_item<float>(s_I, it.x, it.z, it.w, A, bars, pre, area, parity);
      else if (s_I.prec == AOB_PREC_BF16)
        mvm_item<__nv_bfloat16>(s_I, it.x, it.z, it.w, A, bars, pre, area, parity);
      else
        mvm_item<__nv_fp8_e4m3>(s_I, it.x, it.z, it.w, A, bars, pre, area, parity);
      parity ^= 1u;
      tables = -1;  // the rows overwrote the tables
    }
    if (tid == 0) s_ticket = (int)nxt;
    __syncthreads();
    t = s_ticket;
  }
  // the last CTA out re-arms the queue for the next launch (all its threads:
  // one pass over the instances instead of a serial chain of round trips)
  __shared__ int s_last;
  if (tid == 0) {
    __threadfence();
    s_last = atomicAdd(&A.ctl[32], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    for (int i = tid; i < A.ninst; i += blockDim.x) {
      A.done[i] = 0u;
      if (__ldg(&A.inst[i].noisy)) A.frames[i] += 1u;
    }
    __syncthreads();
    if (tid == 0) {
      A.ctl[0] = 0u;
      A.ctl[32] = 0u;
      __threadfence();
    }
  }
}

}  // namespace aob

using namespace aob;

aob_batch::aob_batch(int device_) : device(device_) {}

aob_batch::~aob_batch() { drop_graphs(); }

void aob_batch::drop_graphs() {
  for (auto &g : graphs)
    if (g) cudaGraphExecDestroy(g);
  graphs[0] = graphs[1] = nullptr;
}

void aob_batch::add(aob_loop *l) {
  AOB_REQUIRE(l != nullptr, "batch.add: null loop");
  AOB_REQUIRE(l->wfs->device == device, "batch.add: loop on another device");
  AOB_REQUIRE(std::find(loops.begin(), loops.end(), l) == loops.end(), "batch.add: loop added twice");
  loops.push_back(l);
  built = false;
}

void aob_batch::set_tuning(int subaps_, int team_, int mvm_kb_, int lag_, int ctas_per_sm_, int order_) {
  AOB_REQUIRE(subaps_ >= 0 && subaps_ <= 1024, "batch.set_tuning: subaps_per_item must be in [0, 1024]");
  AOB_REQUIRE(team_ == 0 || team_ == 32 || team_ == 64 || team_ == 128 || team_ == 256,
              "batch.set_tuning: team_threads must be 0, 32, 64, 128 or 256");
  AOB_REQUIRE(mvm_kb_ >= 0 && mvm_kb_ <= 200, "batch.set_tuning: mvm_kb must be in [0, 200]");
  AOB_REQUIRE(lag_ >= 0 && lag_ <= 1024, "batch.set_tuning: lag must be in [0, 1024]");
  AOB_REQUIRE(ctas_per_sm_ >= 0 && ctas_per_sm_ <= 4, "batch.set_tuning: ctas_per_sm must be in [0, 4]");
  AOB_REQUIRE(order_ == 0 || order_ == 1, "batch.set_tuning: order must be 0 or 1");
  subaps = subaps_;
  team = team_;
  mvm_kb = mvm_kb_;
  lag = lag_;
  ctas_per_sm = ctas_per_sm_;
  order = order_;
  built = false;
}

uint64_t aob_batch::key(bool noise) const {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&h](const void *p, size_t n) {
    const unsigned char *b = (const unsigned char *)p;
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  };
  mix(&noise, sizeof noise);
  const int tune[6] = {subaps, team, mvm_kb, lag, ctas_per_sm, order};
  mix(tune, sizeof tune);
  for (const aob_loop *l : loops) {
    const uint64_t k = l->key(noise);
    mix(&k, sizeof k);
    const void *p[4] = {l->ls->com(), l->ls->com_clipped.p, l->ls->centroids.p, l->wfs->phase.p};
    mix(p, sizeof p);
  }
  return h;
}

// Snapshot every instance's parameters, cut the work into items and upload.
void aob_batch::build(bool noise) {
  AOB_REQUIRE(!loops.empty(), "batch: no instances added");
  AOB_CUDA(cudaSetDevice(device));
  const int n = (int)loops.size();
  const int nsm = num_sms(device);
  std::vector<BatchInst> hi(n);
  std::vector<int64_t> cost(n);
  phase_off.assign(n, 0);
  volt_off.assign(n, 0);
  int64_t pf = 0, vf = 0;
  for (int i = 0; i < n; ++i) {
    phase_off[i] = pf;
    volt_off[i] = vf;
    pf += (int64_t)loops[i]->wfs->npup * loops[i]->wfs->npup;
    vf += loops[i]->ls->nactu;
  }
  if (phase_all.n != pf) phase_all.alloc(pf);
  if (volt_all.n != vf) volt_all.alloc(vf);
  if (frames.n != n) frames.alloc(n);
  if (done.n != n) done.alloc(n);
  if (ctl.n != 64) ctl.alloc(64);
  if (status.n != 1) status.alloc(1);
  AOB_CUDA(cudaMemset(done.p, 0, done.bytes()));
  AOB_CUDA(cudaMemset(ctl.p, 0, ctl.bytes()));
  AOB_CUDA(cudaMemset(status.p, 0, status.bytes()));
  std::vector<uint32_t> hf(n);
  frame_seen.assign(n, 0);
  h_frames.assign(n, 0);

  // dynamic shared memory per CTA (static shared memory and the per-block
  // reservation come on top), minus a fixed header for BATCH_MAX_ROWS rows of
  // barriers and epilogue inputs, is what one item may use
  const int cps = ctas_per_sm > 0 ? ctas_per_sm : 2;
  const size_t smem_cap = std::min<size_t>((size_t)226 * 1024, ((size_t)228 / cps - 2) * 1024);
  const size_t item_cap = smem_cap - batch_bars_bytes(BATCH_MAX_ROWS) - batch_pre_bytes(BATCH_MAX_ROWS);
  const size_t kb = mvm_kb > 0 ? (size_t)mvm_kb * 1024 : (size_t)48 * 1024;
  std::vector<int> S(n), RPI(n);
  int rmax = 1;
  alg_bytes = 0;
  for (int i = 0; i < n; ++i) {
    aob_loop *l = loops[i];
    aob_sh *w = l->wfs;
    aob_ls *c = l->ls;
    bool perturbed = false;
    for (auto &kv : c->perturb) perturbed |= kv.second.on;
    AOB_REQUIRE(!perturbed && !c->open_loop && c->delay == 0.f && c->kind == AOB_CTRL_LS && !l->wfs->fs_n &&
                    !l->wfs->fakecam,
                "batch: instance " + std::to_string(i) +
                    ": needs an LS controller with delay 0, closed loop, no perturbation, no field stop, no fakecam");
    AOB_REQUIRE(w->nfft == 16 || w->nfft == 32, "batch: instance " + std::to_string(i) + ": nfft must be 16 or 32");
    c->ensure_packed(c->prec);
    BatchInst &I = hi[i];
    std::memset(&I, 0, sizeof I);
    aob_centro *fc = w->make_args(noise, c->centroids.p, frames.p + i, I.sh);
    AOB_REQUIRE(fc == l->centro, "batch: instance " + std::to_string(i) + ": centroider cannot be fused");
    const int esize = c->prec == AOB_PREC_F32 ? 4 : (c->prec == AOB_PREC_BF16 ? 2 : 1);
    const int V = 16 / esize;
    I.prec = c->prec;
    I.ld = (c->nslope + V - 1) / V * V;
    I.mat = c->prec == AOB_PREC_F32 ? (const void *)c->cm_f32.p
                                    : (c->prec == AOB_PREC_BF16 ? (const void *)c->cm_bf16.p : (const void *)c->cm_fp8.p);
    I.rscale = c->prec == AOB_PREC_FP8 ? c->row_scale.p : nullptr;
    I.nrow = c->nactu;
    I.ncol = c->nslope;
    I.err = c->err.p;
    I.com = c->com();
    I.volt = c->com_clipped.p;
    I.volt_out = volt_all.p + volt_off[i];
    I.mgain = c->gains.p;
    I.gain = c->gain;
    I.vmin = c->volt_min;
    I.vmax = c->volt_max;
    I.do_clip = c->volt_min < c->volt_max ? 1 : 0;
    I.cls = (w->nfft == 16 ? 0 : 1) + (w->nphase == 6 ? 0 : 2);
    I.noisy = (noise && w->noise > -1.f) ? 1 : 0;
    hf[i] = (uint32_t)w->frame;
    frame_seen[i] = w->frame;
    // sensor items: `subaps` sub-apertures each, split over the CTA's teams
    const int npix2 = w->npix * w->npix;
    const int tm = team_threads();
    int s = std::max(1, std::min(subaps > 0 ? subaps : 32, w->nvalid));
    auto sh_bytes = [&](int b) {
      const int smax = (b + BATCH_THREADS / tm - 1) / (BATCH_THREADS / tm);
      const ShSmem L(w->nfft, w->nu, w->nv, w->nphase, w->nrebin * w->nrebin * npix2, npix2, smax);
      return L.team_bytes(BATCH_THREADS / tm);
    };
    while (s > 1 && sh_bytes(s) > item_cap) --s;
    AOB_REQUIRE(sh_bytes(s) <= item_cap, "batch: instance " + std::to_string(i) + ": a sensor item does not fit");
    S[i] = s;
    I.smax = (s + BATCH_THREADS / tm - 1) / (BATCH_THREADS / tm);
    I.nsensor = (w->nvalid + s - 1) / s;
    // MVM items: about `kb` bytes of rows each
    const size_t row_bytes = (size_t)I.ld * esize;
    const size_t slope_b = sizeof(float) * swizzled_slope_floats(I.ld, V);
    int r = (int)std::max<size_t>(1, kb / row_bytes);
    r = std::min(r, c->nactu);
    auto mvm_bytes = [&](int rr) { return (size_t)rr * row_bytes + slope_b + sizeof(float) * BATCH_SLOTS * rr; };
    r = std::min(r, BATCH_MAX_ROWS);
    while (r > 1 && mvm_bytes(r) > item_cap) --r;
    AOB_REQUIRE(mvm_bytes(r) <= item_cap, "batch: instance " + std::to_string(i) + ": a command-matrix row does not fit");
    // even split of the rows over the items
    const int nit = (c->nactu + r - 1) / r;
    RPI[i] = (c->nactu + nit - 1) / nit;
    rmax = std::max(rmax, RPI[i]);
    cost[i] = (int64_t)w->nvalid * w->nfft * w->nfft + (int64_t)c->nactu * I.ld * esize / 8;
    const int64_t pd2 = (int64_t)w->nphase * w->nphase;
    alg_bytes += (int64_t)c->nactu * I.ld * esize             // command matrix
                 + 2 * 4 * pd2 * w->nvalid                     // phase + pupil samples
                 + 2 * 4 * (int64_t)c->nslope                  // slopes written, read back
                 + 4 * 4 * (int64_t)c->nactu;                  // com read + write, err, voltage
  }
  // the area must hold every item's shared memory with the final rows_max
  size_t area = 0;
  for (int i = 0; i < n; ++i) {
    aob_loop *l = loops[i];
    aob_sh *w = l->wfs;
    const int npix2 = w->npix * w->npix;
    const ShSmem L(w->nfft, w->nu, w->nv, w->nphase, w->nrebin * w->nrebin * npix2, npix2, hi[i].smax);
    const int esize = hi[i].prec == AOB_PREC_F32 ? 4 : (hi[i].prec == AOB_PREC_BF16 ? 2 : 1);
    const int V = 16 / esize;
    const size_t mv = (size_t)RPI[i] * hi[i].ld * esize + sizeof(float) * swizzled_slope_floats(hi[i].ld, V) +
                      sizeof(float) * BATCH_SLOTS * RPI[i];
    area = std::max(area, std::max(L.team_bytes(BATCH_THREADS / team_threads()), mv));
  }
  smem = batch_bars_bytes(rmax) + batch_pre_bytes(rmax) + area;
  AOB_REQUIRE(smem <= smem_cap, "batch: shared memory per CTA exceeds the budget");
  rows_max = rmax;

  // queue: sensor items of instance k, then MVM items of instance k - lag
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  if (order == 0) std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<int4> items;
  auto emit_sensor = [&](int i) {
    const int nv = loops[i]->wfs->nvalid;
    for (int f = 0; f < nv; f += S[i]) items.push_back(make_int4(i, BI_SENSOR, f, std::min(S[i], nv - f)));
  };
  auto emit_mvm = [&](int i) {
    const int na = loops[i]->ls->nactu;
    for (int r0 = 0; r0 < na; r0 += RPI[i]) items.push_back(make_int4(i, BI_MVM, r0, std::min(RPI[i], na - r0)));
  };
  for (int k = 0; k < n + lag; ++k) {
    if (k < n) emit_sensor(ord[k]);
    if (k - lag >= 0) emit_mvm(ord[k - lag]);
  }
  nitems = (int)items.size();
  d_items.alloc(nitems);
  AOB_CUDA(cudaMemcpy(d_items.p, items.data(), sizeof(int4) * nitems, cudaMemcpyHostToDevice));
  AOB_CUDA(cudaMemcpy(frames.p, hf.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
  // two instance tables: phases read from each sensor's buffer, or from the staging buffer
  for (int v = 0; v < 2; ++v) {
    std::vector<BatchInst> t = hi;
    if (v == 1)
      for (int i = 0; i < n; ++i) t[i].sh.phase = phase_all.p + phase_off[i];
    d_inst[v].alloc((int64_t)sizeof(BatchInst) * n);
    AOB_CUDA(cudaMemcpy(d_inst[v].p, t.data(), sizeof(BatchInst) * n, cudaMemcpyHostToDevice));
  }
  auto kern = cps <= 2 ? batch_step_kernel<2> : batch_step_kernel<4>;
  smem_opt_in(reinterpret_cast<const void *>(kern), (int)smem);  // only ever raised, per device
  int per_sm = 0;
  AOB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BATCH_THREADS, smem));
  AOB_REQUIRE(per_sm >= 1, "batch: the kernel does not fit on an SM");
  grid = nsm * std::min(per_sm, cps);
  // the resets above ran on the legacy stream; the steps may use any stream
  AOB_CUDA(cudaDeviceSynchronize());
  drop_graphs();
  built = true;
  built_key = key(noise);
}

void aob_batch::launch(bool staged, cudaStream_t s) {
  BatchArgs A{};
  A.inst = reinterpret_cast<const BatchInst *>(d_inst[staged ? 1 : 0].p);
  A.items = d_items.p;
  A.nitems = nitems;
  A.ninst = (int)loops.size();
  A.ctl = ctl.p;
  A.done = done.p;
  A.frames = frames.p;
  A.status = status.p;
  A.rows_max = rows_max;
  A.team = team_threads();
  A.dep_polls = test_dep_polls ? test_dep_polls : DEP_MAX_POLLS;
  A.dep_extra = test_dep_extra;
  if (ctas_per_sm == 0 || ctas_per_sm <= 2)
    batch_step_kernel<2><<<grid, BATCH_THREADS, smem, s>>>(A);
  else
    batch_step_kernel<4><<<grid, BATCH_THREADS, smem, s>>>(A);
  AOB_LAUNCH_CHECK("batch_step_kernel");
}

// One step of every instance.  staged: phases come from the staging buffer
// (host copies), otherwise from each sensor's own phase buffer.
void aob_batch::device_step(bool noise, bool staged, cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  const uint64_t k = key(noise);
  if (!built || k != built_key) {
    AOB_CUDA(cudaStreamSynchronize(s));
    build(noise);
  }
  // a sensor stepped outside the batch moved its frame: re-sync the device copies
  bool resync = false;
  for (size_t i = 0; i < loops.size(); ++i) {
    h_frames[i] = (uint32_t)loops[i]->wfs->frame;
    resync |= loops[i]->wfs->frame != frame_seen[i];
  }
  if (resync) {
    // pageable source: the copy is staged before the call returns
    AOB_CUDA(cudaMemcpyAsync(frames.p, h_frames.data(), sizeof(uint32_t) * loops.size(), cudaMemcpyHostToDevice, s));
    for (size_t i = 0; i < loops.size(); ++i) frame_seen[i] = loops[i]->wfs->frame;
  }
  const int v = staged ? 1 : 0;
  if (!use_graph) {
    launch(staged, s);
  } else {
    if (!graphs[v]) {
      cudaStream_t cs;
      AOB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        try {
          launch(staged, cs);
        } catch (...) {
          cudaStreamEndCapture(cs, &g);
          if (g) cudaGraphDestroy(g);
          cudaStreamDestroy(cs);
          throw;
        }
        e = cudaStreamEndCapture(cs, &g);
      }
      cudaStreamDestroy(cs);
      AOB_CUDA(e);
      cudaGraphExec_t ge = nullptr;
      e = cudaGraphInstantiate(&ge, g, 0);
      cudaGraphDestroy(g);
      AOB_CUDA(e);
      graphs[v] = ge;
    }
    AOB_CUDA(cudaGraphLaunch(graphs[v], s));
  }
  // host mirrors of what the kernel advanced
  for (size_t i = 0; i < loops.size(); ++i) {
    aob_sh *w = loops[i]->wfs;
    if (noise && w->noise > -1.f) {
      ++w->frame;
      ++frame_seen[i];
    }
    ++w->image_gen;
  }
}

void aob_batch::step_host(const float *host_phase, float *host_volt, bool noise, cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  const uint64_t k = key(noise);
  if (!built || k != built_key) {
    AOB_CUDA(cudaStreamSynchronize(s));
    build(noise);
  }
  if (host_phase)
    AOB_CUDA(cudaMemcpyAsync(phase_all.p, host_phase, phase_all.bytes(), cudaMemcpyHostToDevice, s));
  device_step(noise, host_phase != nullptr, s);
  if (host_volt) {
    AOB_CUDA(cudaMemcpyAsync(host_volt, volt_all.p, volt_all.bytes(), cudaMemcpyDeviceToHost, s));
    AOB_CUDA(cudaStreamSynchronize(s));
  }
}

// ---------------------------------------------------------------------------
extern "C" {

#define BATCH_TRY try {
#define BATCH_END                   \
  return AOB_OK;                    \
  }                                 \
  catch (const std::exception &e) { \
    aob::set_last_error(e.what());  \
    return AOB_ERR;                 \
  }
#define BATCH_NEED(p) \
  if (!(p)) throw aob::Error(std::string(__func__) + ": null handle or pointer")

int aob_batch_create(aob_batch **out, int device) {
  BATCH_TRY BATCH_NEED(out);
  *out = nullptr;
  AOB_CUDA(cudaSetDevice(device));
  *out = new aob_batch(device);
  BATCH_END
}
int aob_batch_destroy(aob_batch *b) {
  BATCH_TRY if (b) {
    cudaSetDevice(b->device);
    delete b;
  }
  BATCH_END
}
int aob_batch_add(aob_batch *b, aob_loop *loop) {
  BATCH_TRY BATCH_NEED(b);
  b->add(loop);
  BATCH_END
}
int aob_batch_set_tuning(aob_batch *b, int subaps_per_item, int team_threads, int mvm_kb, int lag, int ctas_per_sm,
                         int order) {
  BATCH_TRY BATCH_NEED(b);
  b->set_tuning(subaps_per_item, team_threads, mvm_kb, lag, ctas_per_sm, order);
  BATCH_END
}
int aob_batch_use_graph(aob_batch *b, int enable) {
  BATCH_TRY BATCH_NEED(b);
  b->use_graph = enable != 0;
  BATCH_END
}
int aob_batch_test_wait_expiry(aob_batch *b, uint32_t polls, int noise, void *stream) {
  BATCH_TRY BATCH_NEED(b);
  AOB_REQUIRE(polls >= 1, "aob_batch_test_wait_expiry: polls >= 1 required");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  struct Restore {
    aob_batch *b;
    bool g;
    ~Restore() {
      b->test_dep_polls = 0;
      b->test_dep_extra = 0;
      b->use_graph = g;
    }
  } restore{b, b->use_graph};
  b->use_graph = false;  // the test values are kernel arguments: a direct launch
  b->test_dep_polls = polls;
  b->test_dep_extra = 1;
  b->device_step(noise != 0, false, s);
  AOB_CUDA(cudaStreamSynchronize(s));
  BATCH_END
}
int aob_batch_refresh(aob_batch *b) {
  BATCH_TRY BATCH_NEED(b);
  b->built = false;
  BATCH_END
}
int aob_batch_step(aob_batch *b, int noise, void *stream) {
  BATCH_TRY BATCH_NEED(b);
  b->device_step(noise != 0, false, reinterpret_cast<cudaStream_t>(stream));
  BATCH_END
}
int aob_batch_step_host(aob_batch *b, const float *host_phases, float *host_volts, int noise, void *stream) {
  BATCH_TRY BATCH_NEED(b);
  b->step_host(host_phases, host_volts, noise != 0, reinterpret_cast<cudaStream_t>(stream));
  BATCH_END
}
int aob_batch_info(aob_batch *b, int64_t *info, int n) {
  BATCH_TRY BATCH_NEED(b);
  BATCH_NEED(info);
  if (!b->built) b->build(true);
  const int64_t v[8] = {(int64_t)b->loops.size(), b->nitems, b->grid, (int64_t)b->smem, b->rows_max,
                        b->alg_bytes, b->phase_all.n, b->volt_all.n};
  for (int i = 0; i < n && i < 8; ++i) info[i] = v[i];
  BATCH_END
}
int aob_batch_offsets(aob_batch *b, int64_t *phase_off, int64_t *volt_off) {
  BATCH_TRY BATCH_NEED(b);
  if (!b->built) b->build(true);
  for (size_t i = 0; i < b->loops.size(); ++i) {
    if (phase_off) phase_off[i] = b->phase_off[i];
    if (volt_off) volt_off[i] = b->volt_off[i];
  }
  BATCH_END
}
int aob_batch_time(aob_batch *b, int noise, int warmup, int iters, float *ms_per_step) {
  BATCH_TRY BATCH_NEED(b);
  BATCH_NEED(ms_per_step);
  AOB_REQUIRE(warmup >= 0 && iters >= 1, "aob_batch_time: warmup >= 0 and iters >= 1 required");
  AOB_CUDA(cudaSetDevice(b->device));
  cudaStream_t s;
  AOB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  try {
    for (int i = 0; i < warmup; ++i) b->device_step(noise != 0, false, s);
    AOB_CUDA(cudaEventRecord(e0, s));
    for (int i = 0; i < iters; ++i) b->device_step(noise != 0, false, s);
    AOB_CUDA(cudaEventRecord(e1, s));
    AOB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    AOB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *ms_per_step = ms / (float)iters;
  } catch (...) {
    cudaStreamSynchronize(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  BATCH_END
}
int aob_batch_status(aob_batch *b, uint32_t *status) {
  BATCH_TRY BATCH_NEED(b);
  BATCH_NEED(status);
  *status = 0;
  if (b->status.p) AOB_CUDA(cudaMemcpy(status, b->status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  BATCH_END
}

}  // extern "C"
