// One RTC iteration with the learned reconstructor in one cooperative kernel:
// Shack-Hartmann image + fused centroids (sh_core.cuh) -> grid barrier -> the
// control step of mlp_fused.cuh (three layers + linear skip, threshold test,
// then the integrator or the LS fallback) -> each command row's voltage (delay
// ring, clip; sutra_controller.cpp:205-263) in the thread that wrote it.
//
// At entry the last warp's first thread prefetches the CTA's slice of the phase
// screen into L2, bulk-copies the sensor tables into shared memory and issues
// the bulk copies of the CTA's rows of the four weight matrices, so the weight
// stream lands while the sensor stages run.  The result equals, bit for bit,
// the same iteration as separate launches (sensor image with fused centroids,
// the fused control step, the voltage kernel).  Every wait is bounded.

#include <algorithm>
#include <map>
#include <mutex>

#include "aob_objects.hpp"
#include "mlp_fused.cuh"
#include "sh_core.cuh"

namespace aob {

constexpr uint32_t RTC_MLP_TABLE_POLLS = 1u << 22;

struct RtcMlpArgs {
  ShKernelArgs sh;  // sensor; sh.c_slopes is the controller's slope vector
  MlpFusedArgs m;   // control step; m.x is the same slope vector
  int batch;        // sub-apertures per CTA and round
  uint32_t sensor_off;  // byte offset of the sensor region in shared memory
  // voltage stage
  float *oldest;
  const float *second;
  float a, b;
  int delayed;
  float vmin, vmax;
  int do_clip;
  float *volt;       // com_clipped
  float *volt_host;  // caller's pinned host voltages (mapped), also written, or null
};

// the voltage of command row r, as voltage_kernel computes it
struct RtcMlpVoltage {
  float *oldest;
  const float *second;
  float a, b;
  int delayed;
  float vmin, vmax;
  int do_clip;
  float *volt, *volt_host;
  __device__ explicit RtcMlpVoltage(const RtcMlpArgs &A)
      : oldest(A.oldest), second(A.second), a(A.a), b(A.b), delayed(A.delayed), vmin(A.vmin), vmax(A.vmax),
        do_clip(A.do_clip), volt(A.volt), volt_host(A.volt_host) {}
  __device__ void operator()(int r, float c) const {
    float v;
    if (delayed) {
      v = a * oldest[r] + b * second[r];
      oldest[r] = c;
    } else {
      v = c;
    }
    if (do_clip) v = fminf(fmaxf(v, vmin), vmax);
    volt[r] = v;
    if (volt_host) volt_host[r] = v;
  }
};

template <int NFFT, int PD>
__global__ void __launch_bounds__(MLP_FUSED_THREADS, 1) rtc_mlp_kernel(RtcMlpArgs A) {
  extern __shared__ __align__(128) unsigned char sm[];
  // shared memory: control step (mbarrier, vectors, weight rows) | table mbarrier |
  //                sensor tables + batch work area
  const MlpFusedSmem L = mlp_fused_layout<float>(A.m);
  uint64_t *tbar = reinterpret_cast<uint64_t *>(sm + A.sensor_off);
  unsigned char *shm = sm + A.sensor_off + 128;
  const int pd = PD > 0 ? PD : A.sh.pdiam;
  const int npix2 = A.sh.npix * A.sh.npix;
  const ShSmem Ls(NFFT, A.sh.nu, A.sh.nv, pd, A.sh.nrebin2 * npix2, npix2, A.batch);
  const ShSmem L1(NFFT, A.sh.nu, A.sh.nv, pd, A.sh.nrebin2 * npix2, npix2, 1);
  const ShTableCopy tcopy(A.sh, L1);
  const int helper = (int)blockDim.x - 32;
  if ((int)threadIdx.x == helper) {
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
    mbar_init(tbar, 1);
    fence_mbar_init();
    mbar_expect_tx(tbar, tcopy.image_bytes + tcopy.wt_bytes);
    bulk_g2s(shm, A.sh.tblob, tcopy.image_bytes, tbar);
    if (tcopy.wt_bytes) bulk_g2s(shm + L1.wt, A.sh.c_weights, tcopy.wt_bytes, tbar);
    mlp_fused_issue(A.m, sm, L);  // the weight rows, in flight during the sensor stages
  }
  bool tables_in = false;
  auto wait_tables = [&]() {  // every thread, before the first stage that reads the tables
    if (!tables_in) {
      if (!mbar_wait(tbar, 0, RTC_MLP_TABLE_POLLS)) atomicOr(A.m.status, (uint32_t)ERR_MBAR_TIMEOUT);
      tables_in = true;
    }
  };
  sh_load_tables<NFFT>(A.sh, shm, threadIdx.x, blockDim.x, true, tcopy.wt_bytes != 0);
  // ---- sensor images and slopes: this CTA's sub-apertures, A.batch per round ----
  const int nvalid = A.sh.nvalid;
  const Team team{(int)threadIdx.x, (int)blockDim.x, 0};
  const bool one_round = A.batch * (int)gridDim.x >= nvalid;
  const int S1 =
      (int)blockIdx.x < nvalid ? min(A.batch, (nvalid - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x) : 0;
  if (one_round) {
    if (S1 > 0)
      sh_batch<NFFT, PD, TEAM_CTA, decltype(wait_tables), true>(A.sh, blockIdx.x, gridDim.x, S1, shm, shm + Ls.hdr,
                                                                Ls, team, wait_tables);
  } else {
    for (int base = blockIdx.x; base < nvalid; base += A.batch * gridDim.x) {
      const int Sb = min(A.batch, (nvalid - base + (int)gridDim.x - 1) / (int)gridDim.x);
      sh_batch<NFFT, PD>(A.sh, base, gridDim.x, Sb, shm, shm + Ls.hdr, Ls, team, wait_tables);
    }
  }
  wait_tables();  // a CTA without sub-apertures
  // ---- all slopes published; the cube and image are written while the others arrive ----
  const unsigned long long ticket = grid_arrive(A.m.gbar, gridDim.x);
  if (one_round && S1 > 0) sh_store_images(A.sh, blockIdx.x, gridDim.x, S1, shm + Ls.hdr, Ls, team);
  grid_wait(A.m.gbar, ticket, A.m.status);
  // ---- the control step on the slopes, each command row's voltage with it ----
  mlp_fused_body<float>(A.m, sm, L, RtcMlpVoltage(A));
}

template <int NFFT, int PD>
static bool launch_rtc_mlp_t(const RtcMlpArgs &A, int grid, size_t smem, cudaStream_t s, bool dry) {
  auto kern = rtc_mlp_kernel<NFFT, PD>;
  struct Fit {
    std::mutex mu;
    std::map<std::pair<int, size_t>, bool> ok;
  };
  static Fit fit;
  int dev = 0;
  AOB_CUDA(cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lock(fit.mu);
    auto it = fit.ok.find({dev, smem});
    if (it == fit.ok.end()) {
      bool ok = true;
      try {
        smem_opt_in(reinterpret_cast<const void *>(kern), (int)smem);  // only ever raised, per device
      } catch (const std::exception &) {
        cudaGetLastError();
        ok = false;
      }
      int per_sm = 0;
      if (ok && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, MLP_FUSED_THREADS, smem) != cudaSuccess ||
                 per_sm < 1)) {
        cudaGetLastError();
        ok = false;
      }
      it = fit.ok.emplace(std::make_pair(dev, smem), ok).first;
    }
    if (!it->second) return false;
  }
  if (dry) return true;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(MLP_FUSED_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  AOB_CUDA(cudaLaunchKernelEx(&cfg, kern, A));
  AOB_LAUNCH_CHECK("rtc_mlp_kernel");
  return true;
}

template <int NFFT>
static bool launch_rtc_mlp_pd(int pd, const RtcMlpArgs &A, int grid, size_t smem, cudaStream_t s, bool dry) {
  switch (pd) {
    case 4: return launch_rtc_mlp_t<NFFT, 4>(A, grid, smem, s, dry);
    case 6: return launch_rtc_mlp_t<NFFT, 6>(A, grid, smem, s, dry);
    case 8: return launch_rtc_mlp_t<NFFT, 8>(A, grid, smem, s, dry);
    default: return launch_rtc_mlp_t<NFFT, 0>(A, grid, smem, s, dry);
  }
}

}  // namespace aob

using namespace aob;

// The fused iteration with the learned reconstructor, or false when the
// configuration does not fit it (then the caller runs separate launches).
bool aob_loop::launch_mlp(aob_mlp *m, float threshold, bool noise, cudaStream_t s, bool dry) {
  aob_sh *w = wfs;
  aob_ls *c = ls;
  bool perturbed = false;
  for (auto &kv : c->perturb) perturbed |= kv.second.on;
  if (perturbed || c->open_loop || centro->type > 2 || c->kind != AOB_CTRL_LS || w->fs_n || w->fakecam ||
      c->prec != AOB_PREC_F32 || m->device != w->device)
    return false;
  RtcMlpArgs A{};
  size_t mlp_bytes = 0;
  if (!m->fused_args(c, threshold, A.m, mlp_bytes)) return false;
  aob_centro *fc = w->make_args(noise, c->centroids.p, nullptr, A.sh);
  if (fc != centro) return false;
  const int grid = num_sms(w->device);  // the control step's rows are split over one CTA per SM
  A.sensor_off = (uint32_t)((mlp_bytes + 127) / 128 * 128);
  const int npix2 = w->npix * w->npix;
  const int share = (w->nvalid + grid - 1) / grid;
  int batch = share;
  auto smem_for = [&](int b) {
    const ShSmem L(w->nfft, w->nu, w->nv, w->nphase, w->nrebin * w->nrebin * npix2, npix2, b);
    return (size_t)A.sensor_off + 128 + L.bytes();
  };
  while (batch > 1 && smem_for(batch) > 227 * 1024) --batch;
  A.batch = std::max(batch, 1);
  const size_t smem = smem_for(A.batch);
  if (smem > 227 * 1024) return false;
  A.a = c->a;
  A.b = c->b;
  A.delayed = c->delay > 0 ? 1 : 0;
  if (A.delayed) {
    AOB_REQUIRE(c->ring.size() >= 2, "loop.step_mlp: the controller's delay ring is too short");
    A.oldest = c->ring[0].p;
    A.second = c->ring[1].p;
  }
  A.vmin = c->volt_min;
  A.vmax = c->volt_max;
  A.do_clip = c->volt_min < c->volt_max ? 1 : 0;
  A.volt = c->com_clipped.p;
  A.volt_host = io_volt;
  bool ok;
  if (w->nfft == 16)
    ok = launch_rtc_mlp_pd<16>(w->nphase, A, grid, smem, s, dry);
  else if (w->nfft == 32)
    ok = launch_rtc_mlp_pd<32>(w->nphase, A, grid, smem, s, dry);
  else
    ok = launch_rtc_mlp_pd<64>(w->nphase, A, grid, smem, s, dry);
  if (!ok || dry) return ok;
  w->after_image(A.sh, fc, false);
  if (A.delayed) {
    // the oldest buffer now holds a copy of the current command and becomes it
    aob::DevBuf<float> t = std::move(c->ring.front());
    c->ring.pop_front();
    c->ring.push_back(std::move(t));
  }
  return true;
}

void aob_loop::step_mlp(aob_mlp *m, float threshold, const float *host_phase, float *host_voltage, bool noise,
                        cudaStream_t s, bool wait) {
  AOB_REQUIRE(!persist_on, "loop.step_mlp: the persistent kernel is running (persist_step / persist_stop)");
  AOB_REQUIRE(m && ls->nslope == m->nin && ls->nactu == m->nout, "loop.step_mlp: the network's sizes differ");
  AOB_CUDA(cudaSetDevice(wfs->device));
  if (host_phase)
    AOB_CUDA(cudaMemcpyAsync(wfs->phase.p, host_phase, wfs->phase.bytes(), cudaMemcpyHostToDevice, s));
  io_volt = (host_io == 1 && host_voltage && mode != 1)
                ? static_cast<float *>(const_cast<void *>(mapped_view(host_voltage)))
                : nullptr;
  struct Reset {
    float *&p;
    ~Reset() { p = nullptr; }
  } reset_io{io_volt};
  bool fused = false;
  if (mode != 1 && !ls->open_loop) fused = launch_mlp(m, threshold, noise, s, false);
  if (fused) {
    last_kernels = 1;
  } else {
    // separate launches: image with fused centroids into the controller, the
    // control step (fused or multi-kernel), the voltages
    last_kernels = 3;
    wfs->comp_image_to(noise, s, ls->centroids.p, nullptr);
    AOB_REQUIRE(aob_mlp_comp_com(m, ls, threshold, s) == AOB_OK, "loop.step_mlp: " + std::string(aob_last_error()));
    ls->comp_voltage(s);
  }
  if (host_voltage) {
    if (!(io_volt && fused))
      AOB_CUDA(cudaMemcpyAsync(host_voltage, ls->com_clipped.p, ls->com_clipped.bytes(), cudaMemcpyDeviceToHost, s));
    if (wait) AOB_CUDA(cudaStreamSynchronize(s));
  }
}

extern "C" int aob_loop_step_mlp(aob_loop *l, aob_mlp *m, float threshold, const float *host_phase,
                                 float *host_voltage, int noise, void *stream) {
  try {
    if (!l || !m) throw Error("aob_loop_step_mlp: null handle");
    l->step_mlp(m, threshold, host_phase, host_voltage, noise != 0, reinterpret_cast<cudaStream_t>(stream), true);
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

extern "C" int aob_loop_step_mlp_async(aob_loop *l, aob_mlp *m, float threshold, const float *host_phase,
                                       float *host_voltage, int noise, void *stream) {
  try {
    if (!l || !m) throw Error("aob_loop_step_mlp_async: null handle");
    l->step_mlp(m, threshold, host_phase, host_voltage, noise != 0, reinterpret_cast<cudaStream_t>(stream), false);
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}
