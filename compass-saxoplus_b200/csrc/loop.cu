// One RTC iteration (sensor image + fused centroids -> MVM + integrator ->
// voltages) bound into one object, optionally replayed from CUDA graphs.
//
// The reference drives these stages as separate Python -> C++ calls, each a
// handful of launches on the default stream with host synchronisation in
// between (CompassSupervisor.next, shesha/shesha/supervisor/
// compassSupervisor.py:175-289).  Here the device part is three kernels on one
// stream: the sensor kernel writes the slopes directly into the controller's
// input vector, the MVM kernel bumps the noise frame counter held in device
// memory (so a captured graph stays valid from one iteration to the next),
// and the voltage kernel applies delay / perturbation / clip.  Because the
// command-history ring rotates every iteration, one graph is captured per
// rotation phase; a graph is rebuilt when a parameter it baked in changes.

#include <cuda.h>

#include <cstring>

#include "aob_objects.hpp"

using namespace aob;

// control-word layout and exit value shared with the kernel (rtc_fused.cu)
namespace aob {
constexpr int PERSIST_DOOR = 0, PERSIST_STOP = 32, PERSIST_DONE = 64, PERSIST_WORDS = 128;
constexpr int PERSIST_CMD = 4, PERSIST_ARG = 8;
constexpr uint32_t PERSIST_DEFAULT_POLLS = 1u << 21;  // ~2 s of polls (an L2 round trip and a 256 ns sleep each)
}

static void cu_check(CUresult r, const char *what) {
  if (r != CUDA_SUCCESS) throw Error(std::string(what) + ": driver error " + std::to_string((int)r));
}

// The driver's stream memory operations, looked up through the runtime (the
// library does not link the driver library itself and still loads on
// machines without it).
using StreamValue32Fn = CUresult (*)(CUstream, CUdeviceptr, cuuint32_t, unsigned int);
static StreamValue32Fn driver_fn(const char *name) {
  void *p = nullptr;
  cudaDriverEntryPointQueryResult q;
  AOB_CUDA(cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q));
  AOB_REQUIRE(p != nullptr && q == cudaDriverEntryPointSuccess, std::string("loop: ") + name + " not available");
  return reinterpret_cast<StreamValue32Fn>(p);
}
static StreamValue32Fn write_value32() {
  static StreamValue32Fn fn = driver_fn("cuStreamWriteValue32");
  return fn;
}
static StreamValue32Fn wait_value32() {
  static StreamValue32Fn fn = driver_fn("cuStreamWaitValue32");
  return fn;
}

aob_loop::aob_loop(aob_sh *w, aob_centro *c, aob_ls *l) : wfs(w), centro(c), ls(l) {
  AOB_REQUIRE(w && c && l, "loop: sensor, centroider and controller are required");
  AOB_REQUIRE(w->device == c->device && w->device == l->device, "loop: objects on different devices");
  AOB_REQUIRE(c->type <= 2, "loop: SH loops need a CoG-family centroider");
  AOB_REQUIRE(2 * w->nvalid == l->nslope, "loop: controller nslope must be 2*nvalid of the sensor");
  AOB_REQUIRE(c->nvalid == w->nvalid, "loop: centroider nvalid differs from the sensor's");
  AOB_CUDA(cudaSetDevice(w->device));
  d_frame.alloc(1);
  gbar.alloc(GRID_WORDS);
  if (c->wfs && c->wfs->fused == c && c->wfs != w) c->wfs->fused = nullptr;
  c->wfs = w;
  w->fused = c;
}

aob_loop::~aob_loop() {
  try {
    persist_stop();
  } catch (...) {
  }
  run_release();
  drop_graphs();
}

void aob_loop::run_release() {
  if (run_copy) {
    cudaStreamSynchronize(run_copy);
    cudaStreamDestroy(run_copy);
    run_copy = nullptr;
  }
  for (cudaEvent_t *e : {&run_entry, &run_copied[0], &run_copied[1], &run_used[0], &run_used[1]})
    if (*e) {
      cudaEventDestroy(*e);
      *e = nullptr;
    }
}

void aob_loop::drop_graphs() {
  for (auto &g : graphs)
    if (g) cudaGraphExecDestroy(g);
  graphs.clear();
  graph_key.clear();
  graph_front.clear();
  graph_kernels.clear();
}

// Everything a captured graph bakes into its kernel parameters.
uint64_t aob_loop::key(bool noise) const {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&h](const void *p, size_t n) {
    const unsigned char *b = (const unsigned char *)p;
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  };
  mix(&noise, sizeof noise);
  mix(&wfs->noise, sizeof wfs->noise);
  mix(&wfs->seed, sizeof wfs->seed);
  mix(&wfs->lambda_um, sizeof wfs->lambda_um);
  mix(&wfs->nphot, sizeof wfs->nphot);
  mix(&centro->params_gen, sizeof centro->params_gen);
  mix(&ls->gain, sizeof ls->gain);
  mix(&ls->a, sizeof ls->a);
  mix(&ls->delay, sizeof ls->delay);  // the delay ring's length and buffers
  const size_t nring = ls->ring.size();
  mix(&nring, sizeof nring);
  mix(&ls->volt_min, sizeof ls->volt_min);
  mix(&ls->volt_max, sizeof ls->volt_max);
  mix(&ls->prec, sizeof ls->prec);
  mix(&ls->nblocks, sizeof ls->nblocks);
  mix(&ls->mvm_kind, sizeof ls->mvm_kind);
  mix(&wfs->batch_override, sizeof wfs->batch_override);
  mix(&mode, sizeof mode);
  mix(&fused_batch, sizeof fused_batch);
  mix(&io_volt, sizeof io_volt);
  const void *pm[4] = {ls->cm_f32.p, ls->cm_bf16.p, ls->cm_fp8.p, centro->weights.p};
  mix(pm, sizeof pm);
  return h;
}

void aob_loop::device_step(bool noise, cudaStream_t s, bool frame_on_device) {
  if (mode != 1) {
    // the fused kernel's grid barrier is a 64-bit arrival counter that every
    // launch raises by exactly its grid size, so it needs no re-arming
    if (launch_fused(noise, s, frame_on_device, true)) {
      if (launch_fused(noise, s, frame_on_device, false)) {
        last_kernels = 1;
        return;
      }
    }
    AOB_REQUIRE(mode != 2, "loop: the fused kernel does not fit this configuration");
  }
  last_kernels = 3;
  const bool noisy = noise && wfs->noise > -1.f;
  wfs->comp_image_to(noise, s, ls->centroids.p, frame_on_device ? d_frame.p : nullptr);
  ls->comp_com(s, (frame_on_device && noisy) ? d_frame.p : nullptr);
  ls->comp_voltage(s);
}

// Device view of pinned, mapped host memory (nullptr for pageable memory).
const void *mapped_view(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

// ---------------------------------------------------------------------------
// Persistent mode: the fused kernel stays resident (its command-matrix rows,
// sensor tables and the integrator state stay in shared memory) and runs one
// step per doorbell.  A step on the caller's stream: the phase copy, a stream
// write of the step id into the doorbell, a stream wait until the kernel
// reports the id done, and the voltages (written into pinned host memory by
// the kernel itself, or copied).  The kernel's waits are bounded; when it
// leaves it sets "done" far ahead, so no stream waits for a step that will
// not run.
void aob_loop::persist_start(bool noise, float *host_voltage, uint32_t door_polls) {
  AOB_REQUIRE(!persist_on, "loop.persist_start: the persistent kernel is already running");
  AOB_CUDA(cudaSetDevice(wfs->device));
  AOB_REQUIRE(ls->delay <= 0.f, "loop.persist_start: the persistent mode needs a controller without delay");
  AOB_REQUIRE(mode != 1, "loop.persist_start: the persistent mode runs the fused kernel (mode 0 or 2)");
  AOB_REQUIRE(launch_fused(noise, nullptr, true, true),
              "loop.persist_start: the fused kernel does not fit this configuration");
  float *volt = nullptr;
  if (host_voltage) {
    volt = static_cast<float *>(const_cast<void *>(mapped_view(host_voltage)));
    AOB_REQUIRE(volt != nullptr, "loop.persist_start: host_voltage must be pinned, mapped host memory");
  }
  if (persist_ctl.n < PERSIST_WORDS) persist_ctl.alloc(PERSIST_WORDS);
  AOB_CUDA(cudaMemset(persist_ctl.p, 0, sizeof(uint32_t) * PERSIST_WORDS));
  // the device frame counter starts at the host's
  frame_host = (uint32_t)wfs->frame;
  AOB_CUDA(cudaMemcpy(d_frame.p, &frame_host, sizeof frame_host, cudaMemcpyHostToDevice));
  frame_mirror = wfs->frame;
  AOB_CUDA(cudaStreamCreateWithFlags(&persist_stream, cudaStreamNonBlocking));
  persist_door_polls = door_polls ? door_polls : PERSIST_DEFAULT_POLLS;
  persist_launch = true;
  io_volt = volt;
  bool ok = false;
  try {
    ok = launch_fused(noise, persist_stream, true, false);
  } catch (...) {
    persist_launch = false;
    io_volt = nullptr;
    cudaStreamDestroy(persist_stream);
    persist_stream = nullptr;
    throw;
  }
  persist_launch = false;
  io_volt = nullptr;
  if (!ok) {
    cudaStreamDestroy(persist_stream);
    persist_stream = nullptr;
    throw Error("loop.persist_start: launch failed");
  }
  persist_on = true;
  persist_noise = noise;
  persist_volt = volt;
  persist_id = 0;
  persist_last = nullptr;
  persist_cmd = 0;
  persist_rtc_steps = 0;
}

void aob_loop::persist_step(const float *host_phase, float *host_voltage, bool noise, cudaStream_t s, bool wait) {
  AOB_REQUIRE(persist_on, "loop.persist_step: the persistent kernel is not running (persist_start)");
  AOB_REQUIRE(noise == persist_noise, "loop.persist_step: the noise setting differs from persist_start's");
  AOB_CUDA(cudaSetDevice(wfs->device));
  if (host_phase)
    AOB_CUDA(cudaMemcpyAsync(wfs->phase.p, host_phase, wfs->phase.bytes(), cudaMemcpyHostToDevice, s));
  const uint32_t id = persist_id + 1;
  CUstream cs = reinterpret_cast<CUstream>(s);
  if (persist_cmd) {  // the previous command was a flush
    cu_check(write_value32()(cs, reinterpret_cast<CUdeviceptr>(persist_ctl.p + PERSIST_CMD), 0u, 0),
             "loop.persist_step: command");
    persist_cmd = 0;
  }
  cu_check(write_value32()(cs, reinterpret_cast<CUdeviceptr>(persist_ctl.p + PERSIST_DOOR), id, 0),
           "loop.persist_step: doorbell");
  cu_check(wait_value32()(cs, reinterpret_cast<CUdeviceptr>(persist_ctl.p + PERSIST_DONE), id,
                          CU_STREAM_WAIT_VALUE_GEQ),
           "loop.persist_step: wait");
  persist_id = id;
  persist_last = s;
  ++persist_rtc_steps;
  if (host_voltage && (persist_volt == nullptr || mapped_view(host_voltage) != persist_volt))
    AOB_CUDA(cudaMemcpyAsync(host_voltage, ls->com_clipped.p, ls->com_clipped.bytes(), cudaMemcpyDeviceToHost, s));
  // host-side state the step corresponds to
  if (noise && wfs->noise > -1.f) {
    ++wfs->frame;
    ++frame_mirror;
  }
  ++wfs->image_gen;
  if (wait) AOB_CUDA(cudaStreamSynchronize(s));
}

void aob_loop::persist_flush(void *dev_buf, size_t bytes, cudaStream_t s) {
  AOB_REQUIRE(persist_on, "loop.persist_flush: the persistent kernel is not running (persist_start)");
  AOB_REQUIRE(dev_buf != nullptr && (reinterpret_cast<uintptr_t>(dev_buf) & 15) == 0 && bytes % 16 == 0,
              "loop.persist_flush: a 16-byte aligned device buffer and a multiple of 16 bytes are required");
  AOB_CUDA(cudaSetDevice(wfs->device));
  const uint32_t id = persist_id + 1;
  CUstream cs = reinterpret_cast<CUstream>(s);
  const uint64_t ptr = reinterpret_cast<uint64_t>(dev_buf), n = bytes;
  const uint32_t w[5] = {1u, (uint32_t)ptr, (uint32_t)(ptr >> 32), (uint32_t)n, (uint32_t)(n >> 32)};
  cu_check(write_value32()(cs, reinterpret_cast<CUdeviceptr>(persist_ctl.p + PERSIST_CMD), w[0], 0),
           "loop.persist_flush: command");
  for (int k = 0; k < 4; ++k)
    cu_check(write_value32()(cs, reinterpret_cast<CUdeviceptr>(persist_ctl.p + PERSIST_ARG + k), w[1 + k], 0),
             "loop.persist_flush: arguments");
  cu_check(write_value32()(cs, reinterpret_cast<CUdeviceptr>(persist_ctl.p + PERSIST_DOOR), id, 0),
           "loop.persist_flush: doorbell");
  cu_check(wait_value32()(cs, reinterpret_cast<CUdeviceptr>(persist_ctl.p + PERSIST_DONE), id,
                          CU_STREAM_WAIT_VALUE_GEQ),
           "loop.persist_flush: wait");
  persist_id = id;
  persist_last = s;
  persist_cmd = 1;
}

void aob_loop::persist_stop() {
  if (!persist_on) return;
  AOB_CUDA(cudaSetDevice(wfs->device));
  persist_on = false;
  // the steps already rung first (the kernel finishes them, or its bounded
  // waits expire and it releases their waits)
  if (persist_last) cudaStreamSynchronize(persist_last);
  // the stop flag through a stream of its own (no implicit ordering with any other)
  cudaStream_t ss = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&ss, cudaStreamNonBlocking);
  if (e == cudaSuccess) {
    CUresult r = CUDA_ERROR_NOT_SUPPORTED;
    try {
      r = write_value32()(reinterpret_cast<CUstream>(ss), reinterpret_cast<CUdeviceptr>(persist_ctl.p + PERSIST_STOP),
                          1u, 0);
    } catch (...) {
    }
    e = r == CUDA_SUCCESS ? cudaStreamSynchronize(ss) : cudaErrorUnknown;
    cudaStreamDestroy(ss);
  }
  const cudaError_t e2 = cudaStreamSynchronize(persist_stream);
  cudaStreamDestroy(persist_stream);
  persist_stream = nullptr;
  persist_last = nullptr;
  persist_volt = nullptr;
  AOB_CUDA(e);
  AOB_CUDA(e2);
}

void aob_loop::step(const float *host_phase, float *host_voltage, bool noise, cudaStream_t s, bool wait) {
  AOB_REQUIRE(!persist_on, "loop.step: the persistent kernel is running (persist_step / persist_stop)");
  AOB_CUDA(cudaSetDevice(wfs->device));
  // the phase copy goes out first: nothing else of the step can start before it lands
  if (host_phase)
    AOB_CUDA(cudaMemcpyAsync(wfs->phase.p, host_phase, wfs->phase.bytes(), cudaMemcpyHostToDevice, s));
  // Direct voltages: with the caller's voltage buffer pinned and mapped, the
  // fused kernel's epilogue writes it as well (posted stores over the bus), so
  // no copy-engine transfer follows the kernel.
  io_volt = (host_io == 1 && host_voltage && mode != 1)
                ? static_cast<float *>(const_cast<void *>(mapped_view(host_voltage)))
                : nullptr;
  struct Reset {
    float *&p;
    ~Reset() { p = nullptr; }
  } reset_io{io_volt};
  bool perturbed = false;
  for (auto &kv : ls->perturb) perturbed |= kv.second.on;
  // A graph only pays for the three-kernel step: the fused step is one
  // kernel, and a one-node graph adds launch latency on the device (measured
  // through aob_loop_step with host buffers: 18.8 k vs 20.7 k steps/s).
  const bool graphable = use_graph && !perturbed && !ls->open_loop && !(mode != 1 && launch_fused(noise, s, false, true));
  if (!graphable) {
    device_step(noise, s, false);
  } else {
    // the ring of command buffers rotates every iteration: the graph for the
    // current rotation is the one captured with the same front buffer
    const void *front = ls->ring.front().p;
    int slot = -1;
    for (size_t i = 0; i < graphs.size(); ++i)
      if (graph_front[i] == front) slot = (int)i;
    if (slot < 0) {
      graphs.push_back(nullptr);
      graph_key.push_back(0);
      graph_front.push_back(front);
      graph_kernels.push_back(0);
      slot = (int)graphs.size() - 1;
    }
    const uint64_t k = key(noise);
    ls->ensure_packed(ls->prec);  // no synchronous copies may happen inside a capture
    // the device frame counter must equal the host one at the start of the step
    if (frame_mirror != wfs->frame) {
      frame_host = (uint32_t)wfs->frame;
      AOB_CUDA(cudaMemcpyAsync(d_frame.p, &frame_host, sizeof frame_host, cudaMemcpyHostToDevice, s));
      frame_mirror = wfs->frame;
    }
    if (!graphs[slot] || graph_key[slot] != k) {
      if (graphs[slot]) cudaGraphExecDestroy(graphs[slot]);
      graphs[slot] = nullptr;
      // capture on a private stream so that the caller's stream may be the legacy default one
      cudaStream_t cs;
      AOB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
      cudaGraph_t g = nullptr;
      const uint64_t frame0 = wfs->frame;
      cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        try {
          device_step(noise, cs, true);
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
      // the capture advanced the host-side state (ring rotation, frame); undo it,
      // the replay below performs the step
      wfs->frame = frame0;
      if (ls->delay > 0) {
        aob::DevBuf<float> t = std::move(ls->ring.back());
        ls->ring.pop_back();
        ls->ring.push_front(std::move(t));
      }
      cudaGraphExec_t ge = nullptr;
      e = cudaGraphInstantiate(&ge, g, 0);
      cudaGraphDestroy(g);
      AOB_CUDA(e);
      graphs[slot] = ge;
      graph_key[slot] = k;
      graph_kernels[slot] = last_kernels;  // set by the captured device step
    }
    AOB_CUDA(cudaGraphLaunch(graphs[slot], s));
    last_kernels = graph_kernels[slot];
    // host-side state the graph's kernels correspond to
    if (noise && wfs->noise > -1.f) {
      ++wfs->frame;
      ++frame_mirror;
    }
    if (ls->delay > 0) {
      aob::DevBuf<float> t = std::move(ls->ring.front());
      ls->ring.pop_front();
      ls->ring.push_back(std::move(t));
    }
    ++wfs->image_gen;
  }
  if (host_voltage) {
    if (!(io_volt && last_kernels == 1))
      AOB_CUDA(cudaMemcpyAsync(host_voltage, ls->com_clipped.p, ls->com_clipped.bytes(), cudaMemcpyDeviceToHost, s));
    if (wait) AOB_CUDA(cudaStreamSynchronize(s));
  }
}

// nsteps iterations with host phases and host voltages, as nsteps calls of
// step() would run them (the same kernels in the same order on s, so the same
// voltages bit for bit), except that the phase of step k + 1 crosses the bus
// while step k computes: it is copied on run_copy into the staging buffer step
// k - 1 used, and step k + 1 starts with a device copy of it into the sensor's
// phase.  Step k reads host_phases[k % nphases] and writes host_volts[k].
void aob_loop::run(const float *host_phases, int nphases, int nsteps, float *host_volts, bool noise, cudaStream_t s,
                   bool wait) {
  AOB_REQUIRE(!persist_on, "loop.run: the persistent kernel is running (persist_step / persist_stop)");
  AOB_REQUIRE(host_phases && nphases >= 1 && nsteps >= 1,
              "loop.run: host_phases, nphases >= 1 and nsteps >= 1 are required");
  AOB_CUDA(cudaSetDevice(wfs->device));
  const int64_t np = wfs->phase.n;
  const size_t pb = wfs->phase.bytes();
  if (!run_copy) {
    AOB_CUDA(cudaStreamCreateWithFlags(&run_copy, cudaStreamNonBlocking));
    AOB_CUDA(cudaEventCreateWithFlags(&run_entry, cudaEventDisableTiming));
    for (int b = 0; b < 2; ++b) {
      AOB_CUDA(cudaEventCreateWithFlags(&run_copied[b], cudaEventDisableTiming));
      AOB_CUDA(cudaEventCreateWithFlags(&run_used[b], cudaEventDisableTiming));
    }
  }
  for (int b = 0; b < 2; ++b)
    if (run_stage[b].n != np) run_stage[b].alloc(np);
  auto phase_of = [&](int k) { return host_phases + (size_t)(k % nphases) * (size_t)np; };
  // the copies start after all the work already queued on s (an earlier run's
  // last steps may still read the staging buffers)
  AOB_CUDA(cudaEventRecord(run_entry, s));
  AOB_CUDA(cudaStreamWaitEvent(run_copy, run_entry, 0));
  AOB_CUDA(cudaMemcpyAsync(run_stage[0].p, phase_of(0), pb, cudaMemcpyHostToDevice, run_copy));
  AOB_CUDA(cudaEventRecord(run_copied[0], run_copy));
  for (int k = 0; k < nsteps; ++k) {
    const int b = k & 1;
    if (k + 1 < nsteps) {
      // buffer 1 - b was last read by step k - 1's device copy
      if (k >= 1) AOB_CUDA(cudaStreamWaitEvent(run_copy, run_used[1 - b], 0));
      AOB_CUDA(cudaMemcpyAsync(run_stage[1 - b].p, phase_of(k + 1), pb, cudaMemcpyHostToDevice, run_copy));
      AOB_CUDA(cudaEventRecord(run_copied[1 - b], run_copy));
    }
    AOB_CUDA(cudaStreamWaitEvent(s, run_copied[b], 0));
    AOB_CUDA(cudaMemcpyAsync(wfs->phase.p, run_stage[b].p, pb, cudaMemcpyDeviceToDevice, s));
    AOB_CUDA(cudaEventRecord(run_used[b], s));
    step(nullptr, host_volts ? host_volts + (size_t)k * (size_t)ls->nactu : nullptr, noise, s, false);
  }
  if (wait) AOB_CUDA(cudaStreamSynchronize(s));
}

extern "C" {

int aob_loop_create(aob_loop **out, aob_sh *wfs, aob_centro *centro, aob_ls *ls) {
  try {
    if (!out) throw Error("aob_loop_create: null out pointer");
    *out = nullptr;
    *out = new aob_loop(wfs, centro, ls);
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

int aob_loop_destroy(aob_loop *l) {
  if (l) {
    cudaSetDevice(l->wfs->device);
    delete l;
  }
  return AOB_OK;
}

int aob_loop_set_host_io(aob_loop *l, int mode) {
  try {
    if (!l) throw Error("aob_loop_set_host_io: null handle");
    AOB_REQUIRE(mode == 0 || mode == 1, "aob_loop_set_host_io: mode must be 0 (copies) or 1 (direct when pinned)");
    l->host_io = mode;
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

int aob_loop_test_wait_expiry(aob_loop *l, uint32_t polls, void *stream) {
  try {
    if (!l) throw Error("aob_loop_test_wait_expiry: null handle");
    AOB_REQUIRE(polls >= 1, "aob_loop_test_wait_expiry: polls >= 1 required");
    AOB_REQUIRE(l->ls->delay == 0.f, "aob_loop_test_wait_expiry: needs a controller without delay");
    AOB_CUDA(cudaSetDevice(l->wfs->device));
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    AOB_REQUIRE(l->launch_fused(false, s, false, true), "aob_loop_test_wait_expiry: the fused kernel does not fit");
    struct Restore {
      aob_loop *l;
      ~Restore() {
        l->test_grid_polls = 0;
        l->test_absent_cta = -1;
      }
    } restore{l};
    l->test_grid_polls = polls;
    l->test_absent_cta = 0;
    AOB_REQUIRE(l->launch_fused(false, s, false, false), "aob_loop_test_wait_expiry: launch failed");
    // CTA 0 never added its arrival: bring the counter back to a multiple of the grid
    AOB_CUDA(cudaMemsetAsync(l->gbar.p, 0, sizeof(unsigned long long) * GRID_WORDS, s));
    AOB_CUDA(cudaStreamSynchronize(s));
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

int aob_loop_persist_start(aob_loop *l, int noise, float *host_voltage, uint32_t door_polls) {
  try {
    if (!l) throw Error("aob_loop_persist_start: null handle");
    l->persist_start(noise != 0, host_voltage, door_polls);
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

int aob_loop_persist_step(aob_loop *l, const float *host_phase, float *host_voltage, int noise, void *stream,
                          int wait) {
  try {
    if (!l) throw Error("aob_loop_persist_step: null handle");
    l->persist_step(host_phase, host_voltage, noise != 0, reinterpret_cast<cudaStream_t>(stream), wait != 0);
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

int aob_loop_persist_flush(aob_loop *l, void *dev_buf, size_t bytes, void *stream) {
  try {
    if (!l) throw Error("aob_loop_persist_flush: null handle");
    l->persist_flush(dev_buf, bytes, reinterpret_cast<cudaStream_t>(stream));
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

int aob_loop_persist_stats(aob_loop *l, uint64_t *steps, uint64_t *busy_ns) {
  try {
    if (!l || !steps || !busy_ns) throw Error("aob_loop_persist_stats: null pointer");
    AOB_REQUIRE(l->persist_ctl.p != nullptr, "aob_loop_persist_stats: the persistent kernel never ran");
    AOB_CUDA(cudaSetDevice(l->wfs->device));
    unsigned long long t = 0;
    // (the control words are read with a copy on a stream of its own: no device-wide wait)
    cudaStream_t ss = nullptr;
    AOB_CUDA(cudaStreamCreateWithFlags(&ss, cudaStreamNonBlocking));
    cudaError_t e = cudaMemcpyAsync(&t, l->persist_ctl.p + 74, sizeof t, cudaMemcpyDeviceToHost, ss);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ss);
    cudaStreamDestroy(ss);
    AOB_CUDA(e);
    *steps = l->persist_rtc_steps;
    *busy_ns = t;
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

int aob_loop_persist_stop(aob_loop *l) {
  try {
    if (!l) throw Error("aob_loop_persist_stop: null handle");
    l->persist_stop();
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

int aob_loop_step(aob_loop *l, const float *host_phase, float *host_voltage, int noise, void *stream) {
  try {
    if (!l) throw Error("aob_loop_step: null handle");
    l->step(host_phase, host_voltage, noise != 0, reinterpret_cast<cudaStream_t>(stream));
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

int aob_loop_step_async(aob_loop *l, const float *host_phase, float *host_voltage, int noise, void *stream) {
  try {
    if (!l) throw Error("aob_loop_step_async: null handle");
    l->step(host_phase, host_voltage, noise != 0, reinterpret_cast<cudaStream_t>(stream), false);
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

int aob_loop_run(aob_loop *l, const float *host_phases, int nphases, int nsteps, float *host_voltages, int noise,
                 void *stream, int wait) {
  try {
    if (!l) throw Error("aob_loop_run: null handle");
    l->run(host_phases, nphases, nsteps, host_voltages, noise != 0, reinterpret_cast<cudaStream_t>(stream),
           wait != 0);
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

int aob_loop_time(aob_loop *l, int noise, int warmup, int iters, float *ms_per_step) {
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  try {
    if (!l || !ms_per_step) throw Error("aob_loop_time: null pointer");
    AOB_REQUIRE(warmup >= 0 && iters >= 1, "aob_loop_time: warmup >= 0 and iters >= 1 required");
    AOB_CUDA(cudaSetDevice(l->wfs->device));
    AOB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    AOB_CUDA(cudaEventCreate(&e0));
    AOB_CUDA(cudaEventCreate(&e1));
    for (int i = 0; i < warmup; ++i) l->step(nullptr, nullptr, noise != 0, s);
    AOB_CUDA(cudaEventRecord(e0, s));
    for (int i = 0; i < iters; ++i) l->step(nullptr, nullptr, noise != 0, s);
    AOB_CUDA(cudaEventRecord(e1, s));
    AOB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    AOB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *ms_per_step = ms / (float)iters;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    return AOB_OK;
  } catch (const std::exception &e) {
    if (s) cudaStreamSynchronize(s);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    set_last_error(e.what());
    return AOB_ERR;
  }
}

int aob_loop_use_graph(aob_loop *l, int enable) {
  if (!l) {
    set_last_error("aob_loop_use_graph: null handle");
    return AOB_ERR;
  }
  l->use_graph = enable != 0;
  if (!l->use_graph) l->drop_graphs();
  return AOB_OK;
}

int aob_loop_kernels_per_step(aob_loop *l, int *n) {
  if (!l || !n) {
    set_last_error("aob_loop_kernels_per_step: null pointer");
    return AOB_ERR;
  }
  *n = l->last_kernels;
  return AOB_OK;
}

int aob_loop_set_mode(aob_loop *l, int mode, int fused_batch) {
  if (!l || mode < 0 || mode > 2 || fused_batch < 0 || fused_batch > 64) {
    set_last_error("aob_loop_set_mode: mode 0..2, fused_batch 0..64");
    return AOB_ERR;
  }
  l->mode = mode;
  l->fused_batch = fused_batch;
  return AOB_OK;
}

}  // extern "C"
