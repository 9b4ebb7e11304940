// Host-side objects behind the C ABI.  Each owns its device buffers; the C
// entry points in capi.cu are thin wrappers that translate exceptions into
// status codes.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "aob200.h"
#include "aob_common.cuh"

struct aob_centro;
namespace aob {
struct MvmArgs;
struct ShKernelArgs;
}

struct aob_mlp;
// Device view of pinned, mapped host memory (nullptr for pageable memory).
const void *mapped_view(const void *p);

// ---------------------------------------------------------------------------
// Shack-Hartmann sensor (replaces SutraWfsSH, libsutra/src.cpp/sutra_wfs_sh.cpp)
struct aob_sh {
  int device = 0;
  int nxsub = 0, nvalid = 0, npix = 0, nphase = 0, nrebin = 0, nfft = 0, ntot = 0, npup = 0;
  float pdiam = 0.f, nphot = 0.f, nphot4imat = 0.f;
  float lambda_um = 0.5f;
  float noise = -1.f;
  int64_t seed = 1234;
  uint64_t frame = 0;
  bool loaded = false;

  // geometry (device)
  aob::DevBuf<float> phase;        // npup x npup guide-star phase [um]
  aob::DevBuf<float> pupil;        // npup x npup amplitude
  aob::DevBuf<int32_t> istart, jstart, validsubsx, validsubsy, binmap;
  aob::DevBuf<int32_t> hrmap;  // nfft^2 positions in the ntot x ntot image (ntot != nfft)
  int fakecam = 0, max_flux_per_pix = 0, max_pix_value = 0;  // uint16 camera frame of each image
  aob::DevBuf<uint16_t> camimg;
  aob::DevBuf<float> cam_dark, cam_flat;
  int fs_n = 0;                // field stop: side of its focal plane (0: none)
  aob::DevBuf<float> fs_mask;  // fs_n x fs_n focal-plane mask (fftshifted)
  aob::DevBuf<float> fs_field; // fs_n x fs_n complex filtered field (float pairs)
  aob::DevBuf<float> offsets, fluxPerSub;
  // geometric slopes (slopes_geom): phase-sample indexes per sub-aperture and
  // the tip/tilt projection matrix, both in the reference's column-major layout
  aob::DevBuf<int32_t> phasemap;  // nphase^2 x nvalid
  aob::DevBuf<float> ttprojmat;   // nphase^2 x 2 nvalid
  // pruned-DFT tables derived from binmap at load time
  int nu = 0, nv = 0;
  aob::DevBuf<int32_t> ulist, vlist, cbin;
  // outputs
  aob::DevBuf<float> bincube, binimg, intensities, slopes;
  aob::DevBuf<float> twiddle;       // exp(-2 pi i m / nfft) as (re, im) pairs
  aob::DevBuf<float> wxy;           // the same values gathered per (frequency, sample)
  aob::DevBuf<int4> tblob;          // shared-memory table image (see ShSmem)
  // centroider whose slopes are fused into comp_image (may be null)
  aob_centro *fused = nullptr;
  uint64_t image_gen = 0;  // bumped whenever binimg changes

  aob_sh(int device, int nxsub, int nvalid, int npix, int nphase, int nrebin, int nfft, int ntot,
         int npup, float pdiam, float nphot, float nphot4imat);
  void set_field_stop(const float *mask, int n);
  void set_fakecam(int enable, int max_flux, int max_pix);
  void digitalize(cudaStream_t s);
  void field_stop_prepare(cudaStream_t s);
  void load_arrays(const int32_t *binmap, const float *offsets, const float *fluxPerSub,
                   const int32_t *validsubsx, const int32_t *validsubsy, const int32_t *istart,
                   const int32_t *jstart, const int32_t *hrmap = nullptr);
  void comp_image(bool noise, cudaStream_t s);
  // slopes_dst: write the fused centroider's slopes there instead of its staging
  // buffer; frame_ptr: read the noise frame number from device memory
  void comp_image_to(bool noise, cudaStream_t s, float *slopes_dst, const uint32_t *frame_ptr);
  void fill_binimage(cudaStream_t s);
  // kernel arguments for one image; returns the fused centroider (or null)
  aob_centro *make_args(bool noise, float *slopes_dst, const uint32_t *frame_ptr, aob::ShKernelArgs &P);
  void after_image(const aob::ShKernelArgs &P, aob_centro *c, bool staged);
  int batch_override = 0;  // sub-apertures per CTA chosen by the autotuner (0 = heuristic)
  size_t smem_bytes(int batch) const;
  int pick_batch() const;
};

// ---------------------------------------------------------------------------
// high-resolution pyramid sensor (replaces SutraWfs_PyrHR)
struct aob_pyr {
  int device = 0;
  int nxsub, nvalid, npix, nphase, nrebin, nfft, ntot, npts = 0;
  int logn = 0;
  float pdiam, nphot, nphot4imat;
  float lambda_um = 0.5f;
  float noise = -1.f;
  int64_t seed = 1234;
  uint64_t frame = 0;
  bool loaded = false;
  uint64_t image_gen = 0;
  aob::DevBuf<float> phase, pupil;                 // ntot x ntot
  aob::DevBuf<float> cx, cy, weights;              // modulation points
  aob::DevBuf<float> submask, sincar;              // nfft x nfft (x fastest)
  aob::DevBuf<float2> phalfxy;                     // exp(i pyramid phase), nfft x nfft
  aob::DevBuf<float2> work;                        // npts x nfft x nfft focal / pupil planes
  aob::DevBuf<float2> conv;                        // nfft x nfft, pixel-transfer convolution
  aob::DevBuf<float> hrimg;                        // nfft x nfft high-resolution image
  aob::DevBuf<float> binimg, partial;              // (nfft/nrebin)^2 image, per-row sums
  aob::DevBuf<int32_t> validsubsx, validsubsy;     // 4 * nvalid pupil-image pixels
  aob::DevBuf<float> fluxPerSub;
  aob::DevBuf<int32_t> phasemap;                   // slopes_geom: nphase^2 x nvalid
  aob::DevBuf<float> ttprojmat;                    // slopes_geom: nphase^2 x 2 nvalid
  aob::DevBuf<float> slopes;                       // 2 nvalid geometric slopes
  bool compute_focalplane = false;                 // accumulate the focal plane image
  aob::DevBuf<float> focalplane;                   // nfft x nfft sum_p w_p |field stop x focal field|^2
  aob::DevBuf<float> focal_work;                   // npts x nfft x nfft, summed in point order

  aob_pyr(int device, int nxsub, int nvalid, int npix, int nphase, int nrebin, int nfft, int ntot, int npts,
          float pdiam, float nphot, float nphot4imat);
  void load_arrays(const float2 *halfxy, const float *cx, const float *cy, const float *weights, const float *sincar,
                   const float *submask, const int32_t *validsubsx, const int32_t *validsubsy,
                   const float *fluxPerSub);
  void set_modulation(const float *cx, const float *cy, const float *weights, int npts);
  void comp_image(bool noise, cudaStream_t s);
  int nbin() const { return nfft / nrebin; }
};

// ---------------------------------------------------------------------------
// centroiders (replaces SutraCentroiderCog / Tcog / Wcog / Pyr)
struct aob_centro {
  int device = 0;
  int type = 0;
  int nvalid = 0;
  int npix = 0;
  float offset = 0.f, scale = 1.f, threshold = 0.f;
  int order = 0;
  aob_sh *wfs = nullptr;
  aob_pyr *pyr = nullptr;       // pyramid centroider: the sensor whose image it reads
  float valid_thresh = 1.e-4f;  // pyramid: flux below which slopes are 0
  int pyr_method = 1;           // pyramid: 0 sinus global, 1 nosinus global, 2 sinus local, 3 nosinus local
  int nmax = 0;                 // bpcog: rank of the threshold pixel (set_nmax)
  aob::DevBuf<int32_t> validx, validy;
  aob::DevBuf<float> ref, weights, intensities;
  aob::DevBuf<float> pyr_partial;  // pyramid slopes: per-CTA flux sums
  int weights_per_sub = 0;  // 0: one npix^2 map, 1: npix^2*nvalid
  // image path when not attached to a sensor (load_img + calibrate_img)
  int img_m = 0, img_n = 0;
  aob::DevBuf<float> img_raw, img, dark, flat;
  aob::DevBuf<uint16_t> img_raw_u16;  // camera frame (Rtc_UFF input)
  bool raw_u16 = false;               // the last loaded frame is uint16
  aob::DevBuf<int32_t> lut;           // pixel look-up table of the calibration
  // fused slopes staged by the sensor kernel
  aob::DevBuf<float> fused_slopes;
  uint64_t fused_gen = ~0ull;     // sensor image generation they belong to
  uint64_t params_gen = 0;        // bumped on every parameter change
  uint64_t fused_params_gen = ~0ull;

  aob_centro(int device, int type, int nvalid, float offset, float scale);
  // slopes this centroider writes: one per valid pixel (maskedpix), else 2 per sub-aperture
  int nslopes() const { return type == AOB_CENTRO_MASKEDPIX ? nvalid : 2 * nvalid; }
  void touch() { ++params_gen; }
  bool fused_ready() const;
  void get_cog(float *dev_slopes, cudaStream_t s);
  void init_calib();
  void calibrate(cudaStream_t s, bool valid_only = false);
};

// ---------------------------------------------------------------------------
// least-squares controller (replaces SutraControllerLs + SutraController)
struct aob_ls {
  int device = 0;
  int nslope = 0, nactu = 0;
  float delay = 0.f, a = 0.f, b = 1.f, gain = 0.f;
  int open_loop = 0;
  float volt_min = -1.0e6f, volt_max = 1.0e6f;
  int prec = 0;
  int nblocks = 0;   // MVM grid size (chosen by the autotuner, 0 = one CTA per SM)
  int mvm_kind = 0;  // 0 auto (bulk copy when it fits), 1 bulk copy, 2 register streaming
  aob::DevBuf<uint32_t> status;  // error word of the MVM kernels

  aob::DevBuf<float> centroids, err, com_clipped, gains, cmat, imat, eigenvals_f;
  std::deque<aob::DevBuf<float>> ring;  // command history, back() = current command
  // packed row-major copies of cmat for the MVM
  int ld = 0;  // elements per packed row
  aob::DevBuf<float> cm_f32;
  aob::DevBuf<uint16_t> cm_bf16;
  aob::DevBuf<uint8_t> cm_fp8;
  aob::DevBuf<float> row_scale;
  bool packed_valid[3] = {false, false, false};
  std::vector<float> h_cmat;  // column-major host copy used for (re)packing
  // FP64 eigen decomposition state (svdec_imat)
  aob::DevBuf<double> U, eig;

  struct Perturb {
    aob::DevBuf<float> buf;
    int n = 0;
    int cpt = 0;
    bool on = true;
  };
  std::map<std::string, Perturb> perturb;

  // generic controller (SutraControllerGeneric): kind AOB_CTRL_GENERIC and its command law
  int kind = AOB_CTRL_LS;
  int law = 0;
  float leaky = 1.f;
  int polc = 0;
  aob::DevBuf<float> decay, matE_rows, imat_rows, ol_meas, com1_tmp;

  aob_ls(int device, int nslope, int nactu, float delay);
  float *com() { return ring.back().p; }
  void set_delay(float d);
  void ensure_packed(int p);
  // use: device flag; when given and 0 the MVM is skipped (learned reconstructor path)
  void comp_com(cudaStream_t s, uint32_t *bump = nullptr, const uint32_t *use = nullptr);
  void launch_mvm(struct aob::MvmArgs &A, cudaStream_t s);
  void comp_voltage(cudaStream_t s);
  void clip(cudaStream_t s);
  void apply_perturb(cudaStream_t s);
  void make_generic();
  void generic_comp_com(cudaStream_t s, uint32_t *bump);
  void set_matE(const float *h_colmajor);
  void set_imat_rows(const float *h_colmajor);
  void svdec_imat();
  void build_cmat(int nfilt);
};

// ---------------------------------------------------------------------------
// one RTC iteration bound to a sensor, a centroider and a controller
struct aob_loop {
  aob_sh *wfs;
  aob_centro *centro;
  aob_ls *ls;
  aob::DevBuf<uint32_t> d_frame;
  bool use_graph = false;
  std::vector<cudaGraphExec_t> graphs;   // one per command-ring rotation
  std::vector<uint64_t> graph_key;       // parameter snapshot each graph was built for
  std::vector<const void *> graph_front; // ring front buffer each graph was built for
  std::vector<int> graph_kernels;        // kernels each graph launches
  uint64_t frame_mirror = ~0ull;         // value held by d_frame
  aob::DevBuf<unsigned long long> gbar;  // grid-barrier arrival counter of the fused kernel
  int mode = 0;                          // 0 auto (fused when it fits), 1 three kernels, 2 fused only
  int fused_batch = 0;                   // max sub-apertures per CTA and round in the fused kernel (0 = all)
  int last_kernels = 3;                  // kernels launched by the last device step
  uint32_t frame_host = 0;
  int host_io = 1;                       // 1: the fused kernel writes pinned host voltages itself
  float *io_volt = nullptr;              // device view of the caller's pinned voltages during a step
  uint32_t test_grid_polls = 0;          // wait-expiry test: grid-barrier poll limit (0 = the default)
  int test_absent_cta = -1;              // wait-expiry test: the CTA that never arrives (-1 = none)
  // persistent mode: the fused kernel resident, one step per doorbell
  aob::DevBuf<uint32_t> persist_ctl;     // doorbell, stop, done, completions (one line each)
  bool persist_on = false;
  bool persist_launch = false;           // launch_fused starts the resident kernel
  bool persist_noise = true;
  uint32_t persist_id = 0;               // id of the last step rung
  uint32_t persist_door_polls = 0;
  cudaStream_t persist_stream = nullptr; // the resident kernel's stream
  cudaStream_t persist_last = nullptr;   // stream of the last step rung
  float *persist_volt = nullptr;         // device view of the pinned voltages the kernel writes
  void persist_start(bool noise, float *host_voltage, uint32_t door_polls);
  void persist_step(const float *host_phase, float *host_voltage, bool noise, cudaStream_t s, bool wait);
  void persist_stop();
  void persist_flush(void *dev_buf, size_t bytes, cudaStream_t s);
  uint32_t persist_cmd = 0;              // last command rung (1: a flush; the next step resets it)
  uint64_t persist_rtc_steps = 0;        // RTC steps rung since persist_start
  // streamed steps (run): the next step's host phase is copied on a stream of
  // its own into one of two staging buffers while the current step computes
  cudaStream_t run_copy = nullptr;
  cudaEvent_t run_entry = nullptr, run_copied[2] = {nullptr, nullptr}, run_used[2] = {nullptr, nullptr};
  aob::DevBuf<float> run_stage[2];
  void run(const float *host_phases, int nphases, int nsteps, float *host_volts, bool noise, cudaStream_t s,
           bool wait);
  void run_release();
  aob_loop(aob_sh *w, aob_centro *c, aob_ls *l);
  ~aob_loop();
  void device_step(bool noise, cudaStream_t s, bool frame_on_device);
  bool launch_fused(bool noise, cudaStream_t s, bool frame_on_device, bool dry);
  // one iteration with the learned reconstructor m (rtc_mlp.cu)
  bool launch_mlp(aob_mlp *m, float threshold, bool noise, cudaStream_t s, bool dry);
  void step_mlp(aob_mlp *m, float threshold, const float *host_phase, float *host_voltage, bool noise,
                cudaStream_t s, bool wait);
  void step(const float *host_phase, float *host_voltage, bool noise, cudaStream_t s, bool wait = true);
  uint64_t key(bool noise) const;
  void drop_graphs();
};

// ---------------------------------------------------------------------------
// many independent loops advanced by one persistent launch per step
// (batched Monte Carlo; no counterpart in the reference)
struct aob_batch {
  int device = 0;
  std::vector<aob_loop *> loops;
  // tuning: sub-apertures per sensor item (0 = 32), threads per sensor team
  // (0 = 32), command-matrix KB per MVM item (0 = 48), MVM items queued `lag`
  // instances after their sensor items, CTAs per SM (0 = 2), instance order
  // (0 = largest first, 1 = as added)
  int subaps = 0, team = 0, mvm_kb = 0, lag = 2, ctas_per_sm = 0, order = 0;
  int team_threads() const { return team > 0 ? team : 32; }
  bool use_graph = true;
  bool built = false;
  uint64_t built_key = 0;
  int grid = 0, nitems = 0, rows_max = 1;
  size_t smem = 0;
  int64_t alg_bytes = 0;  // algorithmic HBM bytes of one step
  std::vector<int64_t> phase_off, volt_off;
  std::vector<uint64_t> frame_seen;  // sensor frames the device counters hold
  std::vector<uint32_t> h_frames;
  aob::DevBuf<unsigned char> d_inst[2];
  aob::DevBuf<int4> d_items;
  aob::DevBuf<unsigned int> ctl, done;
  aob::DevBuf<uint32_t> frames, status;
  aob::DevBuf<float> phase_all, volt_all;  // staging for host phases / gathered voltages
  cudaGraphExec_t graphs[2] = {nullptr, nullptr};
  uint32_t test_dep_polls = 0;  // wait-expiry test: dependency-wait poll limit (0 = the default)
  uint32_t test_dep_extra = 0;  // wait-expiry test: sensor items an MVM item waits for beyond its instance's

  explicit aob_batch(int device);
  ~aob_batch();
  void add(aob_loop *l);
  void set_tuning(int subaps, int team, int mvm_kb, int lag, int ctas_per_sm, int order);
  uint64_t key(bool noise) const;
  void build(bool noise);
  void launch(bool staged, cudaStream_t s);
  void device_step(bool noise, bool staged, cudaStream_t s);
  void step_host(const float *host_phase, float *host_volt, bool noise, cudaStream_t s);
  void drop_graphs();
};

// ---------------------------------------------------------------------------
// learned reconstructor: MLP slopes -> DM commands with a linear skip path
// (no counterpart in the reference)
namespace aob {
struct MlpFusedArgs;
}

struct aob_mlp {
  int device = 0;
  int nin, nh1, nh2, nout;  // as given
  int pin, ph1, ph2, pout;  // padded to multiples of 8
  float in_scale = 1.f, out_scale = 1.f;
  float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  int64_t t = 0;  // Adam steps taken
  // parameters: FP32 masters, BF16 copies, Adam moments, gradients
  // layers 0..2: in -> h1 -> h2 -> out; layer 3: the linear skip in -> out (no bias)
  aob::DevBuf<float> w[4], b[3], mw[4], vw[4], mb[3], vb[3], gw[4], gb[3];
  aob::DevBuf<uint16_t> wb[4];
  // batch workspace
  int cap = 0;
  aob::DevBuf<uint16_t> xb, h1b, h2b, dy, dz2, dz1;
  aob::DevBuf<float> z1, z2, y, loss_part;
  // batch-1 inference
  aob::DevBuf<float> ix, ih1, ih2, iy;
  aob::DevBuf<uint32_t> use_ls, fallbacks;
  // single-launch control step (comp_com_fused)
  int fused_mode = 0;  // 0: fused kernel when it fits, 1: multi-kernel path
  int gemm_kind = 1;   // training GEMMs: 0 mma.sync kernel, 1 tcgen05 kernel
  aob::DevBuf<uint32_t> tc_status;  // bounded waits of the tcgen05 GEMM that expired
  aob::DevBuf<float> splitk;        // split-K partial products of the weight gradients
  aob::DevBuf<float> colsum_part;   // row-chunk partial sums of the bias gradients
  aob::DevBuf<float> partial;
  aob::DevBuf<unsigned long long> gbar;

  aob_mlp(int device, int nin, int nh1, int nh2, int nout);
  int rows(int l) const { return l == 0 ? ph1 : (l == 1 ? ph2 : pout); }
  int cols(int l) const { return l == 0 ? pin : (l == 1 ? ph1 : (l == 2 ? ph2 : pin)); }
  void set_params(int layer, const float *w_host, const float *b_host);
  void get_params(int layer, float *w_host, float *b_host);
  void ensure_batch(int batch);
  void forward(const float *x, int batch, float *y_out, cudaStream_t s);
  void backward(const float *target, int batch, float *loss, cudaStream_t s);
  void adam(float lr, cudaStream_t s);
  void infer(const float *x, float *y_out, cudaStream_t s);
  bool comp_com_fused(aob_ls *ls, float threshold, cudaStream_t s);
  bool fused_args(aob_ls *ls, float threshold, aob::MlpFusedArgs &A, size_t &smem_bytes);
  void colsum(const __nv_bfloat16 *d, int batch, int cols, float *out, cudaStream_t s);
};

namespace aob {
int num_sms(int device);
}
