// Host objects of the closed-loop support (sim.cu).
#pragma once

#include <memory>
#include <vector>

#include "aob_common.cuh"

namespace aob {

constexpr int RAY_MAX = 8;
struct RaySources {
  int n;
  const float *data[RAY_MAX];
  int dim[RAY_MAX];
  float xoff[RAY_MAX], yoff[RAY_MAX];
};

void raytrace(float *out, int nx, int ny, const RaySources &S, bool reset, cudaStream_t s);

// One extrusion step (sim.cu): the new column/row y = A z + amp B xi + ref from the
// stencil of `screen`, then the shift of the screen by one sample with y inserted.
__global__ void extrude_gemv_kernel(const float *screen, int n, int nst, const float *Arm, const float *Brm,
                                    const uint32_t *ist, int x0ref, float amp, uint32_t k0, uint32_t k1,
                                    uint32_t counter, uint32_t layer, float *y);
__global__ void extrude_shift_kernel(float *dst, const float *src, const float *y, int n, int dir);

// The same extrusion for several independent layers in one launch (sim.cu):
// one job per layer, each writing the next screen `dst` from the current `src`.
constexpr int EXTRUDE_MAX_JOBS = 16;
struct ExtrudeJob {
  const float *src;
  float *dst;
  const float *Arm, *Brm;
  const uint32_t *ist;
  int n, nst, dir, x0ref;
  float amp;
  uint32_t k0, k1, counter, layer;
};
struct ExtrudeBatch {
  int njobs;
  ExtrudeJob job[EXTRUDE_MAX_JOBS];
};
void launch_extrude(const ExtrudeBatch &B, int device, cudaStream_t s);
void kolmo_factor_ab(int device, int n, int nst, const double *zz, const double *xz, const double *xx, float *A,
                     float *B);

}  // namespace aob

struct aob_atmos {
  struct Layer {
    int dim, nst;
    float r0_pix, altitude, deltax, deltay, amplitude;
    float accumx = 0.f, accumy = 0.f;
    int64_t seed;
    uint64_t counter = 0;  // extrusions so far (noise stream counter)
    int cur = 0;           // which of the two screens is current
    int device = 0;        // the atmosphere's device (grid sizing)
    aob::DevBuf<float> scr[2], Arm, Brm;
    aob::DevBuf<uint32_t> istx, isty;
    Layer(int dim, int nst, float r0, float alt, float dx, float dy, int64_t seed);
    // the next extrusion as a job (current screen -> the other one); flips the
    // current screen and advances the noise counter, the launch is the caller's
    aob::ExtrudeJob next_job(int dir, int layer_index);
    void extrude(int dir, int layer_index, cudaStream_t s);
  };
  int device = 0;
  std::vector<std::unique_ptr<Layer>> layers;
  explicit aob_atmos(int dev) : device(dev) {}
  int add_screen(int dim, int nst, float r0_pix, float alt, float dx, float dy, const float *A, const float *B,
                 const uint32_t *istx, const uint32_t *isty, int64_t seed);
  void refresh(int idx, cudaStream_t s);
  void move(cudaStream_t s);
};

struct aob_dm {
  int device, dim, nact, influsize;
  int64_t nnz = 0;
  aob::DevBuf<int32_t> rowptr, actidx;
  aob::DevBuf<float> weight, shape, com;
  aob_dm(int device, int dim, int nact, int influsize, const float *influ, const int32_t *i1, const int32_t *j1);
  void comp_shape(const float *dev_com, cudaStream_t s);
};

struct aob_target {
  int device, npup, nfft;
  float lambda;
  int64_t npts = 0;
  int le_count = 0;
  aob::DevBuf<float> mask, phase, se, le;
  aob::DevBuf<float2> amp;
  aob::DevBuf<unsigned int> maxes;
  aob::DevBuf<unsigned long long> fit_best;  // argmax key of the sinc fit
  aob::DevBuf<float> fit_win;                // its 7 x 7 window
  aob_target(int device, int npup, int nfft, const float *pupil, float lambda_um);
  void comp_image(const float *dev_phase, bool comp_le, cudaStream_t s);
  void strehl(float *sr_se, float *sr_le, cudaStream_t s);
  void reset_le(cudaStream_t s);
  float fit_peak(const float *img, cudaStream_t s);
  void strehl_fit(float *sr_se, float *sr_le, cudaStream_t s);
};
