// Geometric slopes of a sensor's phase (SutraWfs::slopes_geom,
// libsutra/src.cpp/sutra_wfs.cpp:199-251), for the Shack-Hartmann and the
// pyramid sensor.  Three methods, as the reference numbers them:
//   0  edge differences: per sub-aperture the mean over the nphase rows of
//      (last - first sample) along x, and over columns along y, times
//      alpha = 0.206265 / subapd * nphase / (nphase - 1)   (reduce_phasex/y,
//      libsutra/src.cu/sutra_wfs.cu:866-910);
//   1  pupil-weighted centred differences (one-sided at the edges) summed over
//      the sub-aperture, / nphase / 2 * alpha / fluxPerSub   (derive_phasex/y,
//      sutra_wfs.cu:912-970);
//   2  the tip/tilt projection: ttprojmat^T times the gathered phase samples
//      (phase_project, sutra_wfs.cu:1049-1082).
// One warp per sub-aperture; the lanes stride over the samples and combine by
// shuffles in a fixed order, so results are deterministic.

#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "aob_objects.hpp"

namespace aob {

struct GeomArgs {
  const float *phase, *pupil, *flux, *ttp;
  const int32_t *pmap;
  float *out;
  int n, nvalid, type;
  float alpha;
};

__global__ void slopes_geom_kernel(GeomArgs A) {
  const int k = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (k >= A.nvalid) return;  // whole warps leave together
  const int n = A.n, n2 = n * n;
  const int32_t *ix = A.pmap + (size_t)k * n2;
  const float *ph = A.phase;
  float sx = 0.f, sy = 0.f;
  if (A.type == 0) {
    for (int t = lane; t < n; t += 32) {
      sx += ph[ix[t * n + n - 1]] - ph[ix[t * n]];
      sy += ph[ix[(n - 1) * n + t]] - ph[ix[t]];
    }
  } else if (A.type == 1) {
    for (int i = lane; i < n2; i += 32) {
      const int a = i % n;
      const float m = A.pupil[ix[i]];
      const float dx = a == 0 ? ph[ix[i + 1]] - ph[ix[i]]
                              : (a == n - 1 ? ph[ix[i]] - ph[ix[i - 1]] : ph[ix[i + 1]] - ph[ix[i - 1]]);
      const float dy = i < n ? ph[ix[i + n]] - ph[ix[i]]
                             : (i >= n * (n - 1) ? ph[ix[i]] - ph[ix[i - n]] : ph[ix[i + n]] - ph[ix[i - n]]);
      sx += dx * m;
      sy += dy * m;
    }
  } else {
    const float *mx = A.ttp + (size_t)k * n2, *my = A.ttp + ((size_t)A.nvalid + k) * n2;
    for (int j = lane; j < n2; j += 32) {
      const float v = ph[ix[j]];
      sx += mx[j] * v;
      sy += my[j] * v;
    }
  }
  sx = warp_sum(sx);
  sy = warp_sum(sy);
  if (lane == 0) {
    if (A.type == 0) {
      A.out[k] = sx / n * A.alpha;
      A.out[A.nvalid + k] = sy / n * A.alpha;
    } else if (A.type == 1) {
      A.out[k] = sx / n * A.alpha / A.flux[k] / 2;
      A.out[A.nvalid + k] = sy / n / 2 * A.alpha / A.flux[k];
    } else {
      A.out[k] = sx;
      A.out[A.nvalid + k] = sy;
    }
  }
}

// host side shared by both sensors
static void slopes_geom_launch(int device, int type, const DevBuf<float> &phase, const DevBuf<float> &pupil,
                               const DevBuf<float> &flux, const DevBuf<int32_t> &pmap, const DevBuf<float> &ttp,
                               int nphase, int nvalid, float subapd, float *out, cudaStream_t s) {
  AOB_REQUIRE(type >= 0 && type <= 2, "slopes_geom: type must be 0 (reduce), 1 (derive) or 2 (projection)");
  AOB_REQUIRE(pmap.p != nullptr && pmap.n == (int64_t)nphase * nphase * nvalid,
              "slopes_geom: the phasemap has not been loaded (load_arrays)");
  AOB_REQUIRE(nphase >= 2, "slopes_geom: nphase must be >= 2");
  AOB_REQUIRE(type != 1 || (flux.p != nullptr && flux.n >= nvalid && pupil.p != nullptr),
              "slopes_geom: method 1 needs fluxPerSub and the pupil");
  AOB_REQUIRE(type != 2 || (ttp.p != nullptr && ttp.n == 2LL * nphase * nphase * nvalid),
              "slopes_geom: method 2 needs the tip/tilt projection matrix (load_arrays ttprojmat)");
  AOB_CUDA(cudaSetDevice(device));
  GeomArgs A{};
  A.phase = phase.p;
  A.pupil = pupil.p;
  A.flux = flux.p;
  A.ttp = ttp.p;
  A.pmap = pmap.p;
  A.out = out;
  A.n = nphase;
  A.nvalid = nvalid;
  A.type = type;
  // the reference evaluates 0.206265 / subapd * nphase / (nphase - 1) in double
  A.alpha = (float)(0.206265 / (double)subapd * nphase / (nphase - 1));
  const int threads = 256, warps = threads / 32;
  slopes_geom_kernel<<<(nvalid + warps - 1) / warps, threads, 0, s>>>(A);
  AOB_LAUNCH_CHECK("slopes_geom_kernel");
}

}  // namespace aob

using namespace aob;

extern "C" int aob_sh_slopes_geom(aob_sh *h, int type, float *dev_slopes, void *stream) {
  try {
    if (!h) throw Error("aob_sh_slopes_geom: null handle");
    slopes_geom_launch(h->device, type, h->phase, h->pupil, h->fluxPerSub, h->phasemap, h->ttprojmat, h->nphase,
                       h->nvalid, h->pdiam, dev_slopes ? dev_slopes : h->slopes.p,
                       reinterpret_cast<cudaStream_t>(stream));
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}

extern "C" int aob_pyr_slopes_geom(aob_pyr *h, int type, float *dev_slopes, void *stream) {
  try {
    if (!h) throw Error("aob_pyr_slopes_geom: null handle");
    if (!dev_slopes && h->slopes.n != 2LL * h->nvalid) {
      AOB_CUDA(cudaSetDevice(h->device));
      h->slopes.alloc(2LL * h->nvalid);
    }
    slopes_geom_launch(h->device, type, h->phase, h->pupil, h->fluxPerSub, h->phasemap, h->ttprojmat, h->nphase,
                       h->nvalid, h->pdiam, dev_slopes ? dev_slopes : h->slopes.p,
                       reinterpret_cast<cudaStream_t>(stream));
    return AOB_OK;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return AOB_ERR;
  }
}
