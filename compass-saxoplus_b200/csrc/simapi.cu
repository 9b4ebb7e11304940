// extern "C" entry points of the closed-loop support objects (sim.cu).

#include <cstring>
#include <string>

#include "aob_objects.hpp"
#include "sim.hpp"

using aob::Error;

#define API_TRY try {
#define API_END                      \
  return AOB_OK;                     \
  }                                  \
  catch (const std::exception &e) {  \
    aob::set_last_error(e.what());   \
    return AOB_ERR;                  \
  }
#define NEED(p) \
  if (!(p)) throw Error(std::string(__func__) + ": null handle or pointer")
static inline cudaStream_t S(void *p) { return reinterpret_cast<cudaStream_t>(p); }

extern "C" {

int aob_atmos_create(aob_atmos **out, int device) {
  API_TRY NEED(out);
  *out = nullptr;
  AOB_CUDA(cudaSetDevice(device));
  *out = new aob_atmos(device);
  API_END
}
int aob_atmos_destroy(aob_atmos *a) {
  API_TRY if (a) {
    cudaSetDevice(a->device);
    delete a;
  }
  API_END
}
int aob_atmos_add_screen(aob_atmos *a, int dim, int nst, float r0, float alt, float dx, float dy, const float *A,
                         const float *B, const uint32_t *istx, const uint32_t *isty, int64_t seed, int *index) {
  API_TRY NEED(a);
  const int i = a->add_screen(dim, nst, r0, alt, dx, dy, A, B, istx, isty, seed);
  if (index) *index = i;
  API_END
}
int aob_atmos_refresh_screen(aob_atmos *a, int idx, void *stream) {
  API_TRY NEED(a);
  a->refresh(idx, S(stream));
  API_END
}
int aob_atmos_move(aob_atmos *a, void *stream) {
  API_TRY NEED(a);
  a->move(S(stream));
  API_END
}
int aob_atmos_screen(aob_atmos *a, int idx, void **p, int *dim, float *ax, float *ay) {
  API_TRY NEED(a);
  if (idx < 0 || idx >= (int)a->layers.size()) throw Error("atmos.screen: index out of range");
  auto &L = *a->layers[idx];
  if (p) *p = L.scr[L.cur].p;
  if (dim) *dim = L.dim;
  if (ax) *ax = L.accumx;
  if (ay) *ay = L.accumy;
  API_END
}
int aob_atmos_nscreens(aob_atmos *a, int *n) {
  API_TRY NEED(a); NEED(n);
  *n = (int)a->layers.size();
  API_END
}
int aob_kolmo_factor_ab(int device, int n, int nst, const double *zz, const double *xz, const double *xx, float *A,
                        float *B) {
  API_TRY NEED(zz); NEED(xz); NEED(xx); NEED(A); NEED(B);
  if (n <= 0 || nst <= 0) throw Error("kolmo_factor_ab: sizes must be > 0");
  aob::kolmo_factor_ab(device, n, nst, zz, xz, xx, A, B);
  API_END
}

int aob_dm_create(aob_dm **out, int device, int dim, int nact, int isz, const float *influ, const int32_t *i1,
                  const int32_t *j1) {
  API_TRY NEED(out);
  *out = nullptr;
  *out = new aob_dm(device, dim, nact, isz, influ, i1, j1);
  API_END
}
int aob_dm_destroy(aob_dm *d) {
  API_TRY if (d) {
    cudaSetDevice(d->device);
    delete d;
  }
  API_END
}
int aob_dm_comp_shape(aob_dm *d, const float *com, void *stream) {
  API_TRY NEED(d);
  d->comp_shape(com, S(stream));
  API_END
}
int aob_dm_buffer(aob_dm *d, const char *which, void **p, int64_t *n) {
  API_TRY NEED(d); NEED(which); NEED(p); NEED(n);
  std::string w(which);
  if (w == "shape") {
    *p = d->shape.p;
    *n = d->shape.n;
  } else if (w == "com") {
    *p = d->com.p;
    *n = d->com.n;
  } else {
    throw Error("dm.buffer: unknown buffer '" + w + "'");
  }
  API_END
}

int aob_raytrace(float *out, int nx, int ny, int nsrc, const float *const *screens, const int *dims, const float *xoff,
                 const float *yoff, int reset, void *stream) {
  API_TRY NEED(out);
  if (nsrc < 0 || nsrc > aob::RAY_MAX) throw Error("raytrace: at most 8 screens per call");
  if (nx <= 0 || ny <= 0) throw Error("raytrace: bad output size");
  aob::RaySources R{};
  R.n = nsrc;
  for (int k = 0; k < nsrc; ++k) {
    NEED(screens[k]);
    R.data[k] = screens[k];
    R.dim[k] = dims[k];
    R.xoff[k] = xoff[k];
    R.yoff[k] = yoff[k];
    if (!(xoff[k] >= 0.f) || !(yoff[k] >= 0.f)) throw Error("raytrace: offsets must be >= 0");
  }
  aob::raytrace(out, nx, ny, R, reset != 0, S(stream));
  API_END
}

int aob_target_create(aob_target **out, int device, int npup, int nfft, const float *pupil, float lambda_um) {
  API_TRY NEED(out); NEED(pupil);
  *out = nullptr;
  *out = new aob_target(device, npup, nfft, pupil, lambda_um);
  API_END
}
int aob_target_destroy(aob_target *t) {
  API_TRY if (t) {
    cudaSetDevice(t->device);
    delete t;
  }
  API_END
}
int aob_target_comp_image(aob_target *t, const float *phase, int comp_le, void *stream) {
  API_TRY NEED(t);
  t->comp_image(phase, comp_le != 0, S(stream));
  API_END
}
int aob_target_strehl(aob_target *t, float *se, float *le, void *stream) {
  API_TRY NEED(t);
  t->strehl(se, le, S(stream));
  API_END
}
int aob_target_strehl_fit(aob_target *t, float *se, float *le, void *stream) {
  API_TRY NEED(t);
  t->strehl_fit(se, le, S(stream));
  API_END
}
int aob_target_reset_le(aob_target *t, void *stream) {
  API_TRY NEED(t);
  t->reset_le(S(stream));
  API_END
}
int aob_target_buffer(aob_target *t, const char *which, void **p, int64_t *n) {
  API_TRY NEED(t); NEED(which); NEED(p); NEED(n);
  std::string w(which);
  if (w == "phase") {
    *p = t->phase.p;
    *n = t->phase.n;
  } else if (w == "image_se") {
    *p = t->se.p;
    *n = t->se.n;
  } else if (w == "image_le") {
    *p = t->le.p;
    *n = t->le.n;
  } else if (w == "amplipup") {
    *p = t->amp.p;
    *n = t->amp.n;
  } else {
    throw Error("target.buffer: unknown buffer '" + w + "'");
  }
  API_END
}

}  // extern "C"
