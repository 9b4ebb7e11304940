// extern "C" entry points declared in include/aob200.h.  Every function
// catches exceptions and returns AOB_OK / AOB_ERR; the message is kept per
// thread for aob_last_error().

#include <memory>
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "aob_objects.hpp"

namespace aob {
static thread_local std::string g_last_error;
void set_last_error(const std::string &m) { g_last_error = m; }

int num_sms(int device) {
  static int cache[64] = {0};
  if (device < 0 || device >= 64) device = 0;
  if (cache[device] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || n <= 0) n = 148;
    cache[device] = n;
  }
  return cache[device];
}
}  // namespace aob

using aob::Error;

#define AOB_API_BEGIN try {
#define AOB_API_END                                  \
  return AOB_OK;                                     \
  }                                                  \
  catch (const std::exception &e) {                  \
    aob::set_last_error(e.what());                   \
    return AOB_ERR;                                  \
  }                                                  \
  catch (...) {                                      \
    aob::set_last_error("unknown error");            \
    return AOB_ERR;                                  \
  }

static inline cudaStream_t S(void *p) { return reinterpret_cast<cudaStream_t>(p); }
#define NEED(ptr) \
  if (!(ptr)) throw Error(std::string(__func__) + ": null handle or pointer")

extern "C" {

const char *aob_last_error(void) { return aob::g_last_error.c_str(); }
const char *aob_version(void) { return "aob200 0.1.0 (sm_100a)"; }

int aob_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int aob_device_name(int device, char *buf, int len, int *num_sms) {
  AOB_API_BEGIN
  NEED(buf);
  cudaDeviceProp prop;
  AOB_CUDA(cudaGetDeviceProperties(&prop, device));
  if (len > 0) {
    std::strncpy(buf, prop.name, (size_t)len - 1);
    buf[len - 1] = 0;
  }
  if (num_sms) *num_sms = prop.multiProcessorCount;
  AOB_API_END
}

int aob_memcpy_d2h(void *dst, const void *src, size_t bytes, void *stream) {
  AOB_API_BEGIN
  if (bytes == 0) return AOB_OK;
  NEED(dst); NEED(src);
  AOB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, S(stream)));
  AOB_CUDA(cudaStreamSynchronize(S(stream)));
  AOB_API_END
}
int aob_memcpy_h2d(void *dst, const void *src, size_t bytes, void *stream) {
  AOB_API_BEGIN
  if (bytes == 0) return AOB_OK;
  NEED(dst); NEED(src);
  AOB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, S(stream)));
  AOB_CUDA(cudaStreamSynchronize(S(stream)));
  AOB_API_END
}
int aob_memcpy_h2d_async(void *dst, const void *src, size_t bytes, void *stream) {
  AOB_API_BEGIN
  if (bytes == 0) return AOB_OK;
  NEED(dst); NEED(src);
  AOB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, S(stream)));
  AOB_API_END
}
int aob_memcpy_d2d(void *dst, const void *src, size_t bytes, void *stream) {
  AOB_API_BEGIN
  if (bytes == 0) return AOB_OK;
  NEED(dst); NEED(src);
  AOB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, S(stream)));
  AOB_API_END
}
int aob_malloc(void **p, size_t bytes, int device) {
  AOB_API_BEGIN
  NEED(p);
  AOB_CUDA(cudaSetDevice(device));
  AOB_CUDA(cudaMalloc(p, bytes));
  AOB_CUDA(cudaMemset(*p, 0, bytes));
  AOB_API_END
}
int aob_free(void *p) {
  AOB_API_BEGIN
  if (p) AOB_CUDA(cudaFree(p));
  AOB_API_END
}
int aob_stream_sync(void *stream) {
  AOB_API_BEGIN
  AOB_CUDA(cudaStreamSynchronize(S(stream)));
  AOB_API_END
}

__global__ void aob_fill_kernel(float *p, size_t n, float v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}
int aob_fill_f32(float *dev, size_t n, float value, void *stream) {
  AOB_API_BEGIN
  if (n == 0) return AOB_OK;
  NEED(dev);
  aob_fill_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, S(stream)>>>(dev, n, value);
  AOB_LAUNCH_CHECK("aob_fill_kernel");
  AOB_API_END
}

// ---------------------------------------------------------------- SH sensor
int aob_sh_create(aob_sh **out, int device, int nxsub, int nvalid, int npix, int nphase, int nrebin, int nfft,
                  int ntot, int npup, float pdiam, float nphot, float nphot4imat) {
  AOB_API_BEGIN
  NEED(out);
  *out = nullptr;
  *out = new aob_sh(device, nxsub, nvalid, npix, nphase, nrebin, nfft, ntot, npup, pdiam, nphot, nphot4imat);
  AOB_API_END
}
int aob_sh_destroy(aob_sh *h) {
  AOB_API_BEGIN
  if (h) {
    cudaSetDevice(h->device);
    if (h->fused) h->fused->wfs = nullptr;
    delete h;
  }
  AOB_API_END
}
// phasemap / ttprojmat (optional): kept for slopes_geom; every phasemap entry
// must index the phase screen
static void load_geom_arrays(int device, aob::DevBuf<int32_t> &pm, aob::DevBuf<float> &tt, const int32_t *phasemap,
                             const float *ttprojmat, int nphase, int nvalid, int64_t nscreen) {
  const int64_t m = (int64_t)nphase * nphase * nvalid;
  AOB_CUDA(cudaSetDevice(device));
  if (phasemap) {
    for (int64_t i = 0; i < m; ++i)
      if (phasemap[i] < 0 || phasemap[i] >= nscreen) throw Error("load_arrays: phasemap entry outside the phase screen");
    if (pm.n != m) pm.alloc(m);
    pm.upload(phasemap, m);
  }
  if (ttprojmat) {
    if (tt.n != 2 * m) tt.alloc(2 * m);
    tt.upload(ttprojmat, 2 * m);
  }
}

int aob_sh_load_arrays(aob_sh *h, const int32_t *phasemap, const int32_t *hrmap, const int32_t *binmap,
                       const float *offsets, const float *flux, const int32_t *vx, const int32_t *vy,
                       const int32_t *istart, const int32_t *jstart, const float *ttprojmat, const float *) {
  AOB_API_BEGIN
  NEED(h);
  h->load_arrays(binmap, offsets, flux, vx, vy, istart, jstart, hrmap);
  load_geom_arrays(h->device, h->phasemap, h->ttprojmat, phasemap, ttprojmat, h->nphase, h->nvalid, h->phase.n);
  AOB_API_END
}
int aob_sh_set_fakecam(aob_sh *h, int enable, int max_flux_per_pix, int max_pix_value) {
  AOB_API_BEGIN
  NEED(h);
  h->set_fakecam(enable, max_flux_per_pix, max_pix_value);
  AOB_API_END
}
int aob_sh_set_dark(aob_sh *h, const float *dark, int n) {
  AOB_API_BEGIN
  NEED(h); NEED(dark);
  if (!h->fakecam) throw Error("sh.set_dark: enable fakecam first");
  if ((int64_t)n * n != h->cam_dark.n) throw Error("sh.set_dark: the dark must match the image size");
  AOB_CUDA(cudaSetDevice(h->device));
  h->cam_dark.upload(dark, h->cam_dark.n);
  AOB_API_END
}
int aob_sh_set_flat(aob_sh *h, const float *flat, int n) {
  AOB_API_BEGIN
  NEED(h); NEED(flat);
  if (!h->fakecam) throw Error("sh.set_flat: enable fakecam first");
  if ((int64_t)n * n != h->cam_flat.n) throw Error("sh.set_flat: the flat must match the image size");
  AOB_CUDA(cudaSetDevice(h->device));
  h->cam_flat.upload(flat, h->cam_flat.n);
  AOB_API_END
}
int aob_sh_set_field_stop(aob_sh *h, const float *mask, int n) {
  AOB_API_BEGIN
  NEED(h);
  h->set_field_stop(mask, n);
  AOB_API_END
}
int aob_sh_set_pupil(aob_sh *h, const float *pupil) {
  AOB_API_BEGIN
  NEED(h); NEED(pupil);
  AOB_CUDA(cudaSetDevice(h->device));
  h->pupil.upload(pupil, h->pupil.n);
  AOB_API_END
}
int aob_sh_set_noise(aob_sh *h, float noise, int64_t seed) {
  AOB_API_BEGIN
  NEED(h);
  h->noise = noise;
  h->seed = seed;
  h->frame = 0;
  AOB_API_END
}
int aob_sh_set_lambda(aob_sh *h, float l) {
  AOB_API_BEGIN
  NEED(h);
  if (!(l > 0.f)) throw Error("sh.set_lambda: wavelength must be > 0");
  h->lambda_um = l;
  AOB_API_END
}
int aob_sh_set_nphot(aob_sh *h, float n) {
  AOB_API_BEGIN
  NEED(h);
  h->nphot = n;
  AOB_API_END
}
int aob_sh_set_frame(aob_sh *h, uint64_t f) {
  AOB_API_BEGIN
  NEED(h);
  h->frame = f;
  AOB_API_END
}
int aob_sh_get_frame(aob_sh *h, uint64_t *f) {
  AOB_API_BEGIN
  NEED(h); NEED(f);
  *f = h->frame;
  AOB_API_END
}
int aob_sh_buffer(aob_sh *h, const char *which, void **p, int64_t *n) {
  AOB_API_BEGIN
  NEED(h); NEED(which); NEED(p); NEED(n);
  std::string w(which);
#define B(name, buf)        \
  if (w == name) {          \
    *p = (void *)h->buf.p;  \
    *n = h->buf.n;          \
    return AOB_OK;          \
  }
  B("phase", phase) B("pupil", pupil) B("bincube", bincube) B("binimg", binimg) B("intensities", intensities)
  B("validsubsx", validsubsx) B("validsubsy", validsubsy) B("fluxPerSub", fluxPerSub) B("binmap", binmap)
  B("offsets", offsets) B("istart", istart) B("jstart", jstart) B("slopes", slopes) B("camimg", camimg)
  B("dark", cam_dark) B("flat", cam_flat) B("hrmap", hrmap) B("submask", fs_mask) B("phasemap", phasemap)
  B("ttprojmat", ttprojmat)
#undef B
  throw Error("sh.buffer: unknown buffer '" + w + "'");
  AOB_API_END
}
int aob_sh_comp_image(aob_sh *h, int noise, void *stream) {
  AOB_API_BEGIN
  NEED(h);
  h->comp_image(noise != 0, S(stream));
  AOB_API_END
}
int aob_sh_fill_binimage(aob_sh *h, void *stream) {
  AOB_API_BEGIN
  NEED(h);
  h->fill_binimage(S(stream));
  AOB_API_END
}
int aob_sh_set_tuning(aob_sh *h, int subaps_per_cta) {
  AOB_API_BEGIN
  NEED(h);
  if (subaps_per_cta < 0 || subaps_per_cta > 32) throw Error("sh.set_tuning: sub-apertures per CTA must be in [0, 32]");
  h->batch_override = subaps_per_cta;
  AOB_API_END
}
int aob_sh_set_bincube(aob_sh *h, const float *host, int64_t n) {
  AOB_API_BEGIN
  NEED(h); NEED(host);
  if (n != h->bincube.n) throw Error("sh.set_bincube: wrong size");
  AOB_CUDA(cudaSetDevice(h->device));
  h->bincube.upload(host, n);
  AOB_API_END
}
int aob_sh_set_binimg(aob_sh *h, const float *host, int64_t n) {
  AOB_API_BEGIN
  NEED(h); NEED(host);
  if (n != h->binimg.n) throw Error("sh.set_binimg: wrong size");
  AOB_CUDA(cudaSetDevice(h->device));
  h->binimg.upload(host, n);
  ++h->image_gen;
  AOB_API_END
}

// ---------------------------------------------------------------- centroider
int aob_centro_create(aob_centro **out, int device, int type, int nvalid, float offset, float scale) {
  AOB_API_BEGIN
  NEED(out);
  *out = nullptr;
  *out = new aob_centro(device, type, nvalid, offset, scale);
  AOB_API_END
}
int aob_centro_destroy(aob_centro *c) {
  AOB_API_BEGIN
  if (c) {
    cudaSetDevice(c->device);
    if (c->wfs && c->wfs->fused == c) c->wfs->fused = nullptr;
    delete c;
  }
  AOB_API_END
}
int aob_centro_attach_wfs(aob_centro *c, aob_sh *h) {
  AOB_API_BEGIN
  NEED(c);
  if (c->wfs && c->wfs->fused == c) c->wfs->fused = nullptr;
  c->wfs = h;
  if (h) {
    if (h->nvalid != c->nvalid) throw Error("centro.attach_wfs: nvalid differs from the sensor's");
    h->fused = c;
  }
  c->touch();
  AOB_API_END
}
int aob_centro_attach_pyr(aob_centro *c, aob_pyr *p) {
  AOB_API_BEGIN
  NEED(c);
  if (c->type != AOB_CENTRO_PYR && c->type != AOB_CENTRO_MASKEDPIX)
    throw Error("centro.attach_pyr: not a pyramid or masked-pixel centroider");
  if (p && c->type == AOB_CENTRO_PYR && p->nvalid != c->nvalid)
    throw Error("centro.attach_pyr: nvalid differs from the sensor's");
  if (p && c->type == AOB_CENTRO_MASKEDPIX && 4 * p->nvalid != c->nvalid)
    throw Error("centro.attach_pyr: a masked-pixel centroider needs nvalid = 4 * the sensor's nvalid");
  c->pyr = p;
  c->touch();
  AOB_API_END
}
int aob_centro_set_nmax(aob_centro *c, int nmax) {
  AOB_API_BEGIN
  NEED(c);
  if (c->type != AOB_CENTRO_BPCOG) throw Error("centro.set_nmax: not a bpcog centroider");
  if (nmax < 0 || nmax >= 1024) throw Error("centro.set_nmax: nmax must be in [0, 1024)");
  c->nmax = nmax;
  c->touch();
  AOB_API_END
}
int aob_centro_set_pyr_method(aob_centro *c, int method) {
  AOB_API_BEGIN
  NEED(c);
  if (method < 0 || method > 3) throw Error("centro.set_pyr_method: method must be 0..3");
  c->pyr_method = method;
  c->touch();
  AOB_API_END
}
int aob_centro_set_pyr_thresh(aob_centro *c, float thresh) {
  AOB_API_BEGIN
  NEED(c);
  c->valid_thresh = thresh;
  c->touch();
  AOB_API_END
}
int aob_centro_set_npix(aob_centro *c, int npix) {
  AOB_API_BEGIN
  NEED(c);
  if (npix <= 0) throw Error("centro.set_npix: npix must be > 0");
  c->npix = npix;
  c->touch();
  AOB_API_END
}
int aob_centro_set_scale(aob_centro *c, float v) {
  AOB_API_BEGIN
  NEED(c);
  c->scale = v;
  c->touch();
  AOB_API_END
}
int aob_centro_set_offset(aob_centro *c, float v) {
  AOB_API_BEGIN
  NEED(c);
  c->offset = v;
  c->touch();
  AOB_API_END
}
int aob_centro_set_threshold(aob_centro *c, float v) {
  AOB_API_BEGIN
  NEED(c);
  c->threshold = v;
  c->touch();
  AOB_API_END
}
int aob_centro_set_slope_order(aob_centro *c, int order) {
  AOB_API_BEGIN
  NEED(c);
  if (order != 0 && order != 1) throw Error("centro.set_slope_order: 0 (untied) or 1 (interleaved)");
  c->order = order;
  c->touch();
  AOB_API_END
}
int aob_centro_load_validpos(aob_centro *c, const int32_t *vx, const int32_t *vy, int n) {
  AOB_API_BEGIN
  NEED(c); NEED(vx); NEED(vy);
  const int want = c->type == AOB_CENTRO_PYR ? 4 * c->nvalid : c->nvalid;
  if (n != want) throw Error("centro.load_validpos: n must equal nvalid (4 * nvalid for a pyramid centroider)");
  AOB_CUDA(cudaSetDevice(c->device));
  if (!c->validx.p || c->validx.n != n) {
    c->validx.alloc(n);
    c->validy.alloc(n);
  }
  c->validx.upload(vx, n);
  c->validy.upload(vy, n);
  c->touch();
  AOB_API_END
}
int aob_centro_set_centroids_ref(aob_centro *c, const float *ref) {
  AOB_API_BEGIN
  NEED(c); NEED(ref);
  AOB_CUDA(cudaSetDevice(c->device));
  c->ref.upload(ref, c->nslopes());
  c->touch();
  AOB_API_END
}
int aob_centro_load_weights(aob_centro *c, const float *w, int64_t n) {
  AOB_API_BEGIN
  NEED(c); NEED(w);
  if (c->npix <= 0) throw Error("centro.load_weights: set npix first");
  const int64_t np2 = (int64_t)c->npix * c->npix;
  if (n != np2 && n != np2 * c->nvalid) throw Error("centro.load_weights: size must be npix^2 or npix^2*nvalid");
  AOB_CUDA(cudaSetDevice(c->device));
  c->weights.alloc(n);
  c->weights.upload(w, n);
  c->weights_per_sub = (n == np2) ? 0 : 1;
  c->touch();
  AOB_API_END
}
int aob_centro_load_img(aob_centro *c, const float *img, int m, int n) {
  AOB_API_BEGIN
  NEED(c); NEED(img);
  if (m <= 0 || n <= 0) throw Error("centro.load_img: bad size");
  AOB_CUDA(cudaSetDevice(c->device));
  if (c->img_raw.n != (int64_t)m * n) c->img_raw.alloc((int64_t)m * n);
  c->img_m = m;
  c->img_n = n;
  c->img_raw.upload(img, (int64_t)m * n);
  c->raw_u16 = false;
  AOB_API_END
}
int aob_centro_load_img_u16(aob_centro *c, const uint16_t *img, int m, int n, int on_device, void *stream) {
  AOB_API_BEGIN
  NEED(c); NEED(img);
  if (m <= 0 || n <= 0) throw Error("centro.load_img: bad size");
  AOB_CUDA(cudaSetDevice(c->device));
  const int64_t mn = (int64_t)m * n;
  if (c->img_raw_u16.n != mn) c->img_raw_u16.alloc(mn);
  c->img_m = m;
  c->img_n = n;
  AOB_CUDA(cudaMemcpyAsync(c->img_raw_u16.p, img, sizeof(uint16_t) * mn,
                           on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, S(stream)));
  if (!on_device) AOB_CUDA(cudaStreamSynchronize(S(stream)));
  c->raw_u16 = true;
  AOB_API_END
}
int aob_centro_set_lut_pix(aob_centro *c, const int32_t *lut, int n) {
  AOB_API_BEGIN
  NEED(c); NEED(lut);
  if (n <= 0) throw Error("centro.set_lutPix: bad size");
  for (int i = 0; i < n; ++i)
    if (lut[i] < 0 || lut[i] >= n) throw Error("centro.set_lutPix: entry outside the image");
  AOB_CUDA(cudaSetDevice(c->device));
  if (c->lut.n != n) c->lut.alloc(n);
  c->lut.upload(lut, n);
  AOB_API_END
}
int aob_centro_calibrate_img_validpix(aob_centro *c, void *stream) {
  AOB_API_BEGIN
  NEED(c);
  c->calibrate(S(stream), true);
  AOB_API_END
}
int aob_centro_set_dark(aob_centro *c, const float *d, int n) {
  AOB_API_BEGIN
  NEED(c); NEED(d);
  AOB_CUDA(cudaSetDevice(c->device));
  if (c->dark.n != (int64_t)n * n) c->dark.alloc((int64_t)n * n);
  c->dark.upload(d, (int64_t)n * n);
  AOB_API_END
}
int aob_centro_set_flat(aob_centro *c, const float *f, int n) {
  AOB_API_BEGIN
  NEED(c); NEED(f);
  AOB_CUDA(cudaSetDevice(c->device));
  if (c->flat.n != (int64_t)n * n) c->flat.alloc((int64_t)n * n);
  c->flat.upload(f, (int64_t)n * n);
  AOB_API_END
}
int aob_centro_calibrate_img(aob_centro *c, void *stream) {
  AOB_API_BEGIN
  NEED(c);
  c->calibrate(S(stream));
  AOB_API_END
}
int aob_centro_get_cog(aob_centro *c, float *dev_slopes, void *stream) {
  AOB_API_BEGIN
  NEED(c); NEED(dev_slopes);
  c->get_cog(dev_slopes, S(stream));
  AOB_API_END
}
int aob_centro_buffer(aob_centro *c, const char *which, void **p, int64_t *n) {
  AOB_API_BEGIN
  NEED(c); NEED(which); NEED(p); NEED(n);
  std::string w(which);
#define B(name, buf)        \
  if (w == name) {          \
    *p = (void *)c->buf.p;  \
    *n = c->buf.n;          \
    return AOB_OK;          \
  }
  B("validx", validx) B("validy", validy) B("centroids_ref", ref) B("weights", weights)
  B("intensities", intensities) B("img", img) B("dark", dark) B("flat", flat) B("lut", lut)
  if (w == "img_raw") {  // the last loaded frame, float32 or uint16
    *p = c->raw_u16 ? (void *)c->img_raw_u16.p : (void *)c->img_raw.p;
    *n = c->raw_u16 ? c->img_raw_u16.n : c->img_raw.n;
    return AOB_OK;
  }
#undef B
  throw Error("centro.buffer: unknown buffer '" + w + "'");
  AOB_API_END
}
int aob_centro_get_params(aob_centro *c, int *type, int *nvalid, int *npix, float *offset, float *scale,
                          float *threshold) {
  AOB_API_BEGIN
  NEED(c);
  if (type) *type = c->type;
  if (nvalid) *nvalid = c->nvalid;
  if (npix) *npix = c->npix;
  if (offset) *offset = c->offset;
  if (scale) *scale = c->scale;
  if (threshold) *threshold = c->threshold;
  AOB_API_END
}

// ---------------------------------------------------------------- LS controller
int aob_ls_create(aob_ls **out, int device, int nslope, int nactu, float delay) {
  AOB_API_BEGIN
  NEED(out);
  *out = nullptr;
  *out = new aob_ls(device, nslope, nactu, delay);
  AOB_API_END
}
int aob_generic_create(aob_ls **out, int device, int nslope, int nactu, float delay) {
  AOB_API_BEGIN
  NEED(out);
  *out = nullptr;
  std::unique_ptr<aob_ls> c(new aob_ls(device, nslope, nactu, delay));
  c->make_generic();
  *out = c.release();
  AOB_API_END
}
int aob_ls_get_kind(aob_ls *c, int *kind, int *law, float *leaky, int *polc) {
  AOB_API_BEGIN
  NEED(c);
  if (kind) *kind = c->kind;
  if (law) *law = c->law;
  if (leaky) *leaky = c->leaky;
  if (polc) *polc = c->polc;
  AOB_API_END
}
int aob_ls_set_commandlaw(aob_ls *c, int law) {
  AOB_API_BEGIN
  NEED(c);
  if (c->kind != AOB_CTRL_GENERIC) throw Error("set_commandlaw: not a generic controller");
  if (law != AOB_LAW_INTEGRATOR && law != AOB_LAW_MODAL_INTEGRATOR && law != AOB_LAW_2MATRICES)
    throw Error("set_commandlaw: law must be integrator (1), modal_integrator (2) or 2matrices (3)");
  c->law = law;
  AOB_API_END
}
int aob_ls_set_leaky_factor(aob_ls *c, float leaky) {
  AOB_API_BEGIN
  NEED(c);
  if (c->kind != AOB_CTRL_GENERIC) throw Error("set_leaky_factor: not a generic controller");
  c->leaky = leaky;
  AOB_API_END
}
int aob_ls_set_polc(aob_ls *c, int polc) {
  AOB_API_BEGIN
  NEED(c);
  if (c->kind != AOB_CTRL_GENERIC) throw Error("set_polc: not a generic controller");
  c->polc = polc ? 1 : 0;
  AOB_API_END
}
int aob_ls_set_decay_factor(aob_ls *c, const float *decay) {
  AOB_API_BEGIN
  NEED(c); NEED(decay);
  if (c->kind != AOB_CTRL_GENERIC) throw Error("set_decayFactor: not a generic controller");
  AOB_CUDA(cudaSetDevice(c->device));
  c->decay.upload(decay, c->nactu);
  AOB_API_END
}
int aob_ls_apply_perturb(aob_ls *c, void *stream) {
  AOB_API_BEGIN
  NEED(c);
  c->apply_perturb(S(stream));
  AOB_API_END
}
int aob_ls_set_matE(aob_ls *c, const float *matE) {
  AOB_API_BEGIN
  NEED(c); NEED(matE);
  if (c->kind != AOB_CTRL_GENERIC) throw Error("set_matE: not a generic controller");
  c->set_matE(matE);
  AOB_API_END
}
int aob_ls_destroy(aob_ls *c) {
  AOB_API_BEGIN
  if (c) {
    cudaSetDevice(c->device);
    delete c;
  }
  AOB_API_END
}
int aob_ls_set_cmat(aob_ls *c, const float *cmat) {
  AOB_API_BEGIN
  NEED(c); NEED(cmat);
  AOB_CUDA(cudaSetDevice(c->device));
  std::memcpy(c->h_cmat.data(), cmat, sizeof(float) * c->h_cmat.size());
  c->cmat.upload(cmat, c->cmat.n);
  c->packed_valid[0] = c->packed_valid[1] = c->packed_valid[2] = false;
  c->ensure_packed(c->prec);
  AOB_API_END
}
int aob_ls_set_imat(aob_ls *c, const float *imat) {
  AOB_API_BEGIN
  NEED(c); NEED(imat);
  AOB_CUDA(cudaSetDevice(c->device));
  if (!c->imat.p) c->imat.alloc((int64_t)c->nslope * c->nactu);
  c->imat.upload(imat, c->imat.n);
  if (c->kind == AOB_CTRL_GENERIC) c->set_imat_rows(imat);  // pseudo-open-loop slopes
  AOB_API_END
}
int aob_ls_set_modal_gains(aob_ls *c, const float *g) {
  AOB_API_BEGIN
  NEED(c); NEED(g);
  AOB_CUDA(cudaSetDevice(c->device));
  c->gains.upload(g, c->nactu);
  AOB_API_END
}
int aob_ls_set_gain(aob_ls *c, float g) {
  AOB_API_BEGIN
  NEED(c);
  c->gain = g;
  AOB_API_END
}
int aob_ls_set_delay(aob_ls *c, float d) {
  AOB_API_BEGIN
  NEED(c);
  c->set_delay(d);
  AOB_API_END
}
int aob_ls_set_open_loop(aob_ls *c, int ol, int reset) {
  AOB_API_BEGIN
  NEED(c);
  c->open_loop = ol;
  if (ol && reset) {
    AOB_CUDA(cudaSetDevice(c->device));
    for (auto &b : c->ring) AOB_CUDA(cudaMemset(b.p, 0, b.bytes()));
  }
  AOB_API_END
}
int aob_ls_set_com_range(aob_ls *c, float lo, float hi) {
  AOB_API_BEGIN
  NEED(c);
  c->volt_min = lo;
  c->volt_max = hi;
  AOB_API_END
}
int aob_ls_set_com(aob_ls *c, const float *com, int n) {
  AOB_API_BEGIN
  NEED(c); NEED(com);
  if (n != c->nactu) throw Error("ls.set_com: wrong dimension of com");
  AOB_CUDA(cudaSetDevice(c->device));
  c->ring.back().upload(com, n);
  c->com_clipped.upload(com, n);
  AOB_API_END
}
int aob_ls_set_centroids(aob_ls *c, const float *s, int n) {
  AOB_API_BEGIN
  NEED(c); NEED(s);
  if (n != c->nslope) throw Error("ls.set_centroids: wrong dimension");
  AOB_CUDA(cudaSetDevice(c->device));
  c->centroids.upload(s, n);
  AOB_API_END
}
int aob_ls_set_precision(aob_ls *c, int prec) {
  AOB_API_BEGIN
  NEED(c);
  if (prec < 0 || prec > 2) throw Error("ls.set_precision: 0=F32, 1=BF16, 2=FP8");
  c->prec = prec;
  c->ensure_packed(prec);
  AOB_API_END
}
int aob_ls_set_tuning(aob_ls *c, int kind, int nblocks) {
  AOB_API_BEGIN
  NEED(c);
  if (kind < 0 || kind > 2 || nblocks < 0) throw Error("ls.set_tuning: kind 0..2, nblocks >= 0");
  c->mvm_kind = kind;
  c->nblocks = nblocks;
  AOB_API_END
}
int aob_ls_status(aob_ls *c, uint32_t *st, int reset) {
  AOB_API_BEGIN
  NEED(c); NEED(st);
  AOB_CUDA(cudaSetDevice(c->device));
  AOB_CUDA(cudaMemcpy(st, c->status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (reset) AOB_CUDA(cudaMemset(c->status.p, 0, sizeof(uint32_t)));
  AOB_API_END
}
int aob_ls_comp_com(aob_ls *c, void *stream) {
  AOB_API_BEGIN
  NEED(c);
  c->comp_com(S(stream));
  AOB_API_END
}
int aob_ls_clip(aob_ls *c, void *stream) {
  AOB_API_BEGIN
  NEED(c);
  c->clip(S(stream));
  AOB_API_END
}
int aob_ls_comp_voltage(aob_ls *c, void *stream) {
  AOB_API_BEGIN
  NEED(c);
  c->comp_voltage(S(stream));
  AOB_API_END
}
int aob_ls_add_perturb(aob_ls *c, const char *name, const float *pert, int n) {
  AOB_API_BEGIN
  NEED(c); NEED(name); NEED(pert);
  if (n <= 0) throw Error("ls.add_perturb: N must be > 0");
  if (c->perturb.count(name)) throw Error("ls.add_perturb: this perturb buffer already exists");
  AOB_CUDA(cudaSetDevice(c->device));
  aob_ls::Perturb &p = c->perturb[name];
  p.buf.alloc((int64_t)n * c->nactu);
  p.buf.upload(pert, (int64_t)n * c->nactu);
  p.n = n;
  p.cpt = 0;
  p.on = true;
  AOB_API_END
}
int aob_ls_remove_perturb(aob_ls *c, const char *name) {
  AOB_API_BEGIN
  NEED(c); NEED(name);
  if (!c->perturb.erase(name)) throw Error("ls.remove_perturb: this perturb buffer does not exist");
  AOB_API_END
}
int aob_ls_enable_perturb(aob_ls *c, const char *name, int en) {
  AOB_API_BEGIN
  NEED(c); NEED(name);
  auto it = c->perturb.find(name);
  if (it == c->perturb.end()) throw Error("ls.enable_perturb: this perturb buffer does not exist");
  it->second.on = en != 0;
  AOB_API_END
}
int aob_ls_reset_perturb(aob_ls *c) {
  AOB_API_BEGIN
  NEED(c);
  c->perturb.clear();
  AOB_API_END
}
int aob_ls_svdec_imat(aob_ls *c) {
  AOB_API_BEGIN
  NEED(c);
  c->svdec_imat();
  AOB_API_END
}
int aob_ls_build_cmat(aob_ls *c, int nfilt) {
  AOB_API_BEGIN
  NEED(c);
  c->build_cmat(nfilt);
  AOB_API_END
}
int aob_ls_buffer(aob_ls *c, const char *which, void **p, int64_t *n) {
  AOB_API_BEGIN
  NEED(c); NEED(which); NEED(p); NEED(n);
  std::string w(which);
#define B(name, buf)        \
  if (w == name) {          \
    *p = (void *)c->buf.p;  \
    *n = c->buf.n;          \
    return AOB_OK;          \
  }
  B("centroids", centroids) B("err", err) B("com_clipped", com_clipped) B("voltage", com_clipped) B("cmat", cmat)
  B("imat", imat) B("eigenvals", eigenvals_f) B("gain", gains)
#undef B
  if (w == "com") {
    *p = (void *)c->ring.back().p;
    *n = c->nactu;
    return AOB_OK;
  }
  if (w == "com0" || w == "com1") {
    const size_t i = (w == "com0") ? 0 : 1;
    if (i >= c->ring.size()) throw Error("ls.buffer: no delayed command buffers (delay == 0)");
    *p = (void *)c->ring[i].p;
    *n = c->nactu;
    return AOB_OK;
  }
  throw Error("ls.buffer: unknown buffer '" + w + "'");
  AOB_API_END
}
int aob_ls_get_params(aob_ls *c, int *nslope, int *nactu, float *delay, float *gain, int *open_loop,
                      float *vmin, float *vmax, int *prec) {
  AOB_API_BEGIN
  NEED(c);
  if (nslope) *nslope = c->nslope;
  if (nactu) *nactu = c->nactu;
  if (delay) *delay = c->delay;
  if (gain) *gain = c->gain;
  if (open_loop) *open_loop = c->open_loop;
  if (vmin) *vmin = c->volt_min;
  if (vmax) *vmax = c->volt_max;
  if (prec) *prec = c->prec;
  AOB_API_END
}

// ---- pyramid sensor ---------------------------------------------------------
int aob_pyr_create(aob_pyr **out, int device, int nxsub, int nvalid, int npix, int nphase, int nrebin, int nfft,
                   int ntot, int npts, float pdiam, float nphot, float nphot4imat) {
  AOB_API_BEGIN
  NEED(out);
  *out = nullptr;
  AOB_CUDA(cudaSetDevice(device));
  *out = new aob_pyr(device, nxsub, nvalid, npix, nphase, nrebin, nfft, ntot, npts, pdiam, nphot, nphot4imat);
  AOB_API_END
}
int aob_pyr_destroy(aob_pyr *h) {
  AOB_API_BEGIN
  if (h) {
    cudaSetDevice(h->device);
    delete h;
  }
  AOB_API_END
}
int aob_pyr_load_arrays(aob_pyr *h, const float *halfxy_c64, const float *cx, const float *cy, const float *weights,
                        const float *sincar, const float *submask, const int32_t *validsubsx,
                        const int32_t *validsubsy, const int32_t *phasemap, const float *fluxPerSub,
                        const float *ttprojmat) {
  AOB_API_BEGIN
  NEED(h);
  AOB_CUDA(cudaSetDevice(h->device));
  h->load_arrays(reinterpret_cast<const float2 *>(halfxy_c64), cx, cy, weights, sincar, submask, validsubsx,
                 validsubsy, fluxPerSub);
  load_geom_arrays(h->device, h->phasemap, h->ttprojmat, phasemap, ttprojmat, h->nphase, h->nvalid, h->phase.n);
  AOB_API_END
}
int aob_pyr_set_submask(aob_pyr *h, const float *submask, int64_t n) {
  AOB_API_BEGIN
  NEED(h); NEED(submask);
  if (n != h->submask.n) throw Error("pyr.set_submask: wrong dimensions (nfft x nfft)");
  AOB_CUDA(cudaSetDevice(h->device));
  h->submask.upload(submask, n);
  AOB_API_END
}
int aob_pyr_set_phalfxy(aob_pyr *h, const float *phalfxy_c64, int64_t n) {
  AOB_API_BEGIN
  NEED(h); NEED(phalfxy_c64);
  if (n != h->phalfxy.n) throw Error("pyr.set_phalfxy: wrong dimensions (nfft x nfft complex)");
  AOB_CUDA(cudaSetDevice(h->device));
  h->phalfxy.upload(reinterpret_cast<const float2 *>(phalfxy_c64), n);
  AOB_API_END
}
int aob_pyr_set_binimg(aob_pyr *h, const float *img, int64_t n) {
  AOB_API_BEGIN
  NEED(h); NEED(img);
  if (n != h->binimg.n) throw Error("pyr.set_binimg: wrong dimensions");
  AOB_CUDA(cudaSetDevice(h->device));
  h->binimg.upload(img, n);
  ++h->image_gen;
  AOB_API_END
}
int aob_pyr_set_compute_focalplane(aob_pyr *h, int enable) {
  AOB_API_BEGIN
  NEED(h);
  h->compute_focalplane = enable != 0;
  AOB_API_END
}
int aob_pyr_set_modulation(aob_pyr *h, const float *cx, const float *cy, const float *weights, int npts) {
  AOB_API_BEGIN
  NEED(h);
  AOB_CUDA(cudaSetDevice(h->device));
  h->set_modulation(cx, cy, weights, npts);
  AOB_API_END
}
int aob_pyr_set_pupil(aob_pyr *h, const float *pupil_host) {
  AOB_API_BEGIN
  NEED(h); NEED(pupil_host);
  AOB_CUDA(cudaSetDevice(h->device));
  h->pupil.upload(pupil_host, h->pupil.n);
  AOB_API_END
}
int aob_pyr_set_noise(aob_pyr *h, float noise, int64_t seed) {
  AOB_API_BEGIN
  NEED(h);
  h->noise = noise;
  h->seed = seed;
  AOB_API_END
}
int aob_pyr_set_lambda(aob_pyr *h, float lambda_um) {
  AOB_API_BEGIN
  NEED(h);
  if (!(lambda_um > 0.f)) throw Error("pyr.set_lambda: lambda must be > 0");
  h->lambda_um = lambda_um;
  AOB_API_END
}
int aob_pyr_set_nphot(aob_pyr *h, float nphot) {
  AOB_API_BEGIN
  NEED(h);
  h->nphot = nphot;
  AOB_API_END
}
int aob_pyr_set_frame(aob_pyr *h, uint64_t frame) {
  AOB_API_BEGIN
  NEED(h);
  h->frame = frame;
  AOB_API_END
}
int aob_pyr_get_frame(aob_pyr *h, uint64_t *frame) {
  AOB_API_BEGIN
  NEED(h); NEED(frame);
  *frame = h->frame;
  AOB_API_END
}
int aob_pyr_buffer(aob_pyr *h, const char *which, void **dev_ptr, int64_t *nelem) {
  AOB_API_BEGIN
  NEED(h); NEED(which); NEED(dev_ptr);
  const std::string w(which);
  void *p = nullptr;
  int64_t n = 0;
  if (w == "phase") { p = h->phase.p; n = h->phase.n; }
  else if (w == "pupil") { p = h->pupil.p; n = h->pupil.n; }
  else if (w == "binimg") { p = h->binimg.p; n = h->binimg.n; }
  else if (w == "hrimg") { p = h->hrimg.p; n = h->hrimg.n; }
  else if (w == "validsubsx") { p = h->validsubsx.p; n = h->validsubsx.n; }
  else if (w == "validsubsy") { p = h->validsubsy.p; n = h->validsubsy.n; }
  else if (w == "fluxPerSub") { p = h->fluxPerSub.p; n = h->fluxPerSub.n; }
  else if (w == "submask") { p = h->submask.p; n = h->submask.n; }
  else if (w == "phalfxy") { p = h->phalfxy.p; n = 2 * h->phalfxy.n; }
  else if (w == "sincar") { p = h->sincar.p; n = h->sincar.n; }
  else if (w == "phasemap") { p = h->phasemap.p; n = h->phasemap.n; }
  else if (w == "ttprojmat") { p = h->ttprojmat.p; n = h->ttprojmat.n; }
  else if (w == "slopes") {
    if (h->slopes.n != 2LL * h->nvalid) {
      AOB_CUDA(cudaSetDevice(h->device));
      h->slopes.alloc(2LL * h->nvalid);
    }
    p = h->slopes.p; n = h->slopes.n;
  }
  else if (w == "pyrfocalplane") {
    if (h->focalplane.n != (int64_t)h->nfft * h->nfft) {
      AOB_CUDA(cudaSetDevice(h->device));
      h->focalplane.alloc((int64_t)h->nfft * h->nfft);
      AOB_CUDA(cudaMemset(h->focalplane.p, 0, sizeof(float) * h->focalplane.n));
    }
    p = h->focalplane.p; n = h->focalplane.n;
  }
  else throw Error("pyr.buffer: unknown buffer '" + w + "'");
  *dev_ptr = p;
  if (nelem) *nelem = n;
  AOB_API_END
}
int aob_pyr_comp_image(aob_pyr *h, int noise, void *stream) {
  AOB_API_BEGIN
  NEED(h);
  h->comp_image(noise != 0, S(stream));
  AOB_API_END
}

}  // extern "C"
