// Centre-of-gravity centroiders on a sensor image (CoG, thresholded CoG,
// weighted CoG) and the raw-image calibration.
//
// Reference kernels: centroids<> in libsutra/src.cu/sutra_centroider_cog.cu:28-81,
// sutra_centroider_tcog.cu:27-81 (writes the thresholded pixels back into the
// image, :63), sutra_centroider_wcog.cu:58-113; calib_krnl in
// sutra_centroider.cu:89-96.  The reference launches one CTA of npix^2
// threads per sub-aperture and reduces with three CUB BlockReduce passes; here
// one warp handles a sub-aperture and reduces with shuffles.  When the
// centroider is attached to a SH sensor the same sums are produced inside the
// sensor kernel (sh_wfs.cu) and this kernel only runs if the image changed
// after that or a parameter was modified.

#include <algorithm>
#include <vector>

#include "aob_objects.hpp"

namespace aob {

struct CogArgs {
  const float *img;
  float *img_out;  // tCoG write-back target (may alias img); null = none
  int size;        // image is size x size
  const int32_t *validx;
  const int32_t *validy;
  int nvalid, npix, kind, order;
  float scale, offset, thresh;
  const float *ref;
  const float *weights;
  int wper;
  float *slopes;
  float *intens;
};

__global__ void cog_kernel(CogArgs A) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int npix2 = A.npix * A.npix;
  const int64_t lim = (int64_t)A.size * A.size;
  for (int k = warp; k < A.nvalid; k += nwarps) {
    const int vx = A.validx[k], vy = A.validy[k];
    float cs = 0.f, cx = 0.f, cy = 0.f;
    for (int p = lane; p < npix2; p += 32) {
      const int x = p % A.npix, y = p / A.npix;
      const int64_t idim = (int64_t)(x + vx) + (int64_t)(y + vy) * A.size;
      if (idim < 0 || idim >= lim) continue;
      float d = A.img[idim];
      if (A.kind == 1 || A.kind == 2) d = (d > A.thresh) ? d - A.thresh : 1.e-6f;
      if (A.kind == 1 && A.img_out) A.img_out[idim] = d;
      if (A.kind == 2) d *= A.weights[p + (A.wper ? k * npix2 : 0)];
      cs += d;
      cx = fmaf(d, (float)x, cx);
      cy = fmaf(d, (float)y, cy);
    }
    cs = warp_sum(cs);
    cx = warp_sum(cx);
    cy = warp_sum(cy);
    if (lane == 0) {
      const int ix = A.order ? 2 * k : k;
      const int iy = A.order ? 2 * k + 1 : k + A.nvalid;
      A.slopes[ix] = (cx / (cs + 1.e-6f) - A.offset) * A.scale - A.ref[ix];
      A.slopes[iy] = (cy / (cs + 1.e-6f) - A.offset) * A.scale - A.ref[iy];
      A.intens[k] = cs;
    }
  }
}

// tCoG side effect for slopes that were produced inside the sensor kernel:
// store the thresholded pixels of every valid sub-aperture into the image.
__global__ void tcog_writeback_kernel(float *img, int size, const int32_t *validx, const int32_t *validy,
                                      int nvalid, int npix, float thresh) {
  const int npix2 = npix * npix;
  const int64_t lim = (int64_t)size * size;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < npix2 * nvalid; t += gridDim.x * blockDim.x) {
    const int k = t / npix2, p = t - k * npix2;
    const int64_t idim = (int64_t)(p % npix + validx[k]) + (int64_t)(p / npix + validy[k]) * size;
    if (idim < 0 || idim >= lim) continue;
    const float d = img[idim];
    img[idim] = (d > thresh) ? d - thresh : 1.e-6f;
  }
}

// Pyramid slopes (pyr2slopes_krnl, libsutra/src.cu/sutra_centroider_pyr.cu:27-69,
// flux as intensities_krnl, sutra_wfs.cu:2041-2054).  Quadrant k of valid
// sub-aperture i is the binned-image pixel (validx[i + k nvalid], validy[...]).
// With a global method (the reference default is nosinus global, method 1) every
// sub-aperture is normalised by the mean flux (fillvalues, carma_obj.cu:194-201);
// the sum runs in a fixed order (per-thread partial sums, then a tree), so
// the slopes are deterministic.  One CTA.
// Pyramid slopes over the whole GPU in two launches: per-CTA sums of the
// sub-aperture fluxes (the intensities written as they are formed), then every
// CTA adds the CTA sums in a fixed order for the global mean and emits the
// slopes of its sub-apertures (the reference's Method_CoG(uint8_t),
// sutra_centroider_pyr.hpp:27-34: 0 sinus global, 1 nosinus global, 2 sinus
// local, 3 nosinus local; pyr2slopes_krnl, sutra_centroider_pyr.cu:27-69).
constexpr int PYR_SLOPE_THREADS = 256;
__device__ __forceinline__ void pyr_quad(const float *img, int ns, const int32_t *vx, const int32_t *vy, int nvalid,
                                         int i, float *q) {
#pragma unroll
  for (int k = 0; k < 4; ++k) q[k] = img[vx[i + k * nvalid] + vy[i + k * nvalid] * ns];
}
__global__ void __launch_bounds__(PYR_SLOPE_THREADS)
    pyr_flux_kernel(const float *img, int ns, const int32_t *vx, const int32_t *vy, int nvalid, float *inten,
                    float *partial) {
  __shared__ float red[PYR_SLOPE_THREADS / 32];
  const int i = blockIdx.x * PYR_SLOPE_THREADS + threadIdx.x;
  float f = 0.f;
  if (i < nvalid) {
    float q[4];
    pyr_quad(img, ns, vx, vy, nvalid, i, q);
    f = q[0] + q[1] + q[2] + q[3];
    inten[i] = f;
  }
  f = warp_sum(f);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = f;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < PYR_SLOPE_THREADS / 32; ++w) t += red[w];
    partial[blockIdx.x] = t;
  }
}
__global__ void __launch_bounds__(PYR_SLOPE_THREADS)
    pyr_slopes_kernel(const float *img, int ns, const int32_t *vx, const int32_t *vy, int nvalid, float scale,
                      float thresh, int method, const float *ref, int order, const float *partial, int nparts,
                      float *slopes, float *inten) {
  __shared__ float s_mean;
  const bool sinus = (method & 1) == 0, local = method > 1;
  if (threadIdx.x < 32) {
    float t = 0.f;
    for (int b = threadIdx.x; b < nparts; b += 32) t += partial[b];
    t = warp_sum(t);
    if (threadIdx.x == 0) s_mean = t / (float)nvalid;
  }
  const int i = blockIdx.x * PYR_SLOPE_THREADS + threadIdx.x;
  float q[4];
  if (i < nvalid) pyr_quad(img, ns, vx, vy, nvalid, i, q);
  __syncthreads();
  if (i >= nvalid) return;
  const float mean = s_mean;
  const float f = local ? inten[i] : mean;
  const int ix = order ? 2 * i : i;
  const int iy = order ? 2 * i + 1 : i + nvalid;
  float sx = 0.f, sy = 0.f;
  if (!(f < thresh)) {
    const float tx = ((q[0] + q[3]) - (q[1] + q[2])) / f;
    const float ty = ((q[0] + q[2]) - (q[1] + q[3])) / f;
    sx = sinus ? scale * sinpif(tx / 2.f) : scale * tx;
    sy = sinus ? scale * sinpif(ty / 2.f) : scale * ty;
  }
  slopes[ix] = sx - ref[ix];
  slopes[iy] = sy - ref[iy];
  if (!local) inten[i] = mean;
}

// Masked-pixel slopes (get_maskedPix_krnl, libsutra/src.cu/sutra_centroider_maskedPix.cu:26-38,
// with fill_intensities_krnl :47-56 and the CUB sum of sutra_centroider_maskedPix.cpp:129-134):
// every valid pixel of the image is a "slope", normalised by the mean flux of
// the valid pixels: s[i] = img[i] / sum * n - ref[i] (-ref[i] when the sum is 0;
// the reference initialises ref to 1).  intens[i] receives the pixel values and
// intens[n] their sum.  One CTA; the sum runs in a fixed order.
constexpr int MASKED_THREADS = 1024;
__global__ void __launch_bounds__(MASKED_THREADS)
    masked_pix_kernel(const float *img, int ns, const int32_t *vx, const int32_t *vy, int n, const float *ref,
                      float *slopes, float *intens) {
  __shared__ float red[MASKED_THREADS];
  float part = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float v = img[vx[i] + (int64_t)vy[i] * ns];
    intens[i] = v;
    part += v;
  }
  red[threadIdx.x] = part;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  const float sum = red[0];
  if (threadIdx.x == 0) intens[n] = sum;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    slopes[i] = sum != 0.f ? img[vx[i] + (int64_t)vy[i] * ns] / sum * (float)n - ref[i] : -ref[i];
}

// Brightest-pixel CoG (centroids<> of libsutra/src.cu/sutra_centroider_bpcog.cu:24-80):
// the reference sorts a sub-aperture's npix^2 pixels -- padded with zeros up
// to its CUB block size (16, 36, 64, 100, 144, 256, 512 or 1024) -- in
// descending order, takes the value of rank nmax as the threshold, keeps
// pix - threshold where pix > threshold (0 elsewhere), writes those values back
// into the image and takes their centre of gravity.  Here one warp handles a
// sub-aperture and finds the value of rank nmax by counting, for each pixel,
// the larger ones (the padding zeros included).
__global__ void bpcog_kernel(float *img, int size, const int32_t *validx, const int32_t *validy, int nvalid,
                             int npix, int nmax, int npad, float scale, float offset, const float *ref, int order,
                             float *slopes, float *intens) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int npix2 = npix * npix;  // <= 1024 (host-checked)
  const int64_t lim = (int64_t)size * size;
  for (int k = warp; k < nvalid; k += nwarps) {
    const int vx = validx[k], vy = validy[k];
    auto pix = [&](int p) -> float {
      const int64_t idim = (int64_t)(p % npix + vx) + (int64_t)(p / npix + vy) * size;
      return (idim >= 0 && idim < lim) ? img[idim] : 0.f;
    };
    // threshold: the value v with (#larger) <= nmax < (#larger) + (#equal), over
    // the pixels and npad zeros; when no pixel holds rank nmax, a padding zero does
    float thr = 0.f;
    bool found = false;
    for (int c0 = 0; c0 < npix2 && !found; c0 += 32) {
      const int c = c0 + lane;
      const float v = c < npix2 ? pix(c) : 0.f;
      int gt = 0, eq = 0;
      for (int p = 0; p < npix2; ++p) {
        const float u = pix(p);
        gt += u > v;
        eq += u == v;
      }
      if (v < 0.f) gt += npad;
      if (v == 0.f) eq += npad;
      const bool hit = c < npix2 && gt <= nmax && nmax < gt + eq;
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (m) {
        thr = __shfl_sync(0xffffffffu, v, __ffs(m) - 1);
        found = true;
      }
    }
    float cs = 0.f, cx = 0.f, cy = 0.f;
    for (int p = lane; p < npix2; p += 32) {
      const int x = p % npix, y = p / npix;
      const int64_t idim = (int64_t)(x + vx) + (int64_t)(y + vy) * size;
      if (idim < 0 || idim >= lim) continue;
      const float v = img[idim];
      const float d = v > thr ? v - thr : 0.f;
      img[idim] = d;
      cs += d;
      cx = fmaf(d, (float)x, cx);
      cy = fmaf(d, (float)y, cy);
    }
    cs = warp_sum(cs);
    cx = warp_sum(cx);
    cy = warp_sum(cy);
    if (lane == 0) {
      const int ix = order ? 2 * k : k;
      const int iy = order ? 2 * k + 1 : k + nvalid;
      slopes[ix] = (cx / (cs + 1.e-6f) - offset) * scale - ref[ix];
      slopes[iy] = (cy / (cs + 1.e-6f) - offset) * scale - ref[iy];
      intens[k] = cs;
    }
  }
}

// CUB block size the reference's bpcog launch picks for npix^2 pixels
// (get_centroids, sutra_centroider_bpcog.cu:86-135)
static int bpcog_block(int n) {
  const int sizes[] = {16, 36, 64, 100, 144, 256, 512, 1024};
  for (int b : sizes)
    if (n <= b) return b;
  return n;
}

// Raw-image calibration through the pixel look-up table (calib_krnl,
// libsutra/src.cu/sutra_centroider.cu:108-115): cal = (raw[lut] - dark) * flat,
// raw in float32 or in the camera's uint16.
template <typename Tin>
__global__ void calib_kernel(const Tin *raw, float *cal, const float *dark, const float *flat, const int32_t *lut,
                             int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    cal[t] = ((float)raw[lut[t]] - dark[t]) * flat[t];
}

// The same calibration on the valid pixels only, the rest of the image at zero
// (calibrate_img_validPix, sutra_centroider.cpp:194-223): the npix x npix window of
// every valid sub-aperture (calibration_validPix_sh_krnl, sutra_centroider.cu:68-90)
// or every listed pixel (calibration_validPix_pyr_krnl, :92-104).
template <typename Tin>
__global__ void calib_valid_kernel(const Tin *raw, float *cal, const float *dark, const float *flat,
                                   const int32_t *lut, const int32_t *vx, const int32_t *vy, int nvalid, int npix,
                                   int size) {
  const int npix2 = npix * npix;
  const int64_t lim = (int64_t)size * size;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)nvalid * npix2;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(t / npix2), p = (int)(t - (int64_t)k * npix2);
    const int64_t i = (int64_t)(p % npix + vx[k]) + (int64_t)(p / npix + vy[k]) * size;
    if (i < lim) cal[i] = ((float)raw[lut[i]] - dark[i]) * flat[i];
  }
}

}  // namespace aob

using namespace aob;

aob_centro::aob_centro(int device_, int type_, int nvalid_, float offset_, float scale_)
    : device(device_), type(type_), nvalid(nvalid_), offset(offset_), scale(scale_) {
  AOB_REQUIRE(nvalid > 0, "centroider: nvalid must be > 0");
  AOB_REQUIRE(type >= 0 && type <= 5, "centroider: unknown type");
  AOB_CUDA(cudaSetDevice(device));
  ref.alloc(nslopes());
  intensities.alloc(type == AOB_CENTRO_MASKEDPIX ? nvalid + 1 : nvalid);  // maskedpix: pixels, then their sum
  fused_slopes.alloc(nslopes());
  if (type == AOB_CENTRO_MASKEDPIX) {  // the reference starts its reference slopes at 1 (maskedPix.cpp:44-45)
    std::vector<float> one(nvalid, 1.f);
    ref.upload(one.data(), nvalid);
  }
}

bool aob_centro::fused_ready() const {
  return wfs != nullptr && wfs->fused == this && fused_gen == wfs->image_gen &&
         fused_params_gen == params_gen;
}

// dark 0, flat 1 and the identity pixel table for an m x n image when absent (init_calib,
// sutra_centroider.cpp:104-127)
void aob_centro::init_calib() {
  const int64_t n = (int64_t)img_m * img_n;
  if (!img.p || img.n != n) img.alloc(n);
  if (!dark.p || dark.n != n) dark.alloc(n);
  if (!flat.p || flat.n != n) {
    flat.alloc(n);
    std::vector<float> one(n, 1.f);
    flat.upload(one.data(), n);
  }
  if (!lut.p || lut.n != n) {
    lut.alloc(n);
    std::vector<int32_t> id(n);
    for (int64_t i = 0; i < n; ++i) id[i] = (int32_t)i;
    lut.upload(id.data(), n);
  }
}

void aob_centro::calibrate(cudaStream_t s, bool valid_only) {
  AOB_REQUIRE(raw_u16 ? img_raw_u16.p != nullptr : img_raw.p != nullptr, "calibrate_img: image not loaded");
  AOB_CUDA(cudaSetDevice(device));
  init_calib();
  const int64_t n = (int64_t)img_m * img_n;
  if (!valid_only) {
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 4096);
    if (raw_u16)
      calib_kernel<uint16_t><<<grid, 256, 0, s>>>(img_raw_u16.p, img.p, dark.p, flat.p, lut.p, n);
    else
      calib_kernel<float><<<grid, 256, 0, s>>>(img_raw.p, img.p, dark.p, flat.p, lut.p, n);
    AOB_LAUNCH_CHECK("calib_kernel");
    return;
  }
  AOB_REQUIRE(validx.p != nullptr, "calibrate_img_validPix: valid positions not loaded");
  // pyramid / masked-pixel centroiders list single pixels; SH ones npix x npix windows
  const bool pixels = type == AOB_CENTRO_PYR || type == AOB_CENTRO_MASKEDPIX;
  const int nv = (int)validx.n, np = pixels ? 1 : npix;
  AOB_REQUIRE(np > 0, "calibrate_img_validPix: npix not set");
  AOB_CUDA(cudaMemsetAsync(img.p, 0, sizeof(float) * n, s));
  const int64_t work = (int64_t)nv * np * np;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, 4096));
  if (raw_u16)
    calib_valid_kernel<uint16_t><<<grid, 256, 0, s>>>(img_raw_u16.p, img.p, dark.p, flat.p, lut.p, validx.p,
                                                      validy.p, nv, np, img_m);
  else
    calib_valid_kernel<float><<<grid, 256, 0, s>>>(img_raw.p, img.p, dark.p, flat.p, lut.p, validx.p, validy.p, nv,
                                                   np, img_m);
  AOB_LAUNCH_CHECK("calib_valid_kernel");
}

void aob_centro::get_cog(float *dev_slopes, cudaStream_t s) {
  if (type == AOB_CENTRO_MASKEDPIX) {
    AOB_REQUIRE(validx.p != nullptr && validx.n >= nvalid, "get_maskedPix: valid pixel positions not loaded");
    const float *im;
    int ns;
    if (pyr) {
      im = pyr->binimg.p;
      ns = pyr->nbin();
    } else {
      AOB_REQUIRE(img.p != nullptr, "get_maskedPix: no image (attach a pyramid sensor or load_img + calibrate_img)");
      im = img.p;
      ns = img_m;
    }
    AOB_CUDA(cudaSetDevice(device));
    masked_pix_kernel<<<1, MASKED_THREADS, 0, s>>>(im, ns, validx.p, validy.p, nvalid, ref.p, dev_slopes,
                                                   intensities.p);
    AOB_LAUNCH_CHECK("masked_pix_kernel");
    return;
  }
  if (type == AOB_CENTRO_BPCOG) {
    AOB_REQUIRE(npix > 0 && npix * npix <= 1024, "get_bpcog: npix not set (or npix^2 > 1024)");
    AOB_REQUIRE(validx.p != nullptr && validx.n >= nvalid, "get_bpcog: valid positions not loaded");
    AOB_REQUIRE(nmax < bpcog_block(npix * npix), "get_bpcog: nmax must be below the padded pixel count");
    float *im;
    int size;
    if (wfs) {
      im = wfs->binimg.p;
      size = wfs->npix * wfs->nxsub;
    } else {
      AOB_REQUIRE(img.p != nullptr, "get_bpcog: no image (load_img + calibrate_img first)");
      im = img.p;
      size = img_m;
    }
    AOB_CUDA(cudaSetDevice(device));
    const int npad = bpcog_block(npix * npix) - npix * npix;
    const int grid = std::max(1, std::min((nvalid + 7) / 8, num_sms(device) * 8));
    bpcog_kernel<<<grid, 256, 0, s>>>(im, size, validx.p, validy.p, nvalid, npix, nmax, npad, scale, offset, ref.p,
                                      order, dev_slopes, intensities.p);
    AOB_LAUNCH_CHECK("bpcog_kernel");
    if (wfs) ++wfs->image_gen;  // the image now holds the thresholded pixels
    return;
  }
  if (type == 3) {
    AOB_REQUIRE(validx.p != nullptr && validx.n >= 4 * (int64_t)nvalid, "get_pyr: 4 * nvalid valid positions not loaded");
    const float *im;
    int ns;
    if (pyr) {
      im = pyr->binimg.p;
      ns = pyr->nbin();
    } else {
      AOB_REQUIRE(img.p != nullptr, "get_pyr: no image (attach a pyramid sensor or load_img + calibrate_img)");
      im = img.p;
      ns = img_m;
    }
    AOB_CUDA(cudaSetDevice(device));
    const int nparts = (nvalid + PYR_SLOPE_THREADS - 1) / PYR_SLOPE_THREADS;
    if (pyr_partial.n < nparts) pyr_partial.alloc(nparts);
    pyr_flux_kernel<<<nparts, PYR_SLOPE_THREADS, 0, s>>>(im, ns, validx.p, validy.p, nvalid, intensities.p,
                                                        pyr_partial.p);
    AOB_LAUNCH_CHECK("pyr_flux_kernel");
    pyr_slopes_kernel<<<nparts, PYR_SLOPE_THREADS, 0, s>>>(im, ns, validx.p, validy.p, nvalid, scale, valid_thresh,
                                                          pyr_method, ref.p, order, pyr_partial.p, nparts, dev_slopes,
                                                          intensities.p);
    AOB_LAUNCH_CHECK("pyr_slopes_kernel");
    return;
  }
  AOB_REQUIRE(type <= 2, "get_cog: not a CoG-family centroider");
  AOB_REQUIRE(npix > 0, "get_cog: npix not set");
  AOB_REQUIRE(validx.p != nullptr && validx.n >= nvalid, "get_cog: valid positions not loaded");
  if (type == 2) AOB_REQUIRE(weights.p != nullptr, "wcog: weights not loaded");
  AOB_CUDA(cudaSetDevice(device));
  if (fused_ready()) {
    AOB_CUDA(cudaMemcpyAsync(dev_slopes, fused_slopes.p, sizeof(float) * 2 * nvalid,
                             cudaMemcpyDeviceToDevice, s));
    if (type == 1) {
      const int n = npix * npix * nvalid;
      tcog_writeback_kernel<<<std::min((n + 255) / 256, 4096), 256, 0, s>>>(
          wfs->binimg.p, wfs->npix * wfs->nxsub, validx.p, validy.p, nvalid, npix, threshold);
      AOB_LAUNCH_CHECK("tcog_writeback_kernel");
      ++wfs->image_gen;  // a second get_cog thresholds again, as the reference does
    }
    return;
  }
  CogArgs A{};
  if (wfs) {
    A.img = wfs->binimg.p;
    A.size = wfs->npix * wfs->nxsub;
  } else {
    AOB_REQUIRE(img.p != nullptr, "get_cog: no image (load_img + calibrate_img first)");
    A.img = img.p;
    A.size = img_m;
  }
  A.img_out = (type == 1) ? const_cast<float *>(A.img) : nullptr;
  A.validx = validx.p;
  A.validy = validy.p;
  A.nvalid = nvalid;
  A.npix = npix;
  A.kind = type;
  A.order = order;
  A.scale = scale;
  A.offset = offset;
  A.thresh = threshold;
  A.ref = ref.p;
  A.weights = weights.p;
  A.wper = weights_per_sub;
  A.slopes = dev_slopes;
  A.intens = intensities.p;
  const int warps_per_block = 8;
  const int grid = std::max(1, std::min((nvalid + warps_per_block - 1) / warps_per_block, num_sms(device) * 8));
  cog_kernel<<<grid, warps_per_block * 32, 0, s>>>(A);
  AOB_LAUNCH_CHECK("cog_kernel");
  if (wfs && type == 1) ++wfs->image_gen;
}
