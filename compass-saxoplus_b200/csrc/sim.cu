// Closed-loop support: turbulent layers (Fried-Clark extrusion), raytracing of
// layers and DM shapes into a pupil phase, DM shape from commands, and the
// target PSF / Strehl.
//
// Reference interfaces replaced (paths within the reference project):
//   SutraTurbuScreen::extrude / refresh_screen   libsutra/src.cpp/sutra_tscreen.cpp:113-220
//   SutraAtmos::move_atmos                       libsutra/src.cpp/sutra_atmos.cpp:82-100
//   iterkolmo.AB factorisation (SVDs)            shesha/shesha/util/iterkolmo.py:201-267
//   generic_raytrace (bilinear)                  libsutra/src.cu/sutra_target.cu:25-70
//   dmshape_krnl / compShape2                    libsutra/src.cu/sutra_dm.cu:43-133
//   SutraSource::comp_image / comp_strehl        libsutra/src.cpp/sutra_source.cpp:397-515
//
// Layout: each layer keeps two n x n screens (x fastest) and ping-pongs between
// them on every extrusion (shift + new column in one pass); A and B are stored
// row-major so that the extrusion GEMVs stream contiguous rows.  The DM keeps a
// pixel-major CSR of (actuator, influence weight) pairs built from the
// influence cube, so the shape is one gather per pixel.

#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "aob_objects.hpp"
#include "fft.cuh"
#include "sim.hpp"

namespace aob {

// ------------------------------------------------------------------ extrusion
__global__ void extrude_gemv_kernel(const float *screen, int n, int nst, const float *Arm, const float *Brm,
                                    const uint32_t *ist, int x0ref, float amp, uint32_t k0, uint32_t k1,
                                    uint32_t counter, uint32_t layer, float *y) {
  extern __shared__ float sh[];
  float *z = sh;
  float *xi = sh + nst;
  const float ref = screen[x0ref];
  for (int t = threadIdx.x; t < nst; t += blockDim.x) z[t] = screen[ist[t]] - ref;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const U4 w = philox4x32_10(U4{(uint32_t)t, counter, 2u, layer}, k0, k1);
    const float u1 = ((float)(w.x >> 8) + 0.5f) * 5.9604644775390625e-08f;
    const float u2 = ((float)(w.z >> 8) + 0.5f) * 5.9604644775390625e-08f;
    xi[t] = sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int i = blockIdx.x * nw + warp; i < n; i += gridDim.x * nw) {
    const float *a = Arm + (size_t)i * nst;
    const float *b = Brm + (size_t)i * n;
    float sa = 0.f, sb = 0.f;
    for (int t = lane; t < nst; t += 32) sa = fmaf(a[t], z[t], sa);
    for (int t = lane; t < n; t += 32) sb = fmaf(b[t], xi[t], sb);
    sa = warp_sum(sa);
    sb = warp_sum(sb);
    if (lane == 0) y[i] = (sa + amp * sb) + ref;
  }
}

// Shift the screen by one sample and insert the new column / row, following
// the direction conventions of SutraTurbuScreen::extrude (dir +-1 along x,
// +-2 along y; negative directions insert at index 0 in reversed order).
__global__ void extrude_shift_kernel(float *dst, const float *src, const float *y, int n, int dir) {
  const int64_t nn = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nn; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % n), j = (int)(t / n);
    float v;
    if (dir == 1)
      v = (i < n - 1) ? src[(i + 1) + (int64_t)j * n] : y[j];
    else if (dir == -1)
      v = (i > 0) ? src[(i - 1) + (int64_t)j * n] : y[n - 1 - j];
    else if (dir == 2)
      v = (j < n - 1) ? src[i + (int64_t)(j + 1) * n] : y[i];
    else
      v = (j > 0) ? src[i + (int64_t)(j - 1) * n] : y[n - 1 - i];
    dst[t] = v;
  }
}

// One extrusion of every job's layer in one launch (blockIdx.y = job): the rows
// of extrude_gemv_kernel write the new column / row straight to its place in
// the next screen, and the grid shifts the rest of the screen by one sample as
// extrude_shift_kernel does.  The arithmetic of both is unchanged (each row's
// dot products keep their order), so the screens equal the two-kernel
// sequence's bit for bit, with one launch per pass of extrusions instead of
// two per layer.  The launch is short and its data cold, so it is bound by
// chains of memory latency, not bytes: a warp loads its first row of A and B
// into registers before anything else (a lane's share fits for nst, n <= 512),
// the stencil's indexes are loaded at entry too and its screen values before
// the noise is generated, and the shift issues four loads per thread before
// their stores.
constexpr int EXTRUDE_PRE = 16;   // values of a row a lane holds, per operand
constexpr int EXTRUDE_PRE_Z = 2;  // stencil points a thread gathers ahead (nst <= 512)
constexpr int EXTRUDE_ILP = 4;    // shift loads in flight per thread

__global__ void __launch_bounds__(256) extrude_fused_kernel(const __grid_constant__ ExtrudeBatch B) {
  if ((int)blockIdx.y >= B.njobs) return;
  const ExtrudeJob &J = B.job[blockIdx.y];
  const int n = J.n, nst = J.nst, dir = J.dir;
  const float *__restrict__ src = J.src;
  float *__restrict__ dst = J.dst;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int r0 = blockIdx.x * nw + warp;
  const bool rows = (int)blockIdx.x * nw < n;  // this block computes rows (block-uniform)
  const bool prez = rows && nst <= EXTRUDE_PRE_Z * (int)blockDim.x;
  const bool pre = r0 < n && nst <= 32 * EXTRUDE_PRE && n <= 32 * EXTRUDE_PRE;
  float ref = 0.f;
  uint32_t iz[EXTRUDE_PRE_Z];
  if (rows) ref = src[J.x0ref];
  if (prez) {
#pragma unroll
    for (int q = 0; q < EXTRUDE_PRE_Z; ++q) {
      const int t = threadIdx.x + q * blockDim.x;
      iz[q] = t < nst ? __ldg(J.ist + t) : 0u;
    }
  }
  float pa[EXTRUDE_PRE], pb[EXTRUDE_PRE];
  if (pre) {
    const float *a = J.Arm + (size_t)r0 * nst;
    const float *b = J.Brm + (size_t)r0 * n;
#pragma unroll
    for (int q = 0; q < EXTRUDE_PRE; ++q) {
      const int t = lane + 32 * q;
      pa[q] = t < nst ? __ldg(a + t) : 0.f;
      pb[q] = t < n ? __ldg(b + t) : 0.f;
    }
  }
  // the shift; the new column / row is left to the rows below.  n*n < 2^31
  // (the stencil and column fit 48 KB of shared memory, so n < 12288).
  const int nn = n * n;
  const int off = dir == 1 ? 1 : dir == -1 ? -1 : dir == 2 ? n : -n;
  const int stride = gridDim.x * blockDim.x;
  for (int t0 = blockIdx.x * blockDim.x + threadIdx.x; t0 < nn; t0 += EXTRUDE_ILP * stride) {
    float v[EXTRUDE_ILP];
    bool keep[EXTRUDE_ILP];
#pragma unroll
    for (int u = 0; u < EXTRUDE_ILP; ++u) {
      const int t = t0 + u * stride;
      const int i = t % n, j = t / n;
      keep[u] = t < nn && (dir == 1 ? i < n - 1 : dir == -1 ? i > 0 : dir == 2 ? j < n - 1 : j > 0);
      v[u] = keep[u] ? src[t + off] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < EXTRUDE_ILP; ++u)
      if (keep[u]) dst[t0 + u * stride] = v[u];
  }
  if (!rows) return;
  extern __shared__ float sh[];
  float *z = sh;
  float *xi = sh + nst;
  float zv[EXTRUDE_PRE_Z];
  if (prez) {
#pragma unroll
    for (int q = 0; q < EXTRUDE_PRE_Z; ++q) zv[q] = (int)(threadIdx.x + q * blockDim.x) < nst ? src[iz[q]] : 0.f;
  } else {
    for (int t = threadIdx.x; t < nst; t += blockDim.x) z[t] = src[J.ist[t]] - ref;
  }
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const U4 w = philox4x32_10(U4{(uint32_t)t, J.counter, 2u, J.layer}, J.k0, J.k1);
    const float u1 = ((float)(w.x >> 8) + 0.5f) * 5.9604644775390625e-08f;
    const float u2 = ((float)(w.z >> 8) + 0.5f) * 5.9604644775390625e-08f;
    xi[t] = sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
  }
  if (prez) {
#pragma unroll
    for (int q = 0; q < EXTRUDE_PRE_Z; ++q) {
      const int t = threadIdx.x + q * blockDim.x;
      if (t < nst) z[t] = zv[q] - ref;
    }
  }
  __syncthreads();
  for (int r = r0; r < n; r += gridDim.x * nw) {
    float sa = 0.f, sb = 0.f;
    if (pre && r == r0) {
#pragma unroll
      for (int q = 0; q < EXTRUDE_PRE; ++q)
        if (lane + 32 * q < nst) sa = fmaf(pa[q], z[lane + 32 * q], sa);
#pragma unroll
      for (int q = 0; q < EXTRUDE_PRE; ++q)
        if (lane + 32 * q < n) sb = fmaf(pb[q], xi[lane + 32 * q], sb);
    } else {
      const float *a = J.Arm + (size_t)r * nst;
      const float *b = J.Brm + (size_t)r * n;
      for (int t = lane; t < nst; t += 32) sa = fmaf(a[t], z[t], sa);
      for (int t = lane; t < n; t += 32) sb = fmaf(b[t], xi[t], sb);
    }
    sa = warp_sum(sa);
    sb = warp_sum(sb);
    if (lane == 0) {
      // where extrude_shift_kernel puts y[r]
      int at;
      if (dir == 1)
        at = (n - 1) + r * n;
      else if (dir == -1)
        at = (n - 1 - r) * n;
      else if (dir == 2)
        at = r + (n - 1) * n;
      else
        at = n - 1 - r;
      dst[at] = (sa + J.amp * sb) + ref;
    }
  }
}

void launch_extrude(const ExtrudeBatch &B, int device, cudaStream_t s) {
  AOB_REQUIRE(B.njobs >= 1 && B.njobs <= EXTRUDE_MAX_JOBS, "extrude: bad job count");
  int nmax = 0;
  size_t sm = 0;
  for (int q = 0; q < B.njobs; ++q) {
    nmax = std::max(nmax, B.job[q].n);
    sm = std::max(sm, sizeof(float) * ((size_t)B.job[q].nst + B.job[q].n));
  }
  const int threads = 256;
  const int rows_per_cta = threads / 32;
  // enough blocks for every row of the widest layer and for four shift loads per thread
  const int64_t nn = (int64_t)nmax * nmax;
  const int64_t want = std::max<int64_t>((nmax + rows_per_cta - 1) / rows_per_cta,
                                         (nn + threads * EXTRUDE_ILP - 1) / (threads * EXTRUDE_ILP));
  const int gx = (int)std::max<int64_t>(1, std::min<int64_t>(want, 4 * num_sms(device)));
  extrude_fused_kernel<<<dim3(gx, B.njobs), threads, sm, s>>>(B);
  AOB_LAUNCH_CHECK("extrude_fused_kernel");
}

// ------------------------------------------------------------------ raytrace
__global__ void raytrace_kernel(float *out, int nx, int ny, RaySources S, int reset) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= nx || y >= ny) return;
  float acc = reset ? 0.f : out[x + y * nx];
  for (int l = 0; l < S.n; ++l) {
    const int N = S.dim[l];
    const float xref = (float)x - nx / 2.0f + nx / 2.0f + S.xoff[l];
    const float yref = (float)y - ny / 2.0f + ny / 2.0f + S.yoff[l];
    const int iref = (int)xref, jref = (int)yref;
    const float xs = xref - iref, ys = yref - jref;
    const float wx1 = 1.0f - xs, wx2 = xs, wy1 = 1.0f - ys, wy2 = ys;
    if (iref + 1 < N && jref + 1 < N) {
      const float *d = S.data[l];
      acc += (wx1 * wy1 * d[iref + jref * N] + wx2 * wy1 * d[iref + 1 + jref * N] +
              wx1 * wy2 * d[iref + (jref + 1) * N] + wx2 * wy2 * d[iref + 1 + (jref + 1) * N]);
    } else {
      acc += 0.0f;
    }
  }
  out[x + y * nx] = acc;
}

// ------------------------------------------------------------------ DM shape
// Each pixel sums its actuators' weighted commands in CSR order.  A group of up
// to 16 entries -- every entry of most pixels -- has its index and weight loads
// issued before its command gathers and those before the sum, which keeps the
// entry order.  On saxo40's DM (77,284 pixels, 1.06 M entries, at most 25 per
// pixel) this takes the kernel from 7.07 to 6.13 us after an L2 flush; larger
// groups and an entry-major (coalesced) copy of the lists were slower.
constexpr int DM_GROUP = 16;

__global__ void dm_shape_kernel(float *shape, int npix, const int32_t *rowptr, const int32_t *act, const float *w,
                                const float *com) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
    const int k0 = __ldg(rowptr + p), k1 = __ldg(rowptr + p + 1);
    float v = 0.f;
    for (int k = k0; k < k1; k += DM_GROUP) {
      int a[DM_GROUP];
      float ww[DM_GROUP], c[DM_GROUP];
#pragma unroll
      for (int u = 0; u < DM_GROUP; ++u) {
        a[u] = k + u < k1 ? __ldg(act + k + u) : 0;
        ww[u] = k + u < k1 ? __ldg(w + k + u) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < DM_GROUP; ++u) c[u] = k + u < k1 ? com[a[u]] : 0.f;
#pragma unroll
      for (int u = 0; u < DM_GROUP; ++u)
        if (k + u < k1) v = fmaf(c[u], ww[u], v);
    }
    shape[p] = v;
  }
}

// ------------------------------------------------------------------ target PSF
__global__ void target_fill_kernel(float2 *amp, const float *phase, const float *mask, float scale, int npup, int nfft) {
  const int64_t n2 = (int64_t)nfft * nfft;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n2; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % nfft), j = (int)(t / nfft);
    float2 v = make_float2(0.f, 0.f);
    if (i < npup && j < npup) {
      const int q = i + j * npup;
      if (mask[q] > 0.f) {
        float s, c;
        sincosf(scale * phase[q], &s, &c);
        v = make_float2(c, s);
      }
    }
    amp[t] = v;
  }
}

__global__ void target_abs2_kernel(float *se, float *le, const float2 *amp, int64_t n2, float norm, int comp_le,
                                   unsigned int *max_se, unsigned int *max_le) {
  unsigned int mse = 0, mle = 0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n2; t += (int64_t)gridDim.x * blockDim.x) {
    const float2 a = amp[t];
    const float v = (a.x * a.x + a.y * a.y) * norm * norm;
    se[t] = v;
    float l = le[t];
    if (comp_le) {
      l += v;
      le[t] = l;
    }
    mse = max(mse, __float_as_uint(v));
    mle = max(mle, __float_as_uint(l));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mse = max(mse, __shfl_xor_sync(0xffffffffu, mse, o));
    mle = max(mle, __shfl_xor_sync(0xffffffffu, mle, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(max_se, mse);
    atomicMax(max_le, mle);
  }
}

// Index of the largest value (the first one on ties, as cuBLAS Isamax used by
// CarmaObj::aimax): one 64-bit max over (value bits, ~index) -- the images are
// non-negative, so their float bits order like their values.
__global__ void argmax_kernel(const float *img, int64_t n, unsigned long long *best) {
  unsigned long long m = 0ull;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long key =
        ((unsigned long long)__float_as_uint(img[t]) << 32) | (unsigned long long)(0xffffffffu - (uint32_t)t);
    m = key > m ? key : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(0xffffffffu, m, o);
    m = v > m ? v : m;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(best, m);
}

// The (2 h + 1)^2 window of an n x n image centred on pixel c, read as if the
// image were periodic (extract_krnl with roll, libcarma/src.cu/carma_obj.cu:454-488).
__global__ void extract_roll_kernel(float *out, const float *img, int n, const unsigned long long *best, int h) {
  const int w = 2 * h + 1;
  const int t = threadIdx.x;
  if (t >= w * w) return;
  const uint32_t c = 0xffffffffu - (uint32_t)(*best & 0xffffffffull);
  const int cy = (int)(c / n), cx = (int)(c % n);
  int y = cy + t / w - h, x = cx + t % w - h;
  y = (y + n) % n;
  x = (x + n) % n;
  out[t] = img[x + (int64_t)y * n];
}

}  // namespace aob

using namespace aob;

// =================================================================== atmosphere
aob_atmos::Layer::Layer(int dim_, int nst_, float r0, float alt, float dx, float dy, int64_t seed_)
    : dim(dim_), nst(nst_), r0_pix(r0), altitude(alt), deltax(dx), deltay(dy), seed(seed_) {
  amplitude = powf(r0, -5.0f / 6.0f) * 0.5f / (2.0f * (float)M_PI);
  scr[0].alloc((int64_t)dim * dim);
  scr[1].alloc((int64_t)dim * dim);
}

aob::ExtrudeJob aob_atmos::Layer::next_job(int dir, int layer_index) {
  const int n = dim;
  aob::ExtrudeJob J;
  J.src = scr[cur].p;
  J.dst = scr[1 - cur].p;
  J.Arm = Arm.p;
  J.Brm = Brm.p;
  J.ist = (dir == 1 || dir == -1) ? istx.p : isty.p;
  J.n = n;
  J.nst = nst;
  J.dir = dir;
  J.x0ref = (dir == 1 || dir == -2) ? n - 1 : n * (n - 1);
  J.amp = amplitude;
  const uint64_t sd = (uint64_t)seed;
  J.k0 = (uint32_t)(sd & 0xffffffffu);
  J.k1 = (uint32_t)(sd >> 32);
  J.counter = (uint32_t)counter;
  J.layer = (uint32_t)layer_index;
  cur = 1 - cur;
  ++counter;
  return J;
}

void aob_atmos::Layer::extrude(int dir, int layer_index, cudaStream_t s) {
  aob::ExtrudeBatch B{};
  B.njobs = 1;
  B.job[0] = next_job(dir, layer_index);
  aob::launch_extrude(B, device, s);
}

int aob_atmos::add_screen(int dim, int nst, float r0_pix, float alt, float dx, float dy, const float *A,
                          const float *B, const uint32_t *istx_h, const uint32_t *isty_h, int64_t seed) {
  AOB_REQUIRE(dim > 2 && nst > 0, "atmos.add_screen: bad sizes");
  AOB_REQUIRE(A && B && istx_h && isty_h, "atmos.add_screen: null arrays");
  AOB_REQUIRE(sizeof(float) * (nst + dim) <= 48 * 1024, "atmos.add_screen: stencil too large");
  for (int t = 0; t < nst; ++t)
    AOB_REQUIRE(istx_h[t] < (uint32_t)(dim * dim) && isty_h[t] < (uint32_t)(dim * dim),
                "atmos.add_screen: stencil index out of range");
  AOB_CUDA(cudaSetDevice(device));
  layers.emplace_back(new Layer(dim, nst, r0_pix, alt, dx, dy, seed));
  Layer &L = *layers.back();
  L.device = device;
  // A: dim x nst and B: dim x dim column-major (the reference's layout) -> row-major copies
  std::vector<float> ar((size_t)dim * nst), br((size_t)dim * dim);
  for (int i = 0; i < dim; ++i) {
    for (int t = 0; t < nst; ++t) ar[(size_t)i * nst + t] = A[i + (size_t)t * dim];
    for (int t = 0; t < dim; ++t) br[(size_t)i * dim + t] = B[i + (size_t)t * dim];
  }
  L.Arm.alloc((int64_t)dim * nst);
  L.Arm.upload(ar.data(), (int64_t)dim * nst);
  L.Brm.alloc((int64_t)dim * dim);
  L.Brm.upload(br.data(), (int64_t)dim * dim);
  L.istx.alloc(nst);
  L.istx.upload(istx_h, nst);
  L.isty.alloc(nst);
  L.isty.upload(isty_h, nst);
  return (int)layers.size() - 1;
}

void aob_atmos::refresh(int idx, cudaStream_t s) {
  AOB_REQUIRE(idx >= 0 && idx < (int)layers.size(), "atmos.refresh_screen: index out of range");
  AOB_CUDA(cudaSetDevice(device));
  Layer &L = *layers[idx];
  AOB_CUDA(cudaMemsetAsync(L.scr[L.cur].p, 0, L.scr[L.cur].bytes(), s));
  L.accumx = L.accumy = 0.f;
  for (int i = 0; i < 2 * L.dim; ++i) L.extrude(L.deltax > 0 ? 1 : -1, idx, s);
}

// Each layer's extrusions of this move run in order (x first, then y, as
// SutraAtmos::move_atmos does); the layers are independent, so pass r of the
// move extrudes every layer that has an r-th extrusion in one launch.
void aob_atmos::move(cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  std::vector<std::vector<int>> dirs(layers.size());
  size_t passes = 0;
  for (size_t l = 0; l < layers.size(); ++l) {
    Layer &L = *layers[l];
    L.accumx += L.deltax;
    L.accumy += L.deltay;
    const int dx = (int)L.accumx, dy = (int)L.accumy;
    const int cx = dx > 0 ? 1 : -1, cy = dy > 0 ? 1 : -1;
    for (int c = 0; c < cx * dx; ++c) dirs[l].push_back(1 * cx);
    L.accumx -= dx;
    for (int c = 0; c < cy * dy; ++c) dirs[l].push_back(2 * cy);
    L.accumy -= dy;
    passes = std::max(passes, dirs[l].size());
  }
  for (size_t r = 0; r < passes; ++r) {
    aob::ExtrudeBatch B{};
    B.njobs = 0;
    for (size_t l = 0; l < layers.size(); ++l) {
      if (r >= dirs[l].size()) continue;
      B.job[B.njobs++] = layers[l]->next_job(dirs[l][r], (int)l);
      if (B.njobs == aob::EXTRUDE_MAX_JOBS) {
        aob::launch_extrude(B, device, s);
        B.njobs = 0;
      }
    }
    if (B.njobs) aob::launch_extrude(B, device, s);
  }
}

namespace {
void cublas_ok(cublasStatus_t st, const char *w) {
  if (st != CUBLAS_STATUS_SUCCESS) throw aob::Error(std::string(w) + ": cublas status " + std::to_string((int)st));
}
void cusolver_ok(cusolverStatus_t st, const char *w) {
  if (st != CUSOLVER_STATUS_SUCCESS) throw aob::Error(std::string(w) + ": cusolver status " + std::to_string((int)st));
}
// symmetric eigen-decomposition in place (ascending eigenvalues)
void dsyevd(cusolverDnHandle_t hs, double *M, double *ev, int n) {
  int lwork = 0;
  cusolver_ok(cusolverDnDsyevd_bufferSize(hs, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, M, n, ev, &lwork),
              "Dsyevd_bufferSize");
  DevBuf<double> work(std::max(lwork, 1));
  DevBuf<int> info(1);
  cusolver_ok(cusolverDnDsyevd(hs, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, M, n, ev, work.p, lwork, info.p),
              "Dsyevd");
  int h = 0;
  AOB_CUDA(cudaMemcpy(&h, info.p, sizeof(int), cudaMemcpyDeviceToHost));
  AOB_REQUIRE(h == 0, "eigen decomposition did not converge");
}
}  // namespace

// iterkolmo.AB after the covariances (iterkolmo.py:225-251), in float64 on the GPU:
// zz^+ from the eigen-decomposition with the smallest mode dropped, A = xz zz^+,
// bbt = xx - A xz^T, B = U sqrt(max(s, 0)) from the eigen-decomposition of bbt.
void aob::kolmo_factor_ab(int device, int n, int nst, const double *zz, const double *xz, const double *xx, float *A,
                          float *B) {
  AOB_CUDA(cudaSetDevice(device));
  DevBuf<double> dzz((int64_t)nst * nst), dxz((int64_t)n * nst), dxx((int64_t)n * n), ev(std::max(n, nst));
  dzz.upload(zz, dzz.n);
  dxz.upload(xz, dxz.n);
  dxx.upload(xx, dxx.n);
  cublasHandle_t hb;
  cusolverDnHandle_t hs;
  cublas_ok(cublasCreate(&hb), "cublasCreate");
  if (cusolverDnCreate(&hs) != CUSOLVER_STATUS_SUCCESS) {
    cublasDestroy(hb);
    throw Error("cusolverDnCreate failed");
  }
  try {
    dsyevd(hs, dzz.p, ev.p, nst);
    std::vector<double> lam(nst);
    AOB_CUDA(cudaMemcpy(lam.data(), ev.p, sizeof(double) * nst, cudaMemcpyDeviceToHost));
    std::vector<double> inv(nst, 0.0);
    for (int i = 1; i < nst; ++i) inv[i] = 1.0 / lam[i];  // smallest mode (index 0) dropped
    std::vector<double> V((size_t)nst * nst);
    AOB_CUDA(cudaMemcpy(V.data(), dzz.p, sizeof(double) * V.size(), cudaMemcpyDeviceToHost));
    for (int c = 0; c < nst; ++c)
      for (int r = 0; r < nst; ++r) V[r + (size_t)c * nst] *= inv[c];
    DevBuf<double> VS((int64_t)nst * nst), pinv((int64_t)nst * nst), dA((int64_t)n * nst), bbt((int64_t)n * n);
    VS.upload(V.data(), VS.n);
    const double one = 1.0, zero = 0.0, mone = -1.0;
    cublas_ok(cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_T, nst, nst, nst, &one, VS.p, nst, dzz.p, nst, &zero, pinv.p, nst),
              "Dgemm pinv");
    cublas_ok(cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_N, n, nst, nst, &one, dxz.p, n, pinv.p, nst, &zero, dA.p, n),
              "Dgemm A");
    AOB_CUDA(cudaMemcpy(bbt.p, dxx.p, sizeof(double) * bbt.n, cudaMemcpyDeviceToDevice));
    cublas_ok(cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_T, n, n, nst, &mone, dA.p, n, dxz.p, n, &one, bbt.p, n),
              "Dgemm bbt");
    dsyevd(hs, bbt.p, ev.p, n);
    std::vector<double> mu(n), U((size_t)n * n), hA((size_t)n * nst);
    AOB_CUDA(cudaMemcpy(mu.data(), ev.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    AOB_CUDA(cudaMemcpy(U.data(), bbt.p, sizeof(double) * U.size(), cudaMemcpyDeviceToHost));
    AOB_CUDA(cudaMemcpy(hA.data(), dA.p, sizeof(double) * hA.size(), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < hA.size(); ++i) A[i] = (float)hA[i];
    for (int c = 0; c < n; ++c) {
      const double sq = std::sqrt(std::max(mu[c], 0.0));
      for (int r = 0; r < n; ++r) B[r + (size_t)c * n] = (float)(U[r + (size_t)c * n] * sq);
    }
  } catch (...) {
    cublasDestroy(hb);
    cusolverDnDestroy(hs);
    throw;
  }
  cublasDestroy(hb);
  cusolverDnDestroy(hs);
}

// =================================================================== DM
aob_dm::aob_dm(int device_, int dim_, int nact_, int isz, const float *influ, const int32_t *i1, const int32_t *j1)
    : device(device_), dim(dim_), nact(nact_), influsize(isz) {
  AOB_REQUIRE(dim > 0 && nact > 0 && isz > 0, "dm: sizes must be > 0");
  AOB_REQUIRE(influ && i1 && j1, "dm: null arrays");
  AOB_CUDA(cudaSetDevice(device));
  // pixel-major CSR: pixel (i1[a]+x, j1[a]+y) receives influ[x, y, a] * com[a]
  const int64_t npix = (int64_t)dim * dim;
  std::vector<int32_t> cnt(npix + 1, 0);
  for (int a = 0; a < nact; ++a)
    for (int y = 0; y < isz; ++y)
      for (int x = 0; x < isz; ++x) {
        const int px = i1[a] + x, py = j1[a] + y;
        if (px >= 0 && px < dim && py >= 0 && py < dim) ++cnt[px + (int64_t)py * dim + 1];
      }
  for (int64_t p = 0; p < npix; ++p) cnt[p + 1] += cnt[p];
  const int64_t nnz = cnt[npix];
  std::vector<int32_t> act(nnz), fill(cnt.begin(), cnt.end() - 1);
  std::vector<float> w(nnz);
  for (int a = 0; a < nact; ++a)
    for (int y = 0; y < isz; ++y)
      for (int x = 0; x < isz; ++x) {
        const int px = i1[a] + x, py = j1[a] + y;
        if (px >= 0 && px < dim && py >= 0 && py < dim) {
          const int64_t p = px + (int64_t)py * dim;
          const int32_t k = fill[p]++;
          act[k] = a;
          w[k] = influ[x + (size_t)y * isz + (size_t)a * isz * isz];
        }
      }
  rowptr.alloc(npix + 1);
  rowptr.upload(cnt.data(), npix + 1);
  actidx.alloc(std::max<int64_t>(nnz, 1));
  actidx.upload(act.data(), nnz);
  weight.alloc(std::max<int64_t>(nnz, 1));
  weight.upload(w.data(), nnz);
  shape.alloc(npix);
  com.alloc(nact);
  this->nnz = nnz;
}

void aob_dm::comp_shape(const float *dev_com, cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  const float *c = dev_com ? dev_com : com.p;
  if (dev_com && dev_com != com.p)
    AOB_CUDA(cudaMemcpyAsync(com.p, dev_com, sizeof(float) * nact, cudaMemcpyDeviceToDevice, s));
  const int64_t npix = (int64_t)dim * dim;
  dm_shape_kernel<<<(int)std::min<int64_t>((npix + 255) / 256, 8192), 256, 0, s>>>(shape.p, (int)npix, rowptr.p,
                                                                                   actidx.p, weight.p, c);
  AOB_LAUNCH_CHECK("dm_shape_kernel");
}

// =================================================================== target
aob_target::aob_target(int device_, int npup_, int nfft_, const float *pupil, float lambda_um)
    : device(device_), npup(npup_), nfft(nfft_), lambda(lambda_um) {
  AOB_REQUIRE(npup > 0 && nfft >= npup && (nfft & (nfft - 1)) == 0, "target: nfft must be a power of two >= npup");
  AOB_CUDA(cudaSetDevice(device));
  mask.alloc((int64_t)npup * npup);
  mask.upload(pupil, (int64_t)npup * npup);
  npts = 0;
  for (int64_t i = 0; i < (int64_t)npup * npup; ++i) npts += pupil[i] > 0.f ? 1 : 0;
  phase.alloc((int64_t)npup * npup);
  amp.alloc((int64_t)nfft * nfft);
  se.alloc((int64_t)nfft * nfft);
  le.alloc((int64_t)nfft * nfft);
  maxes.alloc(2);
}

void aob_target::comp_image(const float *dev_phase, bool comp_le, cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  const int64_t n2 = (int64_t)nfft * nfft;
  const float scale = (float)(2.0 * M_PI / (double)lambda);
  target_fill_kernel<<<(int)std::min<int64_t>((n2 + 255) / 256, 8192), 256, 0, s>>>(
      amp.p, dev_phase ? dev_phase : phase.p, mask.p, scale, npup, nfft);
  AOB_LAUNCH_CHECK("target_fill_kernel");
  fft2d(amp.p, nfft, 1, false, device, s);
  AOB_CUDA(cudaMemsetAsync(maxes.p, 0, 2 * sizeof(unsigned int), s));
  target_abs2_kernel<<<std::min<int64_t>((n2 + 255) / 256, 2 * 148), 256, 0, s>>>(
      se.p, le.p, amp.p, n2, 1.0f / (float)npts, comp_le ? 1 : 0, maxes.p, maxes.p + 1);
  AOB_LAUNCH_CHECK("target_abs2_kernel");
  if (comp_le) ++le_count;
}

void aob_target::strehl(float *sr_se, float *sr_le, cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  unsigned int m[2];
  AOB_CUDA(cudaMemcpyAsync(m, maxes.p, sizeof(m), cudaMemcpyDeviceToHost, s));
  AOB_CUDA(cudaStreamSynchronize(s));
  float fse, fle;
  std::memcpy(&fse, &m[0], 4);
  std::memcpy(&fle, &m[1], 4);
  if (sr_se) *sr_se = fse;
  if (sr_le) *sr_le = le_count > 0 ? fle / (float)le_count : fse;
}

// SutraSource::fitmax2x1dSinc (libsutra/src.cpp/sutra_source.cpp:451-488): a
// parabola through the 3-pixel cross around the maximum gives its sub-pixel
// position (x0, y0); the peak there is the Shannon (sinc) interpolation of the
// 7 x 7 window, which the well-sampled image allows.  The window is read on the
// device, the fit on the host, as in the reference.
static float sinc_of(double x) {
  if (x == 0) return 1;
  x *= M_PI;
  return (float)(std::sin(x) / x);
}

float aob_target::fit_peak(const float *img, cudaStream_t s) {
  constexpr int H = 3, W = 2 * H + 1;
  const int64_t n2 = (int64_t)nfft * nfft;
  AOB_CUDA(cudaMemsetAsync(fit_best.p, 0, sizeof(unsigned long long), s));
  argmax_kernel<<<(int)std::min<int64_t>((n2 + 255) / 256, 2 * 148), 256, 0, s>>>(img, n2, fit_best.p);
  AOB_LAUNCH_CHECK("argmax_kernel");
  extract_roll_kernel<<<1, 64, 0, s>>>(fit_win.p, img, nfft, fit_best.p, H);
  AOB_LAUNCH_CHECK("extract_roll_kernel");
  float w[W * W];
  AOB_CUDA(cudaMemcpyAsync(w, fit_win.p, sizeof(w), cudaMemcpyDeviceToHost, s));
  AOB_CUDA(cudaStreamSynchronize(s));
  const int center = (W * W - 1) / 2;
  const float A = 0.5 * (w[center - W] + w[center + W]) - w[center];
  const float B = 0.5 * (w[center - 1] + w[center + 1]) - w[center];
  if (A * B == 0) return 0.f;  // (the reference reports it cannot estimate the Strehl)
  const float x0 = -0.5 * (w[center + W] - w[center - W]) / 2. / A;
  const float y0 = -0.5 * (w[center + 1] - w[center - 1]) / 2. / B;
  float val = 0.f;
  int ind = 0;
  for (int i = -H; i < H + 1; ++i) {
    const float ti = sinc_of(x0 - i);
    for (int j = -H; j < H + 1; ++j) {
      const float tj = sinc_of(y0 - j);
      val += ti * tj * w[ind++];
    }
  }
  return val;
}

void aob_target::strehl_fit(float *sr_se, float *sr_le, cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  if (!fit_best.p) {
    fit_best.alloc(1);
    fit_win.alloc(64);
  }
  const float fse = fit_peak(se.p, s);
  const float fle = fit_peak(le.p, s);
  if (sr_se) *sr_se = fse;
  if (sr_le) *sr_le = le_count > 0 ? fle / (float)le_count : fse;
}

void aob_target::reset_le(cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  AOB_CUDA(cudaMemsetAsync(le.p, 0, le.bytes(), s));
  le_count = 0;
}

// =================================================================== raytrace
void aob::raytrace(float *out, int nx, int ny, const RaySources &S, bool reset, cudaStream_t s) {
  dim3 th(32, 8), gr((nx + 31) / 32, (ny + 7) / 8);
  raytrace_kernel<<<gr, th, 0, s>>>(out, nx, ny, S, reset ? 1 : 0);
  AOB_LAUNCH_CHECK("raytrace_kernel");
}
