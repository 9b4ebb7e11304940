// Learned reconstructor: a 3-layer MLP from slopes to DM commands
// (in -> h1 -> h2 -> out, GELU on the hidden layers) plus a linear skip path
// in -> out, y = W3 h2 + b3 + Ws x.  With Ws set to the least-squares command
// matrix and W3 = 0 the untrained network is the LS reconstructor; training
// learns the non-linear correction on top of it.  Trained on the GPU with
// the project's own BF16 tensor-core GEMMs (tcgen05 / TMEM in mlp_tc.cuh, or
// mma.sync in mlp_gemm.cuh) and Adam, run in the
// loop by three batch-1 GEMV kernels, and backed by the least-squares MVM:
// when the norm of the predicted commands exceeds a threshold the step uses
// the LS commands instead.  There is no counterpart in the reference.
//
// Numerics: weights are FP32 masters with BF16 copies; inputs and hidden
// activations are rounded to BF16, every product is accumulated in FP32.
// The network works on scaled quantities: x = slopes * in_scale,
// commands = y * out_scale.  All dimensions are padded to multiples of 8
// (padding weights stay zero).

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "aob_objects.hpp"
#include "mlp_gemm.cuh"
#include "mlp_tc.cuh"
#include "mvm_core.cuh"
#include "mlp_fused.cuh"

namespace aob {

__global__ void f32_to_bf16_kernel(const float *src, __nv_bfloat16 *dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = __float2bfloat16_rn(src[i]);
}

// x [batch][nin] float -> xb [batch][pin] bf16 of x * scale, zero padding
// (the row loops below take four elements per thread and pass, all loads
// issued before any use, so that enough bytes are in flight per SM)
__global__ void mlp_input_kernel(const float *x, int nin, int pin, int batch, float scale, __nv_bfloat16 *xb) {
  const int nt = blockDim.x;
  for (int b = blockIdx.x; b < batch; b += gridDim.x)
    for (int i0 = threadIdx.x; i0 < pin; i0 += 4 * nt) {
      float v[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int i = i0 + k * nt;
        v[k] = i < nin ? __ldcs(x + (int64_t)b * nin + i) : 0.f;
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int i = i0 + k * nt;
        if (i < pin) xb[(int64_t)b * pin + i] = __float2bfloat16_rn(v[k] * scale);
      }
    }
}

__global__ void mlp_output_kernel(const float *y, int nout, int pout, int batch, float scale, float *out) {
  for (int b = blockIdx.x; b < batch; b += gridDim.x)
    for (int o = threadIdx.x; o < nout; o += blockDim.x) out[(int64_t)b * nout + o] = y[(int64_t)b * pout + o] * scale;
}

// Mean-squared error on the scaled outputs: d = y - t / out_scale; the loss
// gradient 2 d / (batch * nout) goes to dy (bf16); per-block partial sums of d^2.
__global__ void mlp_loss_kernel(const float *y, const float *t, int nout, int pout, int batch, float inv_out_scale,
                                __nv_bfloat16 *dy, float *part) {
  __shared__ float red[256];
  const float g = 2.f / ((float)batch * (float)nout);
  float acc = 0.f;
  const int nt = blockDim.x;
  for (int b = blockIdx.x; b < batch; b += gridDim.x)
    for (int o0 = threadIdx.x; o0 < pout; o0 += 4 * nt) {
      float yv[4], tv[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int o = o0 + k * nt;
        yv[k] = o < nout ? y[(int64_t)b * pout + o] : 0.f;
        tv[k] = o < nout ? __ldcs(t + (int64_t)b * nout + o) : 0.f;
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int o = o0 + k * nt;
        if (o >= pout) continue;
        float d = 0.f;
        if (o < nout) d = yv[k] - tv[k] * inv_out_scale;
        dy[(int64_t)b * pout + o] = __float2bfloat16_rn(g * d);
        acc += d * d;
      }
    }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void mlp_loss_final_kernel(const float *part, int nblocks, float denom, float *loss) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float s = 0.f;
    for (int i = 0; i < nblocks; ++i) s += part[i];
    *loss = s / denom;
  }
}

// bias gradient: column sums of a [batch][cols] bf16 matrix, batch order
// Column sums of d [batch][cols] (bias gradients) in two deterministic passes:
// partial sums over row chunks (block 32 columns x 8 row lanes, coalesced
// rows), then the chunks added in order.
constexpr int COLSUM_CHUNKS = 16;
// Partial column sums over a chunk of rows: a thread takes two adjacent
// columns (cols even: one 4-byte load per row, 128 bytes per warp) and rows
// r0 + ty + 8 j, four rows' loads issued before they are added (in row order).
__global__ void mlp_colsum_part_kernel(const __nv_bfloat16 *d, int batch, int cols, float *part) {
  __shared__ float red[8][2][33];
  const int c = 2 * (blockIdx.x * 32 + threadIdx.x);
  const int rchunk = (batch + gridDim.y - 1) / gridDim.y;
  const int r0 = blockIdx.y * rchunk, r1 = min(batch, r0 + rchunk);
  float s0 = 0.f, s1 = 0.f;
  if (c < cols)
    for (int b0 = r0 + threadIdx.y; b0 < r1; b0 += 32) {
      __nv_bfloat162 v[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int b = b0 + 8 * k;
        v[k] = b < r1 ? *reinterpret_cast<const __nv_bfloat162 *>(d + (int64_t)b * cols + c)
                      : __floats2bfloat162_rn(0.f, 0.f);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (b0 + 8 * k >= r1) break;
        const float2 f = __bfloat1622float2(v[k]);
        s0 += f.x;
        s1 += f.y;
      }
    }
  red[threadIdx.y][0][threadIdx.x] = s0;
  red[threadIdx.y][1][threadIdx.x] = s1;
  __syncthreads();
  if (threadIdx.y < 2) {
    const int cc = c + threadIdx.y;
    if (cc < cols) {
      float t = 0.f;
      for (int y = 0; y < 8; ++y) t += red[y][threadIdx.y][threadIdx.x];
      part[(int64_t)blockIdx.y * cols + cc] = t;
    }
  }
}
__global__ void mlp_colsum_final_kernel(const float *part, int nchunk, int cols, float *out) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int y = 0; y < nchunk; ++y) s += part[(int64_t)y * cols + c];
    out[c] = s;
  }
}

// Adam (Kingma & Ba 2015) on FP32 masters; refreshes the BF16 copy.
__global__ void mlp_adam_kernel(float *w, float *m, float *v, const float *g, __nv_bfloat16 *wb, int64_t n, float lr,
                                float b1, float b2, float eps, float c1, float c2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

// Partial dot product of one bf16 row (nchunk 16-byte chunks) with x (float,
// shared memory) over the chunks lane, lane + 32, ...: GEMV_U loads in flight.
constexpr int GEMV_U = 8;
__device__ __forceinline__ float gemv_row(const uint4 *row, const float *x, int nchunk, int lane) {
  float acc = 0.f;
  for (int c0 = lane; c0 < nchunk; c0 += 32 * GEMV_U) {
    uint4 q[GEMV_U];
#pragma unroll
    for (int u = 0; u < GEMV_U; ++u) {
      const int c = c0 + 32 * u;
      q[u] = c < nchunk ? __ldg(row + c) : make_uint4(0u, 0u, 0u, 0u);
    }
#pragma unroll
    for (int u = 0; u < GEMV_U; ++u) {
      const int c = c0 + 32 * u;
      if (c < nchunk) {
        const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q[u]);
        const float4 x0 = *reinterpret_cast<const float4 *>(x + 8 * c);
        const float4 x1 = *reinterpret_cast<const float4 *>(x + 8 * c + 4);
        const float2 f0 = __bfloat1622float2(h[0]), f1 = __bfloat1622float2(h[1]);
        const float2 f2 = __bfloat1622float2(h[2]), f3 = __bfloat1622float2(h[3]);
        acc = fmaf(f0.x, x0.x, acc);
        acc = fmaf(f0.y, x0.y, acc);
        acc = fmaf(f1.x, x0.z, acc);
        acc = fmaf(f1.y, x0.w, acc);
        acc = fmaf(f2.x, x1.x, acc);
        acc = fmaf(f2.y, x1.y, acc);
        acc = fmaf(f3.x, x1.z, acc);
        acc = fmaf(f3.y, x1.w, acc);
      }
    }
  }
  return acc;
}

// One layer for a single input vector: y[r] = act(W[r] . bf16(x * xscale) + b[r]) * yscale
// for r < rows_real (0 in the padding).  One warp per row, 16-byte weight loads.
// With Ws set, y[r] also gets + Ws[r] . bf16(xs_in * xs_scale) (the skip path).
__global__ void mlp_gemv_kernel(const __nv_bfloat16 *W, const float *bias, const float *x, int nin_real, int ld,
                                float xscale, int rows, int rows_real, int gelu, float yscale, float *y,
                                const __nv_bfloat16 *Ws, const float *xs_in, int nskip_real, int lds,
                                float xs_scale) {
  extern __shared__ float xs[];
  float *xk = xs + ld;  // skip input
  for (int k = threadIdx.x; k < ld; k += blockDim.x) xs[k] = k < nin_real ? bf16_round(x[k] * xscale) : 0.f;
  if (Ws)
    for (int k = threadIdx.x; k < lds; k += blockDim.x) xk[k] = k < nskip_real ? bf16_round(xs_in[k] * xs_scale) : 0.f;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int nchunk = ld / 8;
  for (int r = blockIdx.x * nw + warp; r < rows; r += gridDim.x * nw) {
    const float acc = warp_sum(gemv_row(reinterpret_cast<const uint4 *>(W + (int64_t)r * ld), xs, nchunk, lane));
    const float sk = Ws ? warp_sum(gemv_row(reinterpret_cast<const uint4 *>(Ws + (int64_t)r * lds), xk, lds / 8, lane))
                        : 0.f;
    if (lane == 0) {
      float v = acc + bias[r] + sk;
      if (gelu) v = gelu_f(v);
      y[r] = r < rows_real ? v * yscale : 0.f;
    }
  }
}

// Reconstruction choice: predicted commands c = y; when ||c|| <= threshold the
// step uses them (err = -c, integrator applied here, LS MVM skipped), otherwise
// the LS MVM runs and the fallback counter is bumped.  One CTA.
__global__ void mlp_select_kernel(const float *y, int n, float threshold, float gain, const float *mgain, float *err,
                                  float *com, uint32_t *use_ls, uint32_t *fallbacks) {
  __shared__ float red[1024];
  float s = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += y[i] * y[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  const bool fallback = !(sqrtf(red[0]) <= threshold);
  if (threadIdx.x == 0) {
    *use_ls = fallback ? 1u : 0u;
    if (fallback) *fallbacks += 1u;
  }
  if (!fallback)
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const float e = -y[i];
      err[i] = e;
      com[i] = gain * (e * mgain[i]) + com[i];
    }
}

// 2-D bf16 tensor map for the tcgen05 GEMM: inner (contiguous) extent, outer
// extent, row stride in elements; box 64 (inner, 128 bytes) x box_outer, 128-byte
// swizzle, zero fill outside the matrix.
// (the driver entry point is looked up through the runtime, so the library
// does not link the driver library itself and still loads on machines without it)
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    AOB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    AOB_REQUIRE(p != nullptr && q == cudaDriverEntryPointSuccess, "mlp gemm: cuTensorMapEncodeTiled not available");
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

static void encode_map(CUtensorMap *m, const void *base, uint64_t inner, uint64_t outer, uint64_t ld, uint32_t box_outer) {
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {ld * 2};
  cuuint32_t box[2] = {64u, box_outer};
  cuuint32_t es[2] = {1u, 1u};
  const CUresult r = encode_tiled_fn()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides,
                                       box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                       CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  AOB_REQUIRE(r == CUDA_SUCCESS, "mlp gemm: tensor map encoding failed (" + std::to_string((int)r) + ")");
}

// kind 0: mma.sync kernel, 1: tcgen05 kernel.  P2 (tcgen05 only, same M, N
// and layouts): a second product added in the same accumulator.
template <bool A_KM, bool B_KN>
static void gemm(const GemmArgs &P, cudaStream_t s, int kind, uint32_t *status, const GemmArgs *P2 = nullptr,
                 aob::DevBuf<float> *work = nullptr) {
  AOB_REQUIRE(P.M > 0 && P.N > 0 && P.K > 0, "mlp gemm: empty product");
  AOB_REQUIRE(P.lda % 8 == 0 && P.ldb % 8 == 0 && ((A_KM && B_KN) || P.K % 8 == 0),
              "mlp gemm: contiguous dimensions must be multiples of 8");
  if (kind == 1) {
    TcArgs T{P, A_KM ? 1 : 0, B_KN ? 1 : 0, status, P2 ? P2->K : 0, 0, nullptr};
    // split K when it shortens the product (plain float products only: no
    // bias, no activation, no accumulate, no bf16 copy).  Cost model, measured
    // on B200: a CTA alone on an SM takes ~0.5 us per 64-deep stage and two
    // co-resident CTAs share the SM, so a product takes ~ceil(CTAs / SMs) x
    // stages per slice x 0.5 us; the slice sum streams (n + 1) M N floats at
    // ~4 TB/s.  Slices keep at least 8 stages.
    const int tiles = ((P.N + TC_BN - 1) / TC_BN) * ((P.M + TC_BM - 1) / TC_BM);
    int dev = 0;
    AOB_CUDA(cudaGetDevice(&dev));
    const int nsm = num_sms(dev);
    int nsplit = 1;
    if (work && !P2 && P.epi == MG_EPI_NONE && !P.bias && !P.accumulate && !P.Cb && P.Cf && P.ldc % 4 == 0 &&
        reinterpret_cast<uintptr_t>(P.Cf) % 16 == 0) {
      const int nkt = (P.K + TC_BK - 1) / TC_BK;
      auto cost_us = [&](int n) {
        const int per = (nkt + n - 1) / n, ns = (nkt + per - 1) / per;
        const double waves = (double)((tiles * ns + nsm - 1) / nsm);
        const double sum = ns > 1 ? (double)(ns + 1) * P.M * P.N * 4.0 / 4.0e6 : 0.0;
        return waves * per * 0.5 + sum;
      };
      double best = cost_us(1);
      for (int n = 2; n <= 16 && nkt / n >= 8; ++n)
        if (cost_us(n) < best) {
          best = cost_us(n);
          nsplit = n;
        }
    }
    if (nsplit > 1) {
      const int per = (((P.K + TC_BK - 1) / TC_BK) + nsplit - 1) / nsplit;
      nsplit = (((P.K + TC_BK - 1) / TC_BK) + per - 1) / per;
      T.kchunk = per * TC_BK;
      const int64_t need = (int64_t)nsplit * P.M * P.ldc;
      if (work->n < need) work->alloc(need);
      T.partial = work->p;
    }
    auto maps = [](const GemmArgs &Q, CUtensorMap &ma, CUtensorMap &mb) {
      if (A_KM)
        encode_map(&ma, Q.A, (uint64_t)Q.M, (uint64_t)Q.K, (uint64_t)Q.lda, 64u);
      else
        encode_map(&ma, Q.A, (uint64_t)Q.K, (uint64_t)Q.M, (uint64_t)Q.lda, (uint32_t)TC_BM);
      if (B_KN)
        encode_map(&mb, Q.B, (uint64_t)Q.N, (uint64_t)Q.K, (uint64_t)Q.ldb, 64u);
      else
        encode_map(&mb, Q.B, (uint64_t)Q.K, (uint64_t)Q.N, (uint64_t)Q.ldb, (uint32_t)TC_BN);
    };
    CUtensorMap ma, mb, ma2, mb2;
    maps(P, ma, mb);
    if (P2) {
      AOB_REQUIRE(P2->M == P.M && P2->N == P.N && P2->K > 0 && P2->lda % 8 == 0 && P2->ldb % 8 == 0,
                  "mlp gemm: the second product must have the first's shape");
      maps(*P2, ma2, mb2);
    } else {
      ma2 = ma;
      mb2 = mb;
    }
    smem_opt_in(reinterpret_cast<const void *>(tc_gemm_kernel), (int)TC_SMEM_BYTES);
    dim3 grid((P.N + TC_BN - 1) / TC_BN, (P.M + TC_BM - 1) / TC_BM, nsplit);
    tc_gemm_kernel<<<grid, TC_THREADS, TC_SMEM_BYTES, s>>>(ma, mb, ma2, mb2, T);
    AOB_LAUNCH_CHECK("tc_gemm_kernel");
    if (nsplit > 1) {
      const int nq = (P.N + 3) / 4;
      dim3 sgrid((nq + 255) / 256, (unsigned)std::min(P.M, 65535));
      tc_splitk_sum_kernel<<<sgrid, 256, 0, s>>>(T.partial, nsplit, P.M, P.N, P.ldc, P.Cf);
      AOB_LAUNCH_CHECK("tc_splitk_sum_kernel");
    }
    return;
  }
  AOB_REQUIRE(P2 == nullptr, "mlp gemm: a second product needs the tcgen05 kernel");
  dim3 grid((P.N + MG_BN - 1) / MG_BN, (P.M + MG_BM - 1) / MG_BM);
  mlp_gemm_kernel<A_KM, B_KN><<<grid, MG_THREADS, 0, s>>>(P);
  AOB_LAUNCH_CHECK("mlp_gemm_kernel");
}

static int grid_for(int64_t n, int device) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 8 * num_sms(device)));
}

}  // namespace aob

using namespace aob;

static int pad8(int v) { return (v + 7) / 8 * 8; }

aob_mlp::aob_mlp(int device_, int nin_, int nh1_, int nh2_, int nout_)
    : device(device_), nin(nin_), nh1(nh1_), nh2(nh2_), nout(nout_) {
  AOB_REQUIRE(nin > 0 && nh1 > 0 && nh2 > 0 && nout > 0, "mlp: sizes must be > 0");
  pin = pad8(nin);
  ph1 = pad8(nh1);
  ph2 = pad8(nh2);
  pout = pad8(nout);
  AOB_CUDA(cudaSetDevice(device));
  for (int l = 0; l < 4; ++l) {
    const int64_t nw = (int64_t)rows(l) * cols(l);
    w[l].alloc(nw);
    mw[l].alloc(nw);
    vw[l].alloc(nw);
    gw[l].alloc(nw);
    wb[l].alloc(nw);
    if (l < 3) {
      b[l].alloc(rows(l));
      mb[l].alloc(rows(l));
      vb[l].alloc(rows(l));
      gb[l].alloc(rows(l));
    }
  }
  ix.alloc(pin);
  ih1.alloc(ph1);
  ih2.alloc(ph2);
  iy.alloc(pout);
  use_ls.alloc(1);
  fallbacks.alloc(1);
  tc_status.alloc(1);
}

static void real_dims(const aob_mlp &m, int l, int &rr, int &cr) {
  rr = l == 0 ? m.nh1 : (l == 1 ? m.nh2 : m.nout);
  cr = l == 0 ? m.nin : (l == 1 ? m.nh1 : (l == 2 ? m.nh2 : m.nin));
}

void aob_mlp::set_params(int l, const float *wh, const float *bh) {
  AOB_REQUIRE(l >= 0 && l < 4 && wh && (bh || l == 3), "mlp.set_params: bad layer or null arrays");
  AOB_CUDA(cudaSetDevice(device));
  int rr, cr;
  real_dims(*this, l, rr, cr);
  std::vector<float> W((size_t)rows(l) * cols(l), 0.f), B(rows(l), 0.f);
  for (int r = 0; r < rr; ++r) {
    for (int c = 0; c < cr; ++c) W[(size_t)r * cols(l) + c] = wh[(size_t)r * cr + c];
    if (bh) B[r] = bh[r];
  }
  w[l].upload(W.data(), (int64_t)W.size());
  AOB_CUDA(cudaMemset(mw[l].p, 0, mw[l].bytes()));
  AOB_CUDA(cudaMemset(vw[l].p, 0, vw[l].bytes()));
  if (l < 3) {
    b[l].upload(B.data(), (int64_t)B.size());
    AOB_CUDA(cudaMemset(mb[l].p, 0, mb[l].bytes()));
    AOB_CUDA(cudaMemset(vb[l].p, 0, vb[l].bytes()));
  }
  f32_to_bf16_kernel<<<grid_for(w[l].n, device), 256>>>(w[l].p, reinterpret_cast<__nv_bfloat16 *>(wb[l].p), w[l].n);
  AOB_LAUNCH_CHECK("f32_to_bf16_kernel");
  AOB_CUDA(cudaDeviceSynchronize());
  t = 0;
}

void aob_mlp::get_params(int l, float *wh, float *bh) {
  AOB_REQUIRE(l >= 0 && l < 4, "mlp.get_params: bad layer");
  AOB_CUDA(cudaSetDevice(device));
  AOB_CUDA(cudaDeviceSynchronize());
  int rr, cr;
  real_dims(*this, l, rr, cr);
  std::vector<float> W((size_t)rows(l) * cols(l)), B(rows(l), 0.f);
  AOB_CUDA(cudaMemcpy(W.data(), w[l].p, w[l].bytes(), cudaMemcpyDeviceToHost));
  if (l < 3) AOB_CUDA(cudaMemcpy(B.data(), b[l].p, b[l].bytes(), cudaMemcpyDeviceToHost));
  if (wh)
    for (int r = 0; r < rr; ++r)
      for (int c = 0; c < cr; ++c) wh[(size_t)r * cr + c] = W[(size_t)r * cols(l) + c];
  if (bh)
    for (int r = 0; r < rr; ++r) bh[r] = B[r];
}

void aob_mlp::ensure_batch(int batch) {
  AOB_REQUIRE(batch > 0, "mlp: batch must be > 0");
  if (batch <= cap) return;
  AOB_CUDA(cudaSetDevice(device));
  cap = batch;
  xb.alloc((int64_t)cap * pin);
  z1.alloc((int64_t)cap * ph1);
  h1b.alloc((int64_t)cap * ph1);
  z2.alloc((int64_t)cap * ph2);
  h2b.alloc((int64_t)cap * ph2);
  y.alloc((int64_t)cap * pout);
  dy.alloc((int64_t)cap * pout);
  dz2.alloc((int64_t)cap * ph2);
  dz1.alloc((int64_t)cap * ph1);
  loss_part.alloc(8 * num_sms(device));
}

static __nv_bfloat16 *bf(aob::DevBuf<uint16_t> &b) { return reinterpret_cast<__nv_bfloat16 *>(b.p); }

void aob_mlp::forward(const float *x, int batch, float *y_out, cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  ensure_batch(batch);
  mlp_input_kernel<<<std::min(batch, 8 * num_sms(device)), 256, 0, s>>>(x, nin, pin, batch, in_scale, bf(xb));
  AOB_LAUNCH_CHECK("mlp_input_kernel");
  GemmArgs P{};
  // h1 = GELU(x W1^T + b1)
  P = GemmArgs{batch, ph1, pin, bf(xb), pin, bf(wb[0]), pin, b[0].p, MG_EPI_GELU, nullptr, z1.p, ph1,
               nullptr, bf(h1b), ph1, 0};
  gemm<false, false>(P, s, gemm_kind, tc_status.p);
  // h2 = GELU(h1 W2^T + b2)
  P = GemmArgs{batch, ph2, ph1, bf(h1b), ph1, bf(wb[1]), ph1, b[1].p, MG_EPI_GELU, nullptr, z2.p, ph2,
               nullptr, bf(h2b), ph2, 0};
  gemm<false, false>(P, s, gemm_kind, tc_status.p);
  // y = h2 W3^T + b3, then y += x Ws^T (skip path)
  P = GemmArgs{batch, pout, ph2, bf(h2b), ph2, bf(wb[2]), ph2, b[2].p, MG_EPI_NONE, nullptr, nullptr, 0,
               y.p, nullptr, pout, 0};
  GemmArgs P2{batch, pout, pin, bf(xb), pin, bf(wb[3]), pin, nullptr, MG_EPI_NONE, nullptr, nullptr, 0,
              y.p, nullptr, pout, 1};
  if (gemm_kind == 1) {
    gemm<false, false>(P, s, gemm_kind, tc_status.p, &P2);  // one K loop over [h2 | x]
  } else {
    gemm<false, false>(P, s, gemm_kind, tc_status.p);
    gemm<false, false>(P2, s, gemm_kind, tc_status.p);
  }
  if (y_out) {
    mlp_output_kernel<<<std::min(batch, 8 * num_sms(device)), 256, 0, s>>>(y.p, nout, pout, batch, out_scale,
                                                                              y_out);
    AOB_LAUNCH_CHECK("mlp_output_kernel");
  }
}

// bias gradient: column sums of a [batch][cols] bf16 matrix
void aob_mlp::colsum(const __nv_bfloat16 *d, int batch, int cols, float *out, cudaStream_t s) {
  if (colsum_part.n < (int64_t)COLSUM_CHUNKS * cols) colsum_part.alloc((int64_t)COLSUM_CHUNKS * cols);
  AOB_REQUIRE(cols % 2 == 0, "mlp.colsum: padded column count must be even");
  mlp_colsum_part_kernel<<<dim3((cols / 2 + 31) / 32, COLSUM_CHUNKS), dim3(32, 8), 0, s>>>(d, batch, cols,
                                                                                        colsum_part.p);
  mlp_colsum_final_kernel<<<(cols + 255) / 256, 256, 0, s>>>(colsum_part.p, COLSUM_CHUNKS, cols, out);
  AOB_LAUNCH_CHECK("mlp_colsum_kernel");
}

// Gradients of the MSE after forward() on the same batch.
void aob_mlp::backward(const float *target, int batch, float *loss, cudaStream_t s) {
  AOB_REQUIRE(batch <= cap, "mlp.backward: run forward on this batch first");
  AOB_CUDA(cudaSetDevice(device));
  const int nb = (int)loss_part.n;
  mlp_loss_kernel<<<nb, 256, 0, s>>>(y.p, target, nout, pout, batch, 1.f / out_scale, bf(dy), loss_part.p);
  AOB_LAUNCH_CHECK("mlp_loss_kernel");
  if (loss) {
    mlp_loss_final_kernel<<<1, 32, 0, s>>>(loss_part.p, nb, (float)batch * (float)nout, loss);
    AOB_LAUNCH_CHECK("mlp_loss_final_kernel");
  }
  GemmArgs P{};
  // layer 3: dW3 = dy^T h2, db3 = sum dy, dz2 = (dy W3) * GELU'(z2)
  colsum(bf(dy), batch, pout, gb[2].p, s);
  P = GemmArgs{pout, ph2, batch, bf(dy), pout, bf(h2b), ph2, nullptr, MG_EPI_NONE, nullptr, nullptr, 0,
               gw[2].p, nullptr, ph2, 0};
  gemm<true, true>(P, s, gemm_kind, tc_status.p, nullptr, &splitk);
  P = GemmArgs{batch, ph2, pout, bf(dy), pout, bf(wb[2]), ph2, nullptr, MG_EPI_DGELU, z2.p, nullptr, ph2,
               nullptr, bf(dz2), ph2, 0};
  gemm<false, true>(P, s, gemm_kind, tc_status.p);
  // layer 2
  colsum(bf(dz2), batch, ph2, gb[1].p, s);
  P = GemmArgs{ph2, ph1, batch, bf(dz2), ph2, bf(h1b), ph1, nullptr, MG_EPI_NONE, nullptr, nullptr, 0,
               gw[1].p, nullptr, ph1, 0};
  gemm<true, true>(P, s, gemm_kind, tc_status.p, nullptr, &splitk);
  P = GemmArgs{batch, ph1, ph2, bf(dz2), ph2, bf(wb[1]), ph1, nullptr, MG_EPI_DGELU, z1.p, nullptr, ph1,
               nullptr, bf(dz1), ph1, 0};
  gemm<false, true>(P, s, gemm_kind, tc_status.p);
  // layer 1
  colsum(bf(dz1), batch, ph1, gb[0].p, s);
  P = GemmArgs{ph1, pin, batch, bf(dz1), ph1, bf(xb), pin, nullptr, MG_EPI_NONE, nullptr, nullptr, 0,
               gw[0].p, nullptr, pin, 0};
  gemm<true, true>(P, s, gemm_kind, tc_status.p, nullptr, &splitk);
  // skip path: dWs = dy^T x
  P = GemmArgs{pout, pin, batch, bf(dy), pout, bf(xb), pin, nullptr, MG_EPI_NONE, nullptr, nullptr, 0,
               gw[3].p, nullptr, pin, 0};
  gemm<true, true>(P, s, gemm_kind, tc_status.p, nullptr, &splitk);
  AOB_LAUNCH_CHECK("mlp_colsum_kernel");
}

void aob_mlp::adam(float lr, cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  ++t;
  const float c1 = 1.f - std::pow(beta1, (float)t), c2 = 1.f - std::pow(beta2, (float)t);
  for (int l = 0; l < 4; ++l) {
    mlp_adam_kernel<<<grid_for(w[l].n, device), 256, 0, s>>>(w[l].p, mw[l].p, vw[l].p, gw[l].p, bf(wb[l]), w[l].n,
                                                             lr, beta1, beta2, eps, c1, c2);
    if (l < 3)
      mlp_adam_kernel<<<grid_for(b[l].n, device), 256, 0, s>>>(b[l].p, mb[l].p, vb[l].p, gb[l].p, nullptr, b[l].n,
                                                               lr, beta1, beta2, eps, c1, c2);
  }
  AOB_LAUNCH_CHECK("mlp_adam_kernel");
}

void aob_mlp::infer(const float *x, float *y_out, cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  const int threads = 256, nw = threads / 32;
  auto layer = [&](int l, const float *in, int nin_real, float xscale, int nrows_real, int gelu, float yscale,
                   float *out, bool skip) {
    const int rws = rows(l), ld = cols(l);
    const int grid = std::max(1, std::min((rws + nw - 1) / nw, 4 * num_sms(device)));
    const size_t sm = sizeof(float) * (ld + (skip ? pin : 0));
    mlp_gemv_kernel<<<grid, threads, sm, s>>>(bf(wb[l]), b[l].p, in, nin_real, ld, xscale, rws, nrows_real, gelu,
                                              yscale, out, skip ? bf(wb[3]) : nullptr, x, nin, pin, in_scale);
    AOB_LAUNCH_CHECK("mlp_gemv_kernel");
  };
  layer(0, x, nin, in_scale, nh1, 1, 1.f, ih1.p, false);
  layer(1, ih1.p, ph1, 1.f, nh2, 1, 1.f, ih2.p, false);
  layer(2, ih2.p, ph2, 1.f, nout, 0, out_scale, y_out ? y_out : iy.p, true);
}


// ---------------------------------------------------------------------------
// the fused control step (mlp_fused_kernel) is in mlp_fused.cuh

using namespace aob;

// One control step through the fused kernel; false when the configuration
// does not fit it (shared memory, co-residency), in which case the caller runs
// the multi-kernel path.
// The arguments of the fused control step for controller ls on a grid of one CTA
// per SM, and its shared-memory bytes; false when it does not fit.
bool aob_mlp::fused_args(aob_ls *ls, float threshold, MlpFusedArgs &A, size_t &smem_bytes) {
  if (fused_mode == 1) return false;
  if (ls->mvm_kind == 2) return false;  // the fallback reproduces the bulk-copy MVM only
  ls->ensure_packed(ls->prec);
  const int G = num_sms(device);
  auto per = [G](int n) { return (n + G - 1) / G; };
  const int esize = ls->prec == AOB_PREC_F32 ? 4 : (ls->prec == AOB_PREC_BF16 ? 2 : 1);
  const int V = 16 / esize;
  const int ld_ls = (ls->nslope + V - 1) / V * V;
  A = MlpFusedArgs{};
  A.W1 = bf(wb[0]);
  A.W2 = bf(wb[1]);
  A.W3 = bf(wb[2]);
  A.Ws = bf(wb[3]);
  A.b1 = b[0].p;
  A.b2 = b[1].p;
  A.b3 = b[2].p;
  A.pin = pin;
  A.ph1 = ph1;
  A.ph2 = ph2;
  A.pout = pout;
  A.nin = nin;
  A.nh1 = nh1;
  A.nh2 = nh2;
  A.nout = nout;
  A.in_scale = in_scale;
  A.out_scale = out_scale;
  A.threshold = threshold;
  A.x = ls->centroids.p;
  A.h1 = ih1.p;
  A.h2 = ih2.p;
  A.y = iy.p;
  if (partial.n < G) partial.alloc(G);
  if (gbar.n < GRID_WORDS) gbar.alloc(GRID_WORDS);
  A.partial = partial.p;
  A.n1 = per(ph1);
  A.n2 = per(ph2);
  A.n3 = per(pout);
  A.nls = per(nout);
  A.gain = ls->gain;
  A.mgain = ls->gains.p;
  A.err = ls->err.p;
  A.com = ls->com();
  A.use_ls = use_ls.p;
  A.fallbacks = fallbacks.p;
  A.status = ls->status.p;
  A.gbar = gbar.p;
  A.lsmat = ls->prec == AOB_PREC_F32 ? (const void *)ls->cm_f32.p
                                     : (ls->prec == AOB_PREC_BF16 ? (const void *)ls->cm_bf16.p : (const void *)ls->cm_fp8.p);
  A.rscale = ls->prec == AOB_PREC_FP8 ? ls->row_scale.p : nullptr;
  A.ld_ls = ld_ls;
  AOB_REQUIRE((int64_t)std::max(pin, pout) * G < (int64_t)1 << 32, "mlp: sizes beyond the row-split range");
  const MlpFusedSmem L(pin, ph1, ph2, A.n1, A.n2, A.n3, A.nls, swizzled_slope_floats(ld_ls, V));
  if (L.bytes > 227 * 1024 || A.nls > MLP_FUSED_THREADS) return false;
  smem_bytes = L.bytes;
  return true;
}

bool aob_mlp::comp_com_fused(aob_ls *ls, float threshold, cudaStream_t s) {
  MlpFusedArgs A{};
  size_t smem = 0;
  if (!fused_args(ls, threshold, A, smem)) return false;
  const int G = num_sms(device);
  auto launch = [&](auto kern) {
    try {
      smem_opt_in(reinterpret_cast<const void *>(kern), (int)smem);  // only ever raised, per device
    } catch (const std::exception &) {
      cudaGetLastError();
      return false;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, MLP_FUSED_THREADS, smem) != cudaSuccess ||
        per_sm < 1) {
      cudaGetLastError();
      return false;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(G);
    cfg.blockDim = dim3(MLP_FUSED_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    AOB_CUDA(cudaLaunchKernelEx(&cfg, kern, A));
    AOB_LAUNCH_CHECK("mlp_fused_kernel");
    return true;
  };
  if (ls->prec == AOB_PREC_F32) return launch(mlp_fused_kernel<float>);
  if (ls->prec == AOB_PREC_BF16) return launch(mlp_fused_kernel<__nv_bfloat16>);
  return launch(mlp_fused_kernel<__nv_fp8_e4m3>);
}

// ---------------------------------------------------------------------------
extern "C" {

#define MLP_TRY try {
#define MLP_END                     \
  return AOB_OK;                    \
  }                                 \
  catch (const std::exception &e) { \
    aob::set_last_error(e.what());  \
    return AOB_ERR;                 \
  }
#define MLP_NEED(p) \
  if (!(p)) throw aob::Error(std::string(__func__) + ": null handle or pointer")
static inline cudaStream_t MS(void *p) { return reinterpret_cast<cudaStream_t>(p); }

int aob_mlp_create(aob_mlp **out, int device, int nin, int nh1, int nh2, int nout) {
  MLP_TRY MLP_NEED(out);
  *out = nullptr;
  AOB_CUDA(cudaSetDevice(device));
  *out = new aob_mlp(device, nin, nh1, nh2, nout);
  MLP_END
}
int aob_mlp_destroy(aob_mlp *m) {
  MLP_TRY if (m) {
    cudaSetDevice(m->device);
    delete m;
  }
  MLP_END
}
int aob_mlp_set_params(aob_mlp *m, int layer, const float *w, const float *b) {
  MLP_TRY MLP_NEED(m);
  m->set_params(layer, w, b);
  MLP_END
}
int aob_mlp_get_params(aob_mlp *m, int layer, float *w, float *b) {
  MLP_TRY MLP_NEED(m);
  m->get_params(layer, w, b);
  MLP_END
}
int aob_mlp_set_scales(aob_mlp *m, float in_scale, float out_scale) {
  MLP_TRY MLP_NEED(m);
  if (!(out_scale != 0.f)) throw aob::Error("mlp.set_scales: out_scale must be non-zero");
  m->in_scale = in_scale;
  m->out_scale = out_scale;
  MLP_END
}
int aob_mlp_forward(aob_mlp *m, const float *dev_x, int batch, float *dev_y, void *stream) {
  MLP_TRY MLP_NEED(m);
  MLP_NEED(dev_x);
  m->forward(dev_x, batch, dev_y, MS(stream));
  MLP_END
}
int aob_mlp_backward(aob_mlp *m, const float *dev_target, int batch, float *dev_loss, void *stream) {
  MLP_TRY MLP_NEED(m);
  MLP_NEED(dev_target);
  m->backward(dev_target, batch, dev_loss, MS(stream));
  MLP_END
}
int aob_mlp_train_step(aob_mlp *m, const float *dev_x, const float *dev_target, int batch, float lr,
                       float *dev_loss, void *stream) {
  MLP_TRY MLP_NEED(m);
  MLP_NEED(dev_x);
  MLP_NEED(dev_target);
  m->forward(dev_x, batch, nullptr, MS(stream));
  m->backward(dev_target, batch, dev_loss, MS(stream));
  m->adam(lr, MS(stream));
  MLP_END
}
int aob_mlp_infer(aob_mlp *m, const float *dev_x, float *dev_y, void *stream) {
  MLP_TRY MLP_NEED(m);
  MLP_NEED(dev_x);
  m->infer(dev_x, dev_y, MS(stream));
  MLP_END
}
int aob_mlp_comp_com(aob_mlp *m, aob_ls *ls, float threshold, void *stream) {
  MLP_TRY MLP_NEED(m);
  MLP_NEED(ls);
  if (ls->nslope != m->nin || ls->nactu != m->nout) throw aob::Error("mlp.comp_com: sizes differ from the controller's");
  if (ls->kind != AOB_CTRL_LS) throw aob::Error("mlp.comp_com: the LS fallback needs an LS controller");
  if (ls->open_loop) return AOB_OK;
  AOB_CUDA(cudaSetDevice(m->device));
  cudaStream_t s = MS(stream);
  if (m->comp_com_fused(ls, threshold, s)) return AOB_OK;
  m->infer(ls->centroids.p, m->iy.p, s);
  mlp_select_kernel<<<1, 1024, 0, s>>>(m->iy.p, m->nout, threshold, ls->gain, ls->gains.p, ls->err.p, ls->com(),
                                       m->use_ls.p, m->fallbacks.p);
  AOB_LAUNCH_CHECK("mlp_select_kernel");
  ls->comp_com(s, nullptr, m->use_ls.p);
  MLP_END
}
int aob_mlp_set_gemm(aob_mlp *m, int kind) {
  MLP_TRY MLP_NEED(m);
  if (kind < 0 || kind > 1) throw aob::Error("mlp.set_gemm: kind must be 0 or 1");
  m->gemm_kind = kind;
  MLP_END
}
int aob_mlp_gemm_status(aob_mlp *m, uint32_t *status, int reset) {
  MLP_TRY MLP_NEED(m);
  MLP_NEED(status);
  AOB_CUDA(cudaSetDevice(m->device));
  AOB_CUDA(cudaMemcpy(status, m->tc_status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (reset) AOB_CUDA(cudaMemset(m->tc_status.p, 0, sizeof(uint32_t)));
  MLP_END
}
int aob_mlp_set_mode(aob_mlp *m, int mode) {
  MLP_TRY MLP_NEED(m);
  if (mode < 0 || mode > 1) throw aob::Error("mlp.set_mode: mode must be 0 or 1");
  m->fused_mode = mode;
  MLP_END
}
int aob_mlp_fallbacks(aob_mlp *m, uint32_t *count, int reset) {
  MLP_TRY MLP_NEED(m);
  MLP_NEED(count);
  AOB_CUDA(cudaSetDevice(m->device));
  AOB_CUDA(cudaMemcpy(count, m->fallbacks.p, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (reset) AOB_CUDA(cudaMemset(m->fallbacks.p, 0, sizeof(uint32_t)));
  MLP_END
}
int aob_mlp_buffer(aob_mlp *m, const char *which, void **dev_ptr, int64_t *nelem) {
  MLP_TRY MLP_NEED(m);
  MLP_NEED(which);
  MLP_NEED(dev_ptr);
  const std::string w(which);
  void *p = nullptr;
  int64_t n = 0;
  auto pick = [&](const char *name, aob::DevBuf<float> *arr) {
    for (int l = 0; l < 3; ++l)
      if (w == std::string(name) + std::to_string(l + 1)) {
        p = arr[l].p;
        n = arr[l].n;
      }
  };
  pick("W", m->w);
  if (w == "Ws") {
    p = m->w[3].p;
    n = m->w[3].n;
  } else if (w == "dWs") {
    p = m->gw[3].p;
    n = m->gw[3].n;
  }
  pick("b", m->b);
  pick("dW", m->gw);
  pick("db", m->gb);
  if (w == "y") {
    p = m->y.p;
    n = m->y.n;
  }
  if (!p) throw aob::Error("mlp.buffer: unknown buffer '" + w + "'");
  *dev_ptr = p;
  if (nelem) *nelem = n;
  MLP_END
}
int aob_mlp_get_dims(aob_mlp *m, int *padded4) {
  MLP_TRY MLP_NEED(m);
  MLP_NEED(padded4);
  padded4[0] = m->pin;
  padded4[1] = m->ph1;
  padded4[2] = m->ph2;
  padded4[3] = m->pout;
  MLP_END
}

}  // extern "C"
