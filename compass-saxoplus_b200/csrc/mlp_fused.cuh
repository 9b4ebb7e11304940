// The learned reconstructor's whole control step as device code shared by the
// standalone cooperative kernel (mlp.cu) and the fused RTC iteration with the
// learned reconstructor (rtc_mlp.cu).
#pragma once

#include <cuda_bf16.h>

#include "aob_common.cuh"
#include "mlp_gemm.cuh"
#include "mvm_core.cuh"

namespace aob {

__device__ __forceinline__ float bf16_round(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// The whole control step of the learned reconstructor in one cooperative
// kernel: every CTA owns a contiguous block of rows of each layer (and of the
// skip path and of the LS matrix) and, at entry, one thread issues the bulk
// copies of its rows of all four weight matrices into shared memory (one
// mbarrier), so the full weight stream is in flight from the first cycle.
//   phase 1: x = bf16(slopes * in_scale) staged; layer-1 rows and skip rows
//   -- grid barrier -- phase 2: h1 staged, layer-2 rows
//   -- grid barrier -- phase 3: h2 staged, layer-3 rows + skip, |y|^2 per CTA
//   -- grid barrier -- phase 4: the threshold test on the summed |y|^2; either
//      the integrator on the network's commands, or the LS fallback: the CTA's
//      rows of the packed command matrix reduced exactly as the bulk-copy LS
//      MVM does (16 warp slots, transposed eight-row reduction), read from
//      global memory.
// Every row product accumulates over the chunks in the order of
// mlp_gemv_kernel, so the commands equal the multi-kernel path's bit for bit.
constexpr int MLP_FUSED_THREADS = 512;
constexpr uint32_t MLP_ROW_MAX_POLLS = 1u << 22;

struct MlpFusedArgs {
  const __nv_bfloat16 *W1, *W2, *W3, *Ws;
  const float *b1, *b2, *b3;
  int pin, ph1, ph2, pout;  // padded sizes (row strides)
  int nin, nh1, nh2, nout;  // real sizes
  float in_scale, out_scale, threshold;
  const float *x;           // slopes
  float *h1, *h2, *y;       // hidden and output vectors (global, read back through L2)
  float *partial;           // per-CTA sums of y^2
  int n1, n2, n3, nls;      // rows per CTA, at most: layer 1, layer 2, layer 3 / skip, LS
  // controller
  float gain;
  const float *mgain;
  float *err, *com;
  uint32_t *use_ls, *fallbacks, *status;
  unsigned long long *gbar;
  // LS fallback
  const void *lsmat;
  const float *rscale;
  int ld_ls;
};

__device__ __forceinline__ void row_block(int nrow, int &r0, int &R) {
  r0 = (int)((blockIdx.x * (uint32_t)nrow) / gridDim.x);
  R = (int)(((blockIdx.x + 1) * (uint32_t)nrow) / gridDim.x) - r0;
}

// dot of a bf16 row in shared memory with a float vector in shared memory,
// chunk order lane, lane + 32, ... (as gemv_row)
__device__ __forceinline__ float smem_row_dot(const uint4 *row, const float *v, int nchunk, int lane) {
  float acc = 0.f;
  for (int c = lane; c < nchunk; c += 32) {
    const uint4 q = row[c];
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
    const float4 x0 = *reinterpret_cast<const float4 *>(v + 8 * c);
    const float4 x1 = *reinterpret_cast<const float4 *>(v + 8 * c + 4);
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
  return acc;
}

struct MlpFusedSmem {
  size_t xs, hs, sk, sl, part, w1, ws, w2, w3, bytes;
  __host__ __device__ static size_t a16(size_t v) { return (v + 15) & ~size_t(15); }
  __host__ __device__ MlpFusedSmem(int pin, int ph1, int ph2, int n1, int n2, int n3, int nls, int sl_floats) {
    size_t o = 128;  // the mbarrier
    xs = o;
    o = a16(o + sizeof(float) * pin);
    hs = o;
    o = a16(o + sizeof(float) * (ph1 > ph2 ? ph1 : ph2));
    sk = o;
    o = a16(o + sizeof(float) * n3);
    sl = o;
    o = a16(o + sizeof(float) * sl_floats);
    part = o;
    o = a16(o + sizeof(float) * 16 * (nls > 0 ? nls : 1));
    w1 = o;
    o += (size_t)n1 * pin * 2;
    ws = o;
    o += (size_t)n3 * pin * 2;
    w2 = o;
    o += (size_t)n2 * ph1 * 2;
    w3 = o;
    o += (size_t)n3 * ph2 * 2;
    bytes = o;
  }
};

// The layout of a CTA's shared memory for the control step (weights of its rows)
template <typename TL>
__device__ __forceinline__ MlpFusedSmem mlp_fused_layout(const MlpFusedArgs &A) {
  return MlpFusedSmem(A.pin, A.ph1, A.ph2, A.n1, A.n2, A.n3, A.nls, swizzled_slope_floats(A.ld_ls, RowPack<TL>::N));
}

// One thread of the CTA: the mbarrier at sm[0] and the bulk copies of the CTA's
// rows of the four weight matrices, all completing on it.
__device__ __forceinline__ void mlp_fused_issue(const MlpFusedArgs &A, unsigned char *sm, const MlpFusedSmem &L) {
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm);
  int r1, R1, r2, R2, r3, R3;
  row_block(A.ph1, r1, R1);
  row_block(A.ph2, r2, R2);
  row_block(A.pout, r3, R3);
  mbar_init(bar, 1);
  fence_mbar_init();
  const uint32_t b1 = (uint32_t)(R1 * A.pin * 2), bs = (uint32_t)(R3 * A.pin * 2);
  const uint32_t b2 = (uint32_t)(R2 * A.ph1 * 2), b3 = (uint32_t)(R3 * A.ph2 * 2);
  mbar_expect_tx(bar, b1 + bs + b2 + b3);
  if (b1) bulk_g2s(sm + L.w1, A.W1 + (size_t)r1 * A.pin, b1, bar);
  if (bs) bulk_g2s(sm + L.ws, A.Ws + (size_t)r3 * A.pin, bs, bar);
  if (b2) bulk_g2s(sm + L.w2, A.W2 + (size_t)r2 * A.ph1, b2, bar);
  if (b3) bulk_g2s(sm + L.w3, A.W3 + (size_t)r3 * A.ph2, b3, bar);
}

// What the control step does with each command it writes (row, value): nothing
// here; the fused RTC iteration computes the row's voltage.
struct MlpNoEpilogue {
  __device__ void operator()(int, float) const {}
};

// The control step after the weight copies were issued: every thread of the CTA.
template <typename TL, class Epi>
__device__ __forceinline__ void mlp_fused_body(const MlpFusedArgs &A, unsigned char *sm, const MlpFusedSmem &L,
                                               const Epi &epi) {
  constexpr int V = RowPack<TL>::N;
  constexpr int Q = V / 4;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = MLP_FUSED_THREADS / 32;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm);
  float *xs = reinterpret_cast<float *>(sm + L.xs);
  float *hs = reinterpret_cast<float *>(sm + L.hs);
  float *sk = reinterpret_cast<float *>(sm + L.sk);
  int r1, R1, r2, R2, r3, R3;
  row_block(A.ph1, r1, R1);
  row_block(A.ph2, r2, R2);
  row_block(A.pout, r3, R3);
  for (int k = tid; k < A.pin; k += blockDim.x) xs[k] = k < A.nin ? bf16_round(__ldcg(A.x + k) * A.in_scale) : 0.f;
  __syncthreads();
  bool ok = mbar_wait(bar, 0, MLP_ROW_MAX_POLLS);
  ok = __syncthreads_and(ok) != 0;
  if (!ok && tid == 0) atomicOr(A.status, (uint32_t)ERR_MBAR_TIMEOUT);
  // ---- phase 1: layer-1 rows and skip rows ----
  if (ok)
    for (int t = warp; t < R1 + R3; t += nw) {
      if (t < R1) {
        const float acc =
            warp_sum(smem_row_dot(reinterpret_cast<const uint4 *>(sm + L.w1) + (size_t)t * (A.pin / 8), xs, A.pin / 8, lane));
        if (lane == 0) {
          const int r = r1 + t;
          float v = acc + __ldg(A.b1 + r) + 0.f;
          v = gelu_f(v);
          A.h1[r] = r < A.nh1 ? v : 0.f;
        }
      } else {
        const int u = t - R1;
        const float acc =
            warp_sum(smem_row_dot(reinterpret_cast<const uint4 *>(sm + L.ws) + (size_t)u * (A.pin / 8), xs, A.pin / 8, lane));
        if (lane == 0) sk[u] = acc;
      }
    }
  // ---- phase 2 ----
  grid_barrier(A.gbar, gridDim.x, A.status);
  for (int k = tid; k < A.ph1; k += blockDim.x) hs[k] = bf16_round(__ldcg(A.h1 + k));
  __syncthreads();
  if (ok)
    for (int t = warp; t < R2; t += nw) {
      const float acc =
          warp_sum(smem_row_dot(reinterpret_cast<const uint4 *>(sm + L.w2) + (size_t)t * (A.ph1 / 8), hs, A.ph1 / 8, lane));
      if (lane == 0) {
        const int r = r2 + t;
        float v = acc + __ldg(A.b2 + r) + 0.f;
        v = gelu_f(v);
        A.h2[r] = r < A.nh2 ? v : 0.f;
      }
    }
  // ---- phase 3 ----
  grid_barrier(A.gbar, gridDim.x, A.status);
  for (int k = tid; k < A.ph2; k += blockDim.x) hs[k] = bf16_round(__ldcg(A.h2 + k));
  __syncthreads();
  float *yl = reinterpret_cast<float *>(sm + L.part);  // this CTA's outputs, in row order
  if (ok)
    for (int t = warp; t < R3; t += nw) {
      const float acc =
          warp_sum(smem_row_dot(reinterpret_cast<const uint4 *>(sm + L.w3) + (size_t)t * (A.ph2 / 8), hs, A.ph2 / 8, lane));
      if (lane == 0) {
        const int r = r3 + t;
        const float v = acc + __ldg(A.b3 + r) + sk[t];
        const float out = r < A.nout ? v * A.out_scale : 0.f;
        A.y[r] = out;
        yl[t] = out;
      }
    }
  __syncthreads();
  if (tid == 0) {
    float s2 = 0.f;
    for (int t = 0; t < R3; ++t) s2 = fmaf(yl[t], yl[t], s2);
    A.partial[blockIdx.x] = s2;
  }
  // ---- phase 4: threshold test, then the integrator or the LS fallback ----
  grid_barrier(A.gbar, gridDim.x, A.status);
  __shared__ int s_fb;
  if (warp == 0) {
    // lane-strided partial sums then a butterfly: the same order in every CTA
    float tot = 0.f;
    for (int c = lane; c < (int)gridDim.x; c += 32) tot += __ldcg(A.partial + c);
    tot = warp_sum(tot);
    if (lane == 0) {
      const int fb = !(sqrtf(tot) <= A.threshold);
      s_fb = fb;
      if (blockIdx.x == 0) {
        *A.use_ls = fb ? 1u : 0u;
        if (fb) atomicAdd(A.fallbacks, 1u);
      }
    }
  }
  __syncthreads();
  if (!s_fb) {
    for (int t = tid; t < R3; t += blockDim.x) {
      const int r = r3 + t;
      if (r < A.nout) {
        const float e = -yl[t];
        A.err[r] = e;
        const float c = A.gain * (e * __ldg(A.mgain + r)) + __ldcg(A.com + r);
        A.com[r] = c;
        epi(r, c);
      }
    }
    return;
  }
  // LS fallback: rows [r0, r0 + R) of the packed matrix, bulk-copy MVM arithmetic
  int r0, R;
  row_block(A.nout, r0, R);
  float *s_sl = reinterpret_cast<float *>(sm + L.sl);
  float *part = reinterpret_cast<float *>(sm + L.part);
  const int nsh = swizzled_slope_floats(A.ld_ls, V);
  for (int g = tid; g < nsh / 4; g += blockDim.x) {
    const int l = g & 31, jq = g >> 5;
    const int j = jq / Q, q = jq - j * Q;
    const int src = (l + 32 * j) * V + 4 * q;
    float4 v4;
    v4.x = src < A.nin ? __ldcg(A.x + src) : 0.f;
    v4.y = src + 1 < A.nin ? __ldcg(A.x + src + 1) : 0.f;
    v4.z = src + 2 < A.nin ? __ldcg(A.x + src + 2) : 0.f;
    v4.w = src + 3 < A.nin ? __ldcg(A.x + src + 3) : 0.f;
    reinterpret_cast<float4 *>(s_sl)[g] = v4;
  }
  __syncthreads();
  const int nchunk = A.ld_ls / V;
  const size_t row_bytes = (size_t)A.ld_ls * sizeof(TL);
  const float4 *sv4 = reinterpret_cast<const float4 *>(s_sl);
  constexpr int RB = 8;
  for (int rb = 0; rb < R; rb += RB) {
    float acc[RB];
#pragma unroll
    for (int u = 0; u < RB; ++u) acc[u] = 0.f;
    for (int jj = warp; 32 * jj + lane < nchunk; jj += nw) {
      const int c = lane + 32 * jj;
      float4 sv[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) sv[q] = sv4[(jj * Q + q) * 32 + lane];
#pragma unroll
      for (int u = 0; u < RB; ++u)
        if (rb + u < R) {
          const uint4 q4 = __ldcs(reinterpret_cast<const uint4 *>(static_cast<const unsigned char *>(A.lsmat) +
                                                                  (size_t)(r0 + rb + u) * row_bytes) + c);
          acc[u] += RowPack<TL>::dot(q4, sv);
        }
    }
    int u;
    const float t = warp_sum8(acc, lane, u);
    if ((lane & 3) == 0 && rb + u < R) part[warp * A.nls + rb + u] = t;
  }
  __syncthreads();
  if (tid < R) {
    float tot = 0.f;
#pragma unroll
    for (int w = 0; w < nw; ++w) tot += part[w * A.nls + tid];
    const int gr = r0 + tid;
    if (A.rscale) tot *= __ldg(A.rscale + gr);
    const float e = -tot;
    A.err[gr] = e;
    const float c = A.gain * (e * __ldg(A.mgain + gr)) + __ldcg(A.com + gr);
    A.com[gr] = c;
    epi(gr, c);
  }
}

template <typename TL>
__global__ void __launch_bounds__(MLP_FUSED_THREADS, 1) mlp_fused_kernel(MlpFusedArgs A) {
  extern __shared__ __align__(128) unsigned char sm[];
  const MlpFusedSmem L = mlp_fused_layout<TL>(A);
  if (threadIdx.x == 0) mlp_fused_issue(A, sm, L);
  mlp_fused_body<TL>(A, sm, L, MlpNoEpilogue{});
}

}  // namespace aob
