// BF16 tensor-core GEMM with FP32 accumulation for the learned reconstructor.
//
// C[M x N] = op(A) op(B)^T over K, where A is stored either M x K (row-major,
// K contiguous: "MK") or K x M (M contiguous: "KM"), and B either N x K ("NK")
// or K x N ("KN").  The three products of an MLP training step need no
// transposed copies:
//   forward       Z  = X  W^T   A = X [batch][in]   (MK),  B = W [out][in]   (NK)
//   data grad     dH = dZ W     A = dZ [batch][out] (MK),  B = W [out][in]   (KN)
//   weight grad   dW = dZ^T H   A = dZ [batch][out] (KM),  B = H [batch][in] (KN)
//
// CTA tile 128 x 128 x 32, 8 warps of 64 x 32, mma.sync m16n8k16 (bf16 in,
// f32 accumulate); operands staged by cp.async (16-byte chunks, zero-filled
// out of range) into double-buffered shared memory and read with ldmatrix
// (.trans for the M- / N-contiguous layouts).  Every stored dimension that is
// contiguous in memory must be a multiple of 8 elements (16 bytes).
//
// Epilogue per output element (m, n): v = acc (+ C[m, n] when accumulating)
// (+ bias[n]); then optionally
// GELU (and the pre-activation kept), or a multiply by GELU'(pre[m, n]) for
// the backward pass; stored as float and / or bf16.
#pragma once

#include <cuda_bf16.h>

#include "aob_common.cuh"

namespace aob {

constexpr int MG_BM = 128, MG_BN = 128, MG_BK = 32;
constexpr int MG_THREADS = 256;
// shared-memory pitches in bf16 elements (padded so ldmatrix is conflict-free)
constexpr int MG_PK = MG_BK + 8;    // tile stored [rows][k]
constexpr int MG_PMN = MG_BM + 8;   // tile stored [k][rows]
constexpr int MG_TILE = (MG_BM * MG_PK > MG_BK * MG_PMN ? MG_BM * MG_PK : MG_BK * MG_PMN);

enum : int { MG_EPI_NONE = 0, MG_EPI_GELU = 1, MG_EPI_DGELU = 2 };

struct GemmArgs {
  int M, N, K;
  const __nv_bfloat16 *A;
  int lda;  // elements between rows of the stored matrix
  const __nv_bfloat16 *B;
  int ldb;
  const float *bias;         // [N] or null
  int epi;                   // MG_EPI_*
  const float *pre_in;       // [M][ldp] pre-activation for MG_EPI_DGELU
  float *pre_out;            // [M][ldp] pre-activation kept by MG_EPI_GELU (may be null)
  int ldp;
  float *Cf;                 // [M][ldc] float output (may be null)
  __nv_bfloat16 *Cb;         // [M][ldc] bf16 output (may be null)
  int ldc;
  int accumulate;            // add the product to the float output already in Cf
};

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad_f(float x) {
  const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * __expf(-0.5f * x * x);
  return cdf + x * pdf;
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  const int n = valid ? 16 : 0;  // zero-fill when out of range
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void ldsm_x4(uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3, const void *p) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(a));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3, const void *p) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(a));
}
__device__ __forceinline__ void mma_bf16(float *d, const uint32_t *a, const uint32_t *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Stage one K-slice (MG_BK) of the A and B tiles.  A_KM / B_KN select the
// stored layouts described above.
template <bool A_KM, bool B_KN>
__device__ __forceinline__ void mg_load_tiles(const GemmArgs &P, int m0, int n0, int k0, __nv_bfloat16 *sa,
                                              __nv_bfloat16 *sb) {
  const int tid = threadIdx.x;
  // 128 x 32 bf16 = 512 chunks of 8 elements per operand: 2 per thread
#pragma unroll
  for (int it = 0; it < 2; ++it) {
    const int c = tid + it * MG_THREADS;
    if (!A_KM) {  // [m][k]: 4 chunks per row
      const int r = c >> 2, kc = (c & 3) * 8;
      const int gm = m0 + r, gk = k0 + kc;
      const bool v = gm < P.M && gk < P.K;
      cp_async16(sa + r * MG_PK + kc, P.A + (size_t)(v ? gm : 0) * P.lda + (v ? gk : 0), v);
    } else {  // [k][m]: 16 chunks per k row
      const int r = c >> 4, mc = (c & 15) * 8;
      const int gk = k0 + r, gm = m0 + mc;
      const bool v = gk < P.K && gm < P.M;
      cp_async16(sa + r * MG_PMN + mc, P.A + (size_t)(v ? gk : 0) * P.lda + (v ? gm : 0), v);
    }
    if (!B_KN) {
      const int r = c >> 2, kc = (c & 3) * 8;
      const int gn = n0 + r, gk = k0 + kc;
      const bool v = gn < P.N && gk < P.K;
      cp_async16(sb + r * MG_PK + kc, P.B + (size_t)(v ? gn : 0) * P.ldb + (v ? gk : 0), v);
    } else {
      const int r = c >> 4, nc = (c & 15) * 8;
      const int gk = k0 + r, gn = n0 + nc;
      const bool v = gk < P.K && gn < P.N;
      cp_async16(sb + r * MG_PMN + nc, P.B + (size_t)(v ? gk : 0) * P.ldb + (v ? gn : 0), v);
    }
  }
}

template <bool A_KM, bool B_KN>
__global__ void __launch_bounds__(MG_THREADS) mlp_gemm_kernel(GemmArgs P) {
  __shared__ __align__(128) __nv_bfloat16 sA[2][MG_TILE];
  __shared__ __align__(128) __nv_bfloat16 sB[2][MG_TILE];
  const int m0 = blockIdx.y * MG_BM, n0 = blockIdx.x * MG_BN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;  // warp tile origin within the CTA tile
  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

  const int nk = (P.K + MG_BK - 1) / MG_BK;
  mg_load_tiles<A_KM, B_KN>(P, m0, n0, 0, sA[0], sB[0]);
  cp_async_commit();
  for (int kt = 0; kt < nk; ++kt) {
    const int cur = kt & 1;
    if (kt + 1 < nk) mg_load_tiles<A_KM, B_KN>(P, m0, n0, (kt + 1) * MG_BK, sA[cur ^ 1], sB[cur ^ 1]);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const __nv_bfloat16 *a = sA[cur];
    const __nv_bfloat16 *b = sB[cur];
#pragma unroll
    for (int kk = 0; kk < MG_BK; kk += 16) {
      uint32_t af[4][4], bf[4][2];
      const int mi = lane & 7, mj = lane >> 3;  // row within an 8x8 matrix, matrix index
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int mb = wm + i * 16;
        if (!A_KM) {
          // matrices: (rows 0-7, k 0-7), (rows 8-15, k 0-7), (rows 0-7, k 8-15), (rows 8-15, k 8-15)
          const __nv_bfloat16 *p = a + (mb + (mj & 1) * 8 + mi) * MG_PK + kk + (mj >> 1) * 8;
          ldsm_x4(af[i][0], af[i][1], af[i][2], af[i][3], p);
        } else {
          const __nv_bfloat16 *p = a + (kk + (mj >> 1) * 8 + mi) * MG_PMN + mb + (mj & 1) * 8;
          ldsm_x4_t(af[i][0], af[i][1], af[i][2], af[i][3], p);
        }
      }
#pragma unroll
      for (int j = 0; j < 4; j += 2) {
        const int nb = wn + j * 8;
        // matrices: (n 0-7, k 0-7), (n 0-7, k 8-15), (n 8-15, k 0-7), (n 8-15, k 8-15)
        if (!B_KN) {
          const __nv_bfloat16 *p = b + (nb + (mj >> 1) * 8 + mi) * MG_PK + kk + (mj & 1) * 8;
          ldsm_x4(bf[j][0], bf[j][1], bf[j + 1][0], bf[j + 1][1], p);
        } else {
          const __nv_bfloat16 *p = b + (kk + (mj & 1) * 8 + mi) * MG_PMN + nb + (mj >> 1) * 8;
          ldsm_x4_t(bf[j][0], bf[j][1], bf[j + 1][0], bf[j + 1][1], p);
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bf[j]);
    }
    __syncthreads();
  }
  cp_async_wait<0>();

  // epilogue: c0,c1 at (row g, cols 2t, 2t+1), c2,c3 at (row g+8, ...)
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = m0 + wm + i * 16 + g + h * 8;
        if (m >= P.M) continue;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int n = n0 + wn + j * 8 + 2 * t + e;
          if (n >= P.N) continue;
          float v = acc[i][j][2 * h + e];
          if (P.accumulate) v += P.Cf[(size_t)m * P.ldc + n];
          if (P.bias) v += P.bias[n];
          if (P.epi == MG_EPI_GELU) {
            if (P.pre_out) P.pre_out[(size_t)m * P.ldp + n] = v;
            v = gelu_f(v);
          } else if (P.epi == MG_EPI_DGELU) {
            v *= gelu_grad_f(P.pre_in[(size_t)m * P.ldp + n]);
          }
          if (P.Cf) P.Cf[(size_t)m * P.ldc + n] = v;
          if (P.Cb) P.Cb[(size_t)m * P.ldc + n] = __float2bfloat16_rn(v);
        }
      }
}

}  // namespace aob
