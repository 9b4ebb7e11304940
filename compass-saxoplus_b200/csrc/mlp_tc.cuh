// BF16 GEMM on the fifth-generation tensor cores (tcgen05) for the learned
// reconstructor's training step.  Same contract as mlp_gemm_kernel (GemmArgs:
// A stored M x K ("MK") or K x M ("KM"), B stored N x K ("NK") or K x N
// ("KN"), the same epilogue), so the three products of a training step run
// without transposed copies: K-major operands use the K-major shared-memory
// descriptor, M- or N-contiguous ones the MN-major descriptor.
//
// One CTA per 128 x 128 output tile, 16 warps, two CTAs per SM (97 KB of
// shared memory and 128 TMEM columns each):
//  * warp 0, one lane: TMA producer -- 2-D tensor loads with 128-byte swizzle
//    (K-major tile: one box of 64 (K) x 128 rows; MN-major: two boxes of
//    64 (M or N) x 64 (K)) into a 3-stage ring, each stage completing on its
//    "full" mbarrier;
//  * warp 1: allocates 128 TMEM columns (the 128 x 128 FP32 accumulator); one
//    lane issues tcgen05.mma.cta_group::1.kind::f16 (M 128, N 128, K 16, four
//    per 64-wide stage) and tcgen05.commit on the stage's "empty" mbarrier,
//    which hands the stage back to the producer once those MMAs completed;
//    after the last stage, a commit on the accumulator barrier;
//  * all 16 warps: the epilogue -- warps w, w + 4, w + 8, w + 12 read TMEM
//    lanes 32 (w & 3) .. + 31 (rows of the tile; a warp may only read its own
//    lane quadrant), one 32-column chunk each, with tcgen05.ld 32x32b, transpose
//    each 32 x 32 chunk through shared memory and apply bias / GELU / GELU'
//    with coalesced row accesses.
// Split K (blockIdx.z slices, each writing its plain FP32 product to a
// workspace that tc_splitk_sum_kernel adds in slice order: deterministic) keeps
// the SMs busy for the weight-gradient products, whose outputs have few tiles
// and whose K is the batch.
// A second operand pair (A2, B2, same layouts, its own K) can follow the first
// in the same K loop, so y = h2 W3^T + x Ws^T is one GEMM with no read-back of
// the output.
// Every mbarrier wait is bounded: on expiry a status bit is set, the kernel
// still waits (bounded) for its MMAs, frees its TMEM and returns.  No cluster,
// no multicast.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "aob_common.cuh"
#include "mlp_gemm.cuh"

namespace aob {

constexpr int TC_BM = 128, TC_BN = 128, TC_BK = 64, TC_STAGES = 3, TC_THREADS = 512;
constexpr int TC_TILE_BYTES = TC_BM * TC_BK * 2;  // one operand tile of a stage (16 KB)
constexpr int TC_STAGE_BYTES = 2 * TC_TILE_BYTES;
constexpr uint32_t TC_MAX_POLLS = 1u << 24;
enum : uint32_t { ERR_TC_TIMEOUT = 8u };

struct TcArgs {
  GemmArgs P;
  int a_mn, b_mn;    // 1: the operand's M (N) index is the contiguous one (KM / KN)
  uint32_t *status;  // error word (bounded waits that expired)
  int K2;            // > 0: a second product A2 B2^T over K2, summed in the same accumulator
  int kchunk;        // split K: blockIdx.z covers K [z kchunk, (z + 1) kchunk) (0: all of K)
  float *partial;    // split K: slice z writes its plain product to partial + z * M * ldc
};

// shared memory bytes of the kernel (stages + barriers + 1024-byte alignment slack)
constexpr size_t TC_SMEM_BYTES = (size_t)TC_STAGES * TC_STAGE_BYTES + 1024 + 256;

// UMMA shared-memory matrix descriptor: start address, leading / stride byte
// offsets (16-byte units), descriptor version 1, 128-byte swizzle.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// instruction descriptor of kind::f16: BF16 x BF16 -> F32, M = 128, N = 128
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(TC_BN >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  const uint32_t z = 0u;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// two CTAs per SM: one CTA's epilogue overlaps the other's main loop
__global__ void __launch_bounds__(TC_THREADS, 2)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                   const __grid_constant__ CUtensorMap mapA2, const __grid_constant__ CUtensorMap mapB2, TcArgs T) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~uintptr_t(1023));
  const GemmArgs &P = T.P;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * TC_BN;
  // K range of this CTA: the whole K (plus K2), or one split-K slice
  int kt0 = 0, nk1 = (P.K + TC_BK - 1) / TC_BK;
  if (T.kchunk > 0) {
    kt0 = (int)blockIdx.z * (T.kchunk / TC_BK);
    nk1 = min(nk1, kt0 + T.kchunk / TC_BK);
  }
  const int nk = nk1 - kt0 + (T.K2 > 0 ? (T.K2 + TC_BK - 1) / TC_BK : 0);
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + TC_STAGES * TC_STAGE_BYTES);
  uint64_t *empty = full + TC_STAGES;
  uint64_t *accb = empty + TC_STAGES;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(accb + 1);
  if (threadIdx.x == 0) {
    for (int s = 0; s < TC_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accb, 1);
    fence_mbar_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"((uint32_t)TC_BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    tc_fence_before();
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  bool ok = true;
  // the other lanes of the two role warps wait at the warp barrier (not in a
  // polling loop that would share the warp's issue slots with the role lane)
  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer ----
      for (int kt = 0; kt < nk; ++kt) {
        const int s = kt % TC_STAGES;
        const uint32_t round = (uint32_t)(kt / TC_STAGES);
        if (kt >= TC_STAGES && !mbar_wait(&empty[s], (round - 1u) & 1u, TC_MAX_POLLS)) {
          ok = false;
          break;
        }
        unsigned char *sa = sm + s * TC_STAGE_BYTES, *sb = sa + TC_TILE_BYTES;
        mbar_expect_tx(&full[s], (uint32_t)TC_STAGE_BYTES);
        const bool second = kt0 + kt >= nk1;
        const CUtensorMap *ma = second ? &mapA2 : &mapA, *mb = second ? &mapB2 : &mapB;
        const int k0 = (second ? kt0 + kt - nk1 : kt0 + kt) * TC_BK;
        if (T.a_mn) {
          tma_load_2d(sa, ma, m0, k0, &full[s]);
          tma_load_2d(sa + TC_TILE_BYTES / 2, ma, m0 + 64, k0, &full[s]);
        } else {
          tma_load_2d(sa, ma, k0, m0, &full[s]);
        }
        if (T.b_mn) {
          tma_load_2d(sb, mb, n0, k0, &full[s]);
          tma_load_2d(sb + TC_TILE_BYTES / 2, mb, n0 + 64, k0, &full[s]);
        } else {
          tma_load_2d(sb, mb, k0, n0, &full[s]);
        }
    }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer ----
      const uint32_t idesc = umma_idesc_bf16(T.a_mn, T.b_mn);
      int issued = 0;
      for (int kt = 0; kt < nk; ++kt) {
        const int s = kt % TC_STAGES;
        if (!mbar_wait(&full[s], (uint32_t)(kt / TC_STAGES) & 1u, TC_MAX_POLLS)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_addr(sm + s * TC_STAGE_BYTES), sb = sa + TC_TILE_BYTES;
  #pragma unroll
        for (int k = 0; k < TC_BK / 16; ++k) {
          // K-major: 16 elements = 32 bytes along the swizzled row; MN-major: 16 rows of 128 bytes
          const uint64_t da = T.a_mn ? umma_desc_sw128(sa + k * 2048, TC_TILE_BYTES / 2, 1024)
                                     : umma_desc_sw128(sa + k * 32, 16, 1024);
          const uint64_t db = T.b_mn ? umma_desc_sw128(sb + k * 2048, TC_TILE_BYTES / 2, 1024)
                                     : umma_desc_sw128(sb + k * 32, 16, 1024);
          umma_bf16(tmem, da, db, idesc, (kt > 0 || k > 0) ? 1u : 0u);
        }
        umma_commit(&empty[s]);
        ++issued;
    }
    umma_commit(accb);  // arrives once every MMA issued above has completed
    (void)issued;
    }
    __syncwarp();
  }
  // ---- epilogue: warp w owns TMEM lanes (tile rows) 32w .. 32w + 31.  Each
  //      32-column chunk goes TMEM -> registers (thread = row) -> shared memory
  //      (the idle stage buffers; padded rows) -> registers (lane = column), so
  //      that every global load and store of the epilogue is a coalesced row ----
  ok &= mbar_wait(accb, 0, TC_MAX_POLLS);
  __syncwarp();
  tc_fence_after();
  // warps w, w + 4, w + 8 and w + 12 share TMEM lane quadrant w & 3 (a warp
  // may only read its own quadrant) and take one 32-column chunk each
  const int quad = warp & 3, part = warp >> 2;
  float *stage = reinterpret_cast<float *>(sm) + warp * 32 * 33;
  const int n_lane = lane;
#pragma unroll 1
  for (int c = part * (TC_BN / 128); c < (part + 1) * (TC_BN / 128); ++c) {
    uint32_t r[32];
    tmem_ld32(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(c * 32), r);
#pragma unroll
    for (int j = 0; j < 32; ++j) stage[lane * 33 + j] = __uint_as_float(r[j]);
    __syncwarp();
    const int n = n0 + c * 32 + n_lane;
    const float bn = (P.bias && n < P.N) ? P.bias[n] : 0.f;
    if (P.epi == MG_EPI_DGELU && T.kchunk == 0 && !P.accumulate && !P.bias) {
      // GELU' epilogue (the data gradients): rows in blocks of 8 whose
      // pre-activations are all requested before any is used, one memory
      // latency per block instead of one per row
#pragma unroll 1
      for (int i0 = 0; i0 < 32; i0 += 8) {
        float pin[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int m = m0 + quad * 32 + i0 + j;
          pin[j] = (ok && m < P.M && n < P.N) ? __ldg(P.pre_in + (size_t)m * P.ldp + n) : 0.f;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int m = m0 + quad * 32 + i0 + j;
          if (!ok || m >= P.M || n >= P.N) continue;
          const float v = stage[(i0 + j) * 33 + n_lane] * gelu_grad_f(pin[j]);
          const size_t o = (size_t)m * P.ldc + n;
          if (P.Cf) P.Cf[o] = v;
          if (P.Cb) P.Cb[o] = __float2bfloat16_rn(v);
        }
      }
    } else {
#pragma unroll 4
      for (int i = 0; i < 32; ++i) {
        const int m = m0 + quad * 32 + i;
        if (!ok || m >= P.M || n >= P.N) continue;
        float v = stage[i * 33 + n_lane];
        const size_t o = (size_t)m * P.ldc + n;
        if (T.kchunk > 0) {  // split K: the plain product of this slice (summed later in slice order)
          T.partial[(size_t)blockIdx.z * P.M * P.ldc + o] = v;
          continue;
        }
        if (P.accumulate) v += P.Cf[o];
        if (P.bias) v += bn;
        if (P.epi == MG_EPI_GELU) {
          if (P.pre_out) P.pre_out[(size_t)m * P.ldp + n] = v;
          v = gelu_f(v);
        } else if (P.epi == MG_EPI_DGELU) {
          v *= gelu_grad_f(P.pre_in[(size_t)m * P.ldp + n]);
        }
        if (P.Cf) P.Cf[o] = v;
        if (P.Cb) P.Cb[o] = __float2bfloat16_rn(v);
      }
    }
    __syncwarp();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TC_BN));
  if (!ok && lane == 0 && T.status) atomicOr(T.status, (uint32_t)ERR_TC_TIMEOUT);
}

// out[m][n] = sum over slices z (in order) of part[z][m][n], n < N (rows of
// stride ld): the split-K reduction.  Rows over blockIdx.y, 16-byte column
// groups over x (ld a multiple of 4, 16-byte aligned buffers: checked on the
// host); the slices are read streaming, the sum keeps the slice order.
__global__ void tc_splitk_sum_kernel(const float *part, int nslice, int M, int N, int ld, float *out) {
  const int64_t total = (int64_t)M * ld;
  const int nq = (N + 3) >> 2;
  for (int m = blockIdx.y; m < M; m += gridDim.y) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
      const int64_t o = (int64_t)m * ld + 4 * q;
      float4 v = __ldcs(reinterpret_cast<const float4 *>(part + o));
      for (int z = 1; z < nslice; ++z) {
        const float4 w = __ldcs(reinterpret_cast<const float4 *>(part + (int64_t)z * total + o));
        v.x += w.x;
        v.y += w.y;
        v.z += w.z;
        v.w += w.w;
      }
      const int n = 4 * q;
      if (n + 3 < N) {
        *reinterpret_cast<float4 *>(out + o) = v;
      } else {
        out[o] = v.x;
        if (n + 1 < N) out[o + 1] = v.y;
        if (n + 2 < N) out[o + 2] = v.z;
      }
    }
  }
}

}  // namespace aob
