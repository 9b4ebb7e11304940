// Pieces shared by the kernels that reduce packed command-matrix rows (the
// fused RTC step, the batched Monte Carlo step, the learned reconstructor's
// LS fallback): the 16-byte chunk dot product and the bounded grid barrier.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include "aob_common.cuh"

namespace aob {

// Dot product of one 16-byte chunk of a packed row with its slopes sv[0 .. N/4)
// (contiguous float4s).  The operation order is the one every MVM kernel of
// this library uses, so their results agree bit for bit.
template <typename T>
struct RowPack;
template <>
struct RowPack<float> {
  static constexpr int N = 4;
  __device__ static float dot(const uint4 &q, const float4 *sv) {
    const float *f = reinterpret_cast<const float *>(&q);
    const float4 s = sv[0];
    return fmaf(f[3], s.w, fmaf(f[2], s.z, fmaf(f[1], s.y, f[0] * s.x)));
  }
};
template <>
struct RowPack<__nv_bfloat16> {
  static constexpr int N = 8;
  __device__ static float dot(const uint4 &q, const float4 *sv) {
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
    float a = 0.f;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const float4 s = sv[i];
      const float2 f0 = __bfloat1622float2(h[2 * i]), f1 = __bfloat1622float2(h[2 * i + 1]);
      a = fmaf(f1.y, s.w, fmaf(f1.x, s.z, fmaf(f0.y, s.y, fmaf(f0.x, s.x, a))));
    }
    return a;
  }
};
template <>
struct RowPack<__nv_fp8_e4m3> {
  static constexpr int N = 16;
  __device__ static float dot(const uint4 &q, const float4 *sv) {
    const __nv_fp8x2_e4m3 *h = reinterpret_cast<const __nv_fp8x2_e4m3 *>(&q);
    float a = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float4 s = sv[i];
      const float2 f0 = static_cast<float2>(h[2 * i]), f1 = static_cast<float2>(h[2 * i + 1]);
      a = fmaf(f1.y, s.w, fmaf(f1.x, s.z, fmaf(f0.y, s.y, fmaf(f0.x, s.x, a))));
    }
    return a;
  }
};

// shared floats for a slope vector staged in the swizzled layout (whole 32-chunk rounds)
__host__ __device__ inline int swizzled_slope_floats(int ld, int v) { return ((ld / v + 31) / 32) * 32 * v; }

enum : uint32_t { ERR_GRID_TIMEOUT = 2u };
constexpr uint32_t GRID_MAX_POLLS = 1u << 24;

// Grid-wide barrier for a cooperative launch.  ``ctr`` counts arrivals over the
// whole life of its owner: launch n raises it from n * G to (n + 1) * G, so a
// CTA's target is the next multiple of G above the value its own arrival saw
// and nothing has to be reset between launches (every CTA arrives exactly
// once per barrier, also when a wait times out).  One thread per CTA arrives
// with a release add (it publishes the CTA's writes, ordered before it by the
// CTA barrier), spins on relaxed loads and closes with one acquire load.  The
// wait is bounded; on expiry ERR_GRID_TIMEOUT is set and false returned.
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long atom_add_release_u64(unsigned long long *p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.add.release.gpu.global.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}
// Arrival half: every thread of the CTA calls it; thread 0 gets the target
// count to wait for (the others 0).  Work placed between grid_arrive and
// grid_wait overlaps the wait but is not published by the barrier.
__device__ __forceinline__ unsigned long long grid_arrive(unsigned long long *ctr, uint32_t nblocks) {
  __syncthreads();
  unsigned long long target = 0;
  if (threadIdx.x == 0) {
    const unsigned long long old = atom_add_release_u64(ctr, 1ull);
    target = (old / nblocks + 1ull) * nblocks;
  }
  return target;
}
// Waiting half: every thread of the CTA calls it with grid_arrive's result;
// at most max_polls polls.
__device__ __forceinline__ bool grid_wait(const unsigned long long *ctr, unsigned long long target, uint32_t *status,
                                          uint32_t max_polls = GRID_MAX_POLLS) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    int ok = 1;
    uint32_t i = 0;
    while (ld_relaxed_u64(ctr) < target) {
      if (++i >= max_polls) {
        ok = 0;
        atomicOr(status, (uint32_t)ERR_GRID_TIMEOUT);
        break;
      }
    }
    (void)ld_acquire_u64(ctr);  // orders this CTA's later reads after the other CTAs' writes
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}
__device__ __forceinline__ bool grid_barrier(unsigned long long *ctr, uint32_t nblocks, uint32_t *status) {
  return grid_wait(ctr, grid_arrive(ctr, nblocks), status);
}

}  // namespace aob
