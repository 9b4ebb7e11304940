// Shared device helpers: error plumbing, Philox4x32-10, noise samplers,
// warp reductions.  sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

namespace aob {

// ---------------------------------------------------------------------------
// host-side error plumbing: every C entry point catches aob::Error and turns
// it into AOB_ERR plus a thread-local message.
struct Error : std::runtime_error {
  explicit Error(const std::string &m) : std::runtime_error(m) {}
};

void set_last_error(const std::string &msg);

inline void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw Error(std::string(what) + ": " + cudaGetErrorString(e));
}
#define AOB_CUDA(call) ::aob::cuda_check((call), #call)
#define AOB_LAUNCH_CHECK(name) ::aob::cuda_check(cudaGetLastError(), name)
#define AOB_REQUIRE(cond, msg)                 \
  do {                                         \
    if (!(cond)) throw ::aob::Error(msg);      \
  } while (0)

// RAII device buffer
template <typename T>
struct DevBuf {
  T *p = nullptr;
  int64_t n = 0;
  DevBuf() = default;
  explicit DevBuf(int64_t count) { alloc(count); }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(int64_t count) {
    release();
    n = count;
    if (count > 0) {
      AOB_CUDA(cudaMalloc(&p, sizeof(T) * (size_t)count));
      AOB_CUDA(cudaMemset(p, 0, sizeof(T) * (size_t)count));
    }
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void upload(const T *host, int64_t count) {
    AOB_REQUIRE(count <= n, "upload larger than buffer");
    if (count > 0) AOB_CUDA(cudaMemcpy(p, host, sizeof(T) * (size_t)count, cudaMemcpyHostToDevice));
  }
  size_t bytes() const { return sizeof(T) * (size_t)n; }
};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11).  Counter layout used by the sensors:
// c0 = pixel index, c1 = frame, c2 = stream tag, c3 = draw number.
struct U4 {
  uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ void mulhilo32(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
#ifdef __CUDA_ARCH__
  hi = __umulhi(a, b);
  lo = a * b;
#else
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
#endif
}

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c.x, hi0, lo0);
    mulhilo32(0xCD9E8D57u, c.z, hi1, lo1);
    U4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

enum : uint32_t { TAG_POISSON = 0 };

__device__ __forceinline__ double u01(uint32_t x) {
  return __dmul_rn(__dadd_rn((double)x, 0.5), 2.3283064365386963e-10);  // (x + 0.5) / 2^32
}
// 24-bit uniform in (0, 1), exact in float32: ((x >> 8) + 0.5) / 2^24
__device__ __forceinline__ float u01f(uint32_t x) { return ((float)(x >> 8) + 0.5f) * 5.9604644775390625e-08f; }

// Photon and readout noise of one pixel.  One Philox block per (pixel, frame,
// draw): draw 0 gives the first Poisson draw (words x, y) and the readout
// noise (words z, w); rejected Poisson draws continue with draws 1, 2, ...
//
// Poisson deviate: inversion for small means (Devroye 1986, X.3), PTRS
// (Hoermann 1993, "The transformed rejection method for generating Poisson
// random variables") otherwise.  Every value that decides the outcome is
// computed with correctly rounded IEEE operations only (explicit _rn
// intrinsics, no contracted multiply-add), so the CPU oracle reproduces it:
//  * inversion: float64, u from word x (32-bit uniform), p0 = exp(-lambda),
//    1/k as the correctly rounded reciprocal;
//  * PTRS fast path (acceptance ~86 % of draws): float32 sqrt / div / mul /
//    add on 24-bit uniforms;
//  * PTRS exact acceptance test: float64 in product form, log(k!) from the
//    table of cumulative log sums (first AOB_LOGFACT_SMEM entries from shared
//    memory), two-term Stirling series beyond the table.
#define AOB_LOGFACT_N 4096
#define AOB_LOGFACT_SMEM 1024
#define AOB_RK_N 1024
struct NoiseTables {
  const double *logfact;  // log(k!) for k < AOB_LOGFACT_N (device memory)
};

__device__ __forceinline__ double log_factorial(double k, const double *lf_smem, const NoiseTables &T) {
  if (k < (double)AOB_LOGFACT_SMEM) return lf_smem[(int)k];
  if (k < (double)AOB_LOGFACT_N) return __ldg(T.logfact + (int)k);
  const double x = __dadd_rn(k, 1.0);
  const double ix = __ddiv_rn(1.0, x);
  double r = __dmul_rn(__dadd_rn(x, -0.5), log(x));
  r = __dadd_rn(__dadd_rn(r, -x), 0.91893853320467274178);
  const double c = __dadd_rn(__dmul_rn(0.08333333333333333, ix), -__dmul_rn(__dmul_rn(0.002777777777777778, ix),
                                                                            __dmul_rn(ix, ix)));
  return __dadd_rn(r, c);
}

// lam: the float32 mean; w0: Philox block of draw 0.
static __device__ __forceinline__ float poisson_sample(float lamf, const U4 &w0, uint32_t idx, uint32_t frame,
                                                    uint32_t k0, uint32_t k1, const double *lf_smem,
                                                    NoiseTables T) {
  if (!(lamf > 0.f)) return 0.f;
  if (lamf < 10.f) {
    const double lam = (double)lamf;
    const double u = u01(w0.x);
    double p = exp(-lam);
    double f = p;
    int k = 0;
    while (u > f && k < AOB_RK_N - 1) {
      k += 1;
      p = __dmul_rn(p, __dmul_rn(lam, __drcp_rn((double)k)));
      f = __dadd_rn(f, p);
    }
    return (float)k;
  }
  const float slam = __fsqrt_rn(lamf);
  const float b = __fadd_rn(0.931f, __fmul_rn(2.53f, slam));
  const float a = __fadd_rn(-0.059f, __fmul_rn(0.02483f, b));
  const float vr = __fadd_rn(0.9277f, -__fdiv_rn(3.6224f, __fadd_rn(b, -2.0f)));
  const float a2 = __fmul_rn(2.0f, a);
  // constants of the exact acceptance test, computed only when a draw needs it
  double loglam = 0.0, invalpha = 0.0;
  bool slow_ready = false;
  U4 w = w0;
  for (uint32_t d = 0; d < 64u; ++d) {
    if (d > 0) w = philox4x32_10(U4{idx, frame, TAG_POISSON, d}, k0, k1);
    const float u = __fadd_rn(u01f(w.x), -0.5f);
    const float v = u01f(w.y);
    const float us = __fadd_rn(0.5f, -fabsf(u));
    const float k = floorf(__fadd_rn(__fadd_rn(__fmul_rn(__fadd_rn(__fdiv_rn(a2, us), b), u), lamf), 0.43f));
    if (us >= 0.07f && v <= vr) return k;
    if (k < 0.f || (us < 0.013f && v > us)) continue;
    if (!slow_ready) {
      loglam = log((double)lamf);
      invalpha = __dadd_rn(1.1239, __ddiv_rn(1.1328, __dadd_rn((double)b, -3.4)));
      slow_ready = true;
    }
    const double usd = (double)us;
    const double lhs =
        __ddiv_rn(__dmul_rn((double)v, invalpha), __dadd_rn(__ddiv_rn((double)a, __dmul_rn(usd, usd)), (double)b));
    const double rhs = exp(__dadd_rn(__dadd_rn(__dmul_rn((double)k, loglam), -(double)lamf),
                                     -log_factorial((double)k, lf_smem, T)));
    if (lhs <= rhs) return k;
  }
  return floorf(__fadd_rn(lamf, 0.5f));
}

// Standard normal deviate by Box-Muller in float32 from words z (u1) and w (u2)
// of the pixel's draw-0 block.  Compared with the CPU oracle within a
// tolerance, not bit for bit.
__device__ __forceinline__ float gauss_sample(const U4 &w0) {
  const float u1 = u01f(w0.z);
  const float u2 = u01f(w0.w);
  return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

// ---------------------------------------------------------------------------
// mbarrier + bulk-copy (TMA engine, non-tensor form) helpers.  Only CTA-local
// barriers and copies from this GPU's own global memory into this CTA's shared
// memory; no cluster multicast anywhere.
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
// global -> shared bulk copy completing on ``bar``; dst, src 16-byte aligned, bytes % 16 == 0
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Bounded wait for phase ``parity`` of ``bar``: true when it completed, false
// after ``max_polls`` unsuccessful polls (the caller records an error).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t max_polls) {
  const uint32_t a = smem_addr(bar);
  for (uint32_t i = 0; i < max_polls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// error word written by kernels whose bounded waits expired
enum : uint32_t { ERR_MBAR_TIMEOUT = 1u };

// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace aob
