// Shared device helpers: error plumbing, Philox4x32-10, noise samplers,
// warp reductions.  sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>

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

// Opt kernel ``fn`` into ``bytes`` of dynamic shared memory on the current
// device.  Recorded per (kernel, device) and only ever raised, under a lock,
// so that every device gets its own opt-in and no caller lowers the limit
// another one relies on.
inline void smem_opt_in(const void *fn, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> done;
  int dev = 0;
  AOB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  int &cur = done[{fn, dev}];
  if (bytes > cur) {
    AOB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    cur = bytes;
  }
}

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

// Photon and readout noise of one pixel.  Philox blocks (pixel, frame, tag 0,
// block b): block 0 gives the first Poisson draw (words x, y) and the readout
// noise (words z, w); rejected Poisson draws continue with block 1 (x, y then
// z, w), block 2, ...
//
// Poisson deviate: inversion for means below 40 (Devroye 1986, X.3; below 40
// it is cheaper than PTRS, whose quick acceptance rate is low for small means),
// PTRS (Hoermann 1993, "The transformed rejection method for generating
// Poisson random variables") otherwise, all in float32.  Every value that decides the
// outcome comes from correctly rounded IEEE operations only (explicit _rn
// intrinsics, no contracted multiply-add) and the project's own exp / log
// below, so the CPU oracle reproduces each sample bit for bit:
//  * inversion: p0 = exp(-lambda), then p *= lambda / k, F += p until F >= u
//    (at most 160 steps);
//  * PTRS: the fast acceptance test as published; the exact test in the log
//    domain with log(k!) in Stirling form, arranged as
//      k log(lambda / (k+1)) - log(k+1) / 2 + (k + 1 - lambda) - log(2 pi) / 2
//      - 1 / (12 (k+1)) + 1 / (360 (k+1)^3)
//    so that no large terms cancel (a table of log(k!) for k < 10).

// exp(x) for x in [-88, 0]: x = n ln2 + r (Cody-Waite split of ln2, n nearest
// integer to x / ln2), |r| <= ln2 / 2, e^r by its degree-7 Taylor polynomial
// (truncation below 1e-8 relative), times 2^n.
__device__ __forceinline__ float aob_expf_neg(float x) {
  const float n = rintf(__fmul_rn(x, 1.44269502f));
  const float r = __fadd_rn(__fadd_rn(x, -__fmul_rn(n, 0.693145752f)), -__fmul_rn(n, 1.42860677e-06f));
  float p = 1.98412701e-04f;
  p = __fadd_rn(__fmul_rn(p, r), 1.38888892e-03f);
  p = __fadd_rn(__fmul_rn(p, r), 8.33333377e-03f);
  p = __fadd_rn(__fmul_rn(p, r), 4.16666679e-02f);
  p = __fadd_rn(__fmul_rn(p, r), 1.66666672e-01f);
  p = __fadd_rn(__fmul_rn(p, r), 0.5f);
  p = __fadd_rn(__fmul_rn(p, r), 1.0f);
  p = __fadd_rn(__fmul_rn(p, r), 1.0f);
  return __fmul_rn(p, __int_as_float(((int)n + 127) << 23));
}

// log(m) for m in [sqrt(1/2), sqrt(2)] and log1p(d) for d in [-1/4, 1/2] through
// atanh: log((1+s)/(1-s)) = 2 s + 2 s^3/3 + ... + 2 s^11/11 (|s| <= 0.2).
__device__ __forceinline__ float aob_log_series(float s) {
  const float s2 = __fmul_rn(s, s);
  float t = 0.181818187f;                              // 2/11
  t = __fadd_rn(__fmul_rn(t, s2), 0.222222224f);       // 2/9
  t = __fadd_rn(__fmul_rn(t, s2), 0.285714298f);       // 2/7
  t = __fadd_rn(__fmul_rn(t, s2), 0.400000006f);       // 2/5
  t = __fadd_rn(__fmul_rn(t, s2), 0.666666687f);       // 2/3
  return __fadd_rn(__fmul_rn(s, 2.0f), __fmul_rn(__fmul_rn(s, s2), t));
}
// log(x) for normal x > 0: x = m 2^e with m in [sqrt(1/2), sqrt(2)].
__device__ __forceinline__ float aob_logf(float x) {
  const int bits = __float_as_int(x);
  int e = ((bits >> 23) & 0xff) - 127;
  float m = __int_as_float((bits & 0x007fffff) | 0x3f800000);
  if (m > 1.41421354f) {
    m = __fmul_rn(m, 0.5f);
    e += 1;
  }
  const float s = __fdiv_rn(__fadd_rn(m, -1.0f), __fadd_rn(m, 1.0f));
  const float fe = (float)e;
  return __fadd_rn(__fmul_rn(fe, 0.693145752f), __fadd_rn(__fmul_rn(fe, 1.42860677e-06f), aob_log_series(s)));
}
// log(1 + d) for -1/4 <= d <= 1/2 (|s| <= 0.2)
__device__ __forceinline__ float aob_log1pf(float d) { return aob_log_series(__fdiv_rn(d, __fadd_rn(2.0f, d))); }

#define AOB_POISSON_INV_KMAX 160
#define AOB_POISSON_INV_MAX_MEAN 40.f
// log(k!) for k < 10, float32 of the exact values
__device__ __forceinline__ float aob_logfact_small(int k) {
  switch (k) {
    case 0: case 1: return 0.f;
    case 2: return 0.693147182f;
    case 3: return 1.79175949f;
    case 4: return 3.17805386f;
    case 5: return 4.78749180f;
    case 6: return 6.57925129f;
    case 7: return 8.52516174f;
    case 8: return 10.6046028f;
    default: return 12.8018274f;
  }
}

// Poisson deviate by inversion (lamf < AOB_POISSON_INV_MAX_MEAN): chop-down
// search four steps per pass with the factors lambda / j from rk[j] (the
// correctly rounded reciprocals of 1..AOB_POISSON_INV_KMAX); the products and
// sums are formed in the sequential order, and since F only grows the first
// step with F >= u is found from the pass's four comparisons.
__device__ __forceinline__ float poisson_inversion(float lamf, const U4 &w0, const float *rk) {
  if (!(lamf > 0.f)) return 0.f;
  const float u = u01f(w0.x);
  float p = aob_expf_neg(-lamf);
  float f = p;
  if (!(u > f)) return 0.f;
  for (int k = 0; k < AOB_POISSON_INV_KMAX; k += 4) {
    const float a1 = __fmul_rn(lamf, rk[k + 1]), a2 = __fmul_rn(lamf, rk[k + 2]);
    const float a3 = __fmul_rn(lamf, rk[k + 3]), a4 = __fmul_rn(lamf, rk[k + 4]);
    const float p1 = __fmul_rn(p, a1), p2 = __fmul_rn(p1, a2), p3 = __fmul_rn(p2, a3), p4 = __fmul_rn(p3, a4);
    const float f1 = __fadd_rn(f, p1), f2 = __fadd_rn(f1, p2), f3 = __fadd_rn(f2, p3), f4 = __fadd_rn(f3, p4);
    if (!(u > f4)) return (float)(k + 4 - (int)!(u > f3) - (int)!(u > f2) - (int)!(u > f1));
    p = p4;
    f = f4;
  }
  return (float)AOB_POISSON_INV_KMAX;
}

// Poisson deviate by PTRS (lamf >= AOB_POISSON_INV_MAX_MEAN); w0: Philox block 0.
__device__ __forceinline__ float poisson_ptrs(float lamf, const U4 &w0, uint32_t idx, uint32_t frame, uint32_t k0,
                                              uint32_t k1) {
  const float slam = __fsqrt_rn(lamf);
  const float b = __fadd_rn(0.931f, __fmul_rn(2.53f, slam));
  const float a = __fadd_rn(-0.059f, __fmul_rn(0.02483f, b));
  const float vr = __fadd_rn(0.9277f, -__fdiv_rn(3.6224f, __fadd_rn(b, -2.0f)));
  const float a2 = __fmul_rn(2.0f, a);
  const float invalpha = __fadd_rn(1.1239f, __fdiv_rn(1.1328f, __fadd_rn(b, -3.4f)));
  U4 w = w0;
  for (uint32_t d = 0; d < 64u; ++d) {
    // draw 0: words x, y of block 0; draw d >= 1: block (d + 1) / 2, words x, y
    // for odd d and z, w for even d
    if (d & 1u) w = philox4x32_10(U4{idx, frame, TAG_POISSON, (d + 1u) >> 1}, k0, k1);
    const uint32_t wu = (d == 0u || (d & 1u)) ? w.x : w.z;
    const uint32_t wv = (d == 0u || (d & 1u)) ? w.y : w.w;
    const float u = __fadd_rn(u01f(wu), -0.5f);
    const float v = u01f(wv);
    const float us = __fadd_rn(0.5f, -fabsf(u));
    const float k = floorf(__fadd_rn(__fadd_rn(__fmul_rn(__fadd_rn(__fdiv_rn(a2, us), b), u), lamf), 0.43f));
    if (us >= 0.07f && v <= vr) return k;
    if (k < 0.f || (us < 0.013f && v > us)) continue;
    // exact test: log(v * invalpha / (a / us^2 + b)) <= log(pmf(k) e^lambda / ...) in log domain
    const float lhs =
        aob_logf(__fdiv_rn(__fmul_rn(v, invalpha), __fadd_rn(__fdiv_rn(a, __fmul_rn(us, us)), b)));
    float rhs;
    if (k < 10.f) {
      rhs = __fadd_rn(__fadd_rn(__fmul_rn(k, aob_logf(lamf)), -lamf), -aob_logfact_small((int)k));
    } else {
      const float x = __fadd_rn(k, 1.0f);
      const float d = __fdiv_rn(__fadd_rn(lamf, -x), x);
      const float lr = (d >= -0.25f && d <= 0.5f) ? aob_log1pf(d) : aob_logf(__fdiv_rn(lamf, x));
      const float ix = __frcp_rn(x);
      const float corr = __fadd_rn(__fmul_rn(0.0833333358f, ix),
                                   -__fmul_rn(__fmul_rn(0.00277777785f, ix), __fmul_rn(ix, ix)));
      rhs = __fadd_rn(__fmul_rn(k, lr), -__fmul_rn(0.5f, aob_logf(x)));
      rhs = __fadd_rn(rhs, __fadd_rn(x, -lamf));
      rhs = __fadd_rn(__fadd_rn(rhs, -0.918938518f), -corr);
    }
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
// Prefetch [src, src + bytes) into L2 (bytes and src: multiples of 16); no
// completion to wait for.
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
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
enum : uint32_t { ERR_MBAR_TIMEOUT = 1u, ERR_DOOR_TIMEOUT = 16u };

// grid-barrier words (mvm_core.cuh) an owner allocates: the arrival counter on
// a 128-byte line of its own
constexpr int GRID_WORDS = 16;

// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Eight warp sums at once (9 shuffles instead of 40): the xor butterfly of
// warp_sum with the eight values spread over the lanes as it goes -- at
// distance 16 a lane keeps four of the values and sends the other four, at
// 8 two, at 4 one.  Every total is formed by the same additions as
// warp_sum(a[i]) (float addition commutes), so the results are bit-identical.
// Returns the total of value ``row`` = 4 (lane>>4 & 1) + 2 (lane>>3 & 1) +
// (lane>>2 & 1), which all four lanes of the group hold.
__device__ __forceinline__ float warp_sum8(const float (&a)[8], int lane, int &row) {
  const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
  float b[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float keep = h16 ? a[i + 4] : a[i], send = h16 ? a[i] : a[i + 4];
    b[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
  float c[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float keep = h8 ? b[i + 2] : b[i], send = h8 ? b[i] : b[i + 2];
    c[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  float d = (h4 ? c[1] : c[0]) + __shfl_xor_sync(0xffffffffu, h4 ? c[0] : c[1], 4);
  d += __shfl_xor_sync(0xffffffffu, d, 2);
  d += __shfl_xor_sync(0xffffffffu, d, 1);
  row = 4 * (int)h16 + 2 * (int)h8 + (int)h4;
  return d;
}

}  // namespace aob
