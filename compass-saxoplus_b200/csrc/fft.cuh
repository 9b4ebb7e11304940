// Batched in-place complex 2-D FFT (fft.cu).
#pragma once

#include <cuda_runtime.h>

namespace aob {

__device__ __forceinline__ uint32_t bitrev(uint32_t x, int logn) { return __brev(x) >> (32 - logn); }

// ---------------------------------------------------------------------------
// Stockham auto-sort FFT in shared memory (natural order in and out), radix-8
// passes with the butterflies in registers and a last radix-2 or radix-4 pass
// when n is not a power of 8 (Govindaraju et al., "High performance discrete
// Fourier transforms on graphics processors", SC'08).  ``cols`` interleaved
// sequences: element m of sequence c is s[m * cols + c] (consecutive threads
// take consecutive c, so accesses are contiguous).  Pass with current
// sub-transform length ns: butterfly j of sequence c reads s[j + r n/R],
// multiplies by W_(ns R)^(r (j mod ns)), transforms in registers and writes
// to ((j / ns) ns R + j mod ns) + r ns.  cuFFT sign convention (forward
// exp(-2 pi i k m / n)), unnormalised.  tw: exp(-2 pi i m / n), m < n/2.

__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by -i (forward) or +i (inverse)
__device__ __forceinline__ float2 c_rot(float2 a, bool inverse) {
  return inverse ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int R>
__device__ __forceinline__ void dft_small(float2 *v, bool inverse);
template <>
__device__ __forceinline__ void dft_small<2>(float2 *v, bool) {
  const float2 a = v[0], b = v[1];
  v[0] = c_add(a, b);
  v[1] = c_sub(a, b);
}
template <>
__device__ __forceinline__ void dft_small<4>(float2 *v, bool inverse) {
  const float2 t0 = c_add(v[0], v[2]), t1 = c_sub(v[0], v[2]);
  const float2 t2 = c_add(v[1], v[3]), t3 = c_rot(c_sub(v[1], v[3]), inverse);
  v[0] = c_add(t0, t2);
  v[2] = c_sub(t0, t2);
  v[1] = c_add(t1, t3);
  v[3] = c_sub(t1, t3);
}
template <>
__device__ __forceinline__ void dft_small<8>(float2 *v, bool inverse) {
  float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
  dft_small<4>(e, inverse);
  dft_small<4>(o, inverse);
  const float h = 0.70710678118654752f;  // cos(pi / 4)
  const float sg = inverse ? 1.f : -1.f;
  // W8^k o[k]: W8 = exp(-/+ i pi / 4)
  const float2 o1 = make_float2(h * (o[1].x - sg * o[1].y), h * (o[1].y + sg * o[1].x));
  const float2 o2 = c_rot(o[2], inverse);
  const float2 o3 = make_float2(h * (-o[3].x - sg * o[3].y), h * (-o[3].y + sg * o[3].x));
  v[0] = c_add(e[0], o[0]);
  v[4] = c_sub(e[0], o[0]);
  v[1] = c_add(e[1], o1);
  v[5] = c_sub(e[1], o1);
  v[2] = c_add(e[2], o2);
  v[6] = c_sub(e[2], o2);
  v[3] = c_add(e[3], o3);
  v[7] = c_sub(e[3], o3);
}

// W_n^m for 0 <= m < n from the half table
__device__ __forceinline__ float2 fft_twiddle(const float2 *tw, int n, int m, bool inverse) {
  float2 w = m < (n >> 1) ? __ldg(tw + m) : __ldg(tw + (m - (n >> 1)));
  if (m >= (n >> 1)) w = make_float2(-w.x, -w.y);
  if (inverse) w.y = -w.y;
  return w;
}

// One Stockham pass of radix R; every thread handles at most MAXT butterflies.
template <int R, int MAXT>
__device__ __forceinline__ void stockham_pass(float2 *s, int n, int cols, int ns, const float2 *tw, bool inverse) {
  const int nb = n / R;
  const int tasks = nb * cols;
  float2 v[MAXT][R];
#pragma unroll
  for (int it = 0; it < MAXT; ++it) {
    const int t = threadIdx.x + it * blockDim.x;
    if (t < tasks) {
      const int j = t / cols, c = t - j * cols;
#pragma unroll
      for (int r = 0; r < R; ++r) v[it][r] = s[(j + r * nb) * cols + c];
      const int k = j & (ns - 1);
      if (ns > 1) {
        const int step = k * (n / (ns * R));
#pragma unroll
        for (int r = 1; r < R; ++r) v[it][r] = c_mul(v[it][r], fft_twiddle(tw, n, r * step, inverse));
      }
      dft_small<R>(v[it], inverse);
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < MAXT; ++it) {
    const int t = threadIdx.x + it * blockDim.x;
    if (t < tasks) {
      const int j = t / cols, c = t - j * cols;
      const int k = j & (ns - 1);
      const int d = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) s[(d + r * ns) * cols + c] = v[it][r];
    }
  }
  __syncthreads();
}

// Transform of ``cols`` interleaved sequences of length n (a power of two,
// 8 <= n <= 2048) in natural order, in place.  MAXT8 bounds the radix-8
// butterflies per thread and pass: (n / 8) * cols <= MAXT8 * blockDim.x.
// Call with all threads of the CTA; ends with a barrier.
template <int MAXT8>
__device__ __forceinline__ void smem_fft_stockham(float2 *s, int n, int cols, const float2 *tw, bool inverse) {
  int ns = 1;
  for (; ns * 8 <= n; ns *= 8) stockham_pass<8, MAXT8>(s, n, cols, ns, tw, inverse);
  if (ns * 4 == n)
    stockham_pass<4, 2 * MAXT8>(s, n, cols, ns, tw, inverse);
  else if (ns * 2 == n)
    stockham_pass<2, 4 * MAXT8>(s, n, cols, ns, tw, inverse);
}

// ---- compile-time variant: length N, COLS interleaved sequences, NT threads,
// all pass parameters constant (divisions by constants, exactly sized
// register blocks).  tws: the N/2 forward twiddles, in shared memory.
template <int R, int N, int COLS, int NT, int NS>
__device__ __forceinline__ void stockham_pass_ct(float2 *s, const float2 *tws, bool inverse) {
  constexpr int NB = N / R;
  constexpr int TASKS = NB * COLS;
  constexpr int MAXT = (TASKS + NT - 1) / NT;
  constexpr int STEP = N / (NS * R);
  float2 v[MAXT][R];
#pragma unroll
  for (int it = 0; it < MAXT; ++it) {
    const int t = threadIdx.x + it * NT;
    if (TASKS % NT == 0 || t < TASKS) {
      const int j = t / COLS, c = t - j * COLS;
#pragma unroll
      for (int r = 0; r < R; ++r) v[it][r] = s[(j + r * NB) * COLS + c];
      if (NS > 1) {
        const int k = j & (NS - 1);
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const int m = r * k * STEP;  // < N
          float2 w = tws[m & (N / 2 - 1)];
          if (m >= N / 2) w = make_float2(-w.x, -w.y);
          if (inverse) w.y = -w.y;
          v[it][r] = c_mul(v[it][r], w);
        }
      }
      dft_small<R>(v[it], inverse);
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < MAXT; ++it) {
    const int t = threadIdx.x + it * NT;
    if (TASKS % NT == 0 || t < TASKS) {
      const int j = t / COLS, c = t - j * COLS;
      const int k = j & (NS - 1);
      const int d = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) s[(d + r * NS) * COLS + c] = v[it][r];
    }
  }
  __syncthreads();
}

template <int N, int COLS, int NT, int NS>
struct StockhamCT {
  static __device__ __forceinline__ void run(float2 *s, const float2 *tws, bool inverse) {
    constexpr int R = (NS * 8 <= N) ? 8 : N / NS;
    stockham_pass_ct<R, N, COLS, NT, NS>(s, tws, inverse);
    if constexpr (NS * R < N) StockhamCT<N, COLS, NT, NS * R>::run(s, tws, inverse);
  }
};

// Transform of COLS interleaved length-N sequences (natural order, in place)
// by a CTA of NT threads; ends with a barrier.
template <int N, int COLS, int NT>
__device__ __forceinline__ void fft_ct(float2 *s, const float2 *tws, bool inverse) {
  StockhamCT<N, COLS, NT, 1>::run(s, tws, inverse);
}

// Radix-2 decimation-in-time transform on bit-reversed input (element m of
// sequence c at s[bitrev(m) * cols + c]); natural-order output.  Kept for
// callers that load in bit-reversed order.
__device__ __forceinline__ void smem_fft(float2 *s, int n, int logn, int cols, const float2 *tw, int inverse) {
  const int nb = (n / 2) * cols;  // butterflies per stage
  for (int st = 0; st < logn; ++st) {
    const int half = 1 << st;
    const int tstep = n >> (st + 1);
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
      const int c = t % cols;
      const int b = t / cols;
      const int grp = b >> st;
      const int pos = b & (half - 1);
      const int i = (grp * 2 * half + pos) * cols + c;
      const int j = i + half * cols;
      float2 w = __ldg(tw + pos * tstep);
      if (inverse) w.y = -w.y;
      const float2 u = s[i], v0 = s[j];
      const float2 v = make_float2(v0.x * w.x - v0.y * w.y, v0.x * w.y + v0.y * w.x);
      s[i] = make_float2(u.x + v.x, u.y + v.y);
      s[j] = make_float2(u.x - v.x, u.y - v.y);
    }
    __syncthreads();
  }
}

// n x n transforms of ``batch`` contiguous images (x fastest), in place.
void fft2d(float2 *data, int n, int batch, bool inverse, int device, cudaStream_t s);
const float2 *fft_twiddles(int device, int n);
}  // namespace aob
