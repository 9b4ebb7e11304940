// Batched in-place complex 2-D FFT (fft.cu).
#pragma once

#include <cuda_runtime.h>

namespace aob {

__device__ __forceinline__ uint32_t bitrev(uint32_t x, int logn) { return __brev(x) >> (32 - logn); }

// In-shared-memory radix-2 decimation-in-time transform of ``cols``
// interleaved sequences of length n: element m of sequence c lives at
// s[m * cols + c] and enters in bit-reversed order (m -> bitrev(m)); the
// result is in natural order.  tw: forward twiddles exp(-2 pi i m / n),
// m < n/2; inverse = conjugated twiddles.  Ends with a CTA barrier.
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
