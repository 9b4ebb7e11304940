// Batched in-place complex 2-D FFT (fft.cu).
#pragma once

#include <cuda_runtime.h>

namespace aob {
// n x n transforms of ``batch`` contiguous images (x fastest), in place.
void fft2d(float2 *data, int n, int batch, bool inverse, int device, cudaStream_t s);
const float2 *fft_twiddles(int device, int n);
}  // namespace aob
