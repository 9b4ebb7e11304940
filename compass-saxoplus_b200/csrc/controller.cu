// Least-squares controller: command-matrix MVM fused with the integrator,
// command delay / latency interpolation / perturbation / clip, and the
// float64 pseudo-inverse of the interaction matrix.
//
// Reference: SutraControllerLs::comp_com (libsutra/src.cpp/sutra_controller_ls.cpp:
// 251-285) runs cuBLAS Sgemv on the column-major cmat, then mult_int_krnl
// (libsutra/src.cu/sutra_utils.cu:631-639).  comp_voltage
// (sutra_controller.cpp:245-263) is a chain of axpy / copy / clip launches.
//
// Layout in HBM: besides the caller-visible column-major float32 cmat, the MVM
// reads a row-major (actuator-major) packed copy -- float32, bfloat16, or FP8
// E4M3 with one float32 scale per actuator row -- with rows padded to 16 bytes.
// Each CTA owns a contiguous block of actuator rows, stages the slope vector in
// shared memory, and each warp streams whole rows with 16-byte loads (8 loads
// in flight per lane), accumulates in float32 and applies the integrator in
// the epilogue.  No cross-CTA reduction is needed, so the result is
// deterministic.

#include <cublas_v2.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "aob_objects.hpp"

namespace aob {

struct MvmArgs {
  const void *mat;        // packed rows
  const float *rscale;    // per-row scale (FP8) or null
  int ld;                 // elements per packed row
  int nrow, ncol;
  const float *s;         // slopes (device)
  float *err;             // -cmat.s
  float *com;             // integrator state
  const float *mgain;     // modal gains (null: 1 for every row)
  float gain;
  float berta;            // integrator state factor: com = gain * e * mgain + berta * com
  int integrate;
  uint32_t *bump;         // incremented once per launch when set (noise frame counter)
  uint32_t *status;       // error word (bounded waits that expired)
  int rows_per_cta;       // bulk kernel: rows staged per CTA (host-checked to fit)
  const uint32_t *use;    // when set and *use == 0 the launch does nothing (the learned
                          // reconstructor's commands were used instead)
};

// Dot product of one 16-byte packed chunk with its slopes sv[STRIDE * q],
// q < V/4.  The slopes are staged in shared memory in a lane-swizzled order:
// the V/4 float4 groups of chunk c = lane + 32*j live at float4 index
// (j*(V/4) + q)*32 + lane, so a warp reads them with conflict-free 128-bit
// loads for every precision (STRIDE = 32 from the staged vector, 1 from a
// register copy).
template <typename T>
struct Pack;
template <>
struct Pack<float> {
  static constexpr int N = 4;
  template <int STRIDE = 32>
  __device__ static float dot(const uint4 &q, const float4 *sv) {
    const float *f = reinterpret_cast<const float *>(&q);
    const float4 s = sv[0];
    float a = f[0] * s.x;
    a = fmaf(f[1], s.y, a);
    a = fmaf(f[2], s.z, a);
    return fmaf(f[3], s.w, a);
  }
};
template <>
struct Pack<__nv_bfloat16> {
  static constexpr int N = 8;
  template <int STRIDE = 32>
  __device__ static float dot(const uint4 &q, const float4 *sv) {
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&q);
    float a = 0.f;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const float4 s = sv[STRIDE * i];
      const float2 f0 = __bfloat1622float2(h[2 * i]);
      const float2 f1 = __bfloat1622float2(h[2 * i + 1]);
      a = fmaf(f0.x, s.x, a);
      a = fmaf(f0.y, s.y, a);
      a = fmaf(f1.x, s.z, a);
      a = fmaf(f1.y, s.w, a);
    }
    return a;
  }
};
template <>
struct Pack<__nv_fp8_e4m3> {
  static constexpr int N = 16;
  template <int STRIDE = 32>
  __device__ static float dot(const uint4 &q, const float4 *sv) {
    const __nv_fp8x2_e4m3 *h = reinterpret_cast<const __nv_fp8x2_e4m3 *>(&q);
    float a = 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float4 s = sv[STRIDE * i];
      const float2 f0 = static_cast<float2>(h[2 * i]);
      const float2 f1 = static_cast<float2>(h[2 * i + 1]);
      a = fmaf(f0.x, s.x, a);
      a = fmaf(f0.y, s.y, a);
      a = fmaf(f1.x, s.z, a);
      a = fmaf(f1.y, s.w, a);
    }
    return a;
  }
};

constexpr int MVM_THREADS = 512;
constexpr int MVM_UNROLL = 8;

// shared floats needed for the swizzled slope vector (whole 32-chunk rounds)
__host__ __device__ inline int mvm_smem_floats(int ld, int v) { return ((ld / v + 31) / 32) * 32 * v; }

template <typename T>
__global__ void __launch_bounds__(MVM_THREADS) ls_mvm_kernel(MvmArgs A) {
  extern __shared__ __align__(16) float s_sh[];
  if (A.use && *A.use == 0u) return;
  constexpr int V = Pack<T>::N;
  constexpr int Q = V / 4;
  const int nchunk = A.ld / V;  // 16-byte chunks per row
  const int nsh = mvm_smem_floats(A.ld, V);
  for (int i = threadIdx.x; i < nsh; i += blockDim.x) {
    // inverse of the swizzle: float i sits in group g = i/4, element e = i%4
    const int g = i >> 2, e = i & 3;
    const int l = g & 31, jq = g >> 5;
    const int j = jq / Q, q = jq - j * Q;
    const int src = (l + 32 * j) * V + 4 * q + e;
    s_sh[i] = (src < A.ncol) ? __ldcg(A.s + src) : 0.f;  // global-space load: may overtake the stores
  }
  if (A.bump && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(A.bump, 1u);
  __syncthreads();
  const float4 *sv = reinterpret_cast<const float4 *>(s_sh);
  const int r0 = (int)((blockIdx.x * (uint32_t)A.nrow) / gridDim.x);  // 32-bit: host-checked range
  const int r1 = (int)(((blockIdx.x + 1) * (uint32_t)A.nrow) / gridDim.x);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  const float4 *svl = sv + lane;
  for (int r = r0 + warp; r < r1; r += nw) {
    const uint4 *row = reinterpret_cast<const uint4 *>(static_cast<const T *>(A.mat) + (size_t)r * A.ld) + lane;
    float acc[MVM_UNROLL];
#pragma unroll
    for (int u = 0; u < MVM_UNROLL; ++u) acc[u] = 0.f;
    int j = 0;
    for (; 32 * (j + MVM_UNROLL - 1) + lane < nchunk; j += MVM_UNROLL) {
      uint4 q[MVM_UNROLL];
#pragma unroll
      for (int u = 0; u < MVM_UNROLL; ++u) q[u] = __ldcs(row + 32 * (j + u));
#pragma unroll
      for (int u = 0; u < MVM_UNROLL; ++u) acc[u] += Pack<T>::dot(q[u], svl + 32 * Q * (j + u));
    }
    for (; 32 * j + lane < nchunk; ++j) acc[0] += Pack<T>::dot(__ldcs(row + 32 * j), svl + 32 * Q * j);
    float tot = 0.f;
#pragma unroll
    for (int u = 0; u < MVM_UNROLL; ++u) tot += acc[u];
    tot = warp_sum(tot);
    if (lane == 0) {
      // all loads before the first store (global-space loads, one round trip)
      const float sc = A.rscale ? __ldg(A.rscale + r) : 1.f;
      const float mg = (A.integrate && A.mgain) ? __ldg(A.mgain + r) : 1.f;
      const float cm = A.integrate ? __ldcg(A.com + r) : 0.f;
      if (A.rscale) tot *= sc;
      const float e = -tot;
      A.err[r] = e;
      if (A.integrate) A.com[r] = fmaf(A.gain, e * mg, A.berta * cm);
    }
  }
}

// Bulk-copy MVM.  Each CTA owns rows [r0, r1) of the packed matrix; one
// thread issues one TMA bulk copy per row into shared memory (each completing
// on its own mbarrier) before anything else happens, so the whole matrix is in
// flight from the first microsecond.  The slopes are staged with 16-byte
// loads; once the rows have landed the CTA reduces them split-K: warp w, lane
// l take chunks c = l + 32 (w + NW i), read each slope chunk once and apply it
// to every row from registers, and the per-warp partial sums are added in
// warp order (deterministic).  Waits are bounded: an expired wait sets
// ERR_MBAR_TIMEOUT in *status and the CTA's rows are skipped.
constexpr uint32_t MBAR_MAX_POLLS = 1u << 22;

__host__ __device__ inline size_t mvm_bars_bytes(int rows) { return 128 * (((size_t)rows * 8 + 127) / 128); }

template <typename T>
__global__ void __launch_bounds__(MVM_THREADS) ls_mvm_bulk_kernel(MvmArgs A) {
  extern __shared__ __align__(128) unsigned char sm[];
  constexpr int V = Pack<T>::N;
  constexpr int Q = V / 4;
  constexpr int NW = MVM_THREADS / 32;
  constexpr int RB = 8;  // rows per register block
  const int nchunk = A.ld / V;
  const int nsh = mvm_smem_floats(A.ld, V);
  const uint32_t row_bytes = (uint32_t)(A.ld * sizeof(T));
  const int r0 = (int)((blockIdx.x * (uint32_t)A.nrow) / gridDim.x);  // 32-bit: host-checked range
  const int r1 = (int)(((blockIdx.x + 1) * (uint32_t)A.nrow) / gridDim.x);
  const int R = r1 - r0;
  if (A.use && *A.use == 0u) return;
  // shared memory: barriers | slopes | rows | per-warp partial sums
  uint64_t *bars = reinterpret_cast<uint64_t *>(sm);
  float *s_sh = reinterpret_cast<float *>(sm + mvm_bars_bytes(A.rows_per_cta));
  unsigned char *rows = reinterpret_cast<unsigned char *>(s_sh + nsh);
  float *part = reinterpret_cast<float *>(rows + (size_t)A.rows_per_cta * row_bytes);
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);  // one barrier for all the rows
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned char *src = static_cast<const unsigned char *>(A.mat) + (size_t)r0 * row_bytes;
    mbar_expect_tx(&bars[0], (uint32_t)R * row_bytes);
    for (int r = 0; r < R; ++r)
      bulk_g2s(rows + (size_t)r * row_bytes, src + (size_t)r * row_bytes, row_bytes, &bars[0]);
  }
  if (A.bump && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(A.bump, 1u);
  // epilogue inputs of this thread's row (R <= blockDim), fetched now
  float e_sc = 1.f, e_mg = 1.f, e_cm = 0.f;
  if ((int)threadIdx.x < R) {
    const int gr = r0 + threadIdx.x;
    if (A.rscale) e_sc = __ldg(A.rscale + gr);
    if (A.integrate) {
      if (A.mgain) e_mg = __ldg(A.mgain + gr);
      e_cm = __ldcg(A.com + gr);
    }
  }
  for (int g = threadIdx.x; g < nsh / 4; g += blockDim.x) {
    const int l = g & 31, jq = g >> 5;
    const int j = jq / Q, q = jq - j * Q;
    const int src = (l + 32 * j) * V + 4 * q;
    float4 v4;
    if (src + 3 < A.ncol) {
      v4 = __ldcg(reinterpret_cast<const float4 *>(A.s + src));
    } else {
      v4.x = src < A.ncol ? __ldcg(A.s + src) : 0.f;
      v4.y = src + 1 < A.ncol ? __ldcg(A.s + src + 1) : 0.f;
      v4.z = src + 2 < A.ncol ? __ldcg(A.s + src + 2) : 0.f;
      v4.w = 0.f;
    }
    reinterpret_cast<float4 *>(s_sh)[g] = v4;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool rows_ok = true;
  rows_ok = mbar_wait(&bars[0], 0, MBAR_MAX_POLLS);
  if (!rows_ok && threadIdx.x == 0 && A.status) atomicOr(A.status, (uint32_t)ERR_MBAR_TIMEOUT);
  const float4 *sv4 = reinterpret_cast<const float4 *>(s_sh);
  for (int rb = 0; rb < R; rb += RB) {
    float acc[RB];
#pragma unroll
    for (int u = 0; u < RB; ++u) acc[u] = 0.f;
    if (rows_ok) {
      for (int jj = warp; 32 * jj + lane < nchunk; jj += NW) {
        const int c = lane + 32 * jj;
        float4 sv[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) sv[q] = sv4[(jj * Q + q) * 32 + lane];
#pragma unroll
        for (int u = 0; u < RB; ++u)
          if (rb + u < R) {
            const uint4 q4 = reinterpret_cast<const uint4 *>(rows + (size_t)(rb + u) * row_bytes)[c];
            acc[u] += Pack<T>::template dot<1>(q4, sv);
          }
      }
    }
    int u;
    const float t = warp_sum8(acc, lane, u);
    if ((lane & 3) == 0 && rb + u < R) part[warp * A.rows_per_cta + rb + u] = t;
  }
  __syncthreads();
  if (rows_ok && (int)threadIdx.x < R) {
    const int r = threadIdx.x;
    float tot = 0.f;
#pragma unroll
    for (int w = 0; w < NW; ++w) tot += part[w * A.rows_per_cta + r];
    const int gr = r0 + r;
    if (A.rscale) tot *= e_sc;
    const float e = -tot;
    A.err[gr] = e;
    if (A.integrate) A.com[gr] = fmaf(A.gain, e * e_mg, A.berta * e_cm);
  }
  // no CTA may exit with a copy still landing in its shared memory
  if (!rows_ok && threadIdx.x == 0)
    mbar_wait(&bars[0], 0, MBAR_MAX_POLLS);
}

// y[i] = alpha * sum_j A[i][j] x[j] + beta * y[i] for a row-major A (lda
// floats per row): the secondary products of the generic controller (the
// pseudo-open-loop slopes, matE in the modal-integrator and two-matrix laws).
// One warp per row; the row sum runs lane-strided, then a butterfly.
__global__ void gemv_rows_kernel(const float *A, int lda, int nrow, int ncol, const float *x, float alpha, float beta,
                                 float *y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int r = warp; r < nrow; r += nw) {
    const float *a = A + (size_t)r * lda;
    float acc = 0.f;
    for (int j = lane; j < ncol; j += 32) acc = fmaf(a[j], x[j], acc);
    acc = warp_sum(acc);
    if (lane == 0) y[r] = beta == 0.f ? alpha * acc : fmaf(alpha, acc, beta * y[r]);
  }
}

// x[i] = x[i] * scale[i] * gain (mult_krnl, libsutra/src.cu/sutra_utils.cu:603-610)
__global__ void mult_vec_kernel(float *x, const float *scale, float gain, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = x[i] * scale[i] * gain;
}
// y[i] += x[i] (axpy with alpha 1)
__global__ void add_vec_kernel(float *y, const float *x, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] += x[i];
}

struct VoltArgs {
  const float *com;
  float *oldest;       // ring[0]: read for latency, then overwritten with com
  const float *second; // ring[1]
  float a, b;
  int delayed;
  const float *pert[8];
  int pn[8];
  int pcpt[8];
  int npert;
  float vmin, vmax;
  int do_clip;
  float *out;
  int n;
};

__global__ void voltage_kernel(VoltArgs A) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
    float v;
    if (A.delayed) {
      v = A.a * A.oldest[i] + A.b * A.second[i];
      A.oldest[i] = A.com[i];
    } else {
      v = A.com[i];
    }
    for (int j = 0; j < A.npert; ++j) v += A.pert[j][A.pcpt[j] + (int64_t)i * A.pn[j]];
    if (A.do_clip) v = fminf(fmaxf(v, A.vmin), A.vmax);
    A.out[i] = v;
  }
}

__global__ void add_perturb_kernel(float *y, const float *buf, int cpt, int nper, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] += buf[cpt + (int64_t)i * nper];
}

__global__ void clip_kernel(float *x, int n, float lo, float hi) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = fminf(fmaxf(x[i], lo), hi);
}

__global__ void d2f_kernel(const double *a, float *b, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
__global__ void f2d_kernel(const float *a, double *b, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (double)a[i];
}
__global__ void scale_cols_kernel(const double *U, const double *w, double *out, int n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < (int64_t)n * n; t += (int64_t)gridDim.x * blockDim.x)
    out[t] = U[t] * w[t / n];
}

}  // namespace aob

using namespace aob;

aob_ls::aob_ls(int device_, int nslope_, int nactu_, float delay_)
    : device(device_), nslope(nslope_), nactu(nactu_) {
  AOB_REQUIRE(nslope > 0 && nactu > 0, "ls: nslope and nactu must be > 0");
  AOB_CUDA(cudaSetDevice(device));
  set_delay(delay_);
  centroids.alloc(nslope);
  status.alloc(1);
  err.alloc(nactu);
  com_clipped.alloc(nactu);
  gains.alloc(nactu);
  std::vector<float> one(nactu, 1.f);
  gains.upload(one.data(), nactu);
  cmat.alloc((int64_t)nactu * nslope);
  h_cmat.assign((size_t)nactu * nslope, 0.f);
}

// The delay and its interpolation weights.  The command ring holds the last
// floor(delay) + 2 commands (1 without delay): ring[0] is read as the command of
// floor(delay) + 1 steps back, so its length follows the delay.  A longer ring
// gets zero buffers in front (the oldest commands); a shorter one drops its
// oldest; the current command (the ring's back) is kept either way.
void aob_ls::set_delay(float d) {
  AOB_REQUIRE(d >= 0.f, "ls.set_delay: the delay must be >= 0");
  delay = d;
  const int fl = (int)d;
  a = d - (float)fl;
  b = 1.f - a;
  const int nring = delay > 0 ? fl + 2 : 1;
  if ((int)ring.size() < nring) {
    AOB_CUDA(cudaSetDevice(device));
    while ((int)ring.size() < nring) ring.emplace_front(nactu);
  }
  while ((int)ring.size() > nring) ring.pop_front();
}

void aob_ls::ensure_packed(int p) {
  if (packed_valid[p]) return;
  AOB_CUDA(cudaSetDevice(device));
  if (p == AOB_PREC_F32) {
    ld = (nslope + 3) / 4 * 4;
    std::vector<float> rows((size_t)nactu * ld, 0.f);
    for (int s = 0; s < nslope; ++s)
      for (int r = 0; r < nactu; ++r) rows[(size_t)r * ld + s] = h_cmat[(size_t)s * nactu + r];
    cm_f32.alloc((int64_t)nactu * ld);
    cm_f32.upload(rows.data(), (int64_t)nactu * ld);
  } else if (p == AOB_PREC_BF16) {
    const int l = (nslope + 7) / 8 * 8;
    std::vector<__nv_bfloat16> rows((size_t)nactu * l, __float2bfloat16(0.f));
    for (int s = 0; s < nslope; ++s)
      for (int r = 0; r < nactu; ++r) rows[(size_t)r * l + s] = __float2bfloat16(h_cmat[(size_t)s * nactu + r]);
    cm_bf16.alloc((int64_t)nactu * l);
    cm_bf16.upload(reinterpret_cast<const uint16_t *>(rows.data()), (int64_t)nactu * l);
  } else {
    const int l = (nslope + 15) / 16 * 16;
    std::vector<__nv_fp8_e4m3> rows((size_t)nactu * l, __nv_fp8_e4m3(0.f));
    std::vector<float> sc(nactu, 1.f);
    for (int r = 0; r < nactu; ++r) {
      float m = 0.f;
      for (int s = 0; s < nslope; ++s) m = std::max(m, std::fabs(h_cmat[(size_t)s * nactu + r]));
      sc[r] = m > 0.f ? m / 448.f : 1.f;  // 448 = largest finite E4M3 value
      const float inv = 1.f / sc[r];
      for (int s = 0; s < nslope; ++s) rows[(size_t)r * l + s] = __nv_fp8_e4m3(h_cmat[(size_t)s * nactu + r] * inv);
    }
    cm_fp8.alloc((int64_t)nactu * l);
    cm_fp8.upload(reinterpret_cast<const uint8_t *>(rows.data()), (int64_t)nactu * l);
    row_scale.alloc(nactu);
    row_scale.upload(sc.data(), nactu);
  }
  packed_valid[p] = true;
}

void aob_ls::comp_com(cudaStream_t s, uint32_t *bump, const uint32_t *use) {
  if (open_loop) return;
  AOB_CUDA(cudaSetDevice(device));
  if (kind == AOB_CTRL_GENERIC) {
    AOB_REQUIRE(!use, "comp_com: the learned reconstructor drives LS controllers only");
    generic_comp_com(s, bump);
    return;
  }
  ensure_packed(prec);
  MvmArgs A{};
  A.nrow = nactu;
  A.ncol = nslope;
  A.s = centroids.p;
  A.err = err.p;
  A.com = com();
  A.mgain = gains.p;
  A.gain = gain;
  A.berta = 1.f;
  A.integrate = 1;
  A.bump = bump;
  A.status = status.p;
  A.use = use;
  if (prec == AOB_PREC_F32) {
    A.mat = cm_f32.p;
    A.ld = (nslope + 3) / 4 * 4;
  } else if (prec == AOB_PREC_BF16) {
    A.mat = cm_bf16.p;
    A.ld = (nslope + 7) / 8 * 8;
  } else {
    A.mat = cm_fp8.p;
    A.rscale = row_scale.p;
    A.ld = (nslope + 15) / 16 * 16;
  }
  launch_mvm(A, s);
}

namespace {
template <typename T>
void launch_mvm_t(const MvmArgs &A0, int grid, bool bulk, cudaStream_t s) {
  MvmArgs A = A0;
  constexpr int V = Pack<T>::N;
  const size_t slope_bytes = sizeof(float) * mvm_smem_floats(A.ld, V);
  if (bulk) {
    A.rows_per_cta = (A.nrow + grid - 1) / grid;
    const size_t sm = mvm_bars_bytes(A.rows_per_cta) + slope_bytes + (size_t)A.rows_per_cta * A.ld * sizeof(T) +
                      sizeof(float) * (MVM_THREADS / 32) * A.rows_per_cta;
    smem_opt_in(reinterpret_cast<const void *>(ls_mvm_bulk_kernel<T>), (int)sm);
    ls_mvm_bulk_kernel<T><<<grid, MVM_THREADS, sm, s>>>(A);
    AOB_LAUNCH_CHECK("ls_mvm_bulk_kernel");
  } else {
    smem_opt_in(reinterpret_cast<const void *>(ls_mvm_kernel<T>), (int)slope_bytes);
    ls_mvm_kernel<T><<<grid, MVM_THREADS, slope_bytes, s>>>(A);
    AOB_LAUNCH_CHECK("ls_mvm_kernel");
  }
}
}  // namespace

// Largest shared-memory budget a CTA may request on sm_100 (227 KB).
constexpr size_t MVM_SMEM_MAX = 227 * 1024;

// Kernel and grid for this matrix: the bulk-copy kernel when a CTA's rows fit in
// shared memory with one CTA per SM, the register-streaming kernel otherwise
// (or when the caller forces it).  ``nblocks`` > 0 overrides the grid size.
void aob_ls::launch_mvm(MvmArgs &A, cudaStream_t s) {
  const int nsm = num_sms(device);
  int esize = prec == AOB_PREC_F32 ? 4 : (prec == AOB_PREC_BF16 ? 2 : 1);
  int V = 16 / esize;
  int grid = nblocks > 0 ? std::min(nblocks, nactu) : std::min(nactu, nsm);
  AOB_REQUIRE((int64_t)nactu * grid < (int64_t)1 << 32, "ls: too many actuators for the MVM row split");
  const size_t slope_bytes = sizeof(float) * mvm_smem_floats(A.ld, V);
  const int rpc = (nactu + grid - 1) / grid;
  const size_t need = mvm_bars_bytes(rpc) + slope_bytes + (size_t)rpc * A.ld * esize +
                      sizeof(float) * (MVM_THREADS / 32) * rpc;
  const bool bulk = (mvm_kind == 0 || mvm_kind == 1) && need <= MVM_SMEM_MAX && mvm_kind != 2 && rpc <= MVM_THREADS;
  if (prec == AOB_PREC_F32)
    launch_mvm_t<float>(A, grid, bulk, s);
  else if (prec == AOB_PREC_BF16)
    launch_mvm_t<__nv_bfloat16>(A, grid, bulk, s);
  else
    launch_mvm_t<__nv_fp8_e4m3>(A, grid, bulk, s);
}

// The command laws of SutraControllerGeneric::comp_com
// (libsutra/src.cpp/sutra_controller_generic.cpp:219-328), single GPU:
//   integrator        com = berta com - gain cmat s
//   modal_integrator  buff = -(cmat s) * modal gains;  com = gain matE buff + berta com
//   2matrices         buff = -(cmat s) * modal gains;  com = (matE com1) * decay + buff
// with berta = leaky factor, and with pseudo-open-loop slopes (polc: s is
// replaced by s - imat com_clipped, SutraController::comp_polc,
// sutra_controller.cpp:349-375) berta = (1 - gain) leaky.  com1 is the previous
// command: a copy of com without delay, the ring's second-newest buffer with
// delay (SutraController::command_delay, sutra_controller.cpp:205-218).
void aob_ls::generic_comp_com(cudaStream_t s, uint32_t *bump) {
  ensure_packed(prec);
  const int thr = 256, grid_v = std::max(1, std::min((nactu + thr - 1) / thr, 1024));
  const float *sin = centroids.p;
  float berta = leaky;
  if (polc) {
    AOB_REQUIRE(imat_rows.p != nullptr, "comp_com: polc needs the interaction matrix (set_imat)");
    AOB_CUDA(cudaMemcpyAsync(ol_meas.p, centroids.p, sizeof(float) * nslope, cudaMemcpyDeviceToDevice, s));
    gemv_rows_kernel<<<std::max(1, std::min((nslope + 7) / 8, 4096)), 256, 0, s>>>(
        imat_rows.p, nactu, nslope, nactu, com_clipped.p, -1.f, 1.f, ol_meas.p);
    AOB_LAUNCH_CHECK("gemv_rows_kernel (polc)");
    sin = ol_meas.p;
    berta = (1.f - gain) * leaky;
  }
  MvmArgs A{};
  A.nrow = nactu;
  A.ncol = nslope;
  A.s = sin;
  A.err = err.p;
  A.com = com();
  A.mgain = nullptr;
  A.gain = gain;
  A.berta = berta;
  A.integrate = law == AOB_LAW_INTEGRATOR ? 1 : 0;
  A.bump = bump;
  A.status = status.p;
  if (prec == AOB_PREC_F32) {
    A.mat = cm_f32.p;
    A.ld = (nslope + 3) / 4 * 4;
  } else if (prec == AOB_PREC_BF16) {
    A.mat = cm_bf16.p;
    A.ld = (nslope + 7) / 8 * 8;
  } else {
    A.mat = cm_fp8.p;
    A.rscale = row_scale.p;
    A.ld = (nslope + 15) / 16 * 16;
  }
  launch_mvm(A, s);
  if (law == AOB_LAW_INTEGRATOR) return;
  // err = -(cmat s); buff = err * modal gains
  AOB_REQUIRE(matE_rows.p != nullptr, "comp_com: this command law needs matE (set_matE)");
  mult_vec_kernel<<<grid_v, thr, 0, s>>>(err.p, gains.p, 1.f, nactu);
  AOB_LAUNCH_CHECK("mult_vec_kernel");
  const int grid_r = std::max(1, std::min((nactu + 7) / 8, 4096));
  if (law == AOB_LAW_MODAL_INTEGRATOR) {
    gemv_rows_kernel<<<grid_r, 256, 0, s>>>(matE_rows.p, nactu, nactu, nactu, err.p, gain, berta, com());
    AOB_LAUNCH_CHECK("gemv_rows_kernel (modal integrator)");
    return;
  }
  // 2matrices
  const float *com1;
  if (delay > 0) {
    com1 = ring[ring.size() - 2].p;
  } else {
    AOB_CUDA(cudaMemcpyAsync(com1_tmp.p, com(), sizeof(float) * nactu, cudaMemcpyDeviceToDevice, s));
    com1 = com1_tmp.p;
  }
  gemv_rows_kernel<<<grid_r, 256, 0, s>>>(matE_rows.p, nactu, nactu, nactu, com1, 1.f, 0.f, com());
  AOB_LAUNCH_CHECK("gemv_rows_kernel (2matrices)");
  mult_vec_kernel<<<grid_v, thr, 0, s>>>(com(), decay.p, 1.f, nactu);
  add_vec_kernel<<<grid_v, thr, 0, s>>>(com(), err.p, nactu);
  AOB_LAUNCH_CHECK("2matrices update");
}

void aob_ls::make_generic() {
  kind = AOB_CTRL_GENERIC;
  law = AOB_LAW_INTEGRATOR;
  AOB_CUDA(cudaSetDevice(device));
  ol_meas.alloc(nslope);
  com1_tmp.alloc(nactu);
  decay.alloc(nactu);
}

void aob_ls::set_matE(const float *h) {
  std::vector<float> rows((size_t)nactu * nactu);
  for (int j = 0; j < nactu; ++j)
    for (int i = 0; i < nactu; ++i) rows[(size_t)i * nactu + j] = h[i + (size_t)j * nactu];
  AOB_CUDA(cudaSetDevice(device));
  if (!matE_rows.p) matE_rows.alloc((int64_t)nactu * nactu);
  matE_rows.upload(rows.data(), (int64_t)nactu * nactu);
}

void aob_ls::set_imat_rows(const float *h) {
  // imat is [nslope, nactu] column-major: row i (slope) = h[i + j nslope]
  std::vector<float> rows((size_t)nslope * nactu);
  for (int j = 0; j < nactu; ++j)
    for (int i = 0; i < nslope; ++i) rows[(size_t)i * nactu + j] = h[i + (size_t)j * nslope];
  AOB_CUDA(cudaSetDevice(device));
  if (!imat_rows.p) imat_rows.alloc((int64_t)nslope * nactu);
  imat_rows.upload(rows.data(), (int64_t)nslope * nactu);
}

void aob_ls::comp_voltage(cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  VoltArgs A{};
  A.com = com();
  A.delayed = delay > 0 ? 1 : 0;
  if (A.delayed) {
    A.oldest = ring[0].p;
    A.second = ring[1].p;
  }
  A.a = a;
  A.b = b;
  for (auto &kv : perturb) {
    Perturb &p = kv.second;
    if (!p.on) continue;
    AOB_REQUIRE(A.npert < 8, "comp_voltage: at most 8 enabled perturbation buffers");
    A.pert[A.npert] = p.buf.p;
    A.pn[A.npert] = p.n;
    A.pcpt[A.npert] = p.cpt;
    ++A.npert;
    p.cpt = (p.cpt < p.n - 1) ? p.cpt + 1 : 0;
  }
  A.vmin = volt_min;
  A.vmax = volt_max;
  A.do_clip = volt_min < volt_max ? 1 : 0;
  A.out = com_clipped.p;
  A.n = nactu;
  voltage_kernel<<<std::max(1, std::min((nactu + 255) / 256, 1024)), 256, 0, s>>>(A);
  AOB_LAUNCH_CHECK("voltage_kernel");
  if (A.delayed) {
    // the oldest buffer now holds a copy of the current command and becomes it
    aob::DevBuf<float> t = std::move(ring.front());
    ring.pop_front();
    ring.push_back(std::move(t));
  }
}

// SutraController::add_perturb (sutra_controller.cpp:266-285): every enabled
// perturbation buffer adds its current row to com_clipped, then advances.
void aob_ls::apply_perturb(cudaStream_t s) {
  AOB_CUDA(cudaSetDevice(device));
  const int grid = std::max(1, std::min((nactu + 255) / 256, 1024));
  for (auto &kv : perturb) {
    Perturb &p = kv.second;
    if (!p.on) continue;
    add_perturb_kernel<<<grid, 256, 0, s>>>(com_clipped.p, p.buf.p, p.cpt, p.n, nactu);
    AOB_LAUNCH_CHECK("add_perturb_kernel");
    p.cpt = (p.cpt < p.n - 1) ? p.cpt + 1 : 0;
  }
}

void aob_ls::clip(cudaStream_t s) {
  if (!(volt_min < volt_max)) return;
  AOB_CUDA(cudaSetDevice(device));
  clip_kernel<<<std::max(1, std::min((nactu + 255) / 256, 1024)), 256, 0, s>>>(com_clipped.p, nactu, volt_min, volt_max);
  AOB_LAUNCH_CHECK("clip_kernel");
}

namespace {
void cublas_check(cublasStatus_t st, const char *w) {
  if (st != CUBLAS_STATUS_SUCCESS) throw aob::Error(std::string(w) + ": cublas status " + std::to_string((int)st));
}
void cusolver_check(cusolverStatus_t st, const char *w) {
  if (st != CUSOLVER_STATUS_SUCCESS) throw aob::Error(std::string(w) + ": cusolver status " + std::to_string((int)st));
}
}  // namespace

// svdec_imat: U = imat^T imat (float64), eigen-decomposed in place with
// cuSOLVER Dsyevd; eigenvalues ascending (sutra_controller_ls.cpp:116-150).
void aob_ls::svdec_imat() {
  AOB_REQUIRE(imat.p != nullptr, "svdec_imat: imat not set");
  AOB_CUDA(cudaSetDevice(device));
  DevBuf<double> D((int64_t)nslope * nactu);
  f2d_kernel<<<1024, 256>>>(imat.p, D.p, D.n);
  AOB_LAUNCH_CHECK("f2d_kernel");
  U.alloc((int64_t)nactu * nactu);
  eig.alloc(nactu);
  cublasHandle_t hb;
  cublas_check(cublasCreate(&hb), "cublasCreate");
  const double one = 1.0, zero = 0.0;
  cublasStatus_t st = cublasDgemm(hb, CUBLAS_OP_T, CUBLAS_OP_N, nactu, nactu, nslope, &one, D.p, nslope, D.p,
                                  nslope, &zero, U.p, nactu);
  cublasDestroy(hb);
  cublas_check(st, "cublasDgemm");
  cusolverDnHandle_t hs;
  cusolver_check(cusolverDnCreate(&hs), "cusolverDnCreate");
  int lwork = 0;
  cusolverStatus_t ss = cusolverDnDsyevd_bufferSize(hs, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nactu,
                                                    U.p, nactu, eig.p, &lwork);
  if (ss != CUSOLVER_STATUS_SUCCESS) { cusolverDnDestroy(hs); cusolver_check(ss, "Dsyevd_bufferSize"); }
  DevBuf<double> work(std::max(lwork, 1));
  DevBuf<int> info(1);
  ss = cusolverDnDsyevd(hs, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, nactu, U.p, nactu, eig.p, work.p,
                        lwork, info.p);
  cusolverDnDestroy(hs);
  cusolver_check(ss, "cusolverDnDsyevd");
  int h_info = 0;
  AOB_CUDA(cudaMemcpy(&h_info, info.p, sizeof(int), cudaMemcpyDeviceToHost));
  AOB_REQUIRE(h_info == 0, "svdec_imat: eigen decomposition did not converge");
  eigenvals_f.alloc(nactu);
  d2f_kernel<<<64, 256>>>(eig.p, eigenvals_f.p, nactu);
  AOB_LAUNCH_CHECK("d2f_kernel");
  AOB_CUDA(cudaDeviceSynchronize());
}

// build_cmat: cmat = U diag(1/ev, first nfilt modes and |ev| <= 1e-9 dropped) U^T imat^T
// (sutra_controller_ls.cpp:174-217), in float64, stored as float32.
void aob_ls::build_cmat(int nfilt) {
  AOB_REQUIRE(U.p != nullptr, "build_cmat: call svdec_imat first");
  AOB_CUDA(cudaSetDevice(device));
  std::vector<double> ev(nactu), inv(nactu, 0.0);
  AOB_CUDA(cudaMemcpy(ev.data(), eig.p, sizeof(double) * nactu, cudaMemcpyDeviceToHost));
  for (int i = std::max(nfilt, 0); i < nactu; ++i) inv[i] = std::fabs(ev[i]) > 1.e-9 ? 1.0 / ev[i] : 0.0;
  DevBuf<double> w(nactu), T1((int64_t)nactu * nactu), T2((int64_t)nactu * nactu), D((int64_t)nslope * nactu),
      C((int64_t)nactu * nslope);
  w.upload(inv.data(), nactu);
  scale_cols_kernel<<<1024, 256>>>(U.p, w.p, T1.p, nactu);
  f2d_kernel<<<1024, 256>>>(imat.p, D.p, D.n);
  AOB_LAUNCH_CHECK("build_cmat prep");
  cublasHandle_t hb;
  cublas_check(cublasCreate(&hb), "cublasCreate");
  const double one = 1.0, zero = 0.0;
  cublasStatus_t st = cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_T, nactu, nactu, nactu, &one, T1.p, nactu, U.p, nactu,
                                  &zero, T2.p, nactu);
  if (st == CUBLAS_STATUS_SUCCESS)
    st = cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_T, nactu, nslope, nactu, &one, T2.p, nactu, D.p, nslope, &zero, C.p,
                     nactu);
  cublasDestroy(hb);
  cublas_check(st, "cublasDgemm");
  d2f_kernel<<<1024, 256>>>(C.p, cmat.p, C.n);
  AOB_LAUNCH_CHECK("d2f_kernel");
  AOB_CUDA(cudaMemcpy(h_cmat.data(), cmat.p, sizeof(float) * h_cmat.size(), cudaMemcpyDeviceToHost));
  packed_valid[0] = packed_valid[1] = packed_valid[2] = false;
}
