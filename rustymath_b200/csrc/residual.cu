// FP64 residual r = b - A x and the normwise backward error, on the device.
//
// The backward error of a solve, max over right-hand sides c of
//   ||b_c - A x_c||_inf / (||A||_inf ||x_c||_inf + ||b_c||_inf),
// is stated beside every result, and the refinement loop tests it. One warp per row of A
// streams the row once from HBM (the kernel is bandwidth-bound: 8 bytes of A per 2*k
// flops) and keeps k running sums per lane; the row's |a| sum gives ||A||_inf for free.
#include "rm_internal.h"

namespace rm {

constexpr int kResWarps = 8;
constexpr int kResRowsPerWarp = 4;
constexpr int kResChunk = 256;  // rows of x staged in shared memory at a time
constexpr int kNormGroup = 16;  // columns per group of norm slots
constexpr int kNormSlots = 1 + 3 * kNormGroup;

__device__ __forceinline__ void atomic_max_nonneg(double* p, double v) {
  // non-negative doubles (and NaN, above +inf) order like their bit patterns
  if (v > 0.0 || v != v) atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}

// r (n x k, ldr) = b - A x, for k <= KC. Each warp owns kResRowsPerWarp rows of A and
// streams them once; x is staged through shared memory kResChunk rows at a time (every
// block reads it from L2). norms (zeroed by the caller) collects by atomic maxima
// norms[0] = ||A||_inf and, per column c, norms[1+c] = ||r_c||_inf (NaN if a residual is
// NaN) and norms[1+2*kNormGroup+c] = ||b_c||_inf.
template <int KC>
__global__ void __launch_bounds__(kResWarps * 32)
    residual_kernel(const double* __restrict__ a, int64_t lda, int64_t n, const double* __restrict__ x, int64_t ldx,
                    const double* __restrict__ b, int64_t ldb, int k, double* __restrict__ r, int64_t ldr,
                    double* __restrict__ norms) {
  __shared__ double xs[KC][kResChunk];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t row0 = ((int64_t)blockIdx.x * kResWarps + warp) * kResRowsPerWarp;
  double s[kResRowsPerWarp][KC];
  double absum[kResRowsPerWarp];
#pragma unroll
  for (int q = 0; q < kResRowsPerWarp; ++q) {
    absum[q] = 0.0;
#pragma unroll
    for (int c = 0; c < KC; ++c) s[q][c] = 0.0;
  }
  for (int64_t j0 = 0; j0 < n; j0 += kResChunk) {
    __syncthreads();
    for (int e = tid; e < KC * kResChunk; e += kResWarps * 32) {
      const int c = e / kResChunk, jj = e % kResChunk;
      xs[c][jj] = (j0 + jj < n && c < k) ? x[(j0 + jj) * ldx + c] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kResRowsPerWarp; ++q) {
      const int64_t row = row0 + q;
      if (row < n) {
        const double* ar = a + row * lda + j0;
        for (int jj = lane; jj < kResChunk && j0 + jj < n; jj += 32) {
          const double v = __ldcs(ar + jj);  // A streams through once
          absum[q] += fabs(v);
#pragma unroll
          for (int c = 0; c < KC; ++c) s[q][c] = fma(v, xs[c][jj], s[q][c]);
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kResRowsPerWarp; ++q) {
#pragma unroll
    for (int off = 16; off; off >>= 1) {
      absum[q] += __shfl_xor_sync(0xffffffffu, absum[q], off);
#pragma unroll
      for (int c = 0; c < KC; ++c) s[q][c] += __shfl_xor_sync(0xffffffffu, s[q][c], off);
    }
    const int64_t row = row0 + q;
    if (row < n) {
      if (lane < k) {
        double mine = 0.0;
#pragma unroll
        for (int c = 0; c < KC; ++c)
          if (c == lane) mine = s[q][c];
        const double bv = b[row * ldb + lane];
        const double rv = bv - mine;
        r[row * ldr + lane] = rv;
        if (norms) {
          atomic_max_nonneg(&norms[1 + lane], fabs(rv));
          atomic_max_nonneg(&norms[1 + 2 * kNormGroup + lane], fabs(bv));
        }
      }
      if (lane == 0 && norms) atomic_max_nonneg(&norms[0], absum[q]);
    }
  }
}

// norms[1+kNormGroup+c] = ||x_c||_inf for the n x k (k <= kNormGroup) row-major x.
__global__ void column_max_kernel(const double* __restrict__ x, int64_t ldx, int64_t n, int k, double* norms) {
  double m[kNormGroup];
#pragma unroll
  for (int c = 0; c < kNormGroup; ++c) m[c] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int c = 0; c < kNormGroup; ++c)
      if (c < k) m[c] = fmax(m[c], fabs(x[i * ldx + c]));
#pragma unroll
  for (int c = 0; c < kNormGroup; ++c) {
    double v = m[c];
#pragma unroll
    for (int off = 16; off; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0 && c < k) atomic_max_nonneg(&norms[1 + kNormGroup + c], v);
  }
}

// out[0] = max_c ||r_c|| / (||A|| ||x_c|| + ||b_c||) over every group of columns (NaN when a
// residual is NaN), out[1] = ||A||_inf.
__global__ void backward_error_kernel(const double* __restrict__ norms, int k, double* out) {
  if (threadIdx.x != 0) return;
  const double anorm = norms[0];
  double worst = 0.0;
  bool nan = false;
  for (int c = 0; c < k; ++c) {
    const double* g = norms + (c / kNormGroup) * kNormSlots;
    const int cc = c % kNormGroup;
    const double rn = g[1 + cc], xn = g[1 + kNormGroup + cc], bn = g[1 + 2 * kNormGroup + cc];
    nan |= rn != rn;
    const double den = anorm * xn + bn;
    worst = fmax(worst, den > 0.0 ? rn / den : rn);
  }
  out[0] = nan ? __longlong_as_double(0x7ff8000000000000ll) : worst;
  out[1] = anorm;
}

size_t residual_norms_bytes(int64_t k) { return (size_t)((k + kNormGroup - 1) / kNormGroup) * kNormSlots * 8 + 64; }

int residual_f64(const double* a, int64_t lda, int64_t n, const double* x, int64_t ldx, const double* b, int64_t ldb,
                 int64_t k, double* r, int64_t ldr, double* norms, cudaStream_t stream) {
  if (n == 0 || k == 0) return RM_OK;
  const int64_t per_block = (int64_t)kResWarps * kResRowsPerWarp;
  const unsigned blocks = (unsigned)((n + per_block - 1) / per_block);
  if (norms) RM_CUDA_TRY(cudaMemsetAsync(norms, 0, residual_norms_bytes(k), stream));
  for (int64_t c0 = 0, g = 0; c0 < k; c0 += kNormGroup, ++g) {
    const int kc = (int)std::min<int64_t>(kNormGroup, k - c0);
    double* ng = norms ? norms + g * kNormSlots : nullptr;
    if (kc <= 4)
      residual_kernel<4><<<blocks, kResWarps * 32, 0, stream>>>(a, lda, n, x + c0, ldx, b + c0, ldb, kc, r + c0, ldr,
                                                                 ng);
    else
      residual_kernel<16><<<blocks, kResWarps * 32, 0, stream>>>(a, lda, n, x + c0, ldx, b + c0, ldb, kc, r + c0, ldr,
                                                                  ng);
    RM_LAUNCHED();
  }
  return RM_OK;
}

int backward_error_f64(const double* x, int64_t ldx, int64_t n, int64_t k, double* norms, double* out,
                       cudaStream_t stream) {
  if (n == 0 || k == 0) {
    RM_CUDA_TRY(cudaMemsetAsync(out, 0, 2 * sizeof(double), stream));
    return RM_OK;
  }
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, 2 * device_sm_count());
  for (int64_t c0 = 0, g = 0; c0 < k; c0 += kNormGroup, ++g) {
    const int kc = (int)std::min<int64_t>(kNormGroup, k - c0);
    column_max_kernel<<<blocks, 256, 0, stream>>>(x + c0, ldx, n, kc, norms + g * kNormSlots);
    RM_LAUNCHED();
  }
  backward_error_kernel<<<1, 32, 0, stream>>>(norms, (int)k, out);
  RM_LAUNCHED();
  return RM_OK;
}

}  // namespace rm
