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

// r (n x k, ldr) = b - A x; rowabs[i] = sum_j |a_ij| (when not NULL). K_MAX >= k.
template <int K_MAX>
__global__ void __launch_bounds__(kResWarps * 32)
    residual_kernel(const double* __restrict__ a, int64_t lda, int64_t n, const double* __restrict__ x, int64_t ldx,
                    const double* __restrict__ b, int64_t ldb, int k, double* __restrict__ r, int64_t ldr,
                    double* __restrict__ rowabs) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * kResWarps + (threadIdx.x >> 5);
  if (row >= n) return;
  const double* ar = a + row * lda;
  double s[K_MAX];
#pragma unroll
  for (int c = 0; c < K_MAX; ++c) s[c] = 0.0;
  double abs_sum = 0.0;
  for (int64_t j = lane; j < n; j += 32) {
    const double v = __ldcs(ar + j);  // streamed once: keep it out of L2's way
    abs_sum += fabs(v);
    const double* xj = x + j * ldx;
#pragma unroll
    for (int c = 0; c < K_MAX; ++c)
      if (c < k) s[c] = fma(v, __ldg(xj + c), s[c]);
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) {
    abs_sum += __shfl_xor_sync(0xffffffffu, abs_sum, off);
#pragma unroll
    for (int c = 0; c < K_MAX; ++c) s[c] += __shfl_xor_sync(0xffffffffu, s[c], off);
  }
  if (lane < k) {
    double mine = 0.0;
#pragma unroll
    for (int c = 0; c < K_MAX; ++c)
      if (c == lane) mine = s[c];
    r[row * ldr + lane] = b[row * ldb + lane] - mine;
  }
  if (lane == 0 && rowabs) rowabs[row] = abs_sum;
}

// norms[0] = max_i rowabs[i]; for each column c: norms[1+3c..] = ||r_c||, ||x_c||, ||b_c||
// (infinity norms); berr_out[0] = max_c ||r_c|| / (||A|| ||x_c|| + ||b_c||).
__global__ void __launch_bounds__(1024) backward_error_kernel(const double* __restrict__ rowabs, int64_t n,
                                                              const double* __restrict__ r, int64_t ldr,
                                                              const double* __restrict__ x, int64_t ldx,
                                                              const double* __restrict__ b, int64_t ldb, int k,
                                                              double* __restrict__ out) {
  __shared__ double red[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  auto block_max = [&](double v) -> double {
#pragma unroll
    for (int off = 16; off; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
#pragma unroll
    for (int off = 16; off; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    return v;
  };
  double amax = 0.0;
  for (int64_t i = tid; i < n; i += blockDim.x) amax = fmax(amax, rowabs[i]);
  amax = block_max(amax);
  double worst = 0.0;
  bool nan = false;
  for (int c = 0; c < k; ++c) {
    double rn = 0.0, xn = 0.0, bn = 0.0;
    for (int64_t i = tid; i < n; i += blockDim.x) {
      const double rv = fabs(r[i * ldr + c]);
      nan |= rv != rv;
      rn = fmax(rn, rv);
      xn = fmax(xn, fabs(x[i * ldx + c]));
      bn = fmax(bn, fabs(b[i * ldb + c]));
    }
    rn = block_max(rn);
    xn = block_max(xn);
    bn = block_max(bn);
    const double den = amax * xn + bn;
    const double e = den > 0.0 ? rn / den : rn;
    worst = fmax(worst, e);
  }
  nan = __syncthreads_or(nan);
  if (tid == 0) {
    out[0] = nan ? __longlong_as_double(0x7ff8000000000000ll) : worst;
    out[1] = amax;
  }
}

int residual_f64(const double* a, int64_t lda, int64_t n, const double* x, int64_t ldx, const double* b, int64_t ldb,
                 int64_t k, double* r, int64_t ldr, double* rowabs, cudaStream_t stream) {
  if (n == 0 || k == 0) return RM_OK;
  const unsigned blocks = (unsigned)((n + kResWarps - 1) / kResWarps);
  for (int64_t c0 = 0; c0 < k; c0 += 16) {
    const int kc = (int)std::min<int64_t>(16, k - c0);
    if (kc <= 4)
      residual_kernel<4><<<blocks, kResWarps * 32, 0, stream>>>(a, lda, n, x + c0, ldx, b + c0, ldb, kc, r + c0, ldr,
                                                                 c0 == 0 ? rowabs : nullptr);
    else
      residual_kernel<16><<<blocks, kResWarps * 32, 0, stream>>>(a, lda, n, x + c0, ldx, b + c0, ldb, kc, r + c0, ldr,
                                                                  c0 == 0 ? rowabs : nullptr);
    RM_LAUNCHED();
  }
  return RM_OK;
}

int backward_error_f64(const double* rowabs, int64_t n, const double* r, int64_t ldr, const double* x, int64_t ldx,
                       const double* b, int64_t ldb, int64_t k, double* out, cudaStream_t stream) {
  backward_error_kernel<<<1, 1024, 0, stream>>>(rowabs, n, r, ldr, x, ldx, b, ldb, (int)k, out);
  RM_LAUNCHED();
  return RM_OK;
}

}  // namespace rm
