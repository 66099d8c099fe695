// What an LU factorization gives besides solves, on the device: the inverse, the determinant
// and its sign and log-magnitude, and solves for stacks of small factorizations in one launch.
//
// Replaces, for float64:
//  - Lu::inverse / lu_inverse (core/src/linalg/factor.rs:150-154, 645-664): U^-1 L^-1 from the
//    identity, skipping the zeros of L^-1 above its diagonal, then the columns permuted by perm;
//  - Lu::determinant and Lu::log_determinant with odd() (factor.rs:174-194): U's diagonal folded
//    in order, the sign from the permutation's parity;
//  - the stack forms Stacked::lu_inverse, det, slogdet, lu_solve (src/linalg/stacked.rs:136-171,
//    190-214), one CTA per matrix of the stack.
#include <cfloat>
#include <vector>

#include "rm_internal.h"

namespace rm {

constexpr int kGetriCols = kSolveCols;  // columns of the identity per pair of chain launches

__global__ void identity_kernel(double* __restrict__ y, int64_t n) {
  const int64_t total = n * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    y[e] = (e / n == e % n) ? 1.0 : 0.0;
}

// out[r][perm[c]] = y[r][c]; a position outside 0..n-1 sets RM_DEV_BAD_INDEX and is skipped.
__global__ void permute_columns_kernel(const double* __restrict__ y, const int64_t* __restrict__ perm, int64_t n,
                                       double* __restrict__ out, unsigned* status) {
  const int64_t total = n * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / n, c = e - r * n;
    const int64_t q = perm[c];
    if (q < 0 || q >= n) {
      flag_error(status, RM_DEV_BAD_INDEX);
      continue;
    }
    out[r * n + q] = y[e];
  }
}

size_t getri_f64_scratch_bytes(int64_t n) {
  const int64_t nblk = (n + kSolveBlock - 1) / kSolveBlock, chunks = (n + kGetriCols - 1) / kGetriCols;
  return ((size_t)n * n * 8 + 255) / 256 * 256 + (diag_blocks_bytes_max(n) + 255) / 256 * 256 +
         (size_t)chunks * 2 * (nblk + 1) * sizeof(int) + 256;
}

int getri_f64(const double* f, int64_t n, const int64_t* perm, double* out, void* scratch, unsigned* status,
              cudaStream_t stream) {
  if (n == 0) return RM_OK;
  if (n > INT32_MAX / 2) return RM_BAD_ARG;
  const int nblk = (int)((n + kSolveBlock - 1) / kSolveBlock);
  const int chunks = (int)((n + kGetriCols - 1) / kGetriCols);
  char* base = static_cast<char*>(scratch);
  double* y = reinterpret_cast<double*>(base);
  double* dinv = reinterpret_cast<double*>(base + ((size_t)n * n * 8 + 255) / 256 * 256);
  int* flags = reinterpret_cast<int*>(reinterpret_cast<char*>(dinv) + (diag_blocks_bytes_max(n) + 255) / 256 * 256);
  // the factors are column-major: unit L below the diagonal, U on and above it
  RM_TRY(invert_diag_blocks_f64(f, n, true, n, dinv, true, false, stream));
  RM_CUDA_TRY(cudaMemsetAsync(flags, 0, (size_t)chunks * 2 * (nblk + 1) * sizeof(int), stream));
  const int blocks = (int)std::min<int64_t>((n * n + 255) / 256, 8 * device_sm_count());
  identity_kernel<<<blocks, 256, 0, stream>>>(y, n);
  RM_LAUNCHED();
  const int ni = (int)n;
  for (int ch = 0; ch < chunks; ++ch) {
    const int c0 = ch * kGetriCols, kc = std::min(kGetriCols, ni - c0);
    // columns c0.. of L^-1 are zero above row c0: the lower solve starts at c0's block row
    const int b0 = c0 / kSolveBlock, r0 = b0 * kSolveBlock;
    int* fl = flags + (size_t)ch * 2 * (nblk + 1);
    RM_TRY(trsv_chain_f64(true, true, f + (int64_t)r0 * n + r0, n, ni - r0,
                          dinv + (size_t)b0 * kDiagMats * kSolveBlock * kSolveBlock, y + (int64_t)r0 * n + c0, n, kc,
                          fl, fl + nblk, status, stream));
    RM_TRY(trsv_chain_f64(false, true, f, n, ni, dinv, y + c0, n, kc, fl + nblk + 1, fl + 2 * nblk + 1, status,
                          stream));
  }
  permute_columns_kernel<<<blocks, 256, 0, stream>>>(y, perm, n, out, status);
  RM_LAUNCHED();
  return RM_OK;
}

// ------------------------------------------------------------------ determinants
constexpr int kDetThreads = 256;
constexpr int kDetChunk = 2048;  // diagonal items staged in shared memory per round

// Matrix blockIdx.x of the stack: the permutation's parity as rustymath's odd() counts it (a
// cycle counts once, at its smallest position; the walks run in parallel over the starting
// positions, each bounded by n steps), then U's diagonal folded in order by one thread from
// shared memory, with the logarithms formed beforehand by all threads.
__global__ void __launch_bounds__(kDetThreads) lu_det_kernel(const double* __restrict__ factors,
                                                             const int64_t* __restrict__ perm, int64_t n,
                                                             double* det, double* sign, double* logabs,
                                                             unsigned* status) {
  __shared__ double dsm[kDetChunk], lsm[kDetChunk];
  __shared__ int cyc[kDetThreads / 32];
  __shared__ int bad;
  const int64_t m = blockIdx.x;
  const double* f = factors + m * n * n;
  const int64_t* p = perm + m * n;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  int cycles = 0;
  for (int64_t start = threadIdx.x; start < n; start += blockDim.x) {
    int64_t i = p[start], steps = 0;
    while (i > start && i < n && steps < n) {
      i = p[i];
      ++steps;
    }
    if (i < 0 || i >= n) {
      bad = 1;
      continue;
    }
    if (i == start) ++cycles;
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) cycles += __shfl_xor_sync(0xffffffffu, cycles, off);
  if ((threadIdx.x & 31) == 0) cyc[threadIdx.x >> 5] = cycles;
  __syncthreads();
  if (bad) {
    if (threadIdx.x == 0) flag_error(status, RM_DEV_BAD_INDEX);
    return;
  }
  int64_t total = 0;
  for (int w = 0; w < kDetThreads / 32; ++w) total += cyc[w];
  const bool odd = (n - total) % 2 == 1;
  double prod = 1.0, s = odd ? -1.0 : 1.0, l = 0.0;
  for (int64_t b = 0; b < n; b += kDetChunk) {
    const int cnt = (int)(n - b < kDetChunk ? n - b : kDetChunk);
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
      const double d = f[(b + e) * n + b + e];
      dsm[e] = d;
      lsm[e] = d != 0.0 ? log(fabs(d)) : 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int e = 0; e < cnt; ++e) {
        const double d = dsm[e], mag = fabs(d);
        prod = prod * d;
        if (mag == 0.0) {
          s = 0.0;
          l = -INFINITY;
        } else {
          s = s * (d * (1.0 / mag));
          l = l + lsm[e];
        }
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (det) det[m] = odd ? -prod : prod;
    if (sign) sign[m] = s;
    if (logabs) logabs[m] = l;
  }
}

// ------------------------------------------------------------------ small stacked solves
constexpr int kSmallSolveMax = 256;  // a thread per row
constexpr int kSmallSolveCols = 64;

// x = A^-1 b (or A^-T b when trans) for matrix blockIdx.x of a stack of n x n column-major
// factorizations, n <= kSmallSolveMax, k right-hand-side columns (row-major n x k, b and x back
// to back too): a thread per row, the triangles column by column (each column of L or U is
// contiguous in the factors, so a step's reads are coalesced), one barrier per column.
__global__ void __launch_bounds__(kSmallSolveMax) lu_solve_small_kernel(const double* __restrict__ factors,
                                                                        const int64_t* __restrict__ perm, int n,
                                                                        const double* b, int k, double* x, int trans,
                                                                        unsigned* status) {
  extern __shared__ double ysm[];  // n x k
  const int64_t m = blockIdx.x;
  const double* f = factors + m * n * n;
  const int64_t* p = perm + m * n;
  const double* bm = b + m * n * k;
  double* xm = x + m * n * k;
  const int i = threadIdx.x;
  if (i < n) {
    const int64_t src = trans ? i : p[i];
    const bool ok = src >= 0 && src < n;
    if (!ok) flag_error(status, RM_DEV_BAD_INDEX);
    for (int c = 0; c < k; ++c) ysm[i * k + c] = ok ? bm[src * k + c] : 0.0;
  }
  __syncthreads();  // b is read in full before x (which may be b) is written
  // item (r, q) of the factored matrix at f[q * n + r]
  if (!trans) {
    for (int q = 0; q < n; ++q) {  // L y = P b, unit lower
      if (i > q && i < n) {
        const double l = f[(int64_t)q * n + i];
        for (int c = 0; c < k; ++c) ysm[i * k + c] = fma(-l, ysm[q * k + c], ysm[i * k + c]);
      }
      __syncthreads();
    }
    for (int q = n - 1; q >= 0; --q) {  // U x = y
      if (i == q)
        for (int c = 0; c < k; ++c) ysm[q * k + c] = ysm[q * k + c] / f[(int64_t)q * n + q];
      __syncthreads();
      if (i < q) {
        const double u = f[(int64_t)q * n + i];
        for (int c = 0; c < k; ++c) ysm[i * k + c] = fma(-u, ysm[q * k + c], ysm[i * k + c]);
      }
      __syncthreads();
    }
    if (i < n)
      for (int c = 0; c < k; ++c) xm[i * k + c] = ysm[i * k + c];
  } else {
    // A^T x = b with P A = L U: U^T z = b (lower), L^T w = z (unit upper), x[perm[r]] = w[r];
    // (U^T)(r, q) = U(q, r) = f[r * n + q]
    for (int q = 0; q < n; ++q) {
      if (i == q)
        for (int c = 0; c < k; ++c) ysm[q * k + c] = ysm[q * k + c] / f[(int64_t)q * n + q];
      __syncthreads();
      if (i > q && i < n) {
        const double u = f[(int64_t)i * n + q];
        for (int c = 0; c < k; ++c) ysm[i * k + c] = fma(-u, ysm[q * k + c], ysm[i * k + c]);
      }
      __syncthreads();
    }
    for (int q = n - 1; q >= 0; --q) {
      if (i < q) {
        const double l = f[(int64_t)i * n + q];
        for (int c = 0; c < k; ++c) ysm[i * k + c] = fma(-l, ysm[q * k + c], ysm[i * k + c]);
      }
      __syncthreads();
    }
    if (i < n) {
      const int64_t dst = p[i];
      if (dst >= 0 && dst < n)
        for (int c = 0; c < k; ++c) xm[dst * k + c] = ysm[i * k + c];
      else
        flag_error(status, RM_DEV_BAD_INDEX);
    }
  }
}

}  // namespace rm

using namespace rm;

extern "C" {

int rm_dlu_inverse(int64_t n, const double* d_factors, const int64_t* d_perm, double* d_out, void* stream) {
  if (n < 0 || (n > 0 && (!d_factors || !d_perm || !d_out))) return RM_BAD_ARG;
  if (n == 0) return RM_OK;
  RM_TRY(check_device());
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  void* scratch = nullptr;
  RM_TRY(scratch_alloc(&scratch, getri_f64_scratch_bytes(n), s));
  const int st = getri_f64(d_factors, n, d_perm, d_out, scratch, device_status(), s);
  scratch_free(scratch, s);
  return st;
}

int rm_dlu_inverse_host(int64_t n, const double* h_factors, const int64_t* h_perm, double* h_out) {
  if (n < 0 || (n > 0 && (!h_factors || !h_perm || !h_out))) return RM_BAD_ARG;
  if (n == 0) return RM_OK;
  RM_TRY(check_device());
  cudaStream_t s;
  RM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  void* buf = nullptr;
  const size_t bytes = (size_t)n * n * 8;
  int st = scratch_alloc(&buf, 2 * bytes + (size_t)n * 8, s);
  if (st == RM_OK) {
    double* df = static_cast<double*>(buf);
    double* dout = df + n * n;
    int64_t* dp = reinterpret_cast<int64_t*>(dout + n * n);
    cudaError_t e = cudaMemcpyAsync(df, h_factors, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dp, h_perm, (size_t)n * 8, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
      set_last_error(e, "copy", __FILE__, __LINE__);
      st = RM_CUDA_ERROR;
    }
    if (st == RM_OK) st = rm_dlu_inverse(n, df, dp, dout, s);
    if (st == RM_OK) {
      e = cudaMemcpyAsync(h_out, dout, bytes, cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) {
        set_last_error(e, "copy", __FILE__, __LINE__);
        st = RM_CUDA_ERROR;
      }
    }
    scratch_free(buf, s);
  }
  if (st == RM_OK) st = take_device_status(s);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  return st;
}

int rm_dlu_determinant(int64_t count, int64_t n, const double* d_factors, const int64_t* d_perm, double* d_det,
                       double* d_sign, double* d_logabs, void* stream) {
  if (count < 0 || n < 0 || (count > 0 && n > 0 && (!d_factors || !d_perm))) return RM_BAD_ARG;
  if (count == 0) return RM_OK;
  RM_TRY(check_device());
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (n == 0) {
    // the empty product: determinant 1, sign 1, log 0 (factor.rs:174-183 fold nothing)
    std::vector<double> one(count, 1.0), zero(count, 0.0);
    if (d_det) RM_CUDA_TRY(cudaMemcpyAsync(d_det, one.data(), count * 8, cudaMemcpyHostToDevice, s));
    if (d_sign) RM_CUDA_TRY(cudaMemcpyAsync(d_sign, one.data(), count * 8, cudaMemcpyHostToDevice, s));
    if (d_logabs) RM_CUDA_TRY(cudaMemcpyAsync(d_logabs, zero.data(), count * 8, cudaMemcpyHostToDevice, s));
    RM_CUDA_TRY(cudaStreamSynchronize(s));
    return RM_OK;
  }
  for (int64_t first = 0; first < count; first += INT32_MAX / 2) {
    const int64_t c = std::min<int64_t>(count - first, INT32_MAX / 2);
    lu_det_kernel<<<(unsigned)c, kDetThreads, 0, s>>>(d_factors + first * n * n, d_perm + first * n, n,
                                                       d_det ? d_det + first : nullptr,
                                                       d_sign ? d_sign + first : nullptr,
                                                       d_logabs ? d_logabs + first : nullptr, device_status());
    RM_LAUNCHED();
  }
  return RM_OK;
}

int rm_dlu_solve_batched(int64_t count, int64_t n, const double* d_factors, const int64_t* d_perm, const double* d_b,
                         int64_t k, double* d_x, int trans, void* stream) {
  if (count < 0 || n < 0 || k < 0 || n > kSmallSolveMax || k > kSmallSolveCols || (trans != 0 && trans != 1))
    return RM_BAD_ARG;
  if (count == 0 || n == 0 || k == 0) return RM_OK;
  if (!d_factors || !d_perm || !d_b || !d_x) return RM_BAD_ARG;
  RM_TRY(check_device());
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const size_t smem = (size_t)n * k * sizeof(double);
  RM_TRY(smem_attribute(lu_solve_small_kernel, (size_t)kSmallSolveMax * kSmallSolveCols * sizeof(double)));
  for (int64_t first = 0; first < count; first += INT32_MAX / 2) {
    const int64_t c = std::min<int64_t>(count - first, INT32_MAX / 2);
    lu_solve_small_kernel<<<(unsigned)c, kSmallSolveMax, smem, s>>>(d_factors + first * n * n, d_perm + first * n,
                                                                     (int)n, d_b + first * n * k, (int)k,
                                                                     d_x + first * n * k, trans, device_status());
    RM_LAUNCHED();
  }
  return RM_OK;
}

}  // extern "C"
