// Products with one output row or column (m == 1 or n == 1): rustymath's by_vector
// (core/src/linalg.rs:1020-1073), which multiplies a matrix by a vector instead of tiling.
// Here they are HBM-bound streams over the matrix, not DMMA tiles (a 64 x 64 tile would use
// one row or column of 64):
//   - rows_dot_kernel: out_i = alpha * <M row i, x> + beta * out_i, a warp per row, lanes along
//     it with 16-byte loads, four independent partial sums per lane, warp shuffle reduction;
//   - col_comb_kernel: out_j = sum_k M[k][j] x_k, a thread per output column (a warp reads 256
//     contiguous bytes of a matrix row per step), the k range split over blockIdx.y so that the
//     grid covers the GPU; each split writes its partial sums, and comb_finish_kernel adds them
//     in split order (deterministic) and applies alpha and beta.
// The C epilogue is the DMMA GEMM's: v = alpha * sum; beta == 0 writes v (C is not read).
// The summation order differs from by_vector's (and from the DMMA tiles'); the results agree
// within the usual k * eps * |A| |x| bound.
#include <algorithm>

#include "rm_internal.h"

namespace rm {

constexpr int kDotThreads = 256;
constexpr int kCombThreads = 256;
constexpr int kCombUnroll = 8;

__device__ __forceinline__ double epilogue(double acc, double alpha, double beta, const double* c) {
  const double v = alpha * acc;
  return beta == 0.0 ? v : fma(beta, *c, v);
}

// out[i * inc_out] for rows i < rows of M (row-major, ld ldm, k items per row); x contiguous
template <bool VEC>
__global__ void __launch_bounds__(kDotThreads) rows_dot_kernel(const double* __restrict__ mat, int64_t ldm, int64_t rows,
                                                              int64_t k, const double* __restrict__ x, double alpha,
                                                              double beta, double* __restrict__ out, int64_t inc_out) {
  griddep_launch_dependents();
  griddep_wait();  // the kernel before this one in the stream has completed
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (kDotThreads / 32);
  for (int64_t i = blockIdx.x * (int64_t)(kDotThreads / 32) + (threadIdx.x >> 5); i < rows; i += warps) {
    const double* row = mat + i * ldm;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    if constexpr (VEC) {
      // 16-byte loads: lane l takes items 2l, 2l+1 of each 64-item chunk; four chunks in flight
      const int64_t k2 = k / 2;
      const double2* r2 = reinterpret_cast<const double2*>(row);
      const double2* x2 = reinterpret_cast<const double2*>(x);
      int64_t q = lane;
      for (; q + 96 < k2; q += 128) {
        const double2 a0 = __ldcs(r2 + q), a1 = __ldcs(r2 + q + 32), a2 = __ldcs(r2 + q + 64), a3 = __ldcs(r2 + q + 96);
        const double2 b0 = x2[q], b1 = x2[q + 32], b2 = x2[q + 64], b3 = x2[q + 96];
        s0 = fma(a0.x, b0.x, s0), s1 = fma(a0.y, b0.y, s1);
        s2 = fma(a1.x, b1.x, s2), s3 = fma(a1.y, b1.y, s3);
        s0 = fma(a2.x, b2.x, s0), s1 = fma(a2.y, b2.y, s1);
        s2 = fma(a3.x, b3.x, s2), s3 = fma(a3.y, b3.y, s3);
      }
      for (; q < k2; q += 32) {
        const double2 a0 = __ldcs(r2 + q), b0 = x2[q];
        s0 = fma(a0.x, b0.x, s0), s1 = fma(a0.y, b0.y, s1);
      }
      if ((k & 1) && lane == 0) s2 = fma(row[k - 1], x[k - 1], s2);
    } else {
      int64_t q = lane;
      for (; q + 96 < k; q += 128) {
        s0 = fma(__ldcs(row + q), x[q], s0);
        s1 = fma(__ldcs(row + q + 32), x[q + 32], s1);
        s2 = fma(__ldcs(row + q + 64), x[q + 64], s2);
        s3 = fma(__ldcs(row + q + 96), x[q + 96], s3);
      }
      for (; q < k; q += 32) s0 = fma(__ldcs(row + q), x[q], s0);
    }
    double s = (s0 + s1) + (s2 + s3);
#pragma unroll
    for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) {
      double* o = out + i * inc_out;
      *o = epilogue(s, alpha, beta, o);
    }
  }
}

// Partial sums over k in [y * kchunk, (y + 1) * kchunk) of M[k][j] x_k (M row-major, ld ldm)
// for columns j < cols: into part[y * cols + j], or, with a single split, the finished result
// into out[j * inc_out]
__global__ void __launch_bounds__(kCombThreads) col_comb_kernel(const double* __restrict__ mat, int64_t ldm, int64_t cols,
                                                               int64_t k, int64_t kchunk, const double* __restrict__ x,
                                                               double* __restrict__ part, double alpha, double beta,
                                                               double* __restrict__ out, int64_t inc_out) {
  griddep_launch_dependents();
  griddep_wait();  // the kernel before this one in the stream has completed
  const int64_t j = blockIdx.x * (int64_t)kCombThreads + threadIdx.x;
  const int64_t k0 = blockIdx.y * kchunk, k1 = std::min(k, k0 + kchunk);
  if (j >= cols) return;
  const double* col = mat + j;
  double s[kCombUnroll];
#pragma unroll
  for (int u = 0; u < kCombUnroll; ++u) s[u] = 0.0;
  int64_t q = k0;
  for (; q + kCombUnroll <= k1; q += kCombUnroll) {
    double v[kCombUnroll];
#pragma unroll
    for (int u = 0; u < kCombUnroll; ++u) v[u] = __ldcs(col + (q + u) * ldm);
#pragma unroll
    for (int u = 0; u < kCombUnroll; ++u) s[u] = fma(v[u], x[q + u], s[u]);
  }
  for (; q < k1; ++q) s[0] = fma(__ldcs(col + q * ldm), x[q], s[0]);
  double acc = 0.0;
#pragma unroll
  for (int u = 0; u < kCombUnroll; ++u) acc += s[u];
  if (gridDim.y == 1) {
    double* o = out + j * inc_out;
    *o = epilogue(acc, alpha, beta, o);
  } else {
    part[blockIdx.y * cols + j] = acc;
  }
}

__global__ void comb_finish_kernel(const double* __restrict__ part, int64_t cols, int splits, double alpha, double beta,
                                   double* __restrict__ out, int64_t inc_out) {
  griddep_launch_dependents();
  griddep_wait();
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < cols; j += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int y = 0; y < splits; ++y) acc += part[y * cols + j];
    double* o = out + j * inc_out;
    *o = epilogue(acc, alpha, beta, o);
  }
}

__global__ void gather_vector_kernel(const double* __restrict__ src, int64_t inc, int64_t k, double* __restrict__ dst) {
  griddep_launch_dependents();
  griddep_wait();
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < k; q += (int64_t)gridDim.x * blockDim.x)
    dst[q] = src[q * inc];
}

static int launch_rows_dot(const double* mat, int64_t ldm, int64_t rows, int64_t k, const double* x, double alpha,
                           double beta, double* out, int64_t inc_out, cudaStream_t s) {
  const int64_t per_cta = kDotThreads / 32;
  const int grid = (int)std::min<int64_t>((rows + per_cta - 1) / per_cta, 8 * (int64_t)device_sm_count());
  const bool vec = (ldm % 2 == 0) && ((reinterpret_cast<uintptr_t>(mat) & 15) == 0) &&
                   ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
  if (vec)
    RM_CUDA_TRY(launch_dependent(rows_dot_kernel<true>, dim3(grid), dim3(kDotThreads), 0, s, mat, ldm, rows, k, x, alpha,
                                 beta, out, inc_out));
  else
    RM_CUDA_TRY(launch_dependent(rows_dot_kernel<false>, dim3(grid), dim3(kDotThreads), 0, s, mat, ldm, rows, k, x,
                                 alpha, beta, out, inc_out));
  note_launch();
  return RM_OK;
}

static int launch_col_comb(const double* mat, int64_t ldm, int64_t cols, int64_t k, const double* x, double alpha,
                           double beta, double* out, int64_t inc_out, double* part, int splits, int64_t kchunk,
                           cudaStream_t s) {
  const int64_t gx = (cols + kCombThreads - 1) / kCombThreads;
  RM_CUDA_TRY(launch_dependent(col_comb_kernel, dim3((unsigned)gx, (unsigned)splits), dim3(kCombThreads), 0, s, mat,
                               ldm, cols, k, kchunk, x, part, alpha, beta, out, inc_out));
  note_launch();
  if (splits > 1) {
    const int grid = (int)std::min<int64_t>((cols + 255) / 256, 4 * (int64_t)device_sm_count());
    RM_CUDA_TRY(launch_dependent(comb_finish_kernel, dim3(grid), dim3(256), 0, s, (const double*)part, cols, splits,
                                 alpha, beta, out, inc_out));
    note_launch();
  }
  return RM_OK;
}

// C = alpha op(A) op(B) + beta C (row-major) for m == 1 or n == 1, k >= 1, alpha != 0
int gemv_device(bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* a, int64_t lda,
                const double* b, int64_t ldb, double beta, double* c, int64_t ldc, cudaStream_t s) {
  // the matrix operand, its vector, and the output's stride
  const bool col_out = n == 1;  // C is a column (stride ldc); else a row (stride 1)
  const double* mat;
  int64_t ldm, outs = col_out ? m : n;
  const double* vec;
  int64_t incv;
  bool dot;  // the outputs are dots of the matrix's stored rows
  if (col_out) {
    mat = a, ldm = lda, dot = !ta;  // op(A)[i][q] = A[i][q] or A[q][i]
    vec = b, incv = tb ? 1 : ldb;   // op(B)[q][0] = B[0][q] or B[q][0]
  } else {
    mat = b, ldm = ldb, dot = tb;  // op(B)[q][j] = B[j][q] or B[q][j]
    vec = a, incv = ta ? lda : 1;  // op(A)[0][q] = A[q][0] or A[0][q]
  }
  const int64_t inc_out = col_out ? ldc : 1;
  // split the k range of the column form so that the grid covers the GPU
  int splits = 1;
  int64_t kchunk = k;
  if (!dot) {
    const int64_t gx = (outs + kCombThreads - 1) / kCombThreads;
    const int64_t want = std::max<int64_t>(1, (4 * (int64_t)device_sm_count() + gx - 1) / gx);
    splits = (int)std::min<int64_t>({want, (k + 255) / 256, 1024});
    kchunk = (k + splits - 1) / splits;
    splits = (int)((k + kchunk - 1) / kchunk);
  }
  // a strided (or, for the dot form, unaligned) vector is gathered first; scratch is
  // stream-ordered, freed behind the launches
  const bool gather = incv != 1 || (dot && (reinterpret_cast<uintptr_t>(vec) & 15));
  const size_t xbytes = gather ? ((size_t)k * sizeof(double) + 255) / 256 * 256 : 0;
  const size_t pbytes = splits > 1 ? (size_t)splits * outs * sizeof(double) : 0;
  void* scratch = nullptr;
  if (xbytes + pbytes) RM_TRY(scratch_alloc(&scratch, xbytes + pbytes, s));
  double* part = pbytes ? reinterpret_cast<double*>(static_cast<char*>(scratch) + xbytes) : nullptr;
  int st = RM_OK;
  if (gather) {
    double* xg = static_cast<double*>(scratch);
    const int grid = (int)std::min<int64_t>((k + 255) / 256, 4 * (int64_t)device_sm_count());
    const cudaError_t e = launch_dependent(gather_vector_kernel, dim3(grid), dim3(256), 0, s, vec, incv, k, xg);
    if (e != cudaSuccess) {
      set_last_error(e, "gather_vector_kernel", __FILE__, __LINE__);
      st = RM_CUDA_ERROR;
    }
    note_launch();
    vec = xg;
  }
  if (st == RM_OK)
    st = dot ? launch_rows_dot(mat, ldm, outs, k, vec, alpha, beta, c, inc_out, s)
             : launch_col_comb(mat, ldm, outs, k, vec, alpha, beta, c, inc_out, part, splits, kchunk, s);
  scratch_free(scratch, s);
  return st;
}

}  // namespace rm
