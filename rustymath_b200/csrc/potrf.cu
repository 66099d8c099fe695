// Cholesky factorization: L L^T = A for a symmetric positive definite A, from its lower triangle.
//
// Replaces rustymath's cholesky (core/src/linalg/factor.rs:267, cholesky_factor 776-795,
// cholesky_panel 750-773) and its stack form (src/linalg/stacked.rs:259-268). The reference
// factors blocks of cholesky_block(n) columns by recursive halving down to 16-column leaves,
// then updates the rest with `gram` (the lower triangle of C - X X^T). Here, on a row-major
// working copy W (ld a multiple of 32):
//   - each 64-column diagonal block is factored column by column in one CTA's shared memory
//     (sqrt of the pivot, the column below divided by it the way rustymath's `divide` does, the
//     later columns of the block reduced by FMAs in column order), and the same CTA inverts L11;
//   - the rows below it become L21 = A21 L11^-T through one float64 tensor-core GEMM (dgemm.cu);
//   - the trailing matrix takes A22 -= L21 L21^T through another (the whole square is formed;
//     only its lower triangle is read again).
// A pivot that is not > 0 (NaN included) marks the matrix not positive definite, as rustymath's
// None; later blocks then work on whatever is left and their results are not used.
// Stacks of small matrices (n <= 128) factor one matrix per CTA, entirely in shared memory, in
// one launch; a matrix that is not positive definite gives NaN everywhere, as rustymath's stacks.
#include <cfloat>

#include "rm_internal.h"

namespace rm {

constexpr int kPotrfBlock = 64;   // columns of a diagonal block
constexpr int kPotrfThreads = 256;
constexpr int kCholSmallMax = 128;  // largest n of the one-CTA stack form

// rustymath's divide: multiply by the reciprocal unless the divisor is subnormal
__device__ __forceinline__ double chol_divide(double x, double d) { return fabs(d) >= DBL_MIN ? x * (1.0 / d) : x / d; }

// Factors the nb x nb lower triangle held in shared memory S (row stride lds) in place, column by
// column; the upper triangle is not touched. Returns false (in every thread) when a pivot is
// not > 0.
__device__ bool chol_in_smem(double* S, int lds, int nb) {
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int c = 0; c < nb; ++c) {
    const double d0 = S[c * lds + c];
    if (!(d0 > 0.0)) {  // every thread reads the same value and leaves together
      if (threadIdx.x == 0) bad = 1;
      break;
    }
    const double d = sqrt(d0);
    for (int i = c + 1 + threadIdx.x; i < nb; i += blockDim.x) S[i * lds + c] = chol_divide(S[i * lds + c], d);
    __syncthreads();
    if (threadIdx.x == 0) S[c * lds + c] = d;
    // the block's later columns lose column c, row by row from their diagonal down
    const int m = nb - c - 1;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int i = c + 1 + e / m, j = c + 1 + e % m;
      if (j <= i) S[i * lds + j] = fma(S[i * lds + c], -S[j * lds + c], S[i * lds + j]);
    }
    __syncthreads();
  }
  __syncthreads();
  return bad == 0;
}

// One diagonal block of the blocked factorization: the nb x nb block at w (row stride ld) is
// factored in shared memory and written back (lower triangle), and its inverse L11^-1 goes to
// linv (row-major kPotrfBlock x kPotrfBlock, zeros above the diagonal and past nb). A block
// that is not positive definite sets *notpd.
__global__ void __launch_bounds__(kPotrfThreads) potrf_diag_kernel(double* __restrict__ w, int64_t ld, int nb,
                                                                   double* __restrict__ linv, int* notpd) {
  extern __shared__ double psm[];
  constexpr int LDS = kPotrfBlock + 1;
  double* S = psm;
  double* X = psm + kPotrfBlock * LDS;
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e / nb, j = e % nb;
    S[i * LDS + j] = j <= i ? w[(int64_t)i * ld + j] : 0.0;
  }
  __syncthreads();
  const bool ok = chol_in_smem(S, LDS, nb);
  if (!ok) {
    if (threadIdx.x == 0) atomicExch(notpd, 1);
    return;
  }
  // column c of L11^-1: X[i][c] = -(sum_{c<=q<i} L[i][q] X[q][c]) / L[i][i], X[c][c] = 1 / L[c][c]
  const int c = threadIdx.x;
  if (c < kPotrfBlock) {
    for (int i = 0; i < kPotrfBlock; ++i) {
      double v = 0.0;
      if (c < nb && i < nb && i >= c) {
        double s = i == c ? 1.0 : 0.0;
        for (int q = c; q < i; ++q) s = fma(-S[i * LDS + q], X[q * LDS + c], s);
        v = s / S[i * LDS + i];
      }
      X[i * LDS + c] = v;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e / nb, j = e % nb;
    if (j <= i) w[(int64_t)i * ld + j] = S[i * LDS + j];
  }
  for (int e = threadIdx.x; e < kPotrfBlock * kPotrfBlock; e += blockDim.x) {
    const int i = e / kPotrfBlock, j = e % kPotrfBlock;
    linv[e] = X[i * LDS + j];
  }
}

// L (row-major n x n, zeros above the diagonal) from W's lower triangle.
__global__ void chol_store_kernel(const double* __restrict__ w, int64_t ld, int64_t n, double* __restrict__ l) {
  const int64_t total = n * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / n, j = e - i * n;
    l[e] = j <= i ? w[i * ld + j] : 0.0;
  }
}

// W (ld) = the lower triangle of the row-major n x n a; the rest of W is zero.
__global__ void chol_load_kernel(const double* __restrict__ a, int64_t n, double* __restrict__ w, int64_t ld) {
  const int64_t total = n * ld;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / ld, j = e - i * ld;
    w[e] = (j < n && j <= i) ? a[i * n + j] : 0.0;
  }
}

// A stack of count matrices of order n <= kCholSmallMax, one per CTA in shared memory: L with
// zeros above the diagonal, or NaN everywhere where the matrix is not positive definite.
__global__ void __launch_bounds__(kPotrfThreads) chol_small_kernel(const double* __restrict__ a, int n,
                                                                   double* __restrict__ l, int32_t* ok) {
  extern __shared__ double psm[];
  const int lds = n + 1;
  const int64_t base = (int64_t)blockIdx.x * n * n;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    psm[i * lds + j] = j <= i ? a[base + e] : 0.0;
  }
  __syncthreads();
  const bool good = chol_in_smem(psm, lds, n);
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e / n, j = e % n;
    l[base + e] = good ? (j <= i ? psm[i * lds + j] : 0.0) : __longlong_as_double(0x7ff8000000000000ll);
  }
  if (ok && threadIdx.x == 0) ok[blockIdx.x] = good ? 1 : 0;
}

size_t potrf_f64_scratch_bytes(int64_t n) {
  const int64_t ld = round_up(std::max<int64_t>(n, 1), 32);
  return ((size_t)n * ld * 8 + 255) / 256 * 256                    // W
         + (size_t)kPotrfBlock * kPotrfBlock * 8                   // L11^-1
         + ((size_t)n * kPotrfBlock * 8 + 255) / 256 * 256 + 256;  // L21 before it goes back, the flag
}

int potrf_f64(const double* a, int64_t n, double* l, void* scratch, int* notpd_host, unsigned* status,
              cudaStream_t stream) {
  if (n == 0) return RM_OK;
  const int64_t ld = round_up(n, 32);
  char* base = static_cast<char*>(scratch);
  double* w = reinterpret_cast<double*>(base);
  double* linv = reinterpret_cast<double*>(base + ((size_t)n * ld * 8 + 255) / 256 * 256);
  double* t = linv + kPotrfBlock * kPotrfBlock;
  int* flag = reinterpret_cast<int*>(reinterpret_cast<char*>(t) + ((size_t)n * kPotrfBlock * 8 + 255) / 256 * 256);
  const int blocks = (int)std::min<int64_t>((n * ld + 255) / 256, 8 * device_sm_count());
  RM_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), stream));
  chol_load_kernel<<<blocks, 256, 0, stream>>>(a, n, w, ld);
  RM_LAUNCHED();
  const size_t smem = (size_t)2 * kPotrfBlock * (kPotrfBlock + 1) * sizeof(double);
  RM_TRY(smem_attribute(potrf_diag_kernel, smem));
  for (int64_t k0 = 0; k0 < n; k0 += kPotrfBlock) {
    const int nb = (int)std::min<int64_t>(kPotrfBlock, n - k0);
    const int64_t rest = n - k0 - nb;
    double* a11 = w + k0 * ld + k0;
    potrf_diag_kernel<<<1, kPotrfThreads, smem, stream>>>(a11, ld, nb, linv, flag);
    RM_LAUNCHED();
    if (rest == 0) break;
    double* a21 = a11 + (int64_t)nb * ld;
    // L21 = A21 L11^-T into t, then back into W
    RM_TRY(dgemm_device(false, true, rest, nb, nb, 1.0, a21, ld, linv, kPotrfBlock, 0.0, t, kPotrfBlock, status,
                        stream));
    RM_CUDA_TRY(cudaMemcpy2DAsync(a21, ld * 8, t, kPotrfBlock * 8, (size_t)nb * 8, rest, cudaMemcpyDeviceToDevice,
                                  stream));
    // A22 -= L21 L21^T
    RM_TRY(dgemm_device(false, true, rest, rest, nb, -1.0, a21, ld, a21, ld, 1.0, a21 + nb, ld, status, stream));
  }
  if (notpd_host) RM_CUDA_TRY(cudaMemcpyAsync(notpd_host, flag, sizeof(int), cudaMemcpyDeviceToHost, stream));
  chol_store_kernel<<<(int)std::min<int64_t>((n * n + 255) / 256, 8 * device_sm_count()), 256, 0, stream>>>(w, ld, n,
                                                                                                          l);
  RM_LAUNCHED();
  return RM_OK;
}

int cholesky_small_batched(int64_t count, int64_t n, const double* a, double* l, int32_t* ok, cudaStream_t stream) {
  if (count == 0 || n == 0) return RM_OK;
  const size_t smem = (size_t)n * (n + 1) * sizeof(double);
  RM_TRY(smem_attribute(chol_small_kernel, (size_t)kCholSmallMax * (kCholSmallMax + 1) * sizeof(double)));
  for (int64_t first = 0; first < count; first += INT32_MAX / 2) {
    const int64_t c = std::min<int64_t>(count - first, INT32_MAX / 2);
    chol_small_kernel<<<(unsigned)c, kPotrfThreads, smem, stream>>>(a + first * n * n, (int)n, l + first * n * n,
                                                                    ok ? ok + first : nullptr);
    RM_LAUNCHED();
  }
  return RM_OK;
}

}  // namespace rm

using namespace rm;

extern "C" {

int rm_dcholesky(int64_t n, const double* d_a, double* d_l, void* stream) {
  if (n < 0 || (n > 0 && (!d_a || !d_l))) return RM_BAD_ARG;
  if (n == 0) return RM_OK;
  RM_TRY(check_device());
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  void* scratch = nullptr;
  RM_TRY(scratch_alloc(&scratch, potrf_f64_scratch_bytes(n), s));
  int notpd = 0;
  const int st = potrf_f64(d_a, n, d_l, scratch, &notpd, device_status(), s);
  scratch_free(scratch, s);
  if (st != RM_OK) return st;
  RM_TRY(take_device_status(s));  // synchronises: notpd is in host memory now
  if (notpd) {
    set_last_message("a pivot is not > 0: the matrix is not positive definite");
    return RM_NOT_POSITIVE_DEFINITE;
  }
  return RM_OK;
}

int rm_dcholesky_host(int64_t n, const double* h_a, double* h_l) {
  if (n < 0 || (n > 0 && (!h_a || !h_l))) return RM_BAD_ARG;
  if (n == 0) return RM_OK;
  RM_TRY(check_device());
  cudaStream_t s;
  RM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  void* buf = nullptr;
  const size_t bytes = (size_t)n * n * 8;
  int st = scratch_alloc(&buf, 2 * bytes, s);
  if (st == RM_OK) {
    double* da = static_cast<double*>(buf);
    double* dl = da + n * n;
    cudaError_t e = cudaMemcpyAsync(da, h_a, bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
      set_last_error(e, "copy", __FILE__, __LINE__);
      st = RM_CUDA_ERROR;
    }
    if (st == RM_OK) st = rm_dcholesky(n, da, dl, s);
    if (st == RM_OK || st == RM_NOT_POSITIVE_DEFINITE) {
      e = cudaMemcpyAsync(h_l, dl, bytes, cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) {
        set_last_error(e, "copy", __FILE__, __LINE__);
        st = RM_CUDA_ERROR;
      }
    }
    scratch_free(buf, s);
  }
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  return st;
}

int rm_dcholesky_batched(int64_t count, int64_t n, const double* d_a, double* d_l, int32_t* d_ok, void* stream) {
  if (count < 0 || n < 0 || n > kCholSmallMax || ((count > 0 && n > 0) && (!d_a || !d_l))) return RM_BAD_ARG;
  if (count == 0 || n == 0) return RM_OK;
  RM_TRY(check_device());
  return cholesky_small_batched(count, n, d_a, d_l, d_ok, reinterpret_cast<cudaStream_t>(stream));
}

int rm_dcholesky_solve(int64_t n, const double* d_l, const double* d_b, int64_t k, double* d_x, void* stream) {
  if (n < 0 || k < 0 || ((n > 0 && k > 0) && (!d_l || !d_b || !d_x))) return RM_BAD_ARG;
  if (n == 0 || k == 0) return RM_OK;
  RM_TRY(check_device());
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (d_x != d_b) RM_CUDA_TRY(cudaMemcpyAsync(d_x, d_b, (size_t)n * k * 8, cudaMemcpyDeviceToDevice, s));
  // L y = b, then L^T x = y, in place
  RM_TRY(rm_dtrsm(RM_LEFT, RM_LOWER, RM_CBLAS_NO_TRANS, RM_NON_UNIT, n, k, d_l, n, d_x, k, stream));
  return rm_dtrsm(RM_LEFT, RM_LOWER, RM_CBLAS_TRANS, RM_NON_UNIT, n, k, d_l, n, d_x, k, stream);
}

}  // extern "C"
