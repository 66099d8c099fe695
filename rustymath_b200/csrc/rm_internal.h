// Internal interfaces between the CUDA translation units of librm_cuda.so.
#pragma once
#include <algorithm>
#include <cstdint>

#include "rm_common.cuh"

namespace rm {

// ---------------------------------------------------------------- GEMM (dgemm.cu)
// C = alpha*op(A)*op(B) + beta*C, row-major; a, b 16-byte aligned with even lda, ldb.
// `force_wide_m` picks the 128-row tile whatever the size, which makes a product whose
// m <= 128 read each column block of B in one CTA (so B may alias C).
int dgemm_device(bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* a, int64_t lda,
                 const double* b, int64_t ldb, double beta, double* c, int64_t ldc, unsigned* status,
                 cudaStream_t stream, bool force_wide_m = false);
int scale_device(double* c, int64_t ldc, int64_t m, int64_t n, double beta, cudaStream_t stream);
// C = alpha op(A) op(B) + beta C for m == 1 or n == 1 (k >= 1, alpha != 0): streams over the
// matrix operand instead of DMMA tiles (gemv.cu)
int gemv_device(bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* a, int64_t lda,
                const double* b, int64_t ldb, double beta, double* c, int64_t ldc, cudaStream_t stream);

// ---------------------------------------------------------------- FP32 tensor-core GEMM (sgemm_tc.cu)
// C = alpha A B^T + beta C in float32 on tcgen05: A m x k and B n x k row-major (k
// contiguous), lda, ldb % 4 == 0, 16-byte bases; C row-major, and when ct is not NULL its
// transpose goes to ct (ldct) too. passes 1: TF32 inputs; passes 3: float32-level products.
// max_ctas > 0 caps the persistent grid (to leave SMs to a kernel on another stream).
int sgemm_tc(int passes, int64_t m, int64_t n, int64_t k, float alpha, const float* a, int64_t lda, const float* b,
             int64_t ldb, float beta, float* c, int64_t ldc, unsigned* status, cudaStream_t stream,
             float* ct = nullptr, int64_t ldct = 0, int max_ctas = 0);
// Two products C = alpha A B^T + beta C with the same n, k, alpha and beta in one persistent
// launch (the first's output tiles first); a product with m == 0 is skipped.
struct SgemmOperands {
  int64_t m;
  const float* a;
  int64_t lda;
  const float* b;
  int64_t ldb;
  float* c;
  int64_t ldc;
  float* ct;  // optional transposed copy of C (beta == 0 only through the TMA epilogue)
  int64_t ldct;
};
int sgemm_tc_pair(int passes, const SgemmOperands& x, const SgemmOperands& y, int64_t n, int64_t k, float alpha,
                  float beta, unsigned* status, cudaStream_t stream, int max_ctas = 0);
// Three-pass C = alpha A B^T + beta C with the low parts of A and B (x - trunc_tf32(x), from
// split_lo_f32) given in global memory, loaded beside A and B instead of formed per tile.
int sgemm_tc_lo(int64_t m, int64_t n, int64_t k, float alpha, const float* a, int64_t lda, const float* a_lo,
                int64_t ldal, const float* b, int64_t ldb, const float* b_lo, int64_t ldbl, float beta, float* c,
                int64_t ldc, unsigned* status, cudaStream_t stream, int max_ctas = 0);
int transpose_f32(const float* src, int64_t lds, int64_t m, int64_t n, float* dst, int64_t ldd, cudaStream_t stream);
int scale_f32(float* c, int64_t ldc, int64_t m, int64_t n, float beta, cudaStream_t stream);
int split_lo_f32(const float* x, int64_t ldx, int64_t m, int64_t k, float* lo, int64_t ldl, cudaStream_t stream);

// ---------------------------------------------------------------- LU (getrf.cu)
// Row-major working matrix W (n rows, ldw >= n, ldw % 32 == 0, 16-byte aligned). On return
// W holds L\U of P*A row by row, ipiv[c] is the row swapped with row c (absolute) and
// perm[i] the source row of row i. `scratch` holds getrf_f64_scratch_bytes(n) bytes.
size_t getrf_f64_scratch_bytes(int64_t n);
int getrf_f64(double* w, int64_t ldw, int64_t n, int64_t* ipiv, int64_t* perm, void* scratch, unsigned* status,
              cudaStream_t stream);

// Copies the row-major n x n `a` (lda) into W (ldw), zeroing W's padding columns, and
// records max |a_ij| (NaN ignored) into *amax (device).
int load_matrix_f64(const double* a, int64_t lda, double* w, int64_t ldw, int64_t n, double* amax,
                    cudaStream_t stream);
// Writes the column-major factors (item (i,j) at f[j*n+i]) from the row-major W.
int store_factors_f64(const double* w, int64_t ldw, int64_t n, double* factors, cudaStream_t stream);
// x = (P^T L U)^-1 b for n <= 256 and k <= 8 in one CTA, in rustymath's single-column order, from
// W after getrf_f64 (row-major) or from rustymath's column-major factors (colmajor, ld = ldw);
// b, x row-major n x k (ld k). A row position outside 0..n-1 sets RM_DEV_BAD_INDEX in *status
// (when not NULL). small_solve_fits: the sizes the solves send there (n <= 192, where it is the
// faster route).
bool small_solve_fits(int64_t n, int64_t k);
int small_solve_f64(const double* w, int64_t ldw, bool colmajor, int64_t n, const int64_t* perm, const double* b,
                    int64_t k, double* x, unsigned* status, cudaStream_t stream);
// *flag = 1 when every |u_ii| > eps*n*amax (LuWork::regular), else 0.
int regular_flag_f64(const double* w, int64_t ldw, int64_t n, const double* amax, int32_t* flag,
                     cudaStream_t stream);

// ---------------------------------------------------------------- solves (getrs.cu)
constexpr int kSolveBlock = 64;  // rows of a block row of the triangular solves
constexpr int kSolveCols = 16;   // right-hand-side columns per solve launch
// Per block row of a triangular solve: the inverses of its two diagonal blocks (L, U) and
// the two couplings to the block solved just before it (inverse x off-diagonal block).
constexpr int kDiagMats = 4;
constexpr size_t diag_blocks_bytes_max(int64_t n) {
  return (size_t)((n + kSolveBlock - 1) / kSolveBlock) * kDiagMats * kSolveBlock * kSolveBlock * sizeof(double);
}
constexpr size_t getrs_scratch_bytes_max(int64_t n, int64_t k) {
  return ((size_t)n * k * sizeof(double) + 255) / 256 * 256 +
         (size_t)(2 * ((n + kSolveBlock - 1) / kSolveBlock + 1)) * sizeof(int) *
             (size_t)((k + kSolveCols - 1) / kSolveCols) +
         256;
}
size_t getrs_f64_scratch_bytes(int64_t n, int64_t k);
// x = (P^T L U)^-1 b, or (P^T L U)^-T b when trans, from L\U held row-major in lu (as W
// after getrf_f64; lu_colmajor false) or column-major (rustymath's factors; lu_colmajor
// true), with leading dimension ld. b, x row-major n x k (may alias). `dinv` holds the
// inverted diagonal blocks from invert_diag_blocks_f64 with the arguments that
// diag_block_args gives for the same (trans, lu_colmajor).
int getrs_f64(const double* lu, int64_t ld, bool lu_colmajor, int64_t n, const int64_t* perm, const double* dinv,
              const double* b, int64_t ldb, int64_t k, double* x, int64_t ldx, void* scratch, unsigned* status,
              cudaStream_t stream, bool trans = false);
size_t diag_blocks_f64_bytes(int64_t n);
// One float64 block-chained triangular solve (a CTA per kSolveBlock-row block) of kc <= kSolveCols
// columns of x in place: the lower or upper triangle of T, T(i, j) at w[i*ldw + j] (w[j*ldw + i]
// when colmajor), with the diagonal-block inverses of invert_diag_blocks_f64; flags[nblk] and
// *counter zero on entry.
int trsv_chain_f64(bool lower, bool colmajor, const double* w, int64_t ldw, int n, const double* dinv, double* x,
                   int64_t ldx, int kc, int* flags, int* counter, unsigned* status, cudaStream_t stream);
// Inverts the diagonal blocks of the lower and upper triangles of T, T(i,j) = w[i*ldw+j]
// (w[j*ldw+i] when colmajor), a unit triangle's diagonal taken as 1.
int invert_diag_blocks_f64(const double* w, int64_t ldw, bool colmajor, int64_t n, double* dinv, bool lower_unit,
                           bool upper_unit, cudaStream_t stream);
struct DiagBlockArgs {
  bool colmajor, lower_unit, upper_unit;
};
inline DiagBlockArgs diag_block_args(bool trans, bool lu_colmajor) {
  return {trans ? !lu_colmajor : lu_colmajor, !trans, trans};
}

// ---------------------------------------------------------------- residual (residual.cu)
// r = b - A x (FP64). When norms is not NULL (residual_norms_bytes(k) bytes) it also gathers
// ||A||_inf and the columns' ||r||_inf and ||b||_inf, which backward_error_f64 completes.
size_t residual_norms_bytes(int64_t k);
int residual_f64(const double* a, int64_t lda, int64_t n, const double* x, int64_t ldx, const double* b, int64_t ldb,
                 int64_t k, double* r, int64_t ldr, double* norms, cudaStream_t stream);
// After residual_f64 filled norms: out[0] = normwise backward error (max over columns of
// ||r_c|| / (||A|| ||x_c|| + ||b_c||)), out[1] = ||A||_inf.
int backward_error_f64(const double* x, int64_t ldx, int64_t n, int64_t k, double* norms, double* out,
                       cudaStream_t stream);

// dst[j*ldd + i] = src[i*lds + j] for an m x n row-major src.
int transpose_f64(const double* src, int64_t lds, int64_t m, int64_t n, double* dst, int64_t ldd, cudaStream_t stream);

// The device-wide sticky status word (RM_DEV_* bits) of the current device.
unsigned* device_status();
// Reads and clears the current device's status word (synchronises `stream`); maps bits to
// an rm status code.
int take_device_status(cudaStream_t stream);
int check_device();
size_t trsm_f64_scratch_bytes(int64_t order, int64_t m, int64_t n, bool right);
int trsm_f64(bool right, bool lower, bool trans, bool unit, int64_t m, int64_t n, const double* a, int64_t lda,
             double* x, int64_t ldx, void* scratch, unsigned* status, cudaStream_t stream);
size_t ozaki_scratch_bytes(int64_t m, int64_t n, int64_t k, int s);
int dgemm_ozaki(int64_t m, int64_t n, int64_t k, const double* a, int64_t lda, const double* b, int64_t ldb,
                double* c, int64_t ldc, int s, void* scratch, unsigned* status, cudaStream_t stream);  // RM_NO_DEVICE without a compute capability 10.x GPU

// ---------------------------------------------------------------- mixed precision (mixed.cu)
size_t getrf_lpp_f32_scratch_bytes(int64_t n);
// float32 LU of the row-major n x n a (lda % 4 == 0) with each 128-column panel pivoted among
// its own 256 rows; perm[i] (int32) = the row of the input that row i of L U comes from.
// dinv (optional): the diagonal blocks' inverses L11^-1, U11^-1 of each 128-column panel go to
// its slots [b][0], [b][1] of the triangular solves' table (kDiagMats matrices of 128^2 per block)
int getrf_lpp_f32(float* a, int64_t lda, int64_t n, int* perm, void* scratch, unsigned* status, cudaStream_t stream,
                  float* dinv = nullptr);
int to_f32(const double* a, int64_t lda, int64_t n, float* f, int64_t ldf, cudaStream_t stream);
// c (float32) = r[perm]; x (float64) = c or x += c.
int gather_f32(const double* r, int64_t ldr, const int* perm, int64_t n, int64_t k, float* c, int64_t ldc,
               cudaStream_t stream);
int accumulate_f64(const float* c, int64_t ldc, int64_t n, int64_t k, double* x, int64_t ldx, bool assign,
                   cudaStream_t stream);
// float32 triangular solves of an unpivoted row-major L\U (getrs.cu)
size_t diag_blocks_f32_bytes(int64_t n);
int invert_diag_blocks_f32(const float* w, int64_t ldw, int64_t n, float* dinv, cudaStream_t stream);
// Entries [2] and [3] of the float32 table (the couplings to the block before), from entries [0]
// and [1], which the factorization's panels wrote
int couplings_f32(const float* w, int64_t ldw, int64_t n, float* dinv, cudaStream_t stream);
size_t trsv_f32_scratch_bytes(int64_t n, int64_t k);
int64_t premultiplied_f32_ld(int64_t n);
size_t premultiplied_f32_bytes(int64_t n);
int premultiply_f32(const float* lu, int64_t ld, int64_t n, const float* dinv, float* pre, cudaStream_t stream);
int lu_solve_f32_nopiv(const float* lu, int64_t ld, int64_t n, const float* dinv, const float* pre, float* x,
                       int64_t ldx, int64_t k, void* scratch, unsigned* status, cudaStream_t stream);

// z = (LU)^-1 P y in float64 through the float32 factors of the mixed solve (y may be z)
struct Precond {
  const float* f;
  int64_t ldf, n;
  const int* perm;
  const float* dinv;
  const float* pre;
  float* c;  // n x k float32 work
  void* trsv;
  unsigned* st;
  int apply(const double* y, double* z, int64_t k, cudaStream_t s) const {
    RM_TRY(gather_f32(y, k, perm, n, k, c, k, s));
    RM_TRY(lu_solve_f32_nopiv(f, ldf, n, dinv, pre, c, k, k, trsv, st, s));
    return accumulate_f64(c, k, n, k, z, k, true, s);
  }
};
size_t gmres_scratch_bytes(int64_t n, int64_t k, int restart);
int gmres_ir(const double* a, int64_t n, const double* b, int64_t k, double* x, const Precond& pc, int restart,
             int max_outer, double tol, double* berr_out, int* outer_out, void* scratch, double* r, double* norms,
             double* berr_dev, cudaStream_t s);

// ---------------------------------------------------------------- Cholesky (potrf.cu)
size_t potrf_f64_scratch_bytes(int64_t n);
// L (row-major n x n, zeros above the diagonal) of the row-major a's lower triangle; when
// notpd_host is not NULL, *notpd_host (host memory) gets 1 once the stream reaches that point
// if a pivot was not > 0.
int potrf_f64(const double* a, int64_t n, double* l, void* scratch, int* notpd_host, unsigned* status,
              cudaStream_t stream);

// ---------------------------------------------------------------- helpers (api.cu)
int64_t round_up(int64_t x, int64_t m);
// True (and counts it) when rm_test_inject_failure armed a failure of `kind` on this thread.
bool injected_failure(int kind);
// The bounded-wait self-test (getrs.cu): a float64 chain solve at n = 256 whose first block
// never runs; the status bits its kernel set go to *bits (synchronises `stream`).
size_t chain_timeout_scratch_bytes();
int chain_timeout_run(uint64_t wait_ns, void* scratch, unsigned* bits, cudaStream_t stream);
// Stream-ordered scratch allocation from the device's default pool.
int scratch_alloc(void** p, size_t bytes, cudaStream_t stream);
void scratch_free(void* p, cudaStream_t stream);

}  // namespace rm
