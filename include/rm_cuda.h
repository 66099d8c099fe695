/* rm_cuda.h: the C ABI of rustymath-b200, a B200 (sm_100a) implementation of rustymath's
 * dense float64 linear-algebra path: GEMM, LU with partial pivoting, the triangular solves
 * and the reusable factorization.
 *
 * The entry points replace these reference interfaces (paths within rustymath 0.1.66):
 *  - rm_dgemm          : Accelerated::xgemm, core/src/linalg/accelerate.rs:211, reached from
 *                        Tiled::gemm (core/src/linalg.rs:772-774) and PlusTimes.inner
 *                        (core/src/linalg.rs:1119-1132). CBLAS row-major shape.
 *  - rm_dlu_factor     : Factor::matrix_lu_into, core/src/linalg/factor.rs:87 (lu_factor,
 *                        factor.rs:617-630), plus the pivot test of LuWork::regular
 *                        (factor.rs:221-226).
 *  - rm_dlu_solve      : Factor::matrix_lu_solve, factor.rs:89 (lu_solve, factor.rs:633-641).
 *  - rm_dsolve         : solve, factor.rs:279 (LuWork::solve, factor.rs:207-209).
 *
 * Conventions (the reference's):
 *  - matrices are row-major float64 with a leading dimension in items;
 *  - LU factors are column-major: item (i, j) at factors[j*n + i] ("row j holds column j"),
 *    unit L strictly below the diagonal, U on and above it;
 *  - perm[i] is the row of the factored matrix that row i of L*U comes from.
 * Pointers named d_* are device pointers and the call is asynchronous on `stream` (a
 * cudaStream_t, NULL for the legacy default stream) unless it says it synchronises.
 * Pointers named h_* are host pointers and the call returns when its results are in
 * host memory. Every entry point returns an rm status code. Calls on different streams,
 * from different threads, are independent.
 */
#ifndef RM_CUDA_H
#define RM_CUDA_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define RM_OK 0
#define RM_BAD_ARG 1          /* a size, pointer, stride or option out of range */
#define RM_NOT_REGULAR 2      /* a pivot at most eps*n*max|a|: the reference takes lstsq here */
#define RM_CUDA_ERROR 3       /* a CUDA call failed; rm_last_error() has the message */
#define RM_TIMEOUT 4          /* a bounded device-side wait gave up */
#define RM_NO_CONVERGENCE 5   /* refinement did not reach the tolerance and fallback was off */
#define RM_NO_DEVICE 6        /* no CUDA device of compute capability 10.0 */
#define RM_OUT_OF_MEMORY 7
#define RM_NOT_POSITIVE_DEFINITE 8 /* a Cholesky pivot is not > 0: rustymath's cholesky gives None */

#define RM_NO_TRANS 0
#define RM_TRANS 1

/* Factorization methods for rm_dsolve. */
#define RM_METHOD_PLAIN_F64 0    /* LU in float64: the drop-in for rustymath's solve */
#define RM_METHOD_F32_IR 1       /* LU in float32 (tensor-core trailing updates) + float64 refinement;
                                    when classical refinement stalls, GMRES-IR (restart
                                    opts->gmres_restart; 0 skips it) with the same factors */
#define RM_METHOD_GMRES_IR 2     /* (reported in method_used) the answer came from GMRES-IR */

typedef struct rm_solve_options {
  int32_t method;          /* RM_METHOD_* */
  int32_t max_iterations;  /* refinement steps before the fallback decision (default 30) */
  int32_t gmres_restart;   /* GMRES-refinement restart length (default 20, as rustymath's GMRES) */
  int32_t fallback;        /* 1: fall back to RM_METHOD_PLAIN_F64 when refinement fails */
  double tolerance;        /* normwise backward error to reach; 0 means n * 2^-53 */
} rm_solve_options;

typedef struct rm_solve_report {
  double backward_error;   /* max over columns of ||b-Ax||inf / (||A||inf ||x||inf + ||b||inf) */
  int32_t iterations;      /* refinement steps taken (0 for the plain method) */
  int32_t method_used;     /* the method whose result was returned */
  int32_t fell_back;       /* 1 when the mixed method fell back to the plain one */
  int32_t regular;         /* LuWork::regular's verdict on the factored matrix */
} rm_solve_report;

/* Library version (major*10000 + minor*100 + patch) and the text of a status code. */
int rm_version(void);
const char *rm_status_string(int status);
/* Copies the calling thread's last error message into buf (always NUL-terminated). */
int rm_last_error(char *buf, size_t len);
/* Kernels this process has launched through the library so far (a diagnostic counter). */
int64_t rm_launch_count(void);
/* Number of CUDA devices usable by this library (compute capability 10.x). */
int rm_device_count(int *count);

/* Errors that kernels find while they run (a row position outside 0..n-1 in a caller's perm,
 * a bounded device-side wait that gave up) are recorded in a status word that each device
 * holds. Entry points that synchronise read and clear it before they return. The asynchronous
 * device forms (rm_dgemm, rm_dgemm_ozaki, rm_dlu_solve, rm_dlu_solve_noalloc, rm_dlu_factor
 * without h_regular, rm_batch_plan_execute, rm_batch_plan_adjoint) cannot: their errors
 * surface in the next call that reads the word.
 * rm_take_status synchronises `stream`, then returns the recorded error as an rm status code
 * (RM_BAD_ARG for a bad row position, RM_TIMEOUT for a wait) and clears the word. The word is
 * per device, not per stream: an error of a call on another stream of the same device, still
 * unread, is reported by whichever call reads the word first. */
int rm_take_status(void *stream);

/* ---- Test hooks. They make failures on the host, never on the GPU: no kernel faults, traps or
 * hangs because of them. */
#define RM_INJECT_OUT_OF_MEMORY 1 /* a scratch allocation reports device memory exhausted */
#define RM_INJECT_CUDA_ERROR 2    /* a scratch allocation fails with a CUDA error */
/* On the calling thread, after the next `after` events of `kind` succeed, `count` more fail
 * as described; count 0 disarms. */
int rm_test_inject_failure(int kind, int after, int count);
/* Runs a small float64 triangular chain solve (n = 256, four 64-row blocks) whose first block
 * row never runs, so the other blocks wait on a flag that nothing sets; every wait gives up
 * after wait_ns nanoseconds (1000 <= wait_ns <= 2e9). Returns RM_TIMEOUT when the kernel
 * reported its waits' expiry as it should (and RM_OK if it did not), on a status word of its
 * own; synchronises. The device stays usable afterwards. */
int rm_test_chain_timeout(int64_t wait_ns);

/* C = alpha*op(A)*op(B) + beta*C, row-major, op(X) = X or X^T (trans* = RM_TRANS).
 * op(A) is m x k, op(B) is k x n, C is m x n. Mirrors Accelerated::xgemm
 * (core/src/linalg/accelerate.rs:211) with order fixed to row-major. */
int rm_dgemm(int transa, int transb, int64_t m, int64_t n, int64_t k, double alpha,
             const double *d_a, int64_t lda, const double *d_b, int64_t ldb, double beta,
             double *d_c, int64_t ldc, void *stream);
int rm_dgemm_host(int transa, int transb, int64_t m, int64_t n, int64_t k, double alpha,
                  const double *h_a, int64_t lda, const double *h_b, int64_t ldb, double beta,
                  double *h_c, int64_t ldc);

/* C = alpha * A * op(B) + beta * C in float32 on the tensor cores (tcgen05, kind::tf32):
 * A is m x k row-major; op(B) = B (k x n row-major) or, with transb = RM_TRANS, B^T (B
 * n x k row-major); C is m x n row-major. passes = 1 reads the inputs as TF32; passes = 3
 * splits each operand into a TF32 part and a low part and sums three products, for
 * float32-level accuracy. The building block of the mixed-precision solve; it has no
 * counterpart in rustymath, whose float32 products run on its CPU kernels. */
int rm_sgemm_tc(int passes, int transb, int64_t m, int64_t n, int64_t k, float alpha,
                const float *d_a, int64_t lda, const float *d_b, int64_t ldb, float beta,
                float *d_c, int64_t ldc, void *stream);

/* LU with partial pivoting of the n x n row-major d_a into column-major d_factors and
 * d_perm (int64), as lu_factor (core/src/linalg/factor.rs:617-630) gives them. When
 * h_regular is not NULL the call synchronises and writes LuWork::regular's verdict
 * (factor.rs:221-226): 1 when every |u_ii| > eps*n*max|a|. */
int rm_dlu_factor(int64_t n, const double *d_a, double *d_factors, int64_t *d_perm,
                  int32_t *h_regular, void *stream);
int rm_dlu_factor_host(int64_t n, const double *h_a, double *h_factors, int64_t *h_perm,
                       int32_t *h_regular);

/* x = A^-1 b (trans = RM_NO_TRANS) or A^-T b (RM_TRANS) for the matrix the factors and
 * perm describe; b and x are n x k row-major (they may alias). Mirrors lu_solve
 * (core/src/linalg/factor.rs:633-641); the transposed form serves the adjoint. */
int rm_dlu_solve(int64_t n, const double *d_factors, const int64_t *d_perm, const double *d_b,
                 int64_t k, double *d_x, int trans, void *stream);
int rm_dlu_solve_host(int64_t n, const double *h_factors, const int64_t *h_perm,
                      const double *h_b, int64_t k, double *h_x, int trans);

/* LU of a stack of `count` n x n row-major matrices (n <= 256, back to back) in one launch:
 * each matrix's factors (column-major) and row positions as rm_dlu_factor gives them, one CTA
 * per matrix; d_regular[i] (optional) as LuWork::regular. Stacked::lu (src/linalg/stacked.rs:
 * 174-187). Partial pivoting by the greatest magnitude, NaN never chosen; among equal
 * magnitudes the lowest row of the input, where rustymath takes the first in its current
 * (already swapped) row order. Asynchronous. */
int rm_dlu_factor_batched(int64_t count, int64_t n, const double *d_a, double *d_factors, int64_t *d_perm,
                          int32_t *d_regular, void *stream);

/* The inverse of the matrix that the factors and perm describe: d_out = A^-1, row-major n x n,
 * as Lu::inverse (core/src/linalg/factor.rs:150-154; lu_inverse, factor.rs:645-664): U^-1 L^-1
 * from the identity, 16 columns at a time, the lower solve of each group of columns starting
 * at the block row of its first column (L^-1 is zero above its diagonal), then the columns
 * permuted by perm. Asynchronous; a bad row position surfaces through rm_take_status. */
int rm_dlu_inverse(int64_t n, const double *d_factors, const int64_t *d_perm, double *d_out, void *stream);
int rm_dlu_inverse_host(int64_t n, const double *h_factors, const int64_t *h_perm, double *h_out);

/* Determinants of a stack of `count` factorizations (n x n column-major factors and n row
 * positions each, back to back): d_det[i] as Lu::determinant (factor.rs:174-176: U's diagonal
 * multiplied in order from 1, negated when perm is odd; odd(), factor.rs:186-194) and d_sign[i],
 * d_logabs[i] as Lu::log_determinant (factor.rs:177-183: sign 0 and log -inf once a diagonal
 * item is 0). Any output may be NULL. The stack forms of Stacked::det and slogdet
 * (src/linalg/stacked.rs:136-171) factor first. Asynchronous. */
int rm_dlu_determinant(int64_t count, int64_t n, const double *d_factors, const int64_t *d_perm,
                       double *d_det, double *d_sign, double *d_logabs, void *stream);

/* x = A^-1 b (A^-T b when trans) for each of a stack of `count` factorizations with n <= 256
 * (column-major factors and row positions back to back) and n x k right-hand sides (k <= 64,
 * row-major, back to back), one launch: Stacked::lu_solve (src/linalg/stacked.rs:190-204).
 * b and x may alias. Asynchronous; a bad row position surfaces through rm_take_status. */
int rm_dlu_solve_batched(int64_t count, int64_t n, const double *d_factors, const int64_t *d_perm,
                         const double *d_b, int64_t k, double *d_x, int trans, void *stream);

/* rm_dlu_solve for callers that cannot allocate device memory during a call (a fixed
 * memory budget or arena that owns all device memory, a real-time loop kept away from the
 * allocator). It has no counterpart in the reference. Its scratch is a fixed __device__
 * array inside the library of RM_NOALLOC_SCRATCH_BYTES (about 8.9 MB: the inverted 64 x 64
 * diagonal blocks and couplings of a 4096-row factorization, 8 MiB, plus a permuted 4096 x 16
 * right-hand side and the solve's flags), held on every GPU that loads the library until
 * the process exits, so it takes n <= RM_NOALLOC_MAX_N and k <= RM_NOALLOC_MAX_K and
 * returns RM_BAD_ARG beyond them. The first call on a device looks the array up (once per
 * device); make that first call before any stream capture. All calls on one GPU share that
 * GPU's array and each leaves its contents for the next: calls that overlap on the same
 * GPU (on different streams) race on it, so the caller serialises them. A bad row position
 * in d_perm is reported through rm_take_status, as for rm_dlu_solve. */
#define RM_NOALLOC_MAX_N 4096
#define RM_NOALLOC_MAX_K 16
#define RM_NOALLOC_SCRATCH_BYTES 8913672
int rm_dlu_solve_noalloc(int64_t n, const double *d_factors, const int64_t *d_perm,
                         const double *d_b, int64_t k, double *d_x, int trans, void *stream);

/* x = A^-1 b for the n x n row-major A and n x k row-major b, by the method in opts (NULL:
 * plain float64). Returns RM_NOT_REGULAR, writing nothing to x, where rustymath's solve
 * would take its least-squares route (factor.rs:207-209). Synchronises on `stream`. */
int rm_dsolve(int64_t n, const double *d_a, const double *d_b, int64_t k, double *d_x,
              const rm_solve_options *opts, rm_solve_report *report, void *stream);
int rm_dsolve_host(int64_t n, const double *h_a, const double *h_b, int64_t k, double *h_x,
                   const rm_solve_options *opts, rm_solve_report *report);

/* X = op(A)^-1 X (side RM_LEFT, A m x m) or X op(A)^-1 (RM_RIGHT, A n x n) in place for the
 * row-major m x n X, with alpha = 1: the shape of Accelerated::xtrsm (core/src/linalg/
 * accelerate.rs:215, 269-275), reached from Tiled::triangular through accelerate::triangular
 * (accelerate.rs:67-74). The codes are CBLAS's, as the reference passes them: side 141/142,
 * uplo 121 (upper) / 122 (lower), trans 111/112, diag 131 (non-unit) / 132 (unit); row-major
 * storage (CBLAS order 101) is implied. Synchronises on `stream`. */
#define RM_LEFT 141
#define RM_RIGHT 142
#define RM_UPPER 121
#define RM_LOWER 122
#define RM_CBLAS_NO_TRANS 111
#define RM_CBLAS_TRANS 112
#define RM_NON_UNIT 131
#define RM_UNIT 132
int rm_dtrsm(int side, int uplo, int trans, int diag, int64_t m, int64_t n, const double *d_a, int64_t lda,
             double *d_x, int64_t ldx, void *stream);
int rm_dtrsm_host(int side, int uplo, int trans, int diag, int64_t m, int64_t n, const double *h_a, int64_t lda,
                  double *h_x, int64_t ldx);

/* C = A B (row-major float64, no transposes) from int8 tensor-core products: each row of A
 * and each column of B is scaled by a power of two and cut into `slices` (1..8) signed 7-bit
 * pieces, the pieces' products of order < slices are formed exactly in int32 and summed in
 * float64 (the Ozaki split scheme). With 8 slices the error is that of float64 rounding;
 * fewer trade accuracy for speed (error ~ k 2^-7slices |A||B| by row and column scale).
 * Inputs must be finite. rustymath's float64 matmul (PlusTimes.inner, core/src/linalg.rs:
 * 1119-1132) is the native product it stands beside (rm_dgemm). Asynchronous on `stream`. */
int rm_dgemm_ozaki(int64_t m, int64_t n, int64_t k, const double *d_a, int64_t lda, const double *d_b,
                   int64_t ldb, double *d_c, int64_t ldc, int slices, void *stream);
int rm_dgemm_ozaki_host(int64_t m, int64_t n, int64_t k, const double *h_a, int64_t lda, const double *h_b,
                        int64_t ldb, double *h_c, int64_t ldc, int slices);

/* ---- Cholesky.
 * L with L L^T = A for the symmetric positive definite n x n row-major A, reading only A's
 * lower triangle; L is row-major with zeros above the diagonal. Mirrors rustymath's cholesky
 * (core/src/linalg/factor.rs:267; cholesky_factor, factor.rs:750-795). Synchronises on
 * `stream`; returns RM_NOT_POSITIVE_DEFINITE where rustymath gives None (a pivot that is not
 * > 0, NaN included), d_l then unspecified. */
int rm_dcholesky(int64_t n, const double *d_a, double *d_l, void *stream);
int rm_dcholesky_host(int64_t n, const double *h_a, double *h_l);
/* A stack of `count` n x n matrices (n <= 128) back to back, in one launch: each L as
 * rm_dcholesky gives it, or NaN in every item where that matrix is not positive definite, as
 * rustymath's stack form (src/linalg/stacked.rs:259-268); d_ok[i] (optional) is 1 or 0.
 * Asynchronous on `stream`. */
int rm_dcholesky_batched(int64_t count, int64_t n, const double *d_a, double *d_l, int32_t *d_ok,
                         void *stream);
/* x = A^-1 b from A's Cholesky factor L (L y = b, then L^T x = y, the triangular solves of
 * rm_dtrsm); b and x n x k row-major, and they may alias. Synchronises. */
int rm_dcholesky_solve(int64_t n, const double *d_l, const double *d_b, int64_t k, double *d_x,
                       void *stream);

/* ---- Batched solves: many small systems of uneven size in one persistent launch.
 * System i is the n[i] x n[i] row-major float64 A at d_a + a_off[i] (items), its right-hand
 * sides the n[i] x k[i] row-major d_b + b_off[i], its solution d_x + x_off[i]; 0 <= n[i] <= 256
 * and 0 <= k[i] <= 8. rustymath solves a stack of same-size systems one LuWork per thread
 * (Stacked::solve, src/linalg/stacked.rs:88-101, each factor.rs:207-209); these entry points
 * take uneven sizes, which a rustymath stack cannot hold. opts->method picks float32 factors
 * + float64 refinement (RM_METHOD_F32_IR, with per-system fallback to float64 when
 * opts->fallback) or float64 factors (RM_METHOD_PLAIN_F64); every system's normwise backward
 * error is measured in float64. A plan holds the sorted order, the scratch and a CUDA graph
 * of the launch; rm_batch_plan_tune picks the panel width of each size bucket by timing. */
typedef struct rm_batch_report {
  double max_backward_error; /* over the systems (NaN if any is NaN) */
  int64_t fell_back;         /* systems answered by the float64 fallback */
  int64_t not_regular;       /* systems whose float64 factors fail rustymath's regular test */
  int64_t no_convergence;    /* systems left unrefined (fallback off) */
  int32_t max_iterations;    /* most refinement steps any system took */
} rm_batch_report;

/* per-system flags from rm_batch_plan_results */
#define RM_BATCH_FELL_BACK 1
#define RM_BATCH_NOT_REGULAR 2
#define RM_BATCH_NO_CONVERGENCE 4

typedef struct rm_batch_plan rm_batch_plan;
int rm_batch_plan_create(int64_t count, const int64_t *h_n, const int64_t *h_k, const int64_t *h_a_off,
                         const int64_t *h_b_off, const int64_t *h_x_off, const rm_solve_options *opts,
                         rm_batch_plan **plan);
/* Times each size bucket's candidate panel widths on these inputs (solving them) and keeps the
 * fastest, then the CTA size (64 or 256 threads) for the systems of n <= 32 and n <= 64;
 * synchronises on `stream`. */
int rm_batch_plan_tune(rm_batch_plan *plan, const double *d_a, const double *d_b, double *d_x, void *stream);
/* rm_batch_plan_tune with a precision axis as well (a plan made with RM_METHOD_F32_IR): each
 * size bucket also times float64 factors without refinement and keeps whichever route is
 * fastest, so every system still meets the plan's tolerance. rustymath's Stacked::solve has no
 * tuner (every stack is float64); this chooses per size bucket. Synchronises on `stream`. */
int rm_batch_plan_tune_precision(rm_batch_plan *plan, const double *d_a, const double *d_b, double *d_x,
                                 void *stream);
/* One persistent kernel launch for all systems, replayed from a CUDA graph; asynchronous on
 * `stream`. */
int rm_batch_plan_execute(rm_batch_plan *plan, const double *d_a, const double *d_b, double *d_x, void *stream);
/* rm_batch_plan_execute from host memory: copies h_a and h_b (packed as for execute) into d_a
 * and d_b, solves, and copies x back into h_x, in groups of consecutive systems so that one
 * group's copies overlap another's solves (h_a, h_b, h_x pinned for the overlap). A plan whose
 * offsets do not follow the systems' order takes one group. Asynchronous on `stream`: h_x holds
 * the solutions once `stream` reaches the end. The results and the adjoint read it as an
 * execute. (rustymath has no host-to-device path; this is the host-memory form of the stack.) */
int rm_batch_plan_execute_host(rm_batch_plan *plan, const double *h_a, const double *h_b, double *h_x, double *d_a,
                               double *d_b, double *d_x, void *stream);
/* Per-system backward errors, refinement steps and RM_BATCH_* flags of the last execute (any
 * pointer may be NULL); synchronises. */
int rm_batch_plan_results(rm_batch_plan *plan, double *h_berr, int32_t *h_iters, int32_t *h_flags,
                          rm_batch_report *summary);
/* The adjoint of the last execute, for reverse-mode differentiation of x = A^-1 b: given
 * d_gx = dL/dx (packed like b), writes d_gb = dL/db = A^-T dL/dx (packed like b) and, unless
 * d_ga is NULL, d_ga = dL/dA = -(dL/db) x^T (packed like a). It reuses the factors the
 * execute left in the plan (d_a and d_x must be that execute's): a transposed solve with the
 * same row order, refined in float64 against A^T when the factors are float32 (an A whose
 * refinement stalls is factored again in float64). rustymath has no derivative of solve; this
 * is the north star's adjoint. Asynchronous on `stream`. */
int rm_batch_plan_adjoint(rm_batch_plan *plan, const double *d_a, const double *d_x, const double *d_gx,
                          double *d_gb, double *d_ga, void *stream);
/* Per-system normwise backward errors of the last adjoint's A^T gb = gx (either pointer may be
 * NULL); synchronises. */
int rm_batch_plan_adjoint_results(rm_batch_plan *plan, double *h_berr, double *h_max_berr);
/* The panel width chosen for size bucket 0..4 (n <= 32, 64, 128, 192, 256). */
int rm_batch_plan_panel_width(const rm_batch_plan *plan, int bucket);
/* The threads per CTA (a thread per row) that solve size bucket 0..4: 64 or 256 (the
 * 64-thread build takes systems of n <= 64 unless the tuner chose otherwise). */
int rm_batch_plan_cta_threads(const rm_batch_plan *plan, int bucket);
/* The route size bucket 0..4 takes: RM_METHOD_F32_IR (float32 factors + float64 refinement) or
 * RM_METHOD_PLAIN_F64 (float64 factors); -1 for a bad argument. */
int rm_batch_plan_precision(const rm_batch_plan *plan, int bucket);
int rm_batch_plan_destroy(rm_batch_plan *plan);
/* create + execute + results + destroy; synchronises. RM_NO_CONVERGENCE when a system stalled
 * with fallback off. */
int rm_dsolve_batched(int64_t count, const int64_t *h_n, const int64_t *h_k, const int64_t *h_a_off,
                      const int64_t *h_b_off, const int64_t *h_x_off, const double *d_a, const double *d_b,
                      double *d_x, const rm_solve_options *opts, rm_batch_report *report, void *stream);
/* The same with host A, B and X (the host-pointer form of every batched entry point above). */
int rm_dsolve_batched_host(int64_t count, const int64_t *h_n, const int64_t *h_k, const int64_t *h_a_off,
                           const int64_t *h_b_off, const int64_t *h_x_off, const double *h_a, const double *h_b,
                           double *h_x, const rm_solve_options *opts, rm_batch_report *report);

#ifdef __cplusplus
}
#endif
#endif
