/* CPU oracle: a C restatement of rustymath's dense f64 path (test infrastructure only).
 *
 * This header belongs to the checker, not the product. Only tests/, the smoke check and
 * bench.py's CPU-baseline leg load the library built from it. Each function names the
 * reference source it restates (paths are relative to the rustymath repository).
 *
 * Layout conventions follow the reference:
 *  - matrices passed in are row-major unless stated otherwise;
 *  - LU factors are column-major ("row j holds column j": item (i, j) at factors[j*n+i]),
 *    unit L below the diagonal, U on and above (core/src/linalg/factor.rs:132-134);
 *  - perm[i] is the source row of row i of L*U (factor.rs:132, 627-629).
 */
#ifndef RM_ORACLE_H
#define RM_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Threads used by the GEMM restatement (OpenMP); 0 leaves OpenMP's default. */
void ora_set_threads(int threads);
int ora_get_threads(void);

/* C = alpha*op(A)*op(B) + beta*C, row-major, op = transpose when ta/tb != 0.
 * Restates gemm (core/src/linalg.rs:799-807): scale for k==0/alpha==0, by_vector for m==1
 * or n==1 (linalg.rs:1020-1073), else native_gemm + product (linalg.rs:1077-1081, 1353-1426),
 * whose result folds each item's products into C in k order with FMA. */
void ora_dgemm(int ta, int tb, int64_t m, int64_t n, int64_t k, double alpha,
               const double *a, int64_t lda, const double *b, int64_t ldb,
               double beta, double *c, int64_t ldc);

/* In-order FMA fold C = beta*C + sum_p alpha*a_ip*b_pj without blocking or threads: the
 * plain statement of what the packed product computes (linalg.rs:1419-1441, micro). */
void ora_dgemm_fold(int64_t m, int64_t n, int64_t k, double alpha, const double *a,
                    const double *b, double beta, double *c);

/* lu_factor (factor.rs:617-630) with lu_panel (580-615): factors column-major n*n. */
void ora_lu_factor(int64_t n, const double *a, double *factors, int64_t *perm);

/* The pivot rows lu_panel records (pivots[c] = row swapped with row c), for tests. */
void ora_lu_factor_pivots(int64_t n, const double *a, double *factors, int64_t *pivots);

/* lu_solve (factor.rs:633-641): x (n*k row-major) from column-major factors and perm. */
void ora_lu_solve(int64_t n, const double *factors, const int64_t *perm,
                  const double *b, int64_t k, double *x);

/* Solves with the transposed matrix: A^T x = b from A's factors (the adjoint's solve).
 * The reference has no such entry; the adjoint checks build it from the same triangular
 * solves: U^T y = b, L^T z = y, x = P^T z. */
void ora_lu_solve_transposed(int64_t n, const double *factors, const int64_t *perm,
                             const double *b, int64_t k, double *x);

/* lu_inverse, rustymath's own kernels' branch (factor.rs:645-664): out n*n row-major. */
void ora_lu_inverse(int64_t n, const double *factors, const int64_t *perm, double *out);

/* Lu::determinant / log_determinant (factor.rs:174-182) with odd (186-194). */
double ora_lu_determinant(int64_t n, const double *factors, const int64_t *perm);
void ora_lu_log_determinant(int64_t n, const double *factors, const int64_t *perm,
                            double *sign, double *logabs);

/* LuWork::regular (factor.rs:221-226): 1 when every |u_ii| > eps*n*max|a|. */
/* L (row-major, zeros above the diagonal) with L L^T = A from A's lower triangle, as
 * rustymath's cholesky (core/src/linalg/factor.rs:750-795); 0 where A is not positive
 * definite (out untouched). */
int ora_cholesky(int64_t n, const double *a, double *out);

int ora_regular(int64_t n, const double *a, const double *factors);

/* solve (factor.rs:279) for a square, regular a: returns 0 and writes x, or returns 1
 * (the reference would fall back to lstsq, which is outside this path) and writes nothing. */
int ora_solve(int64_t n, const double *a, const double *b, int64_t k, double *x);

/* Normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) with the
 * residual formed in double-double (Dekker/Knuth TwoProd/TwoSum), per right-hand side
 * column; writes the largest over columns. */
double ora_backward_error(int64_t n, const double *a, const double *x, const double *b,
                          int64_t k);

/* Residual r = b - A x (n*k row-major) accumulated in double-double, rounded once. */
void ora_residual_dd(int64_t n, const double *a, const double *x, const double *b,
                     int64_t k, double *r);

#ifdef __cplusplus
}
#endif
#endif
