/* CPU oracle for the dense f64 path: a C restatement of rustymath's algorithms.
 *
 * TEST INFRASTRUCTURE ONLY. tests/, the smoke check and bench.py's CPU-baseline leg use it
 * as the checker and as the timed CPU baseline; the product path never calls it.
 *
 * The reference (rustymath 0.1.66) is Rust and cannot be compiled in this environment, so
 * this file restates its algorithms from the source, keeping their operation order:
 *  - FMA exactly where the reference calls `mul_acc` (core/src/linalg/scalar.rs:52 with
 *    FUSED on x86-64-v3, core/src/float.rs:5); no other contraction (-ffp-contract=off);
 *  - the packed product folds each result's products into C in k order
 *    (core/src/linalg.rs:1353-1441), so any blocking or thread split gives the same bits;
 *  - lu_panel's recursion, LEAF=16, NS=32, stride() padding, pivot rule (first largest
 *    magnitude, NaN skipped) and divide-by-reciprocal (factor.rs:72-82, 476-508, 572-630);
 *  - the triangular solves forward/backward/single (factor.rs:668-748).
 * Parity of this file with the reference is pinned by the reference's own known-answer
 * tests (tests/linalg.rs), restated in tests/test_oracle.py.
 */
#include "rm_oracle.h"

#include <float.h>
#include <immintrin.h>
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

enum { LEAF = 16, NS = 32, KC = 256, MC = 128, NC = 2048, MR = 6, NR = 8, NARROW = 8 };

static int g_threads = 0;
void ora_set_threads(int threads) { g_threads = threads; }
int ora_get_threads(void) { return g_threads > 0 ? g_threads : omp_get_max_threads(); }

/* A strided matrix view, stored row-major with rows `ld` apart, read transposed when `t`
 * (core/src/linalg.rs:646-708, Matrix with Op::Normal / Op::Transpose). */
typedef struct { const double *data; int64_t ld; int t; } view;

static inline view vrows(const double *d, int64_t ld) { view v = {d, ld, 0}; return v; }
static inline view vtr(view v) { v.t = !v.t; return v; }
static inline double vat(view v, int64_t i, int64_t j) { return v.t ? v.data[j * v.ld + i] : v.data[i * v.ld + j]; }
static inline view voff(view v, int64_t row, int64_t col) { v.data += v.t ? col * v.ld + row : row * v.ld + col; return v; }

static int64_t stride_of(int64_t n) { return (n > 0 && n % 128 == 0) ? n + 8 : n; } /* factor.rs:72 */

/* ---------------------------------------------------------------- scalar helpers */

/* axpy: y += a x with y = x.mul_acc(a, y) = fma(x, a, y)   (factor.rs:452) */
static inline void axpy(double *y, double a, const double *x, int64_t n) {
    for (int64_t i = 0; i < n; i++) y[i] = fma(x[i], a, y[i]);
}

/* dot: eight running sums, folded from zero in order, then the tail (factor.rs:466-473) */
static double dot(const double *x, const double *y, int64_t n) {
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t whole = n / 8 * 8;
    for (int64_t c = 0; c < whole; c += 8)
        for (int k = 0; k < 8; k++) s[k] = fma(x[c + k], y[c + k], s[k]);
    double t = 0.0;
    for (int k = 0; k < 8; k++) t = t + s[k];
    for (int64_t i = whole; i < n; i++) t = fma(x[i], y[i], t);
    return t;
}

/* divide: multiply by the reciprocal unless the divisor is subnormal (factor.rs:506-508) */
static void divide(double *x, int64_t n, double d) {
    if (fabs(d) >= DBL_MIN) {
        double r = 1.0 / d;
        for (int64_t i = 0; i < n; i++) x[i] = x[i] * r;
    } else {
        for (int64_t i = 0; i < n; i++) x[i] = x[i] / d;
    }
}

/* greatest |x| ignoring NaN, from 0 (factor.rs:488, float.rs:200) */
static double greatest_abs(const double *x, int64_t n, int64_t step) {
    double top = 0.0;
    for (int64_t i = 0; i < n; i++) { double v = fabs(x[i * step]); if (v > top) top = v; }
    return top;
}

/* largest: position of the first item whose |x| equals the greatest, or 0 (factor.rs:476) */
static int64_t largest(const double *x, int64_t n) {
    double top = greatest_abs(x, n, 1);
    for (int64_t i = 0; i < n; i++) if (fabs(x[i]) == top) return i;
    return 0;
}

/* ---------------------------------------------------------------- GEMM */

static void scale_c(double *c, int64_t ldc, int64_t m, int64_t n, double beta) { /* linalg.rs:1000-1008 */
    if (beta == 1.0) return;
    for (int64_t i = 0; i < m; i++)
        for (int64_t j = 0; j < n; j++) c[i * ldc + j] = beta == 0.0 ? 0.0 : beta * c[i * ldc + j];
}

/* narrow_sums (linalg.rs:937-953): up to NARROW results, four interleaved sets of rows. The
 * reference sends the rows whose 8-wide read would pass the end of its buffer to the last
 * loop; here every row counts as whole, which differs only in rounding order. */
static void narrow_sums(double *out, int64_t n, const double *data, int64_t ld, const double *w, int64_t k) {
    double acc[4][NARROW];
    memset(acc, 0, sizeof acc);
    int64_t quads = k / 4;
    for (int64_t q = 0; q < quads; q++)
        for (int s = 0; s < 4; s++)
            for (int64_t t = 0; t < n; t++) acc[s][t] = fma(data[(4 * q + s) * ld + t], w[4 * q + s], acc[s][t]);
    for (int64_t p = 4 * quads; p < k; p++)
        for (int64_t t = 0; t < n; t++) acc[0][t] = fma(data[p * ld + t], w[p], acc[0][t]);
    for (int64_t t = 0; t < n; t++) out[t] = (acc[0][t] + acc[2][t]) + (acc[1][t] + acc[3][t]);
}

/* dots (linalg.rs:903-918) and narrow_dots (921-935) over stored rows of k items */
static void row_dots(double *out, int64_t rows, const double *data, int64_t ld, const double *x, int64_t k) {
    if (k <= NARROW) {
        for (int64_t i = 0; i < rows; i++) {
            double s[2] = {0.0, 0.0};
            for (int64_t l = 0; l < k; l++) s[l % 2] = fma(data[i * ld + l], x[l], s[l % 2]);
            out[i] = s[0] + s[1];
        }
        return;
    }
    int64_t quads = rows / 4, whole = k / 8 * 8;
    for (int64_t q = 0; q < quads; q++) {
        double s[4][8];
        memset(s, 0, sizeof s);
        for (int64_t c = 0; c < whole; c += 8)
            for (int r = 0; r < 4; r++)
                for (int l = 0; l < 8; l++) s[r][l] = fma(data[(4 * q + r) * ld + c + l], x[c + l], s[r][l]);
        for (int r = 0; r < 4; r++) {
            double t = ((s[r][0] + s[r][4]) + (s[r][2] + s[r][6])) + ((s[r][1] + s[r][5]) + (s[r][3] + s[r][7]));
            for (int64_t p = whole; p < k; p++) t = fma(data[(4 * q + r) * ld + p], x[p], t);
            out[4 * q + r] = t;
        }
    }
    for (int64_t i = 4 * quads; i < rows; i++) out[i] = dot(data + i * ld, x, k);
}

/* by_vector (linalg.rs:1020-1073): a product with m == 1 or n == 1. */
static int by_vector(double *c, int64_t ldc, view a, double alpha, view b, int64_t m, int64_t k, int64_t n, double beta) {
    view mat, vec;
    int64_t rows, step;
    if (n == 1) { mat = a; vec = vtr(b); rows = m; step = ldc; }
    else if (m == 1) { mat = vtr(b); vec = a; rows = n; step = 1; }
    else return 0;
    int narrow = (mat.t ? rows : k) <= NARROW;
    int64_t vs = vec.t ? vec.ld : 1;
    double *x = malloc((size_t)k * sizeof(double));
    for (int64_t p = 0; p < k; p++) x[p] = vec.data[p * vs];
    int one = alpha == 1.0, start = beta == 0.0;
    int direct = step == 1 && one && start;
    double *y = direct ? c : calloc((size_t)rows, sizeof(double));
    if (mat.t) {
        if (narrow) narrow_sums(y, rows, mat.data, mat.ld, x, k);
        else {
            /* scaled_runs: every result folds the stored rows in order from zero */
            for (int64_t i = 0; i < rows; i++) {
                double acc = 0.0;
                for (int64_t p = 0; p < k; p++) acc = fma(x[p], mat.data[p * mat.ld + i], acc);
                y[i] = acc;
            }
        }
    } else {
        row_dots(y, rows, mat.data, mat.ld, x, k);
    }
    if (!direct) {
        for (int64_t i = 0; i < rows; i++) {
            double v = one ? y[i] : alpha * y[i];
            double *z = &c[i * step];
            *z = start ? v : fma(beta, *z, v);
        }
        free(y);
    }
    free(x);
    return 1;
}

/* The 6x8 AVX2 tile of the packed product: folds kc steps into t, which starts at zero
 * when `zero`, else at C's items (linalg.rs:1282 times64, 1435-1441 micro). */
static void micro_6x8(int64_t kc, const double *ap, const double *bp, double *t /* 6x8 */, int zero) {
    __m256d acc[MR][2];
    for (int r = 0; r < MR; r++) {
        acc[r][0] = zero ? _mm256_setzero_pd() : _mm256_loadu_pd(t + r * NR);
        acc[r][1] = zero ? _mm256_setzero_pd() : _mm256_loadu_pd(t + r * NR + 4);
    }
    for (int64_t p = 0; p < kc; p++) {
        __m256d b0 = _mm256_loadu_pd(bp + p * NR), b1 = _mm256_loadu_pd(bp + p * NR + 4);
        for (int r = 0; r < MR; r++) {
            __m256d av = _mm256_broadcast_sd(ap + p * MR + r);
            acc[r][0] = _mm256_fmadd_pd(av, b0, acc[r][0]);
            acc[r][1] = _mm256_fmadd_pd(av, b1, acc[r][1]);
        }
    }
    for (int r = 0; r < MR; r++) { _mm256_storeu_pd(t + r * NR, acc[r][0]); _mm256_storeu_pd(t + r * NR + 4, acc[r][1]); }
}

/* product (linalg.rs:1353-1426) for f64 PlusTimes: C = (start ? 0 : C) + fold_k (alpha a) b */
static void packed_product(double *c, int64_t ldc, view a, double alpha, view b, int64_t m, int64_t k, int64_t n, int start) {
    int threads = ora_get_threads();
    int64_t work = m * k * n;
    if (work < (1 << 20)) threads = 1;
    double *bpack = malloc((size_t)((NC + NR) * KC) * sizeof(double));
    #pragma omp parallel num_threads(threads)
    {
        double *apack = malloc((size_t)((MC + MR) * KC) * sizeof(double));
        double tile[MR * NR];
        for (int64_t jc = 0; jc < n; jc += NC) {
            int64_t nc = n - jc < NC ? n - jc : NC;
            int64_t strips = (nc + NR - 1) / NR;
            for (int64_t pc = 0; pc < k; pc += KC) {
                int64_t kc = k - pc < KC ? k - pc : KC;
                int load = pc > 0 || !start;
                #pragma omp for schedule(static)
                for (int64_t s = 0; s < strips; s++) {
                    double *dst = bpack + s * NR * kc;
                    for (int64_t p = 0; p < kc; p++)
                        for (int l = 0; l < NR; l++) {
                            int64_t j = jc + s * NR + l;
                            dst[p * NR + l] = j < n ? vat(b, pc + p, j) : 0.0;
                        }
                }
                /* implicit barrier: B is packed */
                #pragma omp for schedule(dynamic, 1)
                for (int64_t ic = 0; ic < m; ic += MC) {
                    int64_t mc = m - ic < MC ? m - ic : MC;
                    int64_t astrips = (mc + MR - 1) / MR;
                    for (int64_t s = 0; s < astrips; s++) {
                        double *dst = apack + s * MR * kc;
                        for (int64_t p = 0; p < kc; p++)
                            for (int r = 0; r < MR; r++) {
                                int64_t i = ic + s * MR + r;
                                double v = i < m ? vat(a, i, pc + p) : 0.0;
                                dst[p * MR + r] = alpha == 1.0 ? v : alpha * v;
                            }
                    }
                    for (int64_t s = 0; s < astrips; s++) {
                        int64_t rows = mc - s * MR < MR ? mc - s * MR : MR;
                        for (int64_t sb = 0; sb < strips; sb++) {
                            int64_t cols = nc - sb * NR < NR ? nc - sb * NR : NR;
                            double *cp = c + (ic + s * MR) * ldc + jc + sb * NR;
                            if (load)
                                for (int64_t r = 0; r < rows; r++)
                                    for (int64_t q = 0; q < cols; q++) tile[r * NR + q] = cp[r * ldc + q];
                            micro_6x8(kc, apack + s * MR * kc, bpack + sb * NR * kc, tile, !load);
                            for (int64_t r = 0; r < rows; r++)
                                for (int64_t q = 0; q < cols; q++) cp[r * ldc + q] = tile[r * NR + q];
                        }
                    }
                }
            }
        }
        free(apack);
    }
    free(bpack);
}

/* gemm (linalg.rs:799-807) on rustymath's own kernels */
static void gemm_v(double *c, int64_t ldc, view a, view b, int64_t m, int64_t k, int64_t n, double alpha, double beta) {
    if (m == 0 || n == 0) return;
    if (k == 0 || alpha == 0.0) { scale_c(c, ldc, m, n, beta); return; }
    if (by_vector(c, ldc, a, alpha, b, m, k, n, beta)) return;
    int start = beta == 0.0;
    if (!start) scale_c(c, ldc, m, n, beta);
    packed_product(c, ldc, a, alpha, b, m, k, n, start);
}

void ora_dgemm(int ta, int tb, int64_t m, int64_t n, int64_t k, double alpha, const double *a, int64_t lda,
               const double *b, int64_t ldb, double beta, double *c, int64_t ldc) {
    view va = {a, lda, ta != 0}, vb = {b, ldb, tb != 0};
    gemm_v(c, ldc, va, vb, m, k, n, alpha, beta);
}

void ora_dgemm_fold(int64_t m, int64_t n, int64_t k, double alpha, const double *a, const double *b, double beta, double *c) {
    for (int64_t i = 0; i < m; i++)
        for (int64_t j = 0; j < n; j++) {
            double acc = beta == 0.0 ? 0.0 : (beta == 1.0 ? c[i * n + j] : beta * c[i * n + j]);
            for (int64_t p = 0; p < k; p++) acc = fma(alpha == 1.0 ? a[i * k + p] : alpha * a[i * k + p], b[p * n + j], acc);
            c[i * n + j] = acc;
        }
}

/* ---------------------------------------------------------------- triangular solves */

/* forward (factor.rs:668-689) */
static void forward(view l, int64_t r0, int64_t r1, double *x, int64_t ldx, int64_t k, int64_t block, int lower, int unit) {
    if (!lower && r1 - r0 > block) {
        int64_t mid = (r0 + r1) / 2;
        double *top = x, *bottom = x + (mid - r0) * ldx;
        forward(l, r0, mid, top, ldx, k, block, 0, unit);
        gemm_v(bottom, ldx, voff(l, mid, r0), vrows(top, ldx), r1 - mid, mid - r0, k, -1.0, 1.0);
        forward(l, mid, r1, bottom, ldx, k, block, 0, unit);
        return;
    }
    for (int64_t i0 = r0; i0 < r1; i0 += block) {
        int64_t i1 = i0 + block < r1 ? i0 + block : r1;
        int64_t width = lower ? i1 : k;
        double *rows = x + (i0 - r0) * ldx;
        for (int64_t i = i0; i < i1; i++) {
            double *row = rows + (i - i0) * ldx;
            for (int64_t j = i0; j < i; j++) axpy(row, -vat(l, i, j), rows + (j - i0) * ldx, width);
            if (!unit) divide(row, width, vat(l, i, i));
        }
        if (i1 < r1)
            gemm_v(x + (i1 - r0) * ldx, ldx, voff(l, i1, i0), vrows(rows, ldx), r1 - i1, i1 - i0, width, -1.0, 1.0);
    }
}

/* backward (factor.rs:693-707) */
static void backward(view u, int64_t r0, int64_t r1, double *x, int64_t ldx, int64_t k, int unit) {
    if (r1 - r0 > NS) {
        int64_t mid = (r0 + r1) / 2;
        double *top = x, *bottom = x + (mid - r0) * ldx;
        backward(u, mid, r1, bottom, ldx, k, unit);
        gemm_v(top, ldx, voff(u, r0, mid), vrows(bottom, ldx), mid - r0, r1 - mid, k, -1.0, 1.0);
        backward(u, r0, mid, top, ldx, k, unit);
        return;
    }
    for (int64_t i = r1 - 1; i >= r0; i--) {
        double *xi = x + (i - r0) * ldx;
        for (int64_t j = i + 1; j < r1; j++) axpy(xi, -vat(u, i, j), x + (j - r0) * ldx, k);
        if (!unit) divide(xi, k, vat(u, i, i));
    }
}

/* single (factor.rs:725-748): one contiguous right-hand side */
static void single(double *x, view a, int64_t m, int lower, int unit) {
    const double *d = a.data;
    int64_t ld = a.ld;
#define SOLVED(v, i) (unit ? (v) : (v) / d[(i) * ld + (i)])
    if (a.t && lower) {
        for (int64_t j = 0; j < m; j++) { x[j] = SOLVED(x[j], j); axpy(x + j + 1, -x[j], d + j * ld + j + 1, m - j - 1); }
    } else if (a.t) {
        for (int64_t j = m - 1; j >= 0; j--) { x[j] = SOLVED(x[j], j); axpy(x, -x[j], d + j * ld, j); }
    } else if (lower) {
        for (int64_t i = 0; i < m; i++) x[i] = SOLVED(x[i] - dot(d + i * ld, x, i), i);
    } else {
        for (int64_t i = m - 1; i >= 0; i--) x[i] = SOLVED(x[i] - dot(d + i * ld + i + 1, x + i + 1, m - i - 1), i);
    }
#undef SOLVED
}

enum { LOWER = 0, UNIT_UPPER = 1 };

/* triangular_native for Side::Left (factor.rs:711-721) */
static void triangular(double *x, int64_t ldx, view a, int64_t m, int64_t n, int triangle) {
    if (m == 0 || n == 0) return;
    int lower = (triangle == LOWER) != a.t, unit = triangle == UNIT_UPPER;
    if (n == 1 && ldx == 1) { single(x, a, m, lower, unit); return; }
    if (lower) forward(a, 0, m, x, ldx, n, n >= m ? LEAF : NS, 0, unit);
    else backward(a, 0, m, x, ldx, n, unit);
}

/* ---------------------------------------------------------------- LU */

/* swap_rows (factor.rs:572-577): columns start ld apart */
static void swap_rows(double *columns, int64_t ncols, int64_t ld, const int64_t *pivots, int64_t npiv, int64_t first) {
    for (int64_t c = 0; c < ncols; c++) {
        double *col = columns + c * ld;
        for (int64_t i = 0; i < npiv; i++) { double t = col[first + i]; col[first + i] = col[pivots[i]]; col[pivots[i]] = t; }
    }
}

/* lu_panel (factor.rs:580-615) */
static void lu_panel(double *f, int64_t n, int64_t ld, int64_t c0, int64_t c1, int64_t *pivots, double *scratch) {
    if (c1 - c0 > LEAF) {
        int64_t mid = (c0 + c1) / 2;
        lu_panel(f, n, ld, c0, mid, pivots, scratch);
        int64_t k = mid - c0, w = c1 - mid, lw = stride_of(w);
        double *half = f + mid * ld;
        swap_rows(half, w, ld, pivots + c0, k, c0);
        for (int64_t r = 0; r < k; r++) {
            for (int64_t j = 0; j < w; j++) scratch[r * lw + j] = half[j * ld + c0 + r];
            for (int64_t j = w; j < lw; j++) scratch[r * lw + j] = 0.0;
        }
        triangular(scratch, lw, vtr(vrows(f + c0 * ld + c0, ld)), k, w, UNIT_UPPER);
        for (int64_t r = 0; r < k; r++)
            for (int64_t j = 0; j < w; j++) half[j * ld + c0 + r] = scratch[r * lw + j];
        gemm_v(half + mid, ld, vtr(vrows(scratch, lw)), vrows(f + c0 * ld + mid, ld), w, k, n - mid, -1.0, 1.0);
        lu_panel(f, n, ld, mid, c1, pivots, scratch);
        swap_rows(f + c0 * ld, k, ld, pivots + mid, w, mid);
        return;
    }
    for (int64_t c = c0; c < c1; c++) {
        int64_t p = c + largest(f + c * ld + c, n - c);
        pivots[c] = p;
        if (p != c)
            for (int64_t j = c0; j < c1; j++) { double t = f[j * ld + c]; f[j * ld + c] = f[j * ld + p]; f[j * ld + p] = t; }
        double pivot = f[c * ld + c];
        if (pivot == 0.0) continue;
        double *l = f + c * ld + c + 1;
        divide(l, n - c - 1, pivot);
        for (int64_t j = c + 1; j < c1; j++) {
            double *column = f + j * ld;
            double u = column[c];
            axpy(column + c + 1, -u, l, n - c - 1);
        }
    }
}

static void lu_factor_impl(int64_t n, const double *a, double *factors, int64_t *perm, int64_t *pivots_out) {
    if (n <= 0) return;
    int64_t ld = stride_of(n);
    double *f = malloc((size_t)(n * ld) * sizeof(double));
    for (int64_t j = 0; j < n; j++) {
        for (int64_t i = 0; i < n; i++) f[j * ld + i] = a[i * n + j];
        for (int64_t i = n; i < ld; i++) f[j * ld + i] = 0.0;
    }
    int64_t *pivots = calloc((size_t)n, sizeof(int64_t));
    int64_t w = n / 2 + 1;
    double *scratch = malloc((size_t)((n / 2 + 1) * (stride_of(w) + 8)) * sizeof(double) + 64);
    lu_panel(f, n, ld, 0, n, pivots, scratch);
    for (int64_t j = 0; j < n; j++) memcpy(factors + j * n, f + j * ld, (size_t)n * sizeof(double));
    if (perm) {
        for (int64_t i = 0; i < n; i++) perm[i] = i;
        for (int64_t c = 0; c < n; c++) { int64_t t = perm[c]; perm[c] = perm[pivots[c]]; perm[pivots[c]] = t; }
    }
    if (pivots_out) memcpy(pivots_out, pivots, (size_t)n * sizeof(int64_t));
    free(scratch);
    free(pivots);
    free(f);
}

void ora_lu_factor(int64_t n, const double *a, double *factors, int64_t *perm) { lu_factor_impl(n, a, factors, perm, NULL); }
void ora_lu_factor_pivots(int64_t n, const double *a, double *factors, int64_t *pivots) { lu_factor_impl(n, a, factors, NULL, pivots); }

void ora_lu_solve(int64_t n, const double *factors, const int64_t *perm, const double *b, int64_t k, double *x) {
    for (int64_t i = 0; i < n; i++) memcpy(x + i * k, b + perm[i] * k, (size_t)k * sizeof(double));
    view p = vtr(vrows(factors, n));
    triangular(x, k, p, n, k, UNIT_UPPER);
    triangular(x, k, p, n, k, LOWER);
}

void ora_lu_solve_transposed(int64_t n, const double *factors, const int64_t *perm, const double *b, int64_t k, double *x) {
    double *z = malloc((size_t)(n * k + 1) * sizeof(double));
    memcpy(z, b, (size_t)(n * k) * sizeof(double));
    /* U^T y = b: U^T is lower with U's diagonal; (U^T)(i,j) = U(j,i) = factors[i*n + j] */
    for (int64_t i = 0; i < n; i++) {
        for (int64_t j = 0; j < i; j++) {
            double u = factors[i * n + j];
            for (int64_t c = 0; c < k; c++) z[i * k + c] = fma(-u, z[j * k + c], z[i * k + c]);
        }
        double d = factors[i * n + i];
        for (int64_t c = 0; c < k; c++) z[i * k + c] = z[i * k + c] / d;
    }
    /* L^T z = y: upper with unit diagonal; (L^T)(i,j) = L(j,i) = factors[i*n + j] for j > i */
    for (int64_t i = n - 1; i >= 0; i--)
        for (int64_t j = i + 1; j < n; j++) {
            double l = factors[i * n + j];
            for (int64_t c = 0; c < k; c++) z[i * k + c] = fma(-l, z[j * k + c], z[i * k + c]);
        }
    for (int64_t i = 0; i < n; i++) memcpy(x + perm[i] * k, z + i * k, (size_t)k * sizeof(double));
    free(z);
}

void ora_lu_inverse(int64_t n, const double *factors, const int64_t *perm, double *out) {
    if (n == 0) return;
    view p = vtr(vrows(factors, n));
    int64_t ld = stride_of(n);
    double *x = calloc((size_t)(n * ld), sizeof(double));
    for (int64_t i = 0; i < n; i++) x[i * ld + i] = 1.0;
    forward(p, 0, n, x, ld, n, NS, 1, 1);
    triangular(x, ld, p, n, n, LOWER);
    for (int64_t r = 0; r < n; r++)
        for (int64_t c = 0; c < n; c++) out[r * n + perm[c]] = x[r * ld + c];
    free(x);
}

static int odd(int64_t n, const int64_t *perm) { /* factor.rs:186-194 */
    int64_t cycles = 0;
    for (int64_t start = 0; start < n; start++) {
        int64_t i = perm[start];
        while (i > start) i = perm[i];
        if (i == start) cycles++;
    }
    return (n - cycles) % 2 == 1;
}

double ora_lu_determinant(int64_t n, const double *factors, const int64_t *perm) {
    double product = 1.0;
    for (int64_t i = 0; i < n; i++) product = product * factors[i * n + i];
    return odd(n, perm) ? -product : product;
}

void ora_lu_log_determinant(int64_t n, const double *factors, const int64_t *perm, double *sign, double *logabs) {
    double s = odd(n, perm) ? -1.0 : 1.0, l = 0.0;
    for (int64_t i = 0; i < n; i++) {
        double d = factors[i * n + i], m = fabs(d);
        if (m == 0.0) { s = 0.0; l = -INFINITY; }
        else { s = s * (d * (1.0 / m)); l = l + log(m); }
    }
    *sign = s;
    *logabs = l;
}

/* ---------------------------------------------------------------- Cholesky */

/* cholesky_panel (factor.rs:750-773): factors columns c0..c1 of the rows-row block that
 * `panel` holds column by column (columns ld apart), halving the columns above LEAF; a leaf
 * column takes d = sqrt(its diagonal), divides the items below by d (divide: the reciprocal
 * unless d is subnormal) and removes itself from the leaf's later columns by axpy. 0 where
 * a diagonal is not > 0 (not positive definite; NaN too). */
static int cholesky_panel(double *panel, int64_t rows, int64_t ld, int64_t c0, int64_t c1) {
    if (c1 - c0 > LEAF) {
        int64_t mid = (c0 + c1) / 2;
        if (!cholesky_panel(panel, rows, ld, c0, mid)) return 0;
        /* columns mid..c1, rows mid..: -= L(rows, c0..mid) L(cols, c0..mid)^T */
        view l = vrows(panel + c0 * ld + mid, ld);
        gemm_v(panel + mid * ld + mid, ld, vtr(l), l, c1 - mid, mid - c0, rows - mid, -1.0, 1.0);
        return cholesky_panel(panel, rows, ld, mid, c1);
    }
    for (int64_t c = c0; c < c1; c++) {
        double d = panel[c * ld + c];
        if (!(d > 0.0)) return 0;
        d = sqrt(d);
        panel[c * ld + c] = d;
        double *lc = panel + c * ld + c + 1;
        divide(lc, rows - c - 1, d);
        for (int64_t j = 0; j < c1 - c - 1; j++) {
            double *column = panel + (c + 1 + j) * ld;
            axpy(column + c + 1 + j, -lc[j], lc + j, rows - c - 1 - j);
        }
    }
    return 1;
}

/* cholesky_factor (factor.rs:776-795): blocks of cholesky_block(n) = clamp(n/8, 32, 128)
 * columns (factor.rs:29) in a copy with rows stride(n) apart; each block's columns factor in
 * a transposed copy (columns stride(rows) apart), go back, and `gram` (linalg.rs:777-779, the
 * lower triangle of C - X X^T) updates the rest. L row-major with zeros above the diagonal;
 * 0 (nothing written) where the matrix is not positive definite. Only a's lower triangle is
 * read. gram computes only the lower triangle; here the whole product is formed, whose lower
 * triangle has the same bits (every item folds its k terms in order on its own). */
int ora_cholesky(int64_t n, const double *a, double *out) {
    if (n == 0) return 1;
    int64_t ld = stride_of(n);
    double *l = calloc((size_t)(n * ld), sizeof(double));
    for (int64_t i = 0; i < n; i++) memcpy(l + i * ld, a + i * n, (size_t)n * sizeof(double));
    int64_t width = n / 8 < 32 ? 32 : (n / 8 > 128 ? 128 : n / 8);
    int64_t pl0 = stride_of(n);
    double *panel = malloc((size_t)(pl0 * width) * sizeof(double));
    int ok = 1;
    for (int64_t k0 = 0; k0 < n; k0 += width) {
        int64_t k1 = k0 + width < n ? k0 + width : n;
        int64_t nb = k1 - k0, rows = n - k0, w = n - k1, pl = stride_of(rows);
        for (int64_t j = 0; j < nb; j++)
            for (int64_t i = 0; i < rows; i++) panel[j * pl + i] = l[(k0 + i) * ld + k0 + j];
        if (!cholesky_panel(panel, rows, pl, 0, nb)) { ok = 0; break; }
        for (int64_t i = 0; i < rows; i++)
            for (int64_t j = 0; j < nb; j++) l[(k0 + i) * ld + k0 + j] = panel[j * pl + i];
        if (w == 0) break;
        view x = vtr(vrows(panel + nb, pl));
        gemm_v(l + k1 * ld + k1, ld, x, vtr(x), w, nb, w, -1.0, 1.0);
    }
    if (ok)
        for (int64_t i = 0; i < n; i++)
            for (int64_t j = 0; j < n; j++) out[i * n + j] = j <= i ? l[i * ld + j] : 0.0;
    free(panel);
    free(l);
    return ok;
}

int ora_regular(int64_t n, const double *a, const double *factors) {
    if (n == 0) return 0;
    double top = greatest_abs(a, n * n, 1);
    double negligible = DBL_EPSILON * (double)n * top;
    for (int64_t i = 0; i < n; i++)
        if (fabs(factors[i * n + i]) <= negligible) return 0;
    return 1;
}

int ora_solve(int64_t n, const double *a, const double *b, int64_t k, double *x) {
    if (n == 0) return 1;
    double *f = malloc((size_t)(n * n) * sizeof(double));
    int64_t *perm = malloc((size_t)n * sizeof(int64_t));
    ora_lu_factor(n, a, f, perm);
    int ok = ora_regular(n, a, f);
    if (ok) ora_lu_solve(n, f, perm, b, k, x);
    free(perm);
    free(f);
    return ok ? 0 : 1;
}

/* ---------------------------------------------------------------- error measures */

static inline void two_sum(double a, double b, double *s, double *e) {
    double x = a + b, z = x - a;
    *s = x;
    *e = (a - (x - z)) + (b - z);
}

void ora_residual_dd(int64_t n, const double *a, const double *x, const double *b, int64_t k, double *r) {
    #pragma omp parallel for schedule(static) num_threads(ora_get_threads())
    for (int64_t i = 0; i < n; i++) {
        for (int64_t c = 0; c < k; c++) {
            double hi = b[i * k + c], lo = 0.0;
            for (int64_t j = 0; j < n; j++) {
                double p = -a[i * n + j] * x[j * k + c];
                double pe = fma(-a[i * n + j], x[j * k + c], -p);
                double s, e;
                two_sum(hi, p, &s, &e);
                hi = s;
                lo = lo + (e + pe);
            }
            r[i * k + c] = hi + lo;
        }
    }
}

double ora_backward_error(int64_t n, const double *a, const double *x, const double *b, int64_t k) {
    if (n == 0 || k == 0) return 0.0;
    double *r = malloc((size_t)(n * k) * sizeof(double));
    ora_residual_dd(n, a, x, b, k, r);
    double anorm = 0.0;
    for (int64_t i = 0; i < n; i++) {
        double s = 0.0;
        for (int64_t j = 0; j < n; j++) s += fabs(a[i * n + j]);
        if (s > anorm) anorm = s;
    }
    double worst = 0.0;
    for (int64_t c = 0; c < k; c++) {
        double rn = 0.0, xn = 0.0, bn = 0.0;
        for (int64_t i = 0; i < n; i++) {
            if (fabs(r[i * k + c]) > rn) rn = fabs(r[i * k + c]);
            if (fabs(x[i * k + c]) > xn) xn = fabs(x[i * k + c]);
            if (fabs(b[i * k + c]) > bn) bn = fabs(b[i * k + c]);
        }
        double den = anorm * xn + bn;
        double e = den > 0.0 ? rn / den : rn;
        if (e > worst || e != e) worst = e;
    }
    free(r);
    return worst;
}
