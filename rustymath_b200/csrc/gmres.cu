// GMRES-based iterative refinement (GMRES-IR) for the mixed-precision solve: the stage
// between classical refinement and the float64 fallback.
//
// When classical refinement x += (LU)^-1 r stalls (kappa(A) times float32's unit roundoff near
// or above 1), the float32 factors can still precondition GMRES: each outer step forms
// r = b - A x in float64, solves A d = r by GMRES on the right-preconditioned system
// A (LU)^-1 u = r, d = (LU)^-1 u, in float64 (the products with the float64 A, the
// preconditioner through the float32 factors), and updates x += d; the backward error is
// tested after every outer step, as classical refinement tests it. Right preconditioning
// makes the minimized residual the true one, r - A d: with (LU)^-1 as large as kappa(A), a
// left-preconditioned residual would say little about it. The preconditioner is applied in
// float32, so it is not exactly the same linear map on every vector; the flexible variant
// (FGMRES) keeps each Z_j = (LU)^-1 V_j and forms d = Z y, which the Arnoldi relation
// A Z_j = sum h_ij V_i holds for exactly as computed. The k right-hand sides run
// in lockstep: their Krylov bases are n x k blocks, one product A V_j serves all of them, and
// each column keeps its own Hessenberg matrix and Givens rotations on the host. Orthogonali-
// zation is classical Gram-Schmidt applied twice (CGS2), so each Arnoldi step is two
// reductions over all previous basis blocks rather than j dependent ones.
//
// rustymath's own GMRES (core/src/optimize.rs) is a general iterative solver; this follows
// the published GMRES-IR scheme (Carson and Higham) for the refinement of a low-precision LU.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "rm_internal.h"

namespace rm {
namespace gm {

constexpr int COLS = 32;          // columns per reduction pass
constexpr int ROWS = 256 / COLS;  // rows a block covers per pass

// part[i][blk][c] = sum over this block's rows of V_i[r][g0 + c] * W[r][g0 + c] (row-major n x k
// blocks, V_i at V + i * vstride): fixed-order partial sums, reduced by coldot_final_kernel.
__global__ void __launch_bounds__(256) coldot_kernel(const double* __restrict__ V, int64_t vstride,
                                                     const double* __restrict__ W, int64_t n, int k, int g0,
                                                     double* __restrict__ part) {
  __shared__ double red[ROWS][COLS];
  const int i = blockIdx.y;
  const int c = threadIdx.x % COLS, rl = threadIdx.x / COLS;
  const int col = g0 + c;
  const double* v = V + (int64_t)i * vstride;
  double acc = 0.0;
  if (col < k)
    for (int64_t r = (int64_t)blockIdx.x * ROWS + rl; r < n; r += (int64_t)gridDim.x * ROWS)
      acc = fma(v[r * k + col], W[r * k + col], acc);
  red[rl][c] = acc;
  __syncthreads();
  if (rl == 0) {
    double s = 0.0;
    for (int q = 0; q < ROWS; ++q) s += red[q][c];
    part[((int64_t)i * gridDim.x + blockIdx.x) * COLS + c] = s;
  }
}

// out[i * k + g0 + c] = sum over blocks of part[i][blk][c], in block order
__global__ void coldot_final_kernel(const double* __restrict__ part, int blocks, int nv, int k, int g0,
                                    double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nv * COLS) return;
  const int i = t / COLS, c = t % COLS;
  if (g0 + c >= k) return;
  double s = 0.0;
  for (int b = 0; b < blocks; ++b) s += part[((int64_t)i * blocks + b) * COLS + c];
  out[(int64_t)i * k + g0 + c] = s;
}

// W[r][c] += sign * sum_{i < nv} coef[i * k + c] V_i[r][c]
__global__ void colaxpy_kernel(const double* __restrict__ V, int64_t vstride, int nv, const double* __restrict__ coef,
                               double* __restrict__ W, int64_t n, int k, double sign) {
  const int64_t total = n * k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % k);
    double s = 0.0;
    for (int i = 0; i < nv; ++i) s = fma(coef[(int64_t)i * k + c], V[(int64_t)i * vstride + e], s);
    W[e] = fma(sign, s, W[e]);
  }
}

// X[r][c] *= scale[c]
__global__ void colscale_kernel(double* __restrict__ X, const double* __restrict__ scale, int64_t n, int k) {
  const int64_t total = n * k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    X[e] *= scale[e % k];
}

}  // namespace gm

namespace {

struct Dots {
  double* part;
  int blocks;
  // out[i][c] = <V_i[:, c], W[:, c]> for i < nv
  int run(const double* V, int64_t vstride, int nv, const double* W, int64_t n, int k, double* out,
          cudaStream_t s) const {
    for (int g0 = 0; g0 < k; g0 += gm::COLS) {
      gm::coldot_kernel<<<dim3(blocks, nv), 256, 0, s>>>(V, vstride, W, n, k, g0, part);
      RM_LAUNCHED();
      gm::coldot_final_kernel<<<(nv * gm::COLS + 255) / 256, 256, 0, s>>>(part, blocks, nv, k, g0, out);
      RM_LAUNCHED();
    }
    return RM_OK;
  }
};

int launch_blocks(int64_t total) { return (int)std::min<int64_t>((total + 255) / 256, 4 * device_sm_count()); }

}  // namespace

size_t gmres_scratch_bytes(int64_t n, int64_t k, int restart) {
  const int blocks = 2 * device_sm_count();
  return ((size_t)(2 * restart + 3) * n * k + (size_t)(restart + 1) * blocks * gm::COLS + 4 * (size_t)(restart + 2) * k +
          (size_t)n * (k + 1) + 2) *
             sizeof(double) +
         1024;
}

int gmres_ir(const double* a, int64_t n, const double* b, int64_t k, double* x, const Precond& pc, int restart,
             int max_outer, double tol, double* berr_out, int* outer_out, void* scratch, double* r, double* norms,
             double* berr_dev, cudaStream_t s) {
  const int m = std::max(1, restart);
  double* V = reinterpret_cast<double*>(scratch);  // (m + 1) blocks of n x k
  const int64_t vs = n * k;
  double* W = V + (size_t)(m + 1) * vs;
  double* Z = W + vs;  // m blocks: Z_j = (LU)^-1 V_j
  double* D = Z + (size_t)m * vs;  // the update
  Dots dots;
  dots.blocks = 2 * device_sm_count();
  dots.part = D + vs;
  double* hdev = dots.part + (size_t)(m + 1) * dots.blocks * gm::COLS;  // (m + 1) x k
  double* h2dev = hdev + (size_t)(m + 1) * k;
  double* scl = h2dev + (size_t)(m + 1) * k;  // k
  // A V_j: TMA needs 16-byte aligned rows of V_j, so a block of odd width (or at an odd
  // offset) goes through a copy with an even row length first
  const int64_t kp = (k + 1) & ~int64_t(1);
  double* vpad = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(scl + k) + 15) & ~uintptr_t(15));
  // and A's rows too: an odd n (or an unaligned A) is copied once to an even row length
  double* apad = nullptr;
  int64_t lda = n;
  if ((reinterpret_cast<uintptr_t>(a) & 15) || (n & 1)) {
    lda = n + 1;
    RM_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&apad), (size_t)n * lda * sizeof(double), s));
    RM_CUDA_TRY(cudaMemcpy2DAsync(apad, lda * sizeof(double), a, n * sizeof(double), n * sizeof(double), n,
                                  cudaMemcpyDeviceToDevice, s));
  }
  struct Free {
    double* p;
    cudaStream_t s;
    ~Free() {
      if (p) cudaFreeAsync(p, s);
    }
  } free_apad{apad, s};
  const double* am = apad ? apad : a;
  auto matvec = [&](const double* vj, double* w) -> int {
    const bool aligned = (reinterpret_cast<uintptr_t>(vj) & 15) == 0 && (k % 2) == 0;
    if (aligned) return dgemm_device(false, false, n, k, n, 1.0, am, lda, vj, k, 0.0, w, k, device_status(), s);
    RM_CUDA_TRY(cudaMemcpy2DAsync(vpad, kp * sizeof(double), vj, k * sizeof(double), k * sizeof(double), n,
                                  cudaMemcpyDeviceToDevice, s));
    return dgemm_device(false, false, n, k, n, 1.0, am, lda, vpad, kp, 0.0, w, k, device_status(), s);
  };
  std::vector<double> H((size_t)(m + 1) * m * k), g((size_t)(m + 1) * k), cs((size_t)m * k), sn((size_t)m * k);
  std::vector<double> hh((size_t)(m + 1) * k), beta(k), y((size_t)m * k);
  double prev = INFINITY, berr = INFINITY;
  int outer = 0;
  const int grid = launch_blocks(vs);
  static const bool trace = std::getenv("RM_TRACE") != nullptr;
  for (;; ++outer) {
    RM_TRY(residual_f64(a, n, n, x, k, b, k, k, r, k, norms, s));
    RM_TRY(backward_error_f64(x, k, n, k, norms, berr_dev, s));
    RM_CUDA_TRY(cudaMemcpyAsync(&berr, berr_dev, sizeof berr, cudaMemcpyDeviceToHost, s));
    RM_TRY(take_device_status(s));
    if (trace) std::fprintf(stderr, "  gmres-ir outer %d: backward error %.3e\n", outer, berr);
    // each restart cycle must make some progress (GMRES is slow, not stalled, while it does)
    if (berr <= tol || !(berr < 0.9 * prev) || outer == max_outer) break;
    prev = berr;
    // V_0 = r / beta
    RM_CUDA_TRY(cudaMemcpyAsync(V, r, vs * sizeof(double), cudaMemcpyDeviceToDevice, s));
    RM_TRY(dots.run(V, vs, 1, V, n, k, hdev, s));
    RM_CUDA_TRY(cudaMemcpyAsync(beta.data(), hdev, k * sizeof(double), cudaMemcpyDeviceToHost, s));
    RM_CUDA_TRY(cudaStreamSynchronize(s));
    for (int c = 0; c < k; ++c) {
      beta[c] = std::sqrt(beta[c]);
      hh[c] = beta[c] > 0.0 ? 1.0 / beta[c] : 0.0;
      g[c] = beta[c];
      for (int j = 1; j <= m; ++j) g[(size_t)j * k + c] = 0.0;
    }
    RM_CUDA_TRY(cudaMemcpyAsync(scl, hh.data(), k * sizeof(double), cudaMemcpyHostToDevice, s));
    gm::colscale_kernel<<<grid, 256, 0, s>>>(V, scl, n, (int)k);
    RM_LAUNCHED();
    int steps = 0;
    for (int j = 0; j < m; ++j) {
      // W = A Z_j, Z_j = M^-1 V_j, orthogonalized against V_0..V_j twice
      RM_TRY(pc.apply(V + (size_t)j * vs, Z + (size_t)j * vs, k, s));
      RM_TRY(matvec(Z + (size_t)j * vs, W));
      RM_TRY(dots.run(V, vs, j + 1, W, n, k, hdev, s));
      gm::colaxpy_kernel<<<grid, 256, 0, s>>>(V, vs, j + 1, hdev, W, n, (int)k, -1.0);
      RM_LAUNCHED();
      RM_TRY(dots.run(V, vs, j + 1, W, n, k, h2dev, s));
      gm::colaxpy_kernel<<<grid, 256, 0, s>>>(V, vs, j + 1, h2dev, W, n, (int)k, -1.0);
      RM_LAUNCHED();
      RM_TRY(dots.run(W, 0, 1, W, n, k, h2dev + (size_t)(j + 1) * k, s));
      std::vector<double> h1((size_t)(j + 1) * k), h2((size_t)(j + 2) * k);
      RM_CUDA_TRY(cudaMemcpyAsync(h1.data(), hdev, h1.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
      RM_CUDA_TRY(cudaMemcpyAsync(h2.data(), h2dev, h2.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
      RM_CUDA_TRY(cudaStreamSynchronize(s));
      bool done = true;
      for (int c = 0; c < k; ++c) {
        double* Hc = &H[0];
        auto Hat = [&](int i, int jj) -> double& { return Hc[((size_t)i * m + jj) * k + c]; };
        for (int i = 0; i <= j; ++i) Hat(i, j) = h1[(size_t)i * k + c] + h2[(size_t)i * k + c];
        const double hn = std::sqrt(h2[(size_t)(j + 1) * k + c]);
        Hat(j + 1, j) = hn;
        hh[c] = hn > 0.0 ? 1.0 / hn : 0.0;
        for (int i = 0; i < j; ++i) {  // earlier rotations
          const double t0 = Hat(i, j), t1 = Hat(i + 1, j);
          Hat(i, j) = cs[(size_t)i * k + c] * t0 + sn[(size_t)i * k + c] * t1;
          Hat(i + 1, j) = -sn[(size_t)i * k + c] * t0 + cs[(size_t)i * k + c] * t1;
        }
        const double p = Hat(j, j), q = Hat(j + 1, j);
        const double rr = std::hypot(p, q);
        const double cj = rr > 0.0 ? p / rr : 1.0, sj = rr > 0.0 ? q / rr : 0.0;
        cs[(size_t)j * k + c] = cj, sn[(size_t)j * k + c] = sj;
        Hat(j, j) = rr, Hat(j + 1, j) = 0.0;
        const double gj = g[(size_t)j * k + c];
        g[(size_t)j * k + c] = cj * gj;
        g[(size_t)(j + 1) * k + c] = -sj * gj;
        if (std::fabs(g[(size_t)(j + 1) * k + c]) > 1e-12 * beta[c]) done = false;
      }
      steps = j + 1;
      if (trace)
        std::fprintf(stderr, "    arnoldi %d: |g| %.3e (column 0, beta %.3e)\n", j, std::fabs(g[(size_t)(j + 1) * k]),
                     beta[0]);
      if (done || j + 1 == m) break;
      // V_{j+1} = W / ||W||
      RM_CUDA_TRY(cudaMemcpyAsync(scl, hh.data(), k * sizeof(double), cudaMemcpyHostToDevice, s));
      RM_CUDA_TRY(cudaMemcpyAsync(V + (size_t)(j + 1) * vs, W, vs * sizeof(double), cudaMemcpyDeviceToDevice, s));
      gm::colscale_kernel<<<grid, 256, 0, s>>>(V + (size_t)(j + 1) * vs, scl, n, (int)k);
      RM_LAUNCHED();
    }
    // y = H^-1 g (upper triangular, per column); x += V y
    for (int c = 0; c < k; ++c)
      for (int i = steps - 1; i >= 0; --i) {
        double t = g[(size_t)i * k + c];
        for (int jj = i + 1; jj < steps; ++jj) t -= H[((size_t)i * m + jj) * k + c] * y[(size_t)jj * k + c];
        const double d = H[((size_t)i * m + i) * k + c];
        y[(size_t)i * k + c] = d != 0.0 ? t / d : 0.0;
      }
    // x += Z y
    RM_CUDA_TRY(cudaMemcpyAsync(hdev, y.data(), (size_t)steps * k * sizeof(double), cudaMemcpyHostToDevice, s));
    gm::colaxpy_kernel<<<grid, 256, 0, s>>>(Z, vs, steps, hdev, x, n, (int)k, 1.0);
    RM_LAUNCHED();
  }
  *berr_out = berr;
  *outer_out = outer;
  return RM_OK;
}

}  // namespace rm
