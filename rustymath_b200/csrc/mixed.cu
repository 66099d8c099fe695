// The mixed-precision solve: float32 LU on the tensor cores with block-local partial
// pivoting, then float64 iterative refinement on the device.
//
// rustymath's solve (core/src/linalg/factor.rs:207-209, 279) factors in the working
// precision with partial pivoting. Here the factorization runs in float32 and float64
// refinement (residual r = b - A x from the original float64 A) brings the normwise backward
// error down to n * 2^-53, the bar of the plain float64 path; when refinement stalls, the
// caller falls back to the plain float64 LU.
//
// On a GPU an LU's critical path is its pivot searches: partial pivoting reduces each column
// over every row below the diagonal, n dependent reductions across the whole device. This
// factorization chooses each pivot among a window of rows instead: a 128-column panel
// pivots among its own 256 rows (the rest of its diagonal block and the next block). A
// panel then lives in one CTA's shared memory and every pivot search is a CTA-local
// reduction. On matrices with randomly mixed rows (the single-system configuration) its
// float32 backward error matches full partial pivoting's (~1e-6 at n = 1024..2048, against
// ~1e-3 without pivoting); on a matrix that needs pivots from far away, refinement stalls
// and the fallback answers.
//
// Per 128-column panel at J0 (T = min(256, n - J0) rows):
//   lpp_panel_kernel : GEPP of the T x 128 panel among its T rows, in 32-column leaves with
//                      a shared-memory block update between leaves; writes L11^-1,
//                      (U11^-1)^T and the panel's row permutation
//   lpp_apply_kernel : that permutation on every other column of rows J0..J0+T, A12^T into
//                      a buffer, and the global permutation
//   sgemm_tc         : U12^T = A12^T (L11^-1)^T, written both to a buffer and over A12
//   sgemm_tc         : L21 = A21 U11^-1 for the rows below the panel, in place
//   sgemm_tc         : A22 -= L21 U12
// All products are 3xTF32 (float32-level) on tcgen05 with TMEM accumulators.
#include <climits>

#include "rm_internal.h"

namespace rm {

constexpr int kLppCols = 128;  // panel width (the trailing update's rank)
constexpr int kLppRows = 256;  // rows a panel's pivots are chosen among
constexpr int kLppLeaf = 32;
constexpr int kLppThreads = 256;
constexpr int kLppStride = kLppCols + 1;

__device__ __forceinline__ void warp_argmax_f32(float& v, int& i) {
#pragma unroll
  for (int off = 16; off; off >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, v, off);
    const int oi = __shfl_xor_sync(0xffffffffu, i, off);
    if (ov > v || (ov == v && oi < i)) {
      v = ov;
      i = oi;
    }
  }
}

// float32 copy of the n x n row-major float64 a, leading dimension ldf (padding zeroed)
__global__ void to_f32_kernel(const double* __restrict__ a, int64_t lda, int64_t n, float* __restrict__ f,
                              int64_t ldf) {
  const int64_t total = n * ldf;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / ldf, j = e - i * ldf;
    f[e] = j < n ? (float)__ldcs(a + i * lda + j) : 0.0f;
  }
}

// ------------------------------------------------------------------ the panel
// Factors the T x nb panel A[j0.., j0..] (T <= 256, nb <= 128) with partial pivoting among
// its T rows: thread r owns row r for the pivot search and the rank-1 updates. Within a
// 32-column leaf each column takes one pivot search (warp argmax, first row on ties, NaN
// never chosen) and a rank-1 update of the leaf; after a leaf, the panel's later columns are
// updated with a register-blocked shared-memory product. Writes the panel back, plocal[i] =
// the panel row that row i came from, linv = L11^-1 and uinvt = (U11^-1)^T (ld 128). A zero
// pivot sets RM_DEV_NAN and leaves its column unreduced.
__global__ void __launch_bounds__(kLppThreads) lpp_panel_kernel(float* __restrict__ a, int64_t lda, int j0, int nb,
                                                                int T, float* __restrict__ linv,
                                                                float* __restrict__ uinvt, int* __restrict__ plocal,
                                                                unsigned* status) {
  extern __shared__ float sm[];
  float(*P)[kLppStride] = reinterpret_cast<float(*)[kLppStride]>(sm);
  float(*X)[kLppStride] = reinterpret_cast<float(*)[kLppStride]>(sm + kLppRows * kLppStride);
  float(*Tm)[33] = reinterpret_cast<float(*)[33]>(sm + (kLppRows + kLppCols) * kLppStride);
  __shared__ int perm_s[kLppRows];
  __shared__ float red_v[kLppThreads / 32];
  __shared__ int red_i[kLppThreads / 32];
  __shared__ int piv_row;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float* blk = a + (int64_t)j0 * lda + j0;
  for (int e = tid; e < kLppRows * kLppCols; e += kLppThreads) {
    const int r = e / kLppCols, c = e % kLppCols;
    P[r][c] = (r < T && c < nb) ? blk[(int64_t)r * lda + c] : (r == c ? 1.0f : 0.0f);
  }
  perm_s[tid] = tid;
  __syncthreads();

  for (int l = 0; l < nb; l += kLppLeaf) {
    const int lend = min(l + kLppLeaf, nb);
    for (int c = l; c < lend; ++c) {
      float v = (tid >= c && tid < T) ? fabsf(P[tid][c]) : -1.0f;
      int idx = tid;
      warp_argmax_f32(v, idx);
      if (lane == 0) {
        red_v[warp] = v;
        red_i[warp] = idx;
      }
      __syncthreads();
      if (warp == 0) {
        v = lane < kLppThreads / 32 ? red_v[lane] : -1.0f;
        idx = lane < kLppThreads / 32 ? red_i[lane] : INT_MAX;
        warp_argmax_f32(v, idx);
        if (lane == 0) piv_row = v < 0.0f ? c : idx;  // every candidate NaN: keep the diagonal
      }
      __syncthreads();
      const int p = piv_row;
      if (p != c) {
        if (tid < kLppCols) {
          const float t = P[c][tid];
          P[c][tid] = P[p][tid];
          P[p][tid] = t;
        }
        if (tid == 0) {
          const int t = perm_s[c];
          perm_s[c] = perm_s[p];
          perm_s[p] = t;
        }
      }
      __syncthreads();
      const float piv = P[c][c];
      if (piv != 0.0f) {
        if (tid > c && tid < T) {
          const float lv = P[tid][c] * (1.0f / piv);
          P[tid][c] = lv;
          for (int cc = c + 1; cc < lend; ++cc) P[tid][cc] = fmaf(-lv, P[c][cc], P[tid][cc]);
        }
      } else if (tid == 0) {
        flag_error(status, RM_DEV_NAN);
      }
      __syncthreads();
    }
    if (lend < nb) {
      // rows l..lend-1 of the later columns: substitution with the leaf's unit lower block
      for (int cc = lend + tid; cc < nb; cc += kLppThreads)
        for (int i = l + 1; i < lend; ++i) {
          float s = P[i][cc];
          for (int q = l; q < i; ++q) s = fmaf(-P[i][q], P[q][cc], s);
          P[i][cc] = s;
        }
      __syncthreads();
      // rows lend..T-1 of the later columns -= L(rows, leaf) U(leaf, columns)
      const int ty = tid >> 4, tx = tid & 15;
      constexpr int RI = kLppRows / 16, CJ = kLppCols / 16;
      float acc[RI][CJ];
#pragma unroll
      for (int i = 0; i < RI; ++i)
#pragma unroll
        for (int j = 0; j < CJ; ++j) acc[i][j] = 0.0f;
      for (int q = l; q < lend; ++q) {
        float rv[RI], cv[CJ];
#pragma unroll
        for (int i = 0; i < RI; ++i) {
          const int r = lend + ty + 16 * i;
          rv[i] = r < T ? P[r][q] : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < CJ; ++j) {
          const int cc = lend + tx + 16 * j;
          cv[j] = cc < nb ? P[q][cc] : 0.0f;
        }
#pragma unroll
        for (int i = 0; i < RI; ++i)
#pragma unroll
          for (int j = 0; j < CJ; ++j) acc[i][j] = fmaf(rv[i], cv[j], acc[i][j]);
      }
#pragma unroll
      for (int i = 0; i < RI; ++i)
#pragma unroll
        for (int j = 0; j < CJ; ++j) {
          const int r = lend + ty + 16 * i, cc = lend + tx + 16 * j;
          if (r < T && cc < nb) P[r][cc] -= acc[i][j];
        }
      __syncthreads();
    }
  }
  for (int e = tid; e < T * nb; e += kLppThreads) {
    const int r = e / nb, c = e % nb;
    blk[(int64_t)r * lda + c] = P[r][c];
  }
  if (tid < T) plocal[tid] = perm_s[tid];

  // ---- L11^-1 (unit lower) into X: 32x32 diagonal blocks by column substitution (a warp
  // each, a lane per column), the blocks below them in order of distance from the diagonal
  for (int e = tid; e < kLppCols * kLppCols; e += kLppThreads) X[e / kLppCols][e % kLppCols] = 0.0f;
  __syncthreads();
  if (warp < 4) {
    const int b0 = warp * 32;
    float x[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      float s = i == lane ? 1.0f : 0.0f;
#pragma unroll
      for (int k2 = 0; k2 < i; ++k2) s = fmaf(-P[b0 + i][b0 + k2], x[k2], s);
      x[i] = i < lane ? 0.0f : s;
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) X[b0 + i][b0 + lane] = x[i];
  }
  __syncthreads();
  for (int gap = 1; gap < 4; ++gap)
    for (int ab = 0; ab + gap < 4; ++ab) {
      const int rb = (ab + gap) * 32, ca = ab * 32;
      for (int e = tid; e < 1024; e += kLppThreads) {  // Tm = sum_{c=a..b-1} L_bc X_ca
        const int i = e >> 5, j = e & 31;
        float s = 0.0f;
        for (int k2 = ca; k2 < rb; ++k2) s = fmaf(P[rb + i][k2], X[k2][ca + j], s);
        Tm[i][j] = s;
      }
      __syncthreads();
      for (int e = tid; e < 1024; e += kLppThreads) {  // X_ba = -D_b^-1 Tm
        const int i = e >> 5, j = e & 31;
        float s = 0.0f;
        for (int k2 = 0; k2 <= i; ++k2) s = fmaf(X[rb + i][rb + k2], Tm[k2][j], s);
        X[rb + i][ca + j] = -s;
      }
      __syncthreads();
    }
  for (int e = tid; e < kLppCols * kLppCols; e += kLppThreads) linv[e] = X[e / kLppCols][e % kLppCols];
  __syncthreads();
  // ---- U11^-1 (upper) into X, written transposed
  for (int e = tid; e < kLppCols * kLppCols; e += kLppThreads) X[e / kLppCols][e % kLppCols] = 0.0f;
  __syncthreads();
  if (warp < 4) {
    const int b0 = warp * 32;
    float x[32];
#pragma unroll
    for (int i = 31; i >= 0; --i) {
      float s = i == lane ? 1.0f : 0.0f;
#pragma unroll
      for (int k2 = i + 1; k2 < 32; ++k2) s = fmaf(-P[b0 + i][b0 + k2], x[k2], s);
      x[i] = i > lane ? 0.0f : s / P[b0 + i][b0 + i];
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) X[b0 + i][b0 + lane] = x[i];
  }
  __syncthreads();
  for (int gap = 1; gap < 4; ++gap)
    for (int ab = 0; ab + gap < 4; ++ab) {
      const int ra = ab * 32, cb = (ab + gap) * 32;
      for (int e = tid; e < 1024; e += kLppThreads) {  // Tm = sum_{c=a+1..b} U_ac X_cb
        const int i = e >> 5, j = e & 31;
        float s = 0.0f;
        for (int k2 = ra + 32; k2 < cb + 32; ++k2) s = fmaf(P[ra + i][k2], X[k2][cb + j], s);
        Tm[i][j] = s;
      }
      __syncthreads();
      for (int e = tid; e < 1024; e += kLppThreads) {  // X_ab = -D_a^-1 Tm
        const int i = e >> 5, j = e & 31;
        float s = 0.0f;
        for (int k2 = i; k2 < 32; ++k2) s = fmaf(X[ra + i][ra + k2], Tm[k2][j], s);
        X[ra + i][cb + j] = -s;
      }
      __syncthreads();
    }
  for (int e = tid; e < kLppCols * kLppCols; e += kLppThreads) uinvt[e] = X[e % kLppCols][e / kLppCols];
}

constexpr size_t kLppSmem = ((size_t)(kLppRows + kLppCols) * kLppStride + 32 * 33) * sizeof(float);

// ------------------------------------------------------------------ the panel's row permutation
constexpr int kApplyCols = 32;

// Rows j0..j0+T of the columns [0, j0) and [j1, n) take the panel's permutation (new row i =
// old row plocal[i]); for columns >= j1 the first nb new rows also go, transposed, to a12t
// (ld 128). Block 0 also permutes perm[j0..j0+T).
__global__ void __launch_bounds__(256) lpp_apply_kernel(float* __restrict__ a, int64_t lda, int n, int j0, int j1,
                                                        int T, const int* __restrict__ plocal, float* __restrict__ a12t,
                                                        int* __restrict__ perm) {
  __shared__ float buf[kLppRows][kApplyCols + 1];
  __shared__ int pl[kLppRows];
  const int tid = threadIdx.x;
  if (tid < T) pl[tid] = plocal[tid];
  __syncthreads();
  const int left_chunks = (j0 + kApplyCols - 1) / kApplyCols;
  int c0, c1;
  bool right;
  if ((int)blockIdx.x < left_chunks) {
    c0 = blockIdx.x * kApplyCols;
    c1 = min(c0 + kApplyCols, j0);
    right = false;
  } else {
    c0 = j1 + (blockIdx.x - left_chunks) * kApplyCols;
    c1 = min(c0 + kApplyCols, n);
    right = true;
  }
  const int w = c1 - c0;
  if (w > 0) {
    for (int e = tid; e < T * kApplyCols; e += 256) {
      const int r = e / kApplyCols, c = e % kApplyCols;
      if (c < w) buf[r][c] = a[(int64_t)(j0 + pl[r]) * lda + c0 + c];
    }
    __syncthreads();
    for (int e = tid; e < T * kApplyCols; e += 256) {
      const int r = e / kApplyCols, c = e % kApplyCols;
      if (c < w && pl[r] != r) a[(int64_t)(j0 + r) * lda + c0 + c] = buf[r][c];
    }
    if (right) {
      const int nb = j1 - j0;
      for (int e = tid; e < nb * kApplyCols; e += 256) {
        const int c = e / nb, r = e % nb;  // consecutive threads: consecutive rows of a12t's row
        if (c < w) a12t[(int64_t)(c0 - j1 + c) * kLppCols + r] = buf[r][c];
      }
    }
  }
  if (blockIdx.x == 0) {
    __syncthreads();
    const int v = tid < T ? perm[j0 + pl[tid]] : 0;
    __syncthreads();
    if (tid < T) perm[j0 + tid] = v;
  }
}

__global__ void iota32_kernel(int* p, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = (int)i;
}

size_t getrf_lpp_f32_scratch_bytes(int64_t n) {
  return (2 * (size_t)kLppCols * kLppCols + 2 * (size_t)n * kLppCols) * sizeof(float) + kLppRows * sizeof(int) +
         2048;
}

int getrf_lpp_f32(float* a, int64_t lda, int64_t n, int* perm, void* scratch, unsigned* status, cudaStream_t stream) {
  if (n <= 0) return RM_OK;
  if (n > INT32_MAX / 2) return RM_BAD_ARG;
  float* linv = reinterpret_cast<float*>(scratch);
  float* uinvt = linv + kLppCols * kLppCols;
  float* a12t = uinvt + kLppCols * kLppCols;   // rest x 128: A12^T
  float* u12t = a12t + (size_t)n * kLppCols;   // rest x 128: U12^T
  int* plocal = reinterpret_cast<int*>(u12t + (size_t)n * kLppCols);
  static bool set = false;
  if (!set) {
    RM_CUDA_TRY(cudaFuncSetAttribute(lpp_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLppSmem));
    set = true;
  }
  iota32_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 1024), 256, 0, stream>>>(perm, n);
  RM_LAUNCHED();
  const int ni = (int)n;
  for (int J0 = 0; J0 < ni; J0 += kLppCols) {
    const int nb = std::min(kLppCols, ni - J0);
    const int T = std::min(kLppRows, ni - J0);
    const int J1 = J0 + nb;
    const int rest = ni - J1;
    lpp_panel_kernel<<<1, kLppThreads, kLppSmem, stream>>>(a, lda, J0, nb, T, linv, uinvt, plocal, status);
    RM_LAUNCHED();
    const int chunks = (J0 + kApplyCols - 1) / kApplyCols + (rest + kApplyCols - 1) / kApplyCols;
    lpp_apply_kernel<<<std::max(chunks, 1), 256, 0, stream>>>(a, lda, ni, J0, J1, T, plocal, a12t, perm);
    RM_LAUNCHED();
    if (rest == 0) break;
    float* a12 = a + (int64_t)J0 * lda + J1;
    // U12^T = A12^T (L11^-1)^T, also written transposed over A12
    RM_TRY(sgemm_tc(3, rest, nb, nb, 1.0f, a12t, kLppCols, linv, kLppCols, 0.0f, u12t, kLppCols, status, stream, a12,
                    lda));
    // L21 = A21 U11^-1 for the rows below the panel (the panel's own rows are done), in place
    const int below = ni - (J0 + T);
    if (below > 0) {
      float* a21b = a + (int64_t)(J0 + T) * lda + J0;
      RM_TRY(sgemm_tc(3, below, nb, nb, 1.0f, a21b, lda, uinvt, kLppCols, 0.0f, a21b, lda, status, stream));
    }
    // A22 -= L21 U12
    RM_TRY(sgemm_tc(3, rest, rest, nb, -1.0f, a + (int64_t)J1 * lda + J0, lda, u12t, kLppCols, 1.0f,
                    a + (int64_t)J1 * lda + J1, lda, status, stream));
  }
  return RM_OK;
}

// ------------------------------------------------------------------ refinement helpers

int to_f32(const double* a, int64_t lda, int64_t n, float* f, int64_t ldf, cudaStream_t stream) {
  if (n == 0) return RM_OK;
  const int blocks = (int)std::min<int64_t>((n * ldf + 255) / 256, 8 * device_sm_count());
  to_f32_kernel<<<blocks, 256, 0, stream>>>(a, lda, n, f, ldf);
  RM_LAUNCHED();
  return RM_OK;
}

// c (float32, n x k) = r[perm] (float64 rows gathered and rounded)
__global__ void gather_f32_kernel(const double* __restrict__ r, int64_t ldr, const int* __restrict__ perm, int64_t n,
                                  int64_t k, float* __restrict__ c, int64_t ldc) {
  const int64_t total = n * k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / k, j = e - i * k;
    c[i * ldc + j] = (float)r[(int64_t)perm[i] * ldr + j];
  }
}

// x (float64) = c (assign) or x += c
__global__ void accumulate_kernel(const float* __restrict__ c, int64_t ldc, int64_t n, int64_t k, double* __restrict__ x,
                                  int64_t ldx, bool assign) {
  const int64_t total = n * k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / k, j = e - i * k;
    const double d = (double)c[i * ldc + j];
    double* p = x + i * ldx + j;
    *p = assign ? d : *p + d;
  }
}

int gather_f32(const double* r, int64_t ldr, const int* perm, int64_t n, int64_t k, float* c, int64_t ldc,
               cudaStream_t stream) {
  if (n * k == 0) return RM_OK;
  gather_f32_kernel<<<(int)std::min<int64_t>((n * k + 255) / 256, 4 * device_sm_count()), 256, 0, stream>>>(
      r, ldr, perm, n, k, c, ldc);
  RM_LAUNCHED();
  return RM_OK;
}

int accumulate_f64(const float* c, int64_t ldc, int64_t n, int64_t k, double* x, int64_t ldx, bool assign,
                   cudaStream_t stream) {
  if (n * k == 0) return RM_OK;
  accumulate_kernel<<<(int)std::min<int64_t>((n * k + 255) / 256, 4 * device_sm_count()), 256, 0, stream>>>(
      c, ldc, n, k, x, ldx, assign);
  RM_LAUNCHED();
  return RM_OK;
}

}  // namespace rm
