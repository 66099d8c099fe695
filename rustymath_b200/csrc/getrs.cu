// Triangular solves with the LU factors: x = U^-1 L^-1 P b (and the transposed form).
//
// Replaces lu_solve and the native triangular solves (core/src/linalg/factor.rs:633-641,
// 668-748). The reference substitutes row by row within 16/32-row leaves and removes
// solved halves with GEMMs. On the GPU each 64-row block row of the triangle belongs to
// one CTA. A CTA takes a ticket (an atomic counter, so tickets follow the order in which
// CTAs start and every dependency is held by a CTA that is already running), subtracts
// the products of its block row of L (or U) with each already-solved block of x as soon as
// that block's flag is set, then multiplies by the inverse of its diagonal block (computed
// once per factorization by invert_diag_blocks) and publishes its block with a release
// flag. Waits on flags are bounded: on expiry the status word records a timeout.
#include "rm_internal.h"

namespace rm {

constexpr int kTB = kSolveBlock;  // rows of a block row
constexpr int kKC = kSolveCols;   // right-hand-side columns per launch
constexpr int kTrsvThreads = 256;

size_t diag_blocks_f64_bytes(int64_t n) { return diag_blocks_bytes_max(n); }

// dinv[b][0] = inverse of the lower diagonal block b, dinv[b][1] = inverse of the upper
// diagonal block b (row-major kTB x kTB; rows/columns past n are identity). A unit triangle
// takes its diagonal as 1 without reading it. The triangles are those of the n x n matrix
// T whose item (i, j) is w[i*ldw + j], or w[j*ldw + i] when COLMAJOR.
template <typename T, bool COLMAJOR>
__global__ void __launch_bounds__(128) invert_diag_blocks_kernel(const T* __restrict__ w, int64_t ldw, int64_t n,
                                                                 T* __restrict__ dinv, bool lower_unit, bool upper_unit) {
  __shared__ T x[kTB][kTB + 1];
  const int b = blockIdx.x, which = blockIdx.y;  // 0: L, 1: U
  const int64_t r0 = (int64_t)b * kTB;
  const int rows = (int)(n - r0 < kTB ? n - r0 : kTB);
  const T* blk = w + r0 * ldw + r0;
  const int col = threadIdx.x;  // threads 0..63 each own one column of the inverse
  auto A = [&](int i, int j) -> T {
    if (i >= rows || j >= rows) return i == j ? T(1) : T(0);
    return COLMAJOR ? blk[(int64_t)j * ldw + i] : blk[(int64_t)i * ldw + j];
  };
  if (col < kTB) {
    if (which == 0) {
      // lower: x_i = (delta_i,col - sum_{col<=k<i} L_ik x_k) / L_ii for i >= col
      for (int i = 0; i < kTB; ++i) {
        T s = i == col ? T(1) : T(0);
        if (i > col)
          for (int k = col; k < i; ++k) s = fma(-A(i, k), x[k][col], s);
        x[i][col] = i < col ? T(0) : (lower_unit ? s : s / A(i, i));
      }
    } else {
      // upper: x_i = (delta_i,col - sum_{i<k<=col} U_ik x_k) / U_ii for i <= col
      for (int i = kTB - 1; i >= 0; --i) {
        T s = i == col ? T(1) : T(0);
        if (i < col)
          for (int k = i + 1; k <= col; ++k) s = fma(-A(i, k), x[k][col], s);
        x[i][col] = i > col ? T(0) : (upper_unit ? s : s / A(i, i));
      }
    }
  }
  __syncthreads();
  T* out = dinv + ((int64_t)b * 2 + which) * kTB * kTB;
  for (int e = threadIdx.x; e < kTB * kTB; e += blockDim.x) out[e] = x[e / kTB][e % kTB];
}

int invert_diag_blocks_f64(const double* w, int64_t ldw, bool colmajor, int64_t n, double* dinv, bool lower_unit,
                           bool upper_unit, cudaStream_t stream) {
  if (n == 0) return RM_OK;
  dim3 grid((unsigned)((n + kTB - 1) / kTB), 2);
  if (colmajor)
    invert_diag_blocks_kernel<double, true><<<grid, 128, 0, stream>>>(w, ldw, n, dinv, lower_unit, upper_unit);
  else
    invert_diag_blocks_kernel<double, false><<<grid, 128, 0, stream>>>(w, ldw, n, dinv, lower_unit, upper_unit);
  RM_LAUNCHED();
  return RM_OK;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Solves T x = y for kc <= kKC columns of y (in place in x), T the lower (LOWER) or upper
// triangle of the matrix whose item (i, j) is w[i*ldw + j] (w[j*ldw + i] when COLMAJOR);
// the diagonal blocks' inverses come from dinv. flags[nblk] and counter start at zero.
// Each thread keeps kTB*kKC/kTrsvThreads of its block's running sums in registers.
template <typename T, bool LOWER, bool COLMAJOR>
__global__ void __launch_bounds__(kTrsvThreads)
    trsv_chain_kernel(const T* __restrict__ w, int64_t ldw, int n, const T* __restrict__ dinv, T* x, int64_t ldx,
                      int kc, int* flags, int* counter, unsigned* status) {
  constexpr int PER = kTB * kKC / kTrsvThreads;
  __shared__ T lblk[kTB][kTB];
  __shared__ T xs[kTB][kKC];
  __shared__ int ticket, good;
  const int tid = threadIdx.x;
  const int nblk = (n + kTB - 1) / kTB;
  if (tid == 0) ticket = atomicAdd(counter, 1);
  __syncthreads();
  const int t = ticket;
  const int b = LOWER ? t : nblk - 1 - t;
  const int r0 = b * kTB, rows = min(kTB, n - r0);

  T acc[PER];
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int e = tid + i * kTrsvThreads, r = e / kKC, c = e % kKC;
    acc[i] = (r < rows && c < kc) ? x[(int64_t)(r0 + r) * ldx + c] : T(0);
  }
  bool ok = true;
  for (int s = 0; s < t; ++s) {
    const int j = LOWER ? s : nblk - 1 - s;  // a solved block, in solve order
    const int c0 = j * kTB, cols = min(kTB, n - c0);
    __syncthreads();  // the previous step's reads of lblk / xs are done
    for (int e = tid; e < kTB * kTB; e += kTrsvThreads) {
      if (COLMAJOR) {  // coalesced along the stored column
        const int c = e / kTB, r = e % kTB;
        lblk[r][c] = (r < rows && c < cols) ? w[(int64_t)(c0 + c) * ldw + r0 + r] : T(0);
      } else {
        const int r = e / kTB, c = e % kTB;
        lblk[r][c] = (r < rows && c < cols) ? w[(int64_t)(r0 + r) * ldw + c0 + c] : T(0);
      }
    }
    if (tid == 0) {
      bool seen = ld_acquire(&flags[j]) != 0;
      if (!seen) {
        const uint64_t start = global_ns();
        while (!(seen = ld_acquire(&flags[j]) != 0)) {
          if (global_ns() - start > kWaitLimitNs) break;
          __nanosleep(32);
        }
      }
      if (!seen) flag_error(status, RM_DEV_TIMEOUT);
      good = seen ? 1 : 0;
    }
    __syncthreads();
    if (!good) {
      ok = false;
      break;
    }
    for (int e = tid; e < kTB * kKC; e += kTrsvThreads) {
      const int r = e / kKC, c = e % kKC;
      xs[r][c] = (r < cols && c < kc) ? __ldcg(&x[(int64_t)(c0 + r) * ldx + c]) : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + i * kTrsvThreads, r = e / kKC, c = e % kKC;
      T s2 = acc[i];
#pragma unroll 16
      for (int q = 0; q < kTB; ++q) s2 = fma(-lblk[r][q], xs[q][c], s2);
      acc[i] = s2;
    }
  }
  __syncthreads();
  if (ok) {
    const T* dv = dinv + ((int64_t)b * 2 + (LOWER ? 0 : 1)) * kTB * kTB;
    for (int e = tid; e < kTB * kTB; e += kTrsvThreads) lblk[e / kTB][e % kTB] = dv[e];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + i * kTrsvThreads;
      xs[e / kKC][e % kKC] = acc[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + i * kTrsvThreads, r = e / kKC, c = e % kKC;
      T s2 = T(0);
#pragma unroll 16
      for (int q = 0; q < kTB; ++q) s2 = fma(lblk[r][q], xs[q][c], s2);
      if (r < rows && c < kc) x[(int64_t)(r0 + r) * ldx + c] = s2;
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) st_release(&flags[b], 1);
}

// Row permutation of an n x k row-major matrix: x[i] = b[perm[i]] (gather), or, with
// SCATTER, x[perm[i]] = b[i]. perm == NULL copies.
// A position outside 0..n-1 (a caller's perm) sets RM_DEV_BAD_INDEX and is skipped.
template <bool SCATTER>
__global__ void permute_rows_kernel(const double* __restrict__ b, int64_t ldb, const int64_t* __restrict__ perm,
                                    int64_t n, int64_t k, double* __restrict__ x, int64_t ldx, unsigned* status) {
  const int64_t total = n * k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / k, c = e - i * k;
    const int64_t p = perm ? perm[i] : i;
    if (p < 0 || p >= n) {
      flag_error(status, RM_DEV_BAD_INDEX);
      continue;
    }
    if (SCATTER) x[p * ldx + c] = b[i * ldb + c];
    else x[i * ldx + c] = b[p * ldb + c];
  }
}

size_t getrs_f64_scratch_bytes(int64_t n, int64_t k) { return getrs_scratch_bytes_max(n, k); }

int getrs_f64(const double* lu, int64_t ld, bool lu_colmajor, int64_t n, const int64_t* perm, const double* dinv,
              const double* b, int64_t ldb, int64_t k, double* x, int64_t ldx, void* scratch, unsigned* status,
              cudaStream_t stream, bool trans) {
  if (n == 0 || k == 0) return RM_OK;
  const int nblk = (int)((n + kTB - 1) / kTB);
  const int chunks = (int)((k + kKC - 1) / kKC);
  // The solved triangle pair: L\U itself, or its transpose for A^T x = b.
  const bool colmajor = trans ? !lu_colmajor : lu_colmajor;
  // b may alias x: the permuted right-hand side goes to a temporary first
  double* tmp = reinterpret_cast<double*>(scratch);
  int* flags = reinterpret_cast<int*>(reinterpret_cast<char*>(scratch) + ((size_t)n * k * sizeof(double) + 255) / 256 * 256);
  const size_t flag_bytes = (size_t)(2 * (nblk + 1)) * sizeof(int) * (size_t)chunks;
  RM_CUDA_TRY(cudaMemsetAsync(flags, 0, flag_bytes, stream));
  const int blocks = (int)std::min<int64_t>((n * k + 255) / 256, 4 * device_sm_count());
  permute_rows_kernel<false><<<blocks, 256, 0, stream>>>(b, ldb, trans ? nullptr : perm, n, k, tmp, k, status);
  RM_LAUNCHED();
  for (int ch = 0; ch < chunks; ++ch) {
    const int kc = (int)std::min<int64_t>(kKC, k - (int64_t)ch * kKC);
    int* f = flags + (size_t)ch * 2 * (nblk + 1);
    double* xc = tmp + ch * kKC;
    if (colmajor) {
      trsv_chain_kernel<double, true, true><<<nblk, kTrsvThreads, 0, stream>>>(lu, ld, (int)n, dinv, xc, k, kc, f,
                                                                                f + nblk, status);
      RM_LAUNCHED();
      trsv_chain_kernel<double, false, true><<<nblk, kTrsvThreads, 0, stream>>>(lu, ld, (int)n, dinv, xc, k, kc,
                                                                                 f + nblk + 1, f + 2 * nblk + 1, status);
      RM_LAUNCHED();
    } else {
      trsv_chain_kernel<double, true, false><<<nblk, kTrsvThreads, 0, stream>>>(lu, ld, (int)n, dinv, xc, k, kc, f,
                                                                                 f + nblk, status);
      RM_LAUNCHED();
      trsv_chain_kernel<double, false, false><<<nblk, kTrsvThreads, 0, stream>>>(lu, ld, (int)n, dinv, xc, k, kc,
                                                                                  f + nblk + 1, f + 2 * nblk + 1, status);
      RM_LAUNCHED();
    }
  }
  permute_rows_kernel<true><<<blocks, 256, 0, stream>>>(tmp, k, trans ? perm : nullptr, n, k, x, ldx, status);
  RM_LAUNCHED();
  return RM_OK;
}

// ------------------------------------------------------------------ float32, no pivoting

size_t diag_blocks_f32_bytes(int64_t n) { return diag_blocks_bytes_max(n) / 2; }

int invert_diag_blocks_f32(const float* w, int64_t ldw, int64_t n, float* dinv, cudaStream_t stream) {
  if (n == 0) return RM_OK;
  dim3 grid((unsigned)((n + kTB - 1) / kTB), 2);
  invert_diag_blocks_kernel<float, false><<<grid, 128, 0, stream>>>(w, ldw, n, dinv, true, false);
  RM_LAUNCHED();
  return RM_OK;
}

size_t trsv_f32_scratch_bytes(int64_t n, int64_t k) {
  return (size_t)(2 * ((n + kTB - 1) / kTB + 1)) * sizeof(int) * (size_t)((k + kKC - 1) / kKC) + 256;
}

// x = U^-1 L^-1 x in place for the row-major float32 L\U (unit L) of an unpivoted LU.
int lu_solve_f32_nopiv(const float* lu, int64_t ld, int64_t n, const float* dinv, float* x, int64_t ldx, int64_t k,
                       void* scratch, unsigned* status, cudaStream_t stream) {
  if (n == 0 || k == 0) return RM_OK;
  const int nblk = (int)((n + kTB - 1) / kTB);
  const int chunks = (int)((k + kKC - 1) / kKC);
  int* flags = reinterpret_cast<int*>(scratch);
  RM_CUDA_TRY(cudaMemsetAsync(flags, 0, (size_t)(2 * (nblk + 1)) * sizeof(int) * chunks, stream));
  for (int ch = 0; ch < chunks; ++ch) {
    const int kc = (int)std::min<int64_t>(kKC, k - (int64_t)ch * kKC);
    int* f = flags + (size_t)ch * 2 * (nblk + 1);
    float* xc = x + ch * kKC;
    trsv_chain_kernel<float, true, false><<<nblk, kTrsvThreads, 0, stream>>>(lu, ld, (int)n, dinv, xc, ldx, kc, f,
                                                                              f + nblk, status);
    RM_LAUNCHED();
    trsv_chain_kernel<float, false, false><<<nblk, kTrsvThreads, 0, stream>>>(lu, ld, (int)n, dinv, xc, ldx, kc,
                                                                               f + nblk + 1, f + 2 * nblk + 1, status);
    RM_LAUNCHED();
  }
  return RM_OK;
}

}  // namespace rm
