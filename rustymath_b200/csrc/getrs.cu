// Triangular solves with the LU factors: x = U^-1 L^-1 P b (and the transposed form).
//
// Replaces lu_solve and the native triangular solves (core/src/linalg/factor.rs:633-641,
// 668-748). The reference substitutes row by row within 16/32-row leaves and removes
// solved halves with GEMMs. On the GPU each block row of the triangle (64 rows in float64,
// 128 in float32) belongs to one CTA. A CTA takes a ticket (an atomic counter, so tickets follow the order in which
// CTAs start and every dependency is held by a CTA that is already running), subtracts
// the products of its block row of L (or U) with each already-solved block of x as soon as
// that block's flag is set, then multiplies by the inverse of its diagonal block (computed
// once per factorization by invert_diag_blocks) and publishes its block with a release
// flag. Waits on flags are bounded: on expiry the status word records a timeout.
#include "rm_internal.h"

namespace rm {

constexpr int kKC = kSolveCols;  // right-hand-side columns per launch
constexpr int kTB64 = kSolveBlock;  // float64 block rows (64)
constexpr int kTB32 = 128;          // float32 block rows

size_t diag_blocks_f64_bytes(int64_t n) { return diag_blocks_bytes_max(n); }

// dinv[b][0] = inverse of the lower diagonal block b, dinv[b][1] = inverse of the upper
// diagonal block b (row-major TB x TB; rows/columns past n are identity). A unit triangle
// takes its diagonal as 1 without reading it. The triangles are those of the n x n matrix
// T whose item (i, j) is w[i*ldw + j], or w[j*ldw + i] when COLMAJOR. Thread c solves for
// column c of the inverse.
template <typename T, bool COLMAJOR, int TB>
__global__ void __launch_bounds__(TB) invert_diag_blocks_kernel(const T* __restrict__ w, int64_t ldw, int64_t n,
                                                                T* __restrict__ dinv, bool lower_unit, bool upper_unit) {
  extern __shared__ uint8_t smraw[];
  T(*x)[TB + 1] = reinterpret_cast<T(*)[TB + 1]>(smraw);
  const int b = blockIdx.x, which = blockIdx.y;  // 0: L, 1: U
  const int64_t r0 = (int64_t)b * TB;
  const int rows = (int)(n - r0 < TB ? n - r0 : TB);
  const T* blk = w + r0 * ldw + r0;
  const int col = threadIdx.x;
  auto A = [&](int i, int j) -> T {
    if (i >= rows || j >= rows) return i == j ? T(1) : T(0);
    return COLMAJOR ? blk[(int64_t)j * ldw + i] : blk[(int64_t)i * ldw + j];
  };
  if (which == 0) {
    // lower: x_i = (delta_i,col - sum_{col<=k<i} L_ik x_k) / L_ii for i >= col
    for (int i = 0; i < TB; ++i) {
      T s = i == col ? T(1) : T(0);
      if (i > col)
        for (int k = col; k < i; ++k) s = fma(-A(i, k), x[k][col], s);
      x[i][col] = i < col ? T(0) : (lower_unit ? s : s / A(i, i));
    }
  } else {
    // upper: x_i = (delta_i,col - sum_{i<k<=col} U_ik x_k) / U_ii for i <= col
    for (int i = TB - 1; i >= 0; --i) {
      T s = i == col ? T(1) : T(0);
      if (i < col)
        for (int k = i + 1; k <= col; ++k) s = fma(-A(i, k), x[k][col], s);
      x[i][col] = i > col ? T(0) : (upper_unit ? s : s / A(i, i));
    }
  }
  __syncthreads();
  T* out = dinv + ((int64_t)b * 2 + which) * TB * TB;
  for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) out[e] = x[e / TB][e % TB];
}

template <typename T, bool COLMAJOR, int TB>
static int launch_invert(const T* w, int64_t ldw, int64_t n, T* dinv, bool lower_unit, bool upper_unit,
                         cudaStream_t stream) {
  const size_t smem = (size_t)TB * (TB + 1) * sizeof(T);
  static bool set = false;
  if (!set) {
    RM_CUDA_TRY(cudaFuncSetAttribute(invert_diag_blocks_kernel<T, COLMAJOR, TB>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    set = true;
  }
  dim3 grid((unsigned)((n + TB - 1) / TB), 2);
  invert_diag_blocks_kernel<T, COLMAJOR, TB><<<grid, TB, smem, stream>>>(w, ldw, n, dinv, lower_unit, upper_unit);
  RM_LAUNCHED();
  return RM_OK;
}

int invert_diag_blocks_f64(const double* w, int64_t ldw, bool colmajor, int64_t n, double* dinv, bool lower_unit,
                           bool upper_unit, cudaStream_t stream) {
  if (n == 0) return RM_OK;
  if (colmajor) return launch_invert<double, true, kTB64>(w, ldw, n, dinv, lower_unit, upper_unit, stream);
  return launch_invert<double, false, kTB64>(w, ldw, n, dinv, lower_unit, upper_unit, stream);
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
// triangle of the matrix whose item (i, j) is w[i*ldw + j] (w[j*ldw + i] when COLMAJOR),
// in block rows of TB; the diagonal blocks' inverses come from dinv. flags[nblk] and
// counter start at zero. Thread t owns row t / 4 and columns 4 (t % 4) .. +3 of its block's
// running sums. The next dependency's block of T is loaded into registers while the current
// one is applied, so each block of T crosses HBM once, overlapped with the arithmetic.
template <typename T, bool LOWER, bool COLMAJOR, int TB>
__global__ void __launch_bounds__(TB * 4)
    trsv_chain_kernel(const T* __restrict__ w, int64_t ldw, int n, const T* __restrict__ dinv, T* x, int64_t ldx,
                      int kc, int* flags, int* counter, unsigned* status) {
  constexpr int THREADS = TB * 4;
  constexpr int LPT = TB * TB / THREADS;  // items of a block of T per thread
  constexpr int LDS = TB + 1;
  extern __shared__ uint8_t smraw[];
  T(*lblk)[LDS] = reinterpret_cast<T(*)[LDS]>(smraw);
  T(*xs)[kKC] = reinterpret_cast<T(*)[kKC]>(smraw + ((size_t)TB * LDS * sizeof(T) + 15) / 16 * 16);
  __shared__ int ticket, good;
  const int tid = threadIdx.x;
  const int nblk = (n + TB - 1) / TB;
  if (tid == 0) ticket = atomicAdd(counter, 1);
  __syncthreads();
  const int t = ticket;
  const int b = LOWER ? t : nblk - 1 - t;
  const int r0 = b * TB, rows = min(TB, n - r0);
  const int my_r = tid >> 2, my_c = (tid & 3) * 4;

  T acc[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int c = my_c + i;
    acc[i] = (my_r < rows && c < kc) ? x[(int64_t)(r0 + my_r) * ldx + c] : T(0);
  }
  // element e of a block: COLMAJOR storage is read along its columns (coalesced)
  auto coord = [&](int e, int& r, int& c) {
    if (COLMAJOR) {
      c = e / TB;
      r = e % TB;
    } else {
      r = e / TB;
      c = e % TB;
    }
  };
  T regs[LPT];
  auto load = [&](int j) {
    const int c0 = j * TB, cols = min(TB, n - c0);
#pragma unroll
    for (int q = 0; q < LPT; ++q) {
      int r, c;
      coord(tid + q * THREADS, r, c);
      regs[q] = (r < rows && c < cols)
                    ? (COLMAJOR ? __ldcs(w + (int64_t)(c0 + c) * ldw + r0 + r) : __ldcs(w + (int64_t)(r0 + r) * ldw + c0 + c))
                    : T(0);
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int q = 0; q < LPT; ++q) {
      int r, c;
      coord(tid + q * THREADS, r, c);
      lblk[r][c] = regs[q];
    }
  };
  // acc[i] += sign * sum_q lblk[my_r][q] xs[q][my_c + i]
  auto apply = [&](T sign) {
#pragma unroll 8
    for (int q = 0; q < TB; ++q) {
      const T l = sign * lblk[my_r][q];
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[i] = fma(l, xs[q][my_c + i], acc[i]);
    }
  };
  // the inverse of this block's diagonal block, row-major, prefetched behind the last dependency
  const T* dv = dinv + ((int64_t)b * 2 + (LOWER ? 0 : 1)) * TB * TB;
  auto load_dinv = [&]() {
#pragma unroll
    for (int q = 0; q < LPT; ++q) regs[q] = __ldg(dv + tid + q * THREADS);
  };
  bool ok = true;
  if (t > 0) load(LOWER ? 0 : nblk - 1);
  else load_dinv();
  for (int s = 0; s < t; ++s) {
    const int j = LOWER ? s : nblk - 1 - s;  // a solved block, in solve order
    const int c0 = j * TB, cols = min(TB, n - c0);
    __syncthreads();  // the previous step's reads of lblk / xs are done
    store();
    if (s + 1 < t) load(LOWER ? s + 1 : nblk - 2 - s);
    else load_dinv();
    if (tid == 0) {
      bool seen = ld_acquire(&flags[j]) != 0;
      if (!seen) {
        const uint64_t start = global_ns();
        while (!(seen = ld_acquire(&flags[j]) != 0)) {
          if (global_ns() - start > kWaitLimitNs) break;
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
    for (int e = tid; e < TB * kKC; e += THREADS) {
      const int r = e / kKC, c = e % kKC;
      xs[r][c] = (r < cols && c < kc) ? __ldcg(&x[(int64_t)(c0 + r) * ldx + c]) : T(0);
    }
    __syncthreads();
    apply(T(-1));
  }
  __syncthreads();
  if (ok) {
#pragma unroll
    for (int q = 0; q < LPT; ++q) {
      const int e = tid + q * THREADS;
      lblk[e / TB][e % TB] = regs[q];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) xs[my_r][my_c + i] = acc[i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[i] = T(0);
    apply(T(1));
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int c = my_c + i;
      if (my_r < rows && c < kc) x[(int64_t)(r0 + my_r) * ldx + c] = acc[i];
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) st_release(&flags[b], 1);
}

template <typename T, bool LOWER, bool COLMAJOR, int TB>
static int launch_trsv(const T* w, int64_t ldw, int n, const T* dinv, T* x, int64_t ldx, int kc, int* flags,
                       int* counter, unsigned* status, cudaStream_t stream) {
  const size_t smem = ((size_t)TB * (TB + 1) * sizeof(T) + 15) / 16 * 16 + (size_t)TB * kKC * sizeof(T);
  static bool set = false;
  if (!set) {
    RM_CUDA_TRY(cudaFuncSetAttribute(trsv_chain_kernel<T, LOWER, COLMAJOR, TB>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    set = true;
  }
  const int nblk = (n + TB - 1) / TB;
  trsv_chain_kernel<T, LOWER, COLMAJOR, TB><<<nblk, TB * 4, smem, stream>>>(w, ldw, n, dinv, x, ldx, kc, flags, counter,
                                                                             status);
  RM_LAUNCHED();
  return RM_OK;
}

// Row permutation of an n x k row-major matrix: x[i] = b[perm[i]] (gather), or, with
// SCATTER, x[perm[i]] = b[i]. perm == NULL copies. A position outside 0..n-1 (a caller's
// perm) sets RM_DEV_BAD_INDEX and is skipped.
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
  const int nblk = (int)((n + kTB64 - 1) / kTB64);
  const int chunks = (int)((k + kKC - 1) / kKC);
  // The solved triangle pair: L\\U itself, or its transpose for A^T x = b.
  const bool colmajor = trans ? !lu_colmajor : lu_colmajor;
  // b may alias x: the permuted right-hand side goes to a temporary first
  double* tmp = reinterpret_cast<double*>(scratch);
  int* flags = reinterpret_cast<int*>(reinterpret_cast<char*>(scratch) + ((size_t)n * k * sizeof(double) + 255) / 256 * 256);
  const size_t flag_bytes = (size_t)(2 * (nblk + 1)) * sizeof(int) * (size_t)chunks;
  RM_CUDA_TRY(cudaMemsetAsync(flags, 0, flag_bytes, stream));
  const int blocks = (int)std::min<int64_t>((n * k + 255) / 256, 4 * device_sm_count());
  permute_rows_kernel<false><<<blocks, 256, 0, stream>>>(b, ldb, trans ? nullptr : perm, n, k, tmp, k, status);
  RM_LAUNCHED();
  const int ni = (int)n;
  for (int ch = 0; ch < chunks; ++ch) {
    const int kc = (int)std::min<int64_t>(kKC, k - (int64_t)ch * kKC);
    int* f = flags + (size_t)ch * 2 * (nblk + 1);
    double* xc = tmp + ch * kKC;
    if (colmajor) {
      RM_TRY((launch_trsv<double, true, true, kTB64>(lu, ld, ni, dinv, xc, k, kc, f, f + nblk, status, stream)));
      RM_TRY((launch_trsv<double, false, true, kTB64>(lu, ld, ni, dinv, xc, k, kc, f + nblk + 1, f + 2 * nblk + 1,
                                                      status, stream)));
    } else {
      RM_TRY((launch_trsv<double, true, false, kTB64>(lu, ld, ni, dinv, xc, k, kc, f, f + nblk, status, stream)));
      RM_TRY((launch_trsv<double, false, false, kTB64>(lu, ld, ni, dinv, xc, k, kc, f + nblk + 1, f + 2 * nblk + 1,
                                                       status, stream)));
    }
  }
  permute_rows_kernel<true><<<blocks, 256, 0, stream>>>(tmp, k, trans ? perm : nullptr, n, k, x, ldx, status);
  RM_LAUNCHED();
  return RM_OK;
}

// ------------------------------------------------------------------ float32, no pivoting

size_t diag_blocks_f32_bytes(int64_t n) { return (size_t)((n + kTB32 - 1) / kTB32) * 2 * kTB32 * kTB32 * sizeof(float); }

int invert_diag_blocks_f32(const float* w, int64_t ldw, int64_t n, float* dinv, cudaStream_t stream) {
  if (n == 0) return RM_OK;
  return launch_invert<float, false, kTB32>(w, ldw, n, dinv, true, false, stream);
}

size_t trsv_f32_scratch_bytes(int64_t n, int64_t k) {
  return (size_t)(2 * ((n + kTB32 - 1) / kTB32 + 1)) * sizeof(int) * (size_t)((k + kKC - 1) / kKC) + 256;
}

// x = U^-1 L^-1 x in place for the row-major float32 L\\U (unit L) of an LU whose row
// permutation the caller has already applied to x.
int lu_solve_f32_nopiv(const float* lu, int64_t ld, int64_t n, const float* dinv, float* x, int64_t ldx, int64_t k,
                       void* scratch, unsigned* status, cudaStream_t stream) {
  if (n == 0 || k == 0) return RM_OK;
  const int nblk = (int)((n + kTB32 - 1) / kTB32);
  const int chunks = (int)((k + kKC - 1) / kKC);
  int* flags = reinterpret_cast<int*>(scratch);
  RM_CUDA_TRY(cudaMemsetAsync(flags, 0, (size_t)(2 * (nblk + 1)) * sizeof(int) * chunks, stream));
  for (int ch = 0; ch < chunks; ++ch) {
    const int kc = (int)std::min<int64_t>(kKC, k - (int64_t)ch * kKC);
    int* f = flags + (size_t)ch * 2 * (nblk + 1);
    float* xc = x + ch * kKC;
    RM_TRY((launch_trsv<float, true, false, kTB32>(lu, ld, (int)n, dinv, xc, ldx, kc, f, f + nblk, status, stream)));
    RM_TRY((launch_trsv<float, false, false, kTB32>(lu, ld, (int)n, dinv, xc, ldx, kc, f + nblk + 1, f + 2 * nblk + 1,
                                                    status, stream)));
  }
  return RM_OK;
}

}  // namespace rm
