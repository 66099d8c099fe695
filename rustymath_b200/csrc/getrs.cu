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
#include "rm_tcgen05.cuh"

namespace rm {

constexpr int kKC = kSolveCols;  // right-hand-side columns per launch
constexpr int kTB64 = kSolveBlock;  // float64 block rows (64)
constexpr int kTB32 = 128;          // float32 block rows
constexpr int kPreKC = 8;           // columns per chain of the scaled float32 solve

size_t diag_blocks_f64_bytes(int64_t n) { return diag_blocks_bytes_max(n); }

// dinv[b][0] = inverse of the lower diagonal block b, dinv[b][1] = inverse of the upper
// diagonal block b (row-major TB x TB; rows/columns past n are identity); dinv[b][2..3] are
// the couplings that coupling_kernel fills in. A unit triangle
// takes its diagonal as 1 without reading it. The triangles are those of the n x n matrix
// T whose item (i, j) is w[i*ldw + j], or w[j*ldw + i] when COLMAJOR. Thread c solves for
// column c of the inverse.
template <typename T, bool COLMAJOR, int TB>
__global__ void __launch_bounds__(TB) invert_diag_blocks_kernel(const T* __restrict__ w, int64_t ldw, int64_t n,
                                                                T* __restrict__ dinv, bool lower_unit, bool upper_unit) {
  extern __shared__ uint8_t smraw[];
  T(*x)[TB + 1] = reinterpret_cast<T(*)[TB + 1]>(smraw);
  T(*t)[TB + 1] = reinterpret_cast<T(*)[TB + 1]>(smraw + (size_t)TB * (TB + 1) * sizeof(T));
  const int b = blockIdx.x, which = blockIdx.y;  // 0: L, 1: U
  const int64_t r0 = (int64_t)b * TB;
  const int rows = (int)(n - r0 < TB ? n - r0 : TB);
  const T* blk = w + r0 * ldw + r0;
  const int col = threadIdx.x;
  // the block in shared memory first (read along its storage order, coalesced); past n, identity
  for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) {
    const int s0 = e / TB, s1 = e % TB;  // s1 runs along the storage
    const int i = COLMAJOR ? s1 : s0, j = COLMAJOR ? s0 : s1;
    t[i][j] = (i >= rows || j >= rows) ? (i == j ? T(1) : T(0))
                                       : (COLMAJOR ? blk[(int64_t)j * ldw + i] : blk[(int64_t)i * ldw + j]);
  }
  __syncthreads();
  auto A = [&](int i, int j) -> T { return t[i][j]; };
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
  T* out = dinv + ((int64_t)b * kDiagMats + which) * TB * TB;
  for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) out[e] = x[e / TB][e % TB];
}

// out (TB x TB, row-major, ld ldo) = dinv block dv (TB x TB row-major) times block (b, pb) of
// the n x n matrix T (item (i, j) at w[i*ldw + j], or at w[j*ldw + i] when COLMAJOR; past n,
// zero). 256 threads, each a (TB/16)^2 piece; smem holds both operands.
template <typename T, bool COLMAJOR, int TB>
__device__ __forceinline__ void block_product(const T* __restrict__ w, int64_t ldw, int64_t n, int b, int pb,
                                              const T* __restrict__ dv, T* __restrict__ out, int64_t ldo) {
  constexpr int R = TB / 16;
  extern __shared__ uint8_t smraw[];
  T(*di)[TB + 1] = reinterpret_cast<T(*)[TB + 1]>(smraw);
  T(*ob)[TB + 1] = reinterpret_cast<T(*)[TB + 1]>(smraw + (size_t)TB * (TB + 1) * sizeof(T));
  const int64_t r0 = (int64_t)b * TB, c0 = (int64_t)pb * TB;
  for (int e = threadIdx.x; e < TB * TB; e += 256) {
    const int i = e / TB, j = e % TB;
    di[i][j] = dv[e];
    // COLMAJOR storage read down its columns (coalesced)
    const int ri = COLMAJOR ? j : i, cj = COLMAJOR ? i : j;
    const int64_t gi = r0 + ri, gj = c0 + cj;
    ob[ri][cj] = (gi < n && gj < n) ? (COLMAJOR ? w[gj * ldw + gi] : w[gi * ldw + gj]) : T(0);
  }
  __syncthreads();
  const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
  T acc[R][R];
#pragma unroll
  for (int i = 0; i < R; ++i)
#pragma unroll
    for (int j = 0; j < R; ++j) acc[i][j] = T(0);
  for (int q = 0; q < TB; ++q) {
    T dvv[R], ov[R];
#pragma unroll
    for (int i = 0; i < R; ++i) dvv[i] = di[ty + 16 * i][q];
#pragma unroll
    for (int j = 0; j < R; ++j) ov[j] = ob[q][tx + 16 * j];
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
      for (int j = 0; j < R; ++j) acc[i][j] = fma(dvv[i], ov[j], acc[i][j]);
  }
#pragma unroll
  for (int i = 0; i < R; ++i)
#pragma unroll
    for (int j = 0; j < R; ++j) out[(int64_t)(ty + 16 * i) * ldo + tx + 16 * j] = acc[i][j];
}

// dinv[b][2] = dinv[b][0] T[b, b-1] and dinv[b][3] = dinv[b][1] T[b, b+1]: the coupling of
// block b to the block the forward (backward) solve finishes just before it, so that block
// b's last step is x_b = z_b - coupling x_prev with z_b formed while it waits. A CTA per
// (block, triangle).
template <typename T, bool COLMAJOR, int TB>
__global__ void __launch_bounds__(256) coupling_kernel(const T* __restrict__ w, int64_t ldw, int64_t n,
                                                       T* __restrict__ dinv) {
  const int b = blockIdx.x, which = blockIdx.y;  // 0: lower (block b-1), 1: upper (block b+1)
  const int nblk = (int)((n + TB - 1) / TB);
  const int pb = which == 0 ? b - 1 : b + 1;
  if (pb < 0 || pb >= nblk) return;
  block_product<T, COLMAJOR, TB>(w, ldw, n, b, pb, dinv + ((int64_t)b * kDiagMats + which) * TB * TB,
                                 dinv + ((int64_t)b * kDiagMats + 2 + which) * TB * TB, TB);
}


template <typename T, bool COLMAJOR, int TB>
static int launch_invert(const T* w, int64_t ldw, int64_t n, T* dinv, bool lower_unit, bool upper_unit,
                         cudaStream_t stream) {
  const size_t smem = (size_t)TB * (TB + 1) * sizeof(T);
  RM_TRY(smem_attribute(invert_diag_blocks_kernel<T, COLMAJOR, TB>, 2 * smem));
  RM_TRY(smem_attribute(coupling_kernel<T, COLMAJOR, TB>, 2 * smem));
  dim3 grid((unsigned)((n + TB - 1) / TB), 2);
  invert_diag_blocks_kernel<T, COLMAJOR, TB><<<grid, TB, 2 * smem, stream>>>(w, ldw, n, dinv, lower_unit,
                                                                              upper_unit);
  RM_LAUNCHED();
  if (grid.x > 1) {
    coupling_kernel<T, COLMAJOR, TB><<<grid, 256, 2 * smem, stream>>>(w, ldw, n, dinv);
    RM_LAUNCHED();
  }
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
// in block rows of TB; dinv holds each block's diagonal inverse and its coupling to the
// block solved just before it. With PRE, w holds the block-Jacobi-scaled triangles
// (premultiply_mma_kernel): block b forms D_b^-1 y_b first and subtracts pre_bj x_j as each x_j
// is released. flags[nblk] and counter start at zero. CTAs take tickets in
// launch order and block rows in solve order; block b subtracts T_bj x_j for every block j
// solved before it but the last, as each x_j is released, then forms z_b = D_b^-1 (...) and,
// once the last one (p) is released, x_b = z_b - (D_b^-1 T_bp) x_p: one TB x TB product
// between seeing p's flag and releasing its own. Thread t owns row t / 4 and columns
// 4 (t % 4) .. +3 of its block's sums. The next matrix a step needs is loaded into registers
// while the current one is applied, so each block of T crosses HBM once.
// Shared-memory layout of a chain CTA. float32 with 128-row blocks multiplies on the tensor
// cores (mma.sync m16n8k8, TF32 inputs split into high and low parts, three products: float32-
// level accuracy); the padded rows keep its fragment loads free of bank conflicts.
template <typename T, int TB>
struct ChainLayout {
  static constexpr bool MMA = sizeof(T) == 4 && TB == 128;
  static constexpr int LDS = MMA ? TB + 4 : TB + 1;  // row stride of a block of T
  static constexpr int XS = MMA ? 24 : kKC;          // row stride of the staged x
  static constexpr size_t bytes() {
    return ((size_t)TB * LDS * sizeof(T) + 15) / 16 * 16 + (size_t)TB * XS * sizeof(T);
  }
};


template <typename T, bool LOWER, bool COLMAJOR, int TB, bool PRE>
__global__ void __launch_bounds__(TB * 4)
    trsv_chain_kernel(const T* __restrict__ w, int64_t ldw, int n, const T* __restrict__ dinv, T* x, int64_t ldx,
                      int kc, int* flags, int* counter, unsigned* status, uint64_t wait_ns) {
  using Lay = ChainLayout<T, TB>;
  constexpr int THREADS = TB * 4;
  constexpr int LPT = TB * TB / THREADS;  // items of a block of T per thread
  constexpr int LDS = Lay::LDS;
  extern __shared__ uint8_t smraw[];
  T(*lblk)[LDS] = reinterpret_cast<T(*)[LDS]>(smraw);
  T(*xs)[Lay::XS] = reinterpret_cast<T(*)[Lay::XS]>(smraw + ((size_t)TB * LDS * sizeof(T) + 15) / 16 * 16);
  __shared__ int ticket;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = (n + TB - 1) / TB;
  if (tid == 0) ticket = atomicAdd(counter, 1);
  __syncthreads();
  const int t = ticket;
  const int b = LOWER ? t : nblk - 1 - t;
  const int r0 = b * TB, rows = min(TB, n - r0);
  auto dep = [&](int s) { return LOWER ? s : nblk - 1 - s; };  // the s-th block solved
  // this thread's four items of the block's sums: (my_r, my_c + i) for the scalar product; for
  // the tensor-core one, the m16n8 fragment of warp (8 row tiles x 2 column tiles):
  // rows fr + 8 (i >> 1), columns fc + (i & 1)
  const int g = lane >> 2, tq = lane & 3;
  const int fr = 16 * (warp >> 1) + g, fc = 8 * (warp & 1) + 2 * tq;
  const int my_r = tid >> 2, my_c = (tid & 3) * 4;
  auto prow = [&](int i) { return Lay::MMA ? fr + 8 * (i >> 1) : my_r; };
  auto pcol = [&](int i) { return Lay::MMA ? fc + (i & 1) : my_c + i; };

  T acc[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = prow(i), c = pcol(i);
    acc[i] = (r < rows && c < kc) ? x[(int64_t)(r0 + r) * ldx + c] : T(0);
  }
  T regs[LPT];
  // a block of T: COLMAJOR storage is read along its columns (coalesced)
  auto load = [&](int j) {
    const int c0 = j * TB, cols = min(TB, n - c0);
#pragma unroll
    for (int q = 0; q < LPT; ++q) {
      const int e = tid + q * THREADS;
      const int r = COLMAJOR ? e % TB : e / TB, c = COLMAJOR ? e / TB : e % TB;
      regs[q] = (r < rows && c < cols)
                    ? (COLMAJOR ? __ldcs(w + (int64_t)(c0 + c) * ldw + r0 + r) : __ldcs(w + (int64_t)(r0 + r) * ldw + c0 + c))
                    : T(0);
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int q = 0; q < LPT; ++q) {
      const int e = tid + q * THREADS;
      const int r = COLMAJOR ? e % TB : e / TB, c = COLMAJOR ? e / TB : e % TB;
      lblk[r][c] = regs[q];
    }
  };
  // a row-major matrix of dinv (the diagonal inverse, m = 0, or the coupling, m = 2)
  auto load_mat = [&](int m) {
    const T* dv = dinv + ((int64_t)b * kDiagMats + m + (LOWER ? 0 : 1)) * TB * TB;
#pragma unroll
    for (int q = 0; q < LPT; ++q) regs[q] = __ldg(dv + tid + q * THREADS);
  };
  auto store_mat = [&]() {
#pragma unroll
    for (int q = 0; q < LPT; ++q) {
      const int e = tid + q * THREADS;
      lblk[e / TB][e % TB] = regs[q];
    }
  };
  // acc += sign * lblk xs (this thread's items)
  auto apply = [&](T sign) {
    if constexpr (Lay::MMA) {
      float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
      for (int k8 = 0; k8 < TB; k8 += 8) {
        const float av[4] = {sign * lblk[fr][k8 + tq], sign * lblk[fr + 8][k8 + tq], sign * lblk[fr][k8 + tq + 4],
                             sign * lblk[fr + 8][k8 + tq + 4]};
        const float bv0 = xs[k8 + tq][8 * (warp & 1) + g], bv1 = xs[k8 + tq + 4][8 * (warp & 1) + g];
        uint32_t ah[4], al[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          ah[i] = tc::to_tf32(av[i]);
          al[i] = tc::to_tf32(av[i] - __uint_as_float(ah[i]));
        }
        const uint32_t bh0 = tc::to_tf32(bv0), bh1 = tc::to_tf32(bv1);
        const uint32_t bl0 = tc::to_tf32(bv0 - __uint_as_float(bh0)), bl1 = tc::to_tf32(bv1 - __uint_as_float(bh1));
        tc::mma_tf32_16x8x8(d, al, bh0, bh1);  // the small terms first
        tc::mma_tf32_16x8x8(d, ah, bl0, bl1);
        tc::mma_tf32_16x8x8(d, ah, bh0, bh1);
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[i] += d[i];
    } else {
#pragma unroll 8
      for (int q = 0; q < TB; ++q) {
        const T l = sign * lblk[my_r][q];
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[i] = fma(l, xs[q][my_c + i], acc[i]);
      }
    }
  };
  auto fetch = [&](int j) -> bool {
    bool seen = ld_acquire(&flags[j]) != 0;
    if (!seen) {
      const uint64_t start = global_ns();
      while (!(seen = ld_acquire(&flags[j]) != 0)) {
        if (global_ns() - start > wait_ns) break;
      }
    }
    if (seen) {
      const int c0 = j * TB, cols = min(TB, n - c0);
      for (int e = tid; e < TB * kKC; e += THREADS) {
        const int r = e / kKC, c = e % kKC;
        xs[r][c] = (r < cols && c < kc) ? __ldcg(&x[(int64_t)(c0 + r) * ldx + c]) : T(0);
      }
    }
    if (!__syncthreads_and(seen ? 1 : 0)) {
      if (tid == 0) flag_error(status, RM_DEV_TIMEOUT);
      return false;
    }
    return true;
  };

  bool ok = true;
  if (PRE) {
    load_mat(0);
    store_mat();
    if (t >= 1) load(dep(0));
#pragma unroll
    for (int i = 0; i < 4; ++i) xs[prow(i)][pcol(i)] = acc[i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[i] = T(0);
    apply(T(1));  // D_b^-1 y_b
    for (int s = 0; s < t; ++s) {
      __syncthreads();
      store();
      if (s + 1 < t) load(dep(s + 1));
      if (!fetch(dep(s))) {
        ok = false;
        break;
      }
      apply(T(-1));
    }
    if (ok) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = prow(i), c = pcol(i);
        if (r < rows && c < kc) x[(int64_t)(r0 + r) * ldx + c] = acc[i];
      }
    }
  } else {
  if (t >= 2) load(dep(0));
  else load_mat(0);
  for (int s = 0; s + 1 < t; ++s) {  // every block solved before this one but the last
    __syncthreads();                 // the previous step's reads of lblk / xs are done
    store();
    if (s + 2 < t) load(dep(s + 1));
    else load_mat(0);
    if (!fetch(dep(s))) {
      ok = false;
      break;
    }
    apply(T(-1));
  }
  if (ok) {
    // z_b = D_b^-1 (y_b - sum ...), while the last block before this one may still be running
    __syncthreads();
    store_mat();
#pragma unroll
    for (int i = 0; i < 4; ++i) xs[prow(i)][pcol(i)] = acc[i];
    if (t >= 1) load_mat(2);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[i] = T(0);
    apply(T(1));
    if (t >= 1) {
      __syncthreads();
      store_mat();
      if (fetch(dep(t - 1))) apply(T(-1));  // x_b = z_b - C_b x_prev
      else ok = false;
    }
    if (ok) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = prow(i), c = pcol(i);
        if (r < rows && c < kc) x[(int64_t)(r0 + r) * ldx + c] = acc[i];
      }
    }
  }
  }
  // every thread's x is written before the barrier; thread 0's release store, ordered after the
  // barrier, publishes them device-wide
  __syncthreads();
  if (tid == 0) st_release(&flags[b], 1);
}

// Launches one chain (a CTA per block row). `ctas` < 0 launches all of them; the bounded-wait
// self-test launches one fewer, having taken the first ticket itself.
template <typename T, bool LOWER, bool COLMAJOR, int TB, bool PRE = false>
static int launch_trsv(const T* w, int64_t ldw, int n, const T* dinv, T* x, int64_t ldx, int kc, int* flags,
                       int* counter, unsigned* status, cudaStream_t stream, uint64_t wait_ns = kWaitLimitNs,
                       int ctas = -1) {
  const size_t smem = ChainLayout<T, TB>::bytes();
  RM_TRY(smem_attribute(trsv_chain_kernel<T, LOWER, COLMAJOR, TB, PRE>, smem));
  const int nblk = (n + TB - 1) / TB;
  trsv_chain_kernel<T, LOWER, COLMAJOR, TB, PRE><<<ctas < 0 ? nblk : ctas, TB * 4, smem, stream>>>(
      w, ldw, n, dinv, x, ldx, kc, flags, counter, status, wait_ns);
  RM_LAUNCHED();
  return RM_OK;
}

// The bounded-wait self-test (rm_test_chain_timeout): a lower-triangular float64 chain at
// n = 256 (four 64-row blocks, all zero: every load stays inside the buffers below) whose
// ticket counter starts at 1, so block 0 never runs and never releases its flag. The three
// CTAs launched (tickets 1..3, blocks 1..3, all resident at once) each wait on that flag, give
// up after wait_ns, set RM_DEV_TIMEOUT in a status word of this call's own and return.
namespace {
constexpr int kTimeoutN = 256;
struct TimeoutLayout {
  static constexpr size_t w = 0;
  static constexpr size_t dinv = w + (size_t)kTimeoutN * kTimeoutN * sizeof(double);
  static constexpr size_t x = dinv + diag_blocks_bytes_max(kTimeoutN);
  static constexpr size_t flags = x + (size_t)kTimeoutN * kKC * sizeof(double);
  static constexpr size_t status = flags + 256;
  static constexpr size_t total = status + 256;
};
}  // namespace

size_t chain_timeout_scratch_bytes() { return TimeoutLayout::total; }

int chain_timeout_run(uint64_t wait_ns, void* scratch, unsigned* bits, cudaStream_t stream) {
  char* base = static_cast<char*>(scratch);
  const int nblk = kTimeoutN / kTB64;
  int* flags = reinterpret_cast<int*>(base + TimeoutLayout::flags);
  unsigned* status = reinterpret_cast<unsigned*>(base + TimeoutLayout::status);
  RM_CUDA_TRY(cudaMemsetAsync(scratch, 0, TimeoutLayout::total, stream));
  const int first_ticket = 1;  // the counter sits after the nblk flags
  RM_CUDA_TRY(cudaMemcpyAsync(flags + nblk, &first_ticket, sizeof(int), cudaMemcpyHostToDevice, stream));
  RM_TRY((launch_trsv<double, true, false, kTB64>(
      reinterpret_cast<const double*>(base + TimeoutLayout::w), kTimeoutN, kTimeoutN,
      reinterpret_cast<const double*>(base + TimeoutLayout::dinv), reinterpret_cast<double*>(base + TimeoutLayout::x),
      kKC, kKC, flags, flags + nblk, status, stream, wait_ns, nblk - 1)));
  RM_CUDA_TRY(cudaMemcpyAsync(bits, status, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
  RM_CUDA_TRY(cudaStreamSynchronize(stream));
  return RM_OK;
}

// The float32 block-Jacobi-scaled chain (PRE, 128-row blocks) with its blocks of the scaled
// triangle brought into shared memory by asynchronous copies, two blocks ahead of the one being
// applied (a ring of three): a step's own time is then its product, not the load latency of
// its block. x_b = D_b^-1 y_b - sum_j pre_bj x_j, each x_j subtracted as it is released, in
// solve order; pre holds full zero-padded 128 x 128 blocks (ld a multiple of 128), so every
// copy is in bounds. The products are float32 FMAs on the CUDA cores: 128 x 128 x 8 per step
// is 2^17 FMAs, about 1024 cycles of one SM's FP32 pipes, which beats three TF32 passes through
// the warp-level tensor-core instructions (their rate is near the FMA rate) and, at so few
// columns, tcgen05 too (an M = 128, K = 8 instruction costs the same at N = 16 as at N = 128).
// A launch runs one chain per kPreKC columns of x (blockIdx.y), each with its own tickets and
// flags, so that the chains of a 16-column right-hand side run side by side on twice the SMs,
// each step half the product and half the reduction. Lane (ks, h) of warp g multiplies rows
// 4 (2 g + h) .. + 3 by the chunk's 8 columns of x over k = ks, ks + 16, ..., a 4 x 8 register
// tile; the partial sums stay in registers from step to step, and the sixteen K-slices of a
// warp half sum them once, at the end.
template <bool LOWER>
__global__ void __launch_bounds__(kTB32 * 4)
    trsv_pre_ring_kernel(const float* __restrict__ pre, int64_t ldp, int n, const float* __restrict__ dinv, float* x,
                         int64_t ldx, int k, int* flags, int* counter, int64_t chain_stride, unsigned* status) {
  constexpr int TB = kTB32, THREADS = TB * 4, LDS = TB + 4, RING = 3, NC = kPreKC, XS = NC + 4;
  x += (int64_t)blockIdx.y * NC;
  flags += (int64_t)blockIdx.y * chain_stride;
  counter += (int64_t)blockIdx.y * chain_stride;
  const int kc = min(NC, k - (int)blockIdx.y * NC);
  extern __shared__ __align__(16) uint8_t smraw[];
  float(*ring)[TB][LDS] = reinterpret_cast<float(*)[TB][LDS]>(smraw);
  // x_j (times -1) or y_b, rows XS floats apart: the eight rows that one phase of a 16-byte load
  // reads fall in eight different 16-byte bank groups (XS / 4 is odd)
  float* xs = reinterpret_cast<float*>(smraw + (size_t)RING * TB * LDS * sizeof(float));
  __shared__ int ticket;
  const int tid = threadIdx.x;
  const int nblk = (n + TB - 1) / TB;
  if (tid == 0) ticket = atomicAdd(counter, 1);
  __syncthreads();
  const int t = ticket;
  const int b = LOWER ? t : nblk - 1 - t;
  const int r0 = b * TB, rows = min(TB, n - r0);
  auto dep = [&](int s) { return LOWER ? s : nblk - 1 - s; };  // the s-th block solved
  const int lane = tid & 31, ks = lane & 15, row0 = 4 * (tid >> 4);

  float acc[4][NC];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[i][c] = 0.0f;
  // item 0 is D_b^-1, item i >= 1 the block (b, dep(i - 1)); an item past t commits an empty
  // group, so that every thread counts the same groups
  auto issue = [&](int it) {
    if (it <= t) {
      const float* src;
      int64_t ld;
      if (it == 0) {
        src = dinv + ((int64_t)b * kDiagMats + (LOWER ? 0 : 1)) * TB * TB;
        ld = TB;
      } else {
        src = pre + (int64_t)b * TB * ldp + (int64_t)dep(it - 1) * TB;
        ld = ldp;
      }
      float(*dst)[LDS] = ring[it % RING];
#pragma unroll
      for (int q = 0; q < TB * TB / 4 / THREADS; ++q) {
        const int e = tid + q * THREADS, r = e >> 5, c = (e & 31) * 4;
        cp_async16(&dst[r][c], src + (int64_t)r * ld + c);
      }
    }
    cp_async_commit();
  };
  // rows c0.. (cols of them valid) of x, times sign, into xs (zero past them and past kc)
  auto put_x = [&](int c0, int cols, float sign) {
#pragma unroll
    for (int q = 0; q < TB * NC / THREADS; ++q) {
      const int e = tid + q * THREADS, r = e / NC, c = e % NC;
      xs[r * XS + c] = (r < cols && c < kc) ? sign * __ldcg(&x[(int64_t)(c0 + r) * ldx + c]) : 0.0f;
    }
  };
  // acc += blk xs over this thread's 4 x 8 tile and K-slice
  auto apply = [&](const float(*blk)[LDS]) {
#pragma unroll 4
    for (int kk = 0; kk < TB / 16; ++kk) {
      const int kr = ks + 16 * kk;
      float a[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = blk[row0 + i][kr];
      const float4 x0 = *reinterpret_cast<const float4*>(xs + kr * XS);
      const float4 x1 = *reinterpret_cast<const float4*>(xs + kr * XS + 4);
      const float xv[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[i][c] = fmaf(a[i], xv[c], acc[i][c]);
    }
  };
  // waits for block j's release, then -x_j into xs; the barrier also publishes the ring's
  // copies that each thread waited for before it
  auto fetch = [&](int j) -> bool {
    bool seen = ld_acquire(&flags[j]) != 0;
    if (!seen) {
      const uint64_t start = global_ns();
      while (!(seen = ld_acquire(&flags[j]) != 0)) {
        if (global_ns() - start > kWaitLimitNs) break;
      }
    }
    if (seen) put_x(j * TB, min(TB, n - j * TB), -1.0f);
    if (!__syncthreads_and(seen ? 1 : 0)) {
      if (tid == 0) flag_error(status, RM_DEV_TIMEOUT);
      return false;
    }
    return true;
  };

  issue(0);
  issue(1);
  issue(2);
  put_x(r0, rows, 1.0f);  // y_b
  cp_async_wait<2>();     // item 0 has landed
  __syncthreads();
  apply(ring[0]);  // z_b = D_b^-1 y_b
  bool ok = true;
  for (int s = 0; s < t; ++s) {
    const int it = s + 1;
    __syncthreads();     // the last apply's reads of its slot and of xs are done
    issue(it + 2);       // into the slot of item it - 1, applied already
    cp_async_wait<2>();  // item it has landed (it + 1 and it + 2 may be in flight)
    if (!fetch(dep(s))) {
      ok = false;
      break;
    }
    apply(ring[it % RING]);
  }
  cp_async_wait_all();  // no copy into shared memory outlives the CTA
  // the sixteen K-slices of a warp half (lanes ks = 0..15) summed, halving the tile at each of
  // four exchanges: rows by ks bits 3 and 2, then columns by bits 1 and 0. Lane ks ends with row
  // row0 + (ks >> 2) and columns 2 (ks & 3), 2 (ks & 3) + 1.
  {
    const bool b3 = ks & 8, b2 = ks & 4, b1 = ks & 2, b0 = ks & 1;
    float v16[16], v8[8], v4[4], v2[2];
#pragma unroll
    for (int j = 0; j < 16; ++j) {  // item j: row j / 8, column j % 8 of the kept half
      const float lo = acc[j / 8][j % 8], hi = acc[2 + j / 8][j % 8];
      v16[j] = (b3 ? hi : lo) + __shfl_xor_sync(0xffffffffu, b3 ? lo : hi, 8);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      v8[j] = (b2 ? v16[8 + j] : v16[j]) + __shfl_xor_sync(0xffffffffu, b2 ? v16[j] : v16[8 + j], 4);
#pragma unroll
    for (int j = 0; j < 4; ++j)
      v4[j] = (b1 ? v8[4 + j] : v8[j]) + __shfl_xor_sync(0xffffffffu, b1 ? v8[j] : v8[4 + j], 2);
#pragma unroll
    for (int j = 0; j < 2; ++j)
      v2[j] = (b0 ? v4[2 + j] : v4[j]) + __shfl_xor_sync(0xffffffffu, b0 ? v4[j] : v4[2 + j], 1);
    const int r = row0 + (ks >> 2), c0 = 2 * (ks & 3);
    if (ok && r < rows) {
#pragma unroll
      for (int j = 0; j < 2; ++j)
        if (c0 + j < kc) x[(int64_t)(r0 + r) * ldx + c0 + j] = v2[j];
    }
  }
  // every thread's x is written before the barrier; thread 0's release store, ordered after it,
  // publishes them device-wide
  __syncthreads();
  if (tid == 0) st_release(&flags[b], 1);
}

template <bool LOWER>
static int launch_trsv_pre_ring(const float* pre, int64_t ldp, int n, const float* dinv, float* x, int64_t ldx, int k,
                                int* flags, int* counter, int64_t chain_stride, unsigned* status, cudaStream_t stream) {
  constexpr size_t smem = (size_t)3 * kTB32 * (kTB32 + 4) * sizeof(float) + (size_t)kTB32 * (kPreKC + 4) * sizeof(float);
  RM_TRY(smem_attribute(trsv_pre_ring_kernel<LOWER>, smem));
  const int nblk = (n + kTB32 - 1) / kTB32;
  const dim3 grid((unsigned)nblk, (unsigned)((k + kPreKC - 1) / kPreKC));
  trsv_pre_ring_kernel<LOWER><<<grid, kTB32 * 4, smem, stream>>>(pre, ldp, n, dinv, x, ldx, k, flags, counter,
                                                                   chain_stride, status);
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

int trsv_chain_f64(bool lower, bool colmajor, const double* w, int64_t ldw, int n, const double* dinv, double* x,
                   int64_t ldx, int kc, int* flags, int* counter, unsigned* status, cudaStream_t stream) {
  if (lower && colmajor)
    return launch_trsv<double, true, true, kTB64>(w, ldw, n, dinv, x, ldx, kc, flags, counter, status, stream);
  if (lower) return launch_trsv<double, true, false, kTB64>(w, ldw, n, dinv, x, ldx, kc, flags, counter, status, stream);
  if (colmajor)
    return launch_trsv<double, false, true, kTB64>(w, ldw, n, dinv, x, ldx, kc, flags, counter, status, stream);
  return launch_trsv<double, false, false, kTB64>(w, ldw, n, dinv, x, ldx, kc, flags, counter, status, stream);
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

// ------------------------------------------------------------------ a triangular solve (TRSM)

size_t trsm_f64_scratch_bytes(int64_t order, int64_t m, int64_t n, bool right) {
  const int64_t nblk = (order + kTB64 - 1) / kTB64, cols = right ? m : n;
  return (diag_blocks_bytes_max(order) + 255) / 256 * 256 +
         ((size_t)(nblk + 1) * sizeof(int) * (size_t)((cols + kKC - 1) / kKC) + 255) / 256 * 256 +
         (right ? (size_t)m * n * sizeof(double) : 0) + 256;
}

// x = op(A)^-1 x (left, A m x m) or x op(A)^-1 (right, A n x n) for the row-major m x n x, A
// triangular (lower or upper, unit or not), op(A) = A or A^T: the block-chained solve of
// getrs on one triangle. A right-side solve is a left-side one on x^T with op(A)^T.
int trsm_f64(bool right, bool lower, bool trans, bool unit, int64_t m, int64_t n, const double* a, int64_t lda,
             double* x, int64_t ldx, void* scratch, unsigned* status, cudaStream_t stream) {
  if (m == 0 || n == 0) return RM_OK;
  const int64_t order = right ? n : m, cols = right ? m : n;
  // the solved triangle T: item (i, j) at a[i*lda + j] (row view) or a[j*lda + i] (column view)
  const bool colview = right ? !trans : trans;
  const bool low = colview ? !lower : lower;
  const int nblk = (int)((order + kTB64 - 1) / kTB64);
  double* dinv = reinterpret_cast<double*>(scratch);
  int* flags = reinterpret_cast<int*>(reinterpret_cast<char*>(scratch) + (diag_blocks_bytes_max(order) + 255) / 256 * 256);
  const int chunks = (int)((cols + kKC - 1) / kKC);
  double* xt = reinterpret_cast<double*>(reinterpret_cast<char*>(flags) +
                                         ((size_t)(nblk + 1) * sizeof(int) * chunks + 255) / 256 * 256);
  RM_TRY(invert_diag_blocks_f64(a, lda, colview, order, dinv, unit, unit, stream));
  RM_CUDA_TRY(cudaMemsetAsync(flags, 0, (size_t)(nblk + 1) * sizeof(int) * chunks, stream));
  double* y = x;
  int64_t ldy = ldx;
  if (right) {  // x^T (n x m) row-major
    RM_TRY(transpose_f64(x, ldx, m, n, xt, m, stream));
    y = xt;
    ldy = m;
  }
  const int no = (int)order;
  for (int ch = 0; ch < chunks; ++ch) {
    const int kc = (int)std::min<int64_t>(kKC, cols - (int64_t)ch * kKC);
    int* f = flags + (size_t)ch * (nblk + 1);
    double* yc = y + ch * kKC;
    if (colview) {
      if (low) RM_TRY((launch_trsv<double, true, true, kTB64>(a, lda, no, dinv, yc, ldy, kc, f, f + nblk, status, stream)));
      else RM_TRY((launch_trsv<double, false, true, kTB64>(a, lda, no, dinv, yc, ldy, kc, f, f + nblk, status, stream)));
    } else {
      if (low) RM_TRY((launch_trsv<double, true, false, kTB64>(a, lda, no, dinv, yc, ldy, kc, f, f + nblk, status, stream)));
      else RM_TRY((launch_trsv<double, false, false, kTB64>(a, lda, no, dinv, yc, ldy, kc, f, f + nblk, status, stream)));
    }
  }
  if (right) {
    RM_TRY(transpose_f64(xt, m, n, m, x, ldx, stream));
  }
  return RM_OK;
}

// ------------------------------------------------------------------ float32, no pivoting

size_t diag_blocks_f32_bytes(int64_t n) {
  return (size_t)((n + kTB32 - 1) / kTB32) * kDiagMats * kTB32 * kTB32 * sizeof(float);
}

int invert_diag_blocks_f32(const float* w, int64_t ldw, int64_t n, float* dinv, cudaStream_t stream) {
  if (n == 0) return RM_OK;
  return launch_invert<float, false, kTB32>(w, ldw, n, dinv, true, false, stream);
}

int couplings_f32(const float* w, int64_t ldw, int64_t n, float* dinv, cudaStream_t stream) {
  const int nblk = (int)((n + kTB32 - 1) / kTB32);
  if (nblk < 2) return RM_OK;
  const size_t smem = (size_t)kTB32 * (kTB32 + 1) * sizeof(float);
  RM_TRY(smem_attribute(coupling_kernel<float, false, kTB32>, 2 * smem));
  coupling_kernel<float, false, kTB32><<<dim3((unsigned)nblk, 2), 256, 2 * smem, stream>>>(w, ldw, n, dinv);
  RM_LAUNCHED();
  return RM_OK;
}

// pre = the block-Jacobi-scaled triangles of the row-major float32 L\U w: block (b, j) of pre is
// dinv[b][0] L_bj below the diagonal blocks (j < b) and dinv[b][1] U_bj above them (j > b);
// the diagonal blocks of pre are not written. With them a triangular solve is
// x_b = D_b^-1 y_b - sum_j pre_bj x_j: every block's last step is a single product.
// On the tensor cores, for 128-row blocks: out = D_b^-1 T_bj with
// 3xTF32 mma.sync (float32-level products), a CTA per 64-column half of a block (104 KB of
// shared memory: two CTAs per SM, so one CTA's loads overlap the other's products). 8 warps,
// warp w the rows 16w .. 16w+15 of the 8 column tiles; the operands in padded shared memory (A
// rows 132 floats apart, B rows 72: both fragment patterns hit 32 distinct banks).
__global__ void __launch_bounds__(256) premultiply_mma_kernel(const float* __restrict__ w, int64_t ldw, int64_t n,
                                                              const float* __restrict__ dinv, float* __restrict__ pre,
                                                              int64_t ldp) {
  constexpr int TB = 128, TN = 64, SA = 132, SB = 72;
  extern __shared__ uint8_t smraw[];
  float(*di)[SA] = reinterpret_cast<float(*)[SA]>(smraw);
  float(*ob)[SB] = reinterpret_cast<float(*)[SB]>(smraw + (size_t)TB * SA * sizeof(float));
  const int nblk = (int)((n + TB - 1) / TB);
  const int half = blockIdx.x & 1, blk = blockIdx.x >> 1;
  const int b = blk / nblk, j = blk % nblk;
  if (b == j) return;
  const int which = j < b ? 0 : 1;
  const int64_t r0 = (int64_t)b * TB, c0 = (int64_t)j * TB + half * TN;
  const float* dv = dinv + ((int64_t)b * kDiagMats + which) * TB * TB;
  {
    // both operands as 16-byte loads, all 24 of a thread's in flight before any store
    constexpr int PA = TB * TB / 4 / 256, PB = TB * TN / 4 / 256;  // float4 items per thread
    float4 va[PA], vb[PB];
#pragma unroll
    for (int q = 0; q < PA; ++q) va[q] = __ldg(reinterpret_cast<const float4*>(dv + (threadIdx.x + q * 256) * 4));
#pragma unroll
    for (int q = 0; q < PB; ++q) {
      const int e = (threadIdx.x + q * 256) * 4;
      const int i = e / TN, c = e % TN;
      const int64_t gi = r0 + i, gj = c0 + c;
      const float* src = w + gi * ldw + gj;
      if (gi < n && gj + 3 < n) {
        vb[q] = __ldcs(reinterpret_cast<const float4*>(src));
      } else {
        vb[q].x = (gi < n && gj < n) ? src[0] : 0.0f;
        vb[q].y = (gi < n && gj + 1 < n) ? src[1] : 0.0f;
        vb[q].z = (gi < n && gj + 2 < n) ? src[2] : 0.0f;
        vb[q].w = (gi < n && gj + 3 < n) ? src[3] : 0.0f;
      }
    }
#pragma unroll
    for (int q = 0; q < PA; ++q) {
      const int e = (threadIdx.x + q * 256) * 4;
      *reinterpret_cast<float4*>(&di[e / TB][e % TB]) = va[q];
    }
#pragma unroll
    for (int q = 0; q < PB; ++q) {
      const int e = (threadIdx.x + q * 256) * 4;
      *reinterpret_cast<float4*>(&ob[e / TN][e % TN]) = vb[q];
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
  const int ra = 16 * warp + g;
  float d[TN / 8][4];
#pragma unroll
  for (int nt = 0; nt < TN / 8; ++nt)
#pragma unroll
    for (int e = 0; e < 4; ++e) d[nt][e] = 0.f;
  for (int k8 = 0; k8 < TB; k8 += 8) {
    const float a[4] = {di[ra][k8 + tq], di[ra + 8][k8 + tq], di[ra][k8 + tq + 4], di[ra + 8][k8 + tq + 4]};
#pragma unroll
    for (int nt = 0; nt < TN / 8; ++nt) tc::mma_3xtf32(d[nt], a, ob[k8 + tq][8 * nt + g], ob[k8 + tq + 4][8 * nt + g]);
  }
  float* out = pre + r0 * ldp + c0;
#pragma unroll
  for (int nt = 0; nt < TN / 8; ++nt) {
    const int col = 8 * nt + 2 * tq;
    *reinterpret_cast<float2*>(out + (int64_t)ra * ldp + col) = make_float2(d[nt][0], d[nt][1]);
    *reinterpret_cast<float2*>(out + (int64_t)(ra + 8) * ldp + col) = make_float2(d[nt][2], d[nt][3]);
  }
}

int64_t premultiplied_f32_ld(int64_t n) { return (n + kTB32 - 1) / kTB32 * kTB32; }
size_t premultiplied_f32_bytes(int64_t n) {
  const int64_t ld = premultiplied_f32_ld(n);
  return (size_t)ld * ld * sizeof(float);
}

int premultiply_f32(const float* lu, int64_t ld, int64_t n, const float* dinv, float* pre, cudaStream_t stream) {
  const int nblk = (int)((n + kTB32 - 1) / kTB32);
  if (nblk < 2) return RM_OK;
  const size_t smem = (size_t)kTB32 * (132 + 72) * sizeof(float);
  RM_TRY(smem_attribute(premultiply_mma_kernel, smem));
  premultiply_mma_kernel<<<2 * nblk * nblk, 256, smem, stream>>>(lu, ld, n, dinv, pre, premultiplied_f32_ld(n));
  RM_LAUNCHED();
  return RM_OK;
}

// flags and tickets of both chains per chunk of columns (chunks of kPreKC, the narrower kind)
size_t trsv_f32_scratch_bytes(int64_t n, int64_t k) {
  return (size_t)(2 * ((n + kTB32 - 1) / kTB32 + 1)) * sizeof(int) * (size_t)((k + kPreKC - 1) / kPreKC) + 256;
}

// x = U^-1 L^-1 x in place for the row-major float32 L\\U (unit L) of an LU whose row
// permutation the caller has already applied to x. With pre (premultiply_f32 of the same
// factors; ld premultiplied_f32_ld(n)) the chains read the scaled triangles instead.
int lu_solve_f32_nopiv(const float* lu, int64_t ld, int64_t n, const float* dinv, const float* pre, float* x,
                       int64_t ldx, int64_t k, void* scratch, unsigned* status, cudaStream_t stream) {
  if (n == 0 || k == 0) return RM_OK;
  const int nblk = (int)((n + kTB32 - 1) / kTB32);
  const int chunks = (int)((k + kKC - 1) / kKC), pre_chunks = (int)((k + kPreKC - 1) / kPreKC);
  int* flags = reinterpret_cast<int*>(scratch);
  const int64_t stride = 2 * (nblk + 1);  // ints per chunk: lower flags + ticket, upper flags + ticket
  RM_CUDA_TRY(cudaMemsetAsync(flags, 0, (size_t)stride * sizeof(int) * (pre ? pre_chunks : chunks), stream));
  const int64_t ldp = premultiplied_f32_ld(n);
  if (pre) {
    // every chunk of kPreKC columns in one launch per triangle, side by side
    RM_TRY(launch_trsv_pre_ring<true>(pre, ldp, (int)n, dinv, x, ldx, (int)k, flags, flags + nblk, stride, status,
                                      stream));
    return launch_trsv_pre_ring<false>(pre, ldp, (int)n, dinv, x, ldx, (int)k, flags + nblk + 1, flags + 2 * nblk + 1,
                                       stride, status, stream);
  }
  for (int ch = 0; ch < chunks; ++ch) {
    const int kc = (int)std::min<int64_t>(kKC, k - (int64_t)ch * kKC);
    int* f = flags + (size_t)ch * stride;
    float* xc = x + ch * kKC;
    RM_TRY((launch_trsv<float, true, false, kTB32>(lu, ld, (int)n, dinv, xc, ldx, kc, f, f + nblk, status, stream)));
    RM_TRY((launch_trsv<float, false, false, kTB32>(lu, ld, (int)n, dinv, xc, ldx, kc, f + nblk + 1, f + 2 * nblk + 1,
                                                    status, stream)));
  }
  return RM_OK;
}

}  // namespace rm
