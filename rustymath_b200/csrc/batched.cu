// Batched solves of many small systems of uneven size (n <= 256, k <= 8) in one persistent
// launch: float32 LU with partial pivoting + float64 refinement per system, falling back to a
// float64 LU for the systems whose refinement stalls, all inside the same kernel.
//
// rustymath solves a stack of systems one LuWork per thread (Stacked::solve,
// src/linalg/stacked.rs:88-101, over parallel::stack, core/src/parallel.rs:118-192), each an
// lu_factor + lu_solve (core/src/linalg/factor.rs:617-641) and, when `regular` fails
// (factor.rs:221-226), least squares. Here a CTA takes one system at a time from a shared
// counter (systems sorted by size, largest first, so the long ones start early) and:
//   - loads A (float64, row-major) into a float32 working copy W in its own slice of a global
//     scratch (W stays in L2 while the CTA works on it); thread r owns row r;
//   - factors W with partial pivoting, implicitly: rows never move, a row chosen as pivot of
//     logical column c records pos = c and leaves the candidates; in panels of NB columns
//     (16 or 32, picked per size bucket by the tuner) each thread keeps its row's panel in
//     registers and each column costs one barrier (every warp posts its best candidate row,
//     every thread picks the winner among the posts: largest |pivot|, lowest row on ties, NaN
//     never chosen over a number); then U12 of the panel's pivot rows (a column per thread)
//     and the update of the rows not chosen yet;
//   - solves L U x = P b with the rows' right-hand sides in registers, block by block (a warp
//     per right-hand side solves each NB x NB diagonal block with shuffles);
//   - refines in float64: r = b - A x (a warp per row of A, x in shared memory), the normwise
//     backward error max_c ||r_c|| / (||A|| ||x_c|| + ||b_c||), and corrections from the
//     float32 factors until it is at most the tolerance (n * 2^-53 by default);
//   - on a stall (the error not halving) or the step limit, redoes the system in float64
//     (the same code on float64 items, reusing the slice) and reports the fallback; a pivot
//     at most eps * n * max|a| there marks the system not regular, as rustymath's `regular`.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <numeric>
#include <vector>

#include "rm_internal.h"

namespace rm {
namespace bt {

constexpr int THREADS = 256;
constexpr int WARPS = THREADS / 32;
constexpr int NMAX = 256;  // rows of a system: a thread per row
constexpr int KMAX = 8;    // right-hand sides of a system
constexpr int SLOT_BYTES = 144;
constexpr int UBT_BYTES = NMAX * 20 * 8;  // U12 transposed: NMAX x (NB + 4) items, either type

// result flags per system
constexpr int FLAG_FELL_BACK = 1;
constexpr int FLAG_NOT_REGULAR = 2;
constexpr int FLAG_NO_CONVERGENCE = 4;

struct Smem {
  alignas(16) unsigned char slot[2][WARPS][SLOT_BYTES];  // posts: NB items, then key (T), row
  alignas(16) unsigned char lp[32 * 36 * 4];              // the panel's pivot rows (NB x (NB + 4) items)
  alignas(16) unsigned char ubt[UBT_BYTES];               // U12 of a panel, transposed
  alignas(16) double xs[NMAX][KMAX + 1];                  // the float64 solution, by unknown (rows
  alignas(16) double rs[NMAX][KMAX + 1];                  //  padded: a warp's rows on distinct banks)
  alignas(16) double vsm[32][KMAX + 1];                   // a diagonal block's right-hand sides
  int piv[NMAX];                                          // logical position -> row
  int act[NMAX];                                          // the rows still unchosen after a panel
  double colsum[NMAX];                                    // column sums of |a| (dominance test)
  double amax_a;                                          // max |a_ij|, NaN ignored
  int wcnt[WARPS];
  double red[WARPS][3 * KMAX + 1];
  double anorm, bnorm[KMAX];
  int zero_pivot;
};

// Rows of the panel multipliers (staged in xs..rs during a factorization) and of U12 (ubt): 144
// bytes, so that a quarter-warp's 16-byte accesses to consecutive rows fall on distinct banks.
template <typename T>
struct Stage {
  static constexpr int LDU = 144 / (int)sizeof(T);
};
static_assert(offsetof(Smem, rs) == offsetof(Smem, xs) + sizeof(Smem::xs), "xs and rs are adjacent");
static_assert(sizeof(Smem::xs) + sizeof(Smem::rs) >= (size_t)NMAX * 144, "the multipliers fit in xs..rs");
static_assert(UBT_BYTES >= NMAX * 144, "U12 fits in ubt");

// n items of a row into registers, 16-byte loads when the whole panel is there (rows and panel
// starts are 16-byte aligned: ld % 4 == 0, panels start at multiples of NB)
template <typename T, int NB>
__device__ __forceinline__ void load_row(const T* src, int cnt, T (&v)[NB]) {
  if (cnt == NB) {
    constexpr int PER = 16 / (int)sizeof(T);
#pragma unroll
    for (int q = 0; q < NB; q += PER) {
      if constexpr (sizeof(T) == 4) {
        const float4 t = *reinterpret_cast<const float4*>(src + q);
        v[q] = t.x, v[q + 1] = t.y, v[q + 2] = t.z, v[q + 3] = t.w;
      } else {
        const double2 t = *reinterpret_cast<const double2*>(src + q);
        v[q] = t.x, v[q + 1] = t.y;
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < NB; ++q) v[q] = q < cnt ? src[q] : T(0);
  }
}

template <typename T, int NB>
__device__ __forceinline__ void store_vec(T* dst, const T (&v)[NB]) {
  constexpr int PER = 16 / (int)sizeof(T);
#pragma unroll
  for (int q = 0; q < NB; q += PER) {
    if constexpr (sizeof(T) == 4)
      *reinterpret_cast<float4*>(dst + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
    else
      *reinterpret_cast<double2*>(dst + q) = make_double2(v[q], v[q + 1]);
  }
}

template <typename T, int NB>
__device__ __forceinline__ void load_vec(const T* src, T (&v)[NB]) {
  constexpr int PER = 16 / (int)sizeof(T);
#pragma unroll
  for (int q = 0; q < NB; q += PER) {
    if constexpr (sizeof(T) == 4) {
      const float4 t = *reinterpret_cast<const float4*>(src + q);
      v[q] = t.x, v[q + 1] = t.y, v[q + 2] = t.z, v[q + 3] = t.w;
    } else {
      const double2 t = *reinterpret_cast<const double2*>(src + q);
      v[q] = t.x, v[q + 1] = t.y;
    }
  }
}

template <typename T>
__device__ __forceinline__ T tabs(T v) {
  return v < T(0) ? -v : v;
}

// rustymath's divide: multiply by the reciprocal unless the pivot is subnormal
__device__ __forceinline__ double bdivide(double x, double piv) {
  return fabs(piv) < DBL_MIN ? x / piv : x * (1.0 / piv);
}
__device__ __forceinline__ float bdivide(float x, float piv) {
  return fabsf(piv) < FLT_MIN ? x / piv : x * __frcp_rn(piv);
}

template <typename T>
__device__ __forceinline__ void warp_argmax(T& v, int& i) {
#pragma unroll
  for (int off = 16; off; off >>= 1) {
    const T ov = __shfl_xor_sync(0xffffffffu, v, off);
    const int oi = __shfl_xor_sync(0xffffffffu, i, off);
    if (ov > v || (ov == v && oi < i)) {
      v = ov;
      i = oi;
    }
  }
}

// Loads the n x n row-major float64 a into W (row-major, ld), converted to T: a warp per
// row, lanes along it.
template <typename T>
__device__ void load_w(const double* __restrict__ a, int n, T* W, int ld) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r = warp; r < n; r += WARPS)
    for (int j = lane; j < n; j += 32) W[(int64_t)r * ld + j] = (T)__ldcs(a + (int64_t)r * n + j);
}

// Relative margin of the column diagonal dominance that lets a factorization skip the pivot
// search: |a_jj| - sum_{i != j} |a_ij| > kDominance * sum_i |a_ij| for every column j.
constexpr double kDominance = 1e-10;

// load_w, and whether a is strictly column diagonally dominant with the margin kDominance
// (the same answer in every thread). On such a matrix partial pivoting chooses the diagonal at
// every step: the Schur complements of a column diagonally dominant matrix keep that dominance
// with at least the same excess, so in column c the diagonal item is larger than the sum, and so
// than the largest, of the others below it. The margin covers the float64 rounding of the
// updates (growth at most 2, n <= 256: far below 1e-10 of a column's sum); NaN or a zero column
// fail the test.
template <typename T>
__device__ bool load_w_dominant(const double* __restrict__ a, int n, T* W, int ld, Smem& sm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int j = threadIdx.x; j < NMAX; j += THREADS) sm.colsum[j] = 0.0;
  __syncthreads();
  double cs[NMAX / 32], amax = 0.0;
#pragma unroll
  for (int q = 0; q < NMAX / 32; ++q) cs[q] = 0.0;
  // two rows per warp at a time: all sixteen of a lane's loads in flight before the first store
  for (int r = warp; r < n; r += 2 * WARPS) {
    const int r1 = r + WARPS;
    double v0[NMAX / 32], v1[NMAX / 32];
#pragma unroll
    for (int q = 0; q < NMAX / 32; ++q) {
      const int j = lane + 32 * q;
      v0[q] = j < n ? __ldcs(a + (int64_t)r * n + j) : 0.0;
      v1[q] = (j < n && r1 < n) ? __ldcs(a + (int64_t)r1 * n + j) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < NMAX / 32; ++q) {
      const int j = lane + 32 * q;
      if (j < n) {
        W[(int64_t)r * ld + j] = (T)v0[q];
        cs[q] += fabs(v0[q]);
        amax = fmax(amax, fabs(v0[q]));
        if (r1 < n) {
          W[(int64_t)r1 * ld + j] = (T)v1[q];
          cs[q] += fabs(v1[q]);
          amax = fmax(amax, fabs(v1[q]));
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < NMAX / 32; ++q)
    if (lane + 32 * q < n) atomicAdd(&sm.colsum[lane + 32 * q], cs[q]);
  // max |a| ignoring NaN (rustymath's greatest, factor.rs:488), for the regular test
#pragma unroll
  for (int off = 16; off; off >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, off));
  if (lane == 0) sm.red[warp][0] = amax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double big = 0.0;
    for (int w = 0; w < WARPS; ++w) big = fmax(big, sm.red[w][0]);
    sm.amax_a = big;
  }
  bool ok = true;
  const int j = threadIdx.x;
  if (j < n) {
    const double d = fabs(a[(int64_t)j * n + j]), sum = sm.colsum[j];
    ok = d - (sum - d) > kDominance * sum;  // false for NaN
  }
  return __syncthreads_and(ok ? 1 : 0) != 0;
}

// After a panel (columns J..J+nbj) is factored: the pivot rows' later columns become U12 =
// L11^-1 A12 (a column per thread; U12 to shared memory) and the nact rows still unchosen,
// sm.act[0..nact) with their multipliers in Lsm, take A22 -= L21 U12. A thread per column does
// the update (reads of a row's columns are coalesced across the warp), the U12 column in
// registers and the row's multipliers broadcast from shared memory; when the columns are few,
// groups of threads take interleaved rows. Ends before the closing barrier.
template <typename T, int NB>
__device__ __forceinline__ void panel_tail(T* W, int ld, int n, Smem& sm, int J, int nbj, int nact) {
  const int tid = threadIdx.x;
  constexpr int LDU = Stage<T>::LDU;
  T(*Lp)[NB + 4] = reinterpret_cast<T(*)[NB + 4]>(sm.lp);
  T* UbT = reinterpret_cast<T*>(sm.ubt);
  const T* Lsm = reinterpret_cast<const T*>(sm.xs);
  const int rc0 = J + nbj, rcols = n - rc0;
  if (rcols <= 0) return;
    // U12 of the panel's pivot rows: u = Lp^-1 (their later columns), a column per thread
    for (int j = tid; j < rcols; j += THREADS) {
      T u[NB];
#pragma unroll
      for (int c = 0; c < NB; ++c) u[c] = c < nbj ? W[(int64_t)sm.piv[J + c] * ld + rc0 + j] : T(0);
#pragma unroll
      for (int c = 1; c < NB; ++c)
#pragma unroll
        for (int q = 0; q < c; ++q) u[c] = fma(-Lp[c][q], u[q], u[c]);
#pragma unroll
      for (int c = 0; c < NB; ++c)
        if (c < nbj) W[(int64_t)sm.piv[J + c] * ld + rc0 + j] = u[c];
      store_vec<T, NB>(UbT + j * LDU, u);
    }
    __syncthreads();
    // the rows not chosen yet: later columns -= L(row, panel) U12, a thread per column (reads of
    // a row's columns coalesced across the warp), the U12 column in registers, the row's
    // multipliers broadcast from shared memory; when the columns are few, groups of threads
    // take interleaved rows
    const int width = (rcols + 31) & ~31;
    const int groups = THREADS / width;
    const int g = tid / width, j = tid - g * width;
    if (g < groups && j < rcols) {
      T u[NB];
      load_vec<T, NB>(UbT + j * LDU, u);
      T* col = W + rc0 + j;
      int idx = g;
      // four rows at a time; the next four rows' items are loaded while these four are updated
      T n0 = T(0), n1 = T(0), n2 = T(0), n3 = T(0);
      if (idx + 3 * groups < nact) {
        n0 = col[(int64_t)sm.act[idx] * ld];
        n1 = col[(int64_t)sm.act[idx + groups] * ld];
        n2 = col[(int64_t)sm.act[idx + 2 * groups] * ld];
        n3 = col[(int64_t)sm.act[idx + 3 * groups] * ld];
      }
      for (; idx + 3 * groups < nact; idx += 4 * groups) {
        const int r0 = sm.act[idx], r1 = sm.act[idx + groups], r2 = sm.act[idx + 2 * groups],
                  r3 = sm.act[idx + 3 * groups];
        T x0 = n0, x1 = n1, x2 = n2, x3 = n3;
        const int nxt = idx + 4 * groups;
        if (nxt + 3 * groups < nact) {
          n0 = col[(int64_t)sm.act[nxt] * ld];
          n1 = col[(int64_t)sm.act[nxt + groups] * ld];
          n2 = col[(int64_t)sm.act[nxt + 2 * groups] * ld];
          n3 = col[(int64_t)sm.act[nxt + 3 * groups] * ld];
        }
        constexpr int PER = 16 / (int)sizeof(T);
#pragma unroll
        for (int c = 0; c < NB; c += PER) {
          T a0[PER], a1[PER], a2[PER], a3[PER];
          load_vec<T, PER>(Lsm + r0 * LDU + c, a0);
          load_vec<T, PER>(Lsm + r1 * LDU + c, a1);
          load_vec<T, PER>(Lsm + r2 * LDU + c, a2);
          load_vec<T, PER>(Lsm + r3 * LDU + c, a3);
#pragma unroll
          for (int q = 0; q < PER; ++q) {
            x0 = fma(-a0[q], u[c + q], x0);
            x1 = fma(-a1[q], u[c + q], x1);
            x2 = fma(-a2[q], u[c + q], x2);
            x3 = fma(-a3[q], u[c + q], x3);
          }
        }
        col[(int64_t)r0 * ld] = x0;
        col[(int64_t)r1 * ld] = x1;
        col[(int64_t)r2 * ld] = x2;
        col[(int64_t)r3 * ld] = x3;
      }
      for (; idx < nact; idx += groups) {
        const int r0 = sm.act[idx];
        T x0 = col[(int64_t)r0 * ld];
        constexpr int PER = 16 / (int)sizeof(T);
#pragma unroll
        for (int c = 0; c < NB; c += PER) {
          T a0[PER];
          load_vec<T, PER>(Lsm + r0 * LDU + c, a0);
#pragma unroll
          for (int q = 0; q < PER; ++q) x0 = fma(-a0[q], u[c + q], x0);
        }
        col[(int64_t)r0 * ld] = x0;
      }
    }
}

// Implicitly pivoted LU of the n x n W (row-major, ld): thread r owns row r; my_pos (in/out)
// is the logical position of row r, -1 before it is chosen; sm.piv[c] is the row chosen for
// column c. Returns with every thread's my_pos set. A zero pivot sets sm.zero_pivot and
// leaves its column unreduced.
template <typename T, int NB>
__device__ void bfactor_pivoted(T* W, int ld, int n, Smem& sm, int& my_pos) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r = tid;
  constexpr int LDU = Stage<T>::LDU;
  static_assert(NB <= LDU, "a staged row holds the panel");
  T(*Lp)[NB + 4] = reinterpret_cast<T(*)[NB + 4]>(sm.lp);
  T* UbT = reinterpret_cast<T*>(sm.ubt);   // NMAX x LDU: column j of U12 at UbT[j * LDU]
  T* Lsm = reinterpret_cast<T*>(sm.xs);    // NMAX x LDU: row r's panel multipliers (xs..rs are free here)
  bool active = r < n;
  my_pos = -1;
  for (int J = 0; J < n; J += NB) {
    const int nbj = min(NB, n - J);
    const bool was_active = active;
    T p[NB];
    T* row = W + (int64_t)r * ld + J;
    if (active) load_row<T, NB>(row, nbj, p);
    else
#pragma unroll
      for (int i = 0; i < NB; ++i) p[i] = T(0);
#pragma unroll
    for (int c = 0; c < NB; ++c) {
      if (c < nbj) {
        unsigned char(*sl)[SLOT_BYTES] = sm.slot[c & 1];
        T key = T(-1);
        int idx = r, bi, bw;
        if (sizeof(T) == 4) {
          // float: |pivot| as an ordered 32-bit key (0 none, 1 NaN, bits + 2), redux max + ballot
          const float v = fabsf((float)p[c]);
          const unsigned uk = active ? (v != v ? 1u : __float_as_uint(v) + 2u) : 0u;
          const unsigned wmax = __reduce_max_sync(0xffffffffu, uk);
          const int wl = __ffs(__ballot_sync(0xffffffffu, uk == wmax)) - 1;
          if (lane == wl) {
            T* post = reinterpret_cast<T*>(sl[warp]);
#pragma unroll
            for (int i = 0; i < NB; ++i) post[i] = p[i];
            *reinterpret_cast<unsigned*>(sl[warp] + 128) = wmax;
            *reinterpret_cast<int*>(sl[warp] + 136) = r;
          }
          __syncthreads();
          const unsigned kq = lane < WARPS ? *reinterpret_cast<const unsigned*>(sl[lane] + 128) : 0u;
          const unsigned gmax = __reduce_max_sync(0xffffffffu, kq);
          const unsigned gball = __ballot_sync(0xffffffffu, lane < WARPS && kq == gmax);
          bw = gball ? __ffs(gball) - 1 : 0;
          bi = *reinterpret_cast<const int*>(sl[bw] + 136);
        } else {
          if (active) {
            const T v = tabs(p[c]);
            key = v != v ? T(-0.5) : v;
          }
          warp_argmax(key, idx);
          if (lane == (idx & 31)) {
            T* post = reinterpret_cast<T*>(sl[warp]);
#pragma unroll
            for (int i = 0; i < NB; ++i) post[i] = p[i];
            *reinterpret_cast<T*>(sl[warp] + 128) = key;
            *reinterpret_cast<int*>(sl[warp] + 136) = idx;
          }
          __syncthreads();
          T bk = *reinterpret_cast<const T*>(sl[0] + 128);
          bi = *reinterpret_cast<const int*>(sl[0] + 136), bw = 0;
#pragma unroll
          for (int w = 1; w < WARPS; ++w) {
            const T k2 = *reinterpret_cast<const T*>(sl[w] + 128);
            const int i2 = *reinterpret_cast<const int*>(sl[w] + 136);
            if (k2 > bk || (k2 == bk && i2 < bi)) {
              bk = k2;
              bi = i2;
              bw = w;
            }
          }
        }
        const T* prow = reinterpret_cast<const T*>(sl[bw]);
        const T piv = prow[c];
        if (warp == (bi >> 5)) {
          if (r == bi) {
            active = false;
            my_pos = J + c;
            sm.piv[J + c] = r;
#pragma unroll
            for (int i = 0; i < NB; ++i) Lp[c][i] = p[i];
          }
        }
        if (active) {
          if (piv != T(0)) {
            const T l = bdivide(p[c], piv);
            p[c] = l;
#pragma unroll
            for (int i = c + 1; i < NB; ++i) p[i] = fma(-l, prow[i], p[i]);
          }
        }
        if (piv == T(0) && tid == 0) sm.zero_pivot = 1;
      }
    }
    if (was_active) {
#pragma unroll
      for (int i = 0; i < NB; ++i)
        if (i < nbj) row[i] = p[i];
    }
    const int rc0 = J + nbj, rcols = n - rc0;
    // the rows still unchosen, in increasing order, and their multipliers in shared memory
    const unsigned ball = __ballot_sync(0xffffffffu, active);
    if (lane == 0) sm.wcnt[warp] = __popc(ball);
    if (active && rcols > 0) store_vec<T, NB>(Lsm + r * LDU, p);
    __syncthreads();
    int base = 0, nact = 0;
#pragma unroll
    for (int w = 0; w < WARPS; ++w) {
      const int c = sm.wcnt[w];
      base += w < warp ? c : 0;
      nact += c;
    }
    if (active) sm.act[base + __popc(ball & ((1u << lane) - 1u))] = r;
    panel_tail<T, NB>(W, ld, n, sm, J, nbj, nact);
    __syncthreads();
  }
}

// The factorization of a matrix that load_w_dominant found column diagonally dominant: the
// pivot of column c is row c, so there is no pivot search and no barrier per column. Per
// panel, warp 0 factors the diagonal block with its rows in registers (lane i holds row J + i,
// the pivot row's items passed by shuffles), then every row below solves its own multipliers
// against U11 from shared memory, then panel_tail. Every item is computed by the same
// operations in the same order as bfactor_pivoted would with those pivots, so the results
// are the same bits.
template <typename T, int NB>
__device__ void bfactor_dominant(T* W, int ld, int n, Smem& sm, int& my_pos) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r = tid;
  constexpr int LDU = Stage<T>::LDU;
  T(*Lp)[NB + 4] = reinterpret_cast<T(*)[NB + 4]>(sm.lp);
  T* Lsm = reinterpret_cast<T*>(sm.xs);
  my_pos = r < n ? r : -1;
  for (int i = tid; i < n; i += THREADS) sm.piv[i] = i;
  for (int J = 0; J < n; J += NB) {
    const int nbj = min(NB, n - J);
    const int rc0 = J + nbj, rcols = n - rc0;
    if (warp == 0) {
      // lane i holds row J + i; at step c every lane reads the pivot row (final since step c - 1)
      // from Lp with 16-byte broadcast loads, and the next pivot row's lane stores its row there
      const bool mine = lane < nbj;
      T p[NB];
      if (mine) load_row<T, NB>(W + (int64_t)(J + lane) * ld + J, nbj, p);
      else
#pragma unroll
        for (int i = 0; i < NB; ++i) p[i] = T(0);
      if (lane == 0) store_vec<T, NB>(&Lp[0][0], p);
      __syncwarp();
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        if (c < nbj) {
          T prow[NB];
          load_vec<T, NB>(&Lp[c][0], prow);
          const T piv = prow[c];
          if (lane > c && mine && piv != T(0)) {
            const T l = bdivide(p[c], piv);
            p[c] = l;
#pragma unroll
            for (int i = c + 1; i < NB; ++i) p[i] = fma(-l, prow[i], p[i]);
          }
          if (piv == T(0) && lane == 0) sm.zero_pivot = 1;
          if (lane == c + 1 && c + 1 < NB) store_vec<T, NB>(&Lp[lane][0], p);
          __syncwarp();
        }
      }
      if (mine) {
        T* row = W + (int64_t)(J + lane) * ld + J;
#pragma unroll
        for (int i = 0; i < NB; ++i)
          if (i < nbj) row[i] = p[i];
      }
    }
    __syncthreads();
    // the rows below the block: their multipliers, against U11 in Lp
    if (r >= rc0 && r < n) {
      T p[NB];
      T* row = W + (int64_t)r * ld + J;
      load_row<T, NB>(row, nbj, p);
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        if (c < nbj) {
          const T piv = Lp[c][c];
          if (piv != T(0)) {
            const T l = bdivide(p[c], piv);
            p[c] = l;
#pragma unroll
            for (int i = c + 1; i < NB; ++i) p[i] = fma(-l, Lp[c][i], p[i]);
          }
        }
      }
#pragma unroll
      for (int i = 0; i < NB; ++i)
        if (i < nbj) row[i] = p[i];
      if (rcols > 0) store_vec<T, NB>(Lsm + r * LDU, p);
    }
    for (int i = tid; i < rcols; i += THREADS) sm.act[i] = rc0 + i;
    panel_tail<T, NB>(W, ld, n, sm, J, nbj, rcols);
    __syncthreads();
  }
}

// LU of the n x n W (row-major, ld) with partial pivoting: thread r owns row r; on return
// my_pos is the logical position of row r and sm.piv[c] the row chosen for column c. A zero
// pivot sets sm.zero_pivot and leaves its column unreduced.
template <typename T, int NB>
__device__ void bfactor(T* W, int ld, int n, Smem& sm, int& my_pos, bool dominant) {
  if (dominant) bfactor_dominant<T, NB>(W, ld, n, sm, my_pos);
  else bfactor_pivoted<T, NB>(W, ld, n, sm, my_pos);
}

// Copies cnt items of a row segment (16-byte aligned, the row padded to a multiple of 16 bytes
// past cnt) to shared memory with 16-byte asynchronous copies, in one commit group of the thread.
template <typename T>
__device__ __forceinline__ void copy_segment(T* dst, const T* src, int cnt) {
  constexpr int PER = 16 / (int)sizeof(T);
  for (int q = 0; q < cnt; q += PER) cp_async16(dst + q, src + q);
  cp_async_commit();
}

// Solves L U x = P v: thread r holds v (its row's k right-hand sides) on entry and x[my_pos]
// on return. W holds the implicitly pivoted factors of bfactor<T, NB>.
template <typename T, int NB, int KK>
__device__ void bsolve(const T* W, int ld, int n, int k, Smem& sm, int my_pos, T (&v)[KK]) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r = tid;
  const T* row = W + (int64_t)r * ld;
  // forward: blocks of NB logical columns. A block's loads (the thread's row segment, and for the
  // solving warps their row of the diagonal block) are issued first, so that their latency
  // overlaps the barrier and the shuffle chain instead of following them.
  for (int J = 0; J < n; J += NB) {
    const int nbj = min(NB, n - J);
    const bool upd = r < n && my_pos >= J + nbj;
    T* seg = reinterpret_cast<T*>(sm.ubt + r * 144);  // this row's segment, copied asynchronously
    if (upd) copy_segment<T>(seg, row + J, nbj);
    T lv[NB];
    if (my_pos >= J && my_pos < J + nbj)
#pragma unroll
      for (int c = 0; c < KK; ++c) sm.vsm[my_pos - J][c] = (double)v[c];
    __syncthreads();
    if (warp < k) {  // a warp per right-hand side: column c = warp, lane = row of the block
      const int c = warp;
      load_row<T, NB>(W + (int64_t)(lane < nbj ? sm.piv[J + lane] : 0) * ld + J, nbj, lv);
      T y = lane < nbj ? (T)sm.vsm[lane][c] : T(0);
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        if (q < nbj) {
          const T yq = __shfl_sync(0xffffffffu, y, q);
          if (lane > q && lane < nbj) y = fma(-lv[q], yq, y);
        }
      }
      if (lane < nbj) sm.vsm[lane][c] = (double)y;
    }
    __syncthreads();
    if (upd) {
      cp_async_wait<0>();
      load_vec<T, NB>(seg, lv);
#pragma unroll
      for (int q = 0; q < NB; ++q)
        if (q < nbj) {
#pragma unroll
          for (int c = 0; c < KK; ++c)
            if (c < k) v[c] = fma(-lv[q], (T)sm.vsm[q][c], v[c]);
        }
    } else if (r < n && my_pos >= J && my_pos < J + nbj) {
#pragma unroll
      for (int c = 0; c < KK; ++c) v[c] = (T)sm.vsm[my_pos - J][c];
    }
    __syncthreads();
  }
  // backward, with the same early loads
  const int last = (n - 1) / NB * NB;
  for (int J = last; J >= 0; J -= NB) {
    const int nbj = min(NB, n - J);
    const bool upd = r < n && my_pos >= 0 && my_pos < J;
    T* seg = reinterpret_cast<T*>(sm.ubt + r * 144);
    if (upd) copy_segment<T>(seg, row + J, nbj);
    T uv[NB];
    if (my_pos >= J && my_pos < J + nbj)
#pragma unroll
      for (int c = 0; c < KK; ++c) sm.vsm[my_pos - J][c] = (double)v[c];
    __syncthreads();
    if (warp < k) {  // a warp per right-hand side
      const int c = warp;
      load_row<T, NB>(W + (int64_t)(lane < nbj ? sm.piv[J + lane] : 0) * ld + J, nbj, uv);
      T y = lane < nbj ? (T)sm.vsm[lane][c] : T(0);
#pragma unroll
      for (int q = NB - 1; q >= 0; --q) {
        if (q < nbj) {
          if (lane == q) y = y / uv[q];
          const T xq = __shfl_sync(0xffffffffu, y, q);
          if (lane < q) y = fma(-uv[q], xq, y);
        }
      }
      if (lane < nbj) sm.vsm[lane][c] = (double)y;
    }
    __syncthreads();
    if (upd) {
      cp_async_wait<0>();
      load_vec<T, NB>(seg, uv);
#pragma unroll
      for (int q = 0; q < NB; ++q)
        if (q < nbj) {
#pragma unroll
          for (int c = 0; c < KK; ++c)
            if (c < k) v[c] = fma(-uv[q], (T)sm.vsm[q][c], v[c]);
        }
    } else if (r < n && my_pos >= J && my_pos < J + nbj) {
#pragma unroll
      for (int c = 0; c < KK; ++c) v[c] = (T)sm.vsm[my_pos - J][c];
    }
    __syncthreads();
  }
}

// sm.rs = b - A sm.xs for the n x n row-major a (a warp per row, lanes along it) and returns
// the normwise backward error (NaN if a residual is NaN). The first call (sm.anorm < 0)
// also forms ||A||_inf and ||b_c||_inf.
template <int KK>
__device__ double bresidual(const double* __restrict__ a, const double* __restrict__ b, int n, int k, Smem& sm) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool first = sm.anorm < 0.0;
  double rmax[KK], bmax[KK], xmax[KK], amax = 0.0;
#pragma unroll
  for (int c = 0; c < KK; ++c) {
    rmax[c] = bmax[c] = 0.0;
    xmax[c] = tid < n ? fabs(sm.xs[tid][c]) : 0.0;
  }
  // the lane's items of a row, all in flight before the first is used; the next row's are
  // loaded while this one is reduced
  double av[NMAX / 32];
#pragma unroll
  for (int q = 0; q < NMAX / 32; ++q)
    av[q] = (warp < n && lane + 32 * q < n) ? __ldcs(a + (int64_t)warp * n + lane + 32 * q) : 0.0;
  for (int r = warp; r < n; r += WARPS) {
    const double bv = lane < k ? b[(int64_t)r * k + lane] : 0.0;  // in flight beside the row
    double nx[NMAX / 32];
    const int rn = r + WARPS;
#pragma unroll
    for (int q = 0; q < NMAX / 32; ++q)
      nx[q] = (rn < n && lane + 32 * q < n) ? __ldcs(a + (int64_t)rn * n + lane + 32 * q) : 0.0;
    double acc[KK], asum = 0.0;
#pragma unroll
    for (int c = 0; c < KK; ++c) acc[c] = 0.0;
#pragma unroll
    for (int q = 0; q < NMAX / 32; ++q) {
      const int j = lane + 32 * q;
      if (j < n) {
        asum += fabs(av[q]);
#pragma unroll
        for (int c = 0; c < KK; ++c)
          if (c < k) acc[c] = fma(av[q], sm.xs[j][c], acc[c]);
      }
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
      asum += __shfl_xor_sync(0xffffffffu, asum, off);
#pragma unroll
      for (int c = 0; c < KK; ++c)
        if (c < k) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], off);
    }
    amax = fmax(amax, asum);
    if (lane < k) {
      double mine = 0.0;
#pragma unroll
      for (int c = 0; c < KK; ++c)
        if (c == lane) mine = acc[c];
      const double rv = bv - mine;
      sm.rs[r][lane] = rv;
#pragma unroll
      for (int c = 0; c < KK; ++c)
        if (c == lane) {
          rmax[c] = (fabs(rv) > rmax[c] || rv != rv) ? fabs(rv) : rmax[c];
          bmax[c] = fmax(bmax[c], fabs(bv));
        }
    }
#pragma unroll
    for (int q = 0; q < NMAX / 32; ++q) av[q] = nx[q];
  }
  // the lanes of a warp hold different columns: combine per warp, then across warps
#pragma unroll
  for (int c = 0; c < KK; ++c) {
    double rv = rmax[c], bv = bmax[c], xv = xmax[c];
#pragma unroll
    for (int off = 16; off; off >>= 1) {
      const double o = __shfl_xor_sync(0xffffffffu, rv, off);
      rv = (o > rv || o != o) ? o : rv;
      bv = fmax(bv, __shfl_xor_sync(0xffffffffu, bv, off));
      xv = fmax(xv, __shfl_xor_sync(0xffffffffu, xv, off));
    }
    rmax[c] = rv, bmax[c] = bv, xmax[c] = xv;
  }
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < KK; ++c) {
      sm.red[warp][c] = rmax[c];
      sm.red[warp][KMAX + c] = bmax[c];
      sm.red[warp][2 * KMAX + c] = xmax[c];
    }
    sm.red[warp][3 * KMAX] = amax;
  }
  __syncthreads();
  double berr = 0.0;
  bool nan = false;
  if (first) {
    double an = 0.0;
    for (int w = 0; w < WARPS; ++w) an = fmax(an, sm.red[w][3 * KMAX]);
    if (tid == 0) sm.anorm = an;
    for (int c = 0; c < k; ++c) {
      double bn = 0.0;
      for (int w = 0; w < WARPS; ++w) bn = fmax(bn, sm.red[w][KMAX + c]);
      if (tid == 0) sm.bnorm[c] = bn;
    }
  }
  __syncthreads();
  for (int c = 0; c < k; ++c) {
    double rn = 0.0, xn = 0.0;
    for (int w = 0; w < WARPS; ++w) {
      const double o = sm.red[w][c];
      rn = (o > rn || o != o) ? o : rn;
      xn = fmax(xn, sm.red[w][2 * KMAX + c]);
    }
    nan |= rn != rn;
    const double den = sm.anorm * xn + sm.bnorm[c];
    berr = fmax(berr, den > 0.0 ? rn / den : rn);
  }
  __syncthreads();
  return nan ? __longlong_as_double(0x7ff8000000000000ll) : berr;
}

struct Batch {
  int first, last;  // items [first, last) of the processing order
  const int* sys;   // item -> system
  const int* nb;    // item -> panel width (16 or 32)
  const int* n;
  const int* k;
  const int64_t* a_off;
  const int64_t* b_off;
  const int64_t* x_off;
  const int64_t* w_off;  // bytes
  const double* a;
  const double* b;
  double* x;
  unsigned char* w;
  int method;  // RM_METHOD_*
  int max_it;
  double tol;  // 0: n * 2^-53
  int fallback;
  double* berr;  // per system
  int* iters;
  int* flags;
  int* counter;
  int* piv;            // per system (at p_off): the row chosen for each logical column
  const int64_t* p_off;
  int* ftype;          // per system: 0 when W holds float32 factors, 1 for float64
};

template <typename T, int NB, int KK>
__device__ bool factor_and_solve(Batch& bt, Smem& sm, int n, int k, int ld, T* W, const double* a, const double* b,
                                 int& my_pos) {
  const bool dominant = load_w_dominant<T>(a, n, W, ld, sm);
  if (threadIdx.x == 0) sm.zero_pivot = 0;
  __syncthreads();
  bfactor<T, NB>(W, ld, n, sm, my_pos, dominant);
  T v[KK];
#pragma unroll
  for (int c = 0; c < KK; ++c) v[c] = (threadIdx.x < n && c < k) ? (T)b[(int64_t)threadIdx.x * k + c] : T(0);
  bsolve<T, NB, KK>(W, ld, n, k, sm, my_pos, v);
  if (my_pos >= 0)
#pragma unroll
    for (int c = 0; c < KK; ++c) sm.xs[my_pos][c] = (double)v[c];
  __syncthreads();
  return sm.zero_pivot == 0;
}

template <typename T, int NB, int KK>
__device__ void correct(Batch& bt, Smem& sm, int n, int k, int ld, const T* W, int my_pos) {
  T v[KK];
#pragma unroll
  for (int c = 0; c < KK; ++c) v[c] = (threadIdx.x < n && c < k) ? (T)sm.rs[threadIdx.x][c] : T(0);
  bsolve<T, NB, KK>(W, ld, n, k, sm, my_pos, v);
  if (my_pos >= 0)
#pragma unroll
    for (int c = 0; c < KK; ++c) sm.xs[my_pos][c] += (double)v[c];
  __syncthreads();
}

// One system with at most KK right-hand sides (the solves and residuals loop over KK columns).
template <int KK>
__device__ void solve_system(Batch& bt, Smem& sm, int n, int k, int nb, int ld, const double* a, const double* b,
                             unsigned char* w, int& my_pos, int& iters, int& flags, double& berr, bool& done) {
  if (bt.method == RM_METHOD_F32_IR) {
    float* W = reinterpret_cast<float*>(w);
    if (nb == 32) factor_and_solve<float, 32, KK>(bt, sm, n, k, ld, W, a, b, my_pos);
    else factor_and_solve<float, 16, KK>(bt, sm, n, k, ld, W, a, b, my_pos);
    const double tol = bt.tol > 0.0 ? bt.tol : (double)n * 0x1.0p-53;
    double prev = INFINITY;
    for (;;) {
      berr = bresidual<KK>(a, b, n, k, sm);
      if (berr <= tol) {
        done = true;
        break;
      }
      if (!(berr < 0.5 * prev) || iters == bt.max_it) break;
      prev = berr;
      if (nb == 32) correct<float, 32, KK>(bt, sm, n, k, ld, W, my_pos);
      else correct<float, 16, KK>(bt, sm, n, k, ld, W, my_pos);
      ++iters;
    }
    if (!done) flags |= bt.fallback ? FLAG_FELL_BACK : FLAG_NO_CONVERGENCE;
  }
  if (!done && (bt.method != RM_METHOD_F32_IR || bt.fallback)) {
    double* W = reinterpret_cast<double*>(w);
    const bool nonzero = factor_and_solve<double, 16, KK>(bt, sm, n, k, ld, W, a, b, my_pos);
    berr = bresidual<KK>(a, b, n, k, sm);
    // rustymath's `regular`: every |u_ii| > eps * n * max|a| (a NaN pivot counts as regular)
    __shared__ int irregular;
    if (threadIdx.x == 0) irregular = nonzero ? 0 : 1;
    __syncthreads();
    const double big = sm.amax_a;  // from the load of this factorization
    if (my_pos >= 0) {
      const double u = W[(int64_t)threadIdx.x * ld + my_pos];
      if (fabs(u) <= DBL_EPSILON * n * big) atomicOr(&irregular, 1);
    }
    __syncthreads();
    if (irregular) flags |= FLAG_NOT_REGULAR;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(THREADS, 2) batch_solve_kernel(Batch bt) {
  extern __shared__ __align__(16) unsigned char dsm[];
  Smem& sm = *reinterpret_cast<Smem*>(dsm);
  __shared__ int item_s;
  for (;;) {
    if (threadIdx.x == 0) item_s = bt.first + atomicAdd(bt.counter, 1);
    __syncthreads();
    const int item = item_s;
    __syncthreads();
    if (item >= bt.last) return;
    const int s = bt.sys[item], nb = bt.nb[item];
    const int n = bt.n[s], k = bt.k[s];
    const int ld = (n + 3) & ~3;
    const double* a = bt.a + bt.a_off[s];
    const double* b = bt.b + bt.b_off[s];
    double* x = bt.x + bt.x_off[s];
    unsigned char* w = bt.w + bt.w_off[s];
    if (threadIdx.x == 0) sm.anorm = -1.0;
    int my_pos = -1, iters = 0, flags = 0;
    double berr = 0.0;
    bool done = false;
    if (k <= 1) solve_system<1>(bt, sm, n, k, nb, ld, a, b, w, my_pos, iters, flags, berr, done);
    else if (k <= 2) solve_system<2>(bt, sm, n, k, nb, ld, a, b, w, my_pos, iters, flags, berr, done);
    else if (k <= 4) solve_system<4>(bt, sm, n, k, nb, ld, a, b, w, my_pos, iters, flags, berr, done);
    else solve_system<KMAX>(bt, sm, n, k, nb, ld, a, b, w, my_pos, iters, flags, berr, done);
    // x (row-major n x k) from xs, by unknown; the factors' row order and type stay for the adjoint
    for (int e = threadIdx.x; e < n * k; e += THREADS) x[e] = sm.xs[e / k][e % k];
    for (int i = threadIdx.x; i < n; i += THREADS) bt.piv[bt.p_off[s] + i] = sm.piv[i];
    if (threadIdx.x == 0) {
      bt.berr[s] = berr;
      bt.iters[s] = iters;
      bt.flags[s] = flags;
      bt.ftype[s] = (bt.method == RM_METHOD_F32_IR && (done || !bt.fallback)) ? 0 : 1;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ the adjoint
// Solves A^T y = g with the implicitly pivoted factors of bfactor (P A = L U, row piv[i] of A
// at logical position i): U^T z = g, then L^T w = z, then y[piv[i]] = w_i. Thread t holds
// v = g_t (column t, the unknowns' order) on entry and w_t on return. U^T and L^T are solved
// in blocks of NB: a warp solves the diagonal block with shuffles; then each thread updates
// its own column from the block's rows (coalesced: consecutive threads, consecutive columns).
template <typename T, int NB>
__device__ void bsolve_t(const T* W, int ld, int n, int k, Smem& sm, T (&v)[KMAX]) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int J = 0; J < n; J += NB) {  // U^T z = g: lower triangle, forward
    const int nbj = min(NB, n - J);
    if (t >= J && t < J + nbj)
#pragma unroll
      for (int c = 0; c < KMAX; ++c) sm.vsm[t - J][c] = (double)v[c];
    __syncthreads();
    if (warp < k) {  // a warp per right-hand side
      const int c = warp;
      T ucol[NB];
      T y = lane < nbj ? (T)sm.vsm[lane][c] : T(0);
#pragma unroll
      for (int q = 0; q < NB; ++q)  // U[J+q][J+lane], q <= lane
        ucol[q] = (lane < nbj && q <= lane) ? W[(int64_t)sm.piv[J + q] * ld + J + lane] : T(0);
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        if (q < nbj) {
          if (lane == q) y = y / ucol[q];
          const T zq = __shfl_sync(0xffffffffu, y, q);
          if (lane > q) y = fma(-ucol[q], zq, y);
        }
      }
      if (lane < nbj) sm.vsm[lane][c] = (double)y;
    }
    __syncthreads();
    if (t < n) {
      if (t >= J + nbj) {
        for (int q = 0; q < nbj; ++q) {
          const T u = W[(int64_t)sm.piv[J + q] * ld + t];
#pragma unroll
          for (int c = 0; c < KMAX; ++c)
            if (c < k) v[c] = fma(-u, (T)sm.vsm[q][c], v[c]);
        }
      } else if (t >= J) {
#pragma unroll
        for (int c = 0; c < KMAX; ++c) v[c] = (T)sm.vsm[t - J][c];
      }
    }
    __syncthreads();
  }
  const int last = (n - 1) / NB * NB;
  for (int J = last; J >= 0; J -= NB) {  // L^T w = z: unit upper triangle, backward
    const int nbj = min(NB, n - J);
    if (t >= J && t < J + nbj)
#pragma unroll
      for (int c = 0; c < KMAX; ++c) sm.vsm[t - J][c] = (double)v[c];
    __syncthreads();
    if (warp < k) {  // a warp per right-hand side
      const int c = warp;
      T lcol[NB];
      T y = lane < nbj ? (T)sm.vsm[lane][c] : T(0);
#pragma unroll
      for (int q = 0; q < NB; ++q)  // L[J+q][J+lane], q > lane
        lcol[q] = (lane < nbj && q > lane && q < nbj) ? W[(int64_t)sm.piv[J + q] * ld + J + lane] : T(0);
#pragma unroll
      for (int q = NB - 1; q >= 0; --q) {
        if (q < nbj) {
          const T wq = __shfl_sync(0xffffffffu, y, q);
          if (lane < q) y = fma(-lcol[q], wq, y);
        }
      }
      if (lane < nbj) sm.vsm[lane][c] = (double)y;
    }
    __syncthreads();
    if (t < n) {
      if (t < J) {
        for (int q = 0; q < nbj; ++q) {
          const T l = W[(int64_t)sm.piv[J + q] * ld + t];
#pragma unroll
          for (int c = 0; c < KMAX; ++c)
            if (c < k) v[c] = fma(-l, (T)sm.vsm[q][c], v[c]);
        }
      } else if (t < J + nbj) {
#pragma unroll
        for (int c = 0; c < KMAX; ++c) v[c] = (T)sm.vsm[t - J][c];
      }
    }
    __syncthreads();
  }
}

// sm.rs[t] = g_t - (A^T y)_t (by column t; y = sm.xs by row) for the n x n row-major a, and
// the normwise backward error of A^T y = g (NaN if a residual is NaN).
__device__ double bresidual_t(const double* __restrict__ a, const double* __restrict__ g, int n, int k, Smem& sm) {
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  double r[KMAX], gv[KMAX], yv[KMAX], asum = 0.0;
#pragma unroll
  for (int c = 0; c < KMAX; ++c) r[c] = gv[c] = yv[c] = 0.0;
  if (t < n) {
    double acc[KMAX];
#pragma unroll
    for (int c = 0; c < KMAX; ++c) acc[c] = 0.0;
#pragma unroll 4
    for (int i = 0; i < n; ++i) {
      const double av = __ldg(a + (int64_t)i * n + t);  // column t: coalesced across threads
      asum += fabs(av);
#pragma unroll
      for (int c = 0; c < KMAX; ++c)
        if (c < k) acc[c] = fma(av, sm.xs[i][c], acc[c]);
    }
#pragma unroll
    for (int c = 0; c < KMAX; ++c)
      if (c < k) {
        gv[c] = g[(int64_t)t * k + c];
        r[c] = gv[c] - acc[c];
        yv[c] = fabs(sm.xs[t][c]);
        sm.rs[t][c] = r[c];
      }
  }
  double rm[KMAX], gm[KMAX], ym[KMAX];
#pragma unroll
  for (int c = 0; c < KMAX; ++c) {
    double rv = fabs(r[c]), gvv = fabs(gv[c]), yvv = yv[c];
#pragma unroll
    for (int off = 16; off; off >>= 1) {
      const double o = __shfl_xor_sync(0xffffffffu, rv, off);
      rv = (o > rv || o != o) ? o : rv;
      gvv = fmax(gvv, __shfl_xor_sync(0xffffffffu, gvv, off));
      yvv = fmax(yvv, __shfl_xor_sync(0xffffffffu, yvv, off));
    }
    rm[c] = rv, gm[c] = gvv, ym[c] = yvv;
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) asum = fmax(asum, __shfl_xor_sync(0xffffffffu, asum, off));
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < KMAX; ++c) {
      sm.red[warp][c] = rm[c];
      sm.red[warp][KMAX + c] = gm[c];
      sm.red[warp][2 * KMAX + c] = ym[c];
    }
    sm.red[warp][3 * KMAX] = asum;
  }
  __syncthreads();
  double an = 0.0, berr = 0.0;
  bool nan = false;
  for (int w = 0; w < WARPS; ++w) an = fmax(an, sm.red[w][3 * KMAX]);
  for (int c = 0; c < k; ++c) {
    double rn = 0.0, gn = 0.0, yn = 0.0;
    for (int w = 0; w < WARPS; ++w) {
      const double o = sm.red[w][c];
      rn = (o > rn || o != o) ? o : rn;
      gn = fmax(gn, sm.red[w][KMAX + c]);
      yn = fmax(yn, sm.red[w][2 * KMAX + c]);
    }
    nan |= rn != rn;
    const double den = an * yn + gn;
    berr = fmax(berr, den > 0.0 ? rn / den : rn);
  }
  __syncthreads();
  return nan ? __longlong_as_double(0x7ff8000000000000ll) : berr;
}

struct Adjoint {
  Batch bt;             // the forward's layout, factors (w), row orders (piv) and types
  const double* g;      // dL/dx, packed like b
  double* gb;           // dL/db = A^-T g, packed like b
  double* ga;           // dL/dA = -gb x^T, packed like a (NULL: not formed)
  double* berr;         // per system: the backward error of A^T gb = g
};

template <typename T, int NB>
__device__ void adjoint_solve(const Adjoint& aj, Smem& sm, int n, int k, int ld, const T* W, const double* g,
                              bool add) {
  T v[KMAX];
#pragma unroll
  for (int c = 0; c < KMAX; ++c)
    v[c] = (threadIdx.x < n && c < k) ? (T)(add ? sm.rs[threadIdx.x][c] : g[(int64_t)threadIdx.x * k + c]) : T(0);
  bsolve_t<T, NB>(W, ld, n, k, sm, v);
  if (threadIdx.x < n) {
    const int row = sm.piv[threadIdx.x];
#pragma unroll
    for (int c = 0; c < KMAX; ++c) sm.xs[row][c] = add ? sm.xs[row][c] + (double)v[c] : (double)v[c];
  }
  __syncthreads();
}

__global__ void __launch_bounds__(THREADS, 2) batch_adjoint_kernel(Adjoint aj) {
  extern __shared__ __align__(16) unsigned char dsm[];
  Smem& sm = *reinterpret_cast<Smem*>(dsm);
  __shared__ int item_s;
  const Batch& bt = aj.bt;
  for (;;) {
    if (threadIdx.x == 0) item_s = bt.first + atomicAdd(bt.counter, 1);
    __syncthreads();
    const int item = item_s;
    __syncthreads();
    if (item >= bt.last) return;
    const int s = bt.sys[item];
    const int n = bt.n[s], k = bt.k[s];
    const int ld = (n + 3) & ~3;
    const double* a = bt.a + bt.a_off[s];
    const double* g = aj.g + bt.b_off[s];
    unsigned char* w = bt.w + bt.w_off[s];
    for (int i = threadIdx.x; i < n; i += THREADS) sm.piv[i] = bt.piv[bt.p_off[s] + i];
    __syncthreads();
    double berr = 0.0;
    const double tol = bt.tol > 0.0 ? bt.tol : (double)n * 0x1.0p-53;
    bool done = false;
    if (bt.ftype[s] == 0) {
      // float32 factors: refine in float64 against A^T
      const float* W = reinterpret_cast<const float*>(w);
      adjoint_solve<float, 32>(aj, sm, n, k, ld, W, g, false);
      double prev = INFINITY;
      for (int it = 0;; ++it) {
        berr = bresidual_t(a, g, n, k, sm);
        if (berr <= tol) {
          done = true;
          break;
        }
        if (!(berr < 0.5 * prev) || it == bt.max_it) break;
        prev = berr;
        adjoint_solve<float, 32>(aj, sm, n, k, ld, W, g, true);
      }
    }
    if (!done) {
      // float64 factors (the forward's, or made here when float32 refinement stalls)
      double* W = reinterpret_cast<double*>(w);
      if (bt.ftype[s] == 0) {
        const bool dominant = load_w_dominant<double>(a, n, W, ld, sm);
        int my_pos;
        bfactor<double, 16>(W, ld, n, sm, my_pos, dominant);
        for (int i = threadIdx.x; i < n; i += THREADS) bt.piv[bt.p_off[s] + i] = sm.piv[i];
        if (threadIdx.x == 0) bt.ftype[s] = 1;
        __syncthreads();
      }
      adjoint_solve<double, 16>(aj, sm, n, k, ld, W, g, false);
      berr = bresidual_t(a, g, n, k, sm);
    }
    // gb (packed like b) and ga = -gb x^T (packed like a)
    double* gb = aj.gb + bt.b_off[s];
    for (int e = threadIdx.x; e < n * k; e += THREADS) gb[e] = sm.xs[e / k][e % k];
    if (aj.ga) {
      const double* x = bt.x + bt.x_off[s];
      for (int e = threadIdx.x; e < n * k; e += THREADS) sm.rs[e / k][e % k] = x[e];
      __syncthreads();
      double* ga = aj.ga + bt.a_off[s];
      for (int e = threadIdx.x; e < n * n; e += THREADS) {
        const int i = e / n, j = e - i * n;
        double acc = 0.0;
        for (int c = 0; c < k; ++c) acc = fma(sm.xs[i][c], sm.rs[j][c], acc);
        ga[e] = -acc;
      }
    }
    if (threadIdx.x == 0) aj.berr[s] = berr;
    __syncthreads();
  }
}

// Stacked::lu (src/linalg/stacked.rs:174-187) in one launch: matrix blockIdx.x of a stack of
// n x n row-major matrices (n <= NMAX, back to back) factored in float64 by bfactor in its own
// slice of wbuf (w_stride bytes apart), then written in rustymath's layout: factors column-
// major, (L U)(i, j) = W[piv[i]][j] at factors[j*n + i] (coalesced over i), perm[i] = piv[i];
// regular[m] (when not NULL) as LuWork::regular (factor.rs:221-226): every |u_ii| > eps n
// max|a|, max ignoring NaN, a NaN pivot counting as regular.
__global__ void __launch_bounds__(THREADS) batch_factor_kernel(const double* __restrict__ a, int n,
                                                               unsigned char* wbuf, int64_t w_stride,
                                                               double* __restrict__ factors, int64_t* __restrict__ perm,
                                                               int32_t* regular) {
  extern __shared__ __align__(16) unsigned char dsm[];
  Smem& sm = *reinterpret_cast<Smem*>(dsm);
  __shared__ int irregular;
  const int64_t m = blockIdx.x;
  const int ld = (n + 3) & ~3;
  double* W = reinterpret_cast<double*>(wbuf + m * w_stride);
  const double* am = a + m * n * n;
  const bool dominant = load_w_dominant<double>(am, n, W, ld, sm);
  if (threadIdx.x == 0) {
    sm.zero_pivot = 0;
    irregular = 0;
  }
  __syncthreads();
  int my_pos = -1;
  bfactor<double, 16>(W, ld, n, sm, my_pos, dominant);
  double* fm = factors + m * n * n;
  for (int e = threadIdx.x; e < n * n; e += THREADS) {
    const int j = e / n, i = e - j * n;
    fm[e] = W[(int64_t)sm.piv[i] * ld + j];
  }
  for (int i = threadIdx.x; i < n; i += THREADS) perm[m * n + i] = sm.piv[i];
  if (regular) {
    const double big = sm.amax_a;
    if (my_pos >= 0 && fabs(W[(int64_t)threadIdx.x * ld + my_pos]) <= DBL_EPSILON * n * big) atomicOr(&irregular, 1);
    __syncthreads();
    if (threadIdx.x == 0) regular[m] = irregular ? 0 : 1;
  }
}

}  // namespace bt

// ------------------------------------------------------------------ the plan (host)
struct BatchPlan {
  int64_t count = 0;
  std::vector<int> n, k, order, nb_item;
  std::vector<int64_t> a_off, b_off, x_off, w_off;
  rm_solve_options opts{};
  int nb_bucket[5] = {16, 16, 32, 32, 32};  // panel width per size bucket (tuned)
  // device
  int *d_sys = nullptr, *d_nb = nullptr, *d_n = nullptr, *d_k = nullptr, *d_iters = nullptr, *d_flags = nullptr,
      *d_counter = nullptr;
  int64_t *d_aoff = nullptr, *d_boff = nullptr, *d_xoff = nullptr, *d_woff = nullptr, *d_poff = nullptr;
  int *d_piv = nullptr, *d_ftype = nullptr;
  double* d_berr = nullptr;
  double* d_adj_berr = nullptr;
  unsigned char* d_w = nullptr;
  size_t w_bytes = 0;
  int grid = 0;
  cudaStream_t stream = nullptr;  // the plan's own stream, for graph capture
  cudaGraphExec_t graph = nullptr;
  const void* g_a = nullptr;
  const void* g_b = nullptr;
  const void* g_x = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
};

static int bucket_of(int n) { return n <= 32 ? 0 : n <= 64 ? 1 : n <= 128 ? 2 : n <= 192 ? 3 : 4; }

static void free_plan(BatchPlan* p) {
  if (!p) return;
  if (p->graph) cudaGraphExecDestroy(p->graph);
  for (void* q : {(void*)p->d_sys, (void*)p->d_nb, (void*)p->d_n, (void*)p->d_k, (void*)p->d_iters,
                  (void*)p->d_flags, (void*)p->d_counter, (void*)p->d_aoff, (void*)p->d_boff, (void*)p->d_xoff,
                  (void*)p->d_woff, (void*)p->d_berr, (void*)p->d_w, (void*)p->d_poff, (void*)p->d_piv,
                  (void*)p->d_ftype, (void*)p->d_adj_berr})
    if (q) cudaFree(q);
  if (p->ev_in) cudaEventDestroy(p->ev_in);
  if (p->ev_out) cudaEventDestroy(p->ev_out);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

template <typename V>
static int upload(V** dst, const std::vector<V>& src) {
  RM_CUDA_TRY(cudaMalloc(dst, std::max<size_t>(src.size(), 1) * sizeof(V)));
  if (!src.empty()) RM_CUDA_TRY(cudaMemcpy(*dst, src.data(), src.size() * sizeof(V), cudaMemcpyHostToDevice));
  return RM_OK;
}

static int plan_build(BatchPlan* p) {
  const int64_t cnt = p->count;
  p->order.resize(cnt);
  std::iota(p->order.begin(), p->order.end(), 0);
  // largest first: the long systems start early and the short ones fill in at the end
  std::stable_sort(p->order.begin(), p->order.end(), [&](int x, int y) { return p->n[x] > p->n[y]; });
  p->w_off.assign(cnt, 0);
  size_t off = 0;
  for (int64_t i = 0; i < cnt; ++i) {
    const int n = p->n[i];
    p->w_off[i] = (int64_t)off;
    off += ((size_t)n * ((n + 3) & ~3) * 8 + 255) / 256 * 256;
  }
  p->w_bytes = std::max<size_t>(off, 256);
  p->nb_item.resize(cnt);
  for (int64_t i = 0; i < cnt; ++i) p->nb_item[i] = p->nb_bucket[bucket_of(p->n[p->order[i]])];
  RM_TRY(upload(&p->d_sys, p->order));
  RM_TRY(upload(&p->d_nb, p->nb_item));
  RM_TRY(upload(&p->d_n, p->n));
  RM_TRY(upload(&p->d_k, p->k));
  RM_TRY(upload(&p->d_aoff, p->a_off));
  RM_TRY(upload(&p->d_boff, p->b_off));
  RM_TRY(upload(&p->d_xoff, p->x_off));
  RM_TRY(upload(&p->d_woff, p->w_off));
  std::vector<int64_t> p_off(cnt);
  int64_t poff = 0;
  for (int64_t i = 0; i < cnt; ++i) p_off[i] = poff, poff += p->n[i];
  RM_TRY(upload(&p->d_poff, p_off));
  RM_CUDA_TRY(cudaMalloc(&p->d_piv, std::max<int64_t>(poff, 1) * sizeof(int)));
  RM_CUDA_TRY(cudaMalloc(&p->d_ftype, std::max<int64_t>(cnt, 1) * sizeof(int)));
  RM_CUDA_TRY(cudaMalloc(&p->d_adj_berr, std::max<int64_t>(cnt, 1) * sizeof(double)));
  RM_CUDA_TRY(cudaMalloc(&p->d_berr, std::max<int64_t>(cnt, 1) * sizeof(double)));
  RM_CUDA_TRY(cudaMalloc(&p->d_iters, std::max<int64_t>(cnt, 1) * sizeof(int)));
  RM_CUDA_TRY(cudaMalloc(&p->d_flags, std::max<int64_t>(cnt, 1) * sizeof(int)));
  RM_CUDA_TRY(cudaMalloc(&p->d_counter, sizeof(int)));
  RM_CUDA_TRY(cudaMalloc(&p->d_w, p->w_bytes));
  RM_TRY(smem_attribute(bt::batch_solve_kernel, sizeof(bt::Smem)));
  RM_TRY(smem_attribute(bt::batch_adjoint_kernel, sizeof(bt::Smem)));
  int per_sm = 0;
  RM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bt::batch_solve_kernel, bt::THREADS,
                                                            sizeof(bt::Smem)));
  p->grid = std::max(1, per_sm) * device_sm_count();
  RM_CUDA_TRY(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  RM_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming));
  RM_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_out, cudaEventDisableTiming));
  return RM_OK;
}

static bt::Batch batch_args(BatchPlan* p, const double* a, const double* b, double* x, int first, int last) {
  bt::Batch q;
  q.first = first, q.last = last;
  q.sys = p->d_sys, q.nb = p->d_nb, q.n = p->d_n, q.k = p->d_k;
  q.a_off = p->d_aoff, q.b_off = p->d_boff, q.x_off = p->d_xoff, q.w_off = p->d_woff;
  q.a = a, q.b = b, q.x = x, q.w = p->d_w;
  q.method = p->opts.method;
  q.max_it = p->opts.max_iterations > 0 ? p->opts.max_iterations : 30;
  q.tol = p->opts.tolerance;
  q.fallback = p->opts.fallback;
  q.berr = p->d_berr, q.iters = p->d_iters, q.flags = p->d_flags, q.counter = p->d_counter;
  q.piv = p->d_piv, q.p_off = p->d_poff, q.ftype = p->d_ftype;
  return q;
}

// the counter reset and the one persistent launch, over items [first, last); a launch being
// captured into the plan's graph is counted when the graph runs, not here
static int launch_batch(BatchPlan* p, const double* a, const double* b, double* x, int first, int last,
                        cudaStream_t s, bool captured = false) {
  RM_CUDA_TRY(cudaMemsetAsync(p->d_counter, 0, sizeof(int), s));
  const int items = last - first;
  const int grid = std::min(p->grid, std::max(items, 1));
  bt::batch_solve_kernel<<<grid, bt::THREADS, sizeof(bt::Smem), s>>>(batch_args(p, a, b, x, first, last));
  if (!captured) note_launch();
  RM_CUDA_TRY(cudaGetLastError());
  return RM_OK;
}

int batch_plan_create(int64_t count, const int64_t* n, const int64_t* k, const int64_t* a_off, const int64_t* b_off,
                      const int64_t* x_off, const rm_solve_options* opts, BatchPlan** out) {
  if (!out || count < 0 || count > INT_MAX || (count > 0 && (!n || !k || !a_off || !b_off || !x_off)))
    return RM_BAD_ARG;
  for (int64_t i = 0; i < count; ++i)
    if (n[i] < 0 || n[i] > bt::NMAX || k[i] < 0 || k[i] > bt::KMAX || a_off[i] < 0 || b_off[i] < 0 || x_off[i] < 0) {
      set_last_message("batched systems take 0 <= n <= 256 and 0 <= k <= 8");
      return RM_BAD_ARG;
    }
  BatchPlan* p = new BatchPlan();
  p->count = count;
  p->n.assign(n, n + count);
  p->k.assign(k, k + count);
  p->a_off.assign(a_off, a_off + count);
  p->b_off.assign(b_off, b_off + count);
  p->x_off.assign(x_off, x_off + count);
  if (opts) p->opts = *opts;
  else p->opts.method = RM_METHOD_F32_IR, p->opts.fallback = 1;
  const int st = plan_build(p);
  if (st != RM_OK) {
    free_plan(p);
    return st;
  }
  *out = p;
  return RM_OK;
}

void batch_plan_destroy(BatchPlan* p) { free_plan(p); }

// One persistent launch over every system, replayed from a CUDA graph captured on the plan's
// own stream (re-captured when the data pointers change); ordered after prior work on s and
// before later work on s.
int batch_plan_execute(BatchPlan* p, const double* a, const double* b, double* x, cudaStream_t s) {
  if (!p) return RM_BAD_ARG;
  if (p->count == 0) return RM_OK;
  if (!p->graph || p->g_a != a || p->g_b != b || p->g_x != x) {
    if (p->graph) {
      cudaGraphExecDestroy(p->graph);
      p->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    RM_CUDA_TRY(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
    const int st = launch_batch(p, a, b, x, 0, (int)p->count, p->stream, true);
    const cudaError_t e = cudaStreamEndCapture(p->stream, &g);
    if (st != RM_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    RM_CUDA_TRY(e);
    const cudaError_t ie = cudaGraphInstantiate(&p->graph, g, 0);
    cudaGraphDestroy(g);
    RM_CUDA_TRY(ie);
    p->g_a = a, p->g_b = b, p->g_x = x;
  }
  RM_CUDA_TRY(cudaEventRecord(p->ev_in, s));
  RM_CUDA_TRY(cudaStreamWaitEvent(p->stream, p->ev_in, 0));
  RM_CUDA_TRY(cudaGraphLaunch(p->graph, p->stream));
  note_launch();  // the graph's kernel
  RM_CUDA_TRY(cudaEventRecord(p->ev_out, p->stream));
  RM_CUDA_TRY(cudaStreamWaitEvent(s, p->ev_out, 0));
  return RM_OK;
}

// Picks the panel width of each size bucket: each candidate (16, 32) runs the bucket's own
// systems (a contiguous range of the size-sorted order) twice, timed by CUDA events; the
// faster stays. The results are the solves of those systems (x is written).
int batch_plan_tune(BatchPlan* p, const double* a, const double* b, double* x, cudaStream_t s) {
  if (!p) return RM_BAD_ARG;
  const int cnt = (int)p->count;
  cudaEvent_t e0, e1;
  RM_CUDA_TRY(cudaEventCreate(&e0));
  RM_CUDA_TRY(cudaEventCreate(&e1));
  int status = RM_OK;
  for (int bk = 0; bk < 5 && status == RM_OK; ++bk) {
    int first = cnt, last = 0;
    for (int i = 0; i < cnt; ++i)
      if (bucket_of(p->n[p->order[i]]) == bk) first = std::min(first, i), last = std::max(last, i + 1);
    if (first >= last) continue;
    float best = INFINITY;
    int best_nb = p->nb_bucket[bk];
    for (int cand : {16, 32}) {
      for (int i = first; i < last; ++i) p->nb_item[i] = cand;
      if (cudaMemcpyAsync(p->d_nb + first, p->nb_item.data() + first, (last - first) * sizeof(int),
                          cudaMemcpyHostToDevice, s) != cudaSuccess) {
        status = RM_CUDA_ERROR;
        break;
      }
      float t = 0.0f;
      for (int rep = 0; rep < 2 && status == RM_OK; ++rep) {
        cudaEventRecord(e0, s);
        status = launch_batch(p, a, b, x, first, last, s);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) status = RM_CUDA_ERROR;
        cudaEventElapsedTime(&t, e0, e1);
      }
      if (t < best) best = t, best_nb = cand;
    }
    p->nb_bucket[bk] = best_nb;
    for (int i = first; i < last; ++i) p->nb_item[i] = best_nb;
    if (cudaMemcpyAsync(p->d_nb + first, p->nb_item.data() + first, (last - first) * sizeof(int),
                        cudaMemcpyHostToDevice, s) != cudaSuccess)
      status = RM_CUDA_ERROR;
  }
  cudaStreamSynchronize(s);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return status;  // the kernel reads the widths from d_nb, so a captured graph stays valid
}

// dL/db = A^-T g and dL/dA = -(dL/db) x^T for every system, from the factors the last
// execute left in the plan (the same a and x); one persistent launch on the plan's stream,
// ordered after prior work on s and before later work on s.
int batch_plan_adjoint(BatchPlan* p, const double* a, const double* x, const double* g, double* gb, double* ga,
                       cudaStream_t s) {
  if (!p) return RM_BAD_ARG;
  if (p->count == 0) return RM_OK;
  RM_CUDA_TRY(cudaEventRecord(p->ev_in, s));
  RM_CUDA_TRY(cudaStreamWaitEvent(p->stream, p->ev_in, 0));
  RM_CUDA_TRY(cudaMemsetAsync(p->d_counter, 0, sizeof(int), p->stream));
  bt::Adjoint aj;
  aj.bt = batch_args(p, a, nullptr, const_cast<double*>(x), 0, (int)p->count);
  aj.g = g, aj.gb = gb, aj.ga = ga, aj.berr = p->d_adj_berr;
  const int grid = std::min<int64_t>(p->grid, p->count);
  bt::batch_adjoint_kernel<<<grid, bt::THREADS, sizeof(bt::Smem), p->stream>>>(aj);
  RM_LAUNCHED();
  RM_CUDA_TRY(cudaEventRecord(p->ev_out, p->stream));
  RM_CUDA_TRY(cudaStreamWaitEvent(s, p->ev_out, 0));
  return RM_OK;
}

int batch_plan_adjoint_results(BatchPlan* p, double* berr, double* max_berr) {
  if (!p) return RM_BAD_ARG;
  std::vector<double> be(p->count);
  RM_CUDA_TRY(cudaStreamSynchronize(p->stream));
  if (p->count) RM_CUDA_TRY(cudaMemcpy(be.data(), p->d_adj_berr, p->count * sizeof(double), cudaMemcpyDeviceToHost));
  if (berr) std::copy(be.begin(), be.end(), berr);
  if (max_berr) {
    *max_berr = 0.0;
    for (double v : be) *max_berr = (v != v || *max_berr != *max_berr) ? NAN : std::max(*max_berr, v);
  }
  return RM_OK;
}

int batch_plan_results(BatchPlan* p, double* berr, int32_t* iters, int32_t* flags, rm_batch_report* summary) {
  if (!p) return RM_BAD_ARG;
  const int64_t cnt = p->count;
  std::vector<double> be(cnt);
  std::vector<int> it(cnt), fl(cnt);
  RM_CUDA_TRY(cudaStreamSynchronize(p->stream));
  if (cnt) {
    RM_CUDA_TRY(cudaMemcpy(be.data(), p->d_berr, cnt * sizeof(double), cudaMemcpyDeviceToHost));
    RM_CUDA_TRY(cudaMemcpy(it.data(), p->d_iters, cnt * sizeof(int), cudaMemcpyDeviceToHost));
    RM_CUDA_TRY(cudaMemcpy(fl.data(), p->d_flags, cnt * sizeof(int), cudaMemcpyDeviceToHost));
  }
  if (berr) std::copy(be.begin(), be.end(), berr);
  if (iters) std::copy(it.begin(), it.end(), iters);
  if (flags) std::copy(fl.begin(), fl.end(), flags);
  if (summary) {
    summary->max_backward_error = 0.0;
    summary->fell_back = summary->not_regular = summary->no_convergence = 0;
    summary->max_iterations = 0;
    for (int64_t i = 0; i < cnt; ++i) {
      summary->max_backward_error = std::max(summary->max_backward_error, be[i]);
      if (be[i] != be[i]) summary->max_backward_error = be[i];
      summary->fell_back += (fl[i] & bt::FLAG_FELL_BACK) != 0;
      summary->not_regular += (fl[i] & bt::FLAG_NOT_REGULAR) != 0;
      summary->no_convergence += (fl[i] & bt::FLAG_NO_CONVERGENCE) != 0;
      summary->max_iterations = std::max(summary->max_iterations, it[i]);
    }
  }
  return RM_OK;
}

}  // namespace rm

// ------------------------------------------------------------------ C ABI
struct rm_batch_plan {
  rm::BatchPlan* p;
};

extern "C" {

int rm_batch_plan_create(int64_t count, const int64_t* h_n, const int64_t* h_k, const int64_t* h_a_off,
                         const int64_t* h_b_off, const int64_t* h_x_off, const rm_solve_options* opts,
                         rm_batch_plan** plan) {
  if (!plan) return RM_BAD_ARG;
  *plan = nullptr;
  RM_TRY(rm::check_device());
  rm::BatchPlan* p = nullptr;
  RM_TRY(rm::batch_plan_create(count, h_n, h_k, h_a_off, h_b_off, h_x_off, opts, &p));
  *plan = new rm_batch_plan{p};
  return RM_OK;
}

int rm_batch_plan_tune(rm_batch_plan* plan, const double* d_a, const double* d_b, double* d_x, void* stream) {
  if (!plan || !d_a || !d_b || !d_x) return RM_BAD_ARG;
  RM_TRY(rm::batch_plan_tune(plan->p, d_a, d_b, d_x, reinterpret_cast<cudaStream_t>(stream)));
  return rm::take_device_status(reinterpret_cast<cudaStream_t>(stream));
}

int rm_batch_plan_execute(rm_batch_plan* plan, const double* d_a, const double* d_b, double* d_x, void* stream) {
  if (!plan || (plan->p->count > 0 && (!d_a || !d_b || !d_x))) return RM_BAD_ARG;
  return rm::batch_plan_execute(plan->p, d_a, d_b, d_x, reinterpret_cast<cudaStream_t>(stream));
}

int rm_batch_plan_results(rm_batch_plan* plan, double* h_berr, int32_t* h_iters, int32_t* h_flags,
                          rm_batch_report* summary) {
  if (!plan) return RM_BAD_ARG;
  return rm::batch_plan_results(plan->p, h_berr, h_iters, h_flags, summary);
}

int rm_batch_plan_adjoint(rm_batch_plan* plan, const double* d_a, const double* d_x, const double* d_gx,
                          double* d_gb, double* d_ga, void* stream) {
  if (!plan || (plan->p->count > 0 && (!d_a || !d_x || !d_gx || !d_gb))) return RM_BAD_ARG;
  return rm::batch_plan_adjoint(plan->p, d_a, d_x, d_gx, d_gb, d_ga, reinterpret_cast<cudaStream_t>(stream));
}

int rm_batch_plan_adjoint_results(rm_batch_plan* plan, double* h_berr, double* h_max_berr) {
  if (!plan) return RM_BAD_ARG;
  RM_TRY(rm::batch_plan_adjoint_results(plan->p, h_berr, h_max_berr));
  return rm::take_device_status(nullptr);
}

int rm_batch_plan_panel_width(const rm_batch_plan* plan, int bucket) {
  return plan && bucket >= 0 && bucket < 5 ? plan->p->nb_bucket[bucket] : 0;
}

int rm_batch_plan_destroy(rm_batch_plan* plan) {
  if (!plan) return RM_OK;
  rm::batch_plan_destroy(plan->p);
  delete plan;
  return RM_OK;
}

int rm_dlu_factor_batched(int64_t count, int64_t n, const double* d_a, double* d_factors, int64_t* d_perm,
                          int32_t* d_regular, void* stream) {
  if (count < 0 || n < 0 || n > rm::bt::NMAX || (count > 0 && n > 0 && (!d_a || !d_factors || !d_perm)))
    return RM_BAD_ARG;
  if (count == 0 || n == 0) return RM_OK;
  RM_TRY(rm::check_device());
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int64_t ld = (n + 3) & ~3;
  const int64_t stride = (n * ld * 8 + 255) / 256 * 256;
  RM_TRY(rm::smem_attribute(rm::bt::batch_factor_kernel, sizeof(rm::bt::Smem)));
  for (int64_t first = 0; first < count; first += 65536) {
    const int64_t c = std::min<int64_t>(count - first, 65536);
    void* w = nullptr;
    RM_TRY(rm::scratch_alloc(&w, (size_t)(c * stride), s));
    rm::bt::batch_factor_kernel<<<(unsigned)c, rm::bt::THREADS, sizeof(rm::bt::Smem), s>>>(
        d_a + first * n * n, (int)n, static_cast<unsigned char*>(w), stride, d_factors + first * n * n,
        d_perm + first * n, d_regular ? d_regular + first : nullptr);
    const cudaError_t e = cudaGetLastError();
    rm::scratch_free(w, s);
    rm::note_launch();
    if (e != cudaSuccess) {
      rm::set_last_error(e, "batch_factor_kernel", __FILE__, __LINE__);
      return RM_CUDA_ERROR;
    }
  }
  return RM_OK;
}

int rm_dsolve_batched(int64_t count, const int64_t* h_n, const int64_t* h_k, const int64_t* h_a_off,
                      const int64_t* h_b_off, const int64_t* h_x_off, const double* d_a, const double* d_b,
                      double* d_x, const rm_solve_options* opts, rm_batch_report* report, void* stream) {
  rm_batch_plan* plan = nullptr;
  RM_TRY(rm_batch_plan_create(count, h_n, h_k, h_a_off, h_b_off, h_x_off, opts, &plan));
  int st = rm_batch_plan_execute(plan, d_a, d_b, d_x, stream);
  if (st == RM_OK) st = rm::take_device_status(reinterpret_cast<cudaStream_t>(stream));
  if (st == RM_OK) st = rm_batch_plan_results(plan, nullptr, nullptr, nullptr, report);
  rm_batch_plan_destroy(plan);
  if (st == RM_OK && report && report->no_convergence > 0) {
    rm::set_last_message("refinement stalled on some systems and fallback was off");
    return RM_NO_CONVERGENCE;
  }
  return st;
}

}  // extern "C"
