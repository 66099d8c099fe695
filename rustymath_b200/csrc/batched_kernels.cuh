// The batched kernels, built once per system-size class: batched.cu includes this with
// RM_BT_NS = bt and RM_BT_NMAX = 256 (a CTA of 256 threads, two per SM), batched_small.cu with
// RM_BT_NS = bt64 and RM_BT_NMAX = 64 (a CTA of 64 threads, eight per SM, so that small systems
// keep every thread busy). A thread owns a row, so a CTA takes systems of order up to
// RM_BT_NMAX.
#include <algorithm>
#include <cfloat>
#include <climits>

#include "rm_internal.h"
#include "batched_args.cuh"

#ifndef RM_BT_NS
#error "define RM_BT_NS, RM_BT_NMAX and RM_BT_MIN_BLOCKS before including batched_kernels.cuh"
#endif

namespace rm {
namespace RM_BT_NS {

constexpr int NMAX = RM_BT_NMAX;  // rows of a system: a thread per row
static_assert(NMAX == MAX_N, "the build's size class");
constexpr int THREADS = NMAX;
constexpr int WARPS = THREADS / 32;
constexpr int KMAX = 8;    // right-hand sides of a system
constexpr int SLOT_BYTES = 144;
constexpr int UBT_BYTES = NMAX * 144;  // U12 transposed (NMAX rows of 144 bytes), or row segments

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
  T* Lsm = reinterpret_cast<T*>(sm.xs);  // NMAX x LDU: row r's panel multipliers (xs..rs are free here)
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

// f(c) for the right-hand sides c = warp, warp + WARPS, ... below k: a warp per right-hand side,
// the whole set in one pass when there are as many warps as right-hand sides can be.
template <typename F>
__device__ __forceinline__ void for_each_rhs(int warp, int k, F&& f) {
  if constexpr (WARPS >= KMAX) {
    if (warp < k) f(warp);
  } else {
    for (int c = warp; c < k; c += WARPS) f(c);
  }
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
    if (warp < k) {  // a warp per right-hand side (c = warp, warp + WARPS, ...), lane = row of the block
      load_row<T, NB>(W + (int64_t)(lane < nbj ? sm.piv[J + lane] : 0) * ld + J, nbj, lv);
      for_each_rhs(warp, k, [&](int c) {
        T y = lane < nbj ? (T)sm.vsm[lane][c] : T(0);
#pragma unroll
        for (int q = 0; q < NB; ++q) {
          if (q < nbj) {
            const T yq = __shfl_sync(0xffffffffu, y, q);
            if (lane > q && lane < nbj) y = fma(-lv[q], yq, y);
          }
        }
        if (lane < nbj) sm.vsm[lane][c] = (double)y;
      });
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
      load_row<T, NB>(W + (int64_t)(lane < nbj ? sm.piv[J + lane] : 0) * ld + J, nbj, uv);
      for_each_rhs(warp, k, [&](int c) {
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
      });
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

using Batch = BatchArgs;

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
__device__ void solve_system(Batch& bt, Smem& sm, int method, int n, int k, int nb, int ld, const double* a,
                             const double* b, unsigned char* w, int& my_pos, int& iters, int& flags, double& berr,
                             bool& done) {
  if (method == RM_METHOD_F32_IR) {
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
  if (!done && (method != RM_METHOD_F32_IR || bt.fallback)) {
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

__global__ void __launch_bounds__(THREADS, RM_BT_MIN_BLOCKS) batch_solve_kernel(Batch bt) {
  extern __shared__ __align__(16) unsigned char dsm[];
  Smem& sm = *reinterpret_cast<Smem*>(dsm);
  __shared__ int item_s;
  for (;;) {
    if (threadIdx.x == 0) item_s = bt.first + atomicAdd(bt.counter, 1);
    __syncthreads();
    const int item = item_s;
    __syncthreads();
    if (item >= bt.last) return;
    const int s = bt.sys[item], code = bt.nb[item], nb = code & 0xff;
    const int method = (code & kItemF64) ? RM_METHOD_PLAIN_F64 : bt.method;
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
    if (k <= 1) solve_system<1>(bt, sm, method, n, k, nb, ld, a, b, w, my_pos, iters, flags, berr, done);
    else if (k <= 2) solve_system<2>(bt, sm, method, n, k, nb, ld, a, b, w, my_pos, iters, flags, berr, done);
    else if (k <= 4) solve_system<4>(bt, sm, method, n, k, nb, ld, a, b, w, my_pos, iters, flags, berr, done);
    else solve_system<KMAX>(bt, sm, method, n, k, nb, ld, a, b, w, my_pos, iters, flags, berr, done);
    // x (row-major n x k) from xs, by unknown; the factors' row order and type stay for the adjoint
    for (int e = threadIdx.x; e < n * k; e += THREADS) x[e] = sm.xs[e / k][e % k];
    for (int i = threadIdx.x; i < n; i += THREADS) bt.piv[bt.p_off[s] + i] = sm.piv[i];
    if (threadIdx.x == 0) {
      bt.berr[s] = berr;
      bt.iters[s] = iters;
      bt.flags[s] = flags;
      bt.ftype[s] = (method == RM_METHOD_F32_IR && (done || !bt.fallback)) ? 0 : 1;
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
      T ucol[NB];
#pragma unroll
      for (int q = 0; q < NB; ++q)  // U[J+q][J+lane], q <= lane
        ucol[q] = (lane < nbj && q <= lane) ? W[(int64_t)sm.piv[J + q] * ld + J + lane] : T(0);
      for_each_rhs(warp, k, [&](int c) {
        T y = lane < nbj ? (T)sm.vsm[lane][c] : T(0);
#pragma unroll
        for (int q = 0; q < NB; ++q) {
          if (q < nbj) {
            if (lane == q) y = y / ucol[q];
            const T zq = __shfl_sync(0xffffffffu, y, q);
            if (lane > q) y = fma(-ucol[q], zq, y);
          }
        }
        if (lane < nbj) sm.vsm[lane][c] = (double)y;
      });
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
      T lcol[NB];
#pragma unroll
      for (int q = 0; q < NB; ++q)  // L[J+q][J+lane], q > lane
        lcol[q] = (lane < nbj && q > lane && q < nbj) ? W[(int64_t)sm.piv[J + q] * ld + J + lane] : T(0);
      for_each_rhs(warp, k, [&](int c) {
        T y = lane < nbj ? (T)sm.vsm[lane][c] : T(0);
#pragma unroll
        for (int q = NB - 1; q >= 0; --q) {
          if (q < nbj) {
            const T wq = __shfl_sync(0xffffffffu, y, q);
            if (lane < q) y = fma(-lcol[q], wq, y);
          }
        }
        if (lane < nbj) sm.vsm[lane][c] = (double)y;
      });
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

using Adjoint = AdjointArgs;

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

__global__ void __launch_bounds__(THREADS, RM_BT_MIN_BLOCKS) batch_adjoint_kernel(Adjoint aj) {
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

// ------------------------------------------------------------------ launches (host)
int prepare(int* per_sm) {
  RM_TRY(smem_attribute(batch_solve_kernel, sizeof(Smem)));
  RM_TRY(smem_attribute(batch_adjoint_kernel, sizeof(Smem)));
  RM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, batch_solve_kernel, THREADS, sizeof(Smem)));
  return RM_OK;
}

void launch_solve(const BatchArgs& q, int grid, cudaStream_t s) {
  batch_solve_kernel<<<grid, THREADS, sizeof(Smem), s>>>(q);
}

void launch_adjoint(const AdjointArgs& q, int grid, cudaStream_t s) {
  batch_adjoint_kernel<<<grid, THREADS, sizeof(Smem), s>>>(q);
}

int launch_factor(const double* a, int n, unsigned char* wbuf, int64_t w_stride, double* factors, int64_t* perm,
                  int32_t* regular, unsigned count, cudaStream_t s) {
  RM_TRY(smem_attribute(batch_factor_kernel, sizeof(Smem)));
  batch_factor_kernel<<<count, THREADS, sizeof(Smem), s>>>(a, n, wbuf, w_stride, factors, perm, regular);
  return RM_OK;
}

}  // namespace RM_BT_NS
}  // namespace rm
