// LU with partial pivoting on the B200: the plain float64 path.
//
// Replaces lu_factor / lu_panel (core/src/linalg/factor.rs:580-630). The reference halves
// columns recursively down to 16-column leaves on a column-major copy. Here the working
// copy stays row-major (row swaps are contiguous and coalesced) and the factorization is
// right-looking in blocks of kOuter columns, so the trailing update is a rank-128 FP64
// product (compute-bound on DMMA) instead of the rank-16..n/2 products of the recursion:
//
//   for each block of kOuter columns at J0:
//     for each 32-column leaf at j0 inside it:
//       panel_kernel     : pivot search, row swap, scale and rank-1 updates of the leaf,
//                          rows spread over a cluster of up to 16 CTAs' shared memory
//       swap_trsm_kernel : the leaf's swaps on the block's other columns, and
//                          U = L^-1 A for the leaf's rows of the block's later columns
//       dgemm            : the block's later columns below the leaf -= L21 U12
//     swap_trsm_kernel   : the block's swaps on every column outside it, and perm
//     invert_unit_lower_f64 : L11^-1 of the block's diagonal (4 CTAs, a 32-column block each)
//     dgemm              : U12 = L11^-1 A12 (in place), then A22 -= L21 U12: the next
//                          block's 128 columns first; for n >= 1024 the rest runs on a side
//                          stream while the next block's leaves factor (look-ahead)
//
// The pivot rule is the reference's `largest` (factor.rs:476): the first row of greatest
// magnitude, NaN never chosen, the diagonal itself when every candidate is NaN; a zero
// pivot leaves its column unreduced (factor.rs:606); `divide` multiplies by the
// reciprocal unless the pivot is subnormal (factor.rs:506-508).
#include <climits>

#include <mutex>
#include <vector>

#include "rm_internal.h"

namespace rm {

constexpr int kLeaf = 32;         // columns of a panel leaf
constexpr int kOuter = 128;       // columns of an outer block (the trailing update's rank)
constexpr int kPanelThreads = 256;
constexpr int kPanelWarps = kPanelThreads / 32;
constexpr int kPanelStride = kLeaf + 1;  // shared row stride (odd: conflict-free column reads)
constexpr int kMaxCluster = 16;
constexpr int kPanelSmemBudget = 200 * 1024;

// ------------------------------------------------------------------ cluster helpers
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_nctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t map_rank(const void* p, uint32_t rank) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
  return a;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void st_cluster(uint32_t a, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void st_cluster(uint32_t a, float v) {
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ void st_cluster(uint32_t a, int v) {
  asm volatile("st.shared::cluster.s32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ double ld_cluster_f64(uint32_t a) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ float ld_cluster_f32(uint32_t a) {
  float v;
  asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(a) : "memory");
  return v;
}
template <typename T>
__device__ __forceinline__ T ld_cluster(uint32_t a) {
  if constexpr (sizeof(T) == 8) return ld_cluster_f64(a);
  else return ld_cluster_f32(a);
}

template <typename T>
__device__ __forceinline__ T min_normal() {
  if constexpr (sizeof(T) == 8) return 2.2250738585072014e-308;
  else return 1.17549435e-38f;
}

// Keeps the larger magnitude, and on equal magnitudes the lower row (the first index).
template <typename T>
__device__ __forceinline__ void argmax_merge(T& v, int& i, T ov, int oi) {
  if (ov > v || (ov == v && oi < i)) {
    v = ov;
    i = oi;
  }
}
template <typename T>
__device__ __forceinline__ void warp_argmax(T& v, int& i) {
#pragma unroll
  for (int off = 16; off; off >>= 1) {
    const T ov = __shfl_xor_sync(0xffffffffu, v, off);
    const int oi = __shfl_xor_sync(0xffffffffu, i, off);
    argmax_merge(v, i, ov, oi);
  }
}

template <typename T>
struct PanelShared {
  T red_v[kPanelWarps];
  int red_i[kPanelWarps];
  T slot_v[2][kMaxCluster];
  int slot_i[2][kMaxCluster];
  T cand[2][kLeaf];
  T diag[2][kLeaf];
  T piv[kLeaf];
  T old[kLeaf];
  int p;
};

// One leaf of up to kLeaf columns: rows j0..n-1, columns j0..j0+jb-1 of W. CTA `rank` of
// the cluster holds rows [rank*rpc, (rank+1)*rpc) of the leaf (in shared memory when
// IN_SMEM, else read and written in place); thread t owns the rows t, t+256, ...
template <typename T, bool IN_SMEM>
__global__ void __launch_bounds__(kPanelThreads)
    panel_kernel(T* __restrict__ w, int64_t ldw, int n, int j0, int jb, int rpc, int64_t* __restrict__ ipiv) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int P = (int)cluster_nctarank();
  const int rank = (int)cluster_ctarank();
  const int M = n - j0;
  const int base = rank * rpc;
  const int cnt = max(0, min(rpc, M - base));
  T* S = reinterpret_cast<T*>(smem);
  const size_t rows_bytes = IN_SMEM ? ((size_t)rpc * kPanelStride * sizeof(T) + 15) / 16 * 16 : 0;
  PanelShared<T>* sh = reinterpret_cast<PanelShared<T>*>(smem + rows_bytes);
  T* g0 = w + (int64_t)(j0 + base) * ldw + j0;  // this CTA's first row, first leaf column

  auto at = [&](int lr, int cc) -> T& {
    if constexpr (IN_SMEM) return S[lr * kPanelStride + cc];
    else return g0[(int64_t)lr * ldw + cc];
  };

  if constexpr (IN_SMEM) {
    for (int e = tid; e < cnt * jb; e += kPanelThreads) {
      const int lr = e / jb, cc = e - lr * jb;
      S[lr * kPanelStride + cc] = g0[(int64_t)lr * ldw + cc];
    }
  }
  __syncthreads();
  if (P > 1) cluster_sync_all();  // every CTA of the cluster runs before any DSMEM access

  for (int c = 0; c < jb; ++c) {
    const int par = c & 1;
    const int d = j0 + c;  // the diagonal row
    // ---- this thread's candidate: first greatest magnitude among its rows >= d
    T bv = T(-1);
    int bi = INT_MAX;
    for (int lr = tid; lr < cnt; lr += kPanelThreads) {
      const int gi = j0 + base + lr;
      if (gi >= d) {
        const T v = fabs(at(lr, c));
        if (v > bv) {  // NaN never compares greater
          bv = v;
          bi = gi;
        }
      }
    }
    warp_argmax(bv, bi);
    if (lane == 0) {
      sh->red_v[warp] = bv;
      sh->red_i[warp] = bi;
    }
    __syncthreads();
    if (warp == 0) {
      bv = lane < kPanelWarps ? sh->red_v[lane] : T(-1);
      bi = lane < kPanelWarps ? sh->red_i[lane] : INT_MAX;
      warp_argmax(bv, bi);
      if (lane < jb) {
        if (bi != INT_MAX) sh->cand[par][lane] = at(bi - j0 - base, lane);
        const int dl = d - j0 - base;
        if (dl >= 0 && dl < cnt) sh->diag[par][lane] = at(dl, lane);
      }
      if (P > 1) {
        if (lane < P) {
          st_cluster(map_rank(&sh->slot_v[par][rank], lane), bv);
          st_cluster(map_rank(&sh->slot_i[par][rank], lane), bi);
        }
      } else if (lane == 0) {
        sh->slot_v[par][0] = bv;
        sh->slot_i[par][0] = bi;
      }
    }
    if (P > 1) cluster_sync_all();
    else __syncthreads();
    if (warp == 0) {
      T v = lane < P ? sh->slot_v[par][lane] : T(-1);
      int i = lane < P ? sh->slot_i[par][lane] : INT_MAX;
      warp_argmax(v, i);
      const int p = i == INT_MAX ? d : i;
      const int owner_p = (p - j0) / rpc, owner_d = (d - j0) / rpc;
      if (lane < jb) {
        T dv, pv;
        if (P > 1) {
          dv = ld_cluster<T>(map_rank(&sh->diag[par][lane], owner_d));
          pv = p == d ? dv : ld_cluster<T>(map_rank(&sh->cand[par][lane], owner_p));
        } else {
          dv = sh->diag[par][lane];
          pv = p == d ? dv : sh->cand[par][lane];
        }
        sh->piv[lane] = pv;
        sh->old[lane] = dv;
      }
      if (lane == 0) sh->p = p;
    }
    __syncthreads();
    const int p = sh->p;
    const T pivot = sh->piv[c];
    if (p != d) {
      const int dl = d - j0 - base, pl = p - j0 - base;
      if (dl >= 0 && dl < cnt && dl % kPanelThreads == tid)
        for (int cc = 0; cc < jb; ++cc) at(dl, cc) = sh->piv[cc];
      if (pl >= 0 && pl < cnt && pl % kPanelThreads == tid)
        for (int cc = 0; cc < jb; ++cc) at(pl, cc) = sh->old[cc];
    }
    if (pivot != T(0)) {
      const bool sub = fabs(pivot) < min_normal<T>();
      const T r = sub ? T(0) : T(1) / pivot;
      for (int lr = tid; lr < cnt; lr += kPanelThreads) {
        if (j0 + base + lr > d) {
          T l = at(lr, c);
          l = sub ? l / pivot : l * r;
          at(lr, c) = l;
#pragma unroll 8
          for (int cc = c + 1; cc < jb; ++cc) at(lr, cc) = fma(l, -sh->piv[cc], at(lr, cc));
        }
      }
    }
    if (rank == 0 && tid == 0) ipiv[d] = p;
  }

  if constexpr (IN_SMEM) {
    __syncthreads();
    for (int e = tid; e < cnt * jb; e += kPanelThreads) {
      const int lr = e / jb, cc = e - lr * jb;
      g0[(int64_t)lr * ldw + cc] = S[lr * kPanelStride + cc];
    }
  }
  if (P > 1) cluster_sync_all();  // no CTA leaves while a peer may still read its memory
}

// ------------------------------------------------------------------ short leaves in one CTA
// A leaf whose rows (M = n - j0 <= 768) fit one CTA: a thread per row, the leaf in shared
// memory, factored in sub-leaves of 8 columns. Rows do not move while the leaf is factored:
// each thread keeps its row's current position (relative to j0), a swap of positions d and p
// only exchanges the two threads' positions, and at the end every row is stored at its final
// position, which is where the explicit swaps of panel_kernel would have put it.
//
// Per sub-leaf, each thread holds its row's 8 items in registers and each column costs one CTA
// barrier: a candidate's key is its magnitude's bits + 1 (0 for NaN and for rows already
// chosen); each warp finds its largest key and, among equal keys, the lowest position (a
// redux.sync of the keys' high words; when several lanes share the largest high word, two
// more for the low words and the positions); its winner posts its sub-leaf row, position, key
// and reciprocal (every candidate forms its reciprocal while the reduction runs); after the
// barrier every warp reduces the posts the same way and reads the winning row. When every
// candidate is NaN the pivot is the diagonal's row (factor.rs:476), posted after a second
// barrier. After the sub-leaf, its pivot rows' later columns are solved against their unit
// lower triangle (a thread per column) and the rows still unchosen take the rank-8 update.
//
// The arithmetic on every item is panel_kernel's: the same reciprocal, and per item the same
// fma per pivot column in the same order (the deferred update applies the sub-leaf's columns
// one fma at a time in column order; a zero pivot's column is skipped, as panel_kernel skips
// it), so the results are the same bits. The sub-leaf loop is not unrolled: the kernel's code
// stays in the instruction cache (a leaf fully unrolled over 32 columns was bound by
// instruction fetch).
constexpr int kShortLeafMaxRows = 768;
constexpr int kShortWarps = kShortLeafMaxRows / 32;
constexpr int kSub = 8;
constexpr int kShortStride = kLeaf + 1;  // doubles per row in shared memory

struct alignas(16) ShortPost {
  double row[kSub];
  unsigned long long key;
  double rcp;
  int pos;
  int pad[3];
};

struct ShortShared {
  ShortPost post[2][kShortWarps + 1];  // a post per warp, and the diagonal's row
  double ub[kSub][kLeaf];              // the sub-leaf's pivot rows, later columns (U12)
  int pv[kSub];                        // the thread (row) of each pivot of the sub-leaf
  int pos[kShortLeafMaxRows];          // final positions
};

constexpr size_t short_leaf_smem(int rows) {
  return (sizeof(ShortShared) + 15) / 16 * 16 + (size_t)rows * kShortStride * sizeof(double);
}

// The lane holding the warp's largest key, the lowest position among equal keys; `zero` when
// every key is 0.
__device__ __forceinline__ int short_reduce(unsigned long long key, unsigned pos, bool& zero) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned top = __ballot_sync(0xffffffffu, hi == mhi);
  zero = false;
  if (__popc(top) == 1) return __ffs(top) - 1;  // mhi > 0 here: at most one lane holds a key of 0
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  const bool tie = hi == mhi && lo == mlo;
  const unsigned pmin = __reduce_min_sync(0xffffffffu, tie ? pos : 0xffffffffu);
  zero = mhi == 0u && mlo == 0u;
  return __ffs(__ballot_sync(0xffffffffu, tie && pos == pmin)) - 1;
}

// 1 / pivot as the cluster panel forms it (0 for a subnormal pivot, which is divided by)
__device__ __forceinline__ double short_rcp(double pv) {
  return fabs(pv) < 2.2250738585072014e-308 ? 0.0 : __drcp_rn(pv);
}

__device__ __forceinline__ void short_post(ShortPost& post, const double (&p)[kSub], int i, int pos,
                                           unsigned long long key, double rcp) {
  double2* dst = reinterpret_cast<double2*>(post.row);
#pragma unroll
  for (int q = i / 2; q < kSub / 2; ++q) dst[q] = make_double2(p[2 * q], p[2 * q + 1]);
  post.rcp = rcp;
  post.key = key;
  post.pos = pos;
}

__global__ void __launch_bounds__(kShortLeafMaxRows, 1)
    short_leaf_kernel(double* __restrict__ w, int64_t ldw, int n, int j0, int jb, int64_t* __restrict__ ipiv) {
  extern __shared__ __align__(16) uint8_t smem[];
  ShortShared& sh = *reinterpret_cast<ShortShared*>(smem);
  double* S = reinterpret_cast<double*>(smem + (sizeof(ShortShared) + 15) / 16 * 16);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int warps = blockDim.x >> 5;
  const int M = n - j0;
  griddep_launch_dependents();
  griddep_wait();  // the kernel before this one in the stream has completed
  // the leaf into shared memory: a warp per row, lanes along it (coalesced)
  for (int r = warp; r < M; r += warps)
    if (lane < jb) S[r * kShortStride + lane] = w[(int64_t)(j0 + r) * ldw + j0 + lane];
  __syncthreads();
  double* row = S + t * kShortStride;
  int pos = t < M ? t : INT_MAX;  // the row's current position; threads past M take no part
  bool active = t < M;
#pragma unroll 1
  for (int c0 = 0; c0 < jb; c0 += kSub) {
    double p[kSub];
#pragma unroll
    for (int i = 0; i < kSub; ++i) p[i] = (t < M && c0 + i < jb) ? row[c0 + i] : 0.0;
    unsigned skip = 0;  // the sub-leaf's columns whose pivot was zero (left unreduced)
#pragma unroll
    for (int i = 0; i < kSub; ++i) {
      const int c = c0 + i;
      if (c >= jb) break;
      ShortPost* pp = sh.post[c & 1];
      const double a = fabs(p[i]);
      const unsigned long long key =
          (active && a == a) ? (unsigned long long)__double_as_longlong(a) + 1ull : 0ull;
      const double myr = short_rcp(p[i]);
      bool none;
      const int wl = short_reduce(key, (unsigned)pos, none);
      if (lane == wl) short_post(pp[warp], p, i, pos, key, myr);
      __syncthreads();
      // every warp reduces the posts: the largest key, the lowest position among equals
      const unsigned long long k2 = lane < warps ? pp[lane].key : 0ull;
      const unsigned p2 = lane < warps ? (unsigned)pp[lane].pos : 0xffffffffu;
      const int bw = short_reduce(k2, p2, none);
      const ShortPost* win = &pp[bw];
      if (none) {  // every candidate is NaN: the diagonal's row is the pivot row
        if (pos == c) short_post(pp[kShortWarps], p, i, pos, 0ull, myr);
        __syncthreads();
        win = &pp[kShortWarps];
      }
      const int pr = win->pos;
      const double pivot = win->row[i];
      const double r = win->rcp;
      if (pos == pr) {
        active = false;
        pos = c;
        sh.pv[i] = t;
      } else if (pos == c) {
        pos = pr;
      }
      if (t == 0) ipiv[j0 + c] = j0 + pr;
      if (pivot == 0.0) skip |= 1u << i;
      if (active && pivot != 0.0) {
        const bool sub = fabs(pivot) < 2.2250738585072014e-308;
        double l = p[i];
        l = sub ? l / pivot : l * r;
        p[i] = l;
        const double2* prow = reinterpret_cast<const double2*>(win->row);
#pragma unroll
        for (int q = (i + 1) / 2; q < kSub / 2; ++q) {
          const double2 u = prow[q];
          if (2 * q > i) p[2 * q] = fma(l, -u.x, p[2 * q]);
          if (2 * q + 1 > i) p[2 * q + 1] = fma(l, -u.y, p[2 * q + 1]);
        }
      }
    }
    if (t < M) {
#pragma unroll
      for (int i = 0; i < kSub; ++i)
        if (c0 + i < jb) row[c0 + i] = p[i];
    }
    const int rc0 = c0 + kSub, rcols = jb - rc0;
    if (rcols <= 0) break;
    __syncthreads();
    // U12: the sub-leaf's pivot rows, later columns, against their unit lower triangle; a
    // thread per column, the same fmas in the same order as the rank-1 updates
    if (t < rcols) {
      double u[kSub];
#pragma unroll
      for (int k = 0; k < kSub; ++k) u[k] = S[sh.pv[k] * kShortStride + rc0 + t];
#pragma unroll
      for (int k = 1; k < kSub; ++k) {
        const double* lrow = S + sh.pv[k] * kShortStride + c0;
#pragma unroll
        for (int q = 0; q < k; ++q)
          if (!((skip >> q) & 1u)) u[k] = fma(lrow[q], -u[q], u[k]);
      }
#pragma unroll
      for (int k = 0; k < kSub; ++k) {
        S[sh.pv[k] * kShortStride + rc0 + t] = u[k];
        sh.ub[k][t] = u[k];
      }
    }
    __syncthreads();
    // the rows still unchosen: later columns, one fma per pivot column in column order
    if (active) {
      for (int j = 0; j < rcols; ++j) {
        double x = row[rc0 + j];
#pragma unroll
        for (int k = 0; k < kSub; ++k)
          if (!((skip >> k) & 1u)) x = fma(p[k], -sh.ub[k][j], x);
        row[rc0 + j] = x;
      }
    }
    __syncthreads();
  }
  // the leaf back, every row at its final position: a warp per row, lanes along it
  if (t < M) sh.pos[t] = pos;
  __syncthreads();
  for (int r2 = warp; r2 < M; r2 += warps)
    if (lane < jb) w[(int64_t)(j0 + sh.pos[r2]) * ldw + j0 + lane] = S[r2 * kShortStride + lane];
}

// ------------------------------------------------------------------ a whole matrix in a cluster
// n <= 256: the whole matrix lives in the shared memory of one cluster of C <= 8 CTAs (a power
// of two, at most 32 rows per CTA; 66 KB per CTA at n = 256) and is factored in one launch,
// column by column, right-looking, with one cluster barrier per pivot column, in place of the
// blocked path's chain of dependent launches (leaves, swaps, inversions, block products). Each
// item takes the fmas of rustymath's packed products in the same order (one per pivot column,
// in column order), so the factors are the oracle's bits. Measured per solve (n = 128 / 192 /
// 256): 0.29 / 0.41 / 0.51 ms against 0.31 / 0.47 / 0.57 ms on the blocked path; a column costs
// ~1.1 us at C = 2 and ~2.2 us at C = 16 (the cluster barrier and the pivot row's reads from one
// CTA's shared memory), so at n = 384..512 the blocked path is faster and keeps those sizes.
//
// Rows do not move. Every warp of a CTA tracks the positions of the CTA's rows (lane = row), so
// a pivot choice only exchanges two positions, as in short_leaf_kernel; at the end each row is
// stored at its final position. Per pivot column j, after the barrier that publishes column j's
// candidates:
//   - every warp reduces the C posts (largest key, lowest position among equals; when every
//     candidate is NaN, the row at position j, which its CTA posts beside its candidate) and
//     forms its rows' multipliers l = a_ij / pivot (the reciprocal as the other panels form it);
//   - warp 0 updates column j + 1 (the pivot row's item read from the winner's shared memory),
//     keeps it, finds its CTA's candidate for column j + 1 and posts it into every CTA's slot;
//   - the other warps update columns j + 2 .. n - 1, 32 columns per warp, the pivot row's items
//     read from the winner's shared memory a lane each and passed on by shuffles.
// Posts are double-buffered by the column's parity: a CTA writes the slot of column j + 2 only
// after the barrier of column j + 1, which every CTA reaches after it has read column j's posts.
// Each item takes one fma per pivot column, in column order; a zero pivot leaves its column
// unreduced (factor.rs:606); the multipliers of column j are written into column j at the next
// step, when no warp reads that column any more. Every CTA runs the same n barriers, so the
// barrier cannot be left waiting.
constexpr int kClusterLuMax = 256;
constexpr int kClusterLuRows = 32;  // rows per CTA at most (a lane each)

struct alignas(16) ClusterPost {
  unsigned long long key;  // |candidate| bits + 1; 0 for NaN or no row left
  double piv;              // the candidate's item
  double dpiv;             // the item of the row at the diagonal's position, when this CTA holds it
  int pos;                 // the candidate's position
  int lrow;                // its row within the CTA
  int drow;                // the CTA's row at the diagonal's position, or -1
  int pad;
};

struct ClusterLuShared {
  ClusterPost post[2][kMaxCluster];  // [column parity][posting CTA]
};

__device__ __forceinline__ void st_cluster_u64(uint32_t a, unsigned long long v) {
  asm volatile("st.shared::cluster.u64 [%0], %1;" ::"r"(a), "l"(v) : "memory");
}

// Warp 0 of each CTA: the CTA's candidate for column `col` (y = this lane's row's item) and, if
// the CTA holds it, the row at position `col`, stored into slot `slot` of every CTA's posts.
__device__ __forceinline__ void cluster_lu_post(ClusterLuShared& sh, int slot, double y, int pos, bool active,
                                                int col, int C, int rank, int lane) {
  const double a = fabs(y);
  const unsigned long long key = (active && a == a) ? (unsigned long long)__double_as_longlong(a) + 1ull : 0ull;
  bool none;
  const int wl = short_reduce(key, (unsigned)pos, none);
  const unsigned long long wkey = __shfl_sync(0xffffffffu, key, wl);
  const double wpiv = __shfl_sync(0xffffffffu, y, wl);
  const int wpos = __shfl_sync(0xffffffffu, pos, wl);
  const unsigned db = __ballot_sync(0xffffffffu, pos == col);
  const int dl = db ? __ffs(db) - 1 : -1;
  const double dpiv = __shfl_sync(0xffffffffu, y, dl < 0 ? 0 : dl);
  if (lane < C) {
    const uint32_t d = map_rank(&sh.post[slot][rank], (uint32_t)lane);
    st_cluster_u64(d + offsetof(ClusterPost, key), wkey);
    st_cluster(d + offsetof(ClusterPost, piv), wpiv);
    st_cluster(d + offsetof(ClusterPost, dpiv), dpiv);
    st_cluster(d + offsetof(ClusterPost, pos), wpos);
    st_cluster(d + offsetof(ClusterPost, lrow), wl);
    st_cluster(d + offsetof(ClusterPost, drow), dl);
  }
}

// W (row-major, ldw) is factored in place: on return row i of W holds row i of the factors (the
// source row perm[i]); ipiv[j] is the position exchanged with j at step j. R rows per CTA, ld
// the shared row stride (odd: a warp's column reads hit distinct banks).
__global__ void __launch_bounds__(32 * (1 + kClusterLuMax / 32), 1)
    cluster_lu_kernel(double* __restrict__ w, int64_t ldw, int n, int R, int ld, int64_t* __restrict__ ipiv,
                      int64_t* __restrict__ perm) {
  extern __shared__ __align__(16) uint8_t smem[];
  ClusterLuShared& sh = *reinterpret_cast<ClusterLuShared*>(smem);
  double* S = reinterpret_cast<double*>(smem + sizeof(ClusterLuShared));
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int nwarps = blockDim.x >> 5;
  const int rank = (int)cluster_ctarank(), C = (int)cluster_nctarank();
  const int g0 = rank * R;
  const int rows = max(0, min(R, n - g0));
  for (int i = warp; i < rows; i += nwarps)
    for (int c = lane; c < n; c += 32) S[i * ld + c] = w[(int64_t)(g0 + i) * ldw + c];
  const bool valid = lane < rows;
  int pos = valid ? g0 + lane : INT_MAX;
  double* myrow = S + (valid ? lane : 0) * ld;
  cluster_sync_all();  // the rows are in, and every CTA of the cluster runs before any DSMEM access
  if (warp == 0) cluster_lu_post(sh, 0, valid ? myrow[0] : 0.0, pos, valid, 0, C, rank, lane);
  cluster_sync_all();
  double lprev = 0.0;  // warp 0: the multiplier of the step before, written one step late
  bool lprev_set = false;
#pragma unroll 1
  for (int j = 0; j < n; ++j) {
    const ClusterPost* pp = sh.post[j & 1];
    const unsigned long long k2 = lane < C ? pp[lane].key : 0ull;
    const unsigned p2 = lane < C ? (unsigned)pp[lane].pos : 0xffffffffu;
    bool none;
    int wr = short_reduce(k2, p2, none);
    int lr, pr;
    double piv;
    if (!none) {
      lr = pp[wr].lrow;
      pr = pp[wr].pos;
      piv = pp[wr].piv;
    } else {  // every candidate is NaN: the row at position j is the pivot row
      const unsigned b = __ballot_sync(0xffffffffu, lane < C && pp[lane].drow >= 0);
      wr = __ffs(b) - 1;
      lr = pp[wr].drow;
      pr = j;
      piv = pp[wr].dpiv;
    }
    if (pos == pr) pos = j;
    else if (pos == j) pos = pr;
    const bool active = valid && pos > j;
    const bool skip = piv == 0.0;
    const bool sub = fabs(piv) < 2.2250738585072014e-308;
    const double rcp = short_rcp(piv);
    double l = 0.0;
    if (active && !skip) {
      const double a = myrow[j];
      l = sub ? a / piv : a * rcp;
    }
    const uint32_t prow = map_rank(S + lr * ld, (uint32_t)wr);  // the pivot row, in CTA wr
    if (warp == 0) {
      if (lprev_set) myrow[j - 1] = lprev;
      lprev = l;
      lprev_set = active && !skip;
      if (j + 1 < n) {
        double y = valid ? myrow[j + 1] : 0.0;
        if (!skip) {
          const double u = ld_cluster_f64(prow + (uint32_t)(j + 1) * 8u);
          if (active) {
            y = fma(l, -u, y);
            myrow[j + 1] = y;
          }
        }
        cluster_lu_post(sh, (j + 1) & 1, y, pos, active, j + 1, C, rank, lane);
      }
    } else if (!skip) {
#pragma unroll 1
      for (int c0 = j + 2 + (warp - 1) * 32; c0 < n; c0 += (nwarps - 1) * 32) {
        const int cc = c0 + lane;
        const double ul = cc < n ? ld_cluster_f64(prow + (uint32_t)cc * 8u) : 0.0;
        const int cend = min(32, n - c0);
        double* rp = myrow + c0;
        if (cend == 32) {
#pragma unroll 8
          for (int q = 0; q < 32; ++q) {
            const double u = __shfl_sync(0xffffffffu, ul, q);
            if (active) rp[q] = fma(l, -u, rp[q]);
          }
        } else {
          for (int q = 0; q < cend; ++q) {
            const double u = __shfl_sync(0xffffffffu, ul, q);
            if (active) rp[q] = fma(l, -u, rp[q]);
          }
        }
      }
    }
    if (rank == 0 && t == 0) ipiv[j] = pr;
    cluster_sync_all();
  }
  // every row to its final position: a warp per row, lanes along it
  for (int i = warp; i < rows; i += nwarps) {
    const int pi = __shfl_sync(0xffffffffu, pos, i);
    for (int c = lane; c < n; c += 32) w[(int64_t)pi * ldw + c] = S[i * ld + c];
  }
  if (warp == 0 && valid) perm[pos] = g0 + lane;
}

constexpr size_t cluster_lu_smem(int R, int ld) {
  return sizeof(ClusterLuShared) + (size_t)R * ld * sizeof(double);
}

// ------------------------------------------------------------------ small solves in one CTA
// x = U^-1 L^-1 b[perm] for n <= 256 and k <= 8 from W (rows at their final positions), in one
// CTA: a thread per row holds its row of x; per column one barrier. The order is that of
// rustymath's single-column solve (`single` on the transposed factors, factor.rs:725-748):
// forward, column j after column j - 1, x_i = fma(l_ij, -x_j, x_i) for i > j; backward, from the
// last column, x_j = x_j / u_jj, then x_i = fma(u_ij, -x_j, x_i) for i < j. With one right-hand
// side the result is the oracle's bits; with more, each column is solved the same way. W comes
// in 32-column blocks through two shared-memory buffers, the next block's copies in flight
// while the current one is used.
constexpr int kSmallSolveMax = 256;
constexpr int kSmallSolveK = 8;
constexpr int kSsCols = 32;
constexpr int kSsStride = kSsCols + 2;  // doubles per staged row (16-byte aligned rows)

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// COLMAJOR: the factors in rustymath's order (item (i, j) at w[j * ldw + i], exactly n columns),
// staged as columns ([32][n] per buffer); else W row-major ([n][kSsStride] per buffer). A row
// position outside 0..n-1 sets RM_DEV_BAD_INDEX in *status (when given) and that row's right-hand
// side is taken as zero.
template <bool COLMAJOR>
__global__ void __launch_bounds__(kSmallSolveMax, 1)
    small_solve_kernel(const double* __restrict__ w, int64_t ldw, int n, const int64_t* __restrict__ perm,
                       const double* b, int k, double* x, unsigned* status) {
  extern __shared__ __align__(16) uint8_t smem[];
  double* buf = reinterpret_cast<double*>(smem);  // two staging buffers of kSsCols * kSsStride * ... doubles
  __shared__ double xs[2][kSmallSolveK];
  const int t = threadIdx.x;
  const bool own = t < n;
  const int nblk = (n + kSsCols - 1) / kSsCols;
  double v[kSmallSolveK];
  {
    const int64_t src = own ? perm[t] : 0;
    const bool in = src >= 0 && src < n;
    if (own && !in && status) flag_error(status, RM_DEV_BAD_INDEX);
#pragma unroll
    for (int c = 0; c < kSmallSolveK; ++c) v[c] = (own && in && c < k) ? b[src * k + c] : 0.0;
  }
  const size_t bufsz = COLMAJOR ? (size_t)kSsCols * n : (size_t)n * kSsStride;
  // stage q: forward blocks 0..nblk-1, then backward blocks nblk-1..0
  auto stage = [&](int q) {
    const int blk = q < nblk ? q : 2 * nblk - 1 - q;
    double* dst = buf + (q & 1) * bufsz;
    if constexpr (COLMAJOR) {  // columns blk*32 .. min(n, blk*32 + 32) - 1, a row item each
      const int c0 = blk * kSsCols, cols = min(kSsCols, n - c0);
      for (int e = t; e < cols * n; e += kSmallSolveMax) {
        const int c = e / n, r = e % n;
        cp_async8(dst + (size_t)c * n + r, w + (int64_t)(c0 + c) * ldw + r);
      }
    } else {
      const double* src = w + (int64_t)blk * kSsCols;
      for (int e = t; e < n * (kSsCols / 2); e += kSmallSolveMax) {
        const int r = e / (kSsCols / 2), h = e % (kSsCols / 2);
        cp_async16(dst + r * kSsStride + 2 * h, src + (int64_t)r * ldw + 2 * h);
      }
    }
    cp_async_commit();
  };
  stage(0);
  for (int q = 0; q < 2 * nblk; ++q) {
    cp_async_wait<0>();
    __syncthreads();  // stage q is in; every thread is done with stage q - 1's buffer
    if (q + 1 < 2 * nblk) stage(q + 1);
    const double* S = buf + (q & 1) * bufsz;
    // item (t, c0 + i) of the staged block is mine[i * step]
    const double* mine = COLMAJOR ? S + (own ? t : 0) : S + (own ? t : 0) * kSsStride;
    const int step = COLMAJOR ? n : 1;
    if (q < nblk) {
      const int c0 = q * kSsCols, c1 = min(n, c0 + kSsCols);
      for (int j = c0; j < c1; ++j) {
        double* xj = xs[j & 1];
        if (t == j)
#pragma unroll
          for (int c = 0; c < kSmallSolveK; ++c)
            if (c < k) xj[c] = v[c];
        __syncthreads();
        if (own && t > j) {
          const double l = mine[(j - c0) * step];
#pragma unroll
          for (int c = 0; c < kSmallSolveK; ++c)
            if (c < k) v[c] = fma(l, -xj[c], v[c]);
        }
      }
    } else {
      const int blk = 2 * nblk - 1 - q, c0 = blk * kSsCols, c1 = min(n, c0 + kSsCols);
      for (int j = c1 - 1; j >= c0; --j) {
        double* xj = xs[j & 1];
        if (t == j) {  // the divisions are on the critical path: only the k columns in use
          const double d = mine[(j - c0) * step];
#pragma unroll
          for (int c = 0; c < kSmallSolveK; ++c)
            if (c < k) xj[c] = v[c] = v[c] / d;
        }
        __syncthreads();
        if (own && t < j) {
          const double u = mine[(j - c0) * step];
#pragma unroll
          for (int c = 0; c < kSmallSolveK; ++c)
            if (c < k) v[c] = fma(u, -xj[c], v[c]);
        }
      }
    }
  }
  if (own)
#pragma unroll
    for (int c = 0; c < kSmallSolveK; ++c)
      if (c < k) x[(int64_t)t * k + c] = v[c];
}

// The plain solve takes this kernel up to n = 192: measured per solve (n = 8 / 32 / 64 / 128 / 192 / 256,
// one right-hand side) 0.051 / 0.092 / 0.142 / 0.244 / 0.380 / 0.513 ms against 0.127 / 0.155 / 0.178 /
// 0.271 / 0.385 / 0.490 ms with the block-chained solves.
constexpr int kSmallSolveRoute = 192;
bool small_solve_fits(int64_t n, int64_t k) { return n >= 1 && n <= kSmallSolveRoute && k >= 1 && k <= kSmallSolveK; }

int small_solve_f64(const double* w, int64_t ldw, bool colmajor, int64_t n, const int64_t* perm, const double* b,
                    int64_t k, double* x, unsigned* status, cudaStream_t stream) {
  if (n < 1 || n > kSmallSolveMax || k < 1 || k > kSmallSolveK) return RM_BAD_ARG;
  if (colmajor) {
    RM_TRY(smem_attribute(small_solve_kernel<true>, (size_t)2 * kSsCols * kSmallSolveMax * sizeof(double)));
    small_solve_kernel<true><<<1, kSmallSolveMax, (size_t)2 * kSsCols * n * sizeof(double), stream>>>(
        w, ldw, (int)n, perm, b, (int)k, x, status);
  } else {
    RM_TRY(smem_attribute(small_solve_kernel<false>, (size_t)2 * kSmallSolveMax * kSsStride * sizeof(double)));
    small_solve_kernel<false><<<1, kSmallSolveMax, (size_t)2 * n * kSsStride * sizeof(double), stream>>>(
        w, ldw, (int)n, perm, b, (int)k, x, status);
  }
  RM_LAUNCHED();
  return RM_OK;
}

// ------------------------------------------------------------------ swaps + unit-lower solve
constexpr int kSwapCols = 16;      // columns per CTA
constexpr int kSwapThreads = 256;
constexpr int kMaxSwaps = kOuter;  // pivots applied by one launch

// Applies the swaps ipiv[j0..j0+jb) in order to the columns [lo1,hi1) and [lo2,hi2) of W.
// With trsm_lo < trsm_hi, rows j0..j0+jb-1 of the columns in that range are then replaced
// by L^-1 times them, L the unit lower triangle of W[j0.., j0..] (jb <= kLeaf). Block 0
// also applies the swaps to perm when perm is not NULL.
template <typename T>
__global__ void __launch_bounds__(kSwapThreads)
    swap_trsm_kernel(T* __restrict__ w, int64_t ldw, int j0, int jb, const int64_t* __restrict__ ipiv, int lo1,
                     int hi1, int lo2, int hi2, int trsm_lo, int trsm_hi, int64_t* __restrict__ perm) {
  __shared__ int pos[2 * kMaxSwaps], src[2 * kMaxSwaps];
  __shared__ int count;
  __shared__ T buf[2 * kMaxSwaps][kSwapCols + 1];
  __shared__ T lblk[kLeaf][kLeaf + 1];
  __shared__ int ipv[kMaxSwaps];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  griddep_launch_dependents();
  griddep_wait();  // the kernel before this one in the stream has completed
  // the swaps' targets, all at once (the loop below is sequential over them)
  for (int q = tid; q < jb; q += kSwapThreads) ipv[q] = (int)ipiv[j0 + q];
  __syncthreads();

  // ---- the net effect of the swaps: row pos[e] receives the old row src[e]
  if (warp == 0) {
    for (int q = lane; q < jb; q += 32) pos[q] = src[q] = j0 + q;
    int cntE = jb;
    for (int i = 0; i < jb; ++i) {
      const int d = j0 + i, p = ipv[i];
      if (p == d) continue;
      int e;
      if (p < j0 + jb) {
        e = p - j0;
      } else {
        e = -1;
        for (int b = jb; b < cntE && e < 0; b += 32) {
          const unsigned hit = __ballot_sync(0xffffffffu, b + lane < cntE && pos[b + lane] == p);
          if (hit) e = b + __ffs(hit) - 1;
        }
        if (e < 0) {
          e = cntE;
          if (lane == 0) pos[e] = src[e] = p;
          ++cntE;
        }
        __syncwarp();
      }
      if (lane == 0) {
        const int t = src[i];
        src[i] = src[e];
        src[e] = t;
      }
      __syncwarp();
    }
    if (lane == 0) count = cntE;
  }
  __syncthreads();
  const int E = count;

  // ---- the columns of this CTA
  const int chunks1 = (hi1 - lo1 + kSwapCols - 1) / kSwapCols;
  int c0, c1;
  if ((int)blockIdx.x < chunks1) {
    c0 = lo1 + blockIdx.x * kSwapCols;
    c1 = min(c0 + kSwapCols, hi1);
  } else {
    c0 = lo2 + (blockIdx.x - chunks1) * kSwapCols;
    c1 = min(c0 + kSwapCols, hi2);
  }
  const int width = c1 - c0;

  if (width > 0) {
    for (int e = tid; e < E * kSwapCols; e += kSwapThreads) {
      const int r = e / kSwapCols, cc = e - r * kSwapCols;
      if (cc < width) buf[r][cc] = w[(int64_t)src[r] * ldw + c0 + cc];
    }
  }
  const bool solve = width > 0 && trsm_lo < trsm_hi && c0 >= trsm_lo && c1 <= trsm_hi;
  if (solve)
    for (int e = tid; e < jb * kLeaf; e += kSwapThreads) {
      const int r = e / kLeaf, cc = e - r * kLeaf;
      lblk[r][cc] = cc < jb ? w[(int64_t)(j0 + r) * ldw + j0 + cc] : T(0);
    }
  __syncthreads();
  if (solve) {
    // one warp per column: lane r holds row r; row i is final once rows < i are removed
    for (int cc = warp; cc < width; cc += kSwapThreads / 32) {
      T x = lane < jb ? buf[lane][cc] : T(0);
      for (int i = 0; i < jb; ++i) {
        const T xi = __shfl_sync(0xffffffffu, x, i);
        if (lane > i && lane < jb) x = fma(-lblk[lane][i], xi, x);
      }
      if (lane < jb) buf[lane][cc] = x;
    }
    __syncthreads();
  }
  if (width > 0) {
    for (int e = tid; e < E * kSwapCols; e += kSwapThreads) {
      const int r = e / kSwapCols, cc = e - r * kSwapCols;
      if (cc < width && (pos[r] != src[r] || (solve && r < jb))) w[(int64_t)pos[r] * ldw + c0 + cc] = buf[r][cc];
    }
  }
  if (perm != nullptr && blockIdx.x == 0) {
    int64_t v[(2 * kMaxSwaps + kSwapThreads - 1) / kSwapThreads];
#pragma unroll
    for (int s = 0; s < (int)(sizeof(v) / sizeof(v[0])); ++s) {
      const int e = tid + s * kSwapThreads;
      v[s] = e < E ? perm[src[e]] : 0;
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < (int)(sizeof(v) / sizeof(v[0])); ++s) {
      const int e = tid + s * kSwapThreads;
      if (e < E) perm[pos[e]] = v[s];
    }
  }
}

// ------------------------------------------------------------------ driver

// The largest cluster (<= kMaxCluster CTAs of kPanelSmemBudget bytes) this device can place.
template <typename T>
static int find_panel_cluster_limit() {
  int limit = 0;
  auto k = panel_kernel<T, true>;
  if (smem_attribute(k, kPanelSmemBudget + 4096) != RM_OK ||
      func_attribute(reinterpret_cast<const void*>(k), cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != RM_OK ||
      func_attribute(reinterpret_cast<const void*>(panel_kernel<T, false>),
                     cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != RM_OK) {
    cudaGetLastError();
    return limit = 8;
  }
  for (int P = kMaxCluster; P >= 1; P /= 2) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = P;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(P);
    cfg.blockDim = dim3(kPanelThreads);
    cfg.dynamicSmemBytes = kPanelSmemBudget;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k, &cfg) == cudaSuccess && clusters > 0) return limit = P;
    cudaGetLastError();
  }
  return limit = 1;
}

// Found once per device (the attributes and the answer belong to that device).
template <typename T>
static int panel_cluster_limit() {
  static std::mutex mu;
  static std::vector<int> limits;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  {
    std::lock_guard<std::mutex> lock(mu);
    if ((int)limits.size() > dev && limits[dev]) return limits[dev];
  }
  const int limit = find_panel_cluster_limit<T>();
  std::lock_guard<std::mutex> lock(mu);
  if ((int)limits.size() <= dev) limits.resize(dev + 1, 0);
  limits[dev] = limit;
  return limit;
}


// Whether this device can place the largest cluster cluster_lu_kernel takes (8 CTAs of 288
// threads and 66 KB of shared memory); found once per device.
constexpr int kClusterLuMaxCtas = kClusterLuMax / kClusterLuRows;
static bool find_cluster_lu_ok() {
  const size_t smem = cluster_lu_smem(kClusterLuRows, kClusterLuMax + 1);
  if (smem_attribute(cluster_lu_kernel, smem) != RM_OK) {
    cudaGetLastError();
    return false;
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kClusterLuMaxCtas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(kClusterLuMaxCtas);
  cfg.blockDim = dim3(32 * (1 + kClusterLuMax / 32));
  cfg.dynamicSmemBytes = smem;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, cluster_lu_kernel, &cfg) == cudaSuccess && clusters > 0) return true;
  cudaGetLastError();
  return false;
}

static bool cluster_lu_ok() {
  static std::mutex mu;
  static std::vector<int> state;  // 0 unknown, 1 yes, 2 no
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  {
    std::lock_guard<std::mutex> lock(mu);
    if ((int)state.size() > dev && state[dev]) return state[dev] == 1;
  }
  const bool ok = find_cluster_lu_ok();
  std::lock_guard<std::mutex> lock(mu);
  if ((int)state.size() <= dev) state.resize(dev + 1, 0);
  state[dev] = ok ? 1 : 2;
  return ok;
}

// n <= kClusterLuMax in one launch: C CTAs (the least power of two giving at most 32 rows each).
static int launch_cluster_lu(double* w, int64_t ldw, int n, int64_t* ipiv, int64_t* perm, cudaStream_t stream) {
  const int need = (n + kClusterLuRows - 1) / kClusterLuRows;
  int C = 1;
  while (C < need) C *= 2;
  const int R = (n + C - 1) / C;
  const int ld = n | 1;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(32 * (1 + (n + 31) / 32));
  cfg.dynamicSmemBytes = cluster_lu_smem(R, ld);
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  RM_CUDA_TRY(cudaLaunchKernelEx(&cfg, cluster_lu_kernel, w, ldw, n, R, ld, ipiv, perm));
  note_launch();
  return RM_OK;
}

template <typename T>
static int launch_panel(T* w, int64_t ldw, int n, int j0, int jb, int64_t* ipiv, cudaStream_t stream) {
  const int M = n - j0;
  if constexpr (sizeof(T) == 8) {
    if (M <= kShortLeafMaxRows) {  // one CTA, a thread per row
      RM_TRY(smem_attribute(short_leaf_kernel, short_leaf_smem(kShortLeafMaxRows)));
      RM_CUDA_TRY(launch_dependent(short_leaf_kernel, dim3(1), dim3((M + 31) / 32 * 32), short_leaf_smem(M), stream, w,
                                   ldw, n, j0, jb, ipiv));
      note_launch();
      return RM_OK;
    }
  }
  const size_t sh = (sizeof(PanelShared<T>) + 15) / 16 * 16;
  const int rows_cap = (int)((kPanelSmemBudget - sh) / (kPanelStride * sizeof(T)));
  const int pmax = panel_cluster_limit<T>();
  int P = 1;
  while (P < pmax && (M + P - 1) / P > rows_cap) P *= 2;
  // spread tall leaves over more CTAs: about 2 rows per thread
  while (P < pmax && (M + P - 1) / P > 2 * kPanelThreads) P *= 2;
  const int rpc = (M + P - 1) / P;
  const bool in_smem = rpc <= rows_cap;
  const size_t smem = (in_smem ? ((size_t)rpc * kPanelStride * sizeof(T) + 15) / 16 * 16 : 0) + sh;

  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = P;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(P);
  cfg.blockDim = dim3(kPanelThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (in_smem) {
    RM_CUDA_TRY(cudaLaunchKernelEx(&cfg, panel_kernel<T, true>, w, ldw, n, j0, jb, rpc, ipiv));
  } else {
    RM_CUDA_TRY(cudaLaunchKernelEx(&cfg, panel_kernel<T, false>, w, ldw, n, j0, jb, rpc, ipiv));
  }
  note_launch();
  return RM_OK;
}

template <typename T>
static int launch_swap(T* w, int64_t ldw, int j0, int jb, const int64_t* ipiv, int lo1, int hi1, int lo2, int hi2,
                       int trsm_lo, int trsm_hi, int64_t* perm, cudaStream_t stream) {
  hi1 = max(hi1, lo1);
  hi2 = max(hi2, lo2);
  const int chunks = (hi1 - lo1 + kSwapCols - 1) / kSwapCols + (hi2 - lo2 + kSwapCols - 1) / kSwapCols;
  const int grid = max(chunks, perm ? 1 : 0);
  if (grid == 0) return RM_OK;
  RM_CUDA_TRY(launch_dependent(swap_trsm_kernel<T>, dim3(grid), dim3(kSwapThreads), 0, stream, w, ldw, j0, jb, ipiv, lo1,
                               hi1, lo2, hi2, trsm_lo, trsm_hi, perm));
  note_launch();
  return RM_OK;
}

// L11^-1 of the unit lower triangle of the nb x nb diagonal block at (j0, j0) (row-major,
// ld kOuter, zeros above the diagonal; identity beyond nb), a 32-column block of it per CTA
// (4 CTAs), everything in shared memory: CTA a forms X_aa = D_a^-1 and then, block row by block
// row, X_ba = -D_b^-1 sum_{c=a..b-1} L_bc X_ca; the diagonal blocks' inverses D_b^-1 first, a
// warp each, a lane per column (forward substitution).
constexpr int kInvS = kOuter + 1;
constexpr size_t kInv64Smem = ((size_t)kOuter * kInvS + (size_t)(4 * kLeaf + kOuter + kLeaf) * (kLeaf + 1)) *
                              sizeof(double);

__global__ void __launch_bounds__(256) invert_unit_lower_f64_kernel(const double* __restrict__ w, int64_t ldw, int j0,
                                                                    int nb, double* __restrict__ out) {
  extern __shared__ __align__(16) uint8_t smraw[];
  double(*M)[kInvS] = reinterpret_cast<double(*)[kInvS]>(smraw);
  double(*Y)[kLeaf + 1] = reinterpret_cast<double(*)[kLeaf + 1]>(smraw + (size_t)kOuter * kInvS * sizeof(double));
  double(*X)[kLeaf + 1] = Y + 4 * kLeaf;  // the column block, rows 0..127
  double(*Tq)[kLeaf + 1] = X + kOuter;     // 32 x 33
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ab = blockIdx.x, a0 = kLeaf * ab;
  const double* l = w + (int64_t)j0 * ldw + j0;
  griddep_launch_dependents();
  griddep_wait();  // the kernel before this one in the stream has completed
  // L from row and column a0 on (strictly lower part; unit diagonal implied)
  for (int i = a0 + warp; i < kOuter; i += 8)
    for (int k = a0 + lane; k < kOuter; k += 32) M[i][k] = (i < nb && k < nb && k < i) ? l[(int64_t)i * ldw + k] : 0.0;
  __syncthreads();
  if (warp < 4 - ab) {  // Y_b = D_b^-1, b = ab + warp
    const int b0 = a0 + kLeaf * warp;
    double x[kLeaf];
#pragma unroll
    for (int i = 0; i < kLeaf; ++i) {
      double acc = i == lane ? 1.0 : 0.0;
#pragma unroll
      for (int k2 = 0; k2 < i; ++k2) acc = fma(-M[b0 + i][b0 + k2], x[k2], acc);
      x[i] = i < lane ? 0.0 : acc;
    }
#pragma unroll
    for (int i = 0; i < kLeaf; ++i) Y[b0 + i][lane] = x[i];
  }
  __syncthreads();
  for (int e = tid; e < kLeaf * kLeaf; e += 256) X[a0 + (e >> 5)][e & 31] = Y[a0 + (e >> 5)][e & 31];
  __syncthreads();
  const int ti = tid >> 4, tj = tid & 15;  // rows ti, ti + 16 and columns tj, tj + 16 of a 32 x 32 block
  for (int b = ab + 1; b < 4; ++b) {
    const int r0 = kLeaf * b + ti, r1 = r0 + 16;
    double t00 = 0.0, t01 = 0.0, t10 = 0.0, t11 = 0.0;
#pragma unroll 4
    for (int k = a0; k < kLeaf * b; ++k) {
      const double m0 = M[r0][k], m1 = M[r1][k], x0 = X[k][tj], x1 = X[k][tj + 16];
      t00 = fma(m0, x0, t00), t01 = fma(m0, x1, t01), t10 = fma(m1, x0, t10), t11 = fma(m1, x1, t11);
    }
    Tq[ti][tj] = t00, Tq[ti][tj + 16] = t01, Tq[ti + 16][tj] = t10, Tq[ti + 16][tj + 16] = t11;
    __syncthreads();
    t00 = t01 = t10 = t11 = 0.0;
#pragma unroll 4
    for (int k2 = 0; k2 < kLeaf; ++k2) {
      const double y0 = Y[r0][k2], y1 = Y[r1][k2], u0 = Tq[k2][tj], u1 = Tq[k2][tj + 16];
      t00 = fma(y0, u0, t00), t01 = fma(y0, u1, t01), t10 = fma(y1, u0, t10), t11 = fma(y1, u1, t11);
    }
    X[r0][tj] = -t00, X[r0][tj + 16] = -t01, X[r1][tj] = -t10, X[r1][tj + 16] = -t11;
    __syncthreads();
  }
  for (int rr = warp; rr < kOuter; rr += 8) out[rr * kOuter + a0 + lane] = rr >= a0 ? X[rr][lane] : 0.0;
}

__global__ void iota_kernel(int64_t* perm, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    perm[i] = i;
}

size_t getrf_f64_scratch_bytes(int64_t n) { return (size_t)kOuter * kOuter * sizeof(double) + 256; }

namespace {
// The look-ahead's streams: the critical chain (hp) at the device's highest stream priority, the
// rest of each trailing update (side) at its lowest, so that the chain's panel clusters take
// SMs first as the update's tiles finish. Released on return (queued work completes first).
struct F64LookAhead {
  cudaStream_t hp = nullptr, side = nullptr;
  cudaEvent_t next_done = nullptr, rest_done = nullptr, entry = nullptr;
  int open() {
    int least = 0, greatest = 0;
    RM_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    RM_CUDA_TRY(cudaStreamCreateWithPriority(&hp, cudaStreamNonBlocking, greatest));
    RM_CUDA_TRY(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, least));
    RM_CUDA_TRY(cudaEventCreateWithFlags(&next_done, cudaEventDisableTiming));
    RM_CUDA_TRY(cudaEventCreateWithFlags(&rest_done, cudaEventDisableTiming));
    RM_CUDA_TRY(cudaEventCreateWithFlags(&entry, cudaEventDisableTiming));
    RM_CUDA_TRY(cudaEventRecord(rest_done, side));  // complete at first, so the first wait passes
    return RM_OK;
  }
  ~F64LookAhead() {
    if (next_done) cudaEventDestroy(next_done);
    if (rest_done) cudaEventDestroy(rest_done);
    if (entry) cudaEventDestroy(entry);
    if (hp) cudaStreamDestroy(hp);
    if (side) cudaStreamDestroy(side);
  }
};
}  // namespace

int getrf_f64(double* w, int64_t ldw, int64_t n64, int64_t* ipiv, int64_t* perm, void* scratch, unsigned* status,
              cudaStream_t caller) {
  if (n64 <= 0) return RM_OK;
  if (n64 > INT32_MAX / 2) return RM_BAD_ARG;
  const int n = (int)n64;
  if (n <= kClusterLuMax && cluster_lu_ok()) return launch_cluster_lu(w, ldw, n, ipiv, perm, caller);
  double* linv = reinterpret_cast<double*>(scratch);
  iota_kernel<<<std::max(1, std::min(n / 256 + 1, 1024)), 256, 0, caller>>>(perm, n);
  RM_LAUNCHED();
  // Look-ahead (n >= 1024): each trailing update does the next block's 128 columns first, on
  // the chain's stream; the rest runs on a side stream while the next block's leaves factor.
  // Only the block's row swaps on the columns right of it wait for that rest (it writes them).
  RM_TRY(smem_attribute(invert_unit_lower_f64_kernel, kInv64Smem));
  F64LookAhead la;
  const bool ahead = n >= 1024;
  cudaStream_t stream = caller;
  if (ahead) {
    RM_TRY(la.open());
    RM_CUDA_TRY(cudaEventRecord(la.entry, caller));
    RM_CUDA_TRY(cudaStreamWaitEvent(la.hp, la.entry, 0));
    stream = la.hp;
  }
  for (int J0 = 0; J0 < n; J0 += kOuter) {
    const int nb = std::min(kOuter, n - J0);
    const int J1 = J0 + nb;
    for (int j0 = J0; j0 < J1; j0 += kLeaf) {
      const int jb = std::min(kLeaf, J1 - j0);
      RM_TRY(launch_panel<double>(w, ldw, n, j0, jb, ipiv, stream));
      // the leaf's swaps on the block's other columns; solve for its rows of later columns
      RM_TRY(launch_swap<double>(w, ldw, j0, jb, ipiv, J0, j0, j0 + jb, J1, j0 + jb, J1, nullptr, stream));
      if (j0 + jb < J1 && j0 + jb < n) {
        const int64_t rows = n - (j0 + jb), cols = J1 - (j0 + jb);
        RM_TRY(dgemm_device(false, false, rows, cols, jb, -1.0, w + (int64_t)(j0 + jb) * ldw + j0, ldw,
                            w + (int64_t)j0 * ldw + j0 + jb, ldw, 1.0, w + (int64_t)(j0 + jb) * ldw + j0 + jb, ldw,
                            status, stream));
      }
    }
    // the block's swaps on every other column, and the row permutation (after the rest of the
    // last trailing update, which writes the columns right of this block)
    if (ahead && J0 > 0) RM_CUDA_TRY(cudaStreamWaitEvent(stream, la.rest_done, 0));
    RM_TRY(launch_swap<double>(w, ldw, J0, nb, ipiv, 0, J0, J1, n, 0, 0, perm, stream));
    if (J1 < n) {
      RM_CUDA_TRY(launch_dependent(invert_unit_lower_f64_kernel, dim3(kOuter / kLeaf), dim3(256), kInv64Smem, stream,
                                   (const double*)w, ldw, J0, nb, linv));
      note_launch();
      double* a12 = w + (int64_t)J0 * ldw + J1;
      RM_TRY(dgemm_device(false, false, nb, n - J1, nb, 1.0, linv, kOuter, a12, ldw, 0.0, a12, ldw, status, stream,
                          /*force_wide_m=*/true));
      const double* l21 = w + (int64_t)J1 * ldw + J0;
      double* a22 = w + (int64_t)J1 * ldw + J1;
      const int rest = n - J1;
      if (!ahead) {
        RM_TRY(dgemm_device(false, false, rest, rest, nb, -1.0, l21, ldw, a12, ldw, 1.0, a22, ldw, status, stream));
        continue;
      }
      const int nn = std::min(kOuter, rest);
      RM_TRY(dgemm_device(false, false, rest, nn, nb, -1.0, l21, ldw, a12, ldw, 1.0, a22, ldw, status, stream));
      if (rest > nn) {
        RM_CUDA_TRY(cudaEventRecord(la.next_done, stream));
        RM_CUDA_TRY(cudaStreamWaitEvent(la.side, la.next_done, 0));
        RM_TRY(dgemm_device(false, false, rest, rest - nn, nb, -1.0, l21, ldw, a12 + nn, ldw, 1.0, a22 + nn, ldw, status,
                            la.side));
        RM_CUDA_TRY(cudaEventRecord(la.rest_done, la.side));
      }
    }
  }
  if (ahead) {
    RM_CUDA_TRY(cudaStreamWaitEvent(stream, la.rest_done, 0));
    RM_CUDA_TRY(cudaEventRecord(la.entry, stream));  // the caller's stream continues after both
    RM_CUDA_TRY(cudaStreamWaitEvent(caller, la.entry, 0));
  }
  return RM_OK;
}

// ------------------------------------------------------------------ load / store / regular

__global__ void load_matrix_kernel(const double* __restrict__ a, int64_t lda, double* __restrict__ w, int64_t ldw,
                                   int64_t n, double* amax) {
  double top = 0.0;
  const int64_t total = n * ldw;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / ldw, j = e - i * ldw;
    double v = 0.0;
    if (j < n) {
      v = a[i * lda + j];
      const double m = fabs(v);
      if (m > top) top = m;
    }
    w[e] = v;
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) top = fmax(top, __shfl_xor_sync(0xffffffffu, top, off));
  if ((threadIdx.x & 31) == 0 && top > 0.0)  // non-negative doubles order like their bits
    atomicMax(reinterpret_cast<unsigned long long*>(amax), (unsigned long long)__double_as_longlong(top));
}

int load_matrix_f64(const double* a, int64_t lda, double* w, int64_t ldw, int64_t n, double* amax,
                    cudaStream_t stream) {
  RM_CUDA_TRY(cudaMemsetAsync(amax, 0, sizeof(double), stream));
  if (n == 0) return RM_OK;
  const int64_t total = n * ldw;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 8 * device_sm_count());
  load_matrix_kernel<<<blocks, 256, 0, stream>>>(a, lda, w, ldw, n, amax);
  RM_LAUNCHED();
  return RM_OK;
}

// factors[j*n + i] = W[i][j]: a 32x32-tiled transpose through shared memory
__global__ void store_factors_kernel(const double* __restrict__ w, int64_t ldw, int64_t n, double* __restrict__ f) {
  __shared__ double tile[32][33];
  const int64_t i0 = (int64_t)blockIdx.y * 32, j0 = (int64_t)blockIdx.x * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t i = i0 + r, j = j0 + threadIdx.x;
    if (i < n && j < n) tile[r][threadIdx.x] = w[i * ldw + j];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t j = j0 + r, i = i0 + threadIdx.x;
    if (i < n && j < n) f[j * n + i] = tile[threadIdx.x][r];
  }
}

int store_factors_f64(const double* w, int64_t ldw, int64_t n, double* factors, cudaStream_t stream) {
  if (n == 0) return RM_OK;
  dim3 grid((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32));
  store_factors_kernel<<<grid, dim3(32, 8), 0, stream>>>(w, ldw, n, factors);
  RM_LAUNCHED();
  return RM_OK;
}

__global__ void regular_kernel(const double* __restrict__ w, int64_t ldw, int64_t n, const double* amax,
                               int32_t* flag) {
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  const double negligible = 2.220446049250313e-16 * (double)n * *amax;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
    if (fabs(w[i * ldw + i]) <= negligible) bad = 1;  // NaN compares false: a NaN pivot is regular
  __syncthreads();
  if (threadIdx.x == 0) *flag = (n > 0 && !bad) ? 1 : 0;
}

int regular_flag_f64(const double* w, int64_t ldw, int64_t n, const double* amax, int32_t* flag,
                     cudaStream_t stream) {
  regular_kernel<<<1, 1024, 0, stream>>>(w, ldw, n, amax, flag);
  RM_LAUNCHED();
  return RM_OK;
}

}  // namespace rm
