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
//   lpp_panel_kernel : GEPP of the T x 128 panel among its T rows, in 16-column leaves with
//                      a shared-memory block update between leaves, and the panel's row
//                      permutation
//   lpp_post_kernel  : L11^-1 and (U11^-1)^T (a 32-column block per CTA), beside the
//                      permutation of the columns right of the panel and A12^T into
//                      a buffer, and the global permutation
//   lpp_apply_kernel : the permutation of the columns left of the panel (off the critical
//                      path: nothing reads them again during the factorization)
//   sgemm_tc_pair    : U12^T = A12^T (L11^-1)^T, written both to a buffer and over A12, and
//                      L21 = A21 U11^-1 for the rows below the panel, in place (one launch)
//   sgemm_tc         : A22 -= L21 U12
// All products are 3xTF32 (float32-level) on tcgen05 with TMEM accumulators. Along this chain
// each kernel is a programmatic dependent of the one before it (its launch and set-up overlap
// that kernel's end; it reads nothing of it before griddepcontrol.wait).
#include <climits>

#include "rm_internal.h"

namespace rm {

constexpr int kLppCols = 128;  // panel width (the trailing update's rank)
constexpr int kLppRows = 256;  // rows a panel's pivots are chosen among
constexpr int kLppLeaf = 16;
constexpr int kLppThreads = 256;  // a thread per row
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
struct alignas(16) LppSlot {
  float row[kLppLeaf];  // a warp's candidate pivot row (its current leaf columns)
  int idx;              // its row
  float rcp;            // 1 / pivot
  int pad[2];
};
static_assert(kLppThreads == 256, "the pivot search reduces 8 warp posts");

// |v| as an unsigned key ordered like the magnitudes: 0 is no candidate, 1 a NaN (never chosen
// over a number), otherwise the float's bits + 2 (non-negative floats order like their bits).
__device__ __forceinline__ unsigned pivot_key(float v) {
  const float a = fabsf(v);
  return a != a ? 1u : __float_as_uint(a) + 2u;
}

// Factors the T x nb panel A[j0.., j0..] (T <= 256, nb <= 128) with partial pivoting among
// its T rows. Thread r owns row r. Pivoting is implicit: rows stay where they are and a row
// chosen as a pivot leaves the candidates; the panel is written back in pivot order at the
// end. Within a 16-column leaf each thread keeps its row's leaf in registers, and each
// column costs one barrier: every warp posts its best candidate (redux.sync max of the keys,
// the lowest lane holding it by ballot), that candidate's row and reciprocal, and after the
// barrier every thread reads the 8 keys (two 16-byte loads) and picks the winner by a
// three-level compare tree in registers (largest |pivot|, lowest warp and so first row on
// ties, NaN never chosen over a number), then reads the pivot row from its post (two
// buffers of posts alternate between columns, so a column's posts are never overwritten
// while read).
// After a leaf: U12 of its pivot rows (unit-lower solve, a column per thread) and the block
// update of the later columns of the rows still unchosen. Then the pivot rows come first in
// choice order and the others follow in their original order: plocal[i] is the panel row
// that row i came from. A zero pivot sets RM_DEV_NAN and leaves its column unreduced.
__global__ void __launch_bounds__(kLppThreads, 1) lpp_panel_kernel(float* __restrict__ a, int64_t lda, int j0, int nb,
                                                                int T, int* __restrict__ plocal, unsigned* status) {
  extern __shared__ float sm[];
  float(*P)[kLppStride] = reinterpret_cast<float(*)[kLppStride]>(sm);
  // the leaf's U12, transposed (column j's 16 values contiguous)
  float(*UbT)[kLppLeaf + 4] = reinterpret_cast<float(*)[kLppLeaf + 4]>(sm + kLppRows * kLppStride);
  __shared__ LppSlot slot[2][kLppThreads / 32];
  __shared__ __align__(16) unsigned skey[2][kLppThreads / 32];  // the posts' keys
  __shared__ __align__(16) float Lp[kLppLeaf][kLppLeaf + 4];
  __shared__ int piv_s[kLppCols];
  __shared__ int order_s[kLppRows];
  __shared__ int wcount[kLppThreads / 32];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r = tid;
  float* blk = a + (int64_t)j0 * lda + j0;
  griddep_launch_dependents();
  griddep_wait();  // the update of these columns has completed
  if (nb == kLppCols) {
    // asynchronous 4-byte copies, every one of a thread's in flight at once: a warp per row,
    // lane l the row's floats 4l..4l+3 (each warp reads 512 contiguous bytes per row), in an
    // order rotated by l / 8 so that the shared-memory writes of a warp hit 32 distinct banks
    const int rot = lane >> 3;
    for (int rr = warp; rr < T; rr += kLppThreads / 32)
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int c = 4 * lane + ((t + rot) & 3);
        cp_async4(&P[rr][c], blk + (int64_t)rr * lda + c);
      }
    cp_async_wait_all();
  } else {
    for (int e = tid; e < T * nb; e += kLppThreads) {
      const int rr = e / nb, c = e % nb;
      P[rr][c] = blk[(int64_t)rr * lda + c];
    }
  }
  bool active = r < T;
  __syncthreads();
  for (int L = 0; L * kLppLeaf < nb; ++L) {
    const int c0 = L * kLppLeaf;
    const bool was_active = active;
    float p[kLppLeaf];
#pragma unroll
    for (int i = 0; i < kLppLeaf; ++i) p[i] = (active && c0 + i < nb) ? P[r][c0 + i] : 0.0f;
#pragma unroll
    for (int c = 0; c < kLppLeaf; ++c) {
      if (c0 + c >= nb) continue;  // the last panel may be narrower than a leaf
      LppSlot* sl = &slot[c & 1][0];
      // the warp's candidate: the largest key (redux), the lowest lane holding it (ballot);
      // every lane's reciprocal is taken while the reduction runs, the winner posts its own
      const unsigned key = active ? pivot_key(p[c]) : 0u;
      const float myrcp = __frcp_rn(p[c]);
      const unsigned wmax = __reduce_max_sync(0xffffffffu, key);
      const int wl = __ffs(__ballot_sync(0xffffffffu, key == wmax)) - 1;
      if (lane == wl) {
        float4* dst = reinterpret_cast<float4*>(sl[warp].row);
#pragma unroll
        for (int i = 0; i < kLppLeaf / 4; ++i) dst[i] = make_float4(p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]);
        *reinterpret_cast<int2*>(&sl[warp].idx) = make_int2(r, __float_as_int(myrcp));
        skey[c & 1][warp] = wmax;
      }
      __syncthreads();
      // the winning post: the largest key, the lowest warp (so the lowest row) among equals
      int bw;
      {
        const uint4 k0 = *reinterpret_cast<const uint4*>(&skey[c & 1][0]);
        const uint4 k1 = *reinterpret_cast<const uint4*>(&skey[c & 1][4]);
        const bool s0 = k0.x >= k0.y, s1 = k0.z >= k0.w, s2 = k1.x >= k1.y, s3 = k1.z >= k1.w;
        const unsigned a0 = s0 ? k0.x : k0.y, a1 = s1 ? k0.z : k0.w, a2 = s2 ? k1.x : k1.y, a3 = s3 ? k1.z : k1.w;
        const int w0 = s0 ? 0 : 1, w1 = s1 ? 2 : 3, w2 = s2 ? 4 : 5, w3 = s3 ? 6 : 7;
        const bool t0 = a0 >= a1, t1 = a2 >= a3;
        const unsigned b0 = t0 ? a0 : a1, b1 = t1 ? a2 : a3;
        const int v0 = t0 ? w0 : w1, v1 = t1 ? w2 : w3;
        bw = b0 >= b1 ? v0 : v1;
      }
      const int2 meta = *reinterpret_cast<const int2*>(&sl[bw].idx);
      const int bi = meta.x;
      const float prcp = __int_as_float(meta.y);
      // the pivot row, as 16-byte reads of the winning post
      float prow[kLppLeaf];
      {
        const float4* src = reinterpret_cast<const float4*>(sl[bw].row);
#pragma unroll
        for (int i = c / 4; i < kLppLeaf / 4; ++i) {
          const float4 v4 = src[i];
          prow[4 * i] = v4.x, prow[4 * i + 1] = v4.y, prow[4 * i + 2] = v4.z, prow[4 * i + 3] = v4.w;
        }
      }
      const float piv = prow[c];
      if (warp == (bi >> 5)) {  // warp-uniform: only the pivot's warp records it
        if (r == bi) {
          active = false;
          piv_s[c0 + c] = r;
          float4* dst = reinterpret_cast<float4*>(Lp[c]);
#pragma unroll
          for (int i = 0; i < kLppLeaf / 4; ++i) dst[i] = make_float4(p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]);
        }
      }
      if (active && piv != 0.0f) {
        const float l = p[c] * prcp;
        p[c] = l;
#pragma unroll
        for (int i = c + 1; i < kLppLeaf; ++i) p[i] = fmaf(-l, prow[i], p[i]);
      }
      if (piv == 0.0f && tid == 0) flag_error(status, RM_DEV_NAN);
    }
    if (was_active) {
#pragma unroll
      for (int i = 0; i < kLppLeaf; ++i)
        if (c0 + i < nb) P[r][c0 + i] = p[i];
    }
    __syncthreads();
    const int rc0 = c0 + kLppLeaf, rcols = nb - rc0;
    if (rcols <= 0) break;
    // U12 of the leaf's pivot rows: u = Lp^-1 (their later columns), a column per thread
    if (tid < rcols) {  // rcols < 128 <= threads
      const int j = tid;
      float u[kLppLeaf];
#pragma unroll
      for (int c = 0; c < kLppLeaf; ++c) u[c] = P[piv_s[c0 + c]][rc0 + j];
#pragma unroll
      for (int c = 1; c < kLppLeaf; ++c)
#pragma unroll
        for (int q = 0; q < c; ++q) u[c] = fmaf(-Lp[c][q], u[q], u[c]);
#pragma unroll
      for (int c = 0; c < kLppLeaf; ++c) {
        P[piv_s[c0 + c]][rc0 + j] = u[c];
        UbT[j][c] = u[c];
      }
    }
    __syncthreads();
    // the rows still unchosen: later columns -= L(row, leaf) U12
    if (active) {
      for (int j = 0; j < rcols; ++j) {
        float a0 = P[r][rc0 + j], a1 = 0.f, a2 = 0.f, a3 = 0.f;  // four chains
        const float4* ub = reinterpret_cast<const float4*>(&UbT[j][0]);
#pragma unroll
        for (int q = 0; q < kLppLeaf / 4; ++q) {
          const float4 u4 = ub[q];
          a0 = fmaf(-p[4 * q], u4.x, a0);
          a1 = fmaf(-p[4 * q + 1], u4.y, a1);
          a2 = fmaf(-p[4 * q + 2], u4.z, a2);
          a3 = fmaf(-p[4 * q + 3], u4.w, a3);
        }
        P[r][rc0 + j] = (a0 + a1) + (a2 + a3);
      }
    }
    __syncthreads();
  }

  // the row order: pivot rows in choice order, then the unchosen rows in their own order
  const bool rest = active;  // r < T and never chosen
  const unsigned msk = __ballot_sync(0xffffffffu, rest);
  if (lane == 0) wcount[warp] = __popc(msk);
  if (tid < nb) order_s[tid] = piv_s[tid];
  __syncthreads();
  if (rest) {
    int before = nb;
    for (int w = 0; w < warp; ++w) before += wcount[w];
    order_s[before + __popc(msk & ((1u << lane) - 1u))] = r;
  }
  __syncthreads();
  if (tid < T) plocal[tid] = order_s[tid];
  // the panel back in that order: a warp per row, lanes along it
  for (int rr = warp; rr < T; rr += kLppThreads / 32) {
    const float* src = P[order_s[rr]];
    float* dst = blk + (int64_t)rr * lda;
    for (int c = lane; c < nb; c += 32) dst[c] = src[c];
  }
}

constexpr size_t kLppSmem = ((size_t)kLppRows * kLppStride + (size_t)kLppCols * (kLppLeaf + 4)) * sizeof(float);

// ------------------------------------------------------------------ the diagonal block's inverses
// X = M^-1 for the lower triangles M = L11 (unit; m = 0) and M = U11^T (m = 1) of the panel's
// factored diagonal block (rows j0.. of a in pivot order, nb x nb; identity beyond nb). CTA
// (m, a) builds X's 32-column block a: X_aa = M_aa^-1, then block row by block row
// X_ba = -M_bb^-1 sum_{c=a..b-1} M_bc X_ca. The diagonal blocks' inverses come first, a warp
// each, a lane per column (forward substitution). Outputs: linv = L11^-1 and
// uinvt = (U11^-1)^T (ld 128), and when dblk is not NULL L11^-1 and U11^-1 row-major as the
// triangular solves' table entries [0] and [1] of this block.
constexpr int kInvStride = kLppCols + 1;
constexpr size_t kInvSmem = ((size_t)kLppCols * kInvStride + (4 * 32 + kLppCols + 32) * 33) * sizeof(float);

__device__ __forceinline__ void lpp_inverse_block(float* sm, int bid, const float* __restrict__ a, int64_t lda,
                                                  int j0, int nb, float* __restrict__ linv, float* __restrict__ uinvt,
                                                  float* __restrict__ dblk) {
  float(*M)[kInvStride] = reinterpret_cast<float(*)[kInvStride]>(sm);        // rows, columns >= a0 used
  float(*Y)[33] = reinterpret_cast<float(*)[33]>(sm + kLppCols * kInvStride);  // M_bb^-1 at rows 32 b
  float(*X)[33] = Y + 4 * 32;                                                  // the column block
  float(*Tq)[33] = X + kLppCols;                                               // 32 x 33
  const int m = bid >> 2, ab = bid & 3, a0 = 32 * ab;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const float* blk = a + (int64_t)j0 * lda + j0;
  // M from row a0 on: a warp per stored row, lanes along it
  if (nb == kLppCols) {
    // asynchronous 4-byte copies, all in flight at once; lane l copies floats 4l..4l+3 of a row
    // in an order rotated by l / 8, so that the shared-memory writes of a warp hit distinct banks
    const int rot = lane >> 3;
    for (int i = a0 + warp; i < kLppCols; i += 8)
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int k = 4 * lane + ((t + rot) & 3);
        cp_async4(m == 0 ? &M[i][k] : &M[k][i], blk + (int64_t)i * lda + k);
      }
    cp_async_wait_all();
  } else {
    for (int i = a0 + warp; i < kLppCols; i += 8)
      for (int k = a0 + lane; k < kLppCols; k += 32) {
        const float v = (i < nb && k < nb) ? blk[(int64_t)i * lda + k] : (i == k ? 1.0f : 0.0f);
        if (m == 0) M[i][k] = v;
        else M[k][i] = v;
      }
  }
  __syncthreads();
  if (warp < 4 - ab) {  // Y_b = M_bb^-1, b = ab + warp
    const int b0 = a0 + 32 * warp;
    float x[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      float acc = i == lane ? 1.0f : 0.0f;
#pragma unroll
      for (int k2 = 0; k2 < i; ++k2) acc = fmaf(-M[b0 + i][b0 + k2], x[k2], acc);
      x[i] = i < lane ? 0.0f : (m == 0 ? acc : acc / M[b0 + i][b0 + i]);
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) Y[b0 + i][lane] = x[i];
  }
  __syncthreads();
  for (int e = tid; e < 32 * 32; e += 256) X[a0 + (e >> 5)][e & 31] = Y[a0 + (e >> 5)][e & 31];
  __syncthreads();
  const int ti = tid >> 4, tj = tid & 15;  // rows ti, ti + 16 and columns tj, tj + 16 of a 32 x 32 block
  for (int b = ab + 1; b < 4; ++b) {
    const int r0 = 32 * b + ti, r1 = r0 + 16;
    float t00 = 0.f, t01 = 0.f, t10 = 0.f, t11 = 0.f;
#pragma unroll 4
    for (int k = a0; k < 32 * b; ++k) {
      const float m0 = M[r0][k], m1 = M[r1][k], x0 = X[k][tj], x1 = X[k][tj + 16];
      t00 = fmaf(m0, x0, t00), t01 = fmaf(m0, x1, t01), t10 = fmaf(m1, x0, t10), t11 = fmaf(m1, x1, t11);
    }
    Tq[ti][tj] = t00, Tq[ti][tj + 16] = t01, Tq[ti + 16][tj] = t10, Tq[ti + 16][tj + 16] = t11;
    __syncthreads();
    t00 = t01 = t10 = t11 = 0.f;
#pragma unroll 4
    for (int k2 = 0; k2 < 32; ++k2) {
      const float y0 = Y[r0][k2], y1 = Y[r1][k2], u0 = Tq[k2][tj], u1 = Tq[k2][tj + 16];
      t00 = fmaf(y0, u0, t00), t01 = fmaf(y0, u1, t01), t10 = fmaf(y1, u0, t10), t11 = fmaf(y1, u1, t11);
    }
    X[r0][tj] = -t00, X[r0][tj + 16] = -t01, X[r1][tj] = -t10, X[r1][tj + 16] = -t11;
    __syncthreads();
  }
  // rows above a0 are zero; X is lower triangular within block a (zeros above the diagonal)
  float* out = m == 0 ? linv : uinvt;
  for (int rr = warp; rr < kLppCols; rr += 8) {
    const float v = rr >= a0 ? X[rr][lane] : 0.0f;
    out[rr * kLppCols + a0 + lane] = v;
    if (dblk && m == 0) dblk[rr * kLppCols + a0 + lane] = v;
  }
  if (dblk && m == 1)  // U11^-1 = X^T row-major: row a0 + c holds X's column c, lanes along it
    for (int c = warp; c < 32; c += 8)
      for (int rr = lane; rr < kLppCols; rr += 32)
        dblk[kLppCols * kLppCols + (a0 + c) * kLppCols + rr] = rr >= a0 ? X[rr][c] : 0.0f;
}

// ------------------------------------------------------------------ the panel's row permutation
constexpr int kApplyCols = 32;
constexpr size_t kApplySmem = (size_t)kLppRows * (kApplyCols + 1) * sizeof(float) + kLppRows * sizeof(int);

// Rows j0..j0+T of a band of columns take the panel's permutation (new row i = old row
// plocal[i]): the columns [j1, n) when right, else [0, j0), 32 columns per CTA. For the right
// band the first nb new rows also go, transposed, to a12t (ld 128), and block 0 permutes
// perm[j0..j0+T). A full 32-column chunk moves as 16-byte accesses, eight per thread in flight:
// thread t covers rows t/8 + 32u and the chunk's float4 t%8, so the shared-memory stores of a
// warp (4 rows x 8 float4 at stride 33) hit 32 distinct banks.
__device__ __forceinline__ void lpp_apply_band(float* sm, int bid, float* __restrict__ a, int64_t lda, int n, int j0,
                                               int j1, int T, const int* __restrict__ plocal,
                                               float* __restrict__ a12t, int* __restrict__ perm, bool right) {
  float(*buf)[kApplyCols + 1] = reinterpret_cast<float(*)[kApplyCols + 1]>(sm);
  int* pl = reinterpret_cast<int*>(sm + kLppRows * (kApplyCols + 1));
  const int tid = threadIdx.x;
  if (tid < T) pl[tid] = plocal[tid];
  __syncthreads();
  const int c0 = right ? j1 + bid * kApplyCols : bid * kApplyCols;
  const int c1 = min(c0 + kApplyCols, right ? n : j0);
  const int w = c1 - c0;
  if (w == kApplyCols) {
    const int q = tid & 7, rb = tid >> 3;
    float4 v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int r = rb + 32 * u;
      v[u] = r < T ? *reinterpret_cast<const float4*>(a + (int64_t)(j0 + pl[r]) * lda + c0 + 4 * q)
                   : make_float4(0, 0, 0, 0);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int r = rb + 32 * u;
      if (r < T) buf[r][4 * q] = v[u].x, buf[r][4 * q + 1] = v[u].y, buf[r][4 * q + 2] = v[u].z, buf[r][4 * q + 3] = v[u].w;
    }
    __syncthreads();  // every source row is read before any is overwritten
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int r = rb + 32 * u;
      if (r < T && pl[r] != r) *reinterpret_cast<float4*>(a + (int64_t)(j0 + r) * lda + c0 + 4 * q) = v[u];
    }
  } else if (w > 0) {
    for (int e = tid; e < T * kApplyCols; e += 256) {
      const int r = e / kApplyCols, c = e % kApplyCols;
      if (c < w) buf[r][c] = a[(int64_t)(j0 + pl[r]) * lda + c0 + c];
    }
    __syncthreads();
    for (int e = tid; e < T * kApplyCols; e += 256) {
      const int r = e / kApplyCols, c = e % kApplyCols;
      if (c < w && pl[r] != r) a[(int64_t)(j0 + r) * lda + c0 + c] = buf[r][c];
    }
  }
  if (right) {
    __syncthreads();
    const int nb = j1 - j0;
    for (int e = tid; e < nb * kApplyCols; e += 256) {
      const int c = e / nb, r = e % nb;  // consecutive threads: consecutive rows of a12t's row
      if (c < w) a12t[(int64_t)(c0 - j1 + c) * kLppCols + r] = buf[r][c];
    }
    if (bid == 0) {
      const int v = tid < T ? perm[j0 + pl[tid]] : 0;
      __syncthreads();
      if (tid < T) perm[j0 + tid] = v;
    }
  }
}

// The left band of a panel's row permutation, 32 columns per CTA.
__global__ void __launch_bounds__(256) lpp_apply_kernel(float* __restrict__ a, int64_t lda, int n, int j0, int j1,
                                                        int T, const int* __restrict__ plocal) {
  extern __shared__ float sm[];
  lpp_apply_band(sm, blockIdx.x, a, lda, n, j0, j1, T, plocal, nullptr, nullptr, false);
}

// What follows a panel on the critical path, in one launch: CTAs 0..7 build the diagonal
// block's inverses, the others permute the right band (32 columns each) and fill a12t.
__global__ void __launch_bounds__(256) lpp_post_kernel(float* __restrict__ a, int64_t lda, int n, int j0, int j1,
                                                       int T, const int* __restrict__ plocal, float* __restrict__ a12t,
                                                       int* __restrict__ perm, float* __restrict__ linv,
                                                       float* __restrict__ uinvt, float* __restrict__ dblk) {
  extern __shared__ float sm[];
  griddep_launch_dependents();
  griddep_wait();  // the panel has completed
  if (blockIdx.x < 8) lpp_inverse_block(sm, blockIdx.x, a, lda, j0, j1 - j0, linv, uinvt, dblk);
  else lpp_apply_band(sm, blockIdx.x - 8, a, lda, n, j0, j1, T, plocal, a12t, perm, true);
}

__global__ void iota32_kernel(int* p, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = (int)i;
}

// SMs the look-ahead leaves free of the trailing update: the panel's and the inverses' CTAs
constexpr int kLookAheadSms = 8;

// The streams and events of the look-ahead; released when the factorization returns (work
// still queued on the other streams completes first).
struct LookAhead {
  cudaStream_t side = nullptr, aux = nullptr;
  cudaEvent_t next_done = nullptr, rest_done = nullptr, panel_done = nullptr, left_done = nullptr;
  int open() {
    RM_CUDA_TRY(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    RM_CUDA_TRY(cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking));
    RM_CUDA_TRY(cudaEventCreateWithFlags(&next_done, cudaEventDisableTiming));
    RM_CUDA_TRY(cudaEventCreateWithFlags(&rest_done, cudaEventDisableTiming));
    RM_CUDA_TRY(cudaEventCreateWithFlags(&panel_done, cudaEventDisableTiming));
    RM_CUDA_TRY(cudaEventCreateWithFlags(&left_done, cudaEventDisableTiming));
    // rest_done starts out complete, so the first wait on it passes
    RM_CUDA_TRY(cudaEventRecord(rest_done, side));
    return RM_OK;
  }
  ~LookAhead() {
    if (next_done) cudaEventDestroy(next_done);
    if (rest_done) cudaEventDestroy(rest_done);
    if (panel_done) cudaEventDestroy(panel_done);
    if (left_done) cudaEventDestroy(left_done);
    if (side) cudaStreamDestroy(side);
    if (aux) cudaStreamDestroy(aux);
  }
};

size_t getrf_lpp_f32_scratch_bytes(int64_t n) {
  // linv, uinvt, a12t, u12t, the low parts of L21 and U12^T; each panel's row permutation
  // (256 ints per panel)
  return (2 * (size_t)kLppCols * kLppCols + 4 * (size_t)n * kLppCols) * sizeof(float) +
         (size_t)((n + kLppCols - 1) / kLppCols) * kLppRows * sizeof(int) + 2048;
}

int getrf_lpp_f32(float* a, int64_t lda, int64_t n, int* perm, void* scratch, unsigned* status, cudaStream_t stream,
                  float* dinv) {
  if (n <= 0) return RM_OK;
  if (n > INT32_MAX / 2) return RM_BAD_ARG;
  float* linv = reinterpret_cast<float*>(scratch);
  float* uinvt = linv + kLppCols * kLppCols;
  float* a12t = uinvt + kLppCols * kLppCols;   // rest x 128: A12^T
  float* u12t = a12t + (size_t)n * kLppCols;   // rest x 128: U12^T
  float* l21lo = u12t + (size_t)n * kLppCols;  // rest x 128: low parts of L21 (ld 128) ...
  float* u12lo = l21lo + (size_t)n * kLppCols;  // ... and of U12^T, for the trailing update
  int* plocal = reinterpret_cast<int*>(u12lo + (size_t)n * kLppCols);
  RM_TRY(smem_attribute(lpp_panel_kernel, kLppSmem));
  RM_TRY(smem_attribute(lpp_post_kernel, kInvSmem));
  iota32_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 1024), 256, 0, stream>>>(perm, n);
  RM_LAUNCHED();
  // Look-ahead: the next panel's 128 columns of each trailing update go first, on `stream`;
  // the rest of the update runs on a side stream on all SMs but 8 while the next panel (one
  // CTA) factors on the SMs left free. After a panel, one launch builds its inverses (8 CTAs)
  // and permutes the columns to the right of it, while a third stream permutes the columns to
  // its left, which nothing reads again during the factorization.
  LookAhead la;
  const bool ahead = n >= 1024 && device_sm_count() > 2 * kLookAheadSms;
  if (ahead) RM_TRY(la.open());
  const int ni = (int)n;
  for (int J0 = 0; J0 < ni; J0 += kLppCols) {
    const int nb = std::min(kLppCols, ni - J0);
    const int T = std::min(kLppRows, ni - J0);
    const int J1 = J0 + nb;
    const int rest = ni - J1;
    float* dblk = dinv ? dinv + (size_t)(J0 / kLppCols) * kDiagMats * kLppCols * kLppCols : nullptr;
    int* pl = plocal + (size_t)(J0 / kLppCols) * kLppRows;
    RM_CUDA_TRY(launch_dependent(lpp_panel_kernel, dim3(1), dim3(kLppThreads), kLppSmem, stream, a, lda, J0, nb, T, pl,
                                 status));
    RM_LAUNCHED();
    const int left_chunks = (J0 + kApplyCols - 1) / kApplyCols, right_chunks = (rest + kApplyCols - 1) / kApplyCols;
    // the left band: on the third stream once the panel is done (in stream order without look-ahead)
    cudaStream_t left_stream = stream;
    if (ahead) {
      RM_CUDA_TRY(cudaEventRecord(la.panel_done, stream));
      RM_CUDA_TRY(cudaStreamWaitEvent(la.aux, la.panel_done, 0));
      left_stream = la.aux;
    }
    if (left_chunks > 0) {
      lpp_apply_kernel<<<left_chunks, 256, kApplySmem, left_stream>>>(a, lda, ni, J0, J1, T, pl);
      RM_LAUNCHED();
    }
    // the inverses and the right band, after the trailing update that writes the right band
    if (ahead && J0 > 0) RM_CUDA_TRY(cudaStreamWaitEvent(stream, la.rest_done, 0));
    RM_CUDA_TRY(launch_dependent(lpp_post_kernel, dim3(8 + std::max(right_chunks, 1)), dim3(256), kInvSmem, stream, a, lda,
                                 ni, J0, J1, T, (const int*)pl, a12t, perm, linv, uinvt, dblk));
    RM_LAUNCHED();
    if (rest == 0) break;
    // in one launch: U12^T = A12^T (L11^-1)^T, also written transposed over A12, and
    // L21 = A21 U11^-1 for the rows below the panel (the panel's own rows are done), in place
    float* a12 = a + (int64_t)J0 * lda + J1;
    const int below = ni - (J0 + T);
    float* a21b = a + (int64_t)(J0 + T) * lda + J0;
    const SgemmOperands u12{rest, a12t, kLppCols, linv, kLppCols, u12t, kLppCols, a12, lda};
    const SgemmOperands l21b{std::max(below, 0), a21b, lda, uinvt, kLppCols, a21b, lda, nullptr, 0};
    RM_TRY(sgemm_tc_pair(3, u12, l21b, nb, nb, 1.0f, 0.0f, status, stream));
    // A22 -= L21 U12: the next panel's columns, then the rest
    const float* l21 = a + (int64_t)J1 * lda + J0;
    float* a22 = a + (int64_t)J1 * lda + J1;
    if (!ahead) {
      RM_TRY(sgemm_tc(3, rest, rest, nb, -1.0f, l21, lda, u12t, kLppCols, 1.0f, a22, lda, status, stream));
      continue;
    }
    const int nn = std::min(kLppCols, rest);
    RM_TRY(sgemm_tc(3, rest, nn, nb, -1.0f, l21, lda, u12t, kLppCols, 1.0f, a22, lda, status, stream));
    if (rest > nn) {
      RM_CUDA_TRY(cudaEventRecord(la.next_done, stream));
      RM_CUDA_TRY(cudaStreamWaitEvent(la.side, la.next_done, 0));
      // the panels' low parts once, then the update loads them beside the panels
      RM_TRY(split_lo_f32(l21, lda, rest, nb, l21lo, kLppCols, la.side));
      RM_TRY(split_lo_f32(u12t + (size_t)nn * kLppCols, kLppCols, rest - nn, nb, u12lo, kLppCols, la.side));
      RM_TRY(sgemm_tc_lo(rest, rest - nn, nb, -1.0f, l21, lda, l21lo, kLppCols, u12t + (size_t)nn * kLppCols, kLppCols,
                         u12lo, kLppCols, 1.0f, a22 + nn, lda, status, la.side, device_sm_count() - kLookAheadSms));
      RM_CUDA_TRY(cudaEventRecord(la.rest_done, la.side));
    }
  }
  if (ahead) {
    RM_CUDA_TRY(cudaStreamWaitEvent(stream, la.rest_done, 0));
    RM_CUDA_TRY(cudaEventRecord(la.left_done, la.aux));  // the last left band
    RM_CUDA_TRY(cudaStreamWaitEvent(stream, la.left_done, 0));
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
