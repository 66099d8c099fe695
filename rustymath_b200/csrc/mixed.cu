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
constexpr int kLppLeaf = 16;
constexpr int kLppThreads = 256;  // a thread per row
constexpr int kLppPRows = 2 * kLppCols;  // rows of the panel buffer (the inverses use its upper half)
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
  unsigned key;         // its |pivot| as an ordered key: bits + 2; 1 for NaN; 0: no candidate
  int idx;              // its row
  float rcp;            // 1 / pivot
  int pad;
};

// |v| as an unsigned key ordered like the magnitudes: 0 is no candidate, 1 a NaN (never chosen
// over a number), otherwise the float's bits + 2 (non-negative floats order like their bits).
__device__ __forceinline__ unsigned pivot_key(float v) {
  const float a = fabsf(v);
  return a != a ? 1u : __float_as_uint(a) + 2u;
}

// Factors the T x nb panel A[j0.., j0..] (T <= 256, nb <= 128) with partial pivoting among
// its T rows. Thread r owns row r. Pivoting is implicit: rows stay where they are and a row
// chosen as a pivot leaves the candidates; the panel is written back in pivot order at the
// end. Within a 32-column leaf each thread keeps its row's leaf in registers, and each
// column costs one barrier: every warp posts its best candidate and that candidate's row, and
// after the barrier every thread picks the winner among 8 posts (largest |pivot|, first row
// on ties, NaN never chosen over a number) and reads the pivot row from it (two buffers of
// posts alternate between columns, so a column's posts are never overwritten while read).
// After a leaf: U12 of its pivot rows (unit-lower solve, a column per thread) and the block
// update of the later columns of the rows still unchosen. Then the pivot rows come first in
// choice order and the others follow in their original order: plocal[i] is the panel row
// that row i came from; linv = L11^-1 and uinvt = (U11^-1)^T (ld 128). A zero pivot sets
// RM_DEV_NAN and leaves its column unreduced.
__global__ void __launch_bounds__(kLppThreads, 1) lpp_panel_kernel(float* __restrict__ a, int64_t lda, int j0, int nb,
                                                                int T, float* __restrict__ linv,
                                                                float* __restrict__ uinvt, int* __restrict__ plocal,
                                                                float* __restrict__ dblk, unsigned* status) {
  extern __shared__ float sm[];
  float(*P)[kLppStride] = reinterpret_cast<float(*)[kLppStride]>(sm);
  float(*X)[kLppStride] = reinterpret_cast<float(*)[kLppStride]>(sm + kLppPRows * kLppStride);
  float(*Tm)[33] = reinterpret_cast<float(*)[33]>(sm + (kLppPRows + kLppCols) * kLppStride);  // 96 x 33
  // during the factorization X's space holds the leaf's U12, transposed (column j's 32 values contiguous)
  float(*UbT)[kLppLeaf + 4] = reinterpret_cast<float(*)[kLppLeaf + 4]>(X);
  __shared__ LppSlot slot[2][kLppThreads / 32];
  __shared__ __align__(16) float Lp[kLppLeaf][kLppLeaf + 4];
  __shared__ int piv_s[kLppCols];
  __shared__ int order_s[kLppRows];
  __shared__ int wcount[kLppThreads / 32];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r = tid;
  float* blk = a + (int64_t)j0 * lda + j0;
  for (int e = tid; e < T * nb; e += kLppThreads) {
    const int rr = e / nb, c = e % nb;
    P[rr][c] = blk[(int64_t)rr * lda + c];
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
      // the warp's candidate: the largest key (redux), the lowest lane holding it (ballot)
      const unsigned key = active ? pivot_key(p[c]) : 0u;
      const unsigned wmax = __reduce_max_sync(0xffffffffu, key);
      const int wl = __ffs(__ballot_sync(0xffffffffu, key == wmax)) - 1;
      if (lane == wl) {
        float4* dst = reinterpret_cast<float4*>(sl[warp].row);
#pragma unroll
        for (int i = 0; i < kLppLeaf / 4; ++i) dst[i] = make_float4(p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]);
        sl[warp].key = wmax;
        sl[warp].idx = r;
        sl[warp].rcp = __frcp_rn(p[c]);
      }
      __syncthreads();
      // the winning post: the largest key, the lowest warp (so the lowest row) among equals
      const unsigned kq = lane < kLppThreads / 32 ? sl[lane].key : 0u;
      const unsigned gmax = __reduce_max_sync(0xffffffffu, kq);
      const unsigned gball = __ballot_sync(0xffffffffu, lane < kLppThreads / 32 && kq == gmax);
      const int bw = gball ? __ffs(gball) - 1 : 0;
      const int bi = sl[bw].idx;
      const float prcp = sl[bw].rcp;
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
  // ---- the inverses. D (P's rows 0..127) = the diagonal block in pivot order: L11 below its
  // diagonal (unit), U11 on and above it. XL (X's space) = L11^-1 and XU (P's rows 128..) =
  // (U11^T)^-1 = (U11^-1)^T are both lower triangles, built the same way: the diagonal 32 x 32
  // blocks first (a warp each, a lane per column, zeros above their diagonals), then the
  // blocks below in order of distance b - a = gap: T = sum_{c=a..b-1} M_bc X_ca in Tm,
  // X_ba = -X_bb T, each thread a 2 x 2 piece of every block of a gap. M_0(i, k) = D[i][k],
  // M_1(i, k) = D[k][i].
  float(*D)[kLppStride] = P;
  float(*XL)[kLppStride] = X;
  float(*XU)[kLppStride] = P + kLppCols;
  for (int rr = warp; rr < kLppCols; rr += kLppThreads / 32) {
    const float* src = P[rr < nb ? order_s[rr] : 0];
    for (int c = lane; c < kLppCols; c += 32) X[rr][c] = (rr < nb && c < nb) ? src[c] : (rr == c ? 1.0f : 0.0f);
  }
  __syncthreads();
  for (int rr = warp; rr < kLppCols; rr += kLppThreads / 32)
    for (int c = lane; c < kLppCols; c += 32) D[rr][c] = X[rr][c];
  __syncthreads();
  for (int job = warp; job < 8; job += kLppThreads / 32) {  // 4 blocks of L11, then 4 of U11^T
    const int b0 = (job & 3) * 32;
    float x[32];
    if (job < 4) {
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        float acc = i == lane ? 1.0f : 0.0f;
#pragma unroll
        for (int k2 = 0; k2 < i; ++k2) acc = fmaf(-D[b0 + i][b0 + k2], x[k2], acc);
        x[i] = i < lane ? 0.0f : acc;
      }
#pragma unroll
      for (int i = 0; i < 32; ++i) XL[b0 + i][b0 + lane] = x[i];
    } else {
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        float acc = i == lane ? 1.0f : 0.0f;
#pragma unroll
        for (int k2 = 0; k2 < i; ++k2) acc = fmaf(-D[b0 + k2][b0 + i], x[k2], acc);
        x[i] = i < lane ? 0.0f : acc / D[b0 + i][b0 + i];
      }
#pragma unroll
      for (int i = 0; i < 32; ++i) XU[b0 + i][b0 + lane] = x[i];
    }
  }
  __syncthreads();
  {
    float(*Tq)[33] = Tm;  // up to 3 blocks of 32 x 33
    for (int gap = 1; gap < 4; ++gap)
      for (int m = 0; m < 2; ++m) {
        float(*Xm)[kLppStride] = m == 0 ? XL : XU;
        for (int a = 0; a + gap < 4; ++a) {
          const int b = a + gap;
          for (int tp = tid; tp < 256; tp += kLppThreads) {  // rows ti, ti+16, columns tj, tj+16
            const int ti = tp >> 4, tj = tp & 15;
            float t00 = 0.f, t01 = 0.f, t10 = 0.f, t11 = 0.f;
            const int r0 = 32 * b + ti, r1 = r0 + 16, c0 = 32 * a + tj, c1 = c0 + 16;
            if (m == 0) {
#pragma unroll 4
              for (int k2 = 32 * a; k2 < 32 * b; ++k2) {
                const float m0 = D[r0][k2], m1 = D[r1][k2], x0 = Xm[k2][c0], x1 = Xm[k2][c1];
                t00 = fmaf(m0, x0, t00), t01 = fmaf(m0, x1, t01), t10 = fmaf(m1, x0, t10), t11 = fmaf(m1, x1, t11);
              }
            } else {
#pragma unroll 4
              for (int k2 = 32 * a; k2 < 32 * b; ++k2) {
                const float m0 = D[k2][r0], m1 = D[k2][r1], x0 = Xm[k2][c0], x1 = Xm[k2][c1];
                t00 = fmaf(m0, x0, t00), t01 = fmaf(m0, x1, t01), t10 = fmaf(m1, x0, t10), t11 = fmaf(m1, x1, t11);
              }
            }
            float(*T1)[33] = Tq + 32 * a;
            T1[ti][tj] = t00, T1[ti][tj + 16] = t01, T1[ti + 16][tj] = t10, T1[ti + 16][tj + 16] = t11;
          }
        }
        __syncthreads();
        for (int a = 0; a + gap < 4; ++a) {
          const int b = a + gap;
          float(*T1)[33] = Tq + 32 * a;
          for (int tp = tid; tp < 256; tp += kLppThreads) {
            const int ti = tp >> 4, tj = tp & 15;
            float t00 = 0.f, t01 = 0.f, t10 = 0.f, t11 = 0.f;
            const int r0 = 32 * b + ti, r1 = r0 + 16;
#pragma unroll 4
            for (int k2 = 0; k2 < 32; ++k2) {
              const float x0 = Xm[r0][32 * b + k2], x1 = Xm[r1][32 * b + k2];
              const float u0 = T1[k2][tj], u1 = T1[k2][tj + 16];
              t00 = fmaf(x0, u0, t00), t01 = fmaf(x0, u1, t01), t10 = fmaf(x1, u0, t10), t11 = fmaf(x1, u1, t11);
            }
            Xm[r0][32 * a + tj] = -t00, Xm[r0][32 * a + tj + 16] = -t01, Xm[r1][32 * a + tj] = -t10,
                            Xm[r1][32 * a + tj + 16] = -t11;
          }
        }
        __syncthreads();
      }
  }
  for (int rr = warp; rr < kLppCols; rr += kLppThreads / 32)
    for (int c = lane; c < kLppCols; c += 32) {
      const float l = rr >= c ? XL[rr][c] : 0.0f, u = rr >= c ? XU[rr][c] : 0.0f;
      linv[rr * kLppCols + c] = l;
      uinvt[rr * kLppCols + c] = u;
      if (dblk) dblk[rr * kLppCols + c] = l;  // the triangular solves' table: L11^-1 ...
    }
  if (dblk)  // ... and U11^-1 row-major (XU's transpose), lanes along the output rows
    for (int c = warp; c < kLppCols; c += kLppThreads / 32)
      for (int rr = lane; rr < kLppCols; rr += 32)
        dblk[kLppCols * kLppCols + c * kLppCols + rr] = rr >= c ? XU[rr][c] : 0.0f;
}

constexpr size_t kLppSmem = ((size_t)(kLppPRows + kLppCols) * kLppStride + 3 * 32 * 33) * sizeof(float);

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

// The side stream and the two events of the look-ahead; released when the factorization returns
// (work still queued on the side stream completes first).
struct LookAhead {
  cudaStream_t side = nullptr;
  cudaEvent_t next_done = nullptr, rest_done = nullptr;
  int open() {
    RM_CUDA_TRY(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    RM_CUDA_TRY(cudaEventCreateWithFlags(&next_done, cudaEventDisableTiming));
    RM_CUDA_TRY(cudaEventCreateWithFlags(&rest_done, cudaEventDisableTiming));
    // rest_done starts out complete, so the first wait on it passes
    RM_CUDA_TRY(cudaEventRecord(rest_done, side));
    return RM_OK;
  }
  ~LookAhead() {
    if (next_done) cudaEventDestroy(next_done);
    if (rest_done) cudaEventDestroy(rest_done);
    if (side) cudaStreamDestroy(side);
  }
};

size_t getrf_lpp_f32_scratch_bytes(int64_t n) {
  return (2 * (size_t)kLppCols * kLppCols + 2 * (size_t)n * kLppCols) * sizeof(float) + kLppRows * sizeof(int) +
         2048;
}

int getrf_lpp_f32(float* a, int64_t lda, int64_t n, int* perm, void* scratch, unsigned* status, cudaStream_t stream,
                  float* dinv) {
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
  // Look-ahead: the next panel's 128 columns of each trailing update go first, on `stream`;
  // the rest of the update runs on a side stream on all SMs but one while the next panel
  // (one CTA) factors on the SM left free; the panel's row permutation then waits for it.
  LookAhead la;
  const bool ahead = n >= 1024 && device_sm_count() > 1;
  if (ahead) RM_TRY(la.open());
  const int ni = (int)n;
  for (int J0 = 0; J0 < ni; J0 += kLppCols) {
    const int nb = std::min(kLppCols, ni - J0);
    const int T = std::min(kLppRows, ni - J0);
    const int J1 = J0 + nb;
    const int rest = ni - J1;
    float* dblk = dinv ? dinv + (size_t)(J0 / kLppCols) * kDiagMats * kLppCols * kLppCols : nullptr;
    lpp_panel_kernel<<<1, kLppThreads, kLppSmem, stream>>>(a, lda, J0, nb, T, linv, uinvt, plocal, dblk, status);
    RM_LAUNCHED();
    if (ahead && J0 > 0) RM_CUDA_TRY(cudaStreamWaitEvent(stream, la.rest_done, 0));
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
      RM_TRY(sgemm_tc(3, rest, rest - nn, nb, -1.0f, l21, lda, u12t + (size_t)nn * kLppCols, kLppCols, 1.0f, a22 + nn,
                      lda, status, la.side, nullptr, 0, device_sm_count() - 1));
      RM_CUDA_TRY(cudaEventRecord(la.rest_done, la.side));
    }
  }
  if (ahead) RM_CUDA_TRY(cudaStreamWaitEvent(stream, la.rest_done, 0));
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
