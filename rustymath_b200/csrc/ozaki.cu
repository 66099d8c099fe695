// FP64-accurate GEMM from int8 tensor-core products (the Ozaki split scheme).
//
// C = A B for float64 A (m x k) and B (k x n), row-major. Each row i of A is scaled by a
// power of two 2^-ea[i] into (-1, 1) and cut into `s` signed 7-bit slices:
//   a_ij = 2^ea[i] sum_{p<s} t_p 2^-7(p+1) + (remainder below 2^(ea[i]-7s)),  t_p in [-127, 127],
// each slice exact in int8 (the scaling and the digit extraction are exact in float64);
// likewise each column j of B with 2^eb[j]. Then
//   C_ij ~= 2^(ea[i]+eb[j]) sum_{d<s} 2^-7(d+2) sum_{p+q=d} (A_p B_q)_ij,
// dropping the products of order p + q >= s (below 2^-7s relative, as the truncation). The
// inner sums are int8 x int8 products accumulated in int32 by tcgen05.mma kind::i8 - exact
// while (d+1) k 127^2 < 2^31, so k is cut into chunks that keep it so - and each order d is
// one persistent launch whose epilogue adds 2^(ea+eb-7(d+2)) acc to C in float64, the
// smallest orders first. With s = 8 the truncation (2^-56 relative to 2^(ea+eb)) is below
// float64 rounding.
//
// The slices live in one scratch buffer: A's as s stacked (mp x kp) int8 planes (rows and
// k padded with zeros to whole tiles), B's transposed (K-major) as s stacked (np x kp) planes.
// rustymath's matmul is float64 throughout (core/src/linalg.rs:1119-1132); this is the
// split-precision product measured against the native float64 GEMM (rm_dgemm).
#include <algorithm>
#include <cfloat>
#include <climits>

#include "rm_internal.h"
#include "rm_tcgen05.cuh"

namespace rm {
namespace oz {

constexpr int BM = 128, BN = 128, BK = 128;  // BK int8 = 128 bytes: one swizzle row
constexpr int TILE_BYTES = BM * BK;          // 16 KB per operand tile
constexpr int STAGES = 5;
constexpr int STAGE_BYTES = 2 * TILE_BYTES;
constexpr int THREADS = 192;                 // TMA warp, MMA warp, 4 epilogue warps
constexpr uint32_t TMEM_COLS = 256;          // two accumulators of BN columns
constexpr int STG = 33;                      // epilogue staging: 32 x 33 doubles per warp
constexpr size_t SMEM = 1024 + (size_t)STAGES * STAGE_BYTES + 4 * 32 * STG * 8 + 512;
constexpr int MAX_SLICES = 8;

// Instruction descriptor, kind::i8: D s32, A and B signed int8, both K-major.
constexpr uint32_t idesc_i8(int m, int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

// frexp-style exponent of the largest |x| of a row: max|x| < 2^e (e = 0 for an all-zero row)
__device__ __forceinline__ int exponent_of(double v) {
  if (v == 0.0 || !(v == v)) return INT_MIN;
  int e;
  frexp(v, &e);
  return e;
}

// ea[i] for each row of the m x k row-major a: a warp per row
__global__ void row_exponent_kernel(const double* __restrict__ a, int64_t lda, int m, int k, int* __restrict__ ea) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= m) return;
  int e = INT_MIN;
  for (int j = lane; j < k; j += 32) e = max(e, exponent_of(fabs(a[(int64_t)warp * lda + j])));
#pragma unroll
  for (int off = 16; off; off >>= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, off));
  if (lane == 0) ea[warp] = e == INT_MIN ? 0 : e;
}

// eb[j] (pre-set to INT_MIN) for each column of the k x n row-major b: 32 x 32 tiles, atomics
__global__ void col_exponent_kernel(const double* __restrict__ b, int64_t ldb, int k, int n, int* __restrict__ eb) {
  __shared__ int cm[32];
  const int j = blockIdx.x * 32 + threadIdx.x;
  if (threadIdx.y == 0) cm[threadIdx.x] = INT_MIN;
  __syncthreads();
  int e = INT_MIN;
  if (j < n)
    for (int r = blockIdx.y * 32 + threadIdx.y; r < k; r += gridDim.y * 32)
      e = max(e, exponent_of(fabs(b[(int64_t)r * ldb + j])));
  atomicMax(&cm[threadIdx.x], e);
  __syncthreads();
  if (threadIdx.y == 0 && j < n && cm[threadIdx.x] != INT_MIN) atomicMax(&eb[j], cm[threadIdx.x]);
}

__global__ void fix_exponent_kernel(int* e, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && e[i] == INT_MIN) e[i] = 0;
}

// The s slices of row i of a (scaled by 2^-ea[i]) into planes [p][i][kk] (row stride kp,
// plane stride mp * kp): a warp per row, lanes along it.
__global__ void split_rows_kernel(const double* __restrict__ a, int64_t lda, int m, int k, const int* __restrict__ ea,
                                  int s, int8_t* __restrict__ out, int64_t kp, int64_t plane) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= m) return;
  const int e = ea[warp];
  for (int j = lane; j < k; j += 32) {
    double r = ldexp(a[(int64_t)warp * lda + j], -e);
    for (int p = 0; p < s; ++p) {
      r *= 128.0;
      const double t = trunc(r);
      r -= t;
      out[p * plane + (int64_t)warp * kp + j] = (int8_t)t;
    }
  }
}

// The s slices of column j of b (scaled by 2^-eb[j]), transposed: planes [q][j][kk] (row
// stride kp). 32 x 32 tiles through shared memory: reads along b's rows, writes along k.
__global__ void split_cols_kernel(const double* __restrict__ b, int64_t ldb, int k, int n, const int* __restrict__ eb,
                                  int s, int8_t* __restrict__ out, int64_t kp, int64_t plane) {
  __shared__ int8_t t8[MAX_SLICES][32][33];
  const int r0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int rr = ty; rr < 32; rr += 8) {
    const int r = r0 + rr, j = j0 + tx;
    double v = (r < k && j < n) ? ldexp(b[(int64_t)r * ldb + j], -eb[j]) : 0.0;
    for (int q = 0; q < s; ++q) {
      v *= 128.0;
      const double t = trunc(v);
      v -= t;
      t8[q][tx][rr] = (int8_t)t;
    }
  }
  __syncthreads();
  for (int jj = ty; jj < 32; jj += 8) {
    const int j = j0 + jj, r = r0 + tx;
    if (j < n && r < k)
      for (int q = 0; q < s; ++q) out[q * plane + (int64_t)j * kp + r] = t8[q][jj][tx];
  }
}

// Output tile t of a persistent walk -> (tile row, tile column), in bands of kBand tile rows:
// down a band's rows first, then across its columns, so that the ~148 tiles in flight at once
// read about kBand row panels of A's slices and 148 / kBand column panels of B's (some tens of
// MB, resident in L2) instead of one row panel and 148 column panels.
constexpr int kBand = 8;
__device__ __forceinline__ void tile_coords(int t, int ntm, int ntn, int& tm, int& tn) {
  const int per_band = kBand * ntn;
  const int band = t / per_band, in = t - band * per_band;
  const int rows = min(kBand, ntm - band * kBand);
  tm = band * kBand + in % rows;
  tn = in / rows;
}

// One order d of the split product over k-range [k0, k0 + kc):
//   C (+)= 2^(ea[i] + eb[j] - 7(d+2)) sum_{p+q=d} A_p B_q^T
// Persistent: warp 0 loads the slice tiles by TMA (rows p*mp + m0 of A's planes, q*np + n0 of
// B's), warp 1 issues kind::i8 MMAs into one of two TMEM accumulators per tile, warps 2..5
// drain them (int32 -> float64, scaled, added to C in coalesced rows through shared memory).
__global__ void __launch_bounds__(THREADS, 1)
    ozaki_order_kernel(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_b,
                       double* __restrict__ c, int64_t ldc, int m, int n, int mp, int np, int k0, int kc, int d,
                       const int* __restrict__ ea, const int* __restrict__ eb, int first, unsigned* status) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  double* stg_all = reinterpret_cast<double*>(smem + STAGES * STAGE_BYTES);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES + 4 * 32 * STG * 8);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;
  uint64_t* tempty = tfull + 2;
  uint64_t* mma_done = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntn = (n + BN - 1) / BN, ntm = (m + BM - 1) / BM;
  const int tiles = ntm * ntn;
  const int ktiles = (kc + BK - 1) / BK;
  const int pairs = d + 1;  // (p, d - p) for p = 0..d

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);
    }
    mbar_init(mma_done, 1);
    fence_barrier_init();
  }
  if (warp == 1) {
    tc::tmem_alloc(tmem_slot, TMEM_COLS);
    tc::fence_before();
  }
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      tma_prefetch_desc(&tm_a);
      tma_prefetch_desc(&tm_b);
      int it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        int tmi, tni;
        tile_coords(tile, ntm, ntn, tmi, tni);
        const int m0 = tmi * BM, n0 = tni * BN;
        for (int pq = 0; pq < pairs && ok; ++pq)
          for (int kt = 0; kt < ktiles; ++kt, ++it) {
            const int s = it % STAGES;
            if (!mbar_wait(&empty[s], ((it / STAGES) & 1u) ^ 1u, status)) {
              ok = false;
              break;
            }
            uint8_t* st = smem + s * STAGE_BYTES;
            mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
            tma_load_2d(st, &tm_a, &full[s], k0 + kt * BK, pq * mp + m0);
            tma_load_2d(st + TILE_BYTES, &tm_b, &full[s], k0 + kt * BK, (d - pq) * np + n0);
          }
      }
      for (int j = (it > STAGES ? it - STAGES : 0); j < it; ++j) mbar_wait(&full[j % STAGES], (j / STAGES) & 1u, status);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_i8(BM, BN);
      int it = 0, lt = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, ++lt) {
        const int buf = lt & 1;
        if (!mbar_wait(&tempty[buf], ((lt >> 1) & 1u) ^ 1u, status)) break;
        tc::fence_after();
        const uint32_t dt = tmem + buf * BN;
        for (int pq = 0; pq < pairs && ok; ++pq)
          for (int kt = 0; kt < ktiles; ++kt, ++it) {
            const int s = it % STAGES;
            if (!mbar_wait(&full[s], (it / STAGES) & 1u, status)) {
              ok = false;
              break;
            }
            tc::fence_after();
            const uint32_t sa = smem_u32(smem + s * STAGE_BYTES), sb = sa + TILE_BYTES;
#pragma unroll
            for (int kk = 0; kk < BK / 32; ++kk) {  // K = 32 int8 = 32 bytes per MMA
              const uint32_t acc = (pq == 0 && kt == 0 && kk == 0) ? 0u : 1u;
              mma_i8(dt, tc::smem_desc(sa + kk * 32), tc::smem_desc(sb + kk * 32), idesc, acc);
            }
            tc::mma_commit(&empty[s]);
          }
        if (ok) tc::mma_commit(&tfull[buf]);
      }
      tc::mma_commit(mma_done);
      mbar_wait(mma_done, 0u, status);
    }
  } else {
    // epilogue: warps 2..5, TMEM lane quarter warp % 4
    const int q = warp & 3;
    double* stg = stg_all + (warp - 2) * 32 * STG;
    int lt = 0;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++lt) {
      const int buf = lt & 1;
      if (!mbar_wait(&tfull[buf], (lt >> 1) & 1u, status)) break;
      tc::fence_after();
      int tmi, tni;
      tile_coords(tile, ntm, ntn, tmi, tni);
      const int m0 = tmi * BM, n0 = tni * BN;
      const int row0 = m0 + q * 32;
#pragma unroll 1
      for (int cb = 0; cb < BN; cb += 32) {
        uint32_t v[32];
        tc::tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + buf * BN + cb, v);
        if (cb == BN - 32) {
          tc::fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&tempty[buf]);
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 32; ++j) stg[lane * STG + j] = (double)(int)v[j];
        __syncwarp();
        const int col = n0 + cb + lane;
        const int ecol = col < n ? eb[col] : 0;
        double cv[32];
        if (!first) {
#pragma unroll
          for (int rr = 0; rr < 32; ++rr) {
            const int row = row0 + rr;
            cv[rr] = (row < m && col < n) ? c[(int64_t)row * ldc + col] : 0.0;
          }
        }
#pragma unroll
        for (int rr = 0; rr < 32; ++rr) {
          const int row = row0 + rr;
          if (row < m && col < n) {
            const double val = ldexp(stg[rr * STG + lane], ea[row] + ecol - 7 * (d + 2));
            c[(int64_t)row * ldc + col] = first ? val : cv[rr] + val;
          }
        }
      }
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 1) {
    tc::fence_after();
    tc::tmem_free(tmem, TMEM_COLS);
  }
}

}  // namespace oz

size_t ozaki_scratch_bytes(int64_t m, int64_t n, int64_t k, int s) {
  const int64_t mp = (m + oz::BM - 1) / oz::BM * oz::BM, np = (n + oz::BN - 1) / oz::BN * oz::BN;
  const int64_t kp = (k + oz::BK - 1) / oz::BK * oz::BK;
  return (size_t)s * (mp + np) * kp + (size_t)(m + n) * sizeof(int) + 1024;
}

__global__ void fill_int_kernel(int* p, int n, int v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

int dgemm_ozaki(int64_t m, int64_t n, int64_t k, const double* a, int64_t lda, const double* b, int64_t ldb,
                double* c, int64_t ldc, int s, void* scratch, unsigned* status, cudaStream_t stream) {
  if (m == 0 || n == 0) return RM_OK;
  if (s < 1 || s > oz::MAX_SLICES || m > INT_MAX / 2 || n > INT_MAX / 2 || k > INT_MAX / 2) return RM_BAD_ARG;
  if (k == 0) {
    RM_CUDA_TRY(cudaMemset2DAsync(c, ldc * sizeof(double), 0, n * sizeof(double), m, stream));
    return RM_OK;
  }
  const int64_t mp = (m + oz::BM - 1) / oz::BM * oz::BM, np = (n + oz::BN - 1) / oz::BN * oz::BN;
  const int64_t kp = (k + oz::BK - 1) / oz::BK * oz::BK;
  int8_t* asl = reinterpret_cast<int8_t*>(scratch);
  int8_t* bsl = asl + (size_t)s * mp * kp;
  int* ea = reinterpret_cast<int*>(bsl + (size_t)s * np * kp);
  int* eb = ea + m;
  RM_TRY(smem_attribute(oz::ozaki_order_kernel, oz::SMEM));
  const int mi = (int)m, ni = (int)n, ki = (int)k;
  // exponents and slices (the padding of the planes stays zero)
  RM_CUDA_TRY(cudaMemsetAsync(asl, 0, (size_t)s * (mp + np) * kp, stream));
  oz::row_exponent_kernel<<<(unsigned)((m * 32 + 255) / 256), 256, 0, stream>>>(a, lda, mi, ki, ea);
  RM_LAUNCHED();
  fill_int_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(eb, ni, INT_MIN);
  RM_LAUNCHED();
  oz::col_exponent_kernel<<<dim3((unsigned)((n + 31) / 32), (unsigned)std::min<int64_t>((k + 31) / 32, 64)),
                            dim3(32, 32), 0, stream>>>(b, ldb, ki, ni, eb);
  RM_LAUNCHED();
  oz::fix_exponent_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(eb, ni);
  RM_LAUNCHED();
  oz::split_rows_kernel<<<(unsigned)((m * 32 + 255) / 256), 256, 0, stream>>>(a, lda, mi, ki, ea, s, asl, kp,
                                                                               mp * kp);
  RM_LAUNCHED();
  oz::split_cols_kernel<<<dim3((unsigned)((n + 31) / 32), (unsigned)((k + 31) / 32)), dim3(32, 8), 0, stream>>>(
      b, ldb, ki, ni, eb, s, bsl, kp, np * kp);
  RM_LAUNCHED();
  CUtensorMap ta, tb;
  RM_TRY(make_tensor_map_2d(&ta, asl, 1, kp, s * mp, kp, oz::BK, oz::BM, true));
  RM_TRY(make_tensor_map_2d(&tb, bsl, 1, kp, s * np, kp, oz::BK, oz::BN, true));
  // k chunks short enough that an order's int32 sums cannot overflow: s k 127^2 < 2^31
  const int64_t kmax = std::max<int64_t>(oz::BK, ((int64_t)INT_MAX / ((int64_t)s * 127 * 127)) / oz::BK * oz::BK);
  const int64_t tiles = (mp / oz::BM) * (np / oz::BN);
  const unsigned grid = (unsigned)std::min<int64_t>(tiles, device_sm_count());
  bool first = true;
  for (int64_t k0 = 0; k0 < k; k0 += kmax) {
    const int kc = (int)std::min<int64_t>(kmax, k - k0);
    for (int d = s - 1; d >= 0; --d) {  // the smallest terms first
      oz::ozaki_order_kernel<<<grid, oz::THREADS, oz::SMEM, stream>>>(ta, tb, c, ldc, mi, ni, (int)mp, (int)np,
                                                                     (int)k0, kc, d, ea, eb, first ? 1 : 0, status);
      RM_LAUNCHED();
      first = false;
    }
  }
  return RM_OK;
}

}  // namespace rm
