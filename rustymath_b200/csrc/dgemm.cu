// FP64 GEMM on the B200's FP64 tensor path: TMA-fed shared-memory tiles, mma.sync f64.
//
// Replaces rustymath's packed product (core/src/linalg.rs:1353-1426) and its AVX2 6x8
// micro-kernel (linalg.rs:1282); the operation is Tiled::gemm (linalg.rs:772-774),
// C = alpha*op(A)*op(B) + beta*C on row-major views. tcgen05 has no f64 kind, so the FP64
// tensor cores are reached through warp-level mma.sync.m16n8k8.f64 (DMMA).
//
// Pipeline: thread 0 issues cp.async.bulk.tensor loads (128-byte swizzle) STAGES-1 k-tiles
// ahead into a ring of stages guarded by full/empty mbarriers; the warps read fragments with
// 8-byte shared loads and run DMMA. (No separate producer warp: a ninth warp would cut every
// thread's register budget to 168 and spill the 64x32 accumulator tile.) The mma row/column each thread's fragment covers
// is mapped to a tile row/column (fragment maps below) so that every fragment load of a
// half-warp touches 16 distinct 8-byte bank pairs under the 128-byte swizzle.
#include "rm_internal.h"

namespace rm {

// Columns of a 16-wide swizzled slice that mma column g (0..7) of the slice's first (h=0)
// or second (h=1) n8 tile reads: {0,1,8,9,2,3,10,11} and the same plus 4.
__device__ __forceinline__ uint32_t rho(uint32_t g, uint32_t h) {
  return ((g & 1u) | ((g & 2u) << 2) | ((g & 4u) >> 1)) + 4u * h;
}

template <int BM_, int BN_, int WM_, int WN_, int STAGES_, bool TA_, bool TB_>
struct DgemmCfg {
  static constexpr int BM = BM_, BN = BN_, WM = WM_, WN = WN_, STAGES = STAGES_;
  static constexpr bool TA = TA_, TB = TB_;
  static constexpr int BK = 16;
  static constexpr int WARPS_M = BM / WM, WARPS_N = BN / WN;
  static constexpr int COMPUTE_WARPS = WARPS_M * WARPS_N;
  static constexpr int THREADS = COMPUTE_WARPS * 32;
  static constexpr int A_BYTES = BM * BK * 8, B_BYTES = BN * BK * 8;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int SMEM = STAGES * STAGE_BYTES + 1024 + 2 * STAGES * 8;
  static constexpr int MI = WM / 16, NJ = WN / 8;
  static_assert(BM % 16 == 0 && BN % 16 == 0 && WM % 16 == 0 && WN % 16 == 0, "tile shape");
  static_assert(BM <= 256 && BN <= 256, "TMA box extent");
};

// Byte offset of operand item (mn, k) in a stage's tile: K-major tiles hold one 128-byte
// row per M/N index; MN-major tiles hold 16-wide boxes of 16 k rows (2 KB each).
template <bool KMAJOR>
__device__ __forceinline__ uint32_t tile_off(uint32_t mn, uint32_t k) {
  if (KMAJOR) return swz128_f64(mn, k);
  return (mn >> 4) * 2048u + swz128_f64(k, mn & 15u);
}

template <class C>
__global__ void __launch_bounds__(C::THREADS, 1)
    dgemm_kernel(const __grid_constant__ CUtensorMap tma_a, const __grid_constant__ CUtensorMap tma_b,
                 double* __restrict__ c, int64_t ldc, int m, int n, int k, double alpha, double beta,
                 unsigned* status) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::STAGES * C::STAGE_BYTES);
  uint64_t* empty = full + C::STAGES;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * C::BM, n0 = blockIdx.x * C::BN;
  const int ktiles = (k + C::BK - 1) / C::BK;
  griddep_launch_dependents();
  griddep_wait();  // the kernel before this one in the stream has completed

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], C::COMPUTE_WARPS);
    }
    fence_barrier_init();
  }
  __syncthreads();

  // Thread 0 also issues the TMA loads: k-tile kt goes to stage kt % STAGES once every warp
  // has released that stage's previous k-tile (kt - STAGES).
  bool producing = true;
  auto issue = [&](int kt) {
    const int s = kt % C::STAGES;
    if (kt >= C::STAGES && !mbar_wait(&empty[s], ((kt - C::STAGES) / C::STAGES) & 1u, status)) {
      producing = false;
      return;
    }
    uint8_t* sa = smem + s * C::STAGE_BYTES;
    uint8_t* sb = sa + C::A_BYTES;
    mbar_arrive_expect_tx(&full[s], C::STAGE_BYTES);
    const int k0 = kt * C::BK;
    if (!C::TA) {
      tma_load_2d(sa, &tma_a, &full[s], k0, m0);
    } else {
#pragma unroll
      for (int b = 0; b < C::BM / 16; ++b) tma_load_2d(sa + b * 2048, &tma_a, &full[s], m0 + 16 * b, k0);
    }
    if (C::TB) {
      tma_load_2d(sb, &tma_b, &full[s], k0, n0);
    } else {
#pragma unroll
      for (int b = 0; b < C::BN / 16; ++b) tma_load_2d(sb + b * 2048, &tma_b, &full[s], n0 + 16 * b, k0);
    }
  };
  int issued = 0;
  if (threadIdx.x == 0) {
    tma_prefetch_desc(&tma_a);
    tma_prefetch_desc(&tma_b);
    for (; issued < C::STAGES - 1 && issued < ktiles && producing; ++issued) issue(issued);
  }

  // ---------------- compute warps
  const int wm0 = (warp / C::WARPS_N) * C::WM, wn0 = (warp % C::WARPS_N) * C::WN;
  const uint32_t g = lane >> 2, t = lane & 3;

  // Fragment maps: tile row of mma row r (0..15) of m16 tile i; tile column of mma column
  // q (0..7) of n8 tile j.
  auto arow = [&](int i, uint32_t r) -> uint32_t {
    return C::TA ? (wm0 + 16 * i + rho(r & 7u, r >> 3)) : (wm0 + 16 * i + 2 * (r & 7u) + (r >> 3));
  };
  auto bcol = [&](int j, uint32_t q) -> uint32_t {
    return C::TB ? (wn0 + 16 * (j >> 1) + 2 * q + (j & 1)) : (wn0 + 16 * (j >> 1) + rho(q, j & 1));
  };

  double acc[C::MI][C::NJ][4];
#pragma unroll
  for (int i = 0; i < C::MI; ++i)
#pragma unroll
    for (int j = 0; j < C::NJ; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

  bool ok = true;
  for (int kt = 0; kt < ktiles; ++kt) {
    if (threadIdx.x == 0 && producing && issued < ktiles) issue(issued++);
    const int s = kt % C::STAGES;
    if (!mbar_wait(&full[s], (kt / C::STAGES) & 1u, status)) { ok = false; break; }
    const uint8_t* sa = smem + s * C::STAGE_BYTES;
    const uint8_t* sb = sa + C::A_BYTES;
#pragma unroll
    for (int kk = 0; kk < C::BK; kk += 8) {
      double af[C::MI][4], bf[C::NJ][2];
#pragma unroll
      for (int i = 0; i < C::MI; ++i) {
        // k offsets kk and kk+4 change the swizzled chunk by XOR, so recompute per k.
        const uint32_t r0 = arow(i, g), r1 = arow(i, g + 8);
        af[i][0] = *reinterpret_cast<const double*>(sa + tile_off<!C::TA>(r0, kk + t));
        af[i][1] = *reinterpret_cast<const double*>(sa + tile_off<!C::TA>(r1, kk + t));
        af[i][2] = *reinterpret_cast<const double*>(sa + tile_off<!C::TA>(r0, kk + t + 4));
        af[i][3] = *reinterpret_cast<const double*>(sa + tile_off<!C::TA>(r1, kk + t + 4));
      }
#pragma unroll
      for (int j = 0; j < C::NJ; ++j) {
        const uint32_t q = bcol(j, g);
        bf[j][0] = *reinterpret_cast<const double*>(sb + tile_off<C::TB>(q, kk + t));
        bf[j][1] = *reinterpret_cast<const double*>(sb + tile_off<C::TB>(q, kk + t + 4));
      }
#pragma unroll
      for (int i = 0; i < C::MI; ++i)
#pragma unroll
        for (int j = 0; j < C::NJ; ++j)
          asm volatile(
              "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
              "{%0,%1,%2,%3};"
              : "+d"(acc[i][j][0]), "+d"(acc[i][j][1]), "+d"(acc[i][j][2]), "+d"(acc[i][j][3])
              : "d"(af[i][0]), "d"(af[i][1]), "d"(af[i][2]), "d"(af[i][3]), "d"(bf[j][0]), "d"(bf[j][1]));
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  if (!ok) {
    // leave no copy in flight behind: wait (bounded) for every issued stage's bytes
    if (threadIdx.x == 0)
      for (int kt = (issued > C::STAGES ? issued - C::STAGES : 0); kt < issued; ++kt)
        mbar_wait(&full[kt % C::STAGES], (kt / C::STAGES) & 1u, status);
    return;
  }

  // ---------------- epilogue: C = alpha*acc + beta*C
#pragma unroll
  for (int i = 0; i < C::MI; ++i)
#pragma unroll
    for (int j = 0; j < C::NJ; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const uint32_t r = g + 8 * (e >> 1), q = 2 * t + (e & 1);
        const int row = m0 + arow(i, r), col = n0 + bcol(j, q);
        if (row < m && col < n) {
          double* p = c + (int64_t)row * ldc + col;
          const double v = alpha * acc[i][j][e];
          *p = beta == 0.0 ? v : fma(beta, *p, v);
        }
      }
}

// ------------------------------------------------------------------ host side

template <class C>
static int launch_cfg(const double* a, int64_t lda, const double* b, int64_t ldb, double* c, int64_t ldc, int m,
                      int n, int k, double alpha, double beta, unsigned* status, cudaStream_t stream) {
  CUtensorMap ta, tb;
  // A: op(A) is m x k. Not transposed: stored m rows of k; transposed: k rows of m.
  if (!C::TA) {
    RM_TRY(make_tensor_map_2d(&ta, a, 8, k, m, lda * 8, 16, C::BM, true));
  } else {
    RM_TRY(make_tensor_map_2d(&ta, a, 8, m, k, lda * 8, 16, 16, true));
  }
  if (!C::TB) {
    RM_TRY(make_tensor_map_2d(&tb, b, 8, n, k, ldb * 8, 16, 16, true));
  } else {
    RM_TRY(make_tensor_map_2d(&tb, b, 8, k, n, ldb * 8, 16, C::BN, true));
  }
  RM_TRY(smem_attribute(dgemm_kernel<C>, C::SMEM));
  dim3 grid((n + C::BN - 1) / C::BN, (m + C::BM - 1) / C::BM);
  RM_CUDA_TRY(launch_dependent(dgemm_kernel<C>, grid, dim3(C::THREADS), C::SMEM, stream, ta, tb, c, ldc, m, n, k, alpha,
                               beta, status));
  note_launch();
  return RM_OK;
}

template <bool TA, bool TB>
static int launch_t(const double* a, int64_t lda, const double* b, int64_t ldb, double* c, int64_t ldc, int m, int n,
                    int k, double alpha, double beta, unsigned* status, cudaStream_t stream, bool wide) {
  const int64_t big_tiles = ((int64_t)(m + 127) / 128) * ((n + 127) / 128);
  if (wide || big_tiles >= device_sm_count()) {
    using Big = DgemmCfg<128, 128, 64, 32, 4, TA, TB>;
    return launch_cfg<Big>(a, lda, b, ldb, c, ldc, m, n, k, alpha, beta, status, stream);
  }
  using Small = DgemmCfg<64, 64, 32, 32, 4, TA, TB>;
  return launch_cfg<Small>(a, lda, b, ldb, c, ldc, m, n, k, alpha, beta, status, stream);
}

int dgemm_device(bool ta, bool tb, int64_t m, int64_t n, int64_t k, double alpha, const double* a, int64_t lda,
                 const double* b, int64_t ldb, double beta, double* c, int64_t ldc, unsigned* status,
                 cudaStream_t stream, bool wide) {
  if (m == 0 || n == 0) return RM_OK;
  if (k == 0 || alpha == 0.0) return scale_device(c, ldc, m, n, beta, stream);
  if (m > INT32_MAX || n > INT32_MAX || k > INT32_MAX) return RM_BAD_ARG;
  if (ta) {
    if (tb) return launch_t<true, true>(a, lda, b, ldb, c, ldc, (int)m, (int)n, (int)k, alpha, beta, status, stream, wide);
    return launch_t<true, false>(a, lda, b, ldb, c, ldc, (int)m, (int)n, (int)k, alpha, beta, status, stream, wide);
  }
  if (tb) return launch_t<false, true>(a, lda, b, ldb, c, ldc, (int)m, (int)n, (int)k, alpha, beta, status, stream, wide);
  return launch_t<false, false>(a, lda, b, ldb, c, ldc, (int)m, (int)n, (int)k, alpha, beta, status, stream, wide);
}

// C = beta*C (beta == 0 writes zeros), the reference's `scale` (linalg.rs:1000-1008).
__global__ void scale_kernel(double* c, int64_t ldc, int64_t m, int64_t n, double beta) {
  const int64_t total = m * n;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = idx / n, j = idx % n;
    double* p = c + i * ldc + j;
    *p = beta == 0.0 ? 0.0 : beta * *p;
  }
}

int scale_device(double* c, int64_t ldc, int64_t m, int64_t n, double beta, cudaStream_t stream) {
  if (beta == 1.0 || m == 0 || n == 0) return RM_OK;
  const int64_t total = m * n;
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, 4 * device_sm_count());
  scale_kernel<<<blocks, 256, 0, stream>>>(c, ldc, m, n, beta);
  RM_LAUNCHED();
  return RM_OK;
}

}  // namespace rm
