// FP32 GEMM on the 5th-generation tensor cores: tcgen05.mma kind::tf32, TMEM accumulators.
//
// C = alpha * A B^T + beta * C, float32: A is m x k and B is n x k, both row-major with k
// contiguous ("K-major"); C is m x n row-major, and optionally its transpose goes to a second
// array as well. The mixed-precision LU's block updates run here.
// One pass reads the inputs as TF32 (the tensor core uses the top 19 bits of each float).
// Three passes recover float32-level products: with x_lo = x - trunc_tf32(x), exact in
// float32, A B ~= A_lo B + A B_lo + A B, each on TF32 inputs with FP32 accumulation in
// TMEM; the dropped A_lo B_lo term is ~2^-22 relative. The low parts are formed in shared
// memory from the tiles TMA brought in, so the operands cross L2 once.
//
// Warp roles (192 threads): warp 0 issues the TMA loads (128-byte swizzle, 3-stage ring),
// warp 1 owns the TMEM allocation and its lane 0 issues the MMAs (M=128, N=128, K=8 per
// instruction) and commits each stage back to the producer, warps 2..5 form the low parts
// of each stage (three passes), then read the 128 x 128 accumulator out of TMEM (one
// 32-lane quarter each) and write C. Every wait is bounded; TMEM is freed on every path.
#include "rm_internal.h"

namespace rm {

namespace tc {

constexpr int BM = 128, BN = 128, BK = 32;  // BK floats = 128 bytes: one swizzle row
constexpr int STAGES = 3;
constexpr int TILE_BYTES = BM * BK * 4;     // 16 KB per operand tile (BM == BN)
constexpr int THREADS = 192;
constexpr uint32_t TMEM_COLS = 128;

// UMMA shared-memory descriptor for a K-major tile written by TMA with 128-byte swizzle
// (box {32 k, 128 rows}): rows of 128 bytes, 8-row groups 1024 bytes apart (stride byte
// offset), leading byte offset unused (1), descriptor version 1 (sm_100), layout type 2.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                              // leading byte offset (>> 4)
  d |= (uint64_t)(1024 >> 4) << 32;                    // stride byte offset (>> 4)
  d |= (uint64_t)1 << 46;                              // version
  d |= (uint64_t)2 << 61;                              // SWIZZLE_128B
  return d;
}

// Instruction descriptor, kind::tf32: D f32, A and B tf32, both K-major.
constexpr uint32_t idesc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t lo_bits(uint32_t x) {
  const float v = __uint_as_float(x);
  return __float_as_uint(v - __uint_as_float(x & 0xFFFFE000u));
}

}  // namespace tc

template <int PASSES>
__global__ void __launch_bounds__(tc::THREADS, 1)
    sgemm_tc_kernel(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_b,
                    float* __restrict__ c, int64_t ldc, float* __restrict__ ct, int64_t ldct, int m, int n, int k,
                    float alpha, float beta, unsigned* status) {
  using namespace tc;
  constexpr int OPS = PASSES == 3 ? 4 : 2;  // tiles per stage: A, B, (A_lo, B_lo)
  constexpr int STAGE_BYTES = OPS * TILE_BYTES;
  constexpr int LOAD_BYTES = 2 * TILE_BYTES;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* lo_ready = empty + STAGES;
  uint64_t* done = lo_ready + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ int failed;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int ktiles = (k + BK - 1) / BK;

  if (threadIdx.x == 0) {
    failed = 0;
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
      mbar_init(&lo_ready[s], 4);  // one arrival per low-part warp
    }
    mbar_init(done, 1);
    fence_barrier_init();
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    tc::fence_before();
  }
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      tma_prefetch_desc(&tm_a);
      tma_prefetch_desc(&tm_b);
      int issued = 0;
      for (int kt = 0; kt < ktiles; ++kt) {
        const int s = kt % STAGES;
        if (!mbar_wait(&empty[s], ((kt / STAGES) & 1u) ^ 1u, status)) {
          failed = 1;
          break;
        }
        uint8_t* st = smem + s * STAGE_BYTES;
        mbar_arrive_expect_tx(&full[s], LOAD_BYTES);
        const int k0 = kt * BK;
        tma_load_2d(st, &tm_a, &full[s], k0, m0);
        tma_load_2d(st + TILE_BYTES, &tm_b, &full[s], k0, n0);
        ++issued;
      }
      // the copies still in flight land before this thread leaves (bounded)
      for (int kt = (issued > STAGES ? issued - STAGES : 0); kt < issued; ++kt)
        mbar_wait(&full[kt % STAGES], (kt / STAGES) & 1u, status);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_tf32(BM, BN);
      for (int kt = 0; kt < ktiles; ++kt) {
        const int s = kt % STAGES;
        const uint32_t par = (kt / STAGES) & 1u;
        if (!mbar_wait(&full[s], par, status) || (PASSES == 3 && !mbar_wait(&lo_ready[s], par, status))) {
          failed = 1;
          break;
        }
        tc::fence_after();
        const uint32_t sa = smem_u32(smem + s * STAGE_BYTES);
        const uint32_t sb = sa + TILE_BYTES;
#pragma unroll
        for (int kk = 0; kk < BK / 8; ++kk) {
          const uint32_t off = kk * 32;  // 8 tf32 = 32 bytes along the swizzled rows
          const uint32_t first = (kt == 0 && kk == 0) ? 0u : 1u;
          const uint64_t da = tc::smem_desc(sa + off), db = tc::smem_desc(sb + off);
          if (PASSES == 3) {
            const uint64_t dalo = tc::smem_desc(sa + 2 * TILE_BYTES + off);
            const uint64_t dblo = tc::smem_desc(sa + 3 * TILE_BYTES + off);
            tc::mma_tf32(tmem, dalo, db, idesc, first);
            tc::mma_tf32(tmem, da, dblo, idesc, 1u);
            tc::mma_tf32(tmem, da, db, idesc, 1u);
          } else {
            tc::mma_tf32(tmem, da, db, idesc, first);
          }
        }
        tc::mma_commit(&empty[s]);  // the stage is free once these MMAs have read it
      }
      tc::mma_commit(done);  // the accumulator is complete once every MMA above has run
    }
  } else {
    // ---------------- warps 2..5: the low parts of each stage, then the epilogue
    const int t = threadIdx.x - 64;  // 0..127
    if (PASSES == 3) {
      for (int kt = 0; kt < ktiles; ++kt) {
        const int s = kt % STAGES;
        if (!mbar_wait(&full[s], (kt / STAGES) & 1u, status)) {
          failed = 1;
          break;
        }
        const uint4* src = reinterpret_cast<const uint4*>(smem + s * STAGE_BYTES);
        uint4* dst = reinterpret_cast<uint4*>(smem + s * STAGE_BYTES + 2 * TILE_BYTES);
#pragma unroll 4
        for (int i = t; i < 2 * TILE_BYTES / 16; i += 128) {  // A then B: same swizzled positions
          const uint4 v = src[i];
          dst[i] = make_uint4(tc::lo_bits(v.x), tc::lo_bits(v.y), tc::lo_bits(v.z), tc::lo_bits(v.w));
        }
        fence_proxy_async();  // the MMA reads these through the async proxy
        __syncwarp();
        if (lane == 0) mbar_arrive(&lo_ready[s]);
      }
    }
    const int q = warp & 3;
    const bool ready = mbar_wait(done, 0u, status);
    tc::fence_after();
    const int row = m0 + q * 32 + lane;
    if (ready && !failed && ktiles > 0) {
#pragma unroll 1
      for (int cb = 0; cb < BN; cb += 32) {
        uint32_t v[32];
        tc::tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + cb, v);
        if (row < m) {
          float* crow = c + (int64_t)row * ldc + n0 + cb;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            if (n0 + cb + j < n) {
              const float d = __uint_as_float(v[j]);
              const float out = beta == 0.0f ? alpha * d : fmaf(beta, crow[j], alpha * d);
              crow[j] = out;
              // the transposed copy: the warp's 32 rows land in 32 consecutive floats
              if (ct) ct[(int64_t)(n0 + cb + j) * ldct + row] = out;
            }
          }
        }
      }
    }
    tc::fence_before();
  }
  __syncthreads();
  if (warp == 1) {
    tc::fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// lo = x - trunc_tf32(x), elementwise over an m x k row-major array (lds, ldd)
__global__ void split_lo_kernel(const float* __restrict__ x, int64_t ldx, int64_t m, int64_t k, float* __restrict__ lo,
                                int64_t ldl) {
  const int64_t total = m * k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / k, j = e - i * k;
    const float v = x[i * ldx + j];
    lo[i * ldl + j] = v - __uint_as_float(__float_as_uint(v) & 0xFFFFE000u);
  }
}

int split_lo_f32(const float* x, int64_t ldx, int64_t m, int64_t k, float* lo, int64_t ldl, cudaStream_t stream) {
  if (m == 0 || k == 0) return RM_OK;
  const int blocks = (int)std::min<int64_t>((m * k + 255) / 256, 8 * device_sm_count());
  split_lo_kernel<<<blocks, 256, 0, stream>>>(x, ldx, m, k, lo, ldl);
  RM_LAUNCHED();
  return RM_OK;
}

__global__ void scale_f32_kernel(float* c, int64_t ldc, int64_t m, int64_t n, float beta) {
  const int64_t total = m * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / n, j = e - i * n;
    float* p = c + i * ldc + j;
    *p = beta == 0.0f ? 0.0f : beta * *p;
  }
}

int scale_f32(float* c, int64_t ldc, int64_t m, int64_t n, float beta, cudaStream_t stream) {
  if (beta == 1.0f || m == 0 || n == 0) return RM_OK;
  const int blocks = (int)std::min<int64_t>((m * n + 255) / 256, 4 * device_sm_count());
  scale_f32_kernel<<<blocks, 256, 0, stream>>>(c, ldc, m, n, beta);
  RM_LAUNCHED();
  return RM_OK;
}

size_t sgemm_tc_smem(int passes) {
  return (size_t)tc::STAGES * (passes == 3 ? 4 : 2) * tc::TILE_BYTES + 1024 + 512;
}

template <int PASSES>
static int launch_sgemm(const CUtensorMap& ta, const CUtensorMap& tb, float* c, int64_t ldc, float* ct, int64_t ldct,
                        int m, int n, int k, float alpha, float beta, unsigned* status, cudaStream_t stream) {
  const size_t smem = sgemm_tc_smem(PASSES);
  static bool set = false;
  if (!set) {
    RM_CUDA_TRY(cudaFuncSetAttribute(sgemm_tc_kernel<PASSES>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    set = true;
  }
  dim3 grid((unsigned)((n + tc::BN - 1) / tc::BN), (unsigned)((m + tc::BM - 1) / tc::BM));
  sgemm_tc_kernel<PASSES><<<grid, tc::THREADS, smem, stream>>>(ta, tb, c, ldc, ct, ldct, m, n, k, alpha, beta,
                                                               status);
  RM_LAUNCHED();
  return RM_OK;
}

int sgemm_tc(int passes, int64_t m, int64_t n, int64_t k, float alpha, const float* a, int64_t lda, const float* b,
             int64_t ldb, float beta, float* c, int64_t ldc, unsigned* status, cudaStream_t stream, float* ct,
             int64_t ldct) {
  if (m == 0 || n == 0) return RM_OK;
  if (passes != 1 && passes != 3) return RM_BAD_ARG;
  if (m > INT32_MAX || n > INT32_MAX || k > INT32_MAX || k == 0) return RM_BAD_ARG;
  CUtensorMap ta, tb;
  RM_TRY(make_tensor_map_2d(&ta, a, 4, k, m, lda * 4, tc::BK, tc::BM, true));
  RM_TRY(make_tensor_map_2d(&tb, b, 4, k, n, ldb * 4, tc::BK, tc::BN, true));
  const int mi = (int)m, ni = (int)n, ki = (int)k;
  if (passes == 3) return launch_sgemm<3>(ta, tb, c, ldc, ct, ldct, mi, ni, ki, alpha, beta, status, stream);
  return launch_sgemm<1>(ta, tb, c, ldc, ct, ldct, mi, ni, ki, alpha, beta, status, stream);
}

// dst (n x m, ldd) = src^T for the m x n row-major float32 src (lds): 32x32 tiles through
// shared memory, both sides coalesced.
__global__ void transpose_f32_kernel(const float* __restrict__ src, int64_t lds, int64_t m, int64_t n,
                                     float* __restrict__ dst, int64_t ldd) {
  __shared__ float tile[32][33];
  const int64_t i0 = (int64_t)blockIdx.y * 32, j0 = (int64_t)blockIdx.x * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t i = i0 + r, j = j0 + threadIdx.x;
    if (i < m && j < n) tile[r][threadIdx.x] = src[i * lds + j];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t j = j0 + r, i = i0 + threadIdx.x;
    if (i < m && j < n) dst[j * ldd + i] = tile[threadIdx.x][r];
  }
}

int transpose_f32(const float* src, int64_t lds, int64_t m, int64_t n, float* dst, int64_t ldd, cudaStream_t stream) {
  if (m == 0 || n == 0) return RM_OK;
  dim3 grid((unsigned)((n + 31) / 32), (unsigned)((m + 31) / 32));
  transpose_f32_kernel<<<grid, dim3(32, 8), 0, stream>>>(src, lds, m, n, dst, ldd);
  RM_LAUNCHED();
  return RM_OK;
}

}  // namespace rm
