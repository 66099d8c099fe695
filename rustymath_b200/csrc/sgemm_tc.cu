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
// Persistent: a CTA per SM walks the output tiles in a fixed stride. Warp 0 issues the TMA
// loads (128-byte swizzle) into a ring of stages; warp 1 owns the TMEM allocation (two
// 128 x 128 FP32 accumulators) and its lane 0 issues the MMAs (M=128, N=128, K=8 per
// instruction), alternating accumulators between tiles so that the next tile's MMAs run
// while the epilogue drains the last one; warps 2..5 are the epilogue (one 32-lane TMEM
// quarter each), in 32 x 32 chunks through six buffers per warp: C's chunks come in by TMA
// five chunks ahead (when beta is not zero), alpha*acc + beta*C is formed in the same
// swizzled shared-memory buffer and goes out as an asynchronous TMA store, so no global
// access stalls these warps; the optional
// transposed copy is written from registers in coalesced columns. (When C's address or row
// stride does not suit TMA, the epilogue stages through shared memory and writes coalesced
// rows itself.) For three passes warps 6..9 form the low parts of each stage. Every wait is
// bounded; TMEM is freed on every path. Launched as a programmatic dependent: barrier set-up
// and the TMEM allocation overlap the end of the kernel before it.
#include "rm_internal.h"
#include "rm_tcgen05.cuh"

namespace rm {

namespace tc {

constexpr int BM = 128, BN = 128, BK = 32;  // BK floats = 128 bytes: one swizzle row
constexpr int TILE_BYTES = BM * BK * 4;     // 16 KB per operand tile (BM == BN)
constexpr uint32_t TMEM_COLS = 256;         // two accumulators of BN columns
constexpr int STG_STRIDE = 33;              // direct epilogue: 32 x 32 floats per warp, padded
constexpr int EPI_BUF = 32 * 32 * 4;        // TMA epilogue: one 32 x 32 chunk, 128-byte swizzle
constexpr int EPI_NBUF = 6;                 // chunk buffers per epilogue warp: C is read 5 chunks ahead
constexpr int STG_BYTES = 4 * EPI_NBUF * EPI_BUF;  // (>= the direct epilogue's staging)

template <int PASSES>
struct Cfg {
  static constexpr int OPS = PASSES == 3 ? 4 : 2;  // tiles per stage: A, B, (A_lo, B_lo)
  static constexpr int STAGES = PASSES == 3 ? 2 : 4;
  static constexpr int STAGE_BYTES = OPS * TILE_BYTES;
  static constexpr int LO_WARPS = PASSES == 3 ? 4 : 0;
  static constexpr int THREADS = 32 * (6 + LO_WARPS);
  static constexpr size_t SMEM = 1024 + (size_t)STAGES * STAGE_BYTES + STG_BYTES + 512;
};

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


__device__ __forceinline__ uint32_t lo_bits(uint32_t x) {
  const float v = __uint_as_float(x);
  return __float_as_uint(v - __uint_as_float(x & 0xFFFFE000u));
}


}  // namespace tc

// One of the (up to) two products of a launch: they share n, k, alpha and beta; the output
// tiles of the first come first.
struct SgemmPart {
  float* c;
  int64_t ldc;
  float* ct;
  int64_t ldct;
  int m;
  int tiles;
};

// LO_G (three passes, one product): the low parts of A and B come from global memory
// (tm_alo, tm_blo: same shapes and coordinates as A and B), loaded by TMA beside A and B, in
// place of warps 6..9 forming them in shared memory.
template <int PASSES, bool TMA_EPI, bool LO_G>
__global__ void __launch_bounds__(tc::Cfg<PASSES>::THREADS, 1)
    sgemm_tc_kernel(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_b,
                    const __grid_constant__ CUtensorMap tm_c, const __grid_constant__ CUtensorMap tm_a2,
                    const __grid_constant__ CUtensorMap tm_b2, const __grid_constant__ CUtensorMap tm_c2,
                    const __grid_constant__ CUtensorMap tm_alo, const __grid_constant__ CUtensorMap tm_blo,
                    const SgemmPart p1, const SgemmPart p2, int n, int k, float alpha, float beta,
                    unsigned* status) {
  using namespace tc;
  using C = Cfg<PASSES>;
  constexpr int S = C::STAGES;
  constexpr int LOAD_BYTES = (LO_G ? 4 : 2) * TILE_BYTES;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  float* stg_all = reinterpret_cast<float*>(smem + S * C::STAGE_BYTES);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * C::STAGE_BYTES + STG_BYTES);
  uint64_t* empty = full + S;
  uint64_t* lo_ready = empty + S;
  uint64_t* tfull = lo_ready + S;   // an accumulator holds a finished tile
  uint64_t* tempty = tfull + 2;     // the epilogue has read an accumulator out
  uint64_t* mma_done = tempty + 2;  // every MMA issued has completed
  uint64_t* cload = mma_done + 1;   // [epilogue warp][buffer]: a chunk of C has landed
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(cload + 4 * EPI_NBUF);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntn = (n + BN - 1) / BN;
  const int tiles = p1.tiles + p2.tiles;
  const int ktiles = (k + BK - 1) / BK;
  // tile -> (its product, its index within it)
  auto part = [&](int tile, int& lt) -> const SgemmPart& {
    const bool second = tile >= p1.tiles;
    lt = second ? tile - p1.tiles : tile;
    return second ? p2 : p1;
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
      mbar_init(&lo_ready[s], C::LO_WARPS > 0 ? C::LO_WARPS : 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);  // one arrival per epilogue warp
    }
    mbar_init(mma_done, 1);
    for (int b = 0; b < 4 * EPI_NBUF; ++b) mbar_init(&cload[b], 1);
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
  // set-up done: the next kernel in the stream may start its own; then wait for the previous
  // one's results (no wait without a programmatic launch)
  griddep_launch_dependents();
  griddep_wait();

  if (warp == 0) {
    // ---------------- TMA producer
    if (lane == 0) {
      tma_prefetch_desc(&tm_a);
      tma_prefetch_desc(&tm_b);
      if (p2.tiles > 0) {
        tma_prefetch_desc(&tm_a2);
        tma_prefetch_desc(&tm_b2);
      }
      if (LO_G) {
        tma_prefetch_desc(&tm_alo);
        tma_prefetch_desc(&tm_blo);
      }
      int it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        int ltile;
        part(tile, ltile);
        const bool second = tile >= p1.tiles;
        const CUtensorMap* ma = second ? &tm_a2 : &tm_a;
        const CUtensorMap* mb = second ? &tm_b2 : &tm_b;
        const int m0 = (ltile / ntn) * BM, n0 = (ltile % ntn) * BN;
        for (int kt = 0; kt < ktiles; ++kt, ++it) {
          const int s = it % S;
          if (!mbar_wait(&empty[s], ((it / S) & 1u) ^ 1u, status)) {
            ok = false;
            break;
          }
          uint8_t* st = smem + s * C::STAGE_BYTES;
          mbar_arrive_expect_tx(&full[s], LOAD_BYTES);
          tma_load_2d(st, ma, &full[s], kt * BK, m0);
          tma_load_2d(st + TILE_BYTES, mb, &full[s], kt * BK, n0);
          if (LO_G) {
            tma_load_2d(st + 2 * TILE_BYTES, &tm_alo, &full[s], kt * BK, m0);
            tma_load_2d(st + 3 * TILE_BYTES, &tm_blo, &full[s], kt * BK, n0);
          }
        }
      }
      // the copies still in flight land before this thread leaves (bounded)
      for (int j = (it > S ? it - S : 0); j < it; ++j) mbar_wait(&full[j % S], (j / S) & 1u, status);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_tf32(BM, BN);
      int it = 0, lt = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, ++lt) {
        const int buf = lt & 1;
        if (!mbar_wait(&tempty[buf], ((lt >> 1) & 1u) ^ 1u, status)) break;
        tc::fence_after();
        const uint32_t d = tmem + buf * BN;
        for (int kt = 0; kt < ktiles; ++kt, ++it) {
          const int s = it % S;
          const uint32_t par = (it / S) & 1u;
          if (!mbar_wait(&full[s], par, status) || (PASSES == 3 && !LO_G && !mbar_wait(&lo_ready[s], par, status))) {
            ok = false;
            break;
          }
          tc::fence_after();
          const uint32_t sa = smem_u32(smem + s * C::STAGE_BYTES);
          const uint32_t sb = sa + TILE_BYTES;
#pragma unroll
          for (int kk = 0; kk < BK / 8; ++kk) {
            const uint32_t off = kk * 32;  // 8 tf32 = 32 bytes along the swizzled rows
            const uint32_t first = (kt == 0 && kk == 0) ? 0u : 1u;
            const uint64_t da = tc::smem_desc(sa + off), db = tc::smem_desc(sb + off);
            if (PASSES == 3) {
              const uint64_t dalo = tc::smem_desc(sa + 2 * TILE_BYTES + off);
              const uint64_t dblo = tc::smem_desc(sa + 3 * TILE_BYTES + off);
              tc::mma_tf32(d, dalo, db, idesc, first);
              tc::mma_tf32(d, da, dblo, idesc, 1u);
              tc::mma_tf32(d, da, db, idesc, 1u);
            } else {
              tc::mma_tf32(d, da, db, idesc, first);
            }
          }
          tc::mma_commit(&empty[s]);  // the stage is free once these MMAs have read it
        }
        if (ok) tc::mma_commit(&tfull[buf]);  // the accumulator is complete once every MMA above has run
      }
      tc::mma_commit(mma_done);
      mbar_wait(mma_done, 0u, status);
    }
  } else if (warp < 6 && TMA_EPI) {
    // ---------------- epilogue through TMA: warps 2..5, TMEM lane quarter warp % 4
    const int q = warp & 3, ew = warp - 2;
    uint8_t* ebuf = reinterpret_cast<uint8_t*>(stg_all) + ew * EPI_NBUF * EPI_BUF;
    uint64_t* cl = cload + EPI_NBUF * ew;
    const bool load_c = beta != 0.0f;
    // Chunk ci (counted over this CTA's tiles, BN / 32 per tile) uses buffer ci % EPI_NBUF, and
    // C's chunks are loaded EPI_NBUF - 1 ahead of the one being formed.
    constexpr int CPT = BN / 32;
    const int my_tiles = (int)blockIdx.x < tiles ? (tiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
    const int chunks = my_tiles * CPT;
    int issued = 0;  // chunks of C whose load has been issued
    // Issues the loads of chunks issued..upto-1. Called once a chunk's store is committed (or
    // before the first), so a buffer's previous store is at most one group back.
    auto prefetch_to = [&](int upto) {
      if (!load_c) return;
      upto = min(upto, chunks);
      for (; issued < upto; ++issued) {
        if (lane == 0) {
          tc::bulk_wait_read<1>();  // the store that last used this buffer has read it
          const int b = issued % EPI_NBUF;
          const int tile = (int)blockIdx.x + (issued / CPT) * (int)gridDim.x, cb = (issued % CPT) * 32;
          int lt2;
          part(tile, lt2);
          mbar_arrive_expect_tx(&cl[b], EPI_BUF);
          tma_load_2d(ebuf + b * EPI_BUF, tile >= p1.tiles ? &tm_c2 : &tm_c, &cl[b], (lt2 % ntn) * BN + cb,
                      (lt2 / ntn) * BM + q * 32);
        }
      }
      __syncwarp();
    };
    int lt = 0, ci = 0;
    bool ok = true;
    prefetch_to(EPI_NBUF - 1);
    for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, ++lt) {
      const int buf = lt & 1;
      if (!mbar_wait(&tfull[buf], (lt >> 1) & 1u, status)) break;
      tc::fence_after();
      int ltile;
      const SgemmPart& P = part(tile, ltile);
      const CUtensorMap* mc = tile >= p1.tiles ? &tm_c2 : &tm_c;
      float* const ct = P.ct;
      const int64_t ldct = P.ldct;
      const int m = P.m;
      const int m0 = (ltile / ntn) * BM, n0 = (ltile % ntn) * BN;
      const int row0 = m0 + q * 32;
#pragma unroll 1
      for (int cb = 0; cb < BN; cb += 32, ++ci) {
        uint32_t v[32];
        tc::tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + buf * BN + cb, v);
        if (cb == BN - 32) {  // the accumulator is in registers: hand it back to the MMA warp
          tc::fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&tempty[buf]);
        }
        const int b = ci % EPI_NBUF;
        uint8_t* eb = ebuf + b * EPI_BUF;
        if (load_c) {
          if (!mbar_wait(&cl[b], (ci / EPI_NBUF) & 1u, status)) {
            ok = false;
            break;
          }
        } else {
          if (lane == 0) tc::bulk_wait_read<EPI_NBUF - 1>();  // the store EPI_NBUF chunks back has read this buffer
          __syncwarp();
        }
        // this lane's row of the chunk: alpha * acc + beta * C, in place
#pragma unroll
        for (int g = 0; g < 8; ++g) {
          float4* p = reinterpret_cast<float4*>(eb + tc::chunk_off(lane, 4 * g));
          float4 o = make_float4(alpha * __uint_as_float(v[4 * g]), alpha * __uint_as_float(v[4 * g + 1]),
                                 alpha * __uint_as_float(v[4 * g + 2]), alpha * __uint_as_float(v[4 * g + 3]));
          if (load_c) {
            const float4 cv = *p;
            o.x = fmaf(beta, cv.x, o.x), o.y = fmaf(beta, cv.y, o.y), o.z = fmaf(beta, cv.z, o.z),
            o.w = fmaf(beta, cv.w, o.w);
          }
          *p = o;
          if (ct) {
            // the transposed copy: column j of the chunk, the warp's 32 rows in 32 consecutive floats
            const int row = row0 + lane;
            const float ov[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int col = n0 + cb + 4 * g + e;
              if (row < m && col < n) ct[(int64_t)col * ldct + row] = ov[e];
            }
          }
        }
        fence_proxy_async();  // the TMA store reads these through the async proxy
        __syncwarp();
        if (lane == 0) {
          tc::tma_store_2d(mc, eb, n0 + cb, row0);
          tc::bulk_commit();
        }
        prefetch_to(ci + EPI_NBUF);  // C's chunk EPI_NBUF - 1 ahead of the next
      }
    }
    // loads of C still in flight (only after a wait gave up) land before the CTA ends (bounded)
    for (int j = ci; j < issued; ++j) mbar_wait(&cl[j % EPI_NBUF], (j / EPI_NBUF) & 1u, status);
    if (lane == 0) tc::bulk_wait_all();  // every store has landed before the CTA ends
    __syncwarp();
  } else if (warp < 6) {
    // ---------------- epilogue, direct: warps 2..5, TMEM lane quarter warp % 4
    const int q = warp & 3;
    float* stg = stg_all + (warp - 2) * 32 * STG_STRIDE;
    int lt = 0;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++lt) {
      const int buf = lt & 1;
      if (!mbar_wait(&tfull[buf], (lt >> 1) & 1u, status)) break;
      tc::fence_after();
      int ltile;
      const SgemmPart& P = part(tile, ltile);
      float* const c = P.c;
      const int64_t ldc = P.ldc;
      float* const ct = P.ct;
      const int64_t ldct = P.ldct;
      const int m = P.m;
      const int m0 = (ltile / ntn) * BM, n0 = (ltile % ntn) * BN;
      const int row0 = m0 + q * 32;
#pragma unroll 1
      for (int cb = 0; cb < BN; cb += 32) {
        uint32_t v[32];
        tc::tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + buf * BN + cb, v);
        if (cb == BN - 32) {  // the accumulator is in registers: hand it back to the MMA warp
          tc::fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&tempty[buf]);
        }
        __syncwarp();  // the last chunk's reads of the staging tile are done
#pragma unroll
        for (int j = 0; j < 32; ++j) stg[lane * STG_STRIDE + j] = __uint_as_float(v[j]);
        __syncwarp();
        // lane = column: each row of the chunk is one coalesced 128-byte access
        const int col = n0 + cb + lane;
        float cv[32];
        if (beta != 0.0f) {
#pragma unroll
          for (int rr = 0; rr < 32; ++rr) {
            const int row = row0 + rr;
            cv[rr] = (row < m && col < n) ? c[(int64_t)row * ldc + col] : 0.0f;
          }
        }
#pragma unroll
        for (int rr = 0; rr < 32; ++rr) {
          const int row = row0 + rr;
          float out = alpha * stg[rr * STG_STRIDE + lane];
          if (beta != 0.0f) out = fmaf(beta, cv[rr], out);
          if (row < m && col < n) c[(int64_t)row * ldc + col] = out;
          if (ct) stg[rr * STG_STRIDE + lane] = out;
        }
        if (ct) {
          // lane = row: each column of the chunk is one coalesced access of the transposed copy
          __syncwarp();
          const int row = row0 + lane;
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (row < m && n0 + cb + j < n) ct[(int64_t)(n0 + cb + j) * ldct + row] = stg[lane * STG_STRIDE + j];
        }
      }
    }
  } else if (PASSES == 3 && !LO_G) {
    // ---------------- warps 6..9: the low parts of each stage
    const int t = threadIdx.x - 192;  // 0..127
    int it = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
      for (int kt = 0; kt < ktiles; ++kt, ++it) {
        const int s = it % S;
        if (!mbar_wait(&full[s], (it / S) & 1u, status)) {
          ok = false;
          break;
        }
        const uint4* src = reinterpret_cast<const uint4*>(smem + s * C::STAGE_BYTES);
        uint4* dst = reinterpret_cast<uint4*>(smem + s * C::STAGE_BYTES + 2 * TILE_BYTES);
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
  }
  tc::fence_before();
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

template <int PASSES, bool TMA_EPI, bool LO_G = false>
static int launch_sgemm(const CUtensorMap* maps, const SgemmPart& p1, const SgemmPart& p2, int n, int k, float alpha,
                        float beta, unsigned* status, cudaStream_t stream, int max_ctas) {
  using C = tc::Cfg<PASSES>;
  RM_TRY(smem_attribute(sgemm_tc_kernel<PASSES, TMA_EPI, LO_G>, C::SMEM));
  const int64_t tiles = (int64_t)p1.tiles + p2.tiles;
  const int ctas = max_ctas > 0 ? std::min(max_ctas, device_sm_count()) : device_sm_count();
  const unsigned grid = (unsigned)std::min<int64_t>(tiles, ctas);
  RM_CUDA_TRY(launch_dependent(sgemm_tc_kernel<PASSES, TMA_EPI, LO_G>, dim3(grid), dim3(C::THREADS), C::SMEM, stream,
                               maps[0], maps[1], maps[2], maps[3], maps[4], maps[5], maps[6], maps[7], p1, p2, n, k,
                               alpha, beta, status));
  RM_LAUNCHED();
  return RM_OK;
}

namespace {
// The tensor maps of one product (A, B and, for the TMA epilogue, C) and its tile count.
int prepare_part(const SgemmOperands& o, int64_t n, int64_t k, bool tma_epi, CUtensorMap* maps, SgemmPart* part) {
  if (o.m > INT32_MAX) return RM_BAD_ARG;
  RM_TRY(make_tensor_map_2d(&maps[0], o.a, 4, k, o.m, o.lda * 4, tc::BK, tc::BM, true));
  RM_TRY(make_tensor_map_2d(&maps[1], o.b, 4, k, n, o.ldb * 4, tc::BK, tc::BN, true));
  if (tma_epi) RM_TRY(make_tensor_map_2d(&maps[2], o.c, 4, n, o.m, o.ldc * 4, 32, 32, true));
  else memset(&maps[2], 0, sizeof maps[2]);
  *part = {o.c, o.ldc, o.ct, o.ldct, (int)o.m, (int)(((o.m + tc::BM - 1) / tc::BM) * ((n + tc::BN - 1) / tc::BN))};
  return RM_OK;
}

// C through TMA when its base and row stride are 16-byte aligned (the transposed copy,
// written directly, only beside beta == 0)
bool tma_epilogue_ok(const SgemmOperands& o, float beta) {
  return (reinterpret_cast<uintptr_t>(o.c) & 15) == 0 && (o.ldc * 4) % 16 == 0 && !(o.ct && beta != 0.0f);
}
}  // namespace

int sgemm_tc_pair(int passes, const SgemmOperands& x, const SgemmOperands& y, int64_t n, int64_t k, float alpha,
                  float beta, unsigned* status, cudaStream_t stream, int max_ctas) {
  if (passes != 1 && passes != 3) return RM_BAD_ARG;
  if (n > INT32_MAX || k > INT32_MAX || k == 0) return RM_BAD_ARG;
  if (n == 0) return RM_OK;
  const SgemmOperands* live[2];
  int cnt = 0;
  if (x.m > 0) live[cnt++] = &x;
  if (y.m > 0) live[cnt++] = &y;
  if (cnt == 0) return RM_OK;
  const bool tma_epi = tma_epilogue_ok(*live[0], beta) && (cnt == 1 || tma_epilogue_ok(*live[1], beta));
  CUtensorMap maps[8];
  SgemmPart p[2];
  RM_TRY(prepare_part(*live[0], n, k, tma_epi, maps, &p[0]));
  if (cnt == 2) {
    RM_TRY(prepare_part(*live[1], n, k, tma_epi, maps + 3, &p[1]));
  } else {
    memcpy(maps + 3, maps, 3 * sizeof(CUtensorMap));
    p[1] = {nullptr, 0, nullptr, 0, 0, 0};
  }
  memcpy(maps + 6, maps, 2 * sizeof(CUtensorMap));  // no low parts from global memory
  const int ni = (int)n, ki = (int)k;
  if (passes == 3)
    return tma_epi ? launch_sgemm<3, true>(maps, p[0], p[1], ni, ki, alpha, beta, status, stream, max_ctas)
                   : launch_sgemm<3, false>(maps, p[0], p[1], ni, ki, alpha, beta, status, stream, max_ctas);
  return tma_epi ? launch_sgemm<1, true>(maps, p[0], p[1], ni, ki, alpha, beta, status, stream, max_ctas)
                 : launch_sgemm<1, false>(maps, p[0], p[1], ni, ki, alpha, beta, status, stream, max_ctas);
}

int sgemm_tc_lo(int64_t m, int64_t n, int64_t k, float alpha, const float* a, int64_t lda, const float* a_lo,
                int64_t ldal, const float* b, int64_t ldb, const float* b_lo, int64_t ldbl, float beta, float* c,
                int64_t ldc, unsigned* status, cudaStream_t stream, int max_ctas) {
  if (m == 0 || n == 0) return RM_OK;
  if (m > INT32_MAX || n > INT32_MAX || k > INT32_MAX || k == 0) return RM_BAD_ARG;
  const SgemmOperands x{m, a, lda, b, ldb, c, ldc, nullptr, 0};
  const bool tma_epi = tma_epilogue_ok(x, beta);
  CUtensorMap maps[8];
  SgemmPart p[2];
  RM_TRY(prepare_part(x, n, k, tma_epi, maps, &p[0]));
  memcpy(maps + 3, maps, 3 * sizeof(CUtensorMap));
  p[1] = {nullptr, 0, nullptr, 0, 0, 0};
  RM_TRY(make_tensor_map_2d(&maps[6], a_lo, 4, k, m, ldal * 4, tc::BK, tc::BM, true));
  RM_TRY(make_tensor_map_2d(&maps[7], b_lo, 4, k, n, ldbl * 4, tc::BK, tc::BN, true));
  return tma_epi ? launch_sgemm<3, true, true>(maps, p[0], p[1], (int)n, (int)k, alpha, beta, status, stream, max_ctas)
                 : launch_sgemm<3, false, true>(maps, p[0], p[1], (int)n, (int)k, alpha, beta, status, stream,
                                                max_ctas);
}

int sgemm_tc(int passes, int64_t m, int64_t n, int64_t k, float alpha, const float* a, int64_t lda, const float* b,
             int64_t ldb, float beta, float* c, int64_t ldc, unsigned* status, cudaStream_t stream, float* ct,
             int64_t ldct, int max_ctas) {
  if (m == 0 || n == 0) return RM_OK;
  if (m > INT32_MAX) return RM_BAD_ARG;
  const SgemmOperands x{m, a, lda, b, ldb, c, ldc, ct, ldct};
  const SgemmOperands none{0, nullptr, 0, nullptr, 0, nullptr, 0, nullptr, 0};
  return sgemm_tc_pair(passes, x, none, n, k, alpha, beta, status, stream, max_ctas);
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
