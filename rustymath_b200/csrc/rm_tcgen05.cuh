// Tensor-core helpers shared by the kernels: for tcgen05 (sgemm_tc.cu, ozaki.cu) shared-memory
// matrix descriptors, MMA completion, TMEM loads, TMA stores and bulk-group waits; for the
// warp-level products inside latency-bound kernels (getrs.cu, mixed.cu) TF32 rounding and
// mma.sync m16n8k8.
#pragma once
#include "rm_internal.h"

namespace rm {
namespace tc {

// UMMA shared-memory descriptor for a K-major tile written by TMA with 128-byte swizzle
// (rows of 128 bytes): 8-row groups 1024 bytes apart (stride byte offset), leading byte
// offset unused (1), descriptor version 1 (sm_100), layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                              // leading byte offset (>> 4)
  d |= (uint64_t)(1024 >> 4) << 32;                    // stride byte offset (>> 4)
  d |= (uint64_t)1 << 46;                              // version
  d |= (uint64_t)2 << 61;                              // SWIZZLE_128B
  return d;
}

// Arrives on the mbarrier once every MMA this thread issued before has completed.
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

__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, const void* src, int x, int y) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(map),
               "r"(smem_u32(src)), "r"(x), "r"(y)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Byte offset of float (row r, column j) in a 32 x 32 chunk written by TMA with 128-byte swizzle.
__device__ __forceinline__ uint32_t chunk_off(int r, int j) {
  return (uint32_t)(r * 128 + ((((j >> 2) ^ (r & 7)) << 4) | ((j & 3) << 2)));
}

// Allocates `cols` TMEM columns (a power of two >= 32) for the CTA: the warp that calls it
// writes the base address to *slot; relinquishes the permit so other CTAs can allocate.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(cols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols));
}

// x rounded to TF32 (round to nearest, ties away), in a 32-bit register
__device__ __forceinline__ uint32_t to_tf32(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return r;
}

// d += A B for a 16 x 8 tile: A 16 x 8 (row), B 8 x 8 (col), TF32 in, float32 accumulate
__device__ __forceinline__ void mma_tf32_16x8x8(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// 3xTF32: d += A B with float32-level products (A = Ah + Al, B = Bh + Bl in TF32; Al Bl dropped)
__device__ __forceinline__ void mma_3xtf32(float (&d)[4], const float (&a)[4], float b0, float b1) {
  uint32_t ah[4], al[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    ah[i] = to_tf32(a[i]);
    al[i] = to_tf32(a[i] - __uint_as_float(ah[i]));
  }
  const uint32_t bh0 = to_tf32(b0), bh1 = to_tf32(b1);
  const uint32_t bl0 = to_tf32(b0 - __uint_as_float(bh0)), bl1 = to_tf32(b1 - __uint_as_float(bh1));
  mma_tf32_16x8x8(d, al, bh0, bh1);  // the small terms first
  mma_tf32_16x8x8(d, ah, bl0, bl1);
  mma_tf32_16x8x8(d, ah, bh0, bh1);
}

}  // namespace tc
}  // namespace rm
