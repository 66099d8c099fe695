// Shared device helpers for the sm_100a kernels: status words, mbarriers, TMA, swizzle.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <utility>

#include "../../include/rm_cuda.h"

namespace rm {

// Bits of the device status word a launch may set (read by the host after the stream
// syncs). A bounded wait that gives up sets RM_DEV_TIMEOUT and returns; nothing traps.
enum : unsigned {
  RM_DEV_TIMEOUT = 1u << 0,
  RM_DEV_BAD_INDEX = 1u << 1,
  RM_DEV_NAN = 1u << 2,
};

// How long a wait on an mbarrier, a flag or a peer may last before it gives up.
constexpr uint64_t kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ void flag_error(unsigned* status, unsigned bits) {
  if (status) atomicOr(status, bits);
}

// ------------------------------------------------------------------ programmatic dependent launch
// A kernel launched with launch_dependent() may start while the kernel before it in the stream
// is still running: it does its set-up, then griddep_wait() returns once that kernel has
// completed and its memory is visible (at once for an ordinary launch). A kernel lets the next
// one start early with griddep_launch_dependents(); without it that happens at its end.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                                   Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// ------------------------------------------------------------------ mbarrier
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 1000000;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Waits for the phase with `parity` to complete; after kWaitLimitNs it gives up, sets the
// status bit and returns false, so that a lost arrival ends the launch instead of hanging it.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned* status) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t start = global_ns();
  for (;;) {
    for (int i = 0; i < 64; ++i)
      if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - start > kWaitLimitNs) break;
  }
  flag_error(status, RM_DEV_TIMEOUT);
  return false;
}

// ------------------------------------------------------------------ TMA
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

// Byte offset of item (row, col) of 8-byte items inside a tile whose rows are 128 B,
// written by TMA with CU_TENSOR_MAP_SWIZZLE_128B (16-byte chunks XOR the row's low 3 bits).
__device__ __forceinline__ uint32_t swz128_f64(uint32_t row, uint32_t col) {
  return row * 128u + ((((col >> 1) ^ (row & 7u)) << 4) | ((col & 1u) << 3));
}
// The same for 4-byte items (32 per 128-byte row).
__device__ __forceinline__ uint32_t swz128_f32(uint32_t row, uint32_t col) {
  return row * 128u + ((((col >> 2) ^ (row & 7u)) << 4) | ((col & 3u) << 2));
}

// ------------------------------------------------------------------ warp helpers
__device__ __forceinline__ bool elect_one() { return (threadIdx.x & 31) == 0; }

// 4-byte asynchronous copy global -> shared (no register staging; completes at cp_async_wait_all)
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// 16-byte asynchronous copy (both addresses 16-byte aligned), in the current commit group
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// waits until at most N of this thread's most recent commit groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

}  // namespace rm

// ------------------------------------------------------------------ host helpers
namespace rm {

#define RM_CUDA_TRY(expr)                                                   \
  do {                                                                      \
    cudaError_t _e = (expr);                                                \
    if (_e != cudaSuccess) {                                                \
      ::rm::set_last_error(_e, #expr, __FILE__, __LINE__);                  \
      return RM_CUDA_ERROR;                                                 \
    }                                                                       \
  } while (0)

// Counts a kernel launch (rm_launch_count) and turns a launch error into RM_CUDA_ERROR.
#define RM_LAUNCHED()                          \
  do {                                         \
    ::rm::note_launch();                       \
    RM_CUDA_TRY(cudaGetLastError());           \
  } while (0)

#define RM_TRY(expr)              \
  do {                            \
    int _s = (expr);              \
    if (_s != RM_OK) return _s;   \
  } while (0)

void set_last_error(cudaError_t e, const char* what, const char* file, int line);
void note_launch();
void set_last_message(const char* msg);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda needed).
// 2-D tensor of `elem_bytes` items: inner extent `inner` (contiguous), `outer` rows
// `row_stride_bytes` apart; box {box_inner, box_outer}; 128-byte swizzle when `swizzle`.
int make_tensor_map_2d(CUtensorMap* map, const void* base, int elem_bytes, uint64_t inner, uint64_t outer,
                       uint64_t row_stride_bytes, uint32_t box_inner, uint32_t box_outer, bool swizzle128);

int device_sm_count();

// Sets a function attribute of `kernel` (cudaFuncSetAttribute) on the current device, once per
// device and value: function attributes belong to one device's context, so a process that
// drives several GPUs sets them on each. Safe to call from several threads.
int func_attribute(const void* kernel, cudaFuncAttribute attr, int value);
template <typename K>
inline int smem_attribute(K* kernel, size_t bytes) {
  return func_attribute(reinterpret_cast<const void*>(kernel), cudaFuncAttributeMaxDynamicSharedMemorySize,
                        (int)bytes);
}

}  // namespace rm
