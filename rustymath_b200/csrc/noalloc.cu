// rm_dlu_solve_noalloc: the LU triangular solves with no device allocation at all.
//
// Some callers cannot allocate device memory during a call: code running under a strict
// memory budget or arena that owns every device allocation, real-time loops that must not
// hit the driver's allocator, and hosts that pre-plan all memory up front. For them this
// entry point runs the same kernels as rm_dlu_solve, with the scratch those kernels need
// (the inverted diagonal blocks, the permuted right-hand side and the solve's dependency
// flags) in one file-scope __device__ array of fixed size instead of stream-ordered
// allocations.
#include <mutex>
#include <vector>

#include "rm_internal.h"

namespace rm {

// Scratch for n <= RM_NOALLOC_MAX_N, k <= RM_NOALLOC_MAX_K: inverted diagonal blocks,
// then the solve's permuted right-hand side and flags.
constexpr size_t kNoallocBytes =
    ((diag_blocks_bytes_max(RM_NOALLOC_MAX_N) + 255) / 256) * 256 + getrs_scratch_bytes_max(RM_NOALLOC_MAX_N, RM_NOALLOC_MAX_K);
static_assert(kNoallocBytes == RM_NOALLOC_SCRATCH_BYTES, "the header states the array's size");

// Every GPU that loads this library holds this array until the process exits. All calls
// share it; each call leaves its contents behind for the next.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

// The device address of g_noalloc_scratch for the current device, looked up once per
// device (in host code the symbol's name is only a stand-in, not a device address).
static int noalloc_scratch(void** out) {
  static std::mutex mu;
  static std::vector<void*> addr;
  int dev = 0;
  RM_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if ((int)addr.size() <= dev) addr.resize(dev + 1, nullptr);
  if (!addr[dev]) {
    void* p = nullptr;
    RM_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    addr[dev] = p;
  }
  *out = addr[dev];
  return RM_OK;
}

}  // namespace rm

using namespace rm;

extern "C" int rm_dlu_solve_noalloc(int64_t n, const double* d_factors, const int64_t* d_perm, const double* d_b,
                                    int64_t k, double* d_x, int trans, void* stream) {
  if (n < 0 || k < 0 || (trans != 0 && trans != 1)) return RM_BAD_ARG;
  if (n > RM_NOALLOC_MAX_N || k > RM_NOALLOC_MAX_K) {
    set_last_message("rm_dlu_solve_noalloc takes n <= RM_NOALLOC_MAX_N and k <= RM_NOALLOC_MAX_K");
    return RM_BAD_ARG;
  }
  if (n == 0 || k == 0) return RM_OK;
  if (!d_factors || !d_perm || !d_b || !d_x) return RM_BAD_ARG;
  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    set_last_message("no CUDA device");
    return RM_NO_DEVICE;
  }
  RM_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  if (major != 10) return RM_NO_DEVICE;
  void* base = nullptr;
  RM_TRY(noalloc_scratch(&base));
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  double* dinv = static_cast<double*>(base);
  void* rest = static_cast<char*>(base) + (diag_blocks_f64_bytes(n) + 255) / 256 * 256;
  // getrs_f64 clears the dependency flags it uses before its kernels run.
  const DiagBlockArgs da = diag_block_args(trans != 0, true);
  RM_TRY(invert_diag_blocks_f64(d_factors, n, da.colmajor, n, dinv, da.lower_unit, da.upper_unit, s));
  return getrs_f64(d_factors, n, true, n, d_perm, dinv, d_b, k, k, d_x, k, rest, device_status(), s, trans != 0);
}
