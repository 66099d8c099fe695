// The C ABI (include/rm_cuda.h): argument checks, scratch, and the call sequences of the
// plain float64 path. Every entry point returns an rm status code; nothing here falls back
// to the CPU.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "rm_internal.h"

namespace rm {

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;

void set_last_message(const char* msg) { g_last_error = msg ? msg : ""; }

void set_last_error(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof buf, "%s: %s (%s:%d)", cudaGetErrorString(e), what, file, line);
  g_last_error = buf;
}

int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

static std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// ------------------------------------------------------------------ device facts
int device_sm_count() {
  static std::mutex mu;
  static std::vector<int> counts;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> lock(mu);
  if ((int)counts.size() <= dev) counts.resize(dev + 1, 0);
  if (counts[dev] == 0) {
    int c = 0;
    if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c <= 0) c = 148;
    counts[dev] = c;
  }
  return counts[dev];
}

int func_attribute(const void* kernel, cudaFuncAttribute attr, int value) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void*, int>, int> done;  // (device, kernel, attribute) -> value
  int dev = 0;
  RM_CUDA_TRY(cudaGetDevice(&dev));
  const auto key = std::make_tuple(dev, kernel, (int)attr);
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = done.find(key);
    if (it != done.end() && it->second == value) return RM_OK;
  }
  RM_CUDA_TRY(cudaFuncSetAttribute(kernel, attr, value));
  std::lock_guard<std::mutex> lock(mu);
  done[key] = value;
  return RM_OK;
}

__device__ unsigned g_device_status;

unsigned* device_status() {
  static std::mutex mu;
  static std::vector<unsigned*> ptrs;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if ((int)ptrs.size() <= dev) ptrs.resize(dev + 1, nullptr);
  if (!ptrs[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_device_status) != cudaSuccess) return nullptr;
    ptrs[dev] = static_cast<unsigned*>(p);
  }
  return ptrs[dev];
}

// Maps a status word read back from the device to a status code and clears the word.
static int status_from_word(unsigned h, unsigned* st, cudaStream_t stream) {
  if (h) {
    RM_CUDA_TRY(cudaMemsetAsync(st, 0, sizeof(unsigned), stream));
    if (h & RM_DEV_TIMEOUT) {
      set_last_message("a bounded device-side wait gave up");
      return RM_TIMEOUT;
    }
    if (h & RM_DEV_BAD_INDEX) {
      set_last_message("a row position is outside 0..n-1");
      return RM_BAD_ARG;
    }
  }
  return RM_OK;
}

int take_device_status(cudaStream_t stream) {
  unsigned* st = device_status();
  if (!st) return RM_CUDA_ERROR;
  unsigned h = 0;
  RM_CUDA_TRY(cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, stream));
  RM_CUDA_TRY(cudaStreamSynchronize(stream));
  return status_from_word(h, st, stream);
}

// What a synchronous call reads back at its end, in page-locked memory so that the copies stay
// asynchronous and the host waits once. One block per host thread, allocated at its first use
// and kept until the process exits.
struct alignas(16) CallResults {
  unsigned status;
  int32_t flag;
  double berr[2];
};

static CallResults* call_results() {
  static thread_local CallResults* p = nullptr;
  if (!p && cudaHostAlloc(reinterpret_cast<void**>(&p), sizeof(CallResults), cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    p = nullptr;
  }
  return p;
}

// Ends a synchronous call with one wait: the device status word, and the int32 flag and two
// doubles at d_flag / d_berr when given, read back together. The status word's errors come first.
static int finish_call(cudaStream_t s, const int32_t* d_flag, int32_t* flag, const double* d_berr, double* berr) {
  unsigned* st = device_status();
  if (!st) return RM_CUDA_ERROR;
  CallResults* h = call_results();
  if (!h) {  // no page-locked block: one pageable read each
    if (d_flag) RM_CUDA_TRY(cudaMemcpyAsync(flag, d_flag, sizeof *flag, cudaMemcpyDeviceToHost, s));
    if (d_berr) RM_CUDA_TRY(cudaMemcpyAsync(berr, d_berr, 2 * sizeof *berr, cudaMemcpyDeviceToHost, s));
    return take_device_status(s);
  }
  RM_CUDA_TRY(cudaMemcpyAsync(&h->status, st, sizeof h->status, cudaMemcpyDeviceToHost, s));
  if (d_flag) RM_CUDA_TRY(cudaMemcpyAsync(&h->flag, d_flag, sizeof h->flag, cudaMemcpyDeviceToHost, s));
  if (d_berr) RM_CUDA_TRY(cudaMemcpyAsync(h->berr, d_berr, sizeof h->berr, cudaMemcpyDeviceToHost, s));
  RM_CUDA_TRY(cudaStreamSynchronize(s));
  if (d_flag) *flag = h->flag;
  if (d_berr) berr[0] = h->berr[0], berr[1] = h->berr[1];
  return status_from_word(h->status, st, s);
}

// ------------------------------------------------------------------ failure injection (tests)
// Per thread and RM_INJECT_* kind: how many events pass before the next failures, and how
// many fail then.
static thread_local int g_inject_after[3] = {0, 0, 0};
static thread_local int g_inject_count[3] = {0, 0, 0};

bool injected_failure(int kind) {
  if (kind < 1 || kind > 2 || g_inject_count[kind] <= 0) return false;
  if (g_inject_after[kind] > 0) {
    --g_inject_after[kind];
    return false;
  }
  --g_inject_count[kind];
  return true;
}

// ------------------------------------------------------------------ scratch
int scratch_alloc(void** p, size_t bytes, cudaStream_t stream) {
  *p = nullptr;
  if (bytes == 0) return RM_OK;
  if (injected_failure(RM_INJECT_CUDA_ERROR)) {
    set_last_message("cudaMallocAsync failed (injected by rm_test_inject_failure)");
    return RM_CUDA_ERROR;
  }
  {
    // Keep freed scratch in each device's default pool between calls instead of returning it
    // to the driver (once per device).
    static std::mutex mu;
    static std::vector<bool> pool_set;
    int dev = 0;
    RM_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if ((int)pool_set.size() <= dev) pool_set.resize(dev + 1, false);
    cudaMemPool_t pool;
    if (!pool_set[dev] && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t threshold = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
      pool_set[dev] = true;
    }
  }
  cudaError_t e = injected_failure(RM_INJECT_OUT_OF_MEMORY) ? cudaErrorMemoryAllocation
                                                            : cudaMallocAsync(p, bytes, stream);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    set_last_message("device memory exhausted");
    return RM_OUT_OF_MEMORY;
  }
  RM_CUDA_TRY(e);
  return RM_OK;
}

void scratch_free(void* p, cudaStream_t stream) {
  if (p) cudaFreeAsync(p, stream);
}

// Carves aligned sub-buffers out of one stream-ordered allocation.
struct Arena {
  std::vector<size_t> offsets;
  size_t total = 0;
  size_t add(size_t bytes) {
    const size_t off = total;
    total = (total + bytes + 255) / 256 * 256;
    return off;
  }
};

struct Scratch {
  void* base = nullptr;
  cudaStream_t stream = nullptr;
  ~Scratch() { scratch_free(base, stream); }
  template <typename T>
  T* at(size_t off) const {
    return reinterpret_cast<T*>(static_cast<char*>(base) + off);
  }
};

// ------------------------------------------------------------------ TMA descriptors
int make_tensor_map_2d(CUtensorMap* map, const void* base, int elem_bytes, uint64_t inner, uint64_t outer,
                       uint64_t row_stride_bytes, uint32_t box_inner, uint32_t box_outer, bool swizzle128) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  if (!encode) {
    set_last_message("cuTensorMapEncodeTiled is unavailable");
    return RM_CUDA_ERROR;
  }
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (row_stride_bytes & 15)) {
    set_last_message("a TMA operand needs a 16-byte aligned base and row stride");
    return RM_BAD_ARG;
  }
  CUtensorMapDataType dt = elem_bytes == 8   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                           : elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                           : elem_bytes == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                             : CU_TENSOR_MAP_DATA_TYPE_UINT8;
  cuuint64_t dims[2] = {inner, std::max<uint64_t>(outer, 1)};
  cuuint64_t strides[1] = {std::max<uint64_t>(row_stride_bytes, 16)};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char buf[160];
    snprintf(buf, sizeof buf, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    set_last_message(buf);
    return RM_CUDA_ERROR;
  }
  return RM_OK;
}

// ------------------------------------------------------------------ transpose
__global__ void transpose_kernel(const double* __restrict__ src, int64_t lds, int64_t m, int64_t n,
                                 double* __restrict__ dst, int64_t ldd) {
  __shared__ double tile[32][33];
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

int transpose_f64(const double* src, int64_t lds, int64_t m, int64_t n, double* dst, int64_t ldd, cudaStream_t stream) {
  if (m == 0 || n == 0) return RM_OK;
  dim3 grid((unsigned)((n + 31) / 32), (unsigned)((m + 31) / 32));
  transpose_kernel<<<grid, dim3(32, 8), 0, stream>>>(src, lds, m, n, dst, ldd);
  RM_LAUNCHED();
  return RM_OK;
}

// ------------------------------------------------------------------ plain solve pieces

// The working copy of an n x n system: W (row-major, ld a multiple of 32), pivots, perm.
struct LuBuffers {
  size_t w, ipiv, perm, amax, flag, dinv, getrf, rowabs, berr;
  int64_t ldw;
};

static LuBuffers plan_lu(Arena& arena, int64_t n) {
  LuBuffers b;
  b.ldw = round_up(std::max<int64_t>(n, 1), 32);
  b.w = arena.add((size_t)n * b.ldw * sizeof(double));
  b.ipiv = arena.add((size_t)n * sizeof(int64_t));
  b.perm = arena.add((size_t)n * sizeof(int64_t));
  b.amax = arena.add(sizeof(double));
  b.flag = arena.add(sizeof(int32_t));
  b.dinv = arena.add(diag_blocks_f64_bytes(n));
  b.getrf = arena.add(getrf_f64_scratch_bytes(n));
  b.rowabs = arena.add(sizeof(double));
  b.berr = arena.add(2 * sizeof(double));
  return b;
}

static cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

int check_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_last_message("no CUDA device");
    return RM_NO_DEVICE;
  }
  int major = 0;
  RM_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  if (major != 10) {
    set_last_message("librm_cuda needs a compute capability 10.x device (B200, sm_100a)");
    return RM_NO_DEVICE;
  }
  return RM_OK;
}

}  // namespace rm

using namespace rm;

// ================================================================== C ABI
extern "C" {

int rm_version(void) { return 100; }

int64_t rm_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

const char* rm_status_string(int status) {
  switch (status) {
    case RM_OK: return "ok";
    case RM_BAD_ARG: return "bad argument";
    case RM_NOT_REGULAR: return "matrix not regular (a pivot at most eps*n*max|a|)";
    case RM_CUDA_ERROR: return "CUDA error";
    case RM_TIMEOUT: return "device-side wait timed out";
    case RM_NO_CONVERGENCE: return "refinement did not converge";
    case RM_NO_DEVICE: return "no compute capability 10.x device";
    case RM_OUT_OF_MEMORY: return "out of device memory";
    case RM_NOT_POSITIVE_DEFINITE: return "matrix not positive definite (a Cholesky pivot is not > 0)";
    default: return "unknown status";
  }
}

int rm_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return RM_BAD_ARG;
  const std::string& s = g_last_error;
  const size_t n = std::min(len - 1, s.size());
  memcpy(buf, s.data(), n);
  buf[n] = 0;
  return RM_OK;
}

int rm_take_status(void* stream) {
  RM_TRY(check_device());
  return take_device_status(as_stream(stream));
}

int rm_test_inject_failure(int kind, int after, int count) {
  if (kind < 1 || kind > 2 || after < 0 || count < 0) return RM_BAD_ARG;
  g_inject_after[kind] = after;
  g_inject_count[kind] = count;
  return RM_OK;
}

int rm_test_chain_timeout(int64_t wait_ns) {
  if (wait_ns < 1000 || wait_ns > 2000000000) return RM_BAD_ARG;
  RM_TRY(check_device());
  cudaStream_t s;
  RM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  int st = RM_OK;
  {
    Scratch sc;
    sc.stream = s;
    st = scratch_alloc(&sc.base, chain_timeout_scratch_bytes(), s);
    unsigned bits = 0;
    if (st == RM_OK) st = chain_timeout_run((uint64_t)wait_ns, sc.base, &bits, s);
    if (st == RM_OK) st = (bits & RM_DEV_TIMEOUT) ? RM_TIMEOUT : RM_OK;
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (st != RM_CUDA_ERROR && e != cudaSuccess) {
    set_last_error(e, "stream synchronize", __FILE__, __LINE__);
    st = RM_CUDA_ERROR;
  }
  cudaStreamDestroy(s);
  return st;
}

int rm_device_count(int* count) {
  if (!count) return RM_BAD_ARG;
  *count = 0;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return RM_OK;
  }
  for (int d = 0; d < n; ++d) {
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, d) == cudaSuccess && major == 10) ++*count;
  }
  return RM_OK;
}

int rm_dtrsm(int side, int uplo, int trans, int diag, int64_t m, int64_t n, const double* d_a, int64_t lda,
             double* d_x, int64_t ldx, void* stream) {
  if ((side != RM_LEFT && side != RM_RIGHT) || (uplo != RM_UPPER && uplo != RM_LOWER) ||
      (trans != RM_CBLAS_NO_TRANS && trans != RM_CBLAS_TRANS) || (diag != RM_NON_UNIT && diag != RM_UNIT) || m < 0 ||
      n < 0)
    return RM_BAD_ARG;
  if (m == 0 || n == 0) return RM_OK;
  const bool right = side == RM_RIGHT;
  const int64_t order = right ? n : m;
  if (lda < order || ldx < n || !d_a || !d_x) return RM_BAD_ARG;
  RM_TRY(check_device());
  cudaStream_t s = as_stream(stream);
  Scratch sc;
  sc.stream = s;
  RM_TRY(scratch_alloc(&sc.base, trsm_f64_scratch_bytes(order, m, n, right), s));
  RM_TRY(trsm_f64(right, uplo == RM_LOWER, trans == RM_CBLAS_TRANS, diag == RM_UNIT, m, n, d_a, lda, d_x, ldx, sc.base,
                  device_status(), s));
  return take_device_status(s);
}

int rm_dgemm_ozaki(int64_t m, int64_t n, int64_t k, const double* d_a, int64_t lda, const double* d_b, int64_t ldb,
                   double* d_c, int64_t ldc, int slices, void* stream) {
  if (m < 0 || n < 0 || k < 0 || slices < 1 || slices > 8) return RM_BAD_ARG;
  if (m == 0 || n == 0) return RM_OK;
  if (ldc < n || (k > 0 && (lda < k || ldb < n)) || !d_c || (k > 0 && (!d_a || !d_b))) return RM_BAD_ARG;
  RM_TRY(check_device());
  cudaStream_t s = as_stream(stream);
  Scratch sc;
  sc.stream = s;
  RM_TRY(scratch_alloc(&sc.base, ozaki_scratch_bytes(m, n, k, slices), s));
  RM_TRY(dgemm_ozaki(m, n, k, d_a, lda, d_b, ldb, d_c, ldc, slices, sc.base, device_status(), s));
  return RM_OK;
}

int rm_dgemm(int transa, int transb, int64_t m, int64_t n, int64_t k, double alpha, const double* d_a, int64_t lda,
             const double* d_b, int64_t ldb, double beta, double* d_c, int64_t ldc, void* stream) {
  if (m < 0 || n < 0 || k < 0 || (transa != 0 && transa != 1) || (transb != 0 && transb != 1)) return RM_BAD_ARG;
  if (m == 0 || n == 0) return RM_OK;
  const int64_t acols = transa ? m : k, bcols = transb ? k : n;
  if (ldc < n || (k > 0 && (lda < std::max<int64_t>(acols, 1) || ldb < std::max<int64_t>(bcols, 1)))) return RM_BAD_ARG;
  if (!d_c || (k > 0 && alpha != 0.0 && (!d_a || !d_b))) return RM_BAD_ARG;
  RM_TRY(check_device());
  cudaStream_t s = as_stream(stream);
  if (k == 0 || alpha == 0.0) return scale_device(d_c, ldc, m, n, beta, s);
  // one output row or column: by_vector's case (linalg.rs:1020-1073), an HBM-bound stream
  if (m == 1 || n == 1) return gemv_device(transa, transb, m, n, k, alpha, d_a, lda, d_b, ldb, beta, d_c, ldc, s);
  // TMA wants 16-byte aligned rows: copy misaligned operands into padded buffers.
  const double* a = d_a;
  const double* b = d_b;
  int64_t la = lda, lb = ldb;
  Scratch sc;
  sc.stream = s;
  const bool fix_a = (reinterpret_cast<uintptr_t>(d_a) & 15) || (lda & 1);
  const bool fix_b = (reinterpret_cast<uintptr_t>(d_b) & 15) || (ldb & 1);
  if (fix_a || fix_b) {
    Arena ar;
    const int64_t arows = transa ? k : m, brows = transb ? n : k;
    const int64_t pa = round_up(acols, 2), pb = round_up(bcols, 2);
    const size_t oa = fix_a ? ar.add((size_t)arows * pa * sizeof(double)) : 0;
    const size_t ob = fix_b ? ar.add((size_t)brows * pb * sizeof(double)) : 0;
    RM_TRY(scratch_alloc(&sc.base, ar.total, s));
    if (fix_a) {
      RM_CUDA_TRY(cudaMemcpy2DAsync(sc.at<double>(oa), pa * sizeof(double), d_a, lda * sizeof(double),
                                    acols * sizeof(double), arows, cudaMemcpyDeviceToDevice, s));
      a = sc.at<double>(oa);
      la = pa;
    }
    if (fix_b) {
      RM_CUDA_TRY(cudaMemcpy2DAsync(sc.at<double>(ob), pb * sizeof(double), d_b, ldb * sizeof(double),
                                    bcols * sizeof(double), brows, cudaMemcpyDeviceToDevice, s));
      b = sc.at<double>(ob);
      lb = pb;
    }
  }
  return dgemm_device(transa != 0, transb != 0, m, n, k, alpha, a, la, b, lb, beta, d_c, ldc, device_status(), s);
}

int rm_dgemm_host(int transa, int transb, int64_t m, int64_t n, int64_t k, double alpha, const double* h_a,
                  int64_t lda, const double* h_b, int64_t ldb, double beta, double* h_c, int64_t ldc) {
  if (m < 0 || n < 0 || k < 0 || (transa != 0 && transa != 1) || (transb != 0 && transb != 1)) return RM_BAD_ARG;
  if (m == 0 || n == 0) return RM_OK;
  const int64_t arows = transa ? k : m, acols = transa ? m : k;
  const int64_t brows = transb ? n : k, bcols = transb ? k : n;
  if (ldc < n || (k > 0 && (lda < std::max<int64_t>(acols, 1) || ldb < std::max<int64_t>(bcols, 1)))) return RM_BAD_ARG;
  if (!h_c || (k > 0 && (!h_a || !h_b))) return RM_BAD_ARG;
  RM_TRY(check_device());
  cudaStream_t s;
  RM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  int st = RM_OK;
  {
    Arena ar;
    const int64_t pa = round_up(std::max<int64_t>(acols, 1), 2), pb = round_up(std::max<int64_t>(bcols, 1), 2);
    const size_t oa = ar.add((size_t)arows * pa * sizeof(double));
    const size_t ob = ar.add((size_t)brows * pb * sizeof(double));
    const size_t oc = ar.add((size_t)m * n * sizeof(double));
    Scratch sc;
    sc.stream = s;
    st = scratch_alloc(&sc.base, ar.total, s);
    if (st == RM_OK) {
      cudaError_t e = cudaSuccess;
      if (k > 0) {
        e = cudaMemcpy2DAsync(sc.at<double>(oa), pa * 8, h_a, lda * 8, acols * 8, arows, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
          e = cudaMemcpy2DAsync(sc.at<double>(ob), pb * 8, h_b, ldb * 8, bcols * 8, brows, cudaMemcpyHostToDevice, s);
      }
      if (e == cudaSuccess && beta != 0.0)
        e = cudaMemcpy2DAsync(sc.at<double>(oc), n * 8, h_c, ldc * 8, n * 8, m, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) {
        set_last_error(e, "host to device copy", __FILE__, __LINE__);
        st = RM_CUDA_ERROR;
      }
      if (st == RM_OK)
        st = rm_dgemm(transa, transb, m, n, k, alpha, sc.at<double>(oa), pa, sc.at<double>(ob), pb, beta,
                      sc.at<double>(oc), n, s);
      if (st == RM_OK) {
        e = cudaMemcpy2DAsync(h_c, ldc * 8, sc.at<double>(oc), n * 8, n * 8, m, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) {
          set_last_error(e, "device to host copy", __FILE__, __LINE__);
          st = RM_CUDA_ERROR;
        }
      }
    }
  }
  if (st == RM_OK) st = take_device_status(s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (st == RM_OK && e != cudaSuccess) {
    set_last_error(e, "stream synchronize", __FILE__, __LINE__);
    st = RM_CUDA_ERROR;
  }
  cudaStreamDestroy(s);
  return st;
}

int rm_sgemm_tc(int passes, int transb, int64_t m, int64_t n, int64_t k, float alpha, const float* d_a, int64_t lda,
                const float* d_b, int64_t ldb, float beta, float* d_c, int64_t ldc, void* stream) {
  if (m < 0 || n < 0 || k < 0 || (passes != 1 && passes != 3) || (transb != 0 && transb != 1)) return RM_BAD_ARG;
  if (m == 0 || n == 0) return RM_OK;
  const int64_t bcols = transb ? k : n;
  if (ldc < n || (k > 0 && (lda < k || ldb < bcols)) || !d_c || (k > 0 && (!d_a || !d_b))) return RM_BAD_ARG;
  RM_TRY(check_device());
  cudaStream_t s = as_stream(stream);
  if (k == 0 || alpha == 0.0f) return scale_f32(d_c, ldc, m, n, beta, s);
  // operands go to 16-byte aligned, padded copies when needed; a k x n B is transposed
  // into n x k (the tensor cores read both operands with k contiguous)
  const bool fix_a = (reinterpret_cast<uintptr_t>(d_a) & 15) || (lda & 3);
  const bool fix_b = !transb || (reinterpret_cast<uintptr_t>(d_b) & 15) || (ldb & 3);
  const int64_t pa = round_up(k, 4), pb = round_up(k, 4);
  // a rank-k update (three passes, k <= 256): the operands' low parts go to global memory once,
  // and the kernel loads them beside the operands instead of forming them per output tile
  const bool lo_g = passes == 3 && k <= 256;
  Arena ar;
  const size_t oa = fix_a ? ar.add((size_t)m * pa * 4) : 0, ob = fix_b ? ar.add((size_t)n * pb * 4) : 0;
  const size_t oal = lo_g ? ar.add((size_t)m * pa * 4) : 0, obl = lo_g ? ar.add((size_t)n * pb * 4) : 0;
  Scratch sc;
  sc.stream = s;
  if (ar.total) RM_TRY(scratch_alloc(&sc.base, ar.total, s));
  const float* a = d_a;
  const float* b = d_b;
  int64_t la = lda, lb = ldb;
  if (fix_a) {
    RM_CUDA_TRY(cudaMemcpy2DAsync(sc.at<float>(oa), pa * 4, d_a, lda * 4, k * 4, m, cudaMemcpyDeviceToDevice, s));
    a = sc.at<float>(oa);
    la = pa;
  }
  if (fix_b) {
    if (transb) {
      RM_CUDA_TRY(cudaMemcpy2DAsync(sc.at<float>(ob), pb * 4, d_b, ldb * 4, k * 4, n, cudaMemcpyDeviceToDevice, s));
    } else {
      RM_TRY(transpose_f32(d_b, ldb, k, n, sc.at<float>(ob), pb, s));
    }
    b = sc.at<float>(ob);
    lb = pb;
  }
  if (lo_g) {
    float* al = sc.at<float>(oal);
    float* bl = sc.at<float>(obl);
    RM_TRY(split_lo_f32(a, la, m, k, al, pa, s));
    RM_TRY(split_lo_f32(b, lb, n, k, bl, pb, s));
    return sgemm_tc_lo(m, n, k, alpha, a, la, al, pa, b, lb, bl, pb, beta, d_c, ldc, device_status(), s);
  }
  return sgemm_tc(passes, m, n, k, alpha, a, la, b, lb, beta, d_c, ldc, device_status(), s);
}

int rm_dlu_factor(int64_t n, const double* d_a, double* d_factors, int64_t* d_perm, int32_t* h_regular, void* stream) {
  if (n < 0 || (n > 0 && (!d_a || !d_factors || !d_perm))) return RM_BAD_ARG;
  if (h_regular) *h_regular = 0;
  if (n == 0) return RM_OK;
  RM_TRY(check_device());
  cudaStream_t s = as_stream(stream);
  Arena ar;
  LuBuffers lb = plan_lu(ar, n);
  Scratch sc;
  sc.stream = s;
  RM_TRY(scratch_alloc(&sc.base, ar.total, s));
  double* w = sc.at<double>(lb.w);
  RM_TRY(load_matrix_f64(d_a, n, w, lb.ldw, n, sc.at<double>(lb.amax), s));
  RM_TRY(getrf_f64(w, lb.ldw, n, sc.at<int64_t>(lb.ipiv), d_perm, sc.at<void>(lb.getrf), device_status(), s));
  RM_TRY(store_factors_f64(w, lb.ldw, n, d_factors, s));
  if (h_regular) {
    RM_TRY(regular_flag_f64(w, lb.ldw, n, sc.at<double>(lb.amax), sc.at<int32_t>(lb.flag), s));
    RM_CUDA_TRY(cudaMemcpyAsync(h_regular, sc.at<int32_t>(lb.flag), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    RM_TRY(take_device_status(s));
  }
  return RM_OK;
}

int rm_dlu_factor_host(int64_t n, const double* h_a, double* h_factors, int64_t* h_perm, int32_t* h_regular) {
  if (n < 0 || (n > 0 && (!h_a || !h_factors || !h_perm))) return RM_BAD_ARG;
  if (h_regular) *h_regular = 0;
  if (n == 0) return RM_OK;
  RM_TRY(check_device());
  cudaStream_t s;
  RM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  int st;
  {
    Arena ar;
    const size_t oa = ar.add((size_t)n * n * 8), of = ar.add((size_t)n * n * 8), op = ar.add((size_t)n * 8);
    Scratch sc;
    sc.stream = s;
    st = scratch_alloc(&sc.base, ar.total, s);
    if (st == RM_OK) {
      cudaError_t e = cudaMemcpyAsync(sc.at<double>(oa), h_a, (size_t)n * n * 8, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) { set_last_error(e, "copy", __FILE__, __LINE__); st = RM_CUDA_ERROR; }
      if (st == RM_OK) st = rm_dlu_factor(n, sc.at<double>(oa), sc.at<double>(of), sc.at<int64_t>(op), h_regular, s);
      if (st == RM_OK) {
        e = cudaMemcpyAsync(h_factors, sc.at<double>(of), (size_t)n * n * 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_perm, sc.at<int64_t>(op), (size_t)n * 8, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) { set_last_error(e, "copy", __FILE__, __LINE__); st = RM_CUDA_ERROR; }
      }
    }
  }
  if (st == RM_OK) st = take_device_status(s);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  return st;
}

int rm_dlu_solve(int64_t n, const double* d_factors, const int64_t* d_perm, const double* d_b, int64_t k, double* d_x,
                 int trans, void* stream) {
  if (n < 0 || k < 0 || (trans != 0 && trans != 1)) return RM_BAD_ARG;
  if (n == 0 || k == 0) return RM_OK;
  if (!d_factors || !d_perm || !d_b || !d_x) return RM_BAD_ARG;
  RM_TRY(check_device());
  cudaStream_t s = as_stream(stream);
  // n <= 192, k <= 8: one CTA in rustymath's single-column order, no scratch
  if (!trans && small_solve_fits(n, k))
    return small_solve_f64(d_factors, n, true, n, d_perm, d_b, k, d_x, device_status(), s);
  Arena ar;
  const size_t od = ar.add(diag_blocks_f64_bytes(n)), os = ar.add(getrs_f64_scratch_bytes(n, k));
  Scratch sc;
  sc.stream = s;
  RM_TRY(scratch_alloc(&sc.base, ar.total, s));
  // The factors are column-major (rustymath's order); the kernels read them in place.
  const DiagBlockArgs da = diag_block_args(trans != 0, true);
  RM_TRY(invert_diag_blocks_f64(d_factors, n, da.colmajor, n, sc.at<double>(od), da.lower_unit, da.upper_unit, s));
  return getrs_f64(d_factors, n, true, n, d_perm, sc.at<double>(od), d_b, k, k, d_x, k, sc.at<void>(os),
                   device_status(), s, trans != 0);
}

int rm_dlu_solve_host(int64_t n, const double* h_factors, const int64_t* h_perm, const double* h_b, int64_t k,
                      double* h_x, int trans) {
  if (n < 0 || k < 0) return RM_BAD_ARG;
  if (n == 0 || k == 0) return RM_OK;
  if (!h_factors || !h_perm || !h_b || !h_x) return RM_BAD_ARG;
  RM_TRY(check_device());
  cudaStream_t s;
  RM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  int st;
  {
    Arena ar;
    const size_t of = ar.add((size_t)n * n * 8), op = ar.add((size_t)n * 8), ob = ar.add((size_t)n * k * 8);
    Scratch sc;
    sc.stream = s;
    st = scratch_alloc(&sc.base, ar.total, s);
    if (st == RM_OK) {
      cudaError_t e = cudaMemcpyAsync(sc.at<double>(of), h_factors, (size_t)n * n * 8, cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(sc.at<int64_t>(op), h_perm, (size_t)n * 8, cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(sc.at<double>(ob), h_b, (size_t)n * k * 8, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) { set_last_error(e, "copy", __FILE__, __LINE__); st = RM_CUDA_ERROR; }
      if (st == RM_OK)
        st = rm_dlu_solve(n, sc.at<double>(of), sc.at<int64_t>(op), sc.at<double>(ob), k, sc.at<double>(ob), trans, s);
      if (st == RM_OK) {
        e = cudaMemcpyAsync(h_x, sc.at<double>(ob), (size_t)n * k * 8, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) { set_last_error(e, "copy", __FILE__, __LINE__); st = RM_CUDA_ERROR; }
      }
    }
  }
  if (st == RM_OK) st = take_device_status(s);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  return st;
}

// The plain float64 solve: LU, LuWork::regular's test, then the two triangular solves.
// Phase timing for the solves, on when the environment sets RM_TRACE: CUDA events recorded
// on the solve's stream between phases, printed to stderr once the solve has synchronised.
struct PhaseTrace {
  static constexpr int kMax = 96;
  bool on = false;
  int count = 0;
  cudaEvent_t ev[kMax];
  const char* name[kMax];
  cudaStream_t stream;
  PhaseTrace(cudaStream_t s, const char* what) : stream(s) {
    static const bool enabled = std::getenv("RM_TRACE") != nullptr;
    on = enabled;
    if (on) {
      std::fprintf(stderr, "rm trace: %s\n", what);
      mark("start");
    }
  }
  void mark(const char* what) {
    if (!on || count == kMax) return;
    if (cudaEventCreate(&ev[count]) != cudaSuccess) return;
    name[count] = what;
    cudaEventRecord(ev[count++], stream);
  }
  ~PhaseTrace() {
    if (!on) return;
    cudaEventSynchronize(ev[count - 1]);
    float total = 0.0f;
    for (int i = 1; i < count; ++i) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, ev[i - 1], ev[i]);
      total += ms;
      std::fprintf(stderr, "  %-14s %9.3f ms\n", name[i], ms);
    }
    std::fprintf(stderr, "  %-14s %9.3f ms\n", "total", total);
    for (int i = 0; i < count; ++i) cudaEventDestroy(ev[i]);
  }
};

static int dsolve_plain(int64_t n, const double* d_a, const double* d_b, int64_t k, double* d_x,
                        rm_solve_report* report, cudaStream_t s) {
  Arena ar;
  LuBuffers lb = plan_lu(ar, n);
  const size_t os = ar.add(getrs_f64_scratch_bytes(n, k));
  const size_t orr = ar.add((size_t)n * k * 8);
  const size_t onorm = ar.add(residual_norms_bytes(k));
  Scratch sc;
  sc.stream = s;
  RM_TRY(scratch_alloc(&sc.base, ar.total, s));
  double* w = sc.at<double>(lb.w);
  PhaseTrace tr(s, "plain float64 solve");
  RM_TRY(load_matrix_f64(d_a, n, w, lb.ldw, n, sc.at<double>(lb.amax), s));
  tr.mark("load");
  RM_TRY(getrf_f64(w, lb.ldw, n, sc.at<int64_t>(lb.ipiv), sc.at<int64_t>(lb.perm), sc.at<void>(lb.getrf),
                   device_status(), s));
  tr.mark("getrf");
  // The regular flag, the backward error and the device status word are read back together at
  // the end: the host waits once per call. A matrix that is not regular still gets
  // RM_NOT_REGULAR; x is then unspecified.
  RM_TRY(regular_flag_f64(w, lb.ldw, n, sc.at<double>(lb.amax), sc.at<int32_t>(lb.flag), s));
  if (small_solve_fits(n, k)) {  // one CTA, rustymath's single-column order
    tr.mark("regular");
    RM_TRY(small_solve_f64(w, lb.ldw, false, n, sc.at<int64_t>(lb.perm), d_b, k, d_x, nullptr, s));
  } else {
    RM_TRY(invert_diag_blocks_f64(w, lb.ldw, false, n, sc.at<double>(lb.dinv), true, false, s));
    tr.mark("regular");
    RM_TRY(getrs_f64(w, lb.ldw, false, n, sc.at<int64_t>(lb.perm), sc.at<double>(lb.dinv), d_b, k, k, d_x, k,
                     sc.at<void>(os), device_status(), s));
  }
  tr.mark("getrs");
  if (report) {
    RM_TRY(residual_f64(d_a, n, n, d_x, k, d_b, k, k, sc.at<double>(orr), k, sc.at<double>(onorm), s));
    RM_TRY(backward_error_f64(d_x, k, n, k, sc.at<double>(onorm), sc.at<double>(lb.berr), s));
    tr.mark("residual");
  }
  int32_t regular = 0;
  double berr[2] = {0, 0};
  RM_TRY(finish_call(s, sc.at<int32_t>(lb.flag), &regular, report ? sc.at<double>(lb.berr) : nullptr, berr));
  if (report) report->regular = regular;
  if (!regular) {
    set_last_message("a pivot is at most eps*n*max|a|; rustymath's solve takes least squares here");
    return RM_NOT_REGULAR;
  }
  if (report) {
    report->backward_error = berr[0];
    report->iterations = 0;
    report->method_used = RM_METHOD_PLAIN_F64;
    report->fell_back = 0;
  }
  return RM_OK;
}

// The mixed-precision solve: float32 LU on the tensor cores (panels pivoted among their own
// 256 rows), then float64 refinement until the backward error reaches the tolerance; a stall
// falls back to the plain float64 solve (opts->fallback) or returns RM_NO_CONVERGENCE.
static int dsolve_mixed(int64_t n, const double* d_a, const double* d_b, int64_t k, double* d_x,
                        const rm_solve_options* opts, rm_solve_report* report, cudaStream_t s) {
  const int64_t ldf = round_up(n, 32);
  const double tol = opts->tolerance > 0.0 ? opts->tolerance : (double)n * 0x1.0p-53;
  const int max_it = opts->max_iterations > 0 ? opts->max_iterations : 30;
  int iterations = 0;
  bool converged = false, gmres = false, timed_out = false;
  double berr_h = 0.0;
  {
    Arena ar;
    const size_t of = ar.add((size_t)n * ldf * 4), operm = ar.add((size_t)n * 4);
    const size_t olu = ar.add(getrf_lpp_f32_scratch_bytes(n)), odinv = ar.add(diag_blocks_f32_bytes(n));
    const size_t oc = ar.add((size_t)n * k * 4), orr = ar.add((size_t)n * k * 8), onorm = ar.add(residual_norms_bytes(k));
    const size_t oberr = ar.add(2 * sizeof(double)), otr = ar.add(trsv_f32_scratch_bytes(n, k));
    const size_t opre = ar.add(premultiplied_f32_bytes(n));
    Scratch sc;
    sc.stream = s;
    RM_TRY(scratch_alloc(&sc.base, ar.total, s));
    float* f = sc.at<float>(of);
    int* perm = sc.at<int>(operm);
    float* c = sc.at<float>(oc);
    unsigned* st = device_status();
    PhaseTrace tr(s, "mixed float32 + float64 refinement solve");
    RM_TRY(to_f32(d_a, n, n, f, ldf, s));
    tr.mark("to_f32");
    // the panels write their diagonal blocks' inverses into the solves' table as they go; long
    // chains (n > 1024) then solve on block-Jacobi-scaled triangles, shorter ones take the
    // blocks' couplings to their predecessors
    float* pre = n > 1024 ? sc.at<float>(opre) : nullptr;  // worth its one-off cost on long chains
    RM_TRY(getrf_lpp_f32(f, ldf, n, perm, sc.at<void>(olu), st, s, sc.at<float>(odinv)));
    tr.mark("getrf_f32");
    if (pre) RM_TRY(premultiply_f32(f, ldf, n, sc.at<float>(odinv), pre, s));
    else RM_TRY(couplings_f32(f, ldf, n, sc.at<float>(odinv), s));
    tr.mark("solve_setup");
    // x0 = (LU)^-1 P b
    RM_TRY(gather_f32(d_b, k, perm, n, k, c, k, s));
    RM_TRY(lu_solve_f32_nopiv(f, ldf, n, sc.at<float>(odinv), pre, c, k, k, sc.at<void>(otr), st, s));
    RM_TRY(accumulate_f64(c, k, n, k, d_x, k, true, s));
    tr.mark("solve");
    double prev = INFINITY;
    for (int it = 0; it <= max_it; ++it) {
      RM_TRY(residual_f64(d_a, n, n, d_x, k, d_b, k, k, sc.at<double>(orr), k, sc.at<double>(onorm), s));
      RM_TRY(backward_error_f64(d_x, k, n, k, sc.at<double>(onorm), sc.at<double>(oberr), s));
      tr.mark("residual");
      double be[2] = {0.0, 0.0};
      const int dst = finish_call(s, nullptr, nullptr, sc.at<double>(oberr), be);  // synchronises once
      berr_h = be[0];
      if (dst != RM_OK && dst != RM_TIMEOUT) return dst;
      if (dst == RM_TIMEOUT) {
        timed_out = true;
        break;
      }
      if (berr_h <= tol) {
        converged = true;
        break;
      }
      if (!(berr_h < 0.5 * prev) || it == max_it) break;  // stalled, diverging, NaN, or out of steps
      prev = berr_h;
      // x += (LU)^-1 P r
      RM_TRY(gather_f32(sc.at<double>(orr), k, perm, n, k, c, k, s));
      RM_TRY(lu_solve_f32_nopiv(f, ldf, n, sc.at<float>(odinv), pre, c, k, k, sc.at<void>(otr), st, s));
      RM_TRY(accumulate_f64(c, k, n, k, d_x, k, false, s));
      tr.mark("solve");
      ++iterations;
    }
    if (!converged && !timed_out && opts->gmres_restart > 0 && berr_h == berr_h) {
      // classical refinement stalled: GMRES-IR with the same float32 factors as preconditioner
      Scratch gs;
      gs.stream = s;
      RM_TRY(scratch_alloc(&gs.base, gmres_scratch_bytes(n, k, opts->gmres_restart), s));
      Precond pc{f, ldf, n, perm, sc.at<float>(odinv), pre, c, sc.at<void>(otr), st};
      int outer = 0;
      double berr_g = INFINITY;
      RM_TRY(gmres_ir(d_a, n, d_b, k, d_x, pc, opts->gmres_restart, max_it, tol, &berr_g, &outer, gs.base,
                      sc.at<double>(orr), sc.at<double>(onorm), sc.at<double>(oberr), s));
      tr.mark("gmres_ir");
      iterations += outer;
      if (berr_g <= tol) {
        converged = true;
        gmres = true;
        berr_h = berr_g;
      }
    }
  }
  if (converged) {
    if (report) {
      report->backward_error = berr_h;
      report->iterations = iterations;
      report->method_used = gmres ? RM_METHOD_GMRES_IR : RM_METHOD_F32_IR;
      report->fell_back = 0;
      report->regular = 1;
    }
    return RM_OK;
  }
  if (!opts->fallback) {
    if (report) {
      report->backward_error = berr_h;
      report->iterations = iterations;
      report->method_used = RM_METHOD_F32_IR;
    }
    set_last_message("mixed-precision refinement stalled above the tolerance");
    return RM_NO_CONVERGENCE;
  }
  const int st = dsolve_plain(n, d_a, d_b, k, d_x, report, s);
  if (report) {
    report->iterations = iterations;
    report->fell_back = 1;
  }
  return st;
}

int rm_dsolve(int64_t n, const double* d_a, const double* d_b, int64_t k, double* d_x, const rm_solve_options* opts,
              rm_solve_report* report, void* stream) {
  if (n < 0 || k < 0) return RM_BAD_ARG;
  if (report) memset(report, 0, sizeof *report);
  if (n == 0) {
    set_last_message("an empty matrix is not regular; rustymath's solve takes least squares here");
    return RM_NOT_REGULAR;
  }
  if (!d_a || (k > 0 && (!d_b || !d_x))) return RM_BAD_ARG;
  const int method = opts ? opts->method : RM_METHOD_PLAIN_F64;
  if (method != RM_METHOD_PLAIN_F64 && method != RM_METHOD_F32_IR) return RM_BAD_ARG;
  RM_TRY(check_device());
  cudaStream_t s = as_stream(stream);
  if (k == 0) return RM_OK;
  if (method == RM_METHOD_F32_IR) return dsolve_mixed(n, d_a, d_b, k, d_x, opts, report, s);
  return dsolve_plain(n, d_a, d_b, k, d_x, report, s);
}

int rm_dsolve_host(int64_t n, const double* h_a, const double* h_b, int64_t k, double* h_x,
                   const rm_solve_options* opts, rm_solve_report* report) {
  if (n < 0 || k < 0) return RM_BAD_ARG;
  if (report) memset(report, 0, sizeof *report);
  if (n == 0) return rm_dsolve(0, nullptr, nullptr, k, nullptr, opts, report, nullptr);
  if (!h_a || (k > 0 && (!h_b || !h_x))) return RM_BAD_ARG;
  RM_TRY(check_device());
  cudaStream_t s;
  RM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  int st;
  {
    Arena ar;
    const size_t oa = ar.add((size_t)n * n * 8), ob = ar.add((size_t)n * k * 8), ox = ar.add((size_t)n * k * 8);
    Scratch sc;
    sc.stream = s;
    st = scratch_alloc(&sc.base, ar.total, s);
    if (st == RM_OK) {
      cudaError_t e = cudaMemcpyAsync(sc.at<double>(oa), h_a, (size_t)n * n * 8, cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess && k > 0) e = cudaMemcpyAsync(sc.at<double>(ob), h_b, (size_t)n * k * 8, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) { set_last_error(e, "copy", __FILE__, __LINE__); st = RM_CUDA_ERROR; }
      if (st == RM_OK) st = rm_dsolve(n, sc.at<double>(oa), sc.at<double>(ob), k, sc.at<double>(ox), opts, report, s);
      if (st == RM_OK && k > 0) {
        e = cudaMemcpyAsync(h_x, sc.at<double>(ox), (size_t)n * k * 8, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) { set_last_error(e, "copy", __FILE__, __LINE__); st = RM_CUDA_ERROR; }
      }
    }
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (st == RM_OK && e != cudaSuccess) { set_last_error(e, "sync", __FILE__, __LINE__); st = RM_CUDA_ERROR; }
  cudaStreamDestroy(s);
  return st;
}

// Host-pointer forms of rm_dtrsm, rm_dgemm_ozaki and rm_dsolve_batched: copy in on a stream of
// their own, run the device form, copy back, synchronise.
namespace {
struct HostCall {
  cudaStream_t s = nullptr;
  Scratch sc;
  int st = RM_OK;
  explicit HostCall(size_t bytes) {
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      st = RM_CUDA_ERROR;
      return;
    }
    sc.stream = s;
    st = scratch_alloc(&sc.base, bytes, s);
  }
  int copy(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
    if (st != RM_OK || bytes == 0) return st;
    const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, s);
    if (e != cudaSuccess) {
      set_last_error(e, "copy", __FILE__, __LINE__);
      st = RM_CUDA_ERROR;
    }
    return st;
  }
  int finish() {
    if (!s) return st;
    const cudaError_t e = cudaStreamSynchronize(s);
    if (st == RM_OK && e != cudaSuccess) {
      set_last_error(e, "sync", __FILE__, __LINE__);
      st = RM_CUDA_ERROR;
    }
    return st;
  }
  ~HostCall() {
    if (s) {
      scratch_free(sc.base, s);
      sc.base = nullptr;
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};
}  // namespace

int rm_dtrsm_host(int side, int uplo, int trans, int diag, int64_t m, int64_t n, const double* h_a, int64_t lda,
                  double* h_x, int64_t ldx) {
  if (m < 0 || n < 0) return RM_BAD_ARG;
  if (m == 0 || n == 0) return rm_dtrsm(side, uplo, trans, diag, m, n, h_a, lda, h_x, ldx, nullptr);
  const int64_t order = side == RM_RIGHT ? n : m;
  if (!h_a || !h_x || lda < order || ldx < n) return RM_BAD_ARG;
  RM_TRY(check_device());
  Arena ar;
  const size_t oa = ar.add((size_t)order * lda * 8), ox = ar.add((size_t)m * ldx * 8);
  HostCall hc(ar.total);
  double* a = hc.sc.at<double>(oa);
  double* x = hc.sc.at<double>(ox);
  hc.copy(a, h_a, (size_t)order * lda * 8, cudaMemcpyHostToDevice);
  hc.copy(x, h_x, (size_t)m * ldx * 8, cudaMemcpyHostToDevice);
  if (hc.st == RM_OK) hc.st = rm_dtrsm(side, uplo, trans, diag, m, n, a, lda, x, ldx, hc.s);
  hc.copy(h_x, x, (size_t)m * ldx * 8, cudaMemcpyDeviceToHost);
  return hc.finish();
}

int rm_dgemm_ozaki_host(int64_t m, int64_t n, int64_t k, const double* h_a, int64_t lda, const double* h_b,
                        int64_t ldb, double* h_c, int64_t ldc, int slices) {
  if (m < 0 || n < 0 || k < 0) return RM_BAD_ARG;
  if (m == 0 || n == 0) return RM_OK;
  if (!h_c || ldc < n || (k > 0 && (!h_a || !h_b || lda < k || ldb < n))) return RM_BAD_ARG;
  RM_TRY(check_device());
  Arena ar;
  const size_t oa = ar.add((size_t)m * std::max<int64_t>(lda, 1) * 8), ob = ar.add((size_t)k * ldb * 8);
  const size_t oc = ar.add((size_t)m * ldc * 8);
  HostCall hc(ar.total);
  hc.copy(hc.sc.at<double>(oa), h_a, (size_t)m * lda * 8 * (k > 0), cudaMemcpyHostToDevice);
  hc.copy(hc.sc.at<double>(ob), h_b, (size_t)k * ldb * 8, cudaMemcpyHostToDevice);
  if (hc.st == RM_OK)
    hc.st = rm_dgemm_ozaki(m, n, k, hc.sc.at<double>(oa), std::max<int64_t>(lda, 1), hc.sc.at<double>(ob),
                           std::max<int64_t>(ldb, 1), hc.sc.at<double>(oc), ldc, slices, hc.s);
  hc.copy(h_c, hc.sc.at<double>(oc), (size_t)m * ldc * 8, cudaMemcpyDeviceToHost);
  return hc.finish();
}

int rm_dsolve_batched_host(int64_t count, const int64_t* h_n, const int64_t* h_k, const int64_t* h_a_off,
                           const int64_t* h_b_off, const int64_t* h_x_off, const double* h_a, const double* h_b,
                           double* h_x, const rm_solve_options* opts, rm_batch_report* report) {
  if (count < 0 || (count > 0 && (!h_n || !h_k || !h_a_off || !h_b_off || !h_x_off))) return RM_BAD_ARG;
  int64_t na = 0, nb = 0, nx = 0;
  for (int64_t i = 0; i < count; ++i) {
    if (h_n[i] < 0 || h_k[i] < 0 || h_a_off[i] < 0 || h_b_off[i] < 0 || h_x_off[i] < 0) return RM_BAD_ARG;
    na = std::max(na, h_a_off[i] + h_n[i] * h_n[i]);
    nb = std::max(nb, h_b_off[i] + h_n[i] * h_k[i]);
    nx = std::max(nx, h_x_off[i] + h_n[i] * h_k[i]);
  }
  if ((na && !h_a) || (nb && !h_b) || (nx && !h_x)) return RM_BAD_ARG;
  RM_TRY(check_device());
  Arena ar;
  const size_t oa = ar.add((size_t)na * 8 + 8), ob = ar.add((size_t)nb * 8 + 8), ox = ar.add((size_t)nx * 8 + 8);
  HostCall hc(ar.total);
  hc.copy(hc.sc.at<double>(oa), h_a, (size_t)na * 8, cudaMemcpyHostToDevice);
  hc.copy(hc.sc.at<double>(ob), h_b, (size_t)nb * 8, cudaMemcpyHostToDevice);
  hc.copy(hc.sc.at<double>(ox), h_x, (size_t)nx * 8, cudaMemcpyHostToDevice);  // x's untouched items survive
  if (hc.st == RM_OK)
    hc.st = rm_dsolve_batched(count, h_n, h_k, h_a_off, h_b_off, h_x_off, hc.sc.at<double>(oa), hc.sc.at<double>(ob),
                              hc.sc.at<double>(ox), opts, report, hc.s);
  if (hc.st == RM_OK || hc.st == RM_NO_CONVERGENCE) {
    const int keep = hc.st;
    hc.st = RM_OK;
    hc.copy(h_x, hc.sc.at<double>(ox), (size_t)nx * 8, cudaMemcpyDeviceToHost);
    if (hc.finish() == RM_OK) return keep;
  }
  return hc.finish();
}

}  // extern "C"
