// FP64 residual r = b - A x and the normwise backward error, on the device.
//
// The backward error of a solve, max over right-hand sides c of
//   ||b_c - A x_c||_inf / (||A||_inf ||x_c||_inf + ||b_c||_inf),
// is stated beside every result, and the refinement loop tests it. A crosses HBM once (the
// kernel is bandwidth-bound: 8 bytes of A per 2*k flops, the flops on the FP64 tensor
// path); the rows' |a| sums give ||A||_inf on the way.
#include "rm_internal.h"

namespace rm {

constexpr int kNormGroup = 16;  // columns per group of norm slots
constexpr int kNormSlots = 1 + 3 * kNormGroup;
constexpr int kResWarps = 8;    // warps of a block; they split the columns of A between them
constexpr int kResRows = 32;    // rows of A per block: two m16 tiles in every warp
constexpr int kResStep = 16;    // columns of A per warp step: two k8 mma steps

__device__ __forceinline__ void atomic_max_nonneg(double* p, double v) {
  // non-negative doubles (and NaN, above +inf) order like their bit patterns
  if (v > 0.0 || v != v) atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double a2, double a3, double b0, double b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

// r (n x k, ldr) = b - A x for k <= 8 NT, on the FP64 tensor path (mma.sync m16n8k8 f64).
// A block owns kResRows rows of A; its warps take the columns in interleaved steps of
// kResStep, load their A items straight from HBM into mma fragments (two steps in flight
// per warp, several warps per SM) and x's from L2, and sum
// their partial products in shared memory in warp order at the end, so the result does not
// depend on scheduling. The mma k index of a step is mapped to columns so that each lane's
// A items are 4 consecutive columns (t = lane % 4 takes columns 4t .. 4t+3 of the step;
// k step s uses 4t+2s for mma k index t and 4t+2s+1 for t+4), which VEC reads as two 16-byte
// loads. norms (zeroed by the caller) collects by atomic maxima norms[0] = ||A||_inf and,
// per column c, norms[1+c] = ||r_c||_inf (NaN if a residual is NaN) and
// norms[1+2*kNormGroup+c] = ||b_c||_inf.
template <int NT, bool VEC>
__global__ void __launch_bounds__(kResWarps * 32, 2)
    residual_kernel(const double* __restrict__ a, int64_t lda, int64_t n, const double* __restrict__ x, int64_t ldx,
                    const double* __restrict__ b, int64_t ldb, int k, double* __restrict__ r, int64_t ldr,
                    double* __restrict__ norms) {
  __shared__ double part[kResWarps][kResRows][kNormGroup + 1];
  __shared__ double apart[kResWarps][kResRows];
  __shared__ double rab[2][kResRows][kNormGroup + 1];
  __shared__ double rowsum[kResRows];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int64_t row0 = (int64_t)blockIdx.x * kResRows;
  // this lane's rows are row0 + g + 8i (i = 2m + h); rows past n are never read
  const double* abase = a + (row0 + g) * lda;
  const int64_t ld8 = 8 * lda;
  const int64_t rows_left = n - row0 - g;
  double acc[2][NT][4], asum[2][2];
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    asum[m][0] = asum[m][1] = 0.0;
#pragma unroll
    for (int q = 0; q < NT; ++q)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[m][q][e] = 0.0;
  }
  auto load_a = [&](int64_t j0, double (&av)[2][2][4]) {
    const int64_t j = j0 + 4 * t;
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const bool rok = 8 * (2 * m + h) < rows_left;
        const double* ar = abase + (2 * m + h) * ld8 + j;
        if (VEC && rok && j + 3 < n) {
          const double2 p = __ldcs(reinterpret_cast<const double2*>(ar));
          const double2 q = __ldcs(reinterpret_cast<const double2*>(ar + 2));
          av[m][h][0] = p.x, av[m][h][1] = p.y, av[m][h][2] = q.x, av[m][h][3] = q.y;
        } else {
#pragma unroll
          for (int u = 0; u < 4; ++u) av[m][h][u] = (rok && j + u < n) ? __ldcs(ar + u) : 0.0;
        }
      }
  };
  const int64_t stride = (int64_t)kResWarps * kResStep;
  int64_t j0 = (int64_t)warp * kResStep;
#pragma unroll 2
  for (; j0 < n; j0 += stride) {
    double av[2][2][4];
    load_a(j0, av);
    double xv[NT][4];
#pragma unroll
    for (int q = 0; q < NT; ++q)
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int64_t j = j0 + 4 * t + u;
        const int c = 8 * q + g;
        xv[q][u] = (j < n && c < k) ? __ldg(x + j * ldx + c) : 0.0;
      }
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int u = 0; u < 4; ++u) asum[m][h] += fabs(av[m][h][u]);
#pragma unroll
    for (int s = 0; s < 2; ++s)
#pragma unroll
      for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int q = 0; q < NT; ++q)
          dmma(acc[m][q], av[m][0][2 * s], av[m][1][2 * s], av[m][0][2 * s + 1], av[m][1][2 * s + 1], xv[q][2 * s],
               xv[q][2 * s + 1]);
  }
  // accumulator (row g / g+8 of tile m, columns 8q + 2t, +1) and row |a| sums to shared memory
#pragma unroll
  for (int m = 0; m < 2; ++m) {
#pragma unroll
    for (int q = 0; q < NT; ++q)
#pragma unroll
      for (int e = 0; e < 4; ++e) part[warp][16 * m + g + 8 * (e >> 1)][8 * q + 2 * t + (e & 1)] = acc[m][q][e];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      double v = asum[m][h];
      v += __shfl_xor_sync(0xffffffffu, v, 1);
      v += __shfl_xor_sync(0xffffffffu, v, 2);
      if (t == 0) apart[warp][16 * m + 8 * h + g] = v;
    }
  }
  __syncthreads();
  for (int e = tid; e < kResRows * kNormGroup; e += kResWarps * 32) {
    const int i = e / kNormGroup, c = e % kNormGroup;
    const int64_t row = row0 + i;
    double rv = 0.0, bv = 0.0;
    if (row < n && c < k && c < 8 * NT) {
      double sum = 0.0;
#pragma unroll
      for (int w = 0; w < kResWarps; ++w) sum += part[w][i][c];
      bv = b[row * ldb + c];
      rv = bv - sum;
      r[row * ldr + c] = rv;
    }
    rab[0][i][c] = fabs(rv);
    rab[1][i][c] = fabs(bv);
  }
  if (tid < kResRows) {
    double sum = 0.0;
#pragma unroll
    for (int w = 0; w < kResWarps; ++w) sum += apart[w][tid];
    rowsum[tid] = sum;
  }
  __syncthreads();
  if (norms && tid <= 2 * kNormGroup) {
    double mx = 0.0;
    if (tid < 2 * kNormGroup) {
      const int which = tid / kNormGroup, c = tid % kNormGroup;
      for (int i = 0; i < kResRows; ++i) {
        const double v = rab[which][i][c];
        mx = (v > mx || v != v) ? v : mx;  // NaN, once seen, stays
      }
      if (c < k) atomic_max_nonneg(&norms[1 + (which ? 2 * kNormGroup : 0) + c], mx);
    } else {
      for (int i = 0; i < kResRows; ++i) {
        const double v = rowsum[i];
        mx = (v > mx || v != v) ? v : mx;
      }
      atomic_max_nonneg(&norms[0], mx);
    }
  }
}

// norms[1+kNormGroup+c] = ||x_c||_inf for the n x k (k <= kNormGroup) row-major x.
__global__ void column_max_kernel(const double* __restrict__ x, int64_t ldx, int64_t n, int k, double* norms) {
  double m[kNormGroup];
#pragma unroll
  for (int c = 0; c < kNormGroup; ++c) m[c] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int c = 0; c < kNormGroup; ++c)
      if (c < k) m[c] = fmax(m[c], fabs(x[i * ldx + c]));
#pragma unroll
  for (int c = 0; c < kNormGroup; ++c) {
    double v = m[c];
#pragma unroll
    for (int off = 16; off; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0 && c < k) atomic_max_nonneg(&norms[1 + kNormGroup + c], v);
  }
}

// out[0] = max_c ||r_c|| / (||A|| ||x_c|| + ||b_c||) over every group of columns (NaN when a
// residual is NaN), out[1] = ||A||_inf.
__global__ void backward_error_kernel(const double* __restrict__ norms, int k, double* out) {
  if (threadIdx.x != 0) return;
  const double anorm = norms[0];
  double worst = 0.0;
  bool nan = false;
  for (int c = 0; c < k; ++c) {
    const double* g = norms + (c / kNormGroup) * kNormSlots;
    const int cc = c % kNormGroup;
    const double rn = g[1 + cc], xn = g[1 + kNormGroup + cc], bn = g[1 + 2 * kNormGroup + cc];
    nan |= rn != rn;
    const double den = anorm * xn + bn;
    worst = fmax(worst, den > 0.0 ? rn / den : rn);
  }
  out[0] = nan ? __longlong_as_double(0x7ff8000000000000ll) : worst;
  out[1] = anorm;
}

size_t residual_norms_bytes(int64_t k) { return (size_t)((k + kNormGroup - 1) / kNormGroup) * kNormSlots * 8 + 64; }

int residual_f64(const double* a, int64_t lda, int64_t n, const double* x, int64_t ldx, const double* b, int64_t ldb,
                 int64_t k, double* r, int64_t ldr, double* norms, cudaStream_t stream) {
  if (n == 0 || k == 0) return RM_OK;
  const unsigned blocks = (unsigned)((n + kResRows - 1) / kResRows);
  const bool vec = reinterpret_cast<uintptr_t>(a) % 16 == 0 && lda % 2 == 0;
  if (norms) RM_CUDA_TRY(cudaMemsetAsync(norms, 0, residual_norms_bytes(k), stream));
  for (int64_t c0 = 0, g = 0; c0 < k; c0 += kNormGroup, ++g) {
    const int kc = (int)std::min<int64_t>(kNormGroup, k - c0);
    double* ng = norms ? norms + g * kNormSlots : nullptr;
    auto go = [&](auto kern) {
      kern<<<blocks, kResWarps * 32, 0, stream>>>(a, lda, n, x + c0, ldx, b + c0, ldb, kc, r + c0, ldr, ng);
    };
    if (kc <= 8) vec ? go(residual_kernel<1, true>) : go(residual_kernel<1, false>);
    else vec ? go(residual_kernel<2, true>) : go(residual_kernel<2, false>);
    RM_LAUNCHED();
  }
  return RM_OK;
}

int backward_error_f64(const double* x, int64_t ldx, int64_t n, int64_t k, double* norms, double* out,
                       cudaStream_t stream) {
  if (n == 0 || k == 0) {
    RM_CUDA_TRY(cudaMemsetAsync(out, 0, 2 * sizeof(double), stream));
    return RM_OK;
  }
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, 2 * device_sm_count());
  for (int64_t c0 = 0, g = 0; c0 < k; c0 += kNormGroup, ++g) {
    const int kc = (int)std::min<int64_t>(kNormGroup, k - c0);
    column_max_kernel<<<blocks, 256, 0, stream>>>(x + c0, ldx, n, kc, norms + g * kNormSlots);
    RM_LAUNCHED();
  }
  backward_error_kernel<<<1, 32, 0, stream>>>(norms, (int)k, out);
  RM_LAUNCHED();
  return RM_OK;
}

}  // namespace rm
