// The mixed-precision solve: a random butterfly transformation, an unpivoted float32 LU with
// 3xTF32 tensor-core block updates, and float64 iterative refinement on the device.
//
// rustymath's solve (core/src/linalg/factor.rs:207-209, 279) factors in the working
// precision with partial pivoting. Here the factorization runs in float32 on the tensor
// cores and float64 refinement (residual r = b - A x from the original float64 A) brings
// the normwise backward error down to n * 2^-53, the same bar as the plain float64 path;
// when refinement stalls, the caller falls back to the plain float64 LU.
//
// Pivot searches are what bound an LU's critical path on a GPU (one reduction over the
// column per pivot). They are avoided with the recursive butterfly transformation of
// Parker (1995), as used by Baboulin, Dongarra, Herrmann and Tomov (2013): A_r = U^T A V
// with U, V random butterflies of depth 2, after which Gaussian elimination without
// pivoting is stable with high probability; x = V y where A_r y = U^T b. A butterfly of
// size N is B = (1/sqrt 2) [R0 R1; R0 -R1] with random diagonal R0, R1 (entries
// exp(u/10), u uniform in [-1/2, 1/2]); depth 2 is diag(B_{N/2}, B_{N/2}) B_N. Indices
// {i, i+N/4, i+N/2, i+3N/4} form closed groups under it, so A_r is formed 4x4 block by 4x4
// block in one pass over A. N is n rounded up to a multiple of 4 ([A 0; 0 I] padding).
//
// LU of A_r (float32, row-major) in blocks of 128 columns, each block:
//   genp_diag_kernel : factors the 128x128 diagonal block in shared memory (no pivoting)
//                      and writes L11^-1 and (U11^-1)^T
//   transpose        : A12^T into a buffer (the tensor cores read both operands K-major)
//   sgemm_tc         : U12^T = A12^T (L11^-1)^T, written both to the buffer and, transposed,
//                      back over A12
//   sgemm_tc         : L21 = A21 U11^-1, in place
//   sgemm_tc         : A22 -= L21 U12
#include "rm_internal.h"

namespace rm {

constexpr int kGenpBlock = 128;

// ------------------------------------------------------------------ butterflies
// r holds, for one depth-2 butterfly of size N (h = N/2, q = N/4): level-1 R0 [0,h), R1
// [h,2h); level-2 upper R0 [2h,2h+q), R1 [2h+q,2h+2q); lower R0 [2h+2q,2h+3q), R1 [2h+3q,2N).
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__global__ void butterfly_params_kernel(double* r, int64_t count, uint64_t seed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    const double u = (double)(splitmix64(seed * 0x100000001B3ull + (uint64_t)i) >> 11) * 0x1.0p-53 - 0.5;
    r[i] = exp(u / 10.0);
  }
}

// W (4x4, z = W x) of the depth-2 butterfly for the index group {i0 + t q}.
__device__ __forceinline__ void butterfly4(const double* __restrict__ r, int64_t N, int64_t i0, double W[4][4]) {
  const int64_t h = N / 2, q = N / 4;
  const double s = 0.70710678118654752440;
  const double a0 = r[i0], b0 = r[h + i0], a1 = r[i0 + q], b1 = r[h + i0 + q];
  const double c0 = r[2 * h + i0], d0 = r[2 * h + q + i0], c1 = r[2 * h + 2 * q + i0], d1 = r[2 * h + 3 * q + i0];
  // level 1: y0 = (a0 x0 + b0 x2) s, y2 = (a0 x0 - b0 x2) s, y1 = (a1 x1 + b1 x3) s, y3 = (a1 x1 - b1 x3) s
  const double L1[4][4] = {{a0 * s, 0, b0 * s, 0}, {0, a1 * s, 0, b1 * s}, {a0 * s, 0, -b0 * s, 0}, {0, a1 * s, 0, -b1 * s}};
  // level 2: z0 = (c0 y0 + d0 y1) s, z1 = (c0 y0 - d0 y1) s, z2 = (c1 y2 + d1 y3) s, z3 = (c1 y2 - d1 y3) s
  const double L2[4][4] = {{c0 * s, d0 * s, 0, 0}, {c0 * s, -d0 * s, 0, 0}, {0, 0, c1 * s, d1 * s}, {0, 0, c1 * s, -d1 * s}};
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) W[i][j] = L2[i][0] * L1[0][j] + L2[i][1] * L1[1][j] + L2[i][2] * L1[2][j] + L2[i][3] * L1[3][j];
}

// ar (float32, N x N, ldr) = U^T [A 0; 0 I] V, A the n x n row-major float64 a (lda).
__global__ void rbt_matrix_kernel(const double* __restrict__ a, int64_t lda, int64_t n, int64_t N,
                                  const double* __restrict__ ru, const double* __restrict__ rv, float* __restrict__ ar,
                                  int64_t ldr) {
  const int64_t q = N / 4;
  const int64_t total = q * q;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i0 = e / q, j0 = e - i0 * q;
    double Wu[4][4], Wv[4][4], blk[4][4], t[4][4];
    butterfly4(ru, N, i0, Wu);
    butterfly4(rv, N, j0, Wv);
#pragma unroll
    for (int s1 = 0; s1 < 4; ++s1)
#pragma unroll
      for (int s2 = 0; s2 < 4; ++s2) {
        const int64_t i = i0 + s1 * q, j = j0 + s2 * q;
        blk[s1][s2] = (i < n && j < n) ? __ldcs(a + i * lda + j) : (i == j ? 1.0 : 0.0);
      }
    // t = blk Wv, then out = Wu^T t
#pragma unroll
    for (int s1 = 0; s1 < 4; ++s1)
#pragma unroll
      for (int s2 = 0; s2 < 4; ++s2)
        t[s1][s2] = blk[s1][0] * Wv[0][s2] + blk[s1][1] * Wv[1][s2] + blk[s1][2] * Wv[2][s2] + blk[s1][3] * Wv[3][s2];
#pragma unroll
    for (int s1 = 0; s1 < 4; ++s1)
#pragma unroll
      for (int s2 = 0; s2 < 4; ++s2) {
        const double v = Wu[0][s1] * t[0][s2] + Wu[1][s1] * t[1][s2] + Wu[2][s1] * t[2][s2] + Wu[3][s1] * t[3][s2];
        ar[(i0 + s1 * q) * ldr + j0 + s2 * q] = (float)v;
      }
  }
}

// c (float32, N x k) = U^T [r; 0] for the n x k float64 r; also zeroes nothing else.
__global__ void rbt_left_kernel(const double* __restrict__ r, int64_t ldr, int64_t n, int64_t N, int64_t k,
                                const double* __restrict__ ru, float* __restrict__ c, int64_t ldc) {
  const int64_t q = N / 4;
  const int64_t total = q * k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i0 = e / k, col = e - i0 * k;
    double Wu[4][4], x[4];
    butterfly4(ru, N, i0, Wu);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int64_t i = i0 + s * q;
      x[s] = i < n ? r[i * ldr + col] : 0.0;
    }
#pragma unroll
    for (int s = 0; s < 4; ++s)
      c[(i0 + s * q) * ldc + col] = (float)(Wu[0][s] * x[0] + Wu[1][s] * x[1] + Wu[2][s] * x[2] + Wu[3][s] * x[3]);
  }
}

// x (float64, n x k) += rows 0..n-1 of V y, y float32 N x k.
__global__ void rbt_right_add_kernel(const float* __restrict__ y, int64_t ldy, int64_t n, int64_t N, int64_t k,
                                     const double* __restrict__ rv, double* __restrict__ x, int64_t ldx, bool assign) {
  const int64_t q = N / 4;
  const int64_t total = q * k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j0 = e / k, col = e - j0 * k;
    double Wv[4][4], v[4];
    butterfly4(rv, N, j0, Wv);
#pragma unroll
    for (int s = 0; s < 4; ++s) v[s] = (double)y[(j0 + s * q) * ldy + col];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int64_t j = j0 + s * q;
      if (j < n) {
        const double d = Wv[s][0] * v[0] + Wv[s][1] * v[1] + Wv[s][2] * v[2] + Wv[s][3] * v[3];
        double* p = x + j * ldx + col;
        *p = assign ? d : *p + d;
      }
    }
  }
}

// ------------------------------------------------------------------ unpivoted diagonal block
// Factors D = A[j0..j0+nb, j0..j0+nb) (nb <= 128) in place without pivoting, then writes
// linv = L11^-1 (unit lower) and uinv = (U11^-1)^T, row-major with leading dimension 128. The inverses' 32x32 diagonal blocks come from column substitution in registers (a
// warp each, a lane per column); the blocks off the diagonal from small products in order
// of their distance from the diagonal. A zero pivot sets RM_DEV_NAN (the refinement then
// fails and the caller falls back).
__global__ void __launch_bounds__(256) genp_diag_kernel(float* __restrict__ a, int64_t lda, int j0, int nb,
                                                        float* __restrict__ linv, float* __restrict__ uinv,
                                                        unsigned* status) {
  extern __shared__ float sm[];
  float(*D)[kGenpBlock + 1] = reinterpret_cast<float(*)[kGenpBlock + 1]>(sm);
  float(*X)[kGenpBlock + 1] = reinterpret_cast<float(*)[kGenpBlock + 1]>(sm + kGenpBlock * (kGenpBlock + 1));
  float(*T)[33] = reinterpret_cast<float(*)[33]>(sm + 2 * kGenpBlock * (kGenpBlock + 1));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tx = tid & 15, ty = tid >> 4;  // a 16x16 thread grid for the updates
  float* blk = a + (int64_t)j0 * lda + j0;
  for (int e = tid; e < kGenpBlock * kGenpBlock; e += 256) {
    const int r = e / kGenpBlock, c = e % kGenpBlock;
    D[r][c] = (r < nb && c < nb) ? blk[(int64_t)r * lda + c] : (r == c ? 1.0f : 0.0f);
  }
  __syncthreads();
  // ---- elimination without pivoting
  for (int c = 0; c < kGenpBlock - 1; ++c) {
    const float piv = D[c][c];
    if (tid == 0 && piv == 0.0f) flag_error(status, RM_DEV_NAN);
    const float rp = 1.0f / piv;
    for (int i = c + 1 + tid; i < kGenpBlock; i += 256) D[i][c] *= rp;
    __syncthreads();
    for (int i = c + 1 + ty; i < kGenpBlock; i += 16) {
      const float l = D[i][c];
      for (int j = c + 1 + tx; j < kGenpBlock; j += 16) D[i][j] = fmaf(-l, D[c][j], D[i][j]);
    }
    __syncthreads();
  }
  for (int e = tid; e < nb * nb; e += 256) {
    const int r = e / nb, c = e % nb;
    blk[(int64_t)r * lda + c] = D[r][c];
  }
  // ---- L11^-1 (unit lower) into X
  for (int e = tid; e < kGenpBlock * kGenpBlock; e += 256) X[e / kGenpBlock][e % kGenpBlock] = 0.0f;
  __syncthreads();
  if (warp < 4) {
    const int b0 = warp * 32;
    float x[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      float s = i == lane ? 1.0f : 0.0f;
#pragma unroll
      for (int k2 = 0; k2 < i; ++k2) s = fmaf(-D[b0 + i][b0 + k2], x[k2], s);
      x[i] = i < lane ? 0.0f : s;
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) X[b0 + i][b0 + lane] = x[i];
  }
  __syncthreads();
  for (int gap = 1; gap < 4; ++gap)
    for (int ab = 0; ab + gap < 4; ++ab) {
      const int rb = (ab + gap) * 32, ca = ab * 32;
      for (int e = tid; e < 1024; e += 256) {  // T = sum_{c=a..b-1} L_bc X_ca
        const int i = e >> 5, j = e & 31;
        float s = 0.0f;
        for (int k2 = ca; k2 < rb; ++k2) s = fmaf(D[rb + i][k2], X[k2][ca + j], s);
        T[i][j] = s;
      }
      __syncthreads();
      for (int e = tid; e < 1024; e += 256) {  // X_ba = -D_b^-1 T, D_b^-1 = X's diagonal block b
        const int i = e >> 5, j = e & 31;
        float s = 0.0f;
        for (int k2 = 0; k2 <= i; ++k2) s = fmaf(X[rb + i][rb + k2], T[k2][j], s);
        X[rb + i][ca + j] = -s;
      }
      __syncthreads();
    }
  for (int e = tid; e < kGenpBlock * kGenpBlock; e += 256) linv[e] = X[e / kGenpBlock][e % kGenpBlock];
  __syncthreads();
  // ---- U11^-1 (upper) into X
  for (int e = tid; e < kGenpBlock * kGenpBlock; e += 256) X[e / kGenpBlock][e % kGenpBlock] = 0.0f;
  __syncthreads();
  if (warp < 4) {
    const int b0 = warp * 32;
    float x[32];
#pragma unroll
    for (int i = 31; i >= 0; --i) {
      float s = i == lane ? 1.0f : 0.0f;
#pragma unroll
      for (int k2 = i + 1; k2 < 32; ++k2) s = fmaf(-D[b0 + i][b0 + k2], x[k2], s);
      x[i] = i > lane ? 0.0f : s / D[b0 + i][b0 + i];
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) X[b0 + i][b0 + lane] = x[i];
  }
  __syncthreads();
  for (int gap = 1; gap < 4; ++gap)
    for (int ab = 0; ab + gap < 4; ++ab) {
      const int ra = ab * 32, cb = (ab + gap) * 32;
      for (int e = tid; e < 1024; e += 256) {  // T = sum_{c=a+1..b} U_ac X_cb
        const int i = e >> 5, j = e & 31;
        float s = 0.0f;
        for (int k2 = ra + 32; k2 < cb + 32; ++k2) s = fmaf(D[ra + i][k2], X[k2][cb + j], s);
        T[i][j] = s;
      }
      __syncthreads();
      for (int e = tid; e < 1024; e += 256) {  // X_ab = -D_a^-1 T, D_a^-1 upper
        const int i = e >> 5, j = e & 31;
        float s = 0.0f;
        for (int k2 = i; k2 < 32; ++k2) s = fmaf(X[ra + i][ra + k2], T[k2][j], s);
        X[ra + i][cb + j] = -s;
      }
      __syncthreads();
    }
  for (int e = tid; e < kGenpBlock * kGenpBlock; e += 256) uinv[e] = X[e % kGenpBlock][e / kGenpBlock];
}

constexpr size_t kGenpDiagSmem = (2 * kGenpBlock * (kGenpBlock + 1) + 32 * 33) * sizeof(float);

size_t getrf_genp_f32_scratch_bytes(int64_t n) {
  return (2 * (size_t)kGenpBlock * kGenpBlock + 2 * (size_t)n * kGenpBlock) * sizeof(float) + 1024;
}

int getrf_genp_f32(float* a, int64_t lda, int64_t n, void* scratch, unsigned* status, cudaStream_t stream) {
  if (n <= 0) return RM_OK;
  float* linv = reinterpret_cast<float*>(scratch);
  float* uinvt = linv + kGenpBlock * kGenpBlock;
  float* a12t = uinvt + kGenpBlock * kGenpBlock;  // rest x 128: A12^T
  float* u12t = a12t + (size_t)n * kGenpBlock;    // rest x 128: U12^T
  static bool set = false;
  if (!set) {
    RM_CUDA_TRY(cudaFuncSetAttribute(genp_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGenpDiagSmem));
    set = true;
  }
  for (int64_t J0 = 0; J0 < n; J0 += kGenpBlock) {
    const int nb = (int)std::min<int64_t>(kGenpBlock, n - J0);
    const int64_t J1 = J0 + nb, rest = n - J1;
    genp_diag_kernel<<<1, 256, kGenpDiagSmem, stream>>>(a, lda, (int)J0, nb, linv, uinvt, status);
    RM_LAUNCHED();
    if (rest == 0) break;
    float* a12 = a + J0 * lda + J1;
    float* a21 = a + J1 * lda + J0;
    RM_TRY(transpose_f32(a12, lda, nb, rest, a12t, kGenpBlock, stream));
    // U12^T = A12^T (L11^-1)^T, also written transposed over A12
    RM_TRY(sgemm_tc(3, rest, nb, nb, 1.0f, a12t, kGenpBlock, linv, kGenpBlock, 0.0f, u12t, kGenpBlock, status, stream,
                    a12, lda));
    // L21 = A21 U11^-1, in place (one tile column: each CTA reads its rows before writing them)
    RM_TRY(sgemm_tc(3, rest, nb, nb, 1.0f, a21, lda, uinvt, kGenpBlock, 0.0f, a21, lda, status, stream));
    // A22 -= L21 U12
    RM_TRY(sgemm_tc(3, rest, rest, nb, -1.0f, a21, lda, u12t, kGenpBlock, 1.0f, a + J1 * lda + J1, lda, status,
                    stream));
  }
  return RM_OK;
}

// ------------------------------------------------------------------ butterfly helpers

int butterfly_params(double* r, int64_t N, uint64_t seed, cudaStream_t stream) {
  const int64_t count = 2 * N;
  butterfly_params_kernel<<<(int)std::min<int64_t>((count + 255) / 256, 1024), 256, 0, stream>>>(r, count, seed);
  RM_LAUNCHED();
  return RM_OK;
}

int rbt_matrix(const double* a, int64_t lda, int64_t n, int64_t N, const double* ru, const double* rv, float* ar,
               int64_t ldr, cudaStream_t stream) {
  const int64_t q = N / 4;
  const int blocks = (int)std::min<int64_t>((q * q + 255) / 256, 16 * device_sm_count());
  rbt_matrix_kernel<<<blocks, 256, 0, stream>>>(a, lda, n, N, ru, rv, ar, ldr);
  RM_LAUNCHED();
  return RM_OK;
}

int rbt_left(const double* r, int64_t ldr, int64_t n, int64_t N, int64_t k, const double* ru, float* c, int64_t ldc,
             cudaStream_t stream) {
  const int64_t total = (N / 4) * k;
  rbt_left_kernel<<<(int)std::min<int64_t>((total + 255) / 256, 4 * device_sm_count()), 256, 0, stream>>>(
      r, ldr, n, N, k, ru, c, ldc);
  RM_LAUNCHED();
  return RM_OK;
}

int rbt_right_add(const float* y, int64_t ldy, int64_t n, int64_t N, int64_t k, const double* rv, double* x,
                  int64_t ldx, bool assign, cudaStream_t stream) {
  const int64_t total = (N / 4) * k;
  rbt_right_add_kernel<<<(int)std::min<int64_t>((total + 255) / 256, 4 * device_sm_count()), 256, 0, stream>>>(
      y, ldy, n, N, k, rv, x, ldx, assign);
  RM_LAUNCHED();
  return RM_OK;
}

}  // namespace rm
