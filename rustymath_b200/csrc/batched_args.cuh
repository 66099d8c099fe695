// The arguments and host launches of the batched kernels (batched_kernels.cuh), shared by their
// builds for systems of order up to 256 (namespace bt, batched.cu) and up to 64 (namespace bt64,
// batched_small.cu).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace rm {

// An item's code in BatchArgs::nb: its float32 panel width (16 or 32) in the low byte, and
// kItemF64 when the precision tuner gave its size bucket float64 factors (no refinement).
constexpr int kItemF64 = 1 << 8;

struct BatchArgs {
  int first, last;  // items [first, last) of the processing order
  const int* sys;   // item -> system
  const int* nb;    // item -> panel width (16 or 32), | kItemF64 for float64 factors
  const int* n;
  const int* k;
  const int64_t* a_off;
  const int64_t* b_off;
  const int64_t* x_off;
  const int64_t* w_off;  // bytes
  const double* a;
  const double* b;
  double* x;
  unsigned char* w;
  int method;  // RM_METHOD_*
  int max_it;
  double tol;  // 0: n * 2^-53
  int fallback;
  double* berr;  // per system
  int* iters;
  int* flags;
  int* counter;
  int* piv;            // per system (at p_off): the row chosen for each logical column
  const int64_t* p_off;
  int* ftype;          // per system: 0 when W holds float32 factors, 1 for float64
};

struct AdjointArgs {
  BatchArgs bt;         // the forward's layout, factors (w), row orders (piv) and types
  const double* g;      // dL/dx, packed like b
  double* gb;           // dL/db = A^-T g, packed like b
  double* ga;           // dL/dA = -gb x^T, packed like a (NULL: not formed)
  double* berr;         // per system: the backward error of A^T gb = g
};

// Each build's launches: prepare sets the kernels' shared-memory attribute on the current
// device and gives the persistent grid's CTAs per SM; the launches are asynchronous on s.
#define RM_BT_LAUNCHES                                                                             \
  int prepare(int* per_sm);                                                                       \
  void launch_solve(const BatchArgs& q, int grid, cudaStream_t s);                                \
  void launch_adjoint(const AdjointArgs& q, int grid, cudaStream_t s);                            \
  int launch_factor(const double* a, int n, unsigned char* wbuf, int64_t w_stride, double* factors, \
                    int64_t* perm, int32_t* regular, unsigned count, cudaStream_t s);

namespace bt {
constexpr int MAX_N = 256;
RM_BT_LAUNCHES
}  // namespace bt
namespace bt64 {
constexpr int MAX_N = 64;
RM_BT_LAUNCHES
}  // namespace bt64
#undef RM_BT_LAUNCHES

}  // namespace rm
