// Batched solves of many small systems of uneven size (n <= 256, k <= 8) in one persistent
// launch: float32 LU with partial pivoting + float64 refinement per system, falling back to a
// float64 LU for the systems whose refinement stalls, all inside the same kernel.
//
// rustymath solves a stack of systems one LuWork per thread (Stacked::solve,
// src/linalg/stacked.rs:88-101, over parallel::stack, core/src/parallel.rs:118-192), each an
// lu_factor + lu_solve (core/src/linalg/factor.rs:617-641) and, when `regular` fails
// (factor.rs:221-226), least squares. Here a CTA takes one system at a time from a shared
// counter (systems sorted by size, largest first, so the long ones start early) and:
//   - loads A (float64, row-major) into a float32 working copy W in its own slice of a global
//     scratch (W stays in L2 while the CTA works on it); thread r owns row r;
//   - factors W with partial pivoting, implicitly: rows never move, a row chosen as pivot of
//     logical column c records pos = c and leaves the candidates; in panels of NB columns
//     (16 or 32, picked per size bucket by the tuner) each thread keeps its row's panel in
//     registers and each column costs one barrier (every warp posts its best candidate row,
//     every thread picks the winner among the posts: largest |pivot|, lowest row on ties, NaN
//     never chosen over a number); then U12 of the panel's pivot rows (a column per thread)
//     and the update of the rows not chosen yet;
//   - solves L U x = P b with the rows' right-hand sides in registers, block by block (a warp
//     per right-hand side solves each NB x NB diagonal block with shuffles);
//   - refines in float64: r = b - A x (a warp per row of A, x in shared memory), the normwise
//     backward error max_c ||r_c|| / (||A|| ||x_c|| + ||b_c||), and corrections from the
//     float32 factors until it is at most the tolerance (n * 2^-53 by default);
//   - on a stall (the error not halving) or the step limit, redoes the system in float64
//     (the same code on float64 items, reusing the slice) and reports the fallback; a pivot
//     at most eps * n * max|a| there marks the system not regular, as rustymath's `regular`.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <numeric>
#include <vector>

#include "rm_internal.h"

#define RM_BT_NS bt
#define RM_BT_NMAX 256
#define RM_BT_MIN_BLOCKS 2
#include "batched_kernels.cuh"

namespace rm {


// ------------------------------------------------------------------ the plan (host)
struct BatchPlan {
  int64_t count = 0;
  std::vector<int> n, k, order, nb_item;
  std::vector<int64_t> a_off, b_off, x_off, w_off;
  rm_solve_options opts{};
  int nb_bucket[5] = {16, 16, 32, 32, 32};  // panel width per size bucket (tuned)
  int f64_bucket[5] = {0, 0, 0, 0, 0};      // 1: the bucket's systems take float64 factors (precision tuner)
  int code(int bucket) const { return nb_bucket[bucket] | (f64_bucket[bucket] ? kItemF64 : 0); }
  // device
  int *d_sys = nullptr, *d_nb = nullptr, *d_n = nullptr, *d_k = nullptr, *d_iters = nullptr, *d_flags = nullptr,
      *d_counter = nullptr;
  int64_t *d_aoff = nullptr, *d_boff = nullptr, *d_xoff = nullptr, *d_woff = nullptr, *d_poff = nullptr;
  int *d_piv = nullptr, *d_ftype = nullptr;
  double* d_berr = nullptr;
  double* d_adj_berr = nullptr;
  unsigned char* d_w = nullptr;
  size_t w_bytes = 0;
  int small_limit = bt64::MAX_N;  // the largest n the 64-thread build takes (64, 32 or 0; tuned)
  int split = 0;  // items [0, split) (n > small_limit) go to the 256-thread kernel, the rest to the 64-thread one
  int grid = 0, grid_small = 0;
  cudaStream_t stream = nullptr;  // the plan's own stream, for graph capture
  cudaStream_t side = nullptr;    // the 64-thread kernel's, beside the other inside the graph
  cudaGraphExec_t graph = nullptr;
  const void* g_a = nullptr;
  const void* g_b = nullptr;
  const void* g_x = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr, ev_fork = nullptr, ev_join = nullptr;
  // execute_host: the systems in groups of consecutive indices (about equal bytes of A), each
  // group's items sorted by size; built on the first call and again after a tune
  int tune_gen = 0, groups_gen = -1;
  std::vector<int> g_first;  // group g: items [g_first[g], g_first[g + 1]) of g_order
  std::vector<int> g_split;  // its first item of n <= small_limit
  std::vector<int> g_order, g_nb;
  int *d_gsys = nullptr, *d_gnb = nullptr;
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  std::vector<cudaEvent_t> g_in, g_done;
  cudaEvent_t ev_start = nullptr, ev_end = nullptr;
};

static int bucket_of(int n) { return n <= 32 ? 0 : n <= 64 ? 1 : n <= 128 ? 2 : n <= 192 ? 3 : 4; }
static constexpr int kBucketMax[5] = {32, 64, 128, 192, 256};

static void free_plan(BatchPlan* p) {
  if (!p) return;
  if (p->graph) cudaGraphExecDestroy(p->graph);
  for (void* q : {(void*)p->d_sys, (void*)p->d_nb, (void*)p->d_n, (void*)p->d_k, (void*)p->d_iters,
                  (void*)p->d_flags, (void*)p->d_counter, (void*)p->d_aoff, (void*)p->d_boff, (void*)p->d_xoff,
                  (void*)p->d_woff, (void*)p->d_berr, (void*)p->d_w, (void*)p->d_poff, (void*)p->d_piv,
                  (void*)p->d_ftype, (void*)p->d_adj_berr})
    if (q) cudaFree(q);
  for (cudaEvent_t e : {p->ev_in, p->ev_out, p->ev_fork, p->ev_join, p->ev_start, p->ev_end})
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : p->g_in) cudaEventDestroy(e);
  for (cudaEvent_t e : p->g_done) cudaEventDestroy(e);
  if (p->d_gsys) cudaFree(p->d_gsys);
  if (p->d_gnb) cudaFree(p->d_gnb);
  for (cudaStream_t q : {p->stream, p->side, p->copy_in, p->copy_out})
    if (q) cudaStreamDestroy(q);
  delete p;
}

template <typename V>
static int upload(V** dst, const std::vector<V>& src) {
  RM_CUDA_TRY(cudaMalloc(dst, std::max<size_t>(src.size(), 1) * sizeof(V)));
  if (!src.empty()) RM_CUDA_TRY(cudaMemcpy(*dst, src.data(), src.size() * sizeof(V), cudaMemcpyHostToDevice));
  return RM_OK;
}

// the first item of the size-sorted order that the 64-thread build takes
static void set_split(BatchPlan* p) {
  p->split = 0;
  while (p->split < (int)p->count && p->n[p->order[p->split]] > p->small_limit) ++p->split;
}

static int plan_build(BatchPlan* p) {
  const int64_t cnt = p->count;
  p->order.resize(cnt);
  std::iota(p->order.begin(), p->order.end(), 0);
  // largest first: the long systems start early and the short ones fill in at the end
  std::stable_sort(p->order.begin(), p->order.end(), [&](int x, int y) { return p->n[x] > p->n[y]; });
  p->w_off.assign(cnt, 0);
  size_t off = 0;
  for (int64_t i = 0; i < cnt; ++i) {
    const int n = p->n[i];
    p->w_off[i] = (int64_t)off;
    off += ((size_t)n * ((n + 3) & ~3) * 8 + 255) / 256 * 256;
  }
  p->w_bytes = std::max<size_t>(off, 256);
  p->nb_item.resize(cnt);
  for (int64_t i = 0; i < cnt; ++i) p->nb_item[i] = p->code(bucket_of(p->n[p->order[i]]));
  RM_TRY(upload(&p->d_sys, p->order));
  RM_TRY(upload(&p->d_nb, p->nb_item));
  RM_TRY(upload(&p->d_n, p->n));
  RM_TRY(upload(&p->d_k, p->k));
  RM_TRY(upload(&p->d_aoff, p->a_off));
  RM_TRY(upload(&p->d_boff, p->b_off));
  RM_TRY(upload(&p->d_xoff, p->x_off));
  RM_TRY(upload(&p->d_woff, p->w_off));
  std::vector<int64_t> p_off(cnt);
  int64_t poff = 0;
  for (int64_t i = 0; i < cnt; ++i) p_off[i] = poff, poff += p->n[i];
  RM_TRY(upload(&p->d_poff, p_off));
  RM_CUDA_TRY(cudaMalloc(&p->d_piv, std::max<int64_t>(poff, 1) * sizeof(int)));
  RM_CUDA_TRY(cudaMalloc(&p->d_ftype, std::max<int64_t>(cnt, 1) * sizeof(int)));
  RM_CUDA_TRY(cudaMalloc(&p->d_adj_berr, std::max<int64_t>(cnt, 1) * sizeof(double)));
  RM_CUDA_TRY(cudaMalloc(&p->d_berr, std::max<int64_t>(cnt, 1) * sizeof(double)));
  RM_CUDA_TRY(cudaMalloc(&p->d_iters, std::max<int64_t>(cnt, 1) * sizeof(int)));
  RM_CUDA_TRY(cudaMalloc(&p->d_flags, std::max<int64_t>(cnt, 1) * sizeof(int)));
  RM_CUDA_TRY(cudaMalloc(&p->d_counter, 2 * sizeof(int)));  // one per kernel
  RM_CUDA_TRY(cudaMalloc(&p->d_w, p->w_bytes));
  set_split(p);
  int per_sm = 0, per_sm_small = 0;
  RM_TRY(bt::prepare(&per_sm));
  RM_TRY(bt64::prepare(&per_sm_small));
  p->grid = std::max(1, per_sm) * device_sm_count();
  p->grid_small = std::max(1, per_sm_small) * device_sm_count();
  RM_CUDA_TRY(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  RM_CUDA_TRY(cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&p->ev_in, &p->ev_out, &p->ev_fork, &p->ev_join})
    RM_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  return RM_OK;
}

static BatchArgs batch_args(BatchPlan* p, const double* a, const double* b, double* x, int first, int last,
                            int* counter) {
  BatchArgs q;
  q.first = first, q.last = last;
  q.sys = p->d_sys, q.nb = p->d_nb, q.n = p->d_n, q.k = p->d_k;
  q.a_off = p->d_aoff, q.b_off = p->d_boff, q.x_off = p->d_xoff, q.w_off = p->d_woff;
  q.a = a, q.b = b, q.x = x, q.w = p->d_w;
  q.method = p->opts.method;
  q.max_it = p->opts.max_iterations > 0 ? p->opts.max_iterations : 30;
  q.tol = p->opts.tolerance;
  q.fallback = p->opts.fallback;
  q.berr = p->d_berr, q.iters = p->d_iters, q.flags = p->d_flags, q.counter = counter;
  q.piv = p->d_piv, q.p_off = p->d_poff, q.ftype = p->d_ftype;
  return q;
}

// Runs big(first, last, stream) over the items [first, last) ∩ [0, split) and small(...) over
// [first, last) ∩ [split, ...), after the counters' reset on s (counting the launches in
// rm_launch_count when `count`). When both have items, the
// 64-thread kernel runs on the plan's side stream, forked from s and joined back, so that its
// CTAs fill the SMs that the 256-thread kernel's CTAs leave at its end; inside a capture the
// fork and join become the graph's edges.
template <typename Big, typename Small>
static int launch_split(BatchPlan* p, int first, int last, int split, cudaStream_t s, bool count, Big&& big,
                        Small&& small) {
  RM_CUDA_TRY(cudaMemsetAsync(p->d_counter, 0, 2 * sizeof(int), s));
  const int b1 = std::min(last, split), s0 = std::max(first, split);
  const bool has_big = first < b1, has_small = s0 < last;
  cudaStream_t ss = s;
  if (has_big && has_small) {
    RM_CUDA_TRY(cudaEventRecord(p->ev_fork, s));
    RM_CUDA_TRY(cudaStreamWaitEvent(p->side, p->ev_fork, 0));
    ss = p->side;
  }
  if (has_big) {
    big(first, b1, s);
    RM_CUDA_TRY(cudaGetLastError());
    if (count) note_launch();
  }
  if (has_small) {
    small(s0, last, ss);
    RM_CUDA_TRY(cudaGetLastError());
    if (count) note_launch();
  }
  if (ss != s) {
    RM_CUDA_TRY(cudaEventRecord(p->ev_join, ss));
    RM_CUDA_TRY(cudaStreamWaitEvent(s, p->ev_join, 0));
  }
  return RM_OK;
}

// The persistent launches over items [first, last); launches being captured into the plan's
// graph are counted when the graph runs, not here.
static int launch_batch(BatchPlan* p, const double* a, const double* b, double* x, int first, int last,
                        cudaStream_t s, bool captured = false) {
  RM_TRY(launch_split(
      p, first, last, p->split, s, !captured,
      [&](int f, int l, cudaStream_t st) {
        bt::launch_solve(batch_args(p, a, b, x, f, l, p->d_counter), std::min(p->grid, l - f), st);
      },
      [&](int f, int l, cudaStream_t st) {
        bt64::launch_solve(batch_args(p, a, b, x, f, l, p->d_counter + 1), std::min(p->grid_small, l - f), st);
      }));
  return RM_OK;
}

int batch_plan_create(int64_t count, const int64_t* n, const int64_t* k, const int64_t* a_off, const int64_t* b_off,
                      const int64_t* x_off, const rm_solve_options* opts, BatchPlan** out) {
  if (!out || count < 0 || count > INT_MAX || (count > 0 && (!n || !k || !a_off || !b_off || !x_off)))
    return RM_BAD_ARG;
  for (int64_t i = 0; i < count; ++i)
    if (n[i] < 0 || n[i] > bt::NMAX || k[i] < 0 || k[i] > bt::KMAX || a_off[i] < 0 || b_off[i] < 0 || x_off[i] < 0) {
      set_last_message("batched systems take 0 <= n <= 256 and 0 <= k <= 8");
      return RM_BAD_ARG;
    }
  BatchPlan* p = new BatchPlan();
  p->count = count;
  p->n.assign(n, n + count);
  p->k.assign(k, k + count);
  p->a_off.assign(a_off, a_off + count);
  p->b_off.assign(b_off, b_off + count);
  p->x_off.assign(x_off, x_off + count);
  if (opts) p->opts = *opts;
  else p->opts.method = RM_METHOD_F32_IR, p->opts.fallback = 1;
  const int st = plan_build(p);
  if (st != RM_OK) {
    free_plan(p);
    return st;
  }
  *out = p;
  return RM_OK;
}

void batch_plan_destroy(BatchPlan* p) { free_plan(p); }

// One persistent launch over every system, replayed from a CUDA graph captured on the plan's
// own stream (re-captured when the data pointers change); ordered after prior work on s and
// before later work on s.
int batch_plan_execute(BatchPlan* p, const double* a, const double* b, double* x, cudaStream_t s) {
  if (!p) return RM_BAD_ARG;
  if (p->count == 0) return RM_OK;
  if (!p->graph || p->g_a != a || p->g_b != b || p->g_x != x) {
    if (p->graph) {
      cudaGraphExecDestroy(p->graph);
      p->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    RM_CUDA_TRY(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
    const int st = launch_batch(p, a, b, x, 0, (int)p->count, p->stream, true);
    const cudaError_t e = cudaStreamEndCapture(p->stream, &g);
    if (st != RM_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    RM_CUDA_TRY(e);
    const cudaError_t ie = cudaGraphInstantiate(&p->graph, g, 0);
    cudaGraphDestroy(g);
    RM_CUDA_TRY(ie);
    p->g_a = a, p->g_b = b, p->g_x = x;
  }
  RM_CUDA_TRY(cudaEventRecord(p->ev_in, s));
  RM_CUDA_TRY(cudaStreamWaitEvent(p->stream, p->ev_in, 0));
  RM_CUDA_TRY(cudaGraphLaunch(p->graph, p->stream));
  note_launch();  // the graph's kernels (one, or the two sizes' side by side)
  if (p->split > 0 && p->split < p->count) note_launch();
  RM_CUDA_TRY(cudaEventRecord(p->ev_out, p->stream));
  RM_CUDA_TRY(cudaStreamWaitEvent(s, p->ev_out, 0));
  return RM_OK;
}

// Picks the panel width of each size bucket: each candidate (16, 32) runs the bucket's own
// systems (a contiguous range of the size-sorted order) twice, timed by CUDA events; the
// faster stays. Then the CTA size for the systems of n <= 64: each choice of the largest n
// that the 64-thread build takes (64, 32, or none: all on 256-thread CTAs) runs those systems
// twice, and the fastest stays. The results are the solves of those systems (x is written).
// With `precision` (a mixed plan only), each bucket also times float64 factors without
// refinement beside the float32 widths and keeps whichever is fastest: the systems then still
// meet the plan's backward-error tolerance, by the float64 route.
int batch_plan_tune(BatchPlan* p, const double* a, const double* b, double* x, cudaStream_t s, bool precision) {
  if (!p) return RM_BAD_ARG;
  const int cnt = (int)p->count;
  cudaEvent_t e0, e1;
  RM_CUDA_TRY(cudaEventCreate(&e0));
  RM_CUDA_TRY(cudaEventCreate(&e1));
  int status = RM_OK;
  for (int bk = 0; bk < 5 && status == RM_OK; ++bk) {
    int first = cnt, last = 0;
    for (int i = 0; i < cnt; ++i)
      if (bucket_of(p->n[p->order[i]]) == bk) first = std::min(first, i), last = std::max(last, i + 1);
    if (first >= last) continue;
    float best = INFINITY;
    int best_nb = p->nb_bucket[bk];
    const bool try_f64 = precision && p->opts.method == RM_METHOD_F32_IR;
    for (int cand : {16, 32, 16 | kItemF64}) {
      if ((cand & kItemF64) && !try_f64) continue;
      for (int i = first; i < last; ++i) p->nb_item[i] = cand;
      if (cudaMemcpyAsync(p->d_nb + first, p->nb_item.data() + first, (last - first) * sizeof(int),
                          cudaMemcpyHostToDevice, s) != cudaSuccess) {
        status = RM_CUDA_ERROR;
        break;
      }
      float t = 0.0f;
      for (int rep = 0; rep < 2 && status == RM_OK; ++rep) {
        cudaEventRecord(e0, s);
        status = launch_batch(p, a, b, x, first, last, s);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) status = RM_CUDA_ERROR;
        cudaEventElapsedTime(&t, e0, e1);
      }
      if (t < best) best = t, best_nb = cand;
    }
    if (best_nb & kItemF64) {
      p->f64_bucket[bk] = 1;  // the float32 width stays as it was
    } else {
      p->f64_bucket[bk] = 0;
      p->nb_bucket[bk] = best_nb;
    }
    for (int i = first; i < last; ++i) p->nb_item[i] = p->code(bk);
    if (cudaMemcpyAsync(p->d_nb + first, p->nb_item.data() + first, (last - first) * sizeof(int),
                        cudaMemcpyHostToDevice, s) != cudaSuccess)
      status = RM_CUDA_ERROR;
  }
  const int old_split = p->split;
  int small_first = 0;
  while (small_first < cnt && p->n[p->order[small_first]] > bt64::MAX_N) ++small_first;
  if (status == RM_OK && small_first < cnt) {
    float best = INFINITY;
    int best_limit = p->small_limit;
    for (int limit : {bt64::MAX_N, 32, 0}) {
      p->small_limit = limit;
      set_split(p);
      float t = 0.0f;
      for (int rep = 0; rep < 2 && status == RM_OK; ++rep) {
        cudaEventRecord(e0, s);
        status = launch_batch(p, a, b, x, small_first, cnt, s);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) status = RM_CUDA_ERROR;
        cudaEventElapsedTime(&t, e0, e1);
      }
      if (t < best) best = t, best_limit = limit;
    }
    p->small_limit = best_limit;
    set_split(p);
  }
  cudaStreamSynchronize(s);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ++p->tune_gen;  // execute_host rebuilds its groups with the new widths and split
  // the kernels read the widths from d_nb, so a captured graph stays valid unless the split moved
  if (p->split != old_split && p->graph) {
    cudaGraphExecDestroy(p->graph);
    p->graph = nullptr;
  }
  return status;
}

// ------------------------------------------------------------------ execute from host memory
// The systems in groups of consecutive indices with about equal bytes of A (one group when the
// packed offsets do not follow the indices), each group's items sorted by size, largest first,
// with their panel widths and the first item of the 64-thread kernel.
constexpr int kHostGroups = 6;

static bool packed_in_order(const BatchPlan* p) {
  for (int64_t i = 0; i + 1 < p->count; ++i) {
    const int64_t n = p->n[i], k = p->k[i];
    if (p->a_off[i + 1] < p->a_off[i] + n * n || p->b_off[i + 1] < p->b_off[i] + n * k ||
        p->x_off[i + 1] < p->x_off[i] + n * k)
      return false;
  }
  return true;
}

static int build_groups(BatchPlan* p) {
  const int cnt = (int)p->count;
  std::vector<int> bounds = {0};
  if (cnt > 1 && packed_in_order(p)) {
    int64_t total = 0, acc = 0;
    for (int i = 0; i < cnt; ++i) total += (int64_t)p->n[i] * p->n[i];
    const int G = std::min(kHostGroups, cnt);
    int g = 1;
    for (int i = 0; i + 1 < cnt && g < G; ++i) {
      acc += (int64_t)p->n[i] * p->n[i];
      if (acc * G >= total * g) bounds.push_back(i + 1), ++g;
    }
  }
  bounds.push_back(cnt);
  const int G = (int)bounds.size() - 1;
  p->g_order.resize(cnt);
  p->g_nb.resize(cnt);
  p->g_first.assign(bounds.begin(), bounds.end());
  p->g_split.assign(G, 0);
  for (int g = 0; g < G; ++g) {
    auto b = p->g_order.begin() + bounds[g], e = p->g_order.begin() + bounds[g + 1];
    std::iota(b, e, bounds[g]);
    std::stable_sort(b, e, [&](int x, int y) { return p->n[x] > p->n[y]; });
    int sp = bounds[g];
    while (sp < bounds[g + 1] && p->n[p->g_order[sp]] > p->small_limit) ++sp;
    p->g_split[g] = sp;
  }
  for (int i = 0; i < cnt; ++i) p->g_nb[i] = p->code(bucket_of(p->n[p->g_order[i]]));
  if (!p->d_gsys) {
    RM_TRY(upload(&p->d_gsys, p->g_order));
    RM_TRY(upload(&p->d_gnb, p->g_nb));
  } else {
    RM_CUDA_TRY(cudaMemcpy(p->d_gsys, p->g_order.data(), cnt * sizeof(int), cudaMemcpyHostToDevice));
    RM_CUDA_TRY(cudaMemcpy(p->d_gnb, p->g_nb.data(), cnt * sizeof(int), cudaMemcpyHostToDevice));
  }
  if (!p->copy_in) {
    RM_CUDA_TRY(cudaStreamCreateWithFlags(&p->copy_in, cudaStreamNonBlocking));
    RM_CUDA_TRY(cudaStreamCreateWithFlags(&p->copy_out, cudaStreamNonBlocking));
    RM_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_start, cudaEventDisableTiming));
    RM_CUDA_TRY(cudaEventCreateWithFlags(&p->ev_end, cudaEventDisableTiming));
  }
  while ((int)p->g_in.size() < G) {
    cudaEvent_t e1 = nullptr, e2 = nullptr;
    RM_CUDA_TRY(cudaEventCreateWithFlags(&e1, cudaEventDisableTiming));
    p->g_in.push_back(e1);
    RM_CUDA_TRY(cudaEventCreateWithFlags(&e2, cudaEventDisableTiming));
    p->g_done.push_back(e2);
  }
  p->groups_gen = p->tune_gen;
  return RM_OK;
}

// The packed range [lo, hi) of items that the systems [s0, s1) use in an array with offsets off
// and per-system sizes n * w (w = n for A, k for b and x).
static void packed_range(const BatchPlan* p, const std::vector<int64_t>& off, bool square, int s0, int s1, int64_t& lo,
                         int64_t& hi) {
  lo = INT64_MAX, hi = 0;
  for (int i = s0; i < s1; ++i) {
    lo = std::min(lo, off[i]);
    hi = std::max(hi, off[i] + (int64_t)p->n[i] * (square ? p->n[i] : p->k[i]));
  }
  if (lo > hi) lo = hi;
}

// Host A and b in, the solves, host x out: group by group, the copies of one group overlap the
// solves of another (copy-in, solve and copy-out each on a stream of their own, ordered by
// events). Ordered after prior work on s and before later work on s.
int batch_plan_execute_host(BatchPlan* p, const double* h_a, const double* h_b, double* h_x, double* d_a, double* d_b,
                            double* d_x, cudaStream_t s) {
  if (!p) return RM_BAD_ARG;
  if (p->count == 0) return RM_OK;
  if (p->groups_gen != p->tune_gen) RM_TRY(build_groups(p));
  const int G = (int)p->g_first.size() - 1;
  RM_CUDA_TRY(cudaEventRecord(p->ev_start, s));
  for (cudaStream_t q : {p->copy_in, p->stream, p->copy_out}) RM_CUDA_TRY(cudaStreamWaitEvent(q, p->ev_start, 0));
  for (int g = 0; g < G; ++g) {
    const int s0 = p->g_first[g], s1 = p->g_first[g + 1];  // systems (and items) of the group
    int64_t lo, hi;
    packed_range(p, p->a_off, true, s0, s1, lo, hi);
    if (hi > lo) RM_CUDA_TRY(cudaMemcpyAsync(d_a + lo, h_a + lo, (hi - lo) * 8, cudaMemcpyHostToDevice, p->copy_in));
    packed_range(p, p->b_off, false, s0, s1, lo, hi);
    if (hi > lo) RM_CUDA_TRY(cudaMemcpyAsync(d_b + lo, h_b + lo, (hi - lo) * 8, cudaMemcpyHostToDevice, p->copy_in));
    RM_CUDA_TRY(cudaEventRecord(p->g_in[g], p->copy_in));
    RM_CUDA_TRY(cudaStreamWaitEvent(p->stream, p->g_in[g], 0));
    auto args = [&](int f, int l, int* counter) {
      BatchArgs q = batch_args(p, d_a, d_b, d_x, f, l, counter);
      q.sys = p->d_gsys, q.nb = p->d_gnb;
      return q;
    };
    RM_TRY(launch_split(
        p, s0, s1, p->g_split[g], p->stream, true,
        [&](int f, int l, cudaStream_t st) { bt::launch_solve(args(f, l, p->d_counter), std::min(p->grid, l - f), st); },
        [&](int f, int l, cudaStream_t st) {
          bt64::launch_solve(args(f, l, p->d_counter + 1), std::min(p->grid_small, l - f), st);
        }));
    RM_CUDA_TRY(cudaEventRecord(p->g_done[g], p->stream));
    RM_CUDA_TRY(cudaStreamWaitEvent(p->copy_out, p->g_done[g], 0));
    packed_range(p, p->x_off, false, s0, s1, lo, hi);
    if (hi > lo) RM_CUDA_TRY(cudaMemcpyAsync(h_x + lo, d_x + lo, (hi - lo) * 8, cudaMemcpyDeviceToHost, p->copy_out));
  }
  RM_CUDA_TRY(cudaEventRecord(p->ev_end, p->copy_out));
  RM_CUDA_TRY(cudaStreamWaitEvent(s, p->ev_end, 0));
  return RM_OK;
}

// dL/db = A^-T g and dL/dA = -(dL/db) x^T for every system, from the factors the last
// execute left in the plan (the same a and x); one persistent launch on the plan's stream,
// ordered after prior work on s and before later work on s.
int batch_plan_adjoint(BatchPlan* p, const double* a, const double* x, const double* g, double* gb, double* ga,
                       cudaStream_t s) {
  if (!p) return RM_BAD_ARG;
  if (p->count == 0) return RM_OK;
  RM_CUDA_TRY(cudaEventRecord(p->ev_in, s));
  RM_CUDA_TRY(cudaStreamWaitEvent(p->stream, p->ev_in, 0));
  auto args = [&](int f, int l, int* counter) {
    AdjointArgs aj;
    aj.bt = batch_args(p, a, nullptr, const_cast<double*>(x), f, l, counter);
    aj.g = g, aj.gb = gb, aj.ga = ga, aj.berr = p->d_adj_berr;
    return aj;
  };
  RM_TRY(launch_split(
      p, 0, (int)p->count, p->split, p->stream, true,
      [&](int f, int l, cudaStream_t st) { bt::launch_adjoint(args(f, l, p->d_counter), std::min(p->grid, l - f), st); },
      [&](int f, int l, cudaStream_t st) {
        bt64::launch_adjoint(args(f, l, p->d_counter + 1), std::min(p->grid_small, l - f), st);
      }));
  RM_CUDA_TRY(cudaEventRecord(p->ev_out, p->stream));
  RM_CUDA_TRY(cudaStreamWaitEvent(s, p->ev_out, 0));
  return RM_OK;
}

int batch_plan_adjoint_results(BatchPlan* p, double* berr, double* max_berr) {
  if (!p) return RM_BAD_ARG;
  std::vector<double> be(p->count);
  RM_CUDA_TRY(cudaStreamSynchronize(p->stream));
  if (p->count) RM_CUDA_TRY(cudaMemcpy(be.data(), p->d_adj_berr, p->count * sizeof(double), cudaMemcpyDeviceToHost));
  if (berr) std::copy(be.begin(), be.end(), berr);
  if (max_berr) {
    *max_berr = 0.0;
    for (double v : be) *max_berr = (v != v || *max_berr != *max_berr) ? NAN : std::max(*max_berr, v);
  }
  return RM_OK;
}

int batch_plan_results(BatchPlan* p, double* berr, int32_t* iters, int32_t* flags, rm_batch_report* summary) {
  if (!p) return RM_BAD_ARG;
  const int64_t cnt = p->count;
  std::vector<double> be(cnt);
  std::vector<int> it(cnt), fl(cnt);
  RM_CUDA_TRY(cudaStreamSynchronize(p->stream));
  if (cnt) {
    RM_CUDA_TRY(cudaMemcpy(be.data(), p->d_berr, cnt * sizeof(double), cudaMemcpyDeviceToHost));
    RM_CUDA_TRY(cudaMemcpy(it.data(), p->d_iters, cnt * sizeof(int), cudaMemcpyDeviceToHost));
    RM_CUDA_TRY(cudaMemcpy(fl.data(), p->d_flags, cnt * sizeof(int), cudaMemcpyDeviceToHost));
  }
  if (berr) std::copy(be.begin(), be.end(), berr);
  if (iters) std::copy(it.begin(), it.end(), iters);
  if (flags) std::copy(fl.begin(), fl.end(), flags);
  if (summary) {
    summary->max_backward_error = 0.0;
    summary->fell_back = summary->not_regular = summary->no_convergence = 0;
    summary->max_iterations = 0;
    for (int64_t i = 0; i < cnt; ++i) {
      summary->max_backward_error = std::max(summary->max_backward_error, be[i]);
      if (be[i] != be[i]) summary->max_backward_error = be[i];
      summary->fell_back += (fl[i] & bt::FLAG_FELL_BACK) != 0;
      summary->not_regular += (fl[i] & bt::FLAG_NOT_REGULAR) != 0;
      summary->no_convergence += (fl[i] & bt::FLAG_NO_CONVERGENCE) != 0;
      summary->max_iterations = std::max(summary->max_iterations, it[i]);
    }
  }
  return RM_OK;
}

}  // namespace rm

// ------------------------------------------------------------------ C ABI
struct rm_batch_plan {
  rm::BatchPlan* p;
};

extern "C" {

int rm_batch_plan_create(int64_t count, const int64_t* h_n, const int64_t* h_k, const int64_t* h_a_off,
                         const int64_t* h_b_off, const int64_t* h_x_off, const rm_solve_options* opts,
                         rm_batch_plan** plan) {
  if (!plan) return RM_BAD_ARG;
  *plan = nullptr;
  RM_TRY(rm::check_device());
  rm::BatchPlan* p = nullptr;
  RM_TRY(rm::batch_plan_create(count, h_n, h_k, h_a_off, h_b_off, h_x_off, opts, &p));
  *plan = new rm_batch_plan{p};
  return RM_OK;
}

int rm_batch_plan_tune(rm_batch_plan* plan, const double* d_a, const double* d_b, double* d_x, void* stream) {
  if (!plan || !d_a || !d_b || !d_x) return RM_BAD_ARG;
  RM_TRY(rm::batch_plan_tune(plan->p, d_a, d_b, d_x, reinterpret_cast<cudaStream_t>(stream), false));
  return rm::take_device_status(reinterpret_cast<cudaStream_t>(stream));
}

int rm_batch_plan_tune_precision(rm_batch_plan* plan, const double* d_a, const double* d_b, double* d_x,
                                 void* stream) {
  if (!plan || !d_a || !d_b || !d_x) return RM_BAD_ARG;
  RM_TRY(rm::batch_plan_tune(plan->p, d_a, d_b, d_x, reinterpret_cast<cudaStream_t>(stream), true));
  return rm::take_device_status(reinterpret_cast<cudaStream_t>(stream));
}

int rm_batch_plan_execute(rm_batch_plan* plan, const double* d_a, const double* d_b, double* d_x, void* stream) {
  if (!plan || (plan->p->count > 0 && (!d_a || !d_b || !d_x))) return RM_BAD_ARG;
  return rm::batch_plan_execute(plan->p, d_a, d_b, d_x, reinterpret_cast<cudaStream_t>(stream));
}

int rm_batch_plan_execute_host(rm_batch_plan* plan, const double* h_a, const double* h_b, double* h_x, double* d_a,
                               double* d_b, double* d_x, void* stream) {
  if (!plan || (plan->p->count > 0 && (!h_a || !h_b || !h_x || !d_a || !d_b || !d_x))) return RM_BAD_ARG;
  return rm::batch_plan_execute_host(plan->p, h_a, h_b, h_x, d_a, d_b, d_x, reinterpret_cast<cudaStream_t>(stream));
}

int rm_batch_plan_results(rm_batch_plan* plan, double* h_berr, int32_t* h_iters, int32_t* h_flags,
                          rm_batch_report* summary) {
  if (!plan) return RM_BAD_ARG;
  return rm::batch_plan_results(plan->p, h_berr, h_iters, h_flags, summary);
}

int rm_batch_plan_adjoint(rm_batch_plan* plan, const double* d_a, const double* d_x, const double* d_gx,
                          double* d_gb, double* d_ga, void* stream) {
  if (!plan || (plan->p->count > 0 && (!d_a || !d_x || !d_gx || !d_gb))) return RM_BAD_ARG;
  return rm::batch_plan_adjoint(plan->p, d_a, d_x, d_gx, d_gb, d_ga, reinterpret_cast<cudaStream_t>(stream));
}

int rm_batch_plan_adjoint_results(rm_batch_plan* plan, double* h_berr, double* h_max_berr) {
  if (!plan) return RM_BAD_ARG;
  RM_TRY(rm::batch_plan_adjoint_results(plan->p, h_berr, h_max_berr));
  return rm::take_device_status(nullptr);
}

int rm_batch_plan_panel_width(const rm_batch_plan* plan, int bucket) {
  return plan && bucket >= 0 && bucket < 5 ? plan->p->nb_bucket[bucket] : 0;
}

int rm_batch_plan_precision(const rm_batch_plan* plan, int bucket) {
  if (!plan || bucket < 0 || bucket >= 5) return -1;
  return plan->p->f64_bucket[bucket] ? RM_METHOD_PLAIN_F64 : plan->p->opts.method;
}

int rm_batch_plan_cta_threads(const rm_batch_plan* plan, int bucket) {
  if (!plan || bucket < 0 || bucket >= 5) return 0;
  return rm::kBucketMax[bucket] <= plan->p->small_limit ? rm::bt64::MAX_N : rm::bt::MAX_N;
}

int rm_batch_plan_destroy(rm_batch_plan* plan) {
  if (!plan) return RM_OK;
  rm::batch_plan_destroy(plan->p);
  delete plan;
  return RM_OK;
}

int rm_dlu_factor_batched(int64_t count, int64_t n, const double* d_a, double* d_factors, int64_t* d_perm,
                          int32_t* d_regular, void* stream) {
  if (count < 0 || n < 0 || n > rm::bt::NMAX || (count > 0 && n > 0 && (!d_a || !d_factors || !d_perm)))
    return RM_BAD_ARG;
  if (count == 0 || n == 0) return RM_OK;
  RM_TRY(rm::check_device());
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int64_t ld = (n + 3) & ~3;
  const int64_t stride = (n * ld * 8 + 255) / 256 * 256;
  for (int64_t first = 0; first < count; first += 65536) {
    const int64_t c = std::min<int64_t>(count - first, 65536);
    void* w = nullptr;
    RM_TRY(rm::scratch_alloc(&w, (size_t)(c * stride), s));
    // a CTA per matrix: 64 threads (eight CTAs per SM) up to n = 64, else 256
    const auto launch = n <= rm::bt64::MAX_N ? rm::bt64::launch_factor : rm::bt::launch_factor;
    const int ls = launch(d_a + first * n * n, (int)n, static_cast<unsigned char*>(w), stride, d_factors + first * n * n,
                          d_perm + first * n, d_regular ? d_regular + first : nullptr, (unsigned)c, s);
    const cudaError_t e = ls == RM_OK ? cudaGetLastError() : cudaErrorInvalidValue;
    rm::scratch_free(w, s);
    rm::note_launch();
    if (e != cudaSuccess) {
      rm::set_last_error(e, "batch_factor_kernel", __FILE__, __LINE__);
      return RM_CUDA_ERROR;
    }
  }
  return RM_OK;
}

int rm_dsolve_batched(int64_t count, const int64_t* h_n, const int64_t* h_k, const int64_t* h_a_off,
                      const int64_t* h_b_off, const int64_t* h_x_off, const double* d_a, const double* d_b,
                      double* d_x, const rm_solve_options* opts, rm_batch_report* report, void* stream) {
  rm_batch_plan* plan = nullptr;
  RM_TRY(rm_batch_plan_create(count, h_n, h_k, h_a_off, h_b_off, h_x_off, opts, &plan));
  int st = rm_batch_plan_execute(plan, d_a, d_b, d_x, stream);
  if (st == RM_OK) st = rm::take_device_status(reinterpret_cast<cudaStream_t>(stream));
  if (st == RM_OK) st = rm_batch_plan_results(plan, nullptr, nullptr, nullptr, report);
  rm_batch_plan_destroy(plan);
  if (st == RM_OK && report && report->no_convergence > 0) {
    rm::set_last_message("refinement stalled on some systems and fallback was off");
    return RM_NO_CONVERGENCE;
  }
  return st;
}

}  // extern "C"
