#!/usr/bin/env python
"""Benchmark: solves/s at FP64 backward error on one B200, the single large system.

Workload: one float64 system, n = 8192, nrhs = 16, A = U diag(s) V^T with U, V the Q factors
of seeded 8192 x 8192 N(0,1) matrices and s log-spaced from 1 to 1e-4 (kappa = 1e4), B with
N(0,1) entries. A "step" is one complete solve of that system through the library's C ABI
(LU, pivot check, triangular solves and, for the mixed method, FP64 refinement to the
backward-error target n * 2^-53). Inputs are generated on the GPU with torch's seeded
generator (an 8192^2 QR in NumPy would take minutes); A is 512 MiB, larger than L2, so no
flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the CPU oracle (a C restatement of rustymath's LU solve; the Rust
reference cannot be built here) on the host cores, on the same system.
One JSON line on stdout (rank 0)."""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s at FP64 backward error: TC+refinement vs plain FP64 LU on one B200"
WORKLOAD = "single system n=8192 nrhs=16, A=U diag(logspace(0,-4)) V^T (kappa=1e4), B~N(0,1)"


def _jsonable(o):
    """NumPy scalars (and anything else json does not know) as plain Python values."""
    if isinstance(o, np.generic):
        return o.item()
    if isinstance(o, np.ndarray):
        return o.tolist()
    return str(o)


_collect = False  # set while the headline run gathers the other configurations' lines


def _emit(line):
    """Prints a workload's JSON line, or hands it back while the headline run collects them."""
    if not _collect:
        print(json.dumps(line, default=_jsonable), flush=True)
    return line


def other_configs(args, local):
    """The other configurations, measured in the same run on one GPU (each its own timed region,
    after the headline's): n = 512 (plain and mixed solves, 512^3 product), the 20,000 uneven
    systems, the 4096-system adjoint and the 16384^3 GEMM. A leg that fails reports its error."""
    global _collect
    out = {}
    _collect = True
    try:
        for name, fn in (("c1_n512", run_small), ("c3_batched_20000", run_batched),
                         ("c4_adjoint_4096x64", run_adjoint), ("c5_gemm_16384", run_gemm)):
            t0 = time.perf_counter()
            try:
                sub = fn(args, 0, 1, local)
                sub["wall_s"] = time.perf_counter() - t0
                out[name] = sub
            except Exception as e:  # noqa: BLE001 - reported in the line, the headline stands
                out[name] = {"error": f"{type(e).__name__}: {e}"}
    finally:
        _collect = False
    return out


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=8192)
    p.add_argument("--nrhs", type=int, default=16)
    p.add_argument("--method", default="auto", choices=["auto", "plain", "mixed"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-other-configs", action="store_true",
                   help="headline only: skip the other configurations' legs of the default run")
    p.add_argument("--solve-only", action="store_true",
                   help="only the timed solves (for profiling): no e2e, roofline or CPU legs")
    p.add_argument("--workload", default="single", choices=["single", "batched", "adjoint", "gemm", "update", "small"],
                   help="single: the n=8192 system (the headline); batched: 20,000 uneven systems")
    p.add_argument("--count", type=int, default=20000, help="systems in the batched workload")
    p.add_argument("--uniform-n", type=int, default=0,
                   help="batched workload with every system of this order (a profiling case; 0: the U{8..256} mix)")
    return p.parse_args()


def make_system(n, nrhs, seed, device):
    """A = U diag(s) V^T (U, V: Q of QR of seeded N(0,1) matrices; U first), B ~ N(0,1)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    u = torch.linalg.qr(torch.randn(n, n, generator=g, device=device, dtype=torch.float64)).Q
    v = torch.linalg.qr(torch.randn(n, n, generator=g, device=device, dtype=torch.float64)).Q
    s = torch.logspace(0, -4, n, device=device, dtype=torch.float64)
    a = (u * s) @ v.T
    b = torch.randn(n, nrhs, generator=g, device=device, dtype=torch.float64)
    del u, v
    return a.contiguous(), b.contiguous()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_baseline(a_host, b_host, threads=None):
    """The oracle's solve (rustymath's algorithm restated in C) on this host's cores."""
    from oracle import oracle as O
    cores = threads or os.cpu_count()
    O.set_threads(cores)
    n, k = b_host.shape
    t0 = time.perf_counter()
    x = O.solve(a_host, b_host)
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"1 full solve n={n} nrhs={k} (oracle lu_factor+lu_solve, OpenMP)", "seconds": dt}, x


def gemm_peak_f64(torch, dev):
    """Measured FP64 GEMM rate of cuBLAS (torch.matmul float64, 8192^3, best of 5)."""
    n = 8192
    a = torch.randn(n, n, device=dev, dtype=torch.float64)
    b = torch.randn(n, n, device=dev, dtype=torch.float64)
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    return 2.0 * n ** 3 / best / 1e12


def time_dgemm_update(torch, lib, dev, n, k=128, reps=10):
    """One representative launch of the dominant kernel: the rank-128 trailing update."""
    m = n - k
    a = torch.randn(m, k, device=dev, dtype=torch.float64)
    b = torch.randn(k, m, device=dev, dtype=torch.float64)
    c = torch.randn(m, m, device=dev, dtype=torch.float64)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(3):
        lib.rm_dgemm(0, 0, m, m, k, -1.0, a.data_ptr(), k, b.data_ptr(), m, 1.0, c.data_ptr(), m, s)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        lib.rm_dgemm(0, 0, m, m, k, -1.0, a.data_ptr(), k, b.data_ptr(), m, 1.0, c.data_ptr(), m, s)
    e1.record()
    e1.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    return 2.0 * m * m * k / t / 1e12, t


def time_sgemm_update(torch, lib, dev, n, k=128, reps=10):
    """One launch of the mixed LU's dominant tensor-core kernel: the rank-128 trailing update
    A22 -= L21 U12 (3xTF32 tcgen05 GEMM, beta = 1) at the first step's size. It is HBM-bound:
    its algorithmic bytes are C read and written once (8 bytes per item) plus the two panels."""
    m = n - k
    a = torch.randn(m, k, device=dev, dtype=torch.float32)
    b = torch.randn(m, k, device=dev, dtype=torch.float32)
    c = torch.randn(m, m, device=dev, dtype=torch.float32)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def go():
        return lib.rm_sgemm_tc(3, 1, m, m, k, -1.0, a.data_ptr(), k, b.data_ptr(), k, 1.0, c.data_ptr(), m, s)

    for _ in range(3):
        assert go() == 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        go()
    e1.record()
    e1.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    bytes_ = m * m * 8 + 2 * m * k * 4
    return bytes_ / t / 1e9, t, bytes_, 3 * 2.0 * m * m * k / t / 1e12


def time_cusolver(torch, a, b, reps=3):
    """A comparison point, not part of the product path: torch.linalg.lu_factor + lu_solve
    (cuSOLVER getrf/getrs) on the same float64 system, timed by CUDA events."""
    prev = torch.backends.cuda.preferred_linalg_library()
    torch.backends.cuda.preferred_linalg_library("cusolver")
    try:
        def go():
            lu, piv = torch.linalg.lu_factor(a)
            return torch.linalg.lu_solve(lu, piv, b)

        go()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            xs = go()
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / reps
        r = (b - a @ xs).abs().max().item()
        berr = r / (a.abs().sum(1).max().item() * xs.abs().max().item() + b.abs().max().item())
        return {"ms_per_solve": 1e3 * t, "solves_per_s": 1.0 / t, "backward_error": berr,
                "what": "torch.linalg.lu_factor + lu_solve with the cuSOLVER backend (getrf + getrs), float64"}
    finally:
        torch.backends.cuda.preferred_linalg_library(prev)


def parity_vs_oracle(a, b, x_oracle, arms, kappa):
    """Each arm's solution against the oracle's (rustymath's lu_factor + lu_solve restated):
    the normwise relative forward difference max_c ||x_c - xo_c||inf / ||xo_c||inf, and the
    backward error of each from the oracle's double-double residual. The plain arm is held to
    n eps, the others to kappa n eps."""
    import scipy.linalg as sl
    from oracle import oracle as O
    n = a.shape[0]
    eps = np.finfo(np.float64).eps

    def fwd_of(x):
        return float((np.abs(x - x_oracle).max(0) / np.abs(x_oracle).max(0)).max())

    # a third float64 LU (LAPACK getrf/getrs through SciPy): how far two correct float64 solves
    # with different rounding orders lie apart on this system
    lapack = sl.lu_solve(sl.lu_factor(a, check_finite=False), b, check_finite=False)
    out = {"oracle_backward_error": O.backward_error(a, x_oracle, b), "kappa": kappa,
           "lapack_vs_oracle": fwd_of(lapack), "n_eps": n * eps,
           "note": "forward error = max over columns of ||x - x_oracle||inf / ||x_oracle||inf; two backward-stable "
                   "float64 solves differ by up to about kappa times their backward errors, so every arm is held to "
                   "kappa n eps; lapack_vs_oracle is the same difference for LAPACK's getrf + getrs"}
    for name, x in arms.items():
        fwd = fwd_of(x)
        bound = kappa * n * eps
        out[name] = {"forward_error_vs_oracle": fwd, "bound": bound, "within_bound": bool(fwd <= bound),
                     "over_n_eps": fwd / (n * eps), "backward_error_dd": O.backward_error(a, x, b)}
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    import torch
    dev = "cuda:0" if torch.cuda.is_available() else "cpu"
    a, b = make_system(args.n, args.nrhs, 0, dev)
    a_h, b_h = a.cpu().numpy(), b.cpu().numpy()
    del a, b
    from oracle import oracle as O
    cores = os.cpu_count()
    O.set_threads(cores)
    for _ in range(max(0, min(args.warmup, 1))):
        O.solve(a_h, b_h)
    times = []
    x = None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        x = O.solve(a_h, b_h)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = args.steps / total
    berr = O.backward_error(a_h, x, b_h)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "method": "oracle restatement of rustymath lu_factor + lu_solve"},
            "backward_error": berr,
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": f"{args.steps} full solves n={args.n} nrhs={args.nrhs}"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line, default=_jsonable), flush=True)


BATCH_METRIC = "solves/s at FP64 backward error, batched uneven systems (FP32 LU + FP64 refinement) on one B200"
BATCH_WORKLOAD = ("20,000 systems, n~U{8..256}, nrhs~U{1..4} (numpy default_rng(1)); A=N(0,1)+n*I, B=N(0,1) "
                  "(torch seeded generator on the GPU)")


# DRAM bytes (read + write) that ncu measured for the timed mixed launch over the first 2,000
# systems of the batched configuration (shapes from default_rng(1)); traffic grows with the
# systems' sum of n^2, so the full batch's is estimated from it
BATCH_TRAFFIC_2000 = 1522427904 + 282152448


def batch_traffic_estimate(ns):
    ref = np.random.default_rng(1).integers(8, 257, 2000).astype(np.int64)
    return BATCH_TRAFFIC_2000 * float((np.asarray(ns, np.int64) ** 2).sum()) / float((ref ** 2).sum())


def make_batch(count, seed, device, uniform_n=0):
    """Shapes from numpy's default_rng(seed) as the configuration states; entries from torch's
    seeded generator on the GPU (same distributions): A = N(0,1) + n I, B = N(0,1). uniform_n > 0
    gives every system that order instead (for profiling one size)."""
    import torch
    rng = np.random.default_rng(seed)
    ns = rng.integers(8, 257, count)
    ks = rng.integers(1, 5, count)
    if uniform_n:
        ns[:] = uniform_n
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    a = torch.randn(int((ns * ns).sum()), generator=g, device=device, dtype=torch.float64)
    b = torch.randn(int((ns * ks).sum()), generator=g, device=device, dtype=torch.float64)
    # + n on each diagonal: flat indices a_off[i] + j (n_i + 1), j < n_i
    a_off = np.concatenate([[0], np.cumsum(ns * ns)[:-1]])
    starts = np.repeat(a_off, ns)
    within = np.arange(int(ns.sum())) - np.repeat(np.concatenate([[0], np.cumsum(ns)[:-1]]), ns)
    idx = starts + within * np.repeat(ns + 1, ns)
    a[torch.as_tensor(idx, device=device)] += torch.as_tensor(np.repeat(ns, ns).astype(np.float64), device=device)
    return ns, ks, a, b


def cpu_batched(ns, ks, a_h, b_h, count_sample):
    """The oracle's solve per system, one system per host thread (as rustymath's parallel::stack)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    O.set_threads(1)
    cores = os.cpu_count()
    a_off = np.concatenate([[0], np.cumsum(ns * ns)[:-1]])
    b_off = np.concatenate([[0], np.cumsum(ns * ks)[:-1]])
    idx = list(range(min(count_sample, len(ns))))

    def one(i):
        n, k = int(ns[i]), int(ks[i])
        return O.solve(a_h[a_off[i]:a_off[i] + n * n].reshape(n, n), b_h[b_off[i]:b_off[i] + n * k].reshape(n, k))

    t0 = time.perf_counter()
    with ThreadPoolExecutor(cores) as ex:
        list(ex.map(one, idx))
    dt = time.perf_counter() - t0
    return {"value": len(idx) / dt, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"the first {len(idx)} systems of the batch, oracle lu_factor+lu_solve, one system per thread"}


def peak_hbm():
    return peak_hbm_source()[0]


def peak_hbm_source():
    """(GB/s, where it comes from): the measured copy bandwidth when MEASURED_PEAKS.json is
    present, else 6650 GB/s, an earlier measurement on this kind of GPU (the fallback)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (burst copy), of measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6650 GB/s (MEASURED_PEAKS.json absent), of fallback"


def run_batched(args, rank, world, local):
    import torch
    dev = f"cuda:{local}"
    torch.cuda.set_device(dev)
    import rustymath_b200 as rb
    from rustymath_b200 import _lib
    lib = _lib.load()
    ns, ks, a, b = make_batch(args.count, 1 + rank, dev, args.uniform_n)
    x = torch.zeros(int((ns * ks).sum()), dtype=torch.float64, device=dev)

    def arm(method, steps, clocks=None, precision=False):
        plan = rb.BatchPlan(ns, ks, method=method)
        widths = plan.tune(a, b, x, precision=precision)
        for _ in range(max(args.warmup, 1)):
            plan.execute(a, b, x)
        torch.cuda.synchronize()
        l0 = lib.rm_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with (clocks if clocks is not None else _Null()):
            e0.record()
            for _ in range(steps):
                plan.execute(a, b, x)
            e1.record()
            torch.cuda.synchronize()
        launches = (lib.rm_launch_count() - l0) // steps
        t = e0.elapsed_time(e1) / 1e3 / steps
        return plan, t, plan.results()[3], widths, int(launches)

    _, t_plain, rep_plain, w_plain, _ = arm("plain", max(1, min(args.steps, 3)))
    x_plain = x.clone()
    clocks = ClockSampler(local)
    plan, t, rep, widths, launches = arm("mixed", args.steps, clocks)
    x_mixed = x.clone()
    # the tuner's precision axis: per size bucket, float32 factors + refinement or float64 factors
    plan_p, t_p, rep_p, _, _ = arm("mixed", max(1, min(args.steps, 3)), precision=True)
    tuned = {"solves_per_s": len(ns) / t_p, "ms_per_step": 1e3 * t_p, "backward_error_max": rep_p.max_backward_error,
             "route_by_bucket": plan_p.precision(), "buckets": "n <= 32, 64, 128, 192, 256",
             "note": "BatchPlan(method='mixed').tune(precision=True): each bucket keeps the faster of float32 "
                     "factors + float64 refinement and float64 factors; every system still <= n 2^-53"}
    del plan_p
    plan.execute(a, b, x)  # x holds the mixed arm's answer again for the copies and checks below
    torch.cuda.synchronize()
    count = len(ns)
    # end to end: pinned host A, B -> device, the launch, X -> host, every step
    a_h = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    b_h = torch.empty(b.shape, dtype=torch.float64, pin_memory=True)
    x_h = torch.empty(x.shape, dtype=torch.float64, pin_memory=True)
    a_h.copy_(a)
    b_h.copy_(b)
    e2e_steps = max(1, min(args.steps, 3))
    plan.execute_host(a_h, b_h, x_h, a, b, x)  # warm-up: builds the plan's copy groups
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        plan.execute_host(a_h, b_h, x_h, a, b, x)  # group by group: copies overlap the solves
        torch.cuda.synchronize()
    e2e_t = (time.perf_counter() - t0) / e2e_steps
    assert torch.equal(x_h, x.cpu())
    a_bytes = int((ns * ns).sum()) * 8
    passes = 1 + rep.max_iterations + 1  # A read to factor, then once per residual
    line = {"metric": BATCH_METRIC, "value": count / t, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": BATCH_WORKLOAD if not args.uniform_n else
                       f"{count} systems n={args.uniform_n}, nrhs~U{{1..4}}, A=N(0,1)+n*I (profiling case)",
                       "count": count, "panel_widths_by_bucket": widths, "cta_threads_by_bucket": plan.cta_threads(),
                       "l2": "inputs larger than L2 (A is %.1f GB)" % (a_bytes / 1e9)},
            "backward_error_max": rep.max_backward_error, "fell_back": rep.fell_back,
            "max_iterations": rep.max_iterations,
            "plain_fp64": {"solves_per_s": count / t_plain, "ms_per_step": 1e3 * t_plain,
                           "backward_error_max": rep_plain.max_backward_error},
            "tuned_precision": tuned,
            "roofline": {"bound": "hbm", "kernel": "batch_solve_kernel (whole batch; the n <= 64 systems on a "
                                                 "second launch beside it when the tuner keeps them there)",
                         "achieved": passes * a_bytes / t / 1e9, "peak": peak_hbm(), "unit": "GB/s",
                         "frac": passes * a_bytes / t / 1e9 / peak_hbm(),
                         "traffic": batch_traffic_estimate(ns),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the timed mixed launch "
                                           "on the first 2,000 systems of this configuration (1.80 GB), scaled by "
                                           "sum(n^2) to these systems (profiles/batch_solve_kernel_n256x1000.md)",
                         "note": "algorithmic bytes: A read once to factor plus once per residual"},
            "e2e": {"value": count / e2e_t, "unit": "solves/s", "h2d_bytes_per_step": a_bytes + int(b.numel()) * 8,
                    "d2h_bytes_per_step": int(x.numel()) * 8, "api": "BatchPlan.execute_host (pinned host buffers; copies overlap the solves)"},
            "gpu_launches": launches, "clocks": clocks.summary()}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_batched(ns, ks, a_h.numpy(), b_h.numpy(), 2000)
        line["parity_vs_oracle"] = batch_parity(ns, ks, a_h.numpy(), b_h.numpy(),
                                                {"plain_fp64": x_plain.cpu().numpy(), "mixed": x_mixed.cpu().numpy()},
                                                sample=500)
    return _emit(line)


def batch_parity(ns, ks, a_h, b_h, arms, sample, seed=0):
    """A seeded sample of the batch against the oracle's solve, system by system: each arm's
    normwise relative forward difference from the oracle's x; the plain arm held to n eps, the
    mixed one to kappa_inf n eps (kappa of the sampled system, from NumPy)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    O.set_threads(1)
    eps = np.finfo(np.float64).eps
    a_off = np.concatenate([[0], np.cumsum(ns * ns)[:-1]])
    b_off = np.concatenate([[0], np.cumsum(ns * ks)[:-1]])
    idx = np.sort(np.random.default_rng(seed).choice(len(ns), min(sample, len(ns)), replace=False))

    def one(i):
        n, k = int(ns[i]), int(ks[i])
        a = a_h[a_off[i]:a_off[i] + n * n].reshape(n, n)
        b = b_h[b_off[i]:b_off[i] + n * k].reshape(n, k)
        xo = O.solve(a, b)
        kappa = float(np.linalg.cond(a, np.inf))
        res = {}
        for name, xs in arms.items():
            x = xs[b_off[i]:b_off[i] + n * k].reshape(n, k)
            fwd = float((np.abs(x - xo).max(0) / np.abs(xo).max(0)).max())
            bound = n * eps if name == "plain_fp64" else kappa * n * eps
            res[name] = (fwd, fwd / bound)
        return res

    # one BLAS thread per worker: NumPy's LAPACK calls (cond) from many threads at once, each
    # multithreaded, oversubscribe the cores (200x slower)
    from threadpoolctl import threadpool_limits
    with threadpool_limits(1), ThreadPoolExecutor(os.cpu_count()) as ex:
        rows = list(ex.map(one, idx))
    out = {"systems_checked": len(idx), "sample": f"{len(idx)} systems drawn by default_rng({seed})"}
    for name in arms:
        fwd = [r[name][0] for r in rows]
        ratio = [r[name][1] for r in rows]
        out[name] = {"max_forward_error_vs_oracle": max(fwd), "max_error_over_bound": max(ratio),
                     "over_bound": int(sum(bool(q > 1) for q in ratio)),
                     "bound": "n eps" if name == "plain_fp64" else "kappa_inf n eps"}
    return out


ADJ_METRIC = "gradient solves/s: forward + adjoint (dA, db) of 4096 systems n=64 nrhs=2 on one B200"


def run_adjoint(args, rank, world, local):
    """4096 systems n = 64, k = 2, A = N(0,1)/8 + I, b ~ N(0,1), loss sum(w * x): the forward
    batched solve and the adjoint kernel (dL/db = A^-T w, dL/dA = -dL/db x^T)."""
    import torch
    dev = f"cuda:{local}"
    torch.cuda.set_device(dev)
    import rustymath_b200 as rb
    from rustymath_b200 import _lib
    lib = _lib.load()
    batch, n, k = 4096, 64, 2
    g = torch.Generator(device=dev)
    g.manual_seed(1 + rank)
    a = (torch.randn(batch, n, n, generator=g, device=dev, dtype=torch.float64) / 8
         + torch.eye(n, device=dev, dtype=torch.float64)).reshape(-1).contiguous()
    b = torch.randn(batch * n * k, generator=g, device=dev, dtype=torch.float64)
    w = torch.randn(batch * n * k, generator=g, device=dev, dtype=torch.float64)
    x = torch.empty_like(b)
    gb = torch.empty_like(b)
    ga = torch.empty_like(a)
    plan = rb.BatchPlan([n] * batch, [k] * batch, method="mixed")

    def step():
        plan.execute(a, b, x)
        plan.adjoint(a, x, w, gb, ga)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    l0 = lib.rm_launch_count()
    clocks = ClockSampler(local)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    fwd = bwd = 0.0
    with clocks:
        for _ in range(args.steps):
            e0.record()
            plan.execute(a, b, x)
            e1.record()
            plan.adjoint(a, x, w, gb, ga)
            e2.record()
            torch.cuda.synchronize()
            fwd += e0.elapsed_time(e1) / 1e3
            bwd += e1.elapsed_time(e2) / 1e3
    launches = (lib.rm_launch_count() - l0) // args.steps
    t = (fwd + bwd) / args.steps
    berr, mx = plan.adjoint_results()
    da_bytes = batch * n * n * 8
    # end to end through the public differentiable call: every step copies A, b and w in from
    # pinned host memory, runs rustymath_b200.autograd.solve and loss.backward(), and copies
    # dL/dA and dL/db back
    from rustymath_b200 import autograd
    a_h = a.view(batch, n, n).cpu().pin_memory()
    b_h = b.view(batch, n, k).cpu().pin_memory()
    w_h = w.view(batch, n, k).cpu().pin_memory()
    ga_h = torch.empty(a_h.shape, dtype=torch.float64).pin_memory()
    gb_h = torch.empty(b_h.shape, dtype=torch.float64).pin_memory()

    def e2e_step():
        ad = a_h.to(dev, non_blocking=True).requires_grad_()
        bd = b_h.to(dev, non_blocking=True).requires_grad_()
        wd = w_h.to(dev, non_blocking=True)
        (autograd.solve(ad, bd) * wd).sum().backward()
        ga_h.copy_(ad.grad, non_blocking=True)
        gb_h.copy_(bd.grad, non_blocking=True)
        torch.cuda.synchronize()

    for _ in range(2):
        e2e_step()
    e2e_steps = max(3, args.steps)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_t = (time.perf_counter() - t0) / e2e_steps
    assert torch.allclose(gb_h.view(-1).to(dev), gb) and torch.allclose(ga_h.view(-1).to(dev), ga)
    e2e = {"value": batch / e2e_t, "unit": "systems/s (forward + backward)",
           "h2d_bytes_per_step": (batch * n * n + 2 * batch * n * k) * 8,
           "d2h_bytes_per_step": (batch * n * n + batch * n * k) * 8,
           "api": "rustymath_b200.autograd.solve + loss.backward(), pinned copies"}
    line = {"metric": ADJ_METRIC, "value": batch / t, "unit": "systems/s (forward + backward)", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "4096 systems n=64 nrhs=2, A=N(0,1)/8+I, b,w~N(0,1) (torch seeded generator)",
                       "forward_ms": 1e3 * fwd / args.steps, "adjoint_ms": 1e3 * bwd / args.steps},
            "adjoint_backward_error_max": mx,
            "roofline": {"bound": "hbm", "kernel": "batch_adjoint_kernel",
                         "achieved": (2 * da_bytes) / (bwd / args.steps) / 1e9, "peak": peak_hbm(), "unit": "GB/s",
                         "frac": (2 * da_bytes) / (bwd / args.steps) / 1e9 / peak_hbm(), "traffic": 212.07e6 + 91.30e6,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the timed launch at "
                                           "full size (profiles/batch_kernels_n64x4096.md)",
                         "note": "algorithmic bytes: A read once (transposed residual) + dA written once"},
            "e2e": e2e, "gpu_launches": launches, "clocks": clocks.summary()}
    return _emit(line)


GEMM_METRIC = "FP64-accurate GEMM TFLOP/s at 16384^3: Ozaki int8 split vs native FP64 on one B200"


def run_gemm(args, rank, world, local):
    """C = A B at 16384^3, A and B ~ U(-1,1) with rows of A (columns of B) scaled by 10^U(-3,3):
    the native FP64 DMMA GEMM (rm_dgemm), the Ozaki int8 split GEMM (rm_dgemm_ozaki, 8 slices)
    and cuBLAS FP64 (torch.matmul) for reference; errors on 4096 sampled entries against
    extended-precision dot products (numpy longdouble)."""
    import torch
    dev = f"cuda:{local}"
    torch.cuda.set_device(dev)
    import rustymath_b200 as rb
    from rustymath_b200 import _lib
    lib = _lib.load()
    n = args.n if args.n != 8192 else 16384
    g = torch.Generator(device=dev)
    g.manual_seed(5 + rank)
    a = (torch.rand(n, n, generator=g, device=dev, dtype=torch.float64) * 2 - 1) * \
        10.0 ** (torch.rand(n, 1, generator=g, device=dev, dtype=torch.float64) * 6 - 3)
    b = (torch.rand(n, n, generator=g, device=dev, dtype=torch.float64) * 2 - 1) * \
        10.0 ** (torch.rand(1, n, generator=g, device=dev, dtype=torch.float64) * 6 - 3)
    c = torch.empty_like(a)
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def native():
        _lib.check(lib.rm_dgemm(0, 0, n, n, n, 1.0, a.data_ptr(), n, b.data_ptr(), n, 0.0, c.data_ptr(), n, sp), "dgemm")

    def ozaki():
        _lib.check(lib.rm_dgemm_ozaki(n, n, n, a.data_ptr(), n, b.data_ptr(), n, c.data_ptr(), n, 8, sp), "ozaki")

    def cublas():
        torch.matmul(a, b, out=c)

    rng = np.random.default_rng(0)
    rows, cols = rng.integers(0, n, 4096), rng.integers(0, n, 4096)
    a_s = a[torch.as_tensor(rows, device=dev)].cpu().numpy().astype(np.longdouble)
    b_s = b[:, torch.as_tensor(cols, device=dev)].cpu().numpy().astype(np.longdouble)
    ref = np.einsum("ij,ji->i", a_s, b_s)
    mag = np.einsum("ij,ji->i", np.abs(a_s), np.abs(b_s))

    def timed(fn, steps, clocks=None):
        for _ in range(max(args.warmup, 3) if steps > 1 else 1):
            fn()
        torch.cuda.synchronize()
        l0 = lib.rm_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with (clocks if clocks is not None else _Null()):
            e0.record()
            for _ in range(steps):
                fn()
            e1.record()
            torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / steps
        got = c[torch.as_tensor(rows, device=dev), torch.as_tensor(cols, device=dev)].cpu().numpy()
        err = np.abs(got.astype(np.longdouble) - ref).astype(np.float64) / mag.astype(np.float64)
        return t, float(err.max()), (lib.rm_launch_count() - l0) // steps

    steps = max(1, min(args.steps, 3))
    t_nat, e_nat, _ = timed(native, steps)
    t_cub, e_cub, _ = timed(cublas, steps)
    clocks = ClockSampler(local)
    t_oz, e_oz, launches = timed(ozaki, steps, clocks)
    fl = 2.0 * n ** 3
    gemv = gemv_legs(torch, lib, a, dev, max(3, steps))
    cross = gemm_cross_check(torch, lib, dev) if not args.no_cpu_baseline else None
    line = {"metric": GEMM_METRIC, "value": fl / t_oz / 1e12, "unit": "TFLOP/s (FP64-equivalent)", "n_gpus": world,
            "steps": steps, "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * t_oz, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int8 slices -> f64", "data": "synthetic",
            "config": {"workload": f"C=A B at {n}^3, U(-1,1) rows/cols scaled by 10^U(-3,3) (torch seeded)",
                       "slices": 8},
            "max_rel_error_vs_|A||B|": {"ozaki": e_oz, "native_fp64": e_nat, "cublas_fp64": e_cub},
            "native_fp64": {"tflops": fl / t_nat / 1e12, "ms": 1e3 * t_nat},
            "cublas_fp64": {"tflops": fl / t_cub / 1e12, "ms": 1e3 * t_cub},
            "cross_check_2048_vs_oracle": cross, "gemv": gemv,
            "gpu_launches": int(launches), "clocks": clocks.summary()}
    return _emit(line)


def gemv_legs(torch, lib, a, dev, steps):
    """y = A x and y = A^T x through rm_dgemm (n = 1: by_vector's shapes, the HBM-bound stream
    kernels) on the n x n operand A of the GEMM legs (larger than L2): GB/s of A read per call
    (CUDA events) against the measured copy bandwidth, and the largest difference from cuBLAS's
    product relative to |A||x|."""
    from rustymath_b200 import _lib
    n = a.shape[0]
    x = torch.rand(n, 1, device=dev, dtype=torch.float64) * 2 - 1
    y = torch.empty(n, 1, device=dev, dtype=torch.float64)
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = {"workload": f"A {n}x{n} float64 ({8 * n * n / 1e9:.1f} GB), x ~ U(-1,1)", "peak_gbs": peak_hbm()}
    for name, ta in (("a_x", 0), ("at_x", 1)):
        def call():
            _lib.check(lib.rm_dgemm(ta, 0, n, 1, n, 1.0, a.data_ptr(), n, x.data_ptr(), 1, 0.0, y.data_ptr(), 1, sp),
                       "gemv")
        for _ in range(3):
            call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            call()
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / steps
        op = a.T if ta else a
        ref = op @ x
        mag = op.abs() @ x.abs()
        gbs = 8.0 * n * n / t / 1e9
        out[name] = {"ms": 1e3 * t, "gbs": gbs, "frac": gbs / peak_hbm(),
                     "max_rel_diff_vs_cublas": float(((y - ref).abs() / mag).max())}
    return out


def gemm_cross_check(torch, lib, dev, n=2048, seed=5):
    """rm_dgemm and rm_dgemm_ozaki (8 slices) at n^3 against the oracle's product (rustymath's
    PlusTimes.inner restated: packed 6 x 8 micro-kernel, in-order FMA), on the same wide-range
    inputs (U(-1,1), rows of A and columns of B scaled by 10^U(-3,3), default_rng(seed)): the
    largest difference of an item relative to (|A||B|)_ij, and the oracle's own time."""
    from oracle import oracle as O
    from rustymath_b200 import _lib
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 1, (n, n)) * 10.0 ** rng.uniform(-3, 3, (n, 1))
    b = rng.uniform(-1, 1, (n, n)) * 10.0 ** rng.uniform(-3, 3, (1, n))
    O.set_threads(os.cpu_count())
    t0 = time.perf_counter()
    ref = O.dgemm(a, b)
    t_cpu = time.perf_counter() - t0
    mag = np.abs(a) @ np.abs(b)
    ta, tb = torch.tensor(a, device=dev), torch.tensor(b, device=dev)
    tc = torch.empty_like(ta)
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = {"n": n, "oracle_seconds": t_cpu, "oracle_threads": os.cpu_count(),
           "what": "max_ij |C_ij - C_oracle_ij| / (|A||B|)_ij"}
    _lib.check(lib.rm_dgemm(0, 0, n, n, n, 1.0, ta.data_ptr(), n, tb.data_ptr(), n, 0.0, tc.data_ptr(), n, sp), "dgemm")
    out["native_fp64"] = float((np.abs(tc.cpu().numpy() - ref) / mag).max())
    _lib.check(lib.rm_dgemm_ozaki(n, n, n, ta.data_ptr(), n, tb.data_ptr(), n, tc.data_ptr(), n, 8, sp), "ozaki")
    out["ozaki_8_slices"] = float((np.abs(tc.cpu().numpy() - ref) / mag).max())
    out["bound"] = n * np.finfo(np.float64).eps
    out["within_bound"] = bool(max(out["native_fp64"], out["ozaki_8_slices"]) <= out["bound"])
    return out


def run_small(args, rank, world, local):
    """The size rustymath already runs on CPU: one n = 512 system (A = N(0,1) + 512 I, b ~ N(0,1),
    nrhs = 1) by the plain and the mixed method, and C = A B at 512^3 (U(-1,1)); against the
    oracle on 1 host thread and on all of them. Device time per call (CUDA events) and the
    host-pointer call's wall time."""
    import torch
    dev = f"cuda:{local}"
    torch.cuda.set_device(dev)
    import rustymath_b200 as rb
    from rustymath_b200 import _lib
    from oracle import oracle as O
    lib = _lib.load()
    n = 512
    rng = np.random.default_rng(0)
    a_h = rng.standard_normal((n, n)) + n * np.eye(n)
    b_h = rng.standard_normal((n, 1))
    ga, gb = rng.uniform(-1, 1, (n, n)), rng.uniform(-1, 1, (n, n))
    a, b = torch.tensor(a_h, device=dev), torch.tensor(b_h, device=dev)
    x = torch.empty_like(b)
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    reps = max(args.steps, 20)

    def dev_time(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    def host_time(fn):
        fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        return (time.perf_counter() - t0) / reps

    out = {}
    for meth in ("plain", "mixed"):
        opts = rb.linalg._options(meth)
        rep = _lib.SolveReport()
        xs = np.zeros((n, 1))
        out[f"solve_{meth}_ms"] = 1e3 * dev_time(lambda: lib.rm_dsolve(n, a.data_ptr(), b.data_ptr(), 1, x.data_ptr(),
                                                                         ctypes.byref(opts), ctypes.byref(rep), sp))
        out[f"solve_{meth}_host_ms"] = 1e3 * host_time(lambda: lib.rm_dsolve_host(
            n, a_h.ctypes.data, b_h.ctypes.data, 1, xs.ctypes.data, ctypes.byref(opts), ctypes.byref(rep)))
        out[f"solve_{meth}_backward_error"] = O.backward_error(a_h, xs, b_h)
        xo = O.solve(a_h, b_h)
        out[f"solve_{meth}_max_rel_diff_vs_oracle"] = float(np.abs(xs - xo).max() / np.abs(xo).max())
    ta, tb = torch.tensor(ga, device=dev), torch.tensor(gb, device=dev)
    tc = torch.empty_like(ta)
    out["matmul_ms"] = 1e3 * dev_time(lambda: lib.rm_dgemm(0, 0, n, n, n, 1.0, ta.data_ptr(), n, tb.data_ptr(), n, 0.0,
                                                             tc.data_ptr(), n, sp))
    cref = O.dgemm(ga, gb)
    out["matmul_max_abs_diff_vs_oracle"] = float(np.abs(tc.cpu().numpy() - cref).max())
    cpu = {}
    for threads in (1, os.cpu_count()):
        O.set_threads(threads)
        cpu[f"solve_ms_{threads}t"] = 1e3 * host_time(lambda: O.solve(a_h, b_h))
        cpu[f"matmul_ms_{threads}t"] = 1e3 * host_time(lambda: O.dgemm(ga, gb))
    line = {"metric": "n=512 solve and 512^3 matmul (the size rustymath runs on CPU)", "value": 1e3 / out["solve_plain_ms"],
            "unit": "solves/s (plain, device time)", "n_gpus": world, "steps": reps, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic", "config": {"workload": "n=512 nrhs=1, A=N(0,1)+512 I; 512^3 U(-1,1)"},
            "gpu": out, "cpu_baseline": {"kind": "port", "cores": os.cpu_count(), **cpu},
            "gflops": {"solve_plain": (2 / 3 * n ** 3 + 2 * n * n) / out["solve_plain_ms"] / 1e6,
                       "matmul": 2 * n ** 3 / out["matmul_ms"] / 1e6}}
    return _emit(line)


def run_update(args, rank, world, local):
    """The headline roofline's kernel alone: the mixed LU's first rank-128 trailing update
    (3xTF32 tcgen05, m = n = n - 128, k = 128, beta = 1), timed by CUDA events (for profiling)."""
    import torch
    dev = f"cuda:{local}"
    torch.cuda.set_device(dev)
    from rustymath_b200 import _lib
    lib = _lib.load()
    gbs, t, bytes_, tf = time_sgemm_update(torch, lib, dev, args.n, reps=max(args.steps, 1))
    print(json.dumps({"workload": f"rank-128 update m=n={args.n - 128} k=128 (3xTF32)", "achieved_gbs": gbs,
                      "peak_gbs": peak_hbm(), "peak_source": peak_hbm_source()[1], "frac": gbs / peak_hbm(),
                      "launch_us": 1e6 * t,
                      "bytes_per_launch": bytes_, "tf32_tflops": tf}), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "batched":
        return run_batched(args, rank, world, local)
    if args.workload == "adjoint":
        return run_adjoint(args, rank, world, local)
    if args.workload == "gemm":
        return run_gemm(args, rank, world, local)
    if args.workload == "update":
        return run_update(args, rank, world, local)
    if args.workload == "small":
        return run_small(args, rank, world, local)

    import torch
    import torch.distributed as dist
    dev = f"cuda:{local}"
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import rustymath_b200 as rb
    from rustymath_b200 import _lib
    from rustymath_b200.parallel import max_over_ranks
    lib = _lib.load()

    n, k = args.n, args.nrhs
    a, b = make_system(n, k, rank, dev)
    x = torch.empty_like(b)
    method = args.method if args.method != "auto" else "mixed"
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    def timed(meth, steps, warmup, clocks=None):
        """(seconds for `steps` solves, max over ranks; report; launches per solve)"""
        opts = rb.linalg._options(meth)
        rep = _lib.SolveReport()

        def step():
            st = lib.rm_dsolve(n, a.data_ptr(), b.data_ptr(), k, x.data_ptr(), ctypes.byref(opts), ctypes.byref(rep),
                               sp)
            _lib.check(st, "rm_dsolve")

        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        launches0 = lib.rm_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with (clocks if clocks is not None else _Null()):
            torch.cuda.synchronize()
            e0.record()
            for _ in range(steps):
                step()
            e1.record()
            torch.cuda.synchronize()
        launches = (lib.rm_launch_count() - launches0) // max(steps, 1)
        elapsed = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        return elapsed, rep, launches

    # the plain float64 LU first (the comparison arm), then the headline method
    plain_t, plain_rep, plain_launches = timed("plain", max(1, min(args.steps, 3)), args.warmup)
    plain = {"solves_per_s": world * max(1, min(args.steps, 3)) / plain_t,
             "ms_per_solve": 1e3 * plain_t / max(1, min(args.steps, 3)), "backward_error": plain_rep.backward_error,
             "gpu_launches": int(plain_launches)}
    x_plain = x.clone()
    clocks = ClockSampler(local)
    elapsed, rep, launches = timed(method, args.steps, args.warmup, clocks)
    x_main = x.clone()
    value = world * args.steps / elapsed
    berr = rep.backward_error
    method_used = "plain FP64 LU" if rep.method_used == _lib.RM_METHOD_PLAIN_F64 else "FP32 LU + FP64 refinement"

    if args.solve_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "solves/s", "n": n, "nrhs": k,
                              "ms_per_step": 1e3 * elapsed / args.steps, "backward_error": rep.backward_error,
                              "method": method_used, "gpu_launches": int(launches), "plain_fp64": plain,
                              "iterations": rep.iterations, "fell_back": rep.fell_back}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    # ---- end to end through the host API, pinned host buffers, copies inside the timed region
    a_h = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
    b_h = torch.empty((n, k), dtype=torch.float64, pin_memory=True)
    x_h = torch.empty((n, k), dtype=torch.float64, pin_memory=True)
    a_h.copy_(a)
    b_h.copy_(b)
    an, bn, xn = a_h.numpy(), b_h.numpy(), x_h.numpy()
    e2e_steps = max(1, min(args.steps, 3))
    opts = rb.linalg._options(method)
    rep = _lib.SolveReport()
    lib.rm_dsolve_host(n, an.ctypes.data, bn.ctypes.data, k, xn.ctypes.data, ctypes.byref(opts), ctypes.byref(rep))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        st = lib.rm_dsolve_host(n, an.ctypes.data, bn.ctypes.data, k, xn.ctypes.data, ctypes.byref(opts),
                                ctypes.byref(rep))
        _lib.check(st, "rm_dsolve_host")
    e2e_t = (time.perf_counter() - t0) / e2e_steps
    e2e = {"value": world / e2e_t, "unit": "solves/s", "h2d_bytes_per_step": (n * n + n * k) * 8,
           "d2h_bytes_per_step": n * k * 8, "api": "rm_dsolve_host (pinned host buffers)"}

    if rank == 0:
        # ---- roofline of the mixed path's dominant tensor-core kernel (the 3xTF32 rank-128
        # update, HBM-bound) and, beside it, the plain path's FP64 DMMA update
        gbs, t_upd, bytes_upd, tf32_tflops = time_sgemm_update(torch, lib, dev, n)
        roofline = {"bound": "hbm", "kernel": "sgemm_tc_kernel<3,TMA> rank-128 update m=n=8064 k=128 (3xTF32)",
                    "achieved": gbs, "peak": peak_hbm(), "unit": "GB/s", "frac": gbs / peak_hbm(),
                    "peak_source": peak_hbm_source()[1],
                    "bytes_per_launch": bytes_upd, "launch_us": 1e6 * t_upd, "tf32_tflops": tf32_tflops,
                    "traffic": 276.83e6 + 200.59e6,
                    "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of this launch at full size "
                                      "(bench.py --workload update, the 4th GEMM launch)",
                    "timing_note": "launch_us is the rm_sgemm_tc call: the two low-part splits of the panels "
                                   "(2 x 4 MB) and the GEMM launch"}
        peak64 = gemm_peak_f64(torch, dev)
        achieved, t_launch = time_dgemm_update(torch, lib, dev, n)
        roofline["plain_path_dgemm"] = {"bound": "tensor", "kernel": "dgemm_kernel<128x128> rank-128 update",
                                        "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                                        "frac": achieved / peak64,
                                        "peak_source": "cuBLAS FP64 GEMM 8192^3 in this run (no FP64 figure in "
                                                       "MEASURED_PEAKS.json)"}
        cusolver = time_cusolver(torch, a, b)
        cpu, parity = None, None
        if not args.no_cpu_baseline:
            cpu, x_cpu = cpu_baseline(a_h.numpy(), b_h.numpy())
            parity = parity_vs_oracle(a_h.numpy(), b_h.numpy(), x_cpu,
                                      {"plain_fp64": x_plain.cpu().numpy(), "headline": x_main.cpu().numpy()},
                                      kappa=1e4)
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
                "plain_fp64": plain, "speedup_vs_plain_fp64": value / plain["solves_per_s"],
                "refinement_iterations": rep.iterations, "fell_back": rep.fell_back,
                "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if method == "plain" else "f32+f64",
                "data": "synthetic",
                "config": {"workload": WORKLOAD, "method": method_used, "n": n, "nrhs": k,
                           "l2": "inputs larger than L2 (A is 512 MiB)", "parallelism": f"replicas x{world}"},
                "backward_error": berr, "backward_error_target": n * 2.0 ** -53,
                "parity_vs_oracle": parity, "cusolver_fp64": cusolver,
                "speedup_vs_cusolver_fp64": value / cusolver["solves_per_s"],
                "plain_vs_cusolver_time_ratio": plain["ms_per_solve"] / cusolver["ms_per_solve"],
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clocks.summary(), "tflops_lu": (2.0 / 3.0) * n ** 3 / (elapsed / args.steps) / 1e12 * world}
        if world == 1 and not args.no_other_configs:
            line["other_configs"] = other_configs(args, local)
        print(json.dumps(line, default=_jsonable), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
