#!/usr/bin/env python
"""Headline benchmark: LU-solve GFLOP/s at n = 8192 to FP64 backward error.

Workload (one step): solve A X = B for a resident 8192 x 8192 FP64 matrix A = U diag(s) V^T,
s_i = kappa^(-i/(n-1)) with kappa = 1e5 (the hardest of {1e2, 1e4, 1e5}), and 16 Gaussian
right-hand sides, to normwise backward error <= n * 2^-53.  GFLOP/s charges the LAPACK nominal
2/3 n^3 + 2 n^2 k flops per solve to every form.  A is 512 MiB, larger than L2, so no flush is
needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--form mixed|plain] [--impl b200|reference]

--impl reference times the reference's own algorithm restated in C++ (the oracle's threaded
ThrMatrixLinEQSolve, all host cores) on the same n = 8192 system: the median of 5 solves after 1
warm-up, whatever --steps / --warmup ask (the line reports the steps it ran).
With N > 1 (torchrun) every rank solves its own system: replicas, no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT, NRHS_DEFAULT, KAPPA_DEFAULT = 8192, 16, 1e5
# DRAM bytes per algorithmic byte of a dominant kernel class, from a single-launch ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum over the bytes the event profiler charges to that
# launch): the tournament leaf of the mixed solve, profiles/tslu_select_n8192_dram.md
NCU_TRAFFIC_RATIO = {"panel": 1.147}
METRIC = "LU-solve GFLOP/s at n=8192 to FP64 backward error: mixed-precision IR vs plain FP64"


def metric_for(n: int) -> str:
    """The headline metric's name; other orders (the C1 case) say which n they ran."""
    return METRIC if n == N_DEFAULT else METRIC.replace("n=8192", f"n={n}")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--form", choices=["mixed", "plain"], default=None)
    p.add_argument("--n", type=int, default=N_DEFAULT)
    p.add_argument("--nrhs", type=int, default=NRHS_DEFAULT)
    p.add_argument("--kappa", type=float, default=KAPPA_DEFAULT)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison steps")
    p.add_argument("--workload", choices=["solve", "gemm", "ozaki", "batched", "adjoint"], default="solve",
                   help="solve: the headline (default); gemm / ozaki: m=n=k=8192 FP64 product with the "
                        "g*2^e distribution; batched: 20,000 uneven systems; adjoint: n=4096 gradient step")
    p.add_argument("--mode", type=int, default=0, help="batched: 0 plain FP64, 1 FP32 + FP64 refinement")
    p.add_argument("--batch-count", type=int, default=20000,
                   help="batched: number of systems (20,000 is the benchmark; smaller counts size profiler captures)")
    p.add_argument("--cpu-runs", type=int, default=3, help="solves in the CPU-baseline sample (median)")
    return p.parse_args()


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 100 ms during the timed region (the
    sampler is running before the region starts; only its samples from then on count)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.first = 0

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a moment to print its first sample: wait for it (at most 3 s) so
            # that the sampling covers the timed region from its start, and count only what
            # arrives after this point
            deadline = time.monotonic() + 3.0
            while not self.lines and time.monotonic() < deadline and self.proc.poll() is None:
                time.sleep(0.02)
            self.first = len(self.lines)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines[self.first:] or self.lines  # a region shorter than one period keeps the last
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- distributed plumbing
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        timeout = datetime.timedelta(seconds=120)
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timeout, device_id=torch.device("cuda", local))
        else:
            # host-only ranks (the reference arm's plumbing, the CPU tests of this code): gloo
            dist.init_process_group("gloo", timeout=timeout)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value: float) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gflops(steps: int, world: int, flops_per_solve: float, ms_max: float) -> float:
    """Whole-job rate: every rank solves its own system each step (replicas), so the job does
    steps x world solves in the slowest rank's time."""
    return steps * world * flops_per_solve / (ms_max / 1e3) / 1e9


# ----------------------------------------------------------------------------- CPU baseline (oracle)
def headline_system_host(n: int, kappa: float, nrhs: int, seed: int):
    """The headline system A = U diag(s) V^T and its right-hand sides as host numpy arrays.  Input
    generation only (torch QR, on the GPU when there is one); it loads nothing of libb2m."""
    import torch

    from mrmath_b200 import inputs  # numpy / torch only
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    A, B = inputs.c2_kappa(n, kappa, nrhs, seed=seed, device=dev)
    a, b = A.cpu().numpy(), B.cpu().numpy()
    del A, B
    if dev == "cuda":
        torch.cuda.empty_cache()
    return a, b


def cpu_solves(a, b, runs: int, warmup: int):
    """The reference's threaded solve (ThrMatrixLinEQSolve, LinAlgLU.pas:986-1128) restated in C++
    (the oracle), on every host core: `warmup` untimed then `runs` timed solves of a x = b."""
    import oracle
    oracle.set_num_threads(os.cpu_count() or 1)
    times, x, rc = [], None, 0
    for i in range(warmup + runs):
        t0 = time.perf_counter()
        rc, x = oracle.thr_lineq_solve(a, b)
        dt = time.perf_counter() - t0
        if i >= warmup:
            times.append(dt)
    return times, x, rc


def cpu_baseline(a, b, runs: int = 3) -> dict:
    """Bounded sample of the headline workload on the host cores: `runs` solves of the same
    n = 8192 system (about 10 s each on 16 cores), median rate."""
    import oracle
    from mrmath_b200 import inputs
    n, k = a.shape[0], b.shape[1]
    times, x, rc = cpu_solves(a, b, runs, 0)
    med = statistics.median(times)
    return {"value": inputs.lu_solve_flops(n, k) / med / 1e9, "unit": "GFLOP/s", "cores": oracle.num_threads(),
            "kind": "port",
            "sample": f"oracle ThrMatrixLinEQSolve restatement on the benchmark system itself (n={n}, {k} RHS), "
                      f"median of {len(times)} solves ({sum(times):.1f} s of CPU work)",
            "backward_error": float(oracle.backward_error(a, x, b)), "status": rc}


def cpu_tuned_blas_context(a, b, runs: int = 3) -> dict:
    """numpy's LAPACK dgesv (OpenBLAS) on the same system and host cores: a tuned CPU BLAS for
    context beside the reference's own algorithm, never the baseline and never on the GPU path."""
    import numpy as np
    from threadpoolctl import threadpool_info

    from mrmath_b200 import inputs
    n, k = a.shape[0], b.shape[1]
    times, x = [], None
    for _ in range(runs):
        t0 = time.perf_counter()
        x = np.linalg.solve(a, b)
        times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    blas = [p for p in threadpool_info() if p.get("user_api") == "blas"]
    r = b - a @ x
    eta = float(np.abs(r).max() / (np.abs(a).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max()))
    return {"what": "numpy.linalg.solve, LAPACK dgesv (tuned CPU BLAS, not the reference; context only)",
            "value": inputs.lu_solve_flops(n, k) / med / 1e9, "unit": "GFLOP/s", "ms_per_step": med * 1e3,
            "threads": blas[0].get("num_threads") if blas else None,
            "library": f"{blas[0].get('internal_api')} {blas[0].get('version')}" if blas else None,
            "sample": f"median of {runs} solves of the benchmark system", "backward_error": eta}


def run_reference(args, world, rank):
    """The reference arm: the reference's own CPU algorithm (the oracle's restatement of
    ThrMatrixLinEQSolve; the Object Pascal reference cannot be compiled in this image) on the same
    n = 8192 system as the B200 arm, median of 5 solves after 1 warm-up.  Nothing of libb2m is loaded."""
    if rank != 0:
        return 0
    import oracle  # noqa: F401  (fails loudly if the oracle is not built)
    from mrmath_b200 import inputs
    n, k = args.n, args.nrhs
    runs, warm = min(args.steps, 5), min(args.warmup, 1)
    a, b = headline_system_host(n, args.kappa, k, seed=15)
    times, x, rc = cpu_solves(a, b, runs, warm)
    med = statistics.median(times)
    fl = inputs.lu_solve_flops(n, k)
    v = fl / med / 1e9
    sample = (f"oracle ThrMatrixLinEQSolve restatement, n={n}, {k} RHS, kappa={args.kappa:g}: median of {runs} "
              f"solves after {warm} warm-up ({sum(times):.1f} s timed)")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GFLOP/s", "n_gpus": args.gpus,
        "steps": runs, "warmup": warm, "requested_steps": args.steps, "requested_warmup": args.warmup,
        "ms_per_step": med * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: A = U diag(s) V^T from MT19937-seeded Gaussians (seed 15), 16 Gaussian RHS",
        "config": {"workload": f"plain FP64 LU solve, n={n}, {k} RHS, kappa={args.kappa:g}", "n": n, "nrhs": k,
                   "kappa": args.kappa, "parallelism": "host threads"},
        "backward_error": float(oracle.backward_error(a, x, b)), "backward_error_bound": n * 2.0 ** -53,
        "status": rc,
        "cpu_baseline": {"value": v, "unit": "GFLOP/s", "cores": oracle.num_threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- B200 arm
def backward_error_torch(A, X, B) -> float:
    import torch
    R = B - A @ X
    na = A.abs().sum(dim=1).max()
    eta = R.abs().amax(dim=0) / (na * X.abs().amax(dim=0) + B.abs().amax(dim=0))
    return float(eta.max().item())


def fp64_peak_tflops() -> float:
    """cuBLAS DGEMM 8192^3 (torch.matmul float64), best of 5: the measured FP64 peak of this GPU."""
    import torch
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2.0 * 8192 ** 3 / best / 1e9


def run_b200(args, world, rank, local):
    import numpy as np
    import torch

    import mrmath_b200
    from mrmath_b200 import inputs, linalg as L

    torch.cuda.set_device(local)
    ctx = mrmath_b200.Context(local)
    n, k = args.n, args.nrhs
    form = args.form or ("mixed" if hasattr(L, "dev_MatrixLinEQSolveMixed") else "plain")
    A, B = inputs.c2_kappa(n, args.kappa, k, seed=15 + rank, device=f"cuda:{local}")
    X = torch.empty_like(B)
    status = torch.zeros(1, dtype=torch.int32, device=A.device)
    flops = inputs.lu_solve_flops(n, k)

    def step():
        if form == "mixed":
            L.dev_MatrixLinEQSolveMixed(A, B, X, status=status, ctx=ctx)
        else:
            L.dev_MatrixLinEQSolve(A, B, X, status=status, ctx=ctx)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    eta = backward_error_torch(A, X, B)

    # ---- timed region: K resident steps, events on torch's stream (the stream libb2m is bound to)
    l0 = ctx.kernel_launches()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(args.steps):
            step()
        ev1.record()
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    barrier(world)
    launches = ctx.kernel_launches() - l0
    ms_max = max_over_ranks(world, ms)
    # the same K steps again with every launch bracketed by CUDA events on its stream: per kernel
    # class device time and algorithmic work for the roofline (kept out of the timed region above)
    ctx.profile(True)
    for _ in range(args.steps):
        step()
    prof = ctx.profile_read()
    ctx.profile(False)
    value = job_gflops(args.steps, world, flops, ms_max)

    # ---- end to end through the host-buffer C ABI (pinned host buffers, copies inside the region)
    e2e = None
    if not args.no_e2e:
        hA = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
        hB = torch.empty((n, k), dtype=torch.float64, pin_memory=True)
        hX = torch.empty((n, k), dtype=torch.float64, pin_memory=True)
        hA.copy_(A)
        hB.copy_(B)
        a_np, b_np, x_np = hA.numpy(), hB.numpy(), hX.numpy()
        ctx.set_stream(0)  # host API on the legacy stream so the events below bracket it
        fn = L.MatrixLinEQSolveMixed if form == "mixed" else L.MatrixLinEQSolve
        fn(a_np, b_np, X=x_np, ctx=ctx)
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        for _ in range(args.steps):
            fn(a_np, b_np, X=x_np, ctx=ctx)
        e1.record(torch.cuda.default_stream())
        torch.cuda.synchronize()
        ems = max_over_ranks(world, e0.elapsed_time(e1))
        eta_e2e = backward_error_torch(A, torch.from_numpy(x_np).to(A.device), B)
        e2e = {"value": job_gflops(args.steps, world, flops, ems), "unit": "GFLOP/s",
               "h2d_bytes_per_step": int(a_np.nbytes + b_np.nbytes), "d2h_bytes_per_step": int(x_np.nbytes),
               "backward_error": eta_e2e, "api": "b2m_MatrixLinEQSolve" + ("Mixed" if form == "mixed" else "")}
        del hA, hB, hX

    # ---- plain FP64 drop-in on the same system (the comparison the metric names)
    plain = None
    if form == "mixed" and not args.no_plain:
        for _ in range(2):
            L.dev_MatrixLinEQSolve(A, B, X, status=status, ctx=ctx)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record()
        for _ in range(args.steps):
            L.dev_MatrixLinEQSolve(A, B, X, status=status, ctx=ctx)
        p1.record()
        torch.cuda.synchronize()
        pms = max_over_ranks(world, p0.elapsed_time(p1))
        pv = job_gflops(args.steps, world, flops, pms)
        plain = {"value": pv, "unit": "GFLOP/s", "ms_per_step": pms / args.steps,
                 "backward_error": backward_error_torch(A, X, B), "mixed_over_plain": value / pv}

    # ---- context only, never the product path: a library FP64 solve (torch.linalg.solve on the
    # cuSOLVER backend: getrf + getrs) of the same system, timed the same way
    library = None
    if form == "mixed" and not args.no_plain:
        try:
            torch.backends.cuda.preferred_linalg_library("cusolver")
            for _ in range(2):
                Xl = torch.linalg.solve(A, B)
            torch.cuda.synchronize()
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            q0.record()
            for _ in range(args.steps):
                Xl = torch.linalg.solve(A, B)
            q1.record()
            torch.cuda.synchronize()
            qms = max_over_ranks(world, q0.elapsed_time(q1))
            library = {"what": "torch.linalg.solve, cuSOLVER getrf + getrs (context only)",
                       "value": job_gflops(args.steps, world, flops, qms), "unit": "GFLOP/s",
                       "ms_per_step": qms / args.steps, "backward_error": backward_error_torch(A, Xl, B)}
            del Xl
        except Exception as exc:
            library = {"what": "torch.linalg.solve (cuSOLVER)", "unavailable": str(exc)[:200]}

    # ---- roofline of the dominant kernel class (by device time in the profiled pass).  The profiler
    # records FLOPs for the tensor-core GEMM classes and HBM bytes for every other class.
    dom_name, d = max(prof.items(), key=lambda kv: kv[1]["ms"])
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    avg_s = d["ms"] / 1e3 / max(1, d["launches"])
    per_launch = d["work"] / max(1, d["launches"])
    share = d["ms"] / max(1e-9, sum(v["ms"] for v in prof.values()))
    if dom_name == "gemm_f64":
        pk = fp64_peak_tflops()
        achieved = per_launch / avg_s / 1e12
        roof = {"bound": "tensor", "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (of measured)"}
        unit = "TFLOP/s"
    elif dom_name == "gemm_tc":
        pk = peaks.get("bf16_tflops", 1590.0) / 2.0
        achieved = per_launch / avg_s / 1e12
        roof = {"bound": "tensor", "peak_source": "TF32 dense = half of measured bf16_tflops (of measured)"}
        unit = "TFLOP/s"
    else:
        pk = peaks.get("hbm_gbs", 6650.0)
        achieved = per_launch / avg_s / 1e9
        roof = {"bound": "hbm", "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks
                else "fallback 6650 GB/s (of fallback)"}
        unit = "GB/s"
    traffic = per_launch * NCU_TRAFFIC_RATIO[dom_name] if (dom_name in NCU_TRAFFIC_RATIO and roof["bound"] == "hbm") else None
    roof.update({"kernel_class": dom_name, "achieved": achieved, "peak": pk, "unit": unit, "frac": achieved / pk,
                 "traffic": traffic, "traffic_unit": "bytes per launch (DRAM read + write, ncu-measured ratio)",
                 "launches": d["launches"], "avg_launch_us": avg_s * 1e6,
                 "work_per_launch": per_launch, "share_of_device_time": share})

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        a_h, b_h = A.cpu().numpy(), B.cpu().numpy()
        try:
            cpu = cpu_baseline(a_h, b_h, runs=args.cpu_runs)
        except Exception as exc:  # the oracle is test infrastructure; report why it is missing
            cpu = {"value": None, "unit": "GFLOP/s", "cores": 0, "kind": "port", "sample": f"unavailable: {exc}"}
        try:
            cpu["tuned_blas_context"] = cpu_tuned_blas_context(a_h, b_h)
        except Exception as exc:
            cpu["tuned_blas_context"] = {"value": None, "what": f"unavailable: {exc}"}

    if rank == 0:
        line = {
            "metric": metric_for(n), "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if form == "plain" else "f32/tf32 factor + f64 refinement",
            "data": "synthetic: A = U diag(s) V^T from MT19937-seeded Gaussians (seed 15 + rank), 16 Gaussian RHS",
            "config": {"workload": f"{'mixed-precision IR' if form == 'mixed' else 'plain FP64'} LU solve, "
                                   f"n={n}, {k} RHS, kappa={args.kappa:g}", "n": n, "nrhs": k,
                       "kappa": args.kappa, "form": form, "parallelism": f"replicas x{world}",
                       "l2": "A (512 MiB) exceeds L2; no flush needed"},
            "backward_error": eta, "backward_error_bound": n * 2.0 ** -53,
            "e2e": e2e, "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu, "plain_fp64": plain,
            "library_fp64_context": library,
            "kernel_classes": {kname: {"launches": v["launches"], "ms": round(v["ms"], 4)}
                               for kname, v in prof.items() if v["launches"]},
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


# ----------------------------------------------------------------------------- secondary workloads
def _timed(fn, steps, warmup):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def run_secondary(args, world, rank, local):
    """The other scope rows, one JSON line each: replicas per rank like the headline."""
    import numpy as np
    import torch

    import mrmath_b200
    from mrmath_b200 import inputs, linalg as L

    torch.cuda.set_device(local)
    ctx = mrmath_b200.Context(local)
    dev = f"cuda:{local}"
    extra = {}
    with ClockSampler(local) as clk:
        if args.workload in ("gemm", "ozaki"):
            n = 8192
            a, b = inputs.c3_gauss_exp(n, n, n, seed=15 + rank)
            A, B = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
            C = torch.empty((n, n), dtype=torch.float64, device=dev)
            if args.workload == "gemm":
                fn = lambda: L.dev_MatrixMultEx(C, A, B, ctx=ctx)
            else:
                fn = lambda: L.dev_MatrixMultOzaki(C, A, B, slices=8, ctx=ctx)
            ms = _timed(fn, args.steps, args.warmup)
            work, unit = 2.0 * n ** 3, "GFLOP/s"
            metric = f"FP64 {'DGEMM (DMMA)' if args.workload == 'gemm' else 'Ozaki int8 GEMM, 8 slices'} GFLOP/s at 8192^3"
            if args.workload == "ozaki":
                ref = torch.empty_like(C)
                L.dev_MatrixMultEx(ref, A, B, ctx=ctx)
                torch.cuda.synchronize()
                scale = (A.abs() @ B.abs()).max()
                extra["max_abs_diff_vs_native_dgemm_over_max_absAabsB"] = float(((C - ref).abs().max() / scale).item())
            config = {"workload": f"C = A B, m=n=k=8192, entries g*2^e (g Gaussian, e uniform in [-8, 8])", "n": n}
            dtype = "f64" if args.workload == "gemm" else "int8 slices -> f64"
        elif args.workload == "batched":
            sizes, nrhs, mats, rhss = inputs.c5_batched(args.batch_count, seed=15 + rank)
            nn, kk, a_off, b_off, Ah, Bh = L.pack_batch(mats, rhss)
            dA, dB = torch.from_numpy(Ah).to(dev), torch.from_numpy(Bh).to(dev)
            dX = torch.zeros_like(dB)
            info = torch.zeros(len(nn), dtype=torch.int32, device=dev)
            iters = torch.zeros_like(info)
            fn = lambda: L.dev_BatchLinEQSolve(nn, kk, a_off, b_off, dA, dB, dX, info, iters, mode=args.mode, ctx=ctx)
            fn()  # the first call with a plan runs the autotuner
            ms = _timed(fn, args.steps, args.warmup)
            work = sum(inputs.lu_solve_flops(int(x), int(y)) for x, y in zip(nn, kk))
            unit = "GFLOP/s"
            metric = f"batched uneven LU solves GFLOP/s ({len(nn):,} systems, n in [8, 256])"
            extra.update({"solves_per_s": len(nn) / (ms / 1e3), "singular": int((info != 0).sum().item()),
                          "tile_shape": L.batch_tune(ctx)})
            if args.mode == 1:
                it = iters.cpu().numpy()
                extra.update({"mean_refinement_steps": float(it[it > 0].mean()), "fp64_fallbacks": int((it < 0).sum())})
            config = {"workload": f"{len(nn):,} systems A = R + n I, 1-4 RHS, {'FP64' if args.mode == 0 else 'FP32 + FP64 IR'}",
                      "count": len(nn), "mode": args.mode}
            dtype = "f64" if args.mode == 0 else "f32 factor + f64 refinement"
        else:  # adjoint
            n = 4096
            r = inputs.rng(4096 + rank)
            a = r.random_sample((n, n)) * 2.0 - 1.0 + n * np.eye(n)
            A = torch.from_numpy(a).to(dev)
            bvec = torch.from_numpy(r.standard_normal((n, 1))).to(dev)
            G = torch.from_numpy(r.standard_normal((n, 1))).to(dev)
            LU = A.clone()
            indx = torch.zeros(n, dtype=torch.int32, device=dev)
            X = torch.empty_like(bvec)
            Lam, dAt = torch.empty_like(bvec), torch.empty_like(A)

            def fn():
                LU.copy_(A)
                L.dev_MatrixLUDecompInPlace(LU, indx, ctx=ctx)
                X.copy_(bvec)
                L.dev_MatrixLUBackSubst(LU, indx, X, ctx=ctx)
                L.dev_MatrixLinEQSolveAdjoint(LU, indx, X, G, Lam, dAt, ctx=ctx)
            ms = _timed(fn, args.steps, args.warmup)
            ms_adj = _timed(lambda: L.dev_MatrixLinEQSolveAdjoint(LU, indx, X, G, Lam, dAt, ctx=ctx), args.steps,
                            args.warmup)
            work = 2.0 / 3.0 * n ** 3 + 4.0 * n * n
            unit = "GFLOP/s"
            metric = "differentiated solve (factor + solve + adjoint with dA) GFLOP/s at n=4096"
            extra.update({"adjoint_only_ms": ms_adj, "adjoint_dA_write_GBs": 8.0 * n * n / (ms_adj / 1e3) / 1e9})
            config = {"workload": "loss = w^T A^-1 b, A = R + 4096 I, dA = -lambda x^T, db = lambda", "n": n}
            dtype = "f64"
    ms_max = max_over_ranks(world, ms)
    if rank == 0:
        line = {"metric": metric, "value": world * work / (ms_max / 1e3) / 1e9, "unit": unit, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic, MT19937-seeded",
                "config": config, "clocks": clk.summary(), **extra}
        print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def main():
    args = parse()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank)
        if args.workload != "solve":
            return run_secondary(args, world, rank, local)
        return run_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
