"""The benchmark's multi-rank plumbing on two host ranks (gloo, world size 2, no GPU).

`bench.py --gpus N` under torchrun runs one independent solve per rank (replicas, no collective on
the data path); the only cross-rank steps are the barriers around the timed region and the maximum
of the ranks' device times.  These tests run that plumbing as two spawned gloo processes:
- `max_over_ranks` returns the slowest rank's time on every rank, and `job_gflops` charges
  steps x world solves to it;
- the reference arm (`--impl reference`) runs on rank 0 alone, prints exactly one JSON line, and the
  other rank exits 0 without work.
The file also checks two host-side pieces of the bench line: the tuned CPU BLAS context and the
clock record (against a fake nvidia-smi).
"""
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank: int, world: int, port: int):
    # host ranks even where GPUs are visible: the gloo path is the one under test
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "CUDA_VISIBLE_DEVICES": ""})
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)


def _plumbing_rank(rank, world, port, q):
    _env(rank, world, port)
    import torch.distributed as dist

    import bench
    w, r, _ = bench.dist_setup()
    try:
        bench.barrier(w)
        ms = 10.0 + 5.0 * r  # rank 1 is the slow one
        q.put((r, w, dist.get_backend(), bench.max_over_ranks(w, ms)))
        bench.barrier(w)
    finally:
        dist.destroy_process_group()


def _reference_rank(rank, world, port, out_dir, q):
    _env(rank, world, port)
    import contextlib
    import io

    import bench
    sys.argv = ["bench.py", "--impl", "reference", "--gpus", str(world), "--steps", "2", "--warmup", "1",
                "--n", "96", "--nrhs", "2", "--kappa", "100"]
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        rc = bench.main()
    q.put((rank, rc, buf.getvalue()))


def _run(target, args, world=2, timeout=300):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, *args, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=timeout) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(out)


def test_max_over_ranks_gloo_two_ranks():
    out = _run(_plumbing_rank, ())
    assert [o[0] for o in out] == [0, 1]
    for _, w, backend, ms_max in out:
        assert w == 2 and backend == "gloo"
        assert ms_max == 15.0


def test_job_rate_counts_every_replica():
    import bench
    flops = 2.0 / 3.0 * 8192 ** 3 + 2.0 * 8192 ** 2 * 16
    one = bench.job_gflops(20, 1, flops, 400.0)
    assert one == pytest.approx(20 * flops / 0.4 / 1e9)
    # two replicas in the same (slowest-rank) time: twice the job's throughput
    assert bench.job_gflops(20, 2, flops, 400.0) == pytest.approx(2 * one)


def test_reference_arm_rank0_only(tmp_path):
    pytest.importorskip("oracle")
    out = _run(_reference_rank, (str(tmp_path),))
    (r0, rc0, s0), (r1, rc1, s1) = out
    assert (r0, r1) == (0, 1) and rc0 == 0 and rc1 == 0
    assert s1.strip() == ""
    lines = [ln for ln in s0.splitlines() if ln.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["config"]["n"] == 96 and line["status"] == 0
    assert line["backward_error"] <= line["backward_error_bound"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"


def test_tuned_blas_context_line():
    """The tuned CPU BLAS context (numpy's dgesv) beside the CPU baseline: labelled as context,
    solves the benchmark's system construction to FP64 backward error."""
    import bench
    a, b = bench.headline_system_host(256, 1e4, 4, seed=15)
    line = bench.cpu_tuned_blas_context(a, b, runs=1)
    assert "not the reference" in line["what"] and line["unit"] == "GFLOP/s"
    assert line["value"] > 0 and line["backward_error"] <= 256 * 2.0 ** -53


def test_clock_sampler_covers_the_region(tmp_path, monkeypatch):
    """The clock record: the sampler waits for nvidia-smi's first sample before the timed region
    starts, counts only the samples taken after that, and reports the median SM clock, the maximum
    and every throttle reason seen active.  A fake nvidia-smi on PATH stands in for the real one."""
    import time

    import bench
    fake = tmp_path / "nvidia-smi"
    fake.write_text(
        "#!/usr/bin/env python3\n"
        "import sys, time\n"
        "time.sleep(0.3)\n"
        "print('0, 1200, 1965, 300, 0x0, Not Active, Not Active, Not Active, Not Active', flush=True)\n"
        "for i in range(100):\n"
        "    time.sleep(0.05)\n"
        "    cap = 'Active' if i == 2 else 'Not Active'\n"
        "    print(f'0, 1965, 1965, 900, 0x4, Not Active, Not Active, Not Active, {cap}', flush=True)\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    with bench.ClockSampler(0) as clk:
        assert clk.first == 1  # the idle sample before the region is excluded
        time.sleep(0.4)
    s = clk.summary()
    assert s["samples"] >= 3 and s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
