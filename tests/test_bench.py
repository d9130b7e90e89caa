"""bench.py's contract on the CPU: the reference arm's JSON line (the reference's own solver built on the CPU, or the
oracle port where that library is absent, on the host cores, run by rank 0 alone under torchrun) and the cross-rank maximum the GPU arm takes of its timings (world size 2 over gloo)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args, env=None):
    e = dict(os.environ, **(env or {}))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True, env=e, timeout=600)


def test_reference_arm_line():
    r = run_bench("--impl", "reference", "--nx", "8", "--steps", "2", "--warmup", "1")
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "cell-updates/s" and line["value"] > 0
    assert line["steps"] == 2 and line["warmup"] == 1 and line["higher_is_better"] is True
    from oracle import ref as R

    assert line["cpu_baseline"]["kind"] == ("reference" if R.available() else "port")
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["config"]["workload"].startswith("3D static Voronoi 8^3")
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_runs_on_rank_0_only():
    r = run_bench("--impl", "reference", "--nx", "8", "--steps", "1", "--warmup", "1", env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def _max_worker(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    got = bench.max_over_ranks(1.5 + rank, dist, device="cpu")
    dist.barrier()
    out.put((rank, got))
    dist.destroy_process_group()


def test_max_over_ranks_two_ranks_gloo():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_max_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results == {0: 2.5, 1: 2.5}
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.0) == 3.0  # one process: the value itself
