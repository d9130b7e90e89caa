"""Benchmark of the hydro step: cell-updates/s of luna-cpp's FiniteVolume<3> step (time_step + step) on a 128^3 static
Voronoi mesh, FP64 against FP32, on N GPUs (one process per GPU; replicas: the step does not shard).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--nx 128] [--impl luna|reference]
    python -m torch.distributed.run --nproc-per-node N bench.py --gpus N ...

Workload: 128^3 generators on a unit periodic lattice with uniform jitter +-0.1 spacing (mt19937_64 seed 1), ideal gas
gamma 5/3, point blast (rho 1, v 0, p 1e-5, E = 1 in the cells whose centroid lies within 2 cell widths of the centre),
MUSCL-Hancock + HLLC with the face-centroid limiter, CFL 0.3. Synthetic inputs of the configuration's shape (the
reference uses no dataset). One step = time_step(0.3) (primitives, sweep, CFL reduction, the read of dt) + step(dt)
(face fluxes, update). The working set (~3 GB) is larger than L2 (126 MB), so no flush is needed between steps.
Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s at 128^3 3D Voronoi (FP64 vs FP32)"
UNIT = "cell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--nx", type=int, default=128)
    ap.add_argument("--impl", default="luna", choices=["luna", "reference"])
    ap.add_argument("--cpu-sample-steps", type=int, default=5)
    ap.add_argument("--cpu-warmup", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="leave out the learned limiter's section")
    ap.add_argument("--no-moving", action="store_true", help="leave out the moving-mesh section")
    ap.add_argument("--no-adjoint", action="store_true", help="leave out the adjoint's cost")
    ap.add_argument("--moving-steps", type=int, default=5)
    ap.add_argument("--curve", default="row", choices=["row", "morton", "hilbert"],
                    help="the cells' numbering along a space-filling curve (voronoi-cpp's Layout::curve)")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "fp32", "single", "grad16"],
                    help="which policies to time (the JSON line needs both; one is for profiling runs)")
    return ap.parse_args()


def algorithmic_bytes(faces_per_cell: float, gradient_bytes: int = 120) -> dict:
    """Algorithmic HBM bytes per cell update of the static step (each array read once per phase, neighbour gathers
    counted once, no stored flux rows), per phase:
      G (gradient sweep): Q 40 + V 8 + centroid 24 + position 24 + CSR start 4 + list entries 4 * 2F/N
                          + face rows 56 F/N (owner+neighbour 8, area 24, centroid 24) + gradient row written
      F (fluxes+update):  face rows 56 F/N + Q read 40 + gradient row read + centroid 24 + position 24 + V 8 + Q 40
    With F/N = 7.95 and FP64 gradient rows (120 B): 728.8 + 701.2 = 1430 B. The kernel split: the sweep is phase G; the
    flux kernel reads the face rows and the cell rows (phase F without the Q traffic); the update reads Q and writes Q;
    the fused pass (crossing faces, then the tiles' fluxes and update) is phase F."""
    fpc = faces_per_cell
    g = 40 + 8 + 24 + 24 + 4 + 4 * 2 * fpc + 56 * fpc + gradient_bytes
    f = 56 * fpc + 40 + gradient_bytes + 24 + 24 + 8 + 40
    return {"step": g + f, "sweep": g, "fluxes": 56 * fpc + gradient_bytes + 24 + 24 + 8 + 40, "update": 80.0 + 4 + 4 * 2 * fpc,
            "primitives": 40 + 8 + 56, "flux_and_update": f}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_cell():
    """DRAM bytes per cell per launch from the committed ncu summary (profiles/ncu_traffic_*.txt), or None."""
    out = {}
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return out
    for name in sorted(os.listdir(pdir)):
        if not (name.startswith("ncu_traffic") and name.endswith(".txt")):
            continue
        for line in open(os.path.join(pdir, name)):
            m = re.match(r"\s*bytes_per_cell\s+(\w+)\s+(\w+)\s*=\s*([0-9.eE+-]+)", line)
            if m:
                out[(m.group(1), m.group(2))] = float(m.group(3))
    return out


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"luna_bench_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def build_workload(nx: int, threads: int, curve: str = "row"):
    from luna_cpp_b200.mesh import build_mesh, curve_order, jittered_points
    from luna_cpp_b200.problems import point_blast

    points = jittered_points((nx, nx, nx), jitter=0.1, seed=1)
    mesh = build_mesh(points[curve_order(points, curve=curve)], threads=threads)
    return mesh, point_blast(mesh)


def workload_name(nx: int) -> str:
    """The configuration both arms run (the same string in both JSON lines)."""
    return (f"3D static Voronoi {nx}^3 jittered (0.1) point blast, MUSCL-Hancock + HLLC, face-centroid limiter, CFL 0.3, "
            "FP64, one step = time_step + step")


def cpu_solver(mesh, threads: int):
    """The reference's CPU path of the step on this mesh: its own FiniteVolume<3> built on the CPU (oracle/_ref, OpenMP)
    where that library exists, else the C restatement of it (the oracle port, OpenMP). OMP_PROC_BIND=close is set before
    either OpenMP runtime starts."""
    os.environ.setdefault("OMP_PROC_BIND", "close")
    from oracle import ref as R

    if R.available():
        used = R.threads(threads)
        return R.ReferenceFV(mesh), "reference", used
    from oracle import oracle as O

    used = O.threads(threads)
    return O.OracleFV(mesh), "port", used


def cpu_steps(fv, steps: int, warmup: int) -> list:
    """Wall time of each of `steps` whole steps (time_step + step) after `warmup` untimed ones."""
    for _ in range(warmup):
        fv.step(fv.time_step(0.3))
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        fv.step(fv.time_step(0.3))
        times.append(time.perf_counter() - t0)
    return times


def cpu_baseline(mesh, q0, steps: int, warmup: int, threads: int):
    """The reference's CPU path on the same mesh and state: the median of `steps` step times after `warmup` steps."""
    fv, kind, used = cpu_solver(mesh, threads)
    fv.set_state(q0)
    times = cpu_steps(fv, steps, warmup)
    med = float(np.median(times))
    what = "the reference's FiniteVolume<3> built on the CPU" if kind == "reference" else "the oracle port"
    return {"value": mesh.n_cells / med, "unit": UNIT, "cores": used, "kind": kind,
            "sample": f"median of {steps} steps of {what} after {warmup} warm-up steps, the same {mesh.n_cells}-cell "
                      f"mesh and state, OMP_PROC_BIND={os.environ.get('OMP_PROC_BIND')}",
            "ms_per_step": 1e3 * med}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path of the step (its own FiniteVolume<3> built on the CPU with OpenMP, or
    the oracle port where that library is absent), all host threads, on the same workload; rank 0 only. Each step is
    timed on its own; the value is the cells over the median step time."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    mesh, q0 = build_workload(args.nx, threads, args.curve)
    fv, kind, used = cpu_solver(mesh, threads)
    fv.set_state(q0)
    times = cpu_steps(fv, args.steps, args.warmup)
    med = float(np.median(times))
    value = mesh.n_cells / med
    what = "the reference's FiniteVolume<3> built on the CPU" if kind == "reference" else "the oracle port"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * med, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_name(args.nx), "n_cells": mesh.n_cells, "n_faces": mesh.n_faces,
                       "parallelism": "replicas"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": kind,
                             "sample": f"median of {args.steps} steps of {what} after {args.warmup} warm-up steps, "
                                       f"OMP_PROC_BIND={os.environ.get('OMP_PROC_BIND')}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def max_over_ranks(x: float, dist=None, device="cuda") -> float:
    """The largest value of x over the ranks (every rank gets it): the job's time is its slowest replica's."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def learned_section(mesh, q0, steps, warmup, stream, torch) -> dict:
    """The learned limiter beside the plain one (the metric's second half, L1 error per GPU time): (1) the FP64 step on
    this mesh with the shipped trained network against the plain step, CUDA events, the same steps; (2) four held-out
    seeded Riemann problems (quasi-1D strips of 1024 x 4 cells, the training's distribution) run to the same time by
    plain and learned at the base resolution and by plain at 1.5x, each judged by the density profile's L1 against the
    method's own 4x run, with the device time of each run (strips this small are bound by launches)."""
    from luna_cpp_b200 import hydro
    from luna_cpp_b200 import limiter_training as T
    from luna_cpp_b200.learned import LimiterMLP, trained_params

    net = LimiterMLP(trained_params())
    step_ms = {}
    for mode in ("plain", "learned"):
        fv = hydro.FiniteVolume(mesh)
        fv.set_stream(stream)
        if mode == "learned":
            fv.set_limiter("learned", net.params)
        fv.set_state(q0)
        for _ in range(warmup):
            fv.step(fv.time_step(0.3))
        step_ms[mode] = timed_steps(fv, steps, torch) / steps
        fv.close()
    rows = T.evaluate(net, [5000, 5001, 5002, 5003], nx=1024, ny=4, resolutions=(1.0, 1.5), log=lambda s: None)
    summary = T.summarize(rows, resolutions=(1.0, 1.5))
    gm, ms = summary["geomean_l1"], summary["mean_device_ms"]
    return {"step_ms_at_this_mesh": step_ms, "learned_step_cost": step_ms["learned"] / step_ms["plain"],
            "riemann_strips": {"problems": 4, "cells": 4096,
                               "plain": {"l1": gm["plain@1.0"], "device_ms": ms["plain@1.0"]},
                               "learned": {"l1": gm["learned@1.0"], "device_ms": ms["learned@1.0"]},
                               "plain_1.5x": {"l1": gm["plain@1.5"], "device_ms": ms["plain@1.5"]},
                               "plain_resolution_of_equal_error": summary["plain_resolution_of_equal_error"]}}


def moving_section(nx, steps, warmup) -> dict:
    """The moving-mesh configuration's step at nx^3 (the point blast on snapped jittered generators, generators moved with
    the gas plus the roundness velocity, fluxes on the old and the new faces, FP32 fluxes with FP64 state: the
    reference's Precision<double, float, float, float>, "single": face states, Riemann solve and flux rows in float),
    with the mesh rebuilt on the GPU every step: the hydro part's device time (CUDA events around the
    hydro kernels, the geometry rows of the new mesh included; the remesh outside, as the reference's hydro part) and
    the whole step's wall time (remesh and taking the new mesh included), after ``warmup`` steps."""
    from luna_cpp_b200 import hydro
    from luna_cpp_b200.mesh import jittered_points
    from luna_cpp_b200.problems import point_blast
    from luna_cpp_b200.remesh import Remesher
    from luna_cpp_b200.studies import run_moving

    grid = 2.0 ** -30
    pts = np.round(jittered_points((nx, nx, nx), jitter=0.1, seed=1) / grid) * grid
    remesher = Remesher(3, (1.0, 1.0, 1.0))
    mesh = remesher.build(pts)
    fv = hydro.FiniteVolume(mesh, precision="single", motion="moving")
    fv.set_state(point_blast(mesh.cells()))
    run_moving(fv, 1.0, max_steps=warmup, remesher=remesher)
    r = run_moving(fv, 1.0, max_steps=steps, remesher=remesher)
    N, n = mesh.n_cells, r["steps"]
    out = {"workload": f"3D moving point blast {nx}^3 jittered (0.1), FP64 state / FP32 fluxes (single), CFL 0.3, remesh on "
                       "the GPU every step",
           "steps": n, "warmup": warmup, "hydro_ms_per_step": r["hydro_device_ms"] / n,
           "hydro_cell_updates_per_s": N * n / (r["hydro_device_ms"] * 1e-3),
           "remesh_ms_per_step": 1e3 * r["remesh_s"] / n, "mesh_load_ms_per_step": 1e3 * r["mesh_load_s"] / n,
           "step_ms": 1e3 * r["wall_s"] / n, "cell_updates_per_s": N * n / r["wall_s"]}
    fv.close()
    remesher.close()
    return out


def adjoint_section(mesh, q0, steps, warmup, stream, torch) -> dict:
    """The adjoint's cost on the bench mesh, FP64: device time of step_adjoint (primitives and the sweep recomputed with
    the fit kept, the faces' Riemann adjoints, the cells' adjoints, the gather) against the forward step (time_step +
    step), both over `steps` calls after `warmup`, CUDA events on the library's stream. The reference measures 2.46x
    (its step_adjoint against its step at 128^3 in double, A100)."""
    from luna_cpp_b200 import hydro

    fv = hydro.FiniteVolume(mesh)
    fv.set_stream(stream)
    fv.set_state(q0)
    for _ in range(warmup):
        fv.step(fv.time_step(0.3))
    fwd_ms = timed_steps(fv, steps, torch) / steps
    dt = fv.time_step(0.3)
    qbar = torch.randn(mesh.n_cells, 5, dtype=torch.float64, device="cuda") * 1e-3
    for _ in range(2):
        fv.step_adjoint(dt, qbar)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for _ in range(steps):
        fv.step_adjoint(dt, qbar)
    end.record()
    torch.cuda.synchronize()
    adj_ms = start.elapsed_time(end) / steps
    fv.close()
    return {"step_ms": fwd_ms, "step_adjoint_ms": adj_ms, "ratio": adj_ms / fwd_ms, "reference_ratio": 2.46,
            "finite": bool(torch.isfinite(qbar).all().item())}


def fused_section(mesh, q0, steps, warmup, stream, torch, two_kernel_ms, two_kernel_bytes) -> dict:
    """The static FP64 step with the fused flux-and-update pass (LUNA_FUSED_STEP=1: a tile's interior faces solved into
    shared memory, the faces between tiles by their own pass), the same workload: its time a step against the default
    two-kernel pass and its device memory."""
    from luna_cpp_b200 import hydro

    old = os.environ.get("LUNA_FUSED_STEP")
    os.environ["LUNA_FUSED_STEP"] = "1"
    try:
        fv = hydro.FiniteVolume(mesh)
        fv.set_stream(stream)
        fv.set_state(q0)
        for _ in range(warmup):
            fv.step(fv.time_step(0.3))
    finally:
        if old is None:
            del os.environ["LUNA_FUSED_STEP"]
        else:
            os.environ["LUNA_FUSED_STEP"] = old
    fv.set_timing(True)
    fv.timings(reset=True)
    ms = timed_steps(fv, steps, torch) / steps
    phases = fv.timings(reset=True)
    fused, crossing = fv.fused_pass()
    out = {"fused": fused, "ms_per_step": ms, "vs_two_kernel": two_kernel_ms / ms,
           "phases_ms_per_step": {"crossing_faces": phases["fluxes"][0] / steps, "tiles": phases["update"][0] / steps,
                                  "sweep": phases["sweep"][0] / steps},
           "crossing_fraction": crossing / mesh.n_faces, "device_bytes": fv.device_bytes(),
           "two_kernel_device_bytes": two_kernel_bytes}
    fv.close()
    return out


def timed_steps(fv, steps, torch):
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for _ in range(steps):
        fv.step(fv.time_step(0.3))
    end.record()
    torch.cuda.synchronize()
    return start.elapsed_time(end)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch

    from luna_cpp_b200 import hydro

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    threads = max(1, (os.cpu_count() or 1) // world)
    mesh, q0 = build_workload(args.nx, threads, args.curve)
    N, F = mesh.n_cells, mesh.n_faces
    stream = torch.cuda.current_stream().cuda_stream

    def barrier():
        if dist is not None:
            dist.barrier()

    results = {}
    for prec in ("single", "fp32", "grad16", "fp64") if args.precision == "both" else (args.precision,):
        fv = hydro.FiniteVolume(mesh, precision=prec)
        fv.set_stream(stream)
        fv.set_state(q0)
        for _ in range(args.warmup):
            fv.step(fv.time_step(0.3))
        fv.set_timing(True)
        fv.timings(reset=True)
        barrier()
        clocks = Clocks(local)
        with clocks:
            ms = timed_steps(fv, args.steps, torch)
        barrier()
        phases = fv.timings(reset=True)
        fv.set_timing(False)
        ms = max_over_ranks(ms, dist)
        results[prec] = {"ms": ms, "phases": phases, "clocks": clocks.summary(), "fallbacks": fv.fallbacks(), "fv": fv,
                         "fused": fv.fused_pass()}

    if args.precision != "both":
        for r in results.values():
            r["fv"].close()
        if rank == 0:
            r = next(iter(results.values()))
            print(json.dumps({"profiling_run": args.precision, "ms_per_step": r["ms"] / args.steps,
                              "phases_ms_per_step": {k: v[0] / args.steps for k, v in r["phases"].items()}}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    # End to end through the public API with host buffers: each step copies Q in from pinned host memory, steps, and
    # copies Q back out.
    fv = results["fp64"]["fv"]
    host_q = torch.from_numpy(q0.copy()).pin_memory()
    host_out = torch.empty_like(host_q).pin_memory()
    e2e_steps = max(3, args.steps // 2)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        hydro.check(hydro.lib().luna_fv_set_state(fv.handle, host_q.data_ptr(), 0))
        fv.step(fv.time_step(0.3))
        hydro.check(hydro.lib().luna_fv_get_state(fv.handle, host_out.data_ptr(), 0))
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist)
    barrier()

    if rank == 0:
        ab = algorithmic_bytes(F / N)
        peak, peak_kind = measured_peaks()
        r64 = results["fp64"]
        phases = r64["phases"]
        fused, crossing = r64["fused"]
        tpc = traffic_per_cell()
        if fused:
            # the fused pass: the crossing faces' kernel (phase "fluxes") and the tiles' kernel (phase "update") together
            # do phase F; against the sweep, the one kernel pair per step
            pair_ms = phases["fluxes"][0] + phases["update"][0]
            dominant = "flux_and_update" if pair_ms > phases["sweep"][0] else "sweep"
            dom_ms, dom_launches = (pair_ms, phases["update"][1]) if dominant != "sweep" else phases["sweep"]
            traffic = tpc.get(("fp64", "fused")) if dominant != "sweep" else tpc.get(("fp64", "sweep"))
        else:
            dominant = max(("sweep", "fluxes", "update", "primitives"), key=lambda k: phases[k][0])
            dom_ms, dom_launches = phases[dominant]
            traffic = tpc.get(("fp64", dominant))
        avg_s = dom_ms / max(dom_launches, 1) / 1e3
        achieved = ab[dominant] * N / avg_s / 1e9
        step_s = r64["ms"] / args.steps / 1e3
        launches = sum(v[1] for v in phases.values())
        value = world * N * args.steps / (r64["ms"] / 1e3)
        fp32_value = world * N * args.steps / (results["single"]["ms"] / 1e3)
        r32_value = world * N * args.steps / (results["fp32"]["ms"] / 1e3)
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": r64["ms"] / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": {
                "workload": workload_name(args.nx),
                "n_cells": N, "n_faces": F, "faces_per_cell": F / N, "parallelism": f"replicas x{world}",
                "l2": "inputs larger than L2 (working set ~3 GB > 126 MB), no flush",
            },
            "face_fluxes_per_s": world * F * args.steps / (r64["ms"] / 1e3),
            "fp32": {"policy": "single: the reference's Precision<double, float, float, float> (gradients, limiter, face "
                               "states and the Riemann solve in float, flux rows stored in float, geometry, primitives and "
                               "the per-cell sums in double)",
                     "value": fp32_value, "ms_per_step": results["single"]["ms"] / args.steps,
                     "speedup_vs_fp64": fp32_value / value,
                     "phases_ms_per_step": {k: v[0] / args.steps for k, v in results["single"]["phases"].items()}},
            "riemann32": {"policy": "riemann32: Precision<double, float, double, float> (as single, flux rows in double)",
                          "value": r32_value, "ms_per_step": results["fp32"]["ms"] / args.steps,
                          "speedup_vs_fp64": r32_value / value,
                          "phases_ms_per_step": {k: v[0] / args.steps for k, v in results["fp32"]["phases"].items()}},
            "grad16": {"policy": "the reference's 3D default (Grad16: binary16 gradient rows, float limiter, double Riemann)",
                       "value": world * N * args.steps / (results["grad16"]["ms"] / 1e3),
                       "ms_per_step": results["grad16"]["ms"] / args.steps,
                       "speedup_vs_fp64": r64["ms"] / results["grad16"]["ms"],
                       "phases_ms_per_step": {k: v[0] / args.steps for k, v in results["grad16"]["phases"].items()}},
            "phases_ms_per_step": {k: v[0] / args.steps for k, v in phases.items()},
            "flux_pass": {"fused": fused, "crossing_faces": crossing, "crossing_fraction": crossing / F if fused else None},
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)",
                         "algorithmic_bytes_per_cell": ab[dominant],
                         "traffic": None if traffic is None else traffic * N},
            "step_roofline": {"algorithmic_bytes_per_cell": ab["step"],
                              "achieved": ab["step"] * N / step_s / 1e9, "peak": peak, "unit": "GB/s",
                              "frac": ab["step"] * N / step_s / 1e9 / peak},
            "clocks": r64["clocks"],
            "e2e": {"value": world * N * e2e_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(q0.nbytes),
                    "d2h_bytes_per_step": int(q0.nbytes), "steps": e2e_steps},
            "gpu_launches": int(launches),
            "fallbacks_last_step": r64["fallbacks"],
        }
        if world == 1 and not args.no_learned:
            line["learned_limiter"] = learned_section(mesh, q0, args.steps, args.warmup, stream, torch)
        if world == 1 and not args.no_adjoint:
            line["adjoint_cost"] = adjoint_section(mesh, q0, args.steps, args.warmup, stream, torch)
        if world == 1:
            line["fused_flux_update"] = fused_section(mesh, q0, args.steps, args.warmup, stream, torch, r64["ms"] / args.steps,
                                                      r64["fv"].device_bytes())
        if world == 1 and not args.no_moving:
            line["moving"] = moving_section(args.nx, args.moving_steps, 2)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(mesh, q0, args.cpu_sample_steps, args.cpu_warmup, os.cpu_count() or 1)
        print(json.dumps(line), flush=True)
    for r in results.values():
        r["fv"].close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
