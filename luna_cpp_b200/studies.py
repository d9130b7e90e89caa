"""Measurement drivers for the benchmark configurations beside the headline step (the GPU path only; the oracle
comparisons of the same configurations are GPU tests).

- ``precision``: 3D static Voronoi mesh from nx^3 jittered generators; (a) the point blast, (b) the plane acoustic wave
  (amplitude 1e-6, background rho 1, p 3/5); 100 steps of the FP64 step and of the reduced policies (FP32 face
  arithmetic; FP32 gradients; FP16 gradient rows) on the FP64 run's dt schedule: relative L1 and Linf of every
  conserved field against the FP64 run, the wave's error relative to its perturbation, conservation, and device time
  per step.
- ``moving``: the moving-mesh point blast (generators on the 2^-30 snapping grid, moved with the gas plus the
  roundness velocity, fluxes on the old and the new faces) on nx^3 jittered generators to t_end, FP32 face
  arithmetic with FP64 state by default (``riemann32``): steps taken, the hydro part's device time and cell-updates/s
  (the remesh, voronoi-cpp's job, is timed apart, as the reference's hydro part is), the radial density profile; and
  ``timed_steps`` moving steps at ``timed_nx``^3 for the hydro part's throughput at that size.
- ``learned``: the learned limiter on the static 3D point blast: its density L1 against the method's own run at 4x the
  resolution per axis, beside the plain limiter at the same and at finer resolutions, with device times; the GPU time
  the plain limiter needs for the learned limiter's error, over the learned run's.
- ``lines``: the 1D solver as the learned limiter's data factory: a batch of seeded Riemann problems on lines of nx
  cells, one launch a step; cell-updates/s.
- ``adjoint``: 2D Voronoi mesh from nx^2 jittered generators, the shear layer with a_k ~ N(0, 1) from the seed, 200
  steps; d/da_k of int rho vy^2 dA at the final time by the hand-written adjoint with checkpoints every 20 steps,
  against central differences (h = 1e-6) on the same dt schedule; device time of the forward and of the backward.

    python -m luna_cpp_b200.studies precision --nx 128 --steps 100 --out precision.json
    python -m luna_cpp_b200.studies adjoint --nx 512 --steps 200 --out adjoint.json
    python -m luna_cpp_b200.studies moving --nx 32 --out moving.json
    python -m luna_cpp_b200.studies learned --nx 48 --out learned.json
    python -m luna_cpp_b200.studies lines --nx 4096 --out lines.json
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

from . import hydro
from .mesh import build_mesh, jittered_points
from .remesh import Remesher
from .problems import acoustic_wave, cell_centres, conserved, point_blast

GAMMA = 5.0 / 3.0


def _phases_ms(fv) -> float:
    return float(sum(ms for ms, _ in fv.timings().values()))


def _field_errors(q, ref, base=None) -> dict:
    """Per conserved field: sum |q - ref| / sum |ref| (relative L1), max |q - ref| / max |ref| (relative Linf); with
    ``base``, also relative to the deviation from it (sum |q - ref| / sum |ref - base|)."""
    d = np.abs(q - ref)
    out = {"rel_l1": (d.sum(0) / np.abs(ref).sum(0)).tolist(), "rel_linf": (d.max(0) / np.abs(ref).max(0)).tolist(),
           "max_abs": d.max(0).tolist()}
    if base is not None:
        dev = np.abs(ref - base).sum(0)
        out["rel_l1_of_perturbation"] = [float(a / b) if b > 0 else None for a, b in zip(d.sum(0), dev)]
    return out


def precision(nx=128, steps=100, courant=0.3, seed=1, threads=0, log=print) -> dict:
    t0 = time.time()
    mesh = build_mesh(jittered_points((nx, nx, nx), jitter=0.1, seed=seed), threads=threads)
    log(f"mesh {nx}^3: {mesh.n_cells} cells, {mesh.n_faces} faces, {time.time() - t0:.1f} s")
    wave_background = conserved(np.array([1.0, 0.0, 0.0, 0.0, 0.6]), GAMMA)[None, :] * mesh.volume[:, None]
    out = {"config": {"cells": mesh.n_cells, "faces": mesh.n_faces, "steps": steps, "courant": courant, "jitter": 0.1,
                      "seed": seed, "schedule": "every policy replays the FP64 run's dt schedule"}}
    for name, q0 in (("blast", point_blast(mesh, GAMMA)), ("wave", acoustic_wave(mesh, GAMMA))):
        result = {}
        ref = hydro.FiniteVolume(mesh, precision="fp64")
        ref.set_state(q0)
        ref.set_timing(True)
        dts = []
        for _ in range(steps):
            dt = ref.time_step(courant)
            ref.step(dt)
            dts.append(dt)
        q64 = ref.get_state()
        result["fp64"] = {"device_ms_per_step": _phases_ms(ref) / steps, "fallbacks": int(ref.fallbacks()),
                          "mass_drift": float(abs(q64[:, 0].sum() - q0[:, 0].sum()) / q0[:, 0].sum()),
                          "energy_drift": float(abs(q64[:, 4].sum() - q0[:, 4].sum()) / q0[:, 4].sum()),
                          "t_end": float(sum(dts))}
        ref.close()
        for policy in ("fp32", "single", "grad32", "grad16"):
            fv = hydro.FiniteVolume(mesh, precision=policy)
            fv.set_state(q0)
            fv.set_timing(True)
            for dt in dts:
                fv.time_step(courant)
                fv.step(dt)
            q = fv.get_state()
            r = {"device_ms_per_step": _phases_ms(fv) / steps}
            r.update(_field_errors(q, q64, wave_background if name == "wave" else None))
            r["mass_drift"] = float(abs(q[:, 0].sum() - q0[:, 0].sum()) / q0[:, 0].sum())
            r["energy_drift"] = float(abs(q[:, 4].sum() - q0[:, 4].sum()) / q0[:, 4].sum())
            fv.close()
            r["speedup_vs_fp64"] = result["fp64"]["device_ms_per_step"] / r["device_ms_per_step"]
            result[policy] = r
            log(f"{name} {policy}: {r['device_ms_per_step']:.3f} ms/step ({r['speedup_vs_fp64']:.2f}x), "
                f"max rel L1 {max(r['rel_l1']):.2e}")
        out[name] = result
    return out


def radial_profile(mesh, q, bins=32) -> np.ndarray:
    """Volume-weighted mean density in ``bins`` equal shells of radius from the box centre, out to half the box."""
    c = cell_centres(mesh) - 0.5 * np.asarray(mesh.box)
    r = np.sqrt((c * c).sum(1)) / (0.5 * min(mesh.box))
    b = np.minimum((r * bins).astype(int), bins)
    mass = np.bincount(b, weights=q[:, 0], minlength=bins + 1)[:bins]
    vol = np.bincount(b, weights=mesh.volume, minlength=bins + 1)[:bins]
    return np.where(vol > 0, mass / np.where(vol > 0, vol, 1.0), 0.0)


def snapped_jittered_mesh(nx, dim=3, seed=1, threads=0):
    """A jittered mesh whose generators sit on the moving step's 2^-30 snapping grid."""
    step = 2.0 ** -30
    pts = np.round(jittered_points((nx,) * dim, jitter=0.1, seed=seed) / step) * step
    return build_mesh(pts, threads=threads)


def run_moving(fv, t_end, courant=0.3, threads=0, max_steps=100000, remesher=None, log=print) -> dict:
    """Moving steps to t_end (the last step shortened). With ``remesher`` (luna_cpp_b200.remesh.Remesher) the
    generators and the mesh stay on the device; otherwise the host builder remeshes. Returns the steps, t, the hydro
    kernels' device ms, and the wall seconds of the remesh, of taking the new mesh (tiles and geometry rows) and of the
    whole steps."""
    t, steps, remesh_s, load_s = 0.0, 0, 0.0, 0.0
    fv.set_timing(True)
    fv.timings()
    lib = hydro.lib()
    wall0 = time.perf_counter()
    while t < t_end and steps < max_steps:
        dt = min(fv.time_step(courant), t_end - t)
        if remesher is None:
            pos = np.empty((fv.n, fv.dim), dtype=np.float64)
            hydro.check(lib.luna_fv_step_moving_begin(fv.handle, dt, pos.ctypes.data, 0))
            t0 = time.perf_counter()
            mesh = build_mesh(pos, box=fv.mesh.box, threads=threads)
            t1 = time.perf_counter()
            keep: list = []
            hydro.check(lib.luna_fv_step_moving_end(fv.handle, ctypes.byref(hydro.mesh_desc(mesh, keep))))
        else:
            ptr = remesher.points_buffer(fv.n)
            hydro.check(lib.luna_fv_step_moving_begin(fv.handle, dt, ptr, 1))
            t0 = time.perf_counter()
            mesh = remesher.build_device(ptr, fv.n)
            t1 = time.perf_counter()
            hydro.check(lib.luna_fv_step_moving_end(fv.handle, ctypes.byref(mesh.desc)))
        load_s += time.perf_counter() - t1
        remesh_s += t1 - t0
        fv.mesh = mesh
        t += dt
        steps += 1
    hydro_ms = _phases_ms(fv)  # synchronises
    wall = time.perf_counter() - wall0
    return {"steps": steps, "t": t, "hydro_device_ms": hydro_ms, "remesh_s": remesh_s, "mesh_load_s": load_s, "wall_s": wall}


def _moving_run(nx, t_end, precision_policy, courant, threads, remesh, max_steps, log, check_final_mesh=False):
    """The moving point blast on nx^3 snapped jittered generators; the initial mesh built where the remesh runs."""
    step = 2.0 ** -30
    pts = np.round(jittered_points((nx, nx, nx), jitter=0.1, seed=1) / step) * step
    remesher = Remesher(3, (1.0, 1.0, 1.0)) if remesh == "device" else None
    t0 = time.time()
    if remesher is not None:
        mesh = remesher.build(pts)
        cells = mesh.cells()
    else:
        mesh = cells = build_mesh(pts, threads=threads)
    log(f"mesh {nx}^3 ({remesh}): {time.time() - t0:.1f} s")
    q0 = point_blast(cells, GAMMA)
    fv = hydro.FiniteVolume(mesh, precision=precision_policy, motion="moving")
    fv.set_state(q0)
    run = run_moving(fv, t_end, courant, threads, max_steps=max_steps, remesher=remesher, log=log)
    q = fv.get_state()
    final = fv.mesh.cells() if remesher is not None else fv.mesh
    N, n = cells.n_cells, run["steps"]
    same = None
    if remesher is not None and check_final_mesh:  # the last device mesh against the host builder on its generators
        dev = fv.mesh.to_host()
        host = build_mesh(dev.positions, threads=threads)
        same = all(np.ascontiguousarray(getattr(dev, f)).tobytes() == np.ascontiguousarray(getattr(host, f)).tobytes()
                   for f in ("owner", "neighbour", "cell_face_start", "cell_face", "area", "face_centroid", "centroid", "volume"))
    out = {"cells": N, "remesh": remesh, **run, "final_mesh_equals_host_builder": same,
           "hydro_ms_per_step": run["hydro_device_ms"] / n, "remesh_ms_per_step": 1e3 * run["remesh_s"] / n,
           "mesh_load_ms_per_step": 1e3 * run["mesh_load_s"] / n, "step_wall_ms": 1e3 * run["wall_s"] / n,
           "hydro_cell_updates_per_s": N * n / (run["hydro_device_ms"] * 1e-3),
           "cell_updates_per_s": N * n / run["wall_s"],
           "mass_drift": float(abs(q[:, 0].sum() - q0[:, 0].sum()) / q0[:, 0].sum()),
           "energy_drift": float(abs(q[:, 4].sum() - q0[:, 4].sum()) / q0[:, 4].sum()),
           "radial_density_profile": radial_profile(final, q).tolist()}
    log(f"moving {nx}^3 to t = {run['t']:.4f}: {n} steps; a step: hydro {out['hydro_ms_per_step']:.2f} ms (device), remesh "
        f"{out['remesh_ms_per_step']:.1f} ms, mesh load {out['mesh_load_ms_per_step']:.1f} ms, whole {out['step_wall_ms']:.1f} ms; "
        f"final mesh equals the host builder's: {same}")
    fv.close()
    if remesher is not None:
        remesher.close()
    return out


def moving(nx=32, t_end=0.05, precision_policy="fp32", scale_nx=(128, 256), scale_steps=(0, 10), courant=0.3, threads=0,
           remesh="device", log=print) -> dict:
    """The moving-mesh configuration: the point blast on snapped jittered generators, generators moved with the gas plus
    AREPO's roundness velocity, fluxes on the old and the new faces, FP64 state with FP32 face arithmetic
    (riemann32). nx^3 runs to t_end; each of ``scale_nx`` runs to t_end (steps 0) or for that many steps. With remesh
    "device" the generators and the meshes stay on the GPU (luna_cpp_b200.remesh); "host" remeshes with the host
    builder."""
    out = {"config": {"t_end": t_end, "precision": precision_policy, "courant": courant, "remesh": remesh,
                      "problem": "point blast, E = 1 within 2 cell widths, moving mesh"}}
    out["run"] = _moving_run(nx, t_end, precision_policy, courant, threads, remesh, 100000, log, check_final_mesh=True)
    out["scale"] = []
    for big, steps in zip(scale_nx, scale_steps):
        out["scale"].append(_moving_run(big, t_end if steps == 0 else 1.0, precision_policy, courant, threads, remesh,
                                        100000 if steps == 0 else steps, log, check_final_mesh=big <= 128))
    return out


def _run_to(fv, t_end, courant):
    """Static steps to t_end (the last one shortened); returns (steps, device ms)."""
    fv.set_timing(True)
    fv.timings()
    t, steps = 0.0, 0
    while t < t_end:
        dt = min(fv.time_step(courant), t_end - t)
        fv.step(dt)
        t += dt
        steps += 1
    return steps, _phases_ms(fv)


def _radial_reference(mesh, q, bins=1024):
    """The density of a (fine) run as a function of radius from the box centre: mass over volume in thin shells out to
    the box's corner, for linear interpolation at other meshes' cell radii."""
    c = cell_centres(mesh) - 0.5 * np.asarray(mesh.box)
    r = np.sqrt((c * c).sum(1))
    edge = float(np.sqrt((0.25 * np.asarray(mesh.box) ** 2).sum()))
    b = np.minimum((r / edge * bins).astype(int), bins - 1)
    mass = np.bincount(b, weights=q[:, 0], minlength=bins)
    vol = np.bincount(b, weights=mesh.volume, minlength=bins)
    centres = (np.arange(bins) + 0.5) * edge / bins
    keep = vol > 0
    return centres[keep], mass[keep] / vol[keep]


def _profile_l1(mesh, q, reference) -> float:
    """Volume-weighted L1 of the cell densities against the reference profile at the cells' radii."""
    c = cell_centres(mesh) - 0.5 * np.asarray(mesh.box)
    r = np.sqrt((c * c).sum(1))
    rho = q[:, 0] / mesh.volume
    want = np.interp(r, reference[0], reference[1])
    return float((mesh.volume * np.abs(rho - want)).sum() / mesh.volume.sum())


def learned_moving(nx=64, plain_nx=(64, 72, 80, 88), cells_factor=4.0, t_end=0.05, courant=0.3, params=None, log=print) -> dict:
    """The learned limiter on the moving point blast (the learned-limiter configuration's evaluation): nx^3 snapped jittered
    generators, E = 1 within 2 cell widths, gamma 5/3, FP64, generators moved with the gas plus the roundness velocity,
    the mesh rebuilt on the GPU every step, to t_end; the learned limiter (``params``, default the shipped network) at nx
    and the plain one at nx and at the finer ``plain_nx``, each judged by the volume-weighted L1 of its density against
    the radial profile of the plain method's own run on cells_factor x the cells (round(nx cells_factor^(1/3))^3). GPU
    time: the hydro kernels' device time, and the whole steps' time (remesh included; it is GPU work). The plain method's
    error and times are interpolated in log-log at the learned run's error."""
    import torch

    from .learned import LimiterMLP, trained_params
    from .remesh import Remesher

    grid = 2.0 ** -30

    def run(n, mode, net=None):
        pts = np.round(jittered_points((n, n, n), jitter=0.1, seed=1) / grid) * grid
        remesher = Remesher(3, (1.0, 1.0, 1.0))
        mesh = remesher.build(pts)
        cells = mesh.cells()
        fv = hydro.FiniteVolume(mesh, motion="moving")
        if mode == "learned":
            fv.set_limiter("learned", net.params)
        fv.set_state(point_blast(cells, GAMMA))
        torch.cuda.synchronize()
        r = run_moving(fv, t_end, courant, remesher=remesher, log=lambda m: None)
        q = fv.get_state()
        final = fv.mesh.cells()
        fv.close()
        remesher.close()
        return r, final, q

    n_ref = int(round(nx * cells_factor ** (1.0 / 3.0)))
    r, final, q = run(n_ref, "plain")
    reference = _radial_reference(final, q)
    out = {"config": {"problem": "moving point blast, E = 1 within 2 cell widths, gamma 5/3, FP64, device remesh",
                      "t_end": t_end, "courant": courant,
                      "reference": {"nx": n_ref, "cells": n_ref ** 3, "cells_over_base": n_ref ** 3 / nx ** 3, "steps": r["steps"],
                                    "hydro_device_ms": r["hydro_device_ms"], "wall_s": r["wall_s"]}},
           "plain": [], "learned": []}
    log(f"reference {n_ref}^3: {r['steps']} steps, {r['wall_s']:.1f} s")
    net = LimiterMLP(trained_params() if params is None else params)
    for n in sorted(set(plain_nx) | {nx}):
        for mode in ("plain", "learned") if n == nx else ("plain",):
            r, final, q = run(n, mode, net)
            row = {"nx": n, "cells": n ** 3, "steps": r["steps"], "hydro_device_ms": r["hydro_device_ms"],
                   "whole_ms": 1e3 * r["wall_s"], "l1": _profile_l1(final, q, reference)}
            out[mode].append(row)
            log(f"{mode} {n}^3: {row['steps']} steps, hydro {row['hydro_device_ms']:.1f} ms, whole {row['whole_ms']:.0f} ms, "
                f"L1 {row['l1']:.4e}")
    plain = sorted(out["plain"], key=lambda r: r["nx"])
    learned = out["learned"][0]
    out["learned_l1_over_plain_l1"] = learned["l1"] / next(r["l1"] for r in plain if r["nx"] == nx)
    le = np.log([r["l1"] for r in plain])
    for key in ("hydro_device_ms", "whole_ms"):
        if np.all(np.diff(le) < 0) and le[-1] <= np.log(learned["l1"]) <= le[0]:
            x = np.interp(np.log(learned["l1"]), le[::-1], np.log([r["nx"] for r in plain])[::-1])
            t = np.interp(x, np.log([r["nx"] for r in plain]), np.log([r[key] for r in plain]))
            out["plain_nx_of_equal_error"] = float(np.exp(x))
            out[f"gpu_time_ratio_at_equal_error_{key}"] = float(np.exp(t) / learned[key])
        else:
            out["plain_nx_of_equal_error"] = None
            out[f"gpu_time_ratio_at_equal_error_{key}"] = None
    return out


def learned_blast(nx=48, factor=4, plain_nx=(48, 56, 64, 72, 80), t_end=0.05, courant=0.3, threads=0, log=print) -> dict:
    """The learned limiter in 3D: the static point blast (E = 1 within 2 cell widths, FP64) on nx^3 jittered generators
    to t_end with the shipped network, and with the plain limiter at nx and at the finer ``plain_nx``, each judged by the
    volume-weighted L1 of its density against the radial profile of the method's own run at factor x nx per axis; with
    the device time of every run. The plain method's error and time are interpolated in log-log at the learned run's
    error: the GPU time the plain limiter needs for the learned limiter's accuracy, over the learned run's."""
    import torch

    from .learned import LimiterMLP, trained_params

    def mesh_of(n):
        t0 = time.time()
        m = build_mesh(jittered_points((n, n, n), jitter=0.1, seed=1), threads=threads)
        log(f"mesh {n}^3: {m.n_cells} cells, {time.time() - t0:.1f} s")
        return m

    fine = mesh_of(factor * nx)
    fv = hydro.FiniteVolume(fine)
    fv.set_state(point_blast(fine, GAMMA))
    steps, ms = _run_to(fv, t_end, courant)
    reference = _radial_reference(fine, fv.get_state())
    fv.close()
    out = {"config": {"problem": "static point blast, E = 1 within 2 cell widths, gamma 5/3, FP64", "t_end": t_end,
                      "courant": courant, "reference": {"cells": fine.n_cells, "steps": steps, "device_ms": ms}},
           "plain": [], "learned": []}
    del fine
    net = LimiterMLP(trained_params())
    for n in sorted(set(plain_nx) | {nx}):
        mesh = mesh_of(n)
        q0 = point_blast(mesh, GAMMA)
        for mode in ("plain", "learned") if n == nx else ("plain",):
            fv = hydro.FiniteVolume(mesh)
            if mode == "learned":
                fv.set_limiter("learned", net.params)
            fv.set_state(q0)
            steps, ms = _run_to(fv, t_end, courant)
            row = {"nx": n, "cells": mesh.n_cells, "steps": steps, "device_ms": ms, "l1": _profile_l1(mesh, fv.get_state(), reference)}
            fv.close()
            out[mode].append(row)
            log(f"{mode} {n}^3: {steps} steps, {ms:.1f} ms, L1 {row['l1']:.4e}")
    torch.cuda.synchronize()
    plain = sorted(out["plain"], key=lambda r: r["nx"])
    learned = out["learned"][0]
    le = np.log([r["l1"] for r in plain])
    if np.all(np.diff(le) < 0) and le[-1] <= np.log(learned["l1"]) <= le[0]:
        # error falls with resolution: interpolate log nx and log time at the learned error
        x = np.interp(np.log(learned["l1"]), le[::-1], np.log([r["nx"] for r in plain])[::-1])
        t = np.interp(x, np.log([r["nx"] for r in plain]), np.log([r["device_ms"] for r in plain]))
        out["plain_nx_of_equal_error"] = float(np.exp(x))
        out["plain_device_ms_at_equal_error"] = float(np.exp(t))
        out["gpu_time_ratio_at_equal_error"] = float(np.exp(t) / learned["device_ms"])
    else:
        out["plain_nx_of_equal_error"] = None
        out["gpu_time_ratio_at_equal_error"] = None
    out["learned_l1_over_plain_l1"] = learned["l1"] / next(r["l1"] for r in plain if r["nx"] == nx)
    return out


def lines(nx=4096, batch=1024, steps=200, courant=0.8, seed=9000, log=print) -> dict:
    """The 1D solver as the learned limiter's data factory: ``batch`` seeded Riemann problems (the training
    distribution) on lines of nx uniform cells between outflow walls, all in one launch a step: ``steps`` fused steps
    (step_and_time_step, LUNA's rule), device time by CUDA events, cell-updates/s."""
    import torch

    from .limiter_training import riemann_problem
    from .line import Line
    from .problems import line_keys, line_state, line_tube

    x = (np.arange(nx) + 0.5) / nx
    keys, order, step, period = line_keys(x, 1.0)
    q0 = np.stack([line_state(line_tube(*((r.rho[k], r.u[k], r.p[k]) for k in (0, 1)), t_end=1.0), keys, step)
                   for r in (riemann_problem(seed + b) for b in range(batch))])
    ln = Line(x, 1.0, lines=batch)
    ln.set_state(q0)
    dt = ln.time_step(courant, "luna")
    for _ in range(5):
        dt = ln.step_and_time_step(dt, courant)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for _ in range(steps):
        dt = ln.step_and_time_step(dt, courant)
    end.record()
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    q = ln.get_state()
    ln.close()
    out = {"config": {"cells": nx, "lines": batch, "steps": steps, "courant": courant, "rule": "luna", "fused": True},
           "device_ms_per_step": ms / steps, "cell_updates_per_s": nx * batch * steps / (ms * 1e-3),
           "finite": bool(np.all(np.isfinite(q)))}
    log(f"{batch} lines x {nx} cells: {ms / steps:.3f} ms/step, {out['cell_updates_per_s'] / 1e9:.2f} G cell-updates/s")
    return out


def adjoint(nx=512, steps=200, every=20, h=1e-6, seed=3, courant=0.3, threads=0, log=print) -> dict:
    import torch

    from .autograd import kinetic_y, last_dts, rollout, shear_layer_torch

    t0 = time.time()
    mesh = build_mesh(jittered_points((nx, nx), jitter=0.1, seed=1), threads=threads)
    log(f"mesh {nx}^2: {mesh.n_cells} cells, {mesh.n_faces} faces, {time.time() - t0:.1f} s")
    dev = torch.device("cuda")
    centres = torch.tensor(cell_centres(mesh), device=dev)
    volume = torch.tensor(mesh.volume, device=dev)
    coefficients = np.random.default_rng(seed).standard_normal(8)
    a = torch.tensor(coefficients, device=dev, requires_grad=True)
    fv = hydro.FiniteVolume(mesh)

    # the plain forward (no checkpoints), for the cost ratio
    with torch.no_grad():
        fv.set_state(shear_layer_torch(centres, volume, a))
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(steps):
        fv.step(fv.time_step(courant))
    torch.cuda.synchronize()
    plain = time.perf_counter() - t

    t = time.perf_counter()
    out = rollout(shear_layer_torch(centres, volume, a), fv, steps, courant=courant, every=every)
    J = kinetic_y(out)
    torch.cuda.synchronize()
    forward = time.perf_counter() - t
    dts = last_dts(out)
    t = time.perf_counter()
    J.backward()
    torch.cuda.synchronize()
    backward = time.perf_counter() - t
    grad = a.grad.detach().cpu().numpy()

    fd = np.zeros(8)
    t = time.perf_counter()
    with torch.no_grad():
        for k in range(8):
            e = torch.zeros(8, dtype=torch.float64, device=dev)
            e[k] = h
            jp = kinetic_y(rollout(shear_layer_torch(centres, volume, a + e), fv, steps, courant=courant, every=every, dts=dts))
            jm = kinetic_y(rollout(shear_layer_torch(centres, volume, a - e), fv, steps, courant=courant, every=every, dts=dts))
            fd[k] = (jp - jm).item() / (2 * h)
    fd_time = time.perf_counter() - t
    err = np.abs(grad - fd)
    res = {"config": {"cells": mesh.n_cells, "faces": mesh.n_faces, "steps": steps, "checkpoint_every": every, "h": h,
                      "seed": seed, "coefficients": coefficients.tolist(), "t_end": float(sum(dts))},
           "objective": float(J.item()), "gradient_adjoint": grad.tolist(), "gradient_fd": fd.tolist(),
           "max_abs_error_over_max_fd": float(err.max() / np.abs(fd).max()),
           "rel_error_per_coefficient": (err / np.abs(fd)).tolist(),
           "seconds": {"plain_forward": plain, "checkpointed_forward": forward, "backward": backward,
                       "finite_differences_16_rollouts": fd_time},
           "backward_over_plain_forward": backward / plain}
    log(json.dumps(res["seconds"]))
    log(f"adjoint vs central differences: max |error| / max |fd| = {res['max_abs_error_over_max_fd']:.2e}")
    fv.close()
    return res


def kernels(case="adjoint", nx=64, repeat=3, log=print) -> dict:
    """Small profiling workloads of the kernels beside the static step, each run `repeat` times after one warm-up on the
    nx^3 jittered point blast (FP64), for ncu captures of one kernel family at a time:
      adjoint  step_adjoint (k_sweep_fit, k_faces_adjoint, k_cell_adjoint, k_gather_adjoint), Q bar on the device;
      tangent  step_tangent (k_tangent_prims, k_tangent_sweep, k_tangent_fluxes, k_tangent_update);
      mlp      the limiter network on nx^3 feature rows: the tensor-core forward (k_mlp_forward_tc) and a training step's
               gradient (k_mlp_train, k_mlp_reduce);
      line     256 Riemann-problem lines of 4096 cells, fused steps (k_line_step);
      tiles    the sweep's tiles cut on the device and the geometry rows of a device mesh (k_morton, k_tiles, ...,
               k_geometry), by taking a device remesh of the generators as the mesh;
      moving   moving steps with the device remesh (k_geometry of each new mesh, the two flux passes)."""
    import torch

    from . import hydro
    from .learned import LimiterMLP, init_params
    from .problems import point_blast

    out = {"case": case, "nx": nx, "repeat": repeat}
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if case in ("adjoint", "tangent"):
        mesh = build_mesh(jittered_points((nx, nx, nx), jitter=0.1, seed=1))
        fv = hydro.FiniteVolume(mesh)
        fv.set_state(point_blast(mesh))
        for _ in range(2):
            fv.step(fv.time_step(0.3))
        q = fv.get_state()
        dt = fv.time_step(0.3)
        bar = torch.randn(mesh.n_cells, 5, dtype=torch.float64, device="cuda") * 1e-3
        call = (lambda: fv.step_adjoint(dt, bar)) if case == "adjoint" else (lambda: (fv.set_state(q), fv.time_step(0.3), fv.step_tangent(dt, bar)))
        call()
        torch.cuda.synchronize()
        start.record()
        for _ in range(repeat):
            call()
        end.record()
        torch.cuda.synchronize()
        out["ms_per_call"] = start.elapsed_time(end) / repeat
        fv.close()
    elif case == "mlp":
        n = nx ** 3
        net = LimiterMLP(init_params(1))
        x = (torch.rand(n, 32, device="cuda") * 2 - 1).to(torch.bfloat16)
        t = torch.rand(n, 5, device="cuda")
        w = torch.ones(n, 5, device="cuda")
        net.forward(x)
        net.gradient(x, t, w)
        torch.cuda.synchronize()
        start.record()
        for _ in range(repeat):
            net.forward(x)
        end.record()
        torch.cuda.synchronize()
        out["forward_ms"] = start.elapsed_time(end) / repeat
        for _ in range(repeat):
            net.gradient(x, t, w)
        torch.cuda.synchronize()
    elif case == "line":
        out.update(lines(nx=4096, batch=256, steps=repeat, log=log))
    elif case in ("tiles", "moving"):
        from .remesh import Remesher

        grid = 2.0 ** -30
        pts = np.round(jittered_points((nx, nx, nx), jitter=0.1, seed=1) / grid) * grid
        remesher = Remesher(3, (1.0, 1.0, 1.0))
        mesh = remesher.build(pts)
        if case == "tiles":
            for _ in range(repeat + 1):
                fv = hydro.FiniteVolume(mesh)
                fv.close()
        else:
            fv = hydro.FiniteVolume(mesh, precision="single", motion="moving")
            fv.set_state(point_blast(mesh.cells()))
            r = run_moving(fv, 1.0, max_steps=repeat + 1, remesher=remesher, log=lambda s: None)
            out["hydro_device_ms_per_step"] = r["hydro_device_ms"] / r["steps"]
            fv.close()
        remesher.close()
    else:
        raise ValueError(case)
    torch.cuda.synchronize()
    log(json.dumps(out))
    return out


def moving_line(nx=131072, steps=2000, courant=0.4, log=print) -> dict:
    """The moving 1D line on Shu-Osher (the left wall holding the entering state and supplying cells, the reference's
    moving pass table, research_notes/inflow_2026-11-06.md:51-64): `steps` steps from t = 0 at nx cells, timed by CUDA
    events over the whole loop (each step reads its dt or its order check back, as the reference's driver does): time_step
    (AREPO's rule) + step, and step_and_time_step (LUNA's rule, one launch a step). Cell updates: the cells of each step,
    summed."""
    import torch

    from .line import MovingLine
    from .problems import line_problem

    pr = line_problem("shu-osher")
    L, o = pr["L"], pr["origin"]
    x = L * (np.arange(nx) + 0.5) / nx
    out = {"config": {"problem": "shu-osher", "cells": nx, "steps": steps, "walls": "inflow (holding the state), outflow",
                      "courant": courant}}
    for path in ("time_step+step", "step_and_time_step"):
        ml = MovingLine(x, L, walls=pr["moving_walls"], inflow=np.array(pr["moving_inflow"]), gamma=pr["gamma"])
        g, V, c = ml.geometry()
        a, b = g + c - 0.5 * V, g + c + 0.5 * V
        ml.set_state(pr["average"](a + o, b + o) * (b - a)[:, None])
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        updates = 0
        torch.cuda.synchronize()
        start.record()
        if path == "time_step+step":
            for _ in range(steps):
                updates += ml.n
                ml.step(ml.time_step(courant, "arepo"))
        else:
            dt = ml.time_step(courant, "luna")
            for _ in range(steps):
                updates += ml.n
                dt = ml.step_and_time_step(dt, courant)
        end.record()
        torch.cuda.synchronize()
        ms = start.elapsed_time(end)
        out[path] = {"device_ms_per_step": ms / steps, "cell_updates_per_s": updates / (ms * 1e-3), "cells_at_end": ml.n,
                     "cells_added": ml.cells_added(), "sorts": ml.stats()["sorts"],
                     "finite": bool(np.all(np.isfinite(ml.get_state())))}
        log(f"{path}: {ms / steps * 1e3:.1f} us/step, {out[path]['cell_updates_per_s'] / 1e9:.2f} G cell-updates/s, "
            f"{ml.n} cells")
        ml.close()
    return out


def moving_derivatives(nx=1024, repeat=5, log=print) -> dict:
    """The cost of the order-1 moving derivatives in 2D, as the reference's --cost-moving measures it
    (hydro_derivatives_test.cpp:1853-1990): an nx^2 jittered periodic mesh on the 2^-30 grid, the reference's wave state,
    medians of `repeat` calls after a warm-up, each from the same state (the reload not timed), CUDA events. The geometry's
    derivative is a null one on the device (zeros), standing in for the mesh library's, as there. The forward step is
    time_step + step with the device remesh; the tangent and the adjoint run that step inside (the adjoint's restore of
    the t^n mesh and state included); every array on the device."""
    import torch

    lib = hydro.lib()
    step = 2.0 ** -30
    rng = np.random.default_rng(5)
    ij = np.stack(np.meshgrid(np.arange(nx), np.arange(nx), indexing="ij"), -1).reshape(-1, 2)
    pts = np.floor((ij + 0.5 + rng.uniform(-0.15, 0.15, ij.shape)) / nx / step) * step
    start_remesh, remesher = Remesher(dim=2, box=(1.0, 1.0)), Remesher(dim=2, box=(1.0, 1.0))
    start = start_remesh.build(pts)
    cells = start.cells()
    c = cells.positions + cells.centroid
    k, gamma = 2 * np.pi, 5.0 / 3.0
    rho = 1 + 0.2 * np.sin(k * c[:, 0]) + rng.uniform(-0.01, 0.01, len(c))
    vx = 0.3 * np.sin(k * c[:, 1]) + rng.uniform(-0.01, 0.01, len(c))
    vy = 0.2 * np.cos(k * c[:, 0]) + rng.uniform(-0.01, 0.01, len(c))
    P = 1 + 0.2 * np.cos(k * (c[:, 0] + c[:, 1])) + rng.uniform(-0.01, 0.01, len(c))
    q0 = np.stack([rho, rho * vx, rho * vy, P / (gamma - 1) + 0.5 * rho * (vx * vx + vy * vy)], -1) * cells.volume[:, None]
    fv = hydro.FiniteVolume(start, hydro.Gas(gamma), order=1, motion="moving")
    N = nx * nx
    dev = dict(device="cuda", dtype=torch.float64)
    q_start = torch.tensor(q0, **dev)
    faces = 4 * N  # above either mesh's faces (about 3 a cell on a jittered 2D lattice)
    zero_cells, zero_points, zero_faces = torch.zeros(N, **dev), torch.zeros(N, 2, **dev), torch.zeros(faces, 2, **dev)
    bar_cells, bar_points, bar_faces, bar_faces2 = (torch.zeros(N, **dev), torch.zeros(N, 2, **dev), torch.zeros(faces, 2, **dev),
                                                    torch.zeros(faces, 2, **dev))
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

    def load():
        fv.set_mesh(start)
        hydro.check(lib.luna_fv_set_state(fv.handle, ptr(q_start), 1))
        torch.cuda.synchronize()

    def forward(dt):
        fv.time_step(0.3)
        fv.step_moving_device(dt, remesher)

    def tangent(dt, dq, dx):
        fv.time_step(0.3)
        hydro.check(lib.luna_fv_step_moving_tangent(fv.handle, dt, ptr(dq), ptr(dx), ptr(zero_cells), ptr(zero_points),
                                                    ptr(zero_faces), ptr(zero_faces), 1))
        fv.step_moving_device(dt, remesher)
        hydro.check(lib.luna_fv_step_moving_tangent_end(fv.handle, dt, ptr(dq), ptr(dx), ptr(zero_cells), ptr(zero_points),
                                                        ptr(zero_faces), ptr(zero_faces), 1))

    def adjoint(dt, qbar, xbar):
        fv.time_step(0.3)
        hydro.check(lib.luna_fv_step_moving_adjoint_begin(fv.handle, dt))
        fv.step_moving_device(dt, remesher)
        hydro.check(lib.luna_fv_step_moving_adjoint_new_mesh(fv.handle, dt, ptr(qbar), ptr(xbar), ptr(bar_faces2), ptr(bar_faces2), 1))
        fv.set_mesh(start)  # the t^n mesh and state back for the first pass
        hydro.check(lib.luna_fv_set_state(fv.handle, ptr(q_start), 1))
        hydro.check(lib.luna_fv_step_moving_adjoint(fv.handle, dt, ptr(qbar), ptr(xbar), ptr(bar_cells), ptr(bar_points),
                                                    ptr(bar_faces), ptr(bar_faces), 1))

    load()
    dt = fv.time_step(0.3)
    out = {"config": {"cells": N, "order": 1, "dim": 2, "repeat": repeat, "geometry_derivative": "null (zeros on the device)",
                      "remesh": "device"}}
    calls = {"forward": lambda a: forward(dt), "tangent": lambda a: tangent(dt, *a), "adjoint": lambda a: adjoint(dt, *a)}
    inputs = {"forward": lambda: (), "tangent": lambda: (torch.full((N, 4), 1e-6, **dev), torch.zeros(N, 2, **dev)),
              "adjoint": lambda: (torch.ones(N, 4, **dev), torch.ones(N, 2, **dev))}
    for name, call in calls.items():
        times = []
        for r in range(repeat + 1):
            load()
            args = inputs[name]()  # filled before the timed region, as the reference fills dq, dx, qbar, xbar
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            call(args)
            e1.record()
            torch.cuda.synchronize()
            if r > 0:
                times.append(e0.elapsed_time(e1))
        out[name] = {"ms": float(np.median(times)), "cell_steps_per_s": N / (float(np.median(times)) * 1e-3)}
    for name in ("tangent", "adjoint"):
        out[name]["x_forward"] = out[name]["ms"] / out["forward"]["ms"]
    log(f"{nx}^2: forward {out['forward']['ms']:.2f} ms, tangent {out['tangent']['ms']:.2f} ms ({out['tangent']['x_forward']:.1f}x), "
        f"adjoint {out['adjoint']['ms']:.2f} ms ({out['adjoint']['x_forward']:.1f}x)")
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("study", choices=["precision", "adjoint", "moving", "learned", "learned_moving", "lines", "moving_line",
                                      "moving_derivatives", "kernels"])
    ap.add_argument("--case", default="adjoint", help="kernels: adjoint, tangent, mlp, line, tiles or moving")
    ap.add_argument("--nx", type=int)
    ap.add_argument("--steps", type=int)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--remesh", choices=["device", "host"], help="moving: where the mesh is rebuilt (default device)")
    ap.add_argument("--scale-steps", help="moving: steps at 128^3,256^3 (0: to t_end), e.g. 0,10")
    ap.add_argument("--out")
    args = ap.parse_args()
    kw = {"threads": args.threads}
    if args.study == "moving" and args.remesh:
        kw["remesh"] = args.remesh
    if args.study == "moving" and args.scale_steps:
        kw["scale_steps"] = tuple(int(x) for x in args.scale_steps.split(","))
    if args.nx:
        kw["nx"] = args.nx
    if args.steps:
        kw["steps"] = args.steps
    if args.study in ("moving", "learned", "learned_moving"):
        kw.pop("steps", None)
    if args.study == "learned_moving":
        kw.pop("threads", None)
    if args.study in ("lines", "moving_line", "moving_derivatives"):
        kw.pop("threads", None)
    if args.study == "moving_derivatives" and args.steps:
        kw["repeat"] = kw.pop("steps")
    if args.study == "kernels":
        kw.pop("threads", None)
        kw["case"] = args.case
        if args.steps:
            kw["repeat"] = kw.pop("steps")
    res = {"precision": precision, "adjoint": adjoint, "moving": moving, "learned": learned_blast,
           "learned_moving": learned_moving, "lines": lines, "moving_line": moving_line,
           "moving_derivatives": moving_derivatives, "kernels": kernels}[args.study](**kw)
    text = json.dumps(res, indent=1)
    if args.out:
        with open(args.out, "w") as f:
            f.write(text)
    print(text)


if __name__ == "__main__":
    main()
