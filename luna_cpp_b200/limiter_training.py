"""Training and judging the learned slope limiter with data the method itself generates.

Data (the learned-limiter configuration): seeded 1D Riemann problems (rho_L, rho_R log-uniform in [0.1, 10], p_L, p_R
log-uniform in [0.01, 10], u_L, u_R uniform in [-1, 1], gamma 1.4) on quasi-1D periodic strips of the 2D solver: a
coarse strip of nx x ny jittered cells and a fine one with 4x the cells along each axis. The fine run (plain limiter) is
coarse-grained onto the coarse cells by lattice index (4 x 4 fine cells a coarse cell, Q summed: conservative); the
coarse sweep on that state gives the features, the admissible factors alpha and the unlimited gradients g; the target of
each (cell, variable) is the fine solution's own sub-cell slope s (volume-weighted least squares of the fine cells'
primitives inside the coarse cell) projected on g, as a fraction of alpha: t = clip((s . g) / (g . g) / alpha, 0, 1).
Training runs the library's tensor-core kernels (forward, backward, Adam). The plain limiter judges: errors are L1 of the
density profile against the fine run, on held-out problems, at equal resolution and against plain runs at higher
resolution.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import hydro
from .learned import LimiterMLP
from .mesh import build_mesh, jittered_points
from .problems import cell_centres, conserved

GAMMA = 1.4


@dataclass
class Riemann:
    rho: tuple
    u: tuple
    p: tuple

    def max_speed(self, gamma=GAMMA) -> float:
        return max(abs(u) + math.sqrt(gamma * p / r) for r, u, p in zip(self.rho, self.u, self.p))


def riemann_problem(seed: int) -> Riemann:
    rng = np.random.default_rng(seed)
    rho = tuple(float(10 ** rng.uniform(-1, 1)) for _ in range(2))
    p = tuple(float(10 ** rng.uniform(-2, 1)) for _ in range(2))
    u = tuple(float(rng.uniform(-1, 1)) for _ in range(2))
    return Riemann(rho, u, p)


def strip(nx: int, ny: int, seed: int = 1):
    """A periodic strip of nx x ny jittered (0.1) cells in the box [0, 1) x [0, ny / nx)."""
    box = (1.0, ny / nx)
    return build_mesh(jittered_points((nx, ny), side=box, jitter=0.1, seed=seed), box=box)


def riemann_state(mesh, prob: Riemann, gamma=GAMMA) -> np.ndarray:
    """The 1D problem across a strip: the left state in [0.25, 0.75), the right one elsewhere."""
    x = cell_centres(mesh)[:, 0]
    left = (x >= 0.25) & (x < 0.75)
    W = np.zeros((mesh.n_cells, 4))
    for a, side in ((0, left), (1, ~left)):
        W[side, 0] = prob.rho[a]
        W[side, 1] = prob.u[a]
        W[side, 3] = prob.p[a]
    return conserved(W, gamma) * mesh.volume[:, None]


def primitives(q, mesh, gamma=GAMMA):
    U = q / mesh.volume[:, None]
    rho = U[:, 0]
    d = U.shape[1] - 2
    v = U[:, 1 : 1 + d] / rho[:, None]
    P = (gamma - 1) * (U[:, 1 + d] - 0.5 * rho * np.sum(v * v, 1))
    return np.column_stack([rho, v, P])


def run_to(fv, t_end: float, courant=0.3, max_steps=200000) -> int:
    """Steps fv to t_end exactly (the last step shortened); returns the steps taken."""
    t, steps = 0.0, 0
    while t < t_end * (1 - 1e-12) and steps < max_steps:
        dt = min(fv.time_step(courant), t_end - t)
        fv.step(dt)
        t += dt
        steps += 1
    return steps


def group_index(nx_f, ny_f, factor):
    """Coarse cell of each fine cell of the strip lattices (jittered_points orders i, then j)."""
    i = np.arange(nx_f * ny_f) // ny_f
    j = np.arange(nx_f * ny_f) % ny_f
    ny_c = ny_f // factor
    return (i // factor) * ny_c + j // factor


def _group_sum(groups, values, n):
    """Per-group sums of the rows of values ([m] or [m, ...]) into n groups (column by column, bincount)."""
    v = np.asarray(values, dtype=np.float64)
    if v.ndim == 1:
        return np.bincount(groups, weights=v, minlength=n)
    flat = v.reshape(v.shape[0], -1)
    out = np.stack([np.bincount(groups, weights=flat[:, c], minlength=n) for c in range(flat.shape[1])], 1)
    return out.reshape((n,) + v.shape[1:])


def coarse_grain(q_fine, groups, n_coarse, coarse_mesh, fine_mesh):
    """Fine Q summed per coarse cell, rescaled to the coarse cell's volume (densities kept, totals conserved up to the
    two meshes' volume difference)."""
    q = _group_sum(groups, q_fine, n_coarse)
    vol = _group_sum(groups, fine_mesh.volume, n_coarse)
    return q * (coarse_mesh.volume / vol)[:, None]


def subcell_slopes(fine_mesh, W_fine, groups, coarse_mesh):
    """Per coarse cell and variable, the volume-weighted least-squares slope of the fine primitives about the coarse
    cell's centroid (nearest periodic image)."""
    box = np.asarray(coarse_mesh.box)
    cc = cell_centres(coarse_mesh)
    cf = cell_centres(fine_mesh)
    d = cf - cc[groups]
    d -= box * np.round(d / box)
    V = fine_mesh.volume
    n = coarse_mesh.n_cells
    sv = _group_sum(groups, V, n)
    dm = _group_sum(groups, V[:, None] * d, n) / sv[:, None]
    wm = _group_sum(groups, V[:, None] * W_fine, n) / sv[:, None]
    dd = d - dm[groups]
    dw = W_fine - wm[groups]
    C = _group_sum(groups, V[:, None, None] * dd[:, :, None] * dd[:, None, :], n)
    B = _group_sum(groups, V[:, None, None] * dd[:, :, None] * dw[:, None, :], n)
    return np.linalg.solve(C, B).transpose(0, 2, 1)  # [n][var][dim]


def slots(dim):
    """The network's output slot of each variable (by role: density 0, velocity 1 .. D, pressure 4), as the library's
    learned_slot."""
    return list(range(dim + 1)) + [4]


def targets(alpha, g, s):
    """t = clip((s . g) / (g . g) / alpha, 0, 1) and weights (1 where alpha > 0 and g != 0), in the variables' slots."""
    g = g.reshape(s.shape)
    gg = np.sum(g * g, 2)
    proj = np.sum(s * g, 2) / np.where(gg > 0, gg, 1.0)
    a = alpha[:, : s.shape[1]]
    ok = (a > 1e-12) & (gg > 1e-300)
    t = np.where(ok, np.clip(proj / np.where(ok, a, 1.0), 0.0, 1.0), 0.0)
    w = ok.astype(np.float32)
    T = np.zeros((s.shape[0], 5), np.float32)
    Wt = np.zeros((s.shape[0], 5), np.float32)
    where = slots(s.shape[2])
    T[:, where] = t
    Wt[:, where] = w
    return T, Wt


@dataclass
class Quadrants:
    """A 2D Riemann problem: four constant states (rho, u, v, P) in the quadrants of the periodic unit box."""
    states: tuple

    def max_speed(self, gamma=GAMMA) -> float:
        return max(math.hypot(u, v) + math.sqrt(gamma * p / r) for r, u, v, p in self.states)


def quadrant_problem(seed: int) -> Quadrants:
    """Four states from the 1D problems' distribution: rho log-uniform in [0.1, 10], P log-uniform in [0.01, 10], each
    velocity component uniform in [-1, 1]."""
    rng = np.random.default_rng(seed)
    return Quadrants(tuple((float(10 ** rng.uniform(-1, 1)), float(rng.uniform(-1, 1)), float(rng.uniform(-1, 1)),
                            float(10 ** rng.uniform(-2, 1))) for _ in range(4)))


def square(n: int, seed: int = 1):
    """A periodic unit square of n x n jittered (0.1) cells."""
    return build_mesh(jittered_points((n, n), jitter=0.1, seed=seed), box=(1.0, 1.0))


def quadrant_state(mesh, prob: Quadrants, gamma=GAMMA) -> np.ndarray:
    c = cell_centres(mesh)
    k = (c[:, 0] >= 0.5).astype(int) + 2 * (c[:, 1] >= 0.5).astype(int)
    W = np.array(prob.states)[k]
    return conserved(W, gamma) * mesh.volume[:, None]


def _dataset(coarse, fine, groups, problems, make_state, gamma, snapshots, travel, log, what):
    """Features, targets and weights of the coarse mesh at `snapshots` of each problem's fine run (plain limiter),
    coarse-grained onto the coarse cells."""
    feats, tars, wts = [], [], []
    t0 = time.time()
    for prob in problems:
        t_end = travel / prob.max_speed(gamma)
        ffv = hydro.FiniteVolume(fine, gas=hydro.Gas(gamma))
        ffv.set_state(make_state(fine, prob, gamma))
        cfv = hydro.FiniteVolume(coarse, gas=hydro.Gas(gamma))
        t_prev = 0.0
        for frac in snapshots:
            run_to(ffv, t_end * frac - t_prev)
            t_prev = t_end * frac
            qf = ffv.get_state()
            qc = coarse_grain(qf, groups, coarse.n_cells, coarse, fine)
            cfv.set_state(qc)
            f, alpha, g = cfv.limiter_inputs()
            s = subcell_slopes(fine, primitives(qf, fine, gamma), groups, coarse)
            T, Wt = targets(alpha.cpu().numpy(), g.cpu().numpy(), s)
            feats.append(f)
            tars.append(torch.tensor(T, device="cuda"))
            wts.append(torch.tensor(Wt, device="cuda"))
        ffv.close()
        cfv.close()
    log(f"dataset ({what}): {len(problems)} problems x {len(snapshots)} snapshots, {sum(x.shape[0] for x in feats)} cells, "
        f"{time.time() - t0:.1f} s")
    return torch.cat(feats), torch.cat(tars), torch.cat(wts)


def build_dataset_2d(problems, n=256, factor=4, gamma=GAMMA, snapshots=(0.25, 0.5, 0.75, 1.0), travel=0.2, log=print):
    """The 2D part of the training data: four-quadrant Riemann problems (seeds) on an n^2 jittered mesh, labelled from
    the method's own run on (factor n)^2 cells, coarse-grained by lattice index (factor^2 fine cells a coarse cell)."""
    coarse, fine = square(n, seed=11), square(factor * n, seed=12)
    groups = group_index(factor * n, factor * n, factor)
    return _dataset(coarse, fine, groups, [quadrant_problem(s) for s in problems], quadrant_state, gamma, snapshots, travel,
                    log, f"2D {n}^2 quadrants, gamma {gamma:g}")


# Directions of the oblique 3D problems: integer normals, so that n . x mod 1 is periodic in the unit cube.
DIRECTIONS = ((1, 1, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, -1, 1), (2, 1, 0), (1, 2, 1), (1, 0, 0))


@dataclass
class Oblique:
    """A 1D Riemann problem across planes of integer normal n in the periodic unit cube: the left state where
    frac(n . x) lies in [0.25, 0.75), the right one elsewhere; the velocity along n."""
    riemann: Riemann
    normal: tuple

    def max_speed(self, gamma=GAMMA) -> float:
        return self.riemann.max_speed(gamma)


def oblique_problem(seed: int) -> Oblique:
    return Oblique(riemann_problem(seed), DIRECTIONS[seed % len(DIRECTIONS)])


def cube(n: int, seed: int = 1):
    """A periodic unit cube of n^3 jittered (0.1) cells."""
    return build_mesh(jittered_points((n, n, n), jitter=0.1, seed=seed), box=(1.0, 1.0, 1.0))


def oblique_state(mesh, prob: Oblique, gamma=GAMMA) -> np.ndarray:
    n = np.asarray(prob.normal, dtype=np.float64)
    s = cell_centres(mesh) @ n
    left = (s - np.floor(s) >= 0.25) & (s - np.floor(s) < 0.75)
    unit = n / np.linalg.norm(n)
    W = np.zeros((mesh.n_cells, 5))
    r = prob.riemann
    for a, side in ((0, left), (1, ~left)):
        W[side, 0] = r.rho[a]
        W[side, 1:4] = r.u[a] * unit
        W[side, 4] = r.p[a]
    return conserved(W, gamma) * mesh.volume[:, None]


def group_index_3d(n_f, factor):
    """Coarse cell of each fine cell of two cubic lattices (jittered_points orders i, j, then k)."""
    idx = np.arange(n_f ** 3)
    i, j, k = idx // (n_f * n_f), (idx // n_f) % n_f, idx % n_f
    n_c = n_f // factor
    return ((i // factor) * n_c + j // factor) * n_c + k // factor


def build_dataset_3d(problems, n=32, factor=4, gamma=GAMMA, snapshots=(0.25, 0.5, 0.75, 1.0), travel=0.2, log=print):
    """3D rows from the 1D problems: each seeded Riemann problem across oblique planes (DIRECTIONS) of an n^3 jittered
    cube, labelled from the method's own run on (factor n)^3 cells, coarse-grained by lattice index. These give the
    network rows in which all three velocity slots are active, as on a 3D mesh."""
    coarse, fine = cube(n, seed=11), cube(factor * n, seed=12)
    groups = group_index_3d(factor * n, factor)
    return _dataset(coarse, fine, groups, [oblique_problem(s) for s in problems], oblique_state, gamma, snapshots, travel,
                    log, f"3D oblique {n}^3, gamma {gamma:g}")


@dataclass
class Blast:
    """A point blast in the periodic unit cube: energy E deposited evenly (by volume) as thermal energy in the cells whose
    centroid lies within r0 of the centre c, in a uniform gas of density rho and pressure p; run to t_end, when a Sedov
    blast wave has reached a radius of about 0.3 (R = 1.15 (E t^2 / rho)^(1/5))."""
    energy: float
    rho: float
    p: float
    r0: float
    centre: tuple

    @property
    def t_end(self) -> float:
        return 0.035 * math.sqrt(self.rho / self.energy)

    def max_speed(self, gamma=GAMMA) -> float:  # as _dataset reads it: travel 0.2 over t_end
        return 0.2 / self.t_end


def blast_problem(seed: int, cell: float = 1.0 / 32) -> Blast:
    """Energy log-uniform in [0.3, 3], density in [0.3, 3], pressure in [1e-6, 1e-3]; the deposit radius 1.5 to 3 coarse
    cells; the centre uniform in [0.4, 0.6]^3."""
    rng = np.random.default_rng(seed)
    return Blast(float(10 ** rng.uniform(np.log10(0.3), np.log10(3))), float(10 ** rng.uniform(np.log10(0.3), np.log10(3))),
                 float(10 ** rng.uniform(-6, -3)), float(rng.uniform(1.5, 3.0) * cell), tuple(float(x) for x in rng.uniform(0.4, 0.6, 3)))


def blast_state(mesh, prob: Blast, gamma=GAMMA) -> np.ndarray:
    d = cell_centres(mesh) - np.asarray(prob.centre)
    d -= np.round(d)
    inside = np.sqrt(np.sum(d * d, 1)) < prob.r0
    W = np.zeros((mesh.n_cells, 5))
    W[:, 0] = prob.rho
    W[:, 4] = prob.p
    Q = conserved(W, gamma) * mesh.volume[:, None]
    Q[inside, 4] += prob.energy * mesh.volume[inside] / mesh.volume[inside].sum()
    return Q


def build_dataset_blast(problems, n=32, factor=4, gamma=5.0 / 3.0, snapshots=(0.2, 0.5, 1.0), log=print):
    """3D rows from point blasts of random energy, density, pressure, deposit radius and centre (seeds) on an n^3 jittered
    cube, labelled from the method's own run on (factor n)^3 cells (the deposit the same physical sphere)."""
    coarse, fine = cube(n, seed=11), cube(factor * n, seed=12)
    groups = group_index_3d(factor * n, factor)
    return _dataset(coarse, fine, groups, [blast_problem(s, 1.0 / n) for s in problems], blast_state, gamma, snapshots, 0.2, log,
                    f"3D point blasts {n}^3, gamma {gamma:g}")


def build_dataset(problems, nx=1024, ny=4, factor=4, gamma=GAMMA, snapshots=(0.25, 0.5, 0.75, 1.0), travel=0.2, log=print):
    """The 1D part of the training data: 1D Riemann problems (seeds) across quasi-1D strips of nx x ny cells, labelled
    from the method's own run on a strip of factor x the cells along each axis."""
    coarse, fine = strip(nx, ny, seed=11), strip(factor * nx, factor * ny, seed=12)
    groups = group_index(factor * nx, factor * ny, factor)
    return _dataset(coarse, fine, groups, [riemann_problem(s) for s in problems], riemann_state, gamma, snapshots, travel,
                    log, f"1D strips {nx}x{ny}, gamma {gamma:g}")


def train(features, target, weight, epochs=20, batch=16384, lr=2e-3, seed=0, log=print) -> LimiterMLP:
    net = LimiterMLP(seed=seed)
    n = features.shape[0]
    g = torch.Generator(device="cpu").manual_seed(seed)
    steps = 0
    for epoch in range(epochs):
        perm = torch.randperm(n, generator=g).to(features.device)
        total, count = 0.0, 0
        for b0 in range(0, n, batch):
            idx = perm[b0 : b0 + batch]
            x, t, w = features[idx].contiguous(), target[idx].contiguous(), weight[idx].contiguous()
            if float(w.sum()) == 0:
                continue
            loss = net.gradient(x, t, w)
            steps += 1
            net.adam(lr=lr * (0.5 ** (epoch / max(epochs / 3, 1))))
            total += float(loss.item())
            count += 1
        log(f"epoch {epoch}: mean batch loss {total / max(count, 1):.5f}")
    return net


def density_profile(mesh, q, bins: int):
    """Volume-weighted mean density in `bins` equal bins of x."""
    x = cell_centres(mesh)[:, 0]
    b = np.minimum((x * bins).astype(int), bins - 1)
    m = np.zeros(bins)
    v = np.zeros(bins)
    np.add.at(m, b, q[:, 0])
    np.add.at(v, b, mesh.volume)
    return m / v


def evaluate(net, problems, nx=1024, ny=4, factor=4, travel=0.2, resolutions=(1.0, 1.5, 2.0), log=print):
    """L1 of the density profile (nx bins) against the 4x fine run, per problem: plain at each resolution and learned at
    the base one; and the device time of each run (sum of the library's per-phase timings)."""
    fine = strip(factor * nx, factor * ny, seed=12)
    meshes = {r: strip(int(round(r * nx)), int(round(r * ny)), seed=11) for r in resolutions}
    rows = []
    for seed in problems:
        prob = riemann_problem(seed)
        t_end = travel / prob.max_speed()
        ffv = hydro.FiniteVolume(fine, gas=hydro.Gas(GAMMA))
        ffv.set_state(riemann_state(fine, prob))
        run_to(ffv, t_end)
        ref = density_profile(fine, ffv.get_state(), nx)
        ffv.close()
        row = {"seed": seed}
        for r, mesh in meshes.items():
            for mode in (("plain", "learned") if r == 1.0 else ("plain",)):
                fv = hydro.FiniteVolume(mesh, gas=hydro.Gas(GAMMA))
                if mode == "learned":
                    fv.set_limiter("learned", net.params)
                fv.set_state(riemann_state(mesh, prob))
                fv.set_timing(True)
                steps = run_to(fv, t_end)
                ms = sum(v[0] for v in fv.timings().values())
                err = float(np.mean(np.abs(density_profile(mesh, fv.get_state(), nx) - ref)))
                row[f"{mode}@{r}"] = {"l1": err, "steps": steps, "device_ms": ms}
                fv.close()
        rows.append(row)
        log(f"problem {seed}: " + ", ".join(f"{k} {v['l1']:.3e}" for k, v in row.items() if k != "seed"))
    return rows


def binned_density(mesh, q, bins: int):
    """Volume-weighted mean density in bins x bins equal squares of the unit box."""
    c = cell_centres(mesh)
    b = np.minimum((c[:, 0] * bins).astype(int), bins - 1) * bins + np.minimum((c[:, 1] * bins).astype(int), bins - 1)
    m = np.bincount(b, weights=q[:, 0], minlength=bins * bins)
    v = np.bincount(b, weights=mesh.volume, minlength=bins * bins)
    return m / np.where(v > 0, v, 1.0)


def evaluate_2d(net, problems, n=256, factor=4, gamma=GAMMA, travel=0.2, resolutions=(1.0, 1.25, 1.5), log=print):
    """The 2D held-out set: each four-quadrant problem run by plain and learned at n^2 and by plain at the finer
    resolutions, judged by the L1 of the density binned on the n x n lattice against the method's own (factor n)^2 run;
    with the device time of each run."""
    fine = square(factor * n, seed=12)
    meshes = {r: square(int(round(r * n)), seed=11) for r in resolutions}
    rows = []
    for seed in problems:
        prob = quadrant_problem(seed)
        t_end = travel / prob.max_speed(gamma)
        ffv = hydro.FiniteVolume(fine, gas=hydro.Gas(gamma))
        ffv.set_state(quadrant_state(fine, prob, gamma))
        run_to(ffv, t_end)
        ref = binned_density(fine, ffv.get_state(), n)
        ffv.close()
        row = {"seed": seed}
        for r, mesh in meshes.items():
            for mode in (("plain", "learned") if r == 1.0 else ("plain",)):
                fv = hydro.FiniteVolume(mesh, gas=hydro.Gas(gamma))
                if mode == "learned":
                    fv.set_limiter("learned", net.params)
                fv.set_state(quadrant_state(mesh, prob, gamma))
                fv.set_timing(True)
                steps = run_to(fv, t_end)
                ms = sum(v[0] for v in fv.timings().values())
                err = float(np.mean(np.abs(binned_density(mesh, fv.get_state(), n) - ref)))
                row[f"{mode}@{r}"] = {"l1": err, "steps": steps, "device_ms": ms}
                fv.close()
        rows.append(row)
        log(f"2D problem {seed}: " + ", ".join(f"{k} {v['l1']:.3e}" for k, v in row.items() if k != "seed"))
    return rows


def summarize(rows, resolutions=(1.0, 1.5, 2.0)):
    """Geometric-mean L1 per configuration, and the plain resolution whose error the learned limiter reaches (log-log
    interpolation of plain's error against resolution) with the device time each needs."""
    keys = [k for k in rows[0] if k != "seed"]
    gm = {k: float(np.exp(np.mean([np.log(r[k]["l1"]) for r in rows]))) for k in keys}
    ms = {k: float(np.mean([r[k]["device_ms"] for r in rows])) for k in keys}
    res = np.array(sorted(resolutions))
    err = np.array([gm[f"plain@{r}"] for r in res])
    target = gm["learned@1.0"]
    # plain's error falls with resolution; where does it cross the learned error?
    equal = None
    if target < err[0]:
        for a in range(len(res) - 1):
            if err[a + 1] <= target <= err[a]:
                u = (np.log(target) - np.log(err[a])) / (np.log(err[a + 1]) - np.log(err[a]))
                equal = float(np.exp(np.log(res[a]) + u * (np.log(res[a + 1]) - np.log(res[a]))))
        if equal is None:
            slope = (np.log(err[-1]) - np.log(err[0])) / (np.log(res[-1]) - np.log(res[0]))
            equal = float(np.exp((np.log(target) - np.log(err[0])) / slope)) if slope < 0 else None
    return {"geomean_l1": gm, "mean_device_ms": ms, "plain_resolution_of_equal_error": equal}


def main():
    import argparse
    import json
    import os

    ap = argparse.ArgumentParser(description="train and judge the learned slope limiter")
    ap.add_argument("--train-problems", type=int, default=48, help="1D Riemann problems (strips)")
    ap.add_argument("--train-problems-2d", type=int, default=16, help="2D four-quadrant problems (n2d^2 meshes)")
    ap.add_argument("--test-problems", type=int, default=8)
    ap.add_argument("--test-problems-2d", type=int, default=4)
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--ny", type=int, default=4)
    ap.add_argument("--n2d", type=int, default=256)
    ap.add_argument("--gammas", default="1.4,1.6666666666666667", help="the data's adiabatic indices")
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--train-problems-3d", type=int, default=12, help="1D problems across oblique planes of n3d^3 cubes")
    ap.add_argument("--n3d", type=int, default=24)
    ap.add_argument("--train-blasts", type=int, default=0, help="3D point blasts of random parameters (gamma 5/3, n3d^3)")
    ap.add_argument("--moving-nx", type=int, default=0, help="also judge on the 3D moving blast at this size (0: no)")
    ap.add_argument("--out", default="limiter_out/limiter")
    args = ap.parse_args()
    os.makedirs(os.path.dirname(args.out) or ".", exist_ok=True)
    lines = []

    def log(s):
        print(s, flush=True)
        lines.append(s)

    t0 = time.time()
    parts = []
    for k, gamma in enumerate(float(g) for g in args.gammas.split(",")):
        parts.append(build_dataset(range(1000 + 100 * k, 1000 + 100 * k + args.train_problems), nx=args.nx, ny=args.ny, gamma=gamma,
                                   log=log))
        if args.train_problems_2d > 0:
            parts.append(build_dataset_2d(range(2000 + 100 * k, 2000 + 100 * k + args.train_problems_2d), n=args.n2d, gamma=gamma,
                                          log=log))
        if args.train_problems_3d > 0:
            parts.append(build_dataset_3d(range(3000 + 100 * k, 3000 + 100 * k + args.train_problems_3d), n=args.n3d, gamma=gamma,
                                          snapshots=(0.5, 1.0), log=log))
    if args.train_blasts > 0:
        parts.append(build_dataset_blast(range(4000, 4000 + args.train_blasts), n=args.n3d, log=log))
    x, t, w = (torch.cat([p[c] for p in parts]) for c in range(3))
    net = train(x, t, w, epochs=args.epochs, log=log)
    np.save(args.out + "_params.npy", net.state())
    report = {"train_problems": args.train_problems, "train_problems_2d": args.train_problems_2d,
              "train_problems_3d": args.train_problems_3d, "n3d": args.n3d, "train_blasts": args.train_blasts, "gammas": args.gammas,
              "epochs": args.epochs, "nx": args.nx, "ny": args.ny, "n2d": args.n2d, "rows": len(x)}
    rows = evaluate(net, range(5000, 5000 + args.test_problems), nx=args.nx, ny=args.ny, log=log)
    report["strips"] = {"summary": summarize(rows), "rows": rows}
    log(json.dumps(report["strips"]["summary"]))
    if args.test_problems_2d > 0:
        rows2 = evaluate_2d(net, range(6000, 6000 + args.test_problems_2d), n=args.n2d, log=log)
        report["quadrants_2d"] = {"summary": summarize(rows2, resolutions=(1.0, 1.25, 1.5)), "rows": rows2}
        log(json.dumps(report["quadrants_2d"]["summary"]))
    if args.moving_nx > 0:
        from .studies import learned_moving

        n = args.moving_nx
        report["moving_blast_3d"] = learned_moving(nx=n, plain_nx=(n, int(n * 1.125), int(n * 1.25), int(n * 1.375)),
                                                   params=net.state(), log=log)
    report["wall_s"] = time.time() - t0
    with open(args.out + "_eval.json", "w") as f:
        json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
