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
    v = U[:, 1:3] / rho[:, None]
    P = (gamma - 1) * (U[:, 3] - 0.5 * rho * np.sum(v * v, 1))
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


def coarse_grain(q_fine, groups, n_coarse, coarse_mesh, fine_mesh):
    """Fine Q summed per coarse cell, rescaled to the coarse cell's volume (densities kept, totals conserved up to the
    two meshes' volume difference)."""
    q = np.zeros((n_coarse, q_fine.shape[1]))
    vol = np.zeros(n_coarse)
    np.add.at(q, groups, q_fine)
    np.add.at(vol, groups, fine_mesh.volume)
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
    # weighted means
    sv = np.zeros(n)
    np.add.at(sv, groups, V)
    dm = np.zeros((n, 2))
    np.add.at(dm, groups, V[:, None] * d)
    dm /= sv[:, None]
    wm = np.zeros((n, W_fine.shape[1]))
    np.add.at(wm, groups, V[:, None] * W_fine)
    wm /= sv[:, None]
    dd = d - dm[groups]
    dw = W_fine - wm[groups]
    C = np.zeros((n, 2, 2))
    np.add.at(C, groups, V[:, None, None] * dd[:, :, None] * dd[:, None, :])
    B = np.zeros((n, 2, W_fine.shape[1]))
    np.add.at(B, groups, V[:, None, None] * dd[:, :, None] * dw[:, None, :])
    return np.linalg.solve(C, B).transpose(0, 2, 1)  # [n][var][dim]


def targets(alpha, g, s):
    """t = clip((s . g) / (g . g) / alpha, 0, 1) and weights (1 where alpha > 0 and g != 0)."""
    g = g.reshape(s.shape)
    gg = np.sum(g * g, 2)
    proj = np.sum(s * g, 2) / np.where(gg > 0, gg, 1.0)
    a = alpha[:, : s.shape[1]]
    ok = (a > 1e-12) & (gg > 1e-300)
    t = np.where(ok, np.clip(proj / np.where(ok, a, 1.0), 0.0, 1.0), 0.0)
    w = ok.astype(np.float32)
    T = np.zeros((s.shape[0], 5), np.float32)
    Wt = np.zeros((s.shape[0], 5), np.float32)
    T[:, : s.shape[1]] = t
    Wt[:, : s.shape[1]] = w
    return T, Wt


def build_dataset(problems, nx=1024, ny=4, factor=4, snapshots=(0.25, 0.5, 0.75, 1.0), travel=0.2, log=print):
    """Features, targets and weights from the fine runs of `problems` (seeds)."""
    coarse = strip(nx, ny, seed=11)
    fine = strip(factor * nx, factor * ny, seed=12)
    groups = group_index(factor * nx, factor * ny, factor)
    feats, tars, wts = [], [], []
    t0 = time.time()
    for seed in problems:
        prob = riemann_problem(seed)
        t_end = travel / prob.max_speed()
        ffv = hydro.FiniteVolume(fine, gas=hydro.Gas(GAMMA))
        ffv.set_state(riemann_state(fine, prob))
        cfv = hydro.FiniteVolume(coarse, gas=hydro.Gas(GAMMA))
        t_prev = 0.0
        for frac in snapshots:
            run_to(ffv, t_end * frac - t_prev)
            t_prev = t_end * frac
            qf = ffv.get_state()
            qc = coarse_grain(qf, groups, coarse.n_cells, coarse, fine)
            cfv.set_state(qc)
            f, alpha, g = cfv.limiter_inputs()
            s = subcell_slopes(fine, primitives(qf, fine), groups, coarse)
            T, Wt = targets(alpha.cpu().numpy(), g.cpu().numpy(), s)
            feats.append(f)
            tars.append(torch.tensor(T, device="cuda"))
            wts.append(torch.tensor(Wt, device="cuda"))
        ffv.close()
        cfv.close()
    log(f"dataset: {len(problems)} problems x {len(snapshots)} snapshots, {sum(x.shape[0] for x in feats)} cells, "
        f"{time.time() - t0:.1f} s")
    return torch.cat(feats), torch.cat(tars), torch.cat(wts)


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
    ap.add_argument("--train-problems", type=int, default=64)
    ap.add_argument("--test-problems", type=int, default=16)
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--ny", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--out", default="limiter_out")
    args = ap.parse_args()
    os.makedirs(os.path.dirname(args.out) or ".", exist_ok=True)
    lines = []

    def log(s):
        print(s, flush=True)
        lines.append(s)

    t0 = time.time()
    x, t, w = build_dataset(range(1000, 1000 + args.train_problems), nx=args.nx, ny=args.ny, log=log)
    net = train(x, t, w, epochs=args.epochs, log=log)
    np.save(args.out + "_params.npy", net.state())
    rows = evaluate(net, range(5000, 5000 + args.test_problems), nx=args.nx, ny=args.ny, log=log)
    summary = summarize(rows)
    log(json.dumps(summary))
    with open(args.out + "_eval.json", "w") as f:
        json.dump({"summary": summary, "rows": rows, "train_problems": args.train_problems, "epochs": args.epochs,
                   "nx": args.nx, "ny": args.ny, "wall_s": time.time() - t0}, f, indent=1)


if __name__ == "__main__":
    main()
