"""The rollout server of luna-cpp (src/examples/rollout.cpp) on libluna_b200: a fixed-dt rollout of the 2D or 3D step
on the Voronoi mesh of the regular n^D lattice of the periodic unit box, and its reverse-mode derivative, served one
command a line on stdin for Python optimisers (the reference's scripts/examples/rollout_client.py drives it unchanged:
``Rollout("luna_cpp_b200/bin/rollout", dim, n, steps, dt, workdir)``).

    python -m luna_cpp_b200.rollout --dim=2 --n=64 --steps=100 --dt=1e-3 [--gamma=5/3] [--courant=0.3] [--moving] [--order=1]

Commands (paths are raw float64 files, C order; cells in lattice C order, the last axis fastest):
    forward <U0 in> <final out>       U0: N x V intensive; runs the steps keeping the tape (on the device); final: N x
                                      (V + D + 1) rows of (Q extensive, x, volume). Answers "ok <ms> <cfl violations>".
    adjoint <bars in> <U0bar out>     bars: N x (V + D + 1) at the end of the last forward; U0bar = dL/dU0 (intensive).
                                      On the static mesh x and the volumes do not depend on U0: their bars drop out.
    tangent <U0 in> <dU0 in> <dQ out> the forward with the tangent dU0 (intensive) beside it; dQ: N x V (extensive) at
                                      the end. Answers "ok <ms>".
    cfl <U0 in>                       "ok <time_step(courant) at U0>".
    geometry <out>                    N x (D + 1) rows of (x, volume). Answers "ok".
    memory                            "ok <peak device bytes> <bytes now>" (the step's buffers and the tape).
    quit
The fixed dt is checked against time_step(courant) of every step; the steps where it is larger are counted.
``--moving``: the moving mesh (Rollout with Motion::moving, rollout.cpp:138-163), remeshed on the device every step;
the forward keeps the positions' tape beside the states' and its final rows carry the moved generators and the final
mesh's volumes; ``cfl`` and ``geometry`` start from the lattice's mesh. ``--order=0|1`` (default 1, as the reference's
server): the scheme's order. The moving derivatives (rollout.cpp:170-271: step_moving_tangent / step_moving_adjoint,
the final volumes' bars onto the positions through the geometry derivative) are served for orders 0 and 1 in 2D, with
the 2D geometry derivative of luna_cpp_b200.geometry_derivative; in 3D ``adjoint`` and ``tangent`` answer an error line
(a 3D geometry derivative is not in the library).
"""
from __future__ import annotations

import sys
import time

import numpy as np


def flag(argv, name, fallback):
    for a in argv:
        if a.startswith(name + "="):
            return a[len(name) + 1:]
    return fallback


def lattice(side: int, dim: int) -> np.ndarray:
    """Rollout::lattice (rollout.cpp:119-133): the cell centres on the 2^-30 grid, C order (the last axis fastest)."""
    step = 2.0 ** -30
    idx = np.stack(np.meshgrid(*[np.arange(side)] * dim, indexing="ij"), -1).reshape(-1, dim)
    return np.floor((idx + 0.5) / side / step) * step


class Server:
    def __init__(self, dim: int, side: int, steps: int, dt: float, gamma: float, courant: float, moving: bool = False,
                 order: int = 1):
        import torch

        from .hydro import FiniteVolume, Gas
        from .mesh import build_mesh

        self.torch = torch
        self.dim, self.steps, self.dt, self.courant, self.moving = dim, steps, dt, courant, moving
        self.V = dim + 2
        self.x0 = lattice(side, dim)
        self.mesh = build_mesh(self.x0, box=(1.0,) * dim)
        self.n = self.mesh.n_cells
        self.V0 = self.mesh.volume.copy()
        self.order = order
        self.fv = FiniteVolume(self.mesh, Gas(gamma), order=order, update="per_face", limiter="face_centroid",
                               motion="moving" if moving else "static_mesh")
        self.tape = torch.empty((steps, self.n, self.V), dtype=torch.float64, device="cuda")
        self.xtape = None
        if moving:
            from .remesh import Remesher

            self.remesher = Remesher(dim, (1.0,) * dim)
            self.xtape = torch.empty((steps, self.n, dim), dtype=torch.float64, device="cuda")
        self.volume_dev = torch.tensor(self.V0, device="cuda")[:, None]
        self.peak = self.now()

    def now(self) -> int:
        tapes = self.tape.numel() + (self.xtape.numel() if self.xtape is not None else 0)
        remesh = self.remesher.device_bytes() if self.moving else 0
        return int(self.fv.device_bytes() + remesh + tapes * 8)

    def load(self, U0: np.ndarray) -> None:
        if self.moving:  # load_positions(x0): back to the lattice's mesh
            self.fv.set_mesh(self.mesh)
        self.fv.set_state(np.ascontiguousarray(U0.reshape(self.n, self.V) * self.V0[:, None]))

    def forward(self, U0: np.ndarray) -> int:
        """Rollout::forward (rollout.cpp:153-168): the tape of states (and of positions, moving) before each step."""
        self.load(U0)
        violations = 0
        for s in range(self.steps):
            self.fv.get_state(out=self.tape[s])
            if self.moving:
                self.xtape[s].copy_(self.torch.from_numpy(self.fv.positions()))
            violations += self.fv.time_step(self.courant) < self.dt
            if self.moving:
                self.fv.step_moving_device(self.dt, self.remesher)
            else:
                self.fv.step(self.dt)
        if self.moving:
            self.final_x = self.fv.positions()  # the final mesh's generators (the adjoint's volume bars)
        return violations

    def final_rows(self) -> np.ndarray:
        """Rollout::final_rows (rollout.cpp:169-183): Q, x and the volumes of the final mesh."""
        w = self.V + self.dim + 1
        rows = np.empty((self.n, w))
        rows[:, :self.V] = self.fv.get_state()
        if self.moving:
            rows[:, self.V:self.V + self.dim] = self.fv.positions()
            rows[:, -1] = self.fv.mesh.cells().volume if hasattr(self.fv.mesh, "cells") else self.fv.mesh.volume
        else:
            rows[:, self.V:self.V + self.dim] = self.x0
            rows[:, -1] = self.V0
        return rows

    def _moving_derivatives(self, what):
        if self.dim != 2:
            raise NotImplementedError(f"the moving mesh's {what} is served in 2D (a 3D geometry derivative is not in "
                                      "libluna_b200)")
        from .geometry_derivative import Geometry2D
        from .mesh import build_mesh

        return Geometry2D, (lambda x: build_mesh(x, box=(1.0,) * self.dim))

    def adjoint(self, bars: np.ndarray) -> np.ndarray:
        if self.moving:
            return self._moving_adjoint(bars)
        w = self.V + self.dim + 1
        qbar = self.torch.tensor(np.ascontiguousarray(bars.reshape(self.n, w)[:, :self.V]), device="cuda")
        for s in range(self.steps - 1, -1, -1):
            self.fv.set_state(self.tape[s])
            self.fv.step_adjoint(self.dt, qbar)
        return (qbar * self.volume_dev).cpu().numpy()

    def _moving_adjoint(self, bars: np.ndarray) -> np.ndarray:
        """Rollout::adjoint, moving (rollout.cpp:228-262): the final mesh's volume bars onto the positions, then each step
        backwards from its taped (Q, x) and the geometry derivative of that step's mesh."""
        Geometry2D, remesh = self._moving_derivatives("adjoint")
        w, D = self.V + self.dim + 1, self.dim
        rows = bars.reshape(self.n, w)
        qbar, xbar = rows[:, :self.V].copy(), rows[:, self.V:self.V + D].copy()
        final = remesh(self.final_x)  # the last forward's final mesh (the host builder's is the device remesh's)
        zero_c, zero_f = np.zeros((self.n, D)), np.zeros((final.n_faces, D))
        xbar += Geometry2D(final).adjoint(rows[:, -1], zero_c, zero_f, zero_f)
        for s in range(self.steps - 1, -1, -1):
            x = self.xtape[s].cpu().numpy()
            self.fv.set_mesh(remesh(x))
            self.fv.set_state(self.tape[s])
            self.fv.time_step(self.courant)  # the point velocities of this state
            # order 1: the step runs again to the next mesh for the second pass, and the start is restored
            qbar, xbar = self.fv.step_moving_adjoint(self.dt, qbar, xbar, Geometry2D, remesh)
        return qbar * self.V0[:, None]

    def _moving_tangent(self, U0: np.ndarray, dU0: np.ndarray) -> np.ndarray:
        """Rollout::tangent, moving (rollout.cpp:170-196): the positions' tangent starts at 0; each step's tangent with
        the geometry derivative of its mesh (order 1: of both meshes), the step inside it (host remesh: the same mesh as
        the device remesh's)."""
        Geometry2D, remesh = self._moving_derivatives("tangent")
        self.load(U0)
        dq = np.ascontiguousarray(dU0.reshape(self.n, self.V) * self.V0[:, None])
        dx = np.zeros((self.n, self.dim))
        for _ in range(self.steps):
            self.fv.time_step(self.courant)
            dq, dx = self.fv.step_moving_tangent(self.dt, dq, dx, Geometry2D, remesh)
        return dq

    def tangent(self, U0: np.ndarray, dU0: np.ndarray) -> np.ndarray:
        """Rollout::tangent (rollout.cpp:170-196), static: time_step then step_tangent every step."""
        if self.moving:
            return self._moving_tangent(U0, dU0)
        self.load(U0)
        dq = self.torch.tensor(np.ascontiguousarray(dU0.reshape(self.n, self.V) * self.V0[:, None]), device="cuda")
        for _ in range(self.steps):
            self.fv.time_step(self.courant)
            self.fv.step_tangent(self.dt, dq)
        return dq.cpu().numpy()

    def cfl(self, U0: np.ndarray) -> float:
        self.load(U0)
        return self.fv.time_step(self.courant)

    def geometry(self) -> np.ndarray:
        return np.concatenate([self.x0, self.V0[:, None]], axis=1)


def now_ms(torch) -> float:
    torch.cuda.synchronize()
    return time.perf_counter() * 1e3


def serve(argv, stdin=sys.stdin, stdout=sys.stdout) -> int:
    dim = int(flag(argv, "--dim", "2"))
    srv = Server(dim, int(flag(argv, "--n", "64")), int(flag(argv, "--steps", "100")), float(flag(argv, "--dt", "1e-3")),
                 float(flag(argv, "--gamma", "1.6666666666666667")), float(flag(argv, "--courant", "0.3")),
                 moving=any(a == "--moving" for a in argv), order=int(flag(argv, "--order", "1")))
    torch = srv.torch
    N, V, w = srv.n, srv.V, srv.V + dim + 1

    def answer(text):
        stdout.write(text + "\n")
        stdout.flush()

    for line in stdin:
        parts = line.split()
        if not parts:
            continue
        cmd, args = parts[0], parts[1:]
        try:
            if cmd == "quit":
                break
            if cmd == "forward":
                U0 = np.fromfile(args[0], dtype=np.float64, count=N * V)
                t0 = now_ms(torch)
                violations = srv.forward(U0)
                ms = now_ms(torch) - t0
                srv.final_rows().tofile(args[1])
                answer(f"ok {ms:.17g} {violations}")
            elif cmd == "adjoint":
                bars = np.fromfile(args[0], dtype=np.float64, count=N * w)
                t0 = now_ms(torch)
                out = srv.adjoint(bars)
                ms = now_ms(torch) - t0
                out.tofile(args[1])
                answer(f"ok {ms:.17g}")
            elif cmd == "cfl":
                answer(f"ok {srv.cfl(np.fromfile(args[0], dtype=np.float64, count=N * V)):.17g}")
            elif cmd == "geometry":
                srv.geometry().tofile(args[0])
                answer("ok")
            elif cmd == "memory":
                answer(f"ok {srv.peak} {srv.now()}")
            elif cmd == "tangent":
                U0 = np.fromfile(args[0], dtype=np.float64, count=N * V)
                dU0 = np.fromfile(args[1], dtype=np.float64, count=N * V)
                t0 = now_ms(torch)
                out = srv.tangent(U0, dU0)
                ms = now_ms(torch) - t0
                out.tofile(args[2])
                answer(f"ok {ms:.17g}")
            else:
                answer("error unknown command")
        except Exception as e:  # one answer a line, as the reference's server: the client raises on anything but ok
            answer(f"error {type(e).__name__}: {e}".replace("\n", " "))
        srv.peak = max(srv.peak, srv.now())  # the derivatives' work arrays too
    return 0


def main():
    argv = sys.argv[1:]
    if "--help" in argv:
        print(__doc__)
        return 0
    return serve(argv)


if __name__ == "__main__":
    sys.exit(main())
