"""The rollout server (luna_cpp_b200/rollout.py, the protocol of the reference's src/examples/rollout.cpp): the host side on
the CPU, the served forward and adjoint on the GPU (checked against central differences through the protocol itself)."""
import os
import subprocess

import numpy as np
import pytest

from luna_cpp_b200 import rollout

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "luna_cpp_b200", "bin", "rollout")


def test_lattice_is_c_order_on_the_grid():
    x = rollout.lattice(4, 3)
    assert x.shape == (64, 3)
    assert np.allclose(x[1], [0.125, 0.125, 0.375]) and np.allclose(x[4], [0.125, 0.375, 0.125])
    assert np.all(np.round(x * 2 ** 30) == x * 2 ** 30)


class Client:
    """A minimal client of the protocol (one command a line, raw float64 files)."""

    def __init__(self, tmp, dim, n, steps, dt, moving=False, order=1):
        self.dim, self.N, self.V, self.tmp = dim, n ** dim, dim + 2, tmp
        extra = (["--moving"] if moving else []) + [f"--order={order}"]
        self.p = subprocess.Popen([BIN, f"--dim={dim}", f"--n={n}", f"--steps={steps}", f"--dt={dt!r}"] + extra,
                                  stdin=subprocess.PIPE, stdout=subprocess.PIPE, text=True, bufsize=1)

    def ask(self, line):
        self.p.stdin.write(line + "\n")
        self.p.stdin.flush()
        return self.p.stdout.readline().split()

    def forward(self, U0):
        U0.astype(np.float64).tofile(self.tmp / "u0.bin")
        out = self.ask(f"forward {self.tmp / 'u0.bin'} {self.tmp / 'fin.bin'}")
        assert out[0] == "ok", out
        return np.fromfile(self.tmp / "fin.bin").reshape(self.N, self.V + self.dim + 1), int(out[2])

    def close(self):
        self.p.stdin.write("quit\n")
        self.p.stdin.flush()
        assert self.p.wait(timeout=60) == 0


@pytest.mark.gpu
def test_served_adjoint_matches_central_differences(cuda, tmp_path):
    """A 2D shear layer on the 32^2 lattice, 12 steps at a fixed dt: dL/dU0 from `adjoint` against central differences of
    `forward` along a smooth direction (L = <bars, final rows>); the served tangent is its transpose (the dot test);
    `cfl`, `geometry` and `memory` answer."""
    c = Client(tmp_path, 2, 32, 12, 2e-3)
    try:
        xc = (np.arange(32) + 0.5) / 32
        X, Y = np.meshgrid(xc, xc, indexing="ij")
        # the shear layer with smooth sides and a little seeded noise: on the lattice an exactly symmetric state puts
        # the limiter's comparisons on ties, kinks at the very point the differences are taken
        noise = np.random.default_rng(8).uniform(-1e-3, 1e-3, (4,) + X.shape)
        layer = np.tanh((0.25 - np.abs(Y - 0.5)) / 0.05)
        rho = 1.5 + 0.5 * layer + noise[0]
        vx = 0.5 * layer + noise[1]
        vy = 0.01 * np.sin(2 * np.pi * X) + noise[2]
        P = 2.5 + noise[3]
        U0 = np.stack([rho, rho * vx, rho * vy, P / (2 / 3) + 0.5 * rho * (vx * vx + vy * vy)], -1).reshape(-1, 4)
        ok = c.ask(f"geometry {tmp_path / 'g.bin'}")
        assert ok == ["ok"]
        g = np.fromfile(tmp_path / "g.bin").reshape(-1, 3)
        assert np.allclose(g[:, 2], 1 / 1024) and np.allclose(g[33, :2], [1.5 / 32, 1.5 / 32])
        U0.tofile(tmp_path / "u0.bin")
        out = c.ask(f"cfl {tmp_path / 'u0.bin'}")
        assert out[0] == "ok" and float(out[1]) > 2e-3
        fin, violations = c.forward(U0)
        assert violations == 0 and np.all(np.isfinite(fin))
        rng = np.random.default_rng(4)
        bars = np.zeros_like(fin)
        bars[:, :4] = rng.standard_normal((fin.shape[0], 4))
        bars.tofile(tmp_path / "bars.bin")
        out = c.ask(f"adjoint {tmp_path / 'bars.bin'} {tmp_path / 'ubar.bin'}")
        assert out[0] == "ok", out
        ubar = np.fromfile(tmp_path / "ubar.bin").reshape(-1, 4)
        # along a smooth direction (a mode of the layer's vy), as the library's adjoint tests: a random field would
        # move the limiter's clips within h, where the adjoint (one branch) and the differences part
        d = np.zeros_like(U0)
        d[:, 2] = (rho * np.sin(4 * np.pi * X)).reshape(-1)
        d[:, 3] = (rho * vy * np.sin(4 * np.pi * X)).reshape(-1)
        h = 1e-7  # the limiter's branches: at 1e-6 some clips switch within +-h over 12 steps (differences off by 8e-4)
        Lp = float((c.forward(U0 + h * d)[0] * bars).sum())
        Lm = float((c.forward(U0 - h * d)[0] * bars).sum())
        fd = (Lp - Lm) / (2 * h)
        assert abs(float((ubar * d).sum()) - fd) <= 1e-6 * abs(fd)
        out = c.ask("memory")
        assert out[0] == "ok" and int(out[1]) >= int(out[2]) > 0
        # the served tangent is the served adjoint's transpose: <dQ(dU0), Qbar> = <dU0, U0bar>
        U0.tofile(tmp_path / "u0.bin")
        d.tofile(tmp_path / "du0.bin")
        out = c.ask(f"tangent {tmp_path / 'u0.bin'} {tmp_path / 'du0.bin'} {tmp_path / 'dq.bin'}")
        assert out[0] == "ok", out
        dQ = np.fromfile(tmp_path / "dq.bin").reshape(-1, 4)
        lhs, rhs = float((dQ * bars[:, :4]).sum()), float((ubar * d).sum())
        assert abs(lhs - rhs) <= 1e-12 * abs(rhs)
    finally:
        c.close()


@pytest.mark.gpu
def test_served_moving_forward(cuda, tmp_path):
    """--moving: a 2D shear layer on the 32^2 lattice, 10 moving steps remeshed on the device. The final rows carry the
    moved generators and the final mesh's volumes (which tile the box), mass and momentum are conserved, a second
    forward from the same U0 restarts from the lattice's mesh (the same bits), and zero bars give a zero U0 bar."""
    c = Client(tmp_path, 2, 32, 10, 2e-3, moving=True)
    try:
        xc = (np.arange(32) + 0.5) / 32
        X, Y = np.meshgrid(xc, xc, indexing="ij")
        layer = np.tanh((0.25 - np.abs(Y - 0.5)) / 0.05)
        rho = 1.5 + 0.5 * layer
        vx = 0.5 * layer
        vy = 0.01 * np.sin(2 * np.pi * X)
        P = 2.5 + 0 * X
        U0 = np.stack([rho, rho * vx, rho * vy, P / (2 / 3) + 0.5 * rho * (vx * vx + vy * vy)], -1).reshape(-1, 4)
        fin, violations = c.forward(U0)
        assert violations == 0 and np.all(np.isfinite(fin))
        x = fin[:, 4:6]
        assert np.max(np.abs(x - rollout.lattice(32, 2))) > 1e-4  # the generators moved with the flow
        assert abs(fin[:, 6].sum() - 1.0) < 1e-12
        Q0 = U0 * (1 / 1024)
        assert np.allclose(fin[:, :3].sum(0), Q0[:, :3].sum(0), rtol=1e-12, atol=1e-14)
        again, _ = c.forward(U0)
        assert again.tobytes() == fin.tobytes()
        bars = np.zeros_like(fin)
        bars.tofile(tmp_path / "bars.bin")
        assert c.ask(f"adjoint {tmp_path / 'bars.bin'} {tmp_path / 'ubar.bin'}")[0] == "ok"
        assert not np.any(np.fromfile(tmp_path / "ubar.bin"))
        out = c.ask("memory")
        assert out[0] == "ok" and int(out[1]) >= int(out[2]) > 0
    finally:
        c.close()


@pytest.mark.gpu
def test_served_moving_derivatives_order_0(cuda, tmp_path):
    """--moving --order=0 in 2D: the served adjoint (the final volumes' bars onto the positions, then each step's
    step_moving_adjoint with the 2D geometry derivative, rollout.cpp:228-262) against central differences of the served
    forward of L = <bars, final rows>, and the served tangent against it by the dot test (1e-10). The lattice start puts
    HLLC's contact speed at zero on the quiet faces (a kink within 1e-5 of U0 along d) and the moved mesh near four-way
    cocircular vertices, so the differences are good to about 1e-6 with bars on Q alone (h = 1e-6; the reference's own
    step_moving_tangent gives 8.5e-8 there) and to about 1e-5 with bars on x and V as well."""
    c = Client(tmp_path, 2, 24, 6, 2e-3, moving=True, order=0)
    try:
        xc = (np.arange(24) + 0.5) / 24
        X, Y = np.meshgrid(xc, xc, indexing="ij")
        noise = np.random.default_rng(8).uniform(-1e-3, 1e-3, (4,) + X.shape)
        layer = np.tanh((0.25 - np.abs(Y - 0.5)) / 0.08)
        rho = 1.5 + 0.5 * layer + noise[0]
        vx = 0.4 * layer + noise[1]
        vy = 0.05 * np.sin(2 * np.pi * X) + noise[2]
        P = 2.5 + noise[3]
        U0 = np.stack([rho, rho * vx, rho * vy, P / (2 / 3) + 0.5 * rho * (vx * vx + vy * vy)], -1).reshape(-1, 4)
        fin, violations = c.forward(U0)
        assert violations == 0
        rng = np.random.default_rng(4)
        bars = rng.standard_normal(fin.shape)
        bars[:, 4:6] *= 10.0  # the positions' and volumes' bars on the scale of Q's effect
        d = rng.standard_normal(U0.shape) * np.abs(U0) * 1e-2
        qbars = np.zeros_like(fin)
        qbars[:, :4] = bars[:, :4]
        h = 1e-6
        plus, minus = c.forward(U0 + h * d)[0], c.forward(U0 - h * d)[0]
        c.forward(U0)  # the adjoint's tape is the last forward's
        for b, bound in ((qbars, 1e-6), (bars, 1e-4)):
            b.tofile(tmp_path / "bars.bin")
            out = c.ask(f"adjoint {tmp_path / 'bars.bin'} {tmp_path / 'ubar.bin'}")
            assert out[0] == "ok", out
            ubar = np.fromfile(tmp_path / "ubar.bin").reshape(-1, 4)
            fd = float(((plus - minus) * b).sum()) / (2 * h)
            assert abs(float((ubar * d).sum()) - fd) <= bound * abs(fd), (float((ubar * d).sum()), fd)
            if b is qbars:
                qbar_u = ubar
        U0.tofile(tmp_path / "u0.bin")
        d.tofile(tmp_path / "du0.bin")
        out = c.ask(f"tangent {tmp_path / 'u0.bin'} {tmp_path / 'du0.bin'} {tmp_path / 'dq.bin'}")
        assert out[0] == "ok", out
        dQ = np.fromfile(tmp_path / "dq.bin").reshape(-1, 4)
        lhs, rhs = float((dQ * bars[:, :4]).sum()), float((qbar_u * d).sum())
        assert abs(lhs - rhs) <= 1e-10 * abs(rhs)
    finally:
        c.close()


@pytest.mark.gpu
def test_served_moving_derivatives_order_1(cuda, tmp_path):
    """--moving (order 1, the default) in 2D: the served tangent and adjoint (two passes a step, the geometry derivative
    of both meshes, the grid steps' derivative taken as dw as in the reference's server) are each other's transpose (the
    dot test, 1e-10), and the adjoint against central differences of the served forward of L = <bars, final rows>. The
    forward moves the points by whole grid steps (2^-30), which the derivative takes as the identity: the difference
    (h = 1e-2 along a direction of 1e-2 of U0, moving the points by about 60 grid steps a step) carries the
    quantisation's error of a few per cent (the reference leaves this check ungated, hydro_derivatives_test.cpp:1693).
    The precise check of these derivatives is the library's against the reference's own (test_gpu_reference)."""
    c = Client(tmp_path, 2, 24, 4, 2e-3, moving=True, order=1)
    try:
        xc = (np.arange(24) + 0.5) / 24
        X, Y = np.meshgrid(xc, xc, indexing="ij")
        noise = np.random.default_rng(8).uniform(-1e-2, 1e-2, (4,) + X.shape)
        k = 2 * np.pi
        rho = 1 + 0.2 * np.sin(k * X) + noise[0]
        vx = 0.3 * np.sin(k * Y) + noise[1]
        vy = 0.2 * np.cos(k * X) + noise[2]
        P = 1 + 0.2 * np.cos(k * (X + Y)) + noise[3]
        U0 = np.stack([rho, rho * vx, rho * vy, P / (2 / 3) + 0.5 * rho * (vx * vx + vy * vy)], -1).reshape(-1, 4)
        fin, violations = c.forward(U0)
        assert violations == 0
        rng = np.random.default_rng(4)
        bars = rng.standard_normal(fin.shape)
        bars[:, 4:6] *= 10.0
        d = rng.standard_normal(U0.shape) * np.abs(U0) * 1e-2
        h = 1e-2
        plus, minus = c.forward(U0 + h * d)[0], c.forward(U0 - h * d)[0]
        c.forward(U0)  # the adjoint's tape is the last forward's
        bars.tofile(tmp_path / "bars.bin")
        out = c.ask(f"adjoint {tmp_path / 'bars.bin'} {tmp_path / 'ubar.bin'}")
        assert out[0] == "ok", out
        ubar = np.fromfile(tmp_path / "ubar.bin").reshape(-1, 4)
        fd = float(((plus - minus) * bars).sum()) / (2 * h)
        print("served order-1 adjoint against central differences:", float((ubar * d).sum()), fd)
        assert abs(float((ubar * d).sum()) - fd) <= 5e-2 * abs(fd), (float((ubar * d).sum()), fd)
        U0.tofile(tmp_path / "u0.bin")
        d.tofile(tmp_path / "du0.bin")
        out = c.ask(f"tangent {tmp_path / 'u0.bin'} {tmp_path / 'du0.bin'} {tmp_path / 'dq.bin'}")
        assert out[0] == "ok", out
        dQ = np.fromfile(tmp_path / "dq.bin").reshape(-1, 4)
        qbars = bars.copy()
        qbars[:, 4:] = 0
        qbars.tofile(tmp_path / "bars.bin")
        c.forward(U0)
        out = c.ask(f"adjoint {tmp_path / 'bars.bin'} {tmp_path / 'ubar.bin'}")
        qbar_u = np.fromfile(tmp_path / "ubar.bin").reshape(-1, 4)
        lhs, rhs = float((dQ * bars[:, :4]).sum()), float((qbar_u * d).sum())
        assert abs(lhs - rhs) <= 1e-10 * abs(rhs), (lhs, rhs)
    finally:
        c.close()
