"""The 1D step's derivatives on the GPU (luna_line_step_tangent / luna_line_step_adjoint, FiniteVolume<1>::step_tangent
and step_adjoint, finite_volume_1d.hpp:852-923): against LUNA's jax.jvp and jax.vjp of five fixed-dt steps
(hydro_derivatives_test.cpp:991-1088, golden vectors in tests/golden/luna_1d_derivatives.json), against central
differences of the CPU oracle's step, and the dot test <w, J dq> = <J^T w, dq> over walls, limiters and solvers."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "luna_1d_derivatives.json")
LIMITERS = {0: "minmod", 1: "face_centroid", 2: "van_leer"}  # LUNA's LIMITER 0, 1, 2


def _golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _line_of(case, problem):
    from luna_cpp_b200.line import Line

    n, L = case["n"], problem["L"]
    x = L * (np.arange(n) + 0.5) / n
    walls = tuple(problem["walls"]) if problem["walls"] else ("outflow", "outflow")
    return Line(x, L, walls=walls, periodic=problem["periodic"], gamma=problem["gamma"], order=1,
                limiter=LIMITERS[case["limiter"]], riemann="hllc")


@pytest.mark.parametrize("name", list(_golden()["cases"]))
def test_line_derivatives_equal_luna_jax(cuda, name):
    """hydro_derivatives_test.cpp's luna_case: U per volume, so J dU = (J dq) / V and J^T w = (J^T (w / V)) V on the
    extensive Q; the tangent's forward after K steps within 1e-12 of LUNA's U, J dU and J^T w within 1e-8 of LUNA's
    largest entry. The flat Sod with MC (no derivative where MC is flat: LUNA's jvp takes its zero branch, the
    reference the unlimited slope) is reported, not gated, as in the reference."""
    g = _golden()
    case = g["cases"][name]
    ln = _line_of(case, g["problems"][case["problem"]])
    V = ln.volume[:, None]
    U0, dU, w = (np.array(case[k]) for k in ("U0", "dU", "w"))
    ln.set_state(U0 * V)
    dq = dU * V
    path = []
    for _ in range(case["steps"]):
        path.append(ln.get_state()[0])
        dq = ln.step_tangent(case["dt"], dq)[0]
    Q = ln.get_state()[0]
    bar = w / V
    for s in reversed(range(case["steps"])):
        ln.set_state(path[s])
        bar = ln.step_adjoint(case["dt"], bar)[0]
    ln.close()

    def rel(ours, theirs):
        theirs = np.array(theirs)
        return float(np.max(np.abs(ours - theirs)) / np.max(np.abs(theirs)))

    forward, jvp, vjp = rel(Q / V, case["U"]), rel(dq / V, case["JdU"]), rel(bar * V, case["JTw"])
    print(f"{name}: forward {forward:.2e}, J dU {jvp:.2e}, J^T w {vjp:.2e}")
    assert forward < g["tolerance"]["forward"], forward
    if case["gate"]:
        assert jvp < g["tolerance"]["derivatives"] and vjp < g["tolerance"]["derivatives"], (jvp, vjp)
    else:
        assert np.isfinite(jvp) and np.isfinite(vjp)


def _state(n, seed, rough=0.05):
    rng = np.random.default_rng(seed)
    x = (np.arange(n) + 0.5) / n
    rho = 1.0 + 0.3 * np.sin(2 * np.pi * x) + rough * rng.uniform(-1, 1, n)
    v = 0.4 * np.cos(2 * np.pi * x) + rough * rng.uniform(-1, 1, n)
    P = 1.0 + 0.2 * np.sin(4 * np.pi * x + 0.3) + rough * rng.uniform(-1, 1, n)
    return np.stack([rho, v, P], axis=1)


def _conserved(W, V, gamma):
    rho, v, P = W[:, 0], W[:, 1], W[:, 2]
    return np.stack([rho, rho * v, P / (gamma - 1) + 0.5 * rho * v * v], axis=1) * V[:, None]


DOT_CASES = [
    # (walls, periodic, limiter, riemann, order)
    (("outflow", "outflow"), True, "face_centroid", "hllc", 1),
    (("outflow", "outflow"), False, "face_centroid", "hllc", 1),
    (("reflective", "reflective"), False, "face_centroid", "hllc", 1),
    (("reflective", "outflow"), False, "minmod", "hllc", 1),
    (("outflow", "reflective"), False, "van_leer", "hllc", 1),
    (("outflow", "outflow"), False, "none", "hllc", 1),
    (("outflow", "outflow"), False, "face_centroid", "hll", 1),
    (("reflective", "reflective"), False, "face_centroid", "hllc", 0),
    (("inflow", "outflow"), False, "face_centroid", "hllc", 1),
]


@pytest.mark.parametrize("walls,periodic,limiter,riemann,order", DOT_CASES)
def test_line_dot_test(cuda, walls, periodic, limiter, riemann, order):
    """<w, J dq> = <J^T w, dq> over 3 steps on a jittered line of 96 cells in a shuffled caller order, three lines of
    different states in one batch (each line's own dt), relative to the sum of the products' magnitudes (the reference's
    dot test, hydro_derivatives_test.cpp:977-985, 1e-13); each line's J dq equals a single-line run's."""
    from luna_cpp_b200.line import Line

    n, lines, gamma, steps = 96, 3, 1.4, 3
    rng = np.random.default_rng(7)
    x = (np.arange(n) + 0.5 + 0.4 * rng.uniform(-0.5, 0.5, n)) / n
    perm = rng.permutation(n)
    x = x[perm]
    inflow = [[1.2, 0.3, 1.1], [1.0, 0.0, 1.0]] if "inflow" in walls else None
    kw = dict(walls=walls, periodic=periodic, inflow=inflow, gamma=gamma, order=order, limiter=limiter, riemann=riemann)
    ln = Line(x, 1.0, lines=lines, **kw)
    V = ln.volume
    q0 = np.stack([_conserved(_state(n, 10 + k), V, gamma) for k in range(lines)])
    dq0 = rng.normal(size=(lines, n, 3)) * np.abs(q0)
    w = rng.normal(size=(lines, n, 3))
    ln.set_state(q0)
    dt = 0.3 * ln.time_step(0.8, "luna")
    path, dq = [], dq0
    for _ in range(steps):
        path.append(ln.get_state())
        dq = ln.step_tangent(dt, dq)
    bar = w
    for s in reversed(range(steps)):
        ln.set_state(path[s])
        bar = ln.step_adjoint(dt, bar)
    for k in range(lines):
        lhs, rhs = float(np.sum(w[k] * dq[k])), float(np.sum(bar[k] * dq0[k]))
        size = float(np.sum(np.abs(w[k] * dq[k])) + np.sum(np.abs(bar[k] * dq0[k])))
        assert abs(lhs - rhs) < 1e-13 * size, (k, lhs, rhs, size)
    one = Line(x, 1.0, lines=1, **kw)
    one.set_state(q0[1])
    d1 = dq0[1]
    for _ in range(steps):
        d1 = one.step_tangent(dt[1], d1)[0]
    assert np.array_equal(d1, dq[1])
    ln.close()
    one.close()


@pytest.mark.parametrize("limiter", ["face_centroid", "minmod", "van_leer"])
@pytest.mark.parametrize("walls,periodic", [(("outflow", "outflow"), True), (("reflective", "outflow"), False)])
def test_line_tangent_equals_oracle_central_differences(cuda, limiter, walls, periodic):
    """J dq of one step against central differences of the CPU oracle's step (h = 1e-6 relative to each entry of dq) on
    a smooth state with 1 % noise: within 1e-6 of the largest entry (the reference's step_test bound,
    hydro_derivatives_test.cpp:508-546),
    or, at a limiter switch within +- h, a one-sided difference within 1e-4; the tangent's own forward equals step()'s
    bit for bit."""
    from luna_cpp_b200.line import Line
    from luna_cpp_b200.problems import line_keys
    from oracle import oracle as O

    n, gamma, h = 64, 1.4, 1e-6
    # jittered generators and a little noise (the reference's smooth step_test, noise 0.01): no two neighbours tie, so
    # the limiter's min / max have a derivative everywhere
    x = (np.arange(n) + 0.5 + 0.3 * np.random.default_rng(5).uniform(-0.5, 0.5, n)) / n
    ln = Line(x, 1.0, walls=walls, periodic=periodic, gamma=gamma, limiter=limiter)
    plain = Line(x, 1.0, walls=walls, periodic=periodic, gamma=gamma, limiter=limiter)
    q0 = _conserved(_state(n, 3, rough=0.01), ln.volume, gamma)
    dq = np.random.default_rng(1).normal(size=(n, 3)) * np.abs(q0)
    ln.set_state(q0)
    plain.set_state(q0)
    dt = float(0.5 * ln.time_step(0.8, "luna")[0])
    J = ln.step_tangent(dt, dq)[0]
    plain.step(dt)
    assert np.array_equal(ln.get_state(), plain.get_state())
    keys, order, step, period = line_keys(x, 1.0)
    oracle = O.OracleLine(keys, step, period, gamma=gamma, walls=walls, periodic=periodic, limiter=limiter)

    def advance(q):
        oracle.set_state(q[order])
        oracle.step(dt)
        out = np.empty_like(q)
        out[order] = oracle.get_state()
        return out

    at, plus, minus = advance(q0), advance(q0 + h * dq), advance(q0 - h * dq)
    fd = (plus - minus) / (2 * h)
    scale = float(np.max(np.abs(fd)))
    cell = np.max(np.abs(J - fd), axis=1) / scale
    # a limiter switch within +- h: there the tangent is one of the one-sided differences (to their O(h) error)
    one_sided = np.minimum(np.max(np.abs(J - (plus - at) / h), axis=1), np.max(np.abs(J - (at - minus) / h), axis=1)) / scale
    switched = cell > 1e-6
    assert np.sum(switched) <= 2 and np.all(one_sided[switched] < 1e-4), (np.max(cell), np.sum(switched))
    ln.close()
    plain.close()


def test_line_derivatives_on_device_buffers(cuda):
    """The same derivatives through device memory (on_device = 1) as through host memory."""
    import ctypes

    import torch

    from luna_cpp_b200.hydro import check, lib
    from luna_cpp_b200.line import Line

    n, gamma = 80, 1.4
    x = (np.arange(n) + 0.5) / n
    a = Line(x, 1.0, walls=("reflective", "outflow"), gamma=gamma)
    b = Line(x, 1.0, walls=("reflective", "outflow"), gamma=gamma)
    q0 = _conserved(_state(n, 5), a.volume, gamma)
    v = np.random.default_rng(2).normal(size=(n, 3))
    for ln in (a, b):
        ln.set_state(q0)
    dt = np.array([0.2 * a.time_step(0.8, "luna")[0]])
    want_t = a.step_tangent(dt, v)[0]
    a.set_state(q0)
    want_a = a.step_adjoint(dt, v)[0]
    for fn, want in (("luna_line_step_tangent", want_t), ("luna_line_step_adjoint", want_a)):
        b.set_state(q0)
        d = torch.tensor(v, device="cuda", dtype=torch.float64)
        check(getattr(lib(), fn)(b._h, dt.ctypes.data, ctypes.c_void_p(d.data_ptr()), 1))
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy(), want), fn
    a.close()
    b.close()


def test_periodic_line_derivatives_need_five_cells(cuda):
    from luna_cpp_b200.hydro import LunaError
    from luna_cpp_b200.line import Line

    ln = Line((np.arange(4) + 0.5) / 4, 1.0, periodic=True)
    ln.set_state(np.tile([1.0, 0.0, 2.5], (4, 1)) * 0.25)
    with pytest.raises(LunaError):
        ln.step_tangent(0.01, np.zeros((4, 3)))
    ln.close()
