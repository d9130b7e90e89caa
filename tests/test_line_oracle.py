"""The 1D oracle (oracle/oracle_line.c, FiniteVolume<1> on a static line) pinned to LUNA's final states and to the
reference's 1D invariants (src/test/hydro1d_test.cpp), on the CPU."""
import json
import os

import numpy as np
import pytest

from luna_cpp_b200.problems import line_keys, line_problem, line_state
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "luna_1d_final_states.json")


def run(ln, t_end, courant, rule):
    """hydro1d_test.cpp's run() (:100-110): to t_end, the last step shortened."""
    t, steps = 0.0, 0
    while t < t_end * (1 - 1e-12):
        dt = min(ln.time_step(courant, rule), t_end - t)
        ln.step(dt)
        t += dt
        steps += 1
    return steps


def primitives(q, volume, gamma):
    U = q / volume[:, None]
    rho = U[:, 0]
    v = U[:, 1] / rho
    return np.stack([rho, v, (gamma - 1) * (U[:, 2] - 0.5 * rho * v * v)], axis=1)


@pytest.mark.parametrize("name", ["sod", "shu-osher", "woodward-colella"])
def test_oracle_equals_luna_final_states(name):
    """hydro1d_test.cpp:266-296: N = 16 uniform cells, LUNA's rule at CFL 0.8, the same step count and every primitive
    within 1e-12 of LUNA's relative to 1e-3 + |W|."""
    golden = json.load(open(GOLDEN))
    case = golden["cases"][name]
    p = line_problem(name)
    n = golden["cells"]
    keys, _, step, period = line_keys(p["L"] * (np.arange(n) + 0.5) / n, p["L"])
    ln = O.OracleLine(keys, step, period, gamma=p["gamma"], walls=p["walls"])
    ln.set_state(line_state(p, keys, step))
    steps = run(ln, p["t_end"], golden["courant"], "luna")
    W = primitives(ln.get_state(), ln.volumes(), p["gamma"])
    want = np.array(case["W"])
    worst = np.max(np.abs(W - want) / (1e-3 + np.abs(want)))
    assert steps == case["steps"]
    assert worst < golden["tolerance"], worst


def jittered_keys(n, L, seed=3, jitter=0.5):
    rng = np.random.default_rng(seed)
    x = L * (np.arange(n) + 0.5 + jitter * rng.uniform(-0.5, 0.5, n)) / n
    return line_keys(x, L)


@pytest.mark.parametrize("walls,periodic", [(("reflective", "reflective"), False), (("outflow", "outflow"), True)])
@pytest.mark.parametrize("limiter", ["face_centroid", "minmod", "van_leer", "none"])
def test_oracle_uniform_state_stays_uniform(walls, periodic, limiter):
    """hydro1d_test.cpp:130-155: a uniform state (at rest between reflective walls, with a bulk velocity on a periodic
    line) stays uniform on a jittered line."""
    keys, _, step, period = jittered_keys(64, 1.0)
    v = 0.0 if not periodic else 0.7
    ln = O.OracleLine(keys, step, period, gamma=1.4, walls=walls, periodic=periodic, limiter=limiter)
    W = np.array([1.3, v, 0.9])
    U = np.array([W[0], W[0] * W[1], W[2] / 0.4 + 0.5 * W[0] * W[1] * W[1]])
    ln.set_state(U[None, :] * ln.volumes()[:, None])
    for _ in range(20):
        ln.step(ln.time_step(0.8, "arepo"))
    Wn = primitives(ln.get_state(), ln.volumes(), 1.4)
    assert np.max(np.abs(Wn - W[None, :])) < 1e-13


@pytest.mark.parametrize("periodic", [False, True])
def test_oracle_conserves(periodic):
    """hydro1d_test.cpp:172-196: mass and energy (and momentum on a periodic line) conserved to round-off through
    reflective walls, on a jittered line with a jump."""
    keys, _, step, period = jittered_keys(128, 1.0, seed=5)
    walls = ("reflective", "reflective")
    ln = O.OracleLine(keys, step, period, gamma=1.4, walls=walls, periodic=periodic)
    p = line_problem("sod")
    q0 = line_state(p, keys, step) if not periodic else None
    if periodic:
        x = keys * step
        rho = np.where(np.abs(x - 0.5) < 0.25, 1.0, 0.125)
        P = np.where(np.abs(x - 0.5) < 0.25, 1.0, 0.1)
        q0 = np.stack([rho, 0.3 * rho, P / 0.4 + 0.5 * rho * 0.09], 1) * ln.volumes()[:, None]
    ln.set_state(q0)
    for _ in range(40):
        ln.step(ln.time_step(0.8, "arepo"))
    q = ln.get_state()
    tot0, tot = q0.sum(0), q.sum(0)
    assert abs(tot[0] - tot0[0]) < 1e-14 * abs(tot0[0])
    assert abs(tot[2] - tot0[2]) < 1e-14 * abs(tot0[2])
    if periodic:
        assert abs(tot[1] - tot0[1]) < 1e-14 * abs(tot0[0])


def test_oracle_forward_of_luna_derivative_cases():
    """The forward of LUNA's derivative cases (src/test/luna_derivative_values.hpp, hydro_derivatives_test.cpp:1054):
    K fixed-dt steps of U0 on N = 64 uniform cells within 1e-12 of LUNA's U, relative to its largest entry, for every
    case (Sod between outflow walls, the periodic sound wave; minmod, MC, van Leer)."""
    golden = json.load(open(os.path.join(os.path.dirname(GOLDEN), "luna_1d_derivatives.json")))
    limiters = {0: "minmod", 1: "face_centroid", 2: "van_leer"}
    for name, case in golden["cases"].items():
        p = golden["problems"][case["problem"]]
        n = case["n"]
        keys, order, step, period = line_keys(p["L"] * (np.arange(n) + 0.5) / n, p["L"])
        walls = tuple(p["walls"]) if p["walls"] else ("outflow", "outflow")
        ln = O.OracleLine(keys, step, period, gamma=p["gamma"], walls=walls, periodic=p["periodic"],
                          limiter=limiters[case["limiter"]])
        V = ln.volumes()[:, None]
        ln.set_state(np.array(case["U0"]) * V)
        for _ in range(case["steps"]):
            ln.step(case["dt"])
        want = np.array(case["U"])
        err = np.max(np.abs(ln.get_state() / V - want)) / np.max(np.abs(want))
        assert err < golden["tolerance"]["forward"], (name, err)
