"""The CUDA line solver (luna_line_*, FiniteVolume<1> on a static line) against LUNA's final states and the CPU oracle."""
import json
import os

import numpy as np
import pytest

from luna_cpp_b200.problems import line_keys, line_problem, line_state

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "luna_1d_final_states.json")


@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("name", ["sod", "shu-osher", "woodward-colella"])
def test_line_equals_luna_final_states(cuda, name, fused):
    """hydro1d_test.cpp:266-296 on the GPU: N = 16, LUNA's rule at CFL 0.8, the same step count, every primitive within
    1e-12 of LUNA's relative to 1e-3 + |W|; also through the fused step (step_and_time_step)."""
    from luna_cpp_b200.line import Line, run_to

    golden = json.load(open(GOLDEN))
    case = golden["cases"][name]
    p = line_problem(name)
    n = golden["cells"]
    x = p["L"] * (np.arange(n) + 0.5) / n
    ln = Line(x, p["L"], walls=p["walls"], gamma=p["gamma"])
    keys, order, step, _ = line_keys(x, p["L"])
    q = np.empty((n, 3))
    q[order] = line_state(p, keys, step)
    ln.set_state(q)
    steps = run_to(ln, p["t_end"], golden["courant"], "luna", fused=fused)
    W = ln.primitives()[0]
    want = np.array(case["W"])
    worst = np.max(np.abs(W[np.argsort(x)] - want) / (1e-3 + np.abs(want)))
    assert int(steps[0]) == case["steps"]
    assert worst < golden["tolerance"], worst


CASES = [
    dict(walls=("reflective", "reflective")),
    dict(walls=("outflow", "reflective"), limiter="minmod"),
    dict(walls=("inflow", "outflow"), inflow=[[1.5, 0.4, 1.2], [0, 0, 0]], limiter="van_leer"),
    dict(walls=("outflow", "outflow"), periodic=True, riemann="hll"),
    dict(walls=("reflective", "outflow"), order=0),
    dict(walls=("outflow", "outflow"), limiter="none"),
]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("rule", ["arepo", "luna"])
def test_line_matches_oracle_on_jittered_lines(cuda, case, rule):
    """A jittered line (generators in shuffled order), 40 steps of a shock tube with every wall, limiter, Riemann solver
    and order, both time-step rules: dt and the state agree with the oracle to 1e-12 relative."""
    from luna_cpp_b200.line import Line
    from oracle import oracle as O

    kw = CASES[case]
    rng = np.random.default_rng(11 + case)
    n = 200
    x = (np.arange(n) + 0.5 + 0.6 * rng.uniform(-0.5, 0.5, n)) / n
    perm = rng.permutation(n)
    x = x[perm]
    p = line_problem("toro-2" if case % 2 else "sod")
    keys, order, step, period = line_keys(x, 1.0)
    q_slots = line_state(p, keys, step)
    inflow = np.array(kw.get("inflow", np.zeros((2, 3))), dtype=np.float64)
    opts = dict(walls=kw["walls"], periodic=kw.get("periodic", False), order=kw.get("order", 1),
                limiter=kw.get("limiter", "face_centroid"), riemann=kw.get("riemann", "hllc"))
    ref = O.OracleLine(keys, step, period, gamma=1.4, inflow=inflow, **opts)
    ref.set_state(q_slots)
    ln = Line(x, 1.0, inflow=inflow if "inflow" in kw else None, gamma=1.4, **opts)
    q = np.empty((n, 3))
    q[order] = q_slots
    ln.set_state(q)
    for _ in range(40):
        dt_ref = ref.time_step(0.8, rule)
        dt = ln.time_step(0.8, rule)[0]
        assert abs(dt - dt_ref) <= 1e-13 * dt_ref
        ref.step(dt_ref)
        ln.step(dt_ref)
    got = ln.get_state()[0][order]
    want = ref.get_state()
    scale = np.abs(want).max(0)
    assert np.max(np.abs(got - want) / scale) < 1e-12


def test_line_batch_equals_single_lines_and_fused_dt(cuda):
    """Lines of a batch are independent (each bit-equal to its own single-line run through the same kernel); the fused
    step's next dt equals time_step by LUNA's rule after it; the fused and the separate step agree to rounding (they are
    separate kernels, whose multiply-add contractions may differ)."""
    from luna_cpp_b200.line import Line

    n = 300
    x = (np.arange(n) + 0.5) / n
    names = ["sod", "toro-2", "toro-3", "toro-5"]
    keys, order, step, _ = line_keys(x, 1.0)
    states = np.stack([line_state(line_problem(k), keys, step) for k in names])
    batch = Line(x, 1.0, lines=len(names))
    batch.set_state(states)
    singles, separate = [], []
    for k in range(len(names)):
        s = Line(x, 1.0)
        s.set_state(states[k])
        singles.append(s)
        t = Line(x, 1.0)
        t.set_state(states[k])
        separate.append(t)
    dt = batch.time_step(0.8, "luna")
    for _ in range(25):
        fused_next = batch.step_and_time_step(dt, 0.8)
        for k, s in enumerate(singles):
            s.step_and_time_step(dt[k], 0.8)
            separate[k].step(dt[k])
        after = batch.time_step(0.8, "luna")
        assert np.array_equal(fused_next, after)
        dt = after
    got = batch.get_state()
    for k, s in enumerate(singles):
        assert np.array_equal(got[k], s.get_state()[0])
        other = separate[k].get_state()[0]
        assert np.max(np.abs(got[k] - other) / np.abs(other).max(0)) < 1e-13


def test_line_batch_conserves_through_reflective_walls(cuda):
    """A batch of 256 random Riemann problems on 2048-cell lines between reflective walls: mass and energy of every
    line conserved to round-off over 200 steps."""
    from luna_cpp_b200.limiter_training import riemann_problem
    from luna_cpp_b200.line import Line
    from luna_cpp_b200.problems import line_tube

    n, lines = 2048, 256
    x = (np.arange(n) + 0.5) / n
    keys, order, step, _ = line_keys(x, 1.0)
    q0 = []
    for k in range(lines):
        r = riemann_problem(9000 + k)
        p = line_tube((r.rho[0], r.u[0], r.p[0]), (r.rho[1], r.u[1], r.p[1]), t_end=0.2, walls=("reflective", "reflective"))
        q0.append(line_state(p, keys, step))
    q0 = np.stack(q0)
    ln = Line(x, 1.0, walls=("reflective", "reflective"), lines=lines)
    ln.set_state(q0)
    dt = ln.time_step(0.8, "arepo")
    for _ in range(200):
        ln.step(dt)
        dt = ln.time_step(0.8, "arepo")
    q = ln.get_state()
    assert np.all(np.isfinite(q))
    for v in (0, 2):
        assert np.max(np.abs(q[..., v].sum(1) - q0[..., v].sum(1)) / np.abs(q0[..., v]).sum(1)) < 1e-13
