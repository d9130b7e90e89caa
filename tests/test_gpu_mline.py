"""The moving 1D line on the GPU (luna_mline_*, FiniteVolume<1> with Motion::moving, finite_volume_1d.hpp): step for step
against the CPU oracle (oracle/oracle_mline.c) — the same positions bit for bit, the same cells added, Q to 1e-12 —
and the reference's own moving-line checks (hydro1d_test.cpp:121-514, tests/mline_checks.py) on the GPU's runs."""
import numpy as np
import pytest

import mline_checks as C
from luna_cpp_b200.problems import _conserved_1d
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def gpu_line(*args, **kw):
    from luna_cpp_b200.line import MovingLine

    return MovingLine(*args, **kw)


def rough_extensive(a, b):
    m = 0.5 * (a + b)
    W = np.stack([1.0 + 0.3 * np.sin(9 * m), 0.4 * np.cos(5 * m), np.where(np.abs(m - 1) < 0.1, 20.0, 1.0)])
    return _conserved_1d(W, 1.4) * (b - a)[:, None]


def same(gpu, ref, what):
    """The two lines hold the same cells: positions bit for bit, Q within 1e-12 of each field's largest."""
    assert gpu.n == ref.n, (what, gpu.n, ref.n)
    assert np.array_equal(gpu.positions(), ref.positions()), what
    g, r = gpu.get_state(), ref.get_state()
    scale = np.abs(r).max(0)
    err = float(np.max(np.abs(g - r) / scale))
    assert err <= 1e-12, (what, err)
    return err


CASES = [
    # (name, options, steps, courant, rule)
    ("periodic order 1 HLLC", dict(periodic=True), 60, 0.4, "arepo"),
    ("periodic order 0 HLL", dict(periodic=True, order=0, riemann="hll"), 40, 0.4, "arepo"),
    ("reflective order 1 minmod", dict(walls=("reflective", "reflective"), limiter="minmod"), 40, 0.8, "luna"),
    ("outflow order 1 van Leer, no regularisation", dict(limiter="van_leer", regularise=False), 40, 0.4, "arepo"),
    ("reflective/outflow order 1 no limiter", dict(walls=("reflective", "outflow"), limiter="none"), 40, 0.4, "arepo"),
]


@pytest.mark.parametrize("name,options,steps,courant,rule", CASES, ids=[c[0] for c in CASES])
def test_moving_line_equals_oracle(cuda, name, options, steps, courant, rule):
    """A rough state with a blast on a jittered line of 400 cells on [0, 2]: each step's dt (time_step) within 1e-13, and
    after the steps the same cells, positions and Q as the oracle's."""
    x = C.points(400, 2.0, 0.5, 8)
    gpu, ref = gpu_line(x, 2.0, gamma=1.4, **options), O.OracleMovingLine(x, 2.0, gamma=1.4, **options)
    for ml in (gpu, ref):
        C.fill(ml, rough_extensive)
    for _ in range(steps):
        dg, dr = float(gpu.time_step(courant, rule)[0]), ref.time_step(courant, rule)
        assert abs(dg - dr) <= 1e-13 * dr
        gpu.step(dr)
        ref.step(dr)
    err = same(gpu, ref, name)
    print(f"{name}: Q within {err:.1e} of the oracle's")
    gpu.close()


def test_moving_line_fused_equals_oracle(cuda):
    """step_and_time_step (one launch: the step, the next dt of LUNA's rule) against the oracle's over 60 steps: the same
    dt sequence to 1e-13, cells and Q."""
    x = C.points(400, 2.0, 0.5, 8)
    for periodic in (True, False):
        opts = dict(periodic=periodic, walls=("reflective", "reflective"))
        gpu, ref = gpu_line(x, 2.0, gamma=1.4, **opts), O.OracleMovingLine(x, 2.0, gamma=1.4, **opts)
        for ml in (gpu, ref):
            C.fill(ml, rough_extensive)
        dg, dr = float(gpu.time_step(0.8, "luna")[0]), ref.time_step(0.8, "luna")
        for _ in range(60):
            assert abs(dg - dr) <= 1e-13 * dr
            dg, dr = float(gpu.step_and_time_step(dr, 0.8)[0]), ref.step_and_time_step(dr, 0.8)
        same(gpu, ref, f"fused, periodic={periodic}")
        gpu.close()


@pytest.mark.parametrize("fixed", [False, True])
def test_shu_osher_with_cells_from_the_wall_equals_oracle(cuda, fixed):
    """Shu-Osher on 512 moving cells to t = 1.8 (AREPO's dt, 0.4): the left wall supplies about 240 cells; the GPU adds
    the same cells at the same steps as the oracle and ends with the same positions and Q; with the zero-gradient wall
    and with the inflow wall holding the state."""
    gpu, pr = C.problem_line(gpu_line, "shu-osher", 512, moving_walls=fixed)
    ref, _ = C.problem_line(O.OracleMovingLine, "shu-osher", 512, moving_walls=fixed)
    t, steps = 0.0, 0
    while t < pr["t_end"] * (1 - 1e-12):
        dt = min(ref.time_step(0.4, "arepo"), pr["t_end"] - t)
        dg = float(gpu.time_step(0.4, "arepo")[0])
        assert abs(min(dg, pr["t_end"] - t) - dt) <= 1e-13 * dt, steps
        gpu.step(dt)
        ref.step(dt)
        t += dt
        steps += 1
        if steps % 500 == 0:
            assert gpu.n == ref.n, steps
    assert gpu.stats() == ref.stats()
    err = same(gpu, ref, "shu-osher")
    print(f"Shu-Osher ({'inflow' if fixed else 'zero-gradient'} wall): {steps} steps, {gpu.n} cells, Q within {err:.1e}")
    gpu.close()


def test_points_that_cross_are_sorted(cuda):
    """Two points driven through each other (unregularised, order 0, a step of twice their meeting time on a periodic line
    of 16): the GPU re-sorts its slots by (key, cell) as the oracle does, and the two lines stay equal over the next
    steps."""
    n = 16
    x = (np.arange(n) + 0.5) / n
    opts = dict(periodic=True, regularise=False, order=0)
    gpu, ref = gpu_line(x, 1.0, gamma=1.4, **opts), O.OracleMovingLine(x, 1.0, gamma=1.4, **opts)
    v = np.zeros(n)
    v[7], v[8] = 1.0, -1.0
    W = np.stack([np.ones(n), v, 0.01 * np.ones(n)])
    for ml in (gpu, ref):
        _, V, _ = ml.geometry()
        ml.set_state(_conserved_1d(W, 1.4) * V[:, None])
        ml.step(0.04)
        ml.step(0.001)
        ml.step(0.001)
    assert ref.stats()["sorts"] >= 1 and gpu.stats() == ref.stats()
    same(gpu, ref, "crossing")
    gpu.close()


# The reference's checks on the GPU's runs (tests/mline_checks.py).
@pytest.mark.parametrize("order", [0, 1])
def test_uniform_states_stay_uniform(cuda, order):
    C.uniform_states_stay_uniform(gpu_line, order)


@pytest.mark.parametrize("periodic", [True, False])
def test_conservation_and_same_bits(cuda, periodic):
    C.conservation_and_same_bits(gpu_line, periodic)


@pytest.mark.parametrize("n,bounds", [(128, (0.0063, 0.0097, 0.0047)), (256, (0.0034, 0.0046, 0.0023))])
def test_sod_within_luna_bounds(cuda, n, bounds):
    C.sod_within_luna_bounds(gpu_line, n, bounds, 0.5)


def test_a_split_at_each_wall(cuda):
    C.a_split_at_each_wall(gpu_line)


@pytest.mark.parametrize("from_left", [True, False])
def test_supersonic_inflow_makes_a_lattice(cuda, from_left):
    C.supersonic_inflow_makes_a_lattice(gpu_line, from_left)


def test_shu_osher_budget_cells_and_mirror(cuda):
    C.shu_osher_budget_cells_and_mirror(gpu_line)


def test_fused_step_conserves_and_is_close(cuda):
    C.fused_step_conserves_and_is_close(gpu_line)


@pytest.mark.parametrize("name", ["sod", "woodward-colella"])
def test_no_cells_where_no_gas_enters(cuda, name):
    C.no_cells_where_no_gas_enters(gpu_line, name)


def test_moving_line_arguments(cuda):
    """The C ABI refuses what the reference refuses: fewer than 3 cells, an unknown wall, an inflow wall without its
    state, a non-positive dt."""
    from luna_cpp_b200.hydro import LunaError

    with pytest.raises(LunaError):
        gpu_line([0.2, 0.6], 1.0)
    with pytest.raises(LunaError):
        gpu_line(C.points(8, 1.0, 0.0, 1), 1.0, walls=("inflow", "outflow"))
    ml = gpu_line(C.points(8, 1.0, 0.0, 1), 1.0)
    C.fill(ml, lambda a, b: _conserved_1d(np.stack([1 + 0 * a, 0 * a, 1 + 0 * a]), 1.4) * (b - a)[:, None])
    with pytest.raises(LunaError):
        ml.step(0.0)
    ml.close()
