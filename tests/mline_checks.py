"""The reference's own checks of the moving 1D line (src/test/hydro1d_test.cpp:121-514), for any implementation of it
(`make(positions, length, **options)`: the oracle's OracleMovingLine or the library's MovingLine): uniform states stay uniform, conservation and the same bits twice, Sod within LUNA's
L1 bounds at AREPO's dt, a split at each wall, supersonic inflow coming out as a lattice, Shu-Osher's budget through
the walls with 1.4-1.55x the cells and no crossing, its mirror image, and no cells where no gas enters."""
import numpy as np
from exact_riemann import ExactRiemann
from luna_cpp_b200.problems import _conserved_1d, line_problem


def points(n, L, jitter, seed):
    """n cell centres on [0, L], each moved by up to jitter / 2 spacings (hydro1d_test.cpp:30-37; seeded numpy)."""
    rng = np.random.default_rng(seed)
    return L * (np.arange(n) + 0.5 + jitter * rng.uniform(-0.5, 0.5, n)) / n


def fill(ml, extensive):
    """Q of each cell from extensive(a, b), its integral over the cell [a, b] (hydro1d_test.cpp:48-60)."""
    g, V, c = ml.geometry()
    a, b = g + c - 0.5 * V, g + c + 0.5 * V
    ml.set_state(extensive(a, b))


def fill_primitives(ml, W, gamma):
    fill(ml, lambda a, b: _conserved_1d(W(0.5 * (a + b)), gamma) * (b - a)[:, None])


def cells(ml, gamma):
    """Per cell the centre, the length and W (hydro1d_test.cpp:73-86)."""
    g, V, c = ml.geometry()
    U = ml.get_state() / V[:, None]
    rho = U[:, 0]
    v = U[:, 1] / rho
    return g + c, V, np.stack([rho, v, (gamma - 1) * (U[:, 2] - 0.5 * rho * v * v)], 1)


def run(ml, t_end, courant, rule):
    t, steps = 0.0, 0
    while t < t_end * (1 - 1e-12):
        dt = min(ml.time_step(courant, rule), t_end - t)
        ml.step(dt)
        t += dt
        steps += 1
    return steps


def problem_line(make, name, n, moving_walls=False, mirrored=False):
    pr = line_problem(name)
    walls, inflow = pr["walls"], None
    if moving_walls and "moving_walls" in pr:
        walls, inflow = pr["moving_walls"], np.array(pr["moving_inflow"])
    if mirrored:
        walls = walls[::-1]
    ml = make(points(n, pr["L"], 0.0, 1), pr["L"], gamma=pr["gamma"], walls=walls, inflow=inflow)
    L, o = pr["L"], pr["origin"]

    def extensive(a, b):
        if mirrored:
            U = pr["average"](L - b + o, L - a + o)
            U = U * np.array([1.0, -1.0, 1.0])
        else:
            U = pr["average"](a + o, b + o)
        return U * (b - a)[:, None]

    fill(ml, extensive)
    return ml, pr


def uniform_states_stay_uniform(make, order):
    """hydro1d_test.cpp:124-156: a uniform state with a bulk velocity on a jittered periodic line, and one at rest between
    reflective walls (HLL), stay uniform to 1e-13 over 20 steps."""
    ml = make(points(200, 1.0, 0.8, 1), 1.0, gamma=1.4, periodic=True, order=order)
    W = np.array([1.3, 0.7, 0.4])
    fill_primitives(ml, lambda x: np.tile(W[:, None], (1, len(x))), 1.4)
    for _ in range(20):
        ml.step(ml.time_step(0.3))
    assert np.max(np.abs(cells(ml, 1.4)[2] - W) / np.abs(W)) < 1e-13
    ml = make(points(200, 2.0, 0.8, 2), 2.0, gamma=1.4, walls=("reflective", "reflective"), order=order, riemann="hll")
    W = np.array([0.8, 0.0, 2.0])
    fill_primitives(ml, lambda x: np.tile(W[:, None], (1, len(x))), 1.4)
    for _ in range(20):
        ml.step(ml.time_step(0.3))
    Wc = cells(ml, 1.4)[2]
    worst = max(np.max(np.abs(Wc[:, 0] - W[0]) / W[0]), np.max(np.abs(Wc[:, 2] - W[2]) / W[2]),
                np.max(np.abs(Wc[:, 1]) / np.sqrt(1.4 * W[2] / W[0])))
    assert worst < 1e-13


def conservation_and_same_bits(make, periodic):
    """hydro1d_test.cpp:159-212: a rough state with a blast in the middle, 40 steps: mass and energy to 1e-14 (and momentum
    on the periodic line), two identical runs give the same bits, states and positions."""
    rng = np.random.default_rng(5)
    table = np.stack([1 + 0.3 * rng.uniform(-1, 1, 300), 0.5 * rng.uniform(-1, 1, 300), 1 + 0.3 * rng.uniform(-1, 1, 300)], 1)

    def extensive(a, b):
        k = np.minimum(299, (150 * (a + b)).astype(int))
        W = table[k].copy()
        W[np.abs(0.5 * (a + b) - 1.0) < 0.1, 2] *= 100
        return _conserved_1d(W.T, 1.4) * (b - a)[:, None]

    runs = []
    for _ in range(2):
        ml = make(points(300, 2.0, 0.8, 3), 2.0, gamma=1.4, periodic=periodic, walls=("reflective", "reflective"))
        fill(ml, extensive)
        before = ml.get_state().sum(0)
        for _ in range(40):
            ml.step(ml.time_step(0.3))
        after = ml.get_state().sum(0)
        runs.append((ml.get_state(), ml.positions()))
    assert abs(after[0] - before[0]) / before[0] < 1e-14 and abs(after[2] - before[2]) / before[2] < 1e-14
    if periodic:
        assert abs(after[1] - before[1]) / np.sqrt(2 * before[0] * before[2]) < 1e-14
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])


def sod_within_luna_bounds(make, n, bounds, jitter):
    """hydro1d_test.cpp:229-264, moving: Sod at AREPO's dt (courant 0.4) to t = 0.25 within LUNA's L1 bounds of the exact
    cell averages."""
    sod = ExactRiemann((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 1.4)
    ml = make(points(n, 1.0, jitter, 6), 1.0, gamma=1.4)

    def extensive(a, b):
        W = np.array([sod.average(lo, hi, 0.5, 1e-12) for lo, hi in zip(a, b)])
        return _conserved_1d(W.T, 1.4) * (b - a)[:, None]

    fill(ml, extensive)
    run(ml, 0.25, 0.4, "arepo")
    x, V, W = cells(ml, 1.4)
    exact = np.array([sod.average(c - 0.5 * v, c + 0.5 * v, 0.5, 0.25) for c, v in zip(x, V)])
    l1 = (V[:, None] * np.abs(W - exact)).sum(0)
    assert np.all(l1 <= np.array(bounds)), l1


def a_split_at_each_wall(make):
    """hydro1d_test.cpp:368-395: 16 points in [0.4, 0.7], spacing 0.04: one call adds a cell at each wall; the totals
    move by < 1e-15 and both halves of each split keep the old state to 1e-14."""
    x = 0.4 + 0.02 * np.arange(16)
    ml = make(x, 1.0, gamma=1.4)
    ml.set_inflow_spacing(0.04)
    fill_primitives(ml, lambda y: np.stack([1.0 + 0.5 * np.sin(9 * y), 0.3 - y, 2.0 + np.cos(7 * y)]), 1.4)
    before, totals = cells(ml, 1.4)[2], ml.get_state().sum(0)
    assert ml.supply_cells() == 2 and ml.n == 18
    after = cells(ml, 1.4)[2]
    assert np.max(np.abs(ml.get_state().sum(0) - totals) / np.abs(totals)) < 1e-15
    # the first cell (id 0) and the new left cell (id 16) keep cell 0's state; the last old cell (15) and id 17 its own
    for new, old in ((16, 0), (0, 0), (17, 15), (15, 15)):
        assert np.max(np.abs(after[new] / before[old] - 1)) < 1e-14


def supersonic_inflow_makes_a_lattice(make, from_left):
    """hydro1d_test.cpp:397-423: supersonic inflow into gas at rest, to t = 0.1 at AREPO's dt: more than 30 cells added,
    the gas behind the entering state stays itself to 1e-12, the new cells a lattice of the set spacing to 1e-9, no
    crossing."""
    n = 128
    inflow_state = np.array([2.0, 3.0 if from_left else -3.0, 1.0])
    rest = np.array([0.5, 0.0, 0.2])
    walls = ["outflow", "outflow"]
    inflow = np.zeros((2, 3))
    walls[0 if from_left else 1] = "inflow"
    inflow[0 if from_left else 1] = inflow_state
    ml = make(points(n, 1.0, 0.0, 4), 1.0, gamma=1.4, walls=tuple(walls), inflow=inflow)
    near = (lambda x: x) if from_left else (lambda x: 1.0 - x)
    fill_primitives(ml, lambda x: np.where(near(x)[None, :] < 0.5, inflow_state[:, None], rest[:, None]), 1.4)
    run(ml, 0.1, 0.4, "arepo")
    x, V, W = cells(ml, 1.4)
    keep = near(x) <= 0.3
    worst = np.max(np.abs(W[keep] - inflow_state) / np.abs(inflow_state))
    xs = np.sort(x[keep])
    uneven = np.max(np.abs(np.diff(xs)[2:-2] - 1.0 / n) * n)
    assert ml.n > n + 30 and worst < 1e-12 and uneven < 1e-9 and ml.stats()["sorts"] == 0, (ml.n, worst, uneven)


def shu_osher_budget_cells_and_mirror(make):
    """hydro1d_test.cpp:425-477: Shu-Osher at N = 512 on the moving line (AREPO's dt, 0.4): the totals follow the budget
    through the walls (1e-11 with a zero-gradient wall, 1e-12 with the inflow wall holding the state), 1.4-1.55x the cells,
    no crossing; a second run gives the same bits; the mirrored problem gives the mirrored result to 1e-9."""
    rhoL, uL, pL, pR, g = 3.857143, 2.629369, 10.33333, 1.0, 1.4
    EL = pL / (g - 1) + 0.5 * rhoL * uL * uL
    ends = []
    for pass_ in range(4):
        mirrored, fixed = pass_ == 2, pass_ == 3
        ml, pr = problem_line(make, "shu-osher", 512, moving_walls=fixed, mirrored=mirrored)
        start = ml.get_state().sum(0)
        run(ml, pr["t_end"], 0.4, "arepo")
        end = ml.get_state().sum(0)
        if not mirrored:
            T = pr["t_end"]
            expected = np.array([rhoL * uL * T, (rhoL * uL * uL + pL - pR) * T, (EL + pL) * uL * T])
            assert np.max(np.abs((end - start) - expected) / expected) < (1e-12 if fixed else 1e-11)
            assert 1.4 * 512 < ml.n < 1.55 * 512
            assert ml.stats()["sorts"] == 0
        if not fixed:
            ends.append(cells(ml, g))
    assert len(ends[0][0]) == len(ends[1][0]) and all(np.array_equal(a, b) for a, b in zip(ends[0], ends[1]))
    a, b = ends[0], ends[2]
    assert len(a[0]) == len(b[0])
    ia, ib = np.argsort(a[0]), np.argsort(-b[0])
    Wa, Wb = a[2][ia], b[2][ib]
    worst = max(np.max(np.abs(Wa[:, 0] - Wb[:, 0])), np.max(np.abs(Wa[:, 1] + Wb[:, 1])), np.max(np.abs(Wa[:, 2] - Wb[:, 2])))
    assert worst < 1e-9, worst


def fused_step_conserves_and_is_close(make):
    """hydro1d_test.cpp:298-343, moving: the fused step (LUNA's rule at 0.8) over 60 steps conserves mass and energy to
    1e-14, gives the same bits twice, and stays within 1.5e-3 of time_step() + step() (its next dt takes w - v of t^n)."""
    for periodic in (True, False):
        def rough(ml):
            fill(ml, lambda a, b: _conserved_1d(np.stack([1.0 + 0.3 * np.sin(9 * (0.5 * (a + b))), 0.4 * np.cos(5 * (0.5 * (a + b))),
                                                          np.where(np.abs(0.5 * (a + b) - 1) < 0.1, 20.0, 1.0)]), 1.4) * (b - a)[:, None])

        def line():
            ml = make(points(400, 2.0, 0.5, 8), 2.0, gamma=1.4, periodic=periodic, walls=("reflective", "reflective"))
            rough(ml)
            return ml

        split, fused, again = line(), line(), line()
        before = fused.get_state().sum(0)
        for _ in range(60):
            split.step(split.time_step(0.8, "luna"))
        for ml in (fused, again):
            dt = ml.time_step(0.8, "luna")
            for _ in range(60):
                dt = ml.step_and_time_step(dt, 0.8)
        after = fused.get_state().sum(0)
        assert np.array_equal(fused.get_state(), again.get_state())
        assert abs(after[0] - before[0]) / before[0] < 1e-14 and abs(after[2] - before[2]) / before[2] < 1e-14
        assert np.max(np.abs(split.get_state() - fused.get_state())) < 1.5e-3


def no_cells_where_no_gas_enters(make, name):
    """hydro1d_test.cpp:498-512: Sod and Woodward-Colella on 256 moving cells keep their count."""
    ml, pr = problem_line(make, name, 256)
    run(ml, pr["t_end"], 0.4, "arepo")
    assert ml.n == 256 and ml.stats()["cells_added"] == 0
