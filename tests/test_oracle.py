"""The CPU oracle against the reference's own known answers (src/test/hydro_test.cpp): LUNA's golden HLL/HLLC fluxes,
the flux invariants, and the mesh invariants of a step. CPU only."""
import json
import os

import numpy as np
import pytest

from conftest import jittered_mesh, random_mesh
from oracle import oracle as O
from luna_cpp_b200.problems import rough_state

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "luna_riemann.json")


def relative(a, b):
    """hydro_test.cpp:25-32: max-norm difference relative to the largest |b|."""
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(b))


@pytest.mark.parametrize("solver", ["hll", "hllc"])
def test_luna_golden_fluxes(solver):
    """hydro_test.cpp:96-104: the solver equals LUNA's on 12 (HLL) / 15 (HLLC) sample faces to 1e-14."""
    g = json.load(open(GOLDEN))
    worst = 0.0
    for c in g[solver]:
        n = np.zeros(3)
        n[c["axis"]] = 1.0
        worst = max(worst, relative(O.riemann(c["L"], c["R"], n, solver=solver), c["F"]))
    assert len(g[solver]) == (12 if solver == "hll" else 15)
    assert worst < 1e-14


def exact_flux(W, n, gamma=5.0 / 3.0):
    U = O.conserved(W, gamma)
    vn = W[1] * n[0] + W[2] * n[1] + W[3] * n[2]
    return np.array([U[0] * vn, U[1] * vn + W[4] * n[0], U[2] * vn + W[4] * n[1], U[3] * vn + W[4] * n[2],
                     (U[4] + W[4]) * vn])


def rotate(v, a):
    angle = np.linalg.norm(a)
    k = a / angle
    return v * np.cos(angle) + np.cross(k, v) * np.sin(angle) + k * (k @ v) * (1 - np.cos(angle))


def rotate_state(s, a):
    return np.concatenate([[s[0]], rotate(np.asarray(s[1:4]), a), [s[4]]])


@pytest.mark.parametrize("solver", ["hll", "hllc"])
def test_flux_invariants(solver):
    """hydro_test.cpp:106-132: consistency, a moving face, symmetry and rotation over random normals."""
    rng = np.random.default_rng(7)
    cons = mov = sym = rot = 0.0
    for _ in range(300):
        n = rng.uniform(-1, 1, 3)
        n /= np.linalg.norm(n)
        w = rng.uniform(-1, 1, 3)
        axis = 3 * rng.uniform(-1, 1, 3)
        L = np.array([1.5 + rng.uniform(-1, 1), *(2 * rng.uniform(-1, 1, 3)), 1.5 + rng.uniform(-1, 1)])
        R = np.array([1.5 + rng.uniform(-1, 1), *(2 * rng.uniform(-1, 1, 3)), 1.5 + rng.uniform(-1, 1)])
        cons = max(cons, relative(O.riemann(L, L, n, solver=solver), exact_flux(L, n)))
        expected = exact_flux(L, n) - (w @ n) * O.conserved(L)
        mov = max(mov, relative(O.riemann(L, L, n, w, solver=solver), expected))
        F = O.riemann(L, R, n, w, solver=solver)
        back = -O.riemann(R, L, -n, w, solver=solver)
        sym = max(sym, relative(F, back))
        turned = O.riemann(rotate_state(L, axis), rotate_state(R, axis), rotate(n, axis), rotate(w, axis), solver=solver)
        rot = max(rot, relative(turned, rotate_state(F, axis)))
    assert cons < 1e-14 and mov < 1e-13 and sym < 1e-14 and rot < 2e-13


def per_volume(fv, mesh):
    return fv.get_state() / mesh.volume[:, None]


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("per_face", [True, False])
@pytest.mark.parametrize("kind", ["jittered", "uniform"])
def test_oracle_uniform_state(order, per_face, kind):
    """hydro_test.cpp:199-213: a uniform state stays uniform over 3 steps (1e-13)."""
    mesh = jittered_mesh(16) if kind == "jittered" else random_mesh(4096)
    W = np.array([1.3, 0.3, -0.2, 0.1, 0.7])
    U = O.conserved(W)
    fv = O.OracleFV(mesh, order=order, per_face=per_face)
    fv.set_state(np.tile(U, (mesh.n_cells, 1)) * mesh.volume[:, None])
    for _ in range(3):
        fv.step(fv.time_step(0.3))
    assert relative(per_volume(fv, mesh), np.tile(U, (mesh.n_cells, 1))) < 1e-13


@pytest.mark.parametrize("order", [0, 1])
def test_oracle_conservation_and_bits(order):
    """hydro_test.cpp:214-254: mass, momentum and energy conserved over 10 steps (1e-14); two runs, the same bits;
    the per-cell and per-face loops agree (on the CPU without contraction: the same bits)."""
    mesh = jittered_mesh(16)
    q0 = rough_state(mesh.n_cells) * mesh.volume[:, None]
    out = []
    for per_face in (True, True, False):
        fv = O.OracleFV(mesh, order=order, per_face=per_face)
        fv.set_state(q0)
        for _ in range(10):
            fv.step(fv.time_step(0.3))
        out.append(fv.get_state())
    before = q0.astype(np.longdouble).sum(0)
    after = out[0].astype(np.longdouble).sum(0)
    scale = float(before[0]) * np.sqrt(float(before[4] / before[0]))
    assert abs(float((after[0] - before[0]) / before[0])) < 1e-14
    assert abs(float((after[4] - before[4]) / before[4])) < 1e-14
    assert np.max(np.abs((after[1:4] - before[1:4]).astype(np.float64))) / scale < 1e-14
    assert np.array_equal(out[0], out[1])
    assert relative(out[2], out[0]) < 1e-12


def test_oracle_float_policy_close_to_double():
    """The riemann32 policy (float gradients, limiter and Riemann solve) stays close to double on a smooth state."""
    mesh = jittered_mesh(16)
    from luna_cpp_b200.problems import acoustic_wave

    q0 = acoustic_wave(mesh, amplitude=1e-2)
    res = {}
    for prec in ("double", "riemann32"):
        fv = O.OracleFV(mesh, precision=prec)
        fv.set_state(q0)
        for _ in range(5):
            fv.step(fv.time_step(0.3))
        res[prec] = fv.get_state()
    rel_l1 = np.abs(res["riemann32"] - res["double"]).sum() / np.abs(res["double"]).sum()
    assert rel_l1 < 1e-5
