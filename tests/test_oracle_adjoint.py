"""The oracle's adjoint of one static step (step_adjoint, finite_volume.hpp:2201-2231) against central finite differences
of its own forward step at fixed dt, on states without ties between neighbours (the limiter's min/max is not
differentiable at a tie; the reference's tests keep only samples whose branch pattern is the same at x +- h)."""
import numpy as np
import pytest

from conftest import jittered_mesh
from oracle import oracle as O
from luna_cpp_b200.problems import acoustic_wave, rough_state


def fd_check(mesh, q0, limiter="face_centroid", riemann="hllc", h=1e-5, trials=3, seed=0):
    fv = O.OracleFV(mesh, limiter=limiter, riemann=riemann)
    fv.set_state(q0)
    dt = fv.time_step(0.3)

    def step(q):
        f = O.OracleFV(mesh, limiter=limiter, riemann=riemann)
        f.set_state(q)
        f.time_step(0.3)
        f.step(dt)
        return f.get_state()

    rng = np.random.default_rng(seed)
    qbar = rng.standard_normal(q0.shape)
    adj = O.OracleFV(mesh, limiter=limiter, riemann=riemann)
    adj.set_state(q0)
    qb0 = adj.step_adjoint(dt, qbar)
    errs = []
    for _ in range(trials):
        dq = rng.standard_normal(q0.shape) * np.abs(q0) * 1e-3
        fd = (step(q0 + h * dq) - step(q0 - h * dq)) / (2 * h)
        lhs, rhs = np.sum(qbar * fd), np.sum(qb0 * dq)
        errs.append(abs(lhs - rhs) / abs(rhs))
    return max(errs)


@pytest.mark.parametrize("riemann", ["hllc", "hll"])
@pytest.mark.parametrize("limiter", ["face_centroid", "none"])
def test_adjoint_against_central_differences_2d(riemann, limiter):
    mesh = jittered_mesh(16, dim=2)
    q0 = rough_state(mesh.n_cells, dim=2) * mesh.volume[:, None]
    assert fd_check(mesh, q0, limiter, riemann) < 1e-6


def test_adjoint_against_central_differences_3d():
    mesh = jittered_mesh(8)
    q0 = rough_state(mesh.n_cells) * mesh.volume[:, None]
    assert fd_check(mesh, q0) < 1e-6


def test_adjoint_smooth_wave():
    mesh = jittered_mesh(16, dim=2)
    q0 = acoustic_wave(mesh, amplitude=1e-2)
    assert fd_check(mesh, q0, trials=2) < 1e-6
