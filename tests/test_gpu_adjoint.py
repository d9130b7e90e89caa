"""The hand-written adjoint kernels (through the C ABI) against the oracle's restatement of the reference's
step_adjoint, and the checkpointed rollout gradient against central finite differences of the same map (fixed dt
schedule, h = 1e-6)."""
import numpy as np
import pytest

from conftest import jittered_mesh
from oracle import oracle as O
from luna_cpp_b200 import hydro
from luna_cpp_b200.problems import rough_state, shear_layer

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("riemann", ["hllc", "hll"])
@pytest.mark.parametrize("limiter", ["face_centroid", "none"])
def test_step_adjoint_matches_oracle(cuda, dim, riemann, limiter):
    mesh = jittered_mesh(32 if dim == 2 else 12, dim=dim)
    q0 = rough_state(mesh.n_cells, dim=dim) * mesh.volume[:, None]
    ora = O.OracleFV(mesh, riemann=riemann, limiter=limiter)
    ora.set_state(q0)
    dt = ora.time_step(0.3)
    qbar = np.random.default_rng(1).standard_normal(q0.shape)
    want = ora.step_adjoint(dt, qbar)
    gpu = hydro.FiniteVolume(mesh, riemann=riemann, limiter=limiter)
    gpu.set_state(q0)
    got = gpu.step_adjoint(dt, qbar)
    again = gpu.step_adjoint(dt, qbar)
    assert np.array_equal(got, again)
    assert np.max(np.abs(got - want)) / np.max(np.abs(want)) < 1e-11
    # Q is left as it was
    assert np.array_equal(gpu.get_state(), q0)


def test_adjoint_requires_fp64_static_order1(cuda):
    mesh = jittered_mesh(8)
    fv = hydro.FiniteVolume(mesh, precision="fp32")
    with pytest.raises(hydro.LunaError):
        fv.step_adjoint(1e-3, np.zeros((mesh.n_cells, 5)))


def test_rollout_gradient_against_central_differences(cuda):
    """The adjoint configuration scaled down: 2D shear layer on a 48^2 jittered mesh, 24 steps with checkpoints every 5,
    objective int rho vy^2 dA; d/d a_k by the adjoint against central differences (h = 1e-6) at the same dt schedule."""
    import torch

    from luna_cpp_b200.autograd import kinetic_y, last_dts, rollout, shear_layer_torch
    from luna_cpp_b200.problems import cell_centres

    mesh = jittered_mesh(48, dim=2)
    dev = torch.device("cuda")
    centres = torch.tensor(cell_centres(mesh), device=dev)
    volume = torch.tensor(mesh.volume, device=dev)
    a = torch.tensor(np.random.default_rng(2).standard_normal(8), device=dev, requires_grad=True)
    fv = hydro.FiniteVolume(mesh)
    q0 = shear_layer_torch(centres, volume, a)
    assert np.allclose(q0.detach().cpu().numpy(), shear_layer(mesh, a.detach().cpu().numpy()), rtol=1e-13, atol=1e-16)
    out = rollout(q0, fv, 24, every=5)
    dts = last_dts(out)
    J = kinetic_y(out)
    J.backward()
    grad = a.grad.detach().cpu().numpy()
    h = 1e-6
    fd = np.zeros(8)
    with torch.no_grad():
        for k in range(8):
            e = torch.zeros(8, dtype=torch.float64, device=dev)
            e[k] = h
            jp = kinetic_y(rollout(shear_layer_torch(centres, volume, a + e), fv, 24, every=5, dts=dts))
            jm = kinetic_y(rollout(shear_layer_torch(centres, volume, a - e), fv, 24, every=5, dts=dts))
            fd[k] = (jp - jm).item() / (2 * h)
    assert np.max(np.abs(grad - fd)) / np.max(np.abs(fd)) < 1e-4


def test_adjoint_config_512_against_oracle(cuda):
    """The adjoint configuration: 2D shear layer (a_k ~ N(0, 1)) on a 512^2 jittered mesh, 200 steps, objective
    J = int rho vy^2 dA. The GPU's step adjoint chained over the 200 steps against the oracle's restatement of the
    reference's step_adjoint, both applied at the oracle's states on its dt schedule, compared as dJ/da_k (Qbar^0
    contracted with dQ^0/da_k): relative difference <= 1e-7. Qbar^0 itself is not compared cell by cell: the layer's
    uniform regions put many cells exactly on limiter kinks (a clip whose factor is 1 to within round-off), where the
    step is continuous but not differentiable and round-off (FMA contraction on the GPU, none in the oracle) picks
    which one-sided derivative a cell's Qbar gets; along the configuration's own parameters both agree. The
    checkpointed rollout is checked against central differences (test_rollout_gradient_against_central_differences;
    at this size luna_cpp_b200.studies.adjoint measures ~1e-9)."""
    from luna_cpp_b200.problems import cell_centres

    mesh = jittered_mesh(512, dim=2)
    a = np.random.default_rng(3).standard_normal(8)
    q0 = shear_layer(mesh, a)
    ora = O.OracleFV(mesh)
    ora.set_state(q0)
    states, dts = [], []
    for _ in range(200):
        states.append(ora.get_state())
        dt = ora.time_step(0.3)
        ora.step(dt)
        dts.append(dt)
    q = ora.get_state()
    qbar = np.zeros_like(q)  # d/dQ of sum Q_my^2 / Q_m
    qbar[:, 0] = -(q[:, 2] / q[:, 0]) ** 2
    qbar[:, 2] = 2 * q[:, 2] / q[:, 0]
    want, got = qbar.copy(), qbar.copy()
    fv = hydro.FiniteVolume(mesh)
    for s in reversed(range(200)):
        ora.set_state(states[s])
        want = ora.step_adjoint(dts[s], want)
        fv.set_state(states[s])
        got = fv.step_adjoint(dts[s], got)
    # dQ^0/da_k: rho vy = rho 0.01 sum a_k sin(2 pi k x) and E = ... + rho vy^2 / 2, per unit volume
    x = cell_centres(mesh)[:, 0]
    rho = q0[:, 0] / mesh.volume
    vy = q0[:, 2] / q0[:, 0]
    basis = 0.01 * np.sin(2 * np.pi * np.arange(1, 9)[None, :] * x[:, None])  # d vy / d a_k
    dq_my = rho[:, None] * basis * mesh.volume[:, None]
    dq_e = rho[:, None] * vy[:, None] * basis * mesh.volume[:, None]
    grad_oracle = want[:, 2] @ dq_my + want[:, 3] @ dq_e
    grad_gpu = got[:, 2] @ dq_my + got[:, 3] @ dq_e
    assert np.max(np.abs(grad_gpu - grad_oracle)) / np.max(np.abs(grad_oracle)) < 1e-7
