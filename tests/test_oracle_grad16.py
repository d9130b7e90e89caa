"""The oracle's Grad16 policy (FP16 gradient rows with one power-of-two exponent per group rho, v, P;
src/hydro/finite_volume.hpp:616-641, precision.hpp half::) against numpy's IEEE binary16 rounding, on the CPU."""
import numpy as np
import pytest

from conftest import jittered_mesh
from luna_cpp_b200.problems import rough_state
from oracle import oracle as O


def numpy_half_round_trip(g, D):
    """The same encoding in numpy: per cell and group, k = clamp(14 - floor(log2 max|g|), -114, 126) (0 for a zero group),
    float32(g 2^k) -> float16 (round to nearest even) -> float32, times 2^-k."""
    g = g.astype(np.float32)
    V = D + 2
    groups = np.array([0 if c < D else 1 if c < D + D * D else 2 for c in range(V * D)])
    out = np.empty_like(g)
    for s in range(3):
        cols = groups == s
        m = np.abs(g[:, cols]).max(axis=1)
        e = ((m.view(np.uint32) >> 23) & 0xFF).astype(np.int64) - 127
        k = np.where(m > 0, np.clip(14 - e, -114, 126), 0)
        scale = np.ldexp(np.float32(1), k).astype(np.float32)[:, None]
        inv = np.ldexp(np.float32(1), -k).astype(np.float32)[:, None]
        out[:, cols] = (g[:, cols] * scale).astype(np.float16).astype(np.float32) * inv
    return out


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_grad16_rounds_the_grad32_gradients(dim):
    mesh = jittered_mesh(10 if dim == 3 else 24, dim=dim)
    q0 = rough_state(mesh.n_cells, dim=dim) * mesh.volume[:, None]
    g32 = O.OracleFV(mesh, precision="grad32")
    g32.set_state(q0)
    g32.time_step(0.3)
    g16 = O.OracleFV(mesh, precision="grad16")
    g16.set_state(q0)
    g16.time_step(0.3)
    want = numpy_half_round_trip(g32.gradients(), dim)
    got = g16.gradients()
    assert np.array_equal(got.astype(np.float32), want)
    rel = np.abs(got - g32.gradients()) / (np.abs(g32.gradients()).max(axis=0) + 1e-300)
    assert rel.max() < 2.0 ** -10  # binary16 keeps 11 bits of the largest component of each group


def test_oracle_grad16_step_conserves_and_stays_close_to_grad32():
    mesh = jittered_mesh(10)
    q0 = rough_state(mesh.n_cells) * mesh.volume[:, None]
    runs = {}
    for p in ("grad32", "grad16"):
        fv = O.OracleFV(mesh, precision=p)
        fv.set_state(q0)
        for _ in range(5):
            fv.step(fv.time_step(0.3))
        runs[p] = fv.get_state()
    assert abs(runs["grad16"][:, 0].sum() - q0[:, 0].sum()) < 1e-13 * q0[:, 0].sum()
    assert np.abs(runs["grad16"] - runs["grad32"]).sum() / np.abs(runs["grad32"]).sum() < 1e-3
