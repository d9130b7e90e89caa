"""The fused flux-and-update pass of the static FP64 step (geometry.cuh::k_tile_flux_update: a tile's interior faces
solved into shared memory, the faces between tiles by their own pass; LUNA_FUSED_STEP=1) against the two-kernel pass
(k_flux_rows then k_update, the default): the same fluxes summed in the same list order, so the same bits, the same
fallback count and the same dt; and a step that leaves the fused pass (the learned limiter's mode) after fused steps."""
import os

import numpy as np
import pytest

from conftest import jittered_mesh
from luna_cpp_b200 import hydro
from luna_cpp_b200.problems import point_blast, rough_state

pytestmark = pytest.mark.gpu


def run(mesh, q0, steps, fused, **kw):
    old = os.environ.get("LUNA_FUSED_STEP")
    os.environ["LUNA_FUSED_STEP"] = "1" if fused else "0"
    try:
        fv = hydro.FiniteVolume(mesh, **kw)
        fv.set_state(q0)
        dts, falls = [], []
        for _ in range(steps):
            dt = fv.time_step(0.3)
            fv.step(dt)
            dts.append(dt)
            falls.append(fv.fallbacks())
        assert fv.fused_pass()[0] == fused
        out = fv.get_state(), dts, falls, fv.device_bytes()
        fv.close()
        return out
    finally:
        if old is None:
            del os.environ["LUNA_FUSED_STEP"]
        else:
            os.environ["LUNA_FUSED_STEP"] = old


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("riemann", ["hllc", "hll"])
def test_fused_step_equals_two_kernel_step(cuda, dim, riemann):
    if dim == 3:
        mesh = jittered_mesh(20)
        q0 = point_blast(mesh, radius_cells=3.0)
    else:
        mesh = jittered_mesh(96, dim=2, jitter=0.3, seed=4)
        q0 = rough_state(mesh.n_cells, dim=2) * mesh.volume[:, None]
    a, dta, fa, bytes_a = run(mesh, q0, 6, True, riemann=riemann)
    b, dtb, fb, bytes_b = run(mesh, q0, 6, False, riemann=riemann)
    assert dta == dtb
    assert fa == fb
    assert a.tobytes() == b.tobytes()
    assert bytes_a < bytes_b  # the fused pass keeps no flux row of an interior face


def test_leaving_the_fused_pass(cuda):
    """Fused steps, then steps with the plain limiter in the learned path's min-factor form (the two-kernel pass, whose
    face and flux rows the fused pass had released), then fused again: the same bits as a run that never fused."""
    mesh = jittered_mesh(16)
    q0 = rough_state(mesh.n_cells) * mesh.volume[:, None]
    states = []
    for fused in (True, False):
        os.environ["LUNA_FUSED_STEP"] = "1" if fused else "0"
        try:
            fv = hydro.FiniteVolume(mesh)
            fv.set_state(q0)
            for k in range(6):
                fv.set_limiter("factors" if k in (2, 3) else "plain")
                fv.step(fv.time_step(0.3))
            states.append(fv.get_state())
            fv.close()
        finally:
            del os.environ["LUNA_FUSED_STEP"]
    assert states[0].tobytes() == states[1].tobytes()
