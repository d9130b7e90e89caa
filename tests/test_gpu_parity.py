"""Parity of the CUDA path (through the C ABI) with the CPU oracle on the same meshes and states, plus the reference's
mesh invariants (src/test/hydro_test.cpp) on the GPU. Tolerances: FP64 one step 1e-13 relative (max norm), 50 steps of
the 32^3 blast 1e-12 relative L1 per conserved field; the FP32 policy against the oracle's same policy 1e-6 relative
(max norm) after one step; conservation 1e-14; bits equal run to run."""
import numpy as np
import pytest

from conftest import jittered_mesh, random_mesh
from oracle import oracle as O
from luna_cpp_b200 import hydro
from luna_cpp_b200.problems import acoustic_wave, point_blast, rough_state, shear_layer

pytestmark = pytest.mark.gpu


def relative(a, b):
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / scale) if scale > 0 else float(np.max(np.abs(a - b)))


def rel_l1(a, b):
    return np.abs(a - b).sum(0) / np.abs(b).sum(0)


def pair(mesh, q0, **kw):
    prec = kw.pop("precision", "fp64")
    gpu = hydro.FiniteVolume(mesh, precision=prec, **kw)
    ora = O.OracleFV(mesh, order=kw.get("order", 1), per_face=kw.get("update", "per_face") == "per_face",
                     limiter=kw.get("limiter", "face_centroid"), riemann=kw.get("riemann", "hllc"),
                     moving=kw.get("motion", "static_mesh") == "moving",
                     precision={"fp32": "riemann32", "grad32": "grad32", "grad16": "grad16", "single": "single"}.get(prec, "double"))
    gpu.set_state(q0)
    ora.set_state(q0)
    return gpu, ora


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("update", ["per_face", "per_cell"])
@pytest.mark.parametrize("riemann", ["hllc", "hll"])
def test_one_step_fp64(cuda, order, update, riemann):
    mesh = jittered_mesh(16)
    q0 = rough_state(mesh.n_cells) * mesh.volume[:, None]
    gpu, ora = pair(mesh, q0, order=order, update=update, riemann=riemann)
    dt_g, dt_o = gpu.time_step(0.3), ora.time_step(0.3)
    assert abs(dt_g - dt_o) <= 1e-14 * dt_o
    assert relative(gpu.prims(), ora.prims()) < 1e-14
    if order == 1:
        assert relative(gpu.gradients(), ora.gradients()) < 1e-11
    gpu.step(dt_o)
    ora.step(dt_o)
    assert relative(gpu.get_state(), ora.get_state()) < 1e-13
    assert gpu.fallbacks() == ora.fallbacks()


def test_limiter_none_and_uniform_random_mesh(cuda):
    mesh = random_mesh(4096)
    q0 = rough_state(mesh.n_cells) * mesh.volume[:, None]
    gpu, ora = pair(mesh, q0, limiter="none")
    for _ in range(2):
        dt = ora.time_step(0.3)
        assert abs(gpu.time_step(0.3) - dt) <= 1e-14 * dt
        gpu.step(dt)
        ora.step(dt)
    assert relative(gpu.get_state(), ora.get_state()) < 1e-12


def ring_mesh():
    """A cell with 600 faces (a centre point inside a ring of 600 points, in a lattice background): more neighbours
    than one tile of the sweep stages, so it takes the single-cell tiles' launch with more shared memory."""
    from luna_cpp_b200.mesh import build_mesh

    th = np.linspace(0, 2 * np.pi, 600, endpoint=False)
    ring = np.stack([0.5 + 0.2 * np.cos(th), 0.5 + 0.2 * np.sin(th)], 1)
    g = (np.arange(24) + 0.5) / 24
    background = np.stack(np.meshgrid(g, g, indexing="ij"), -1).reshape(-1, 2)
    background = background[np.hypot(background[:, 0] - 0.5, background[:, 1] - 0.5) > 0.3]
    return build_mesh(np.concatenate([[[0.5, 0.5]], ring, background]), (1.0, 1.0))


@pytest.mark.parametrize("precision", ["fp64", "grad32"])
def test_cell_with_more_faces_than_a_tile(cuda, precision):
    mesh = ring_mesh()
    assert mesh.cell_face_start[1] - mesh.cell_face_start[0] == 600
    q0 = rough_state(mesh.n_cells, dim=2) * mesh.volume[:, None]
    gpu, ora = pair(mesh, q0, precision=precision)
    tol = 1e-12 if precision == "fp64" else 1e-6  # grad32: the float gradients' rounding differs from the oracle's
    for _ in range(3):
        dt = ora.time_step(0.3)
        assert abs(gpu.time_step(0.3) - dt) <= tol * dt
        gpu.step(dt)
        ora.step(dt)
    assert relative(gpu.get_state(), ora.get_state()) < tol


def test_blast_32_fp64_50_steps(cuda):
    """The plain-method configuration: 32^3 jittered (0.1) mesh, point blast, MUSCL-Hancock + HLLC, CFL 0.3, 50 steps,
    FP64, against the oracle: relative L1 <= 1e-12 for every conserved field (each side takes its own dt)."""
    mesh = jittered_mesh(32)
    q0 = point_blast(mesh)
    gpu, ora = pair(mesh, q0)
    for _ in range(50):
        gpu.step(gpu.time_step(0.3))
        ora.step(ora.time_step(0.3))
    g, o = gpu.get_state(), ora.get_state()
    assert np.all(np.isfinite(g))
    assert np.max(rel_l1(g, o)) < 1e-12
    assert gpu.fallbacks() == ora.fallbacks()


@pytest.mark.parametrize("precision", ["fp32", "grad32", "grad16", "single"])
def test_reduced_policy_matches_oracle_policy(cuda, precision):
    mesh = jittered_mesh(16)
    q0 = rough_state(mesh.n_cells) * mesh.volume[:, None]
    gpu, ora = pair(mesh, q0, precision=precision)
    dt = ora.time_step(0.3)
    assert abs(gpu.time_step(0.3) - dt) <= 1e-14 * dt
    if precision == "grad16":
        # the binary16 rows: the same roundings as the oracle's, but for the components whose float value differs by an
        # ulp (multiply-add contraction) right at a binary16 rounding boundary: those differ by one binary16 step
        g, o = gpu.gradients(), ora.gradients()
        D = 3
        groups = [slice(0, D), slice(D, D + D * D), slice(D + D * D, 5 * D)]
        step = np.concatenate([np.repeat(np.abs(o[:, s]).max(1, keepdims=True), s.stop - s.start, 1) for s in groups], 1) * 2.0 ** -10
        assert np.all(np.abs(g - o) <= step + 1e-300)
        assert np.mean(g == o) > 0.99
    gpu.step(dt)
    ora.step(dt)
    assert relative(gpu.get_state(), ora.get_state()) < (1e-4 if precision == "grad16" else 1e-6)


@pytest.mark.parametrize("problem", ["blast", "wave"])
def test_precision_config_128_fp64_against_oracle(cuda, problem):
    """The precision configuration's FP64 reference run: 128^3 jittered (0.1) mesh, the point blast or the 1e-6 plane
    acoustic wave, 100 steps on the oracle's dt schedule (each dt also checked). Blast: relative L1 <= 1e-12 for every
    conserved field. Wave: the fields are O(1) backgrounds plus a 1e-6 perturbation (and rounding-level transverse
    momenta), so the difference is measured against the perturbation: sum |gpu - oracle| / sum |oracle - background|
    (x-momentum: against itself) <= 1e-8 for density, x-momentum and energy, i.e. ~1e-14 of the fields. (The reduced
    policies are measured against this run by luna_cpp_b200.studies.precision.)"""
    mesh = jittered_mesh(128)
    q0 = point_blast(mesh) if problem == "blast" else acoustic_wave(mesh, amplitude=1e-6)
    gpu, ora = pair(mesh, q0)
    for _ in range(100):
        dt = ora.time_step(0.3)
        assert abs(gpu.time_step(0.3) - dt) <= 1e-13 * dt
        gpu.step(dt)
        ora.step(dt)
    got, want = gpu.get_state(), ora.get_state()
    if problem == "blast":
        assert np.all(rel_l1(got, want) < 1e-12)
    else:
        perturbation = np.abs(want - acoustic_wave(mesh, amplitude=0.0)).sum(0)
        err = np.abs(got - want).sum(0)
        assert np.all(err[[0, 1, 4]] / perturbation[[0, 1, 4]] < 1e-8), err / perturbation


@pytest.mark.parametrize("problem", ["wave", "blast"])
def test_reduced_policies_against_fp64(cuda, problem):
    """The reduced policies against FP64 (20 steps, each run its own dt): relative L1 of Q within 1e-5 for both. On the
    1e-6 acoustic wave also the error of the perturbation (Q minus the background): the double Riemann solve of grad32
    keeps it within 1e-5; the float Riemann solve of fp32 sees the O(1) face states at float's resolution (6e-8), i.e.
    the 1e-6 perturbation to a few per cent, which is bounded here and stated, not hidden."""
    mesh = jittered_mesh(16)
    q0 = acoustic_wave(mesh, amplitude=1e-6) if problem == "wave" else point_blast(mesh, radius_cells=2.5)
    res = {}
    for prec in ("fp64", "fp32", "grad32", "single"):
        fv = hydro.FiniteVolume(mesh, precision=prec)
        fv.set_state(q0)
        for _ in range(20):
            fv.step(fv.time_step(0.3))
        res[prec] = fv.get_state()
    for prec in ("fp32", "grad32", "single"):
        assert np.abs(res[prec] - res["fp64"]).sum() / np.abs(res["fp64"]).sum() < 1e-5
    if problem == "wave":
        background = acoustic_wave(mesh, amplitude=0.0)
        p64 = res["fp64"] - background
        pert = {prec: np.abs(res[prec] - res["fp64"]).sum() / np.abs(p64).sum() for prec in ("fp32", "grad32", "single")}
        assert pert["grad32"] < 1e-5
        assert pert["fp32"] < 0.2 and pert["single"] < 0.2


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("precision", ["fp64", "fp32", "grad32", "grad16", "single"])
def test_uniform_state_stays_uniform(cuda, order, precision):
    mesh = jittered_mesh(16)
    W = np.array([1.3, 0.3, -0.2, 0.1, 0.7])
    U = O.conserved(W)
    fv = hydro.FiniteVolume(mesh, order=order, precision=precision)
    fv.set_state(np.tile(U, (mesh.n_cells, 1)) * mesh.volume[:, None])
    for _ in range(3):
        fv.step(fv.time_step(0.3))
    got = fv.get_state() / mesh.volume[:, None]
    assert relative(got, np.tile(U, (mesh.n_cells, 1))) < (1e-13 if precision == "fp64" else 1e-6)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "grad32", "grad16", "single"])
def test_conservation_and_determinism(cuda, precision):
    mesh = jittered_mesh(16)
    q0 = rough_state(mesh.n_cells) * mesh.volume[:, None]
    outs = []
    for _ in range(2):
        fv = hydro.FiniteVolume(mesh, precision=precision)
        fv.set_state(q0)
        for _ in range(10):
            fv.step(fv.time_step(0.3))
        outs.append(fv.get_state())
    assert np.array_equal(outs[0], outs[1])
    before = q0.astype(np.longdouble).sum(0)
    after = outs[0].astype(np.longdouble).sum(0)
    assert abs(float((after[0] - before[0]) / before[0])) < 1e-14
    assert abs(float((after[4] - before[4]) / before[4])) < 1e-14
    scale = float(before[0]) * np.sqrt(float(before[4] / before[0]))
    assert np.max(np.abs((after[1:4] - before[1:4]).astype(np.float64))) / scale < 1e-14


def test_per_cell_and_per_face_agree(cuda):
    mesh = jittered_mesh(16)
    q0 = rough_state(mesh.n_cells) * mesh.volume[:, None]
    outs = []
    for update in ("per_face", "per_cell"):
        fv = hydro.FiniteVolume(mesh, update=update)
        fv.set_state(q0)
        for _ in range(10):
            fv.step(fv.time_step(0.3))
        outs.append(fv.get_state())
    assert relative(outs[1], outs[0]) < 1e-12


def test_2d_shear_layer_matches_oracle(cuda):
    mesh = jittered_mesh(32, dim=2)
    a = np.random.default_rng(3).standard_normal(8)
    q0 = shear_layer(mesh, a)
    gpu, ora = pair(mesh, q0)
    for _ in range(5):
        dt = ora.time_step(0.3)
        assert abs(gpu.time_step(0.3) - dt) <= 1e-14 * dt
        gpu.step(dt)
        ora.step(dt)
    assert relative(gpu.get_state(), ora.get_state()) < 1e-12


def test_moving_step_matches_oracle(cuda):
    """step_moving on a moving mesh: the t^n fluxes, the drift on the 2^-30 grid, the remesh, the t^n+1 fluxes."""
    from luna_cpp_b200.mesh import build_mesh

    mesh = jittered_mesh(12)
    step = 2.0 ** -30
    mesh = build_mesh(np.round(mesh.positions / step) * step)  # generators on the snapping grid
    q0 = point_blast(mesh, radius_cells=2.5)
    gpu, ora = pair(mesh, q0, motion="moving")
    remesh = lambda pos: build_mesh(pos)
    for _ in range(3):
        dt = ora.time_step(0.3)
        assert abs(gpu.time_step(0.3) - dt) <= 1e-14 * dt
        assert relative(gpu.point_velocities(), ora.point_velocities()) < 1e-13
        mg = gpu.step_moving(dt, remesh)
        mo = ora.step_moving(dt, remesh)
        assert np.array_equal(mg.positions, mo.positions)
    g, o = gpu.get_state(), ora.get_state()
    assert relative(g, o) < 1e-12
    before = q0.sum(0)
    assert abs((g[:, 0].sum() - before[0]) / before[0]) < 1e-14
    assert abs((g[:, 4].sum() - before[4]) / before[4]) < 1e-14


@pytest.mark.parametrize("precision", ["fp64", "fp32", "single"])
def test_moving_config_radial_profile_against_oracle(cuda, precision):
    """The moving-mesh configuration scaled down: the point blast on 16^3 snapped jittered generators, moving mesh, to
    t = 0.05, each side its own dt, positions and remesh; the radial density profile (32 shells) against the oracle's
    run of the same policy: relative L1 <= 1e-8 (FP64) or 1e-4 (FP32 face arithmetic: riemann32, and single with its
    float flux rows). Also the steps taken agree and mass and energy are conserved to round-off."""
    from luna_cpp_b200.mesh import build_mesh
    from luna_cpp_b200.studies import radial_profile, snapped_jittered_mesh

    mesh = snapped_jittered_mesh(16)
    q0 = point_blast(mesh)
    gpu, ora = pair(mesh, q0, motion="moving", precision=precision)
    remesh = lambda pos: build_mesh(pos)
    t_end, profiles = 0.05, []
    for fv in (gpu, ora):
        t, steps, m = 0.0, 0, mesh
        while t < t_end:
            dt = min(fv.time_step(0.3), t_end - t)
            m = fv.step_moving(dt, remesh)
            t += dt
            steps += 1
        q = fv.get_state()
        profiles.append((steps, radial_profile(m, q)))
        assert abs(q[:, 0].sum() - q0[:, 0].sum()) / q0[:, 0].sum() < 1e-13
        assert abs(q[:, 4].sum() - q0[:, 4].sum()) / q0[:, 4].sum() < 1e-13
    (sg, pg), (so, po) = profiles
    assert sg == so
    assert np.abs(pg - po).sum() / np.abs(po).sum() < (1e-8 if precision == "fp64" else 1e-4)


def test_errors_are_status_codes(cuda):
    mesh = jittered_mesh(8)
    fv = hydro.FiniteVolume(mesh)
    with pytest.raises(hydro.LunaError) as e:
        fv.step(-1.0)
    assert e.value.status == 1
    with pytest.raises(hydro.LunaError) as e:
        hydro.lib()
        hydro.check(hydro.lib().luna_fv_step_moving_end(fv.handle, None))
    assert e.value.status in (1, 6)
    with pytest.raises(hydro.LunaError):
        hydro.FiniteVolume(mesh, motion="moving", update="per_cell")


def test_full_size_properties(cuda):
    """The 128^3 blast (the benchmark's workload) at full size: 3 steps stay finite, conserve mass and energy to 1e-14,
    and repeat bit for bit."""
    mesh = jittered_mesh(128)
    q0 = point_blast(mesh)
    outs = []
    for _ in range(2):
        fv = hydro.FiniteVolume(mesh)
        fv.set_state(q0)
        for _ in range(3):
            dt = fv.time_step(0.3)
            assert dt > 0
            fv.step(dt)
        outs.append(fv.get_state())
        fv.close()
    assert np.all(np.isfinite(outs[0]))
    assert np.array_equal(outs[0], outs[1])
    before = q0.astype(np.longdouble).sum(0)
    after = outs[0].astype(np.longdouble).sum(0)
    assert abs(float((after[0] - before[0]) / before[0])) < 1e-14
    assert abs(float((after[4] - before[4]) / before[4])) < 1e-13
