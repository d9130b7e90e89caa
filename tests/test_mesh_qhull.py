"""The mesh builder against an independent Voronoi implementation: qhull (through scipy.spatial), run on the 27
periodic images of the generators. The device remesher equals the host builder bit for bit (tests/test_gpu_remesh.py),
so this pins both to a third-party construction: the same face pairs, area vectors, face centroids and cell volumes to
round-off. CPU only."""
import itertools

import numpy as np
import pytest

from luna_cpp_b200.mesh import build_mesh, jittered_points

scipy_spatial = pytest.importorskip("scipy.spatial")


def periodic_qhull(pts, box):
    """Faces {(i, j): (area vector out of i, centroid relative to i's generator)} and volumes of the periodic Voronoi
    mesh of pts, from qhull's Voronoi diagram of the 3^D images (the central image's cells)."""
    n, D = pts.shape
    shifts = np.array(list(itertools.product((-1, 0, 1), repeat=D)), dtype=float)
    zero = int(np.where((shifts == 0).all(1))[0][0])
    allp = np.concatenate([pts + s * box for s in shifts])
    vor = scipy_spatial.Voronoi(allp)
    base = zero * n
    faces = {}
    for (p, q), rv in zip(vor.ridge_points, vor.ridge_vertices):
        for a, b in ((p, q), (q, p)):
            if not base <= a < base + n:
                continue
            assert -1 not in rv
            i, j = a - base, b % n
            V = vor.vertices[rv]
            nrm = (allp[b] - allp[a]) / np.linalg.norm(allp[b] - allp[a])
            if D == 3:  # the ridge's polygon ordered around its mean, fanned from its first vertex
                c0 = V.mean(0)
                u = np.cross(nrm, [1.0, 0, 0] if abs(nrm[0]) < 0.6 else [0, 1.0, 0])
                u /= np.linalg.norm(u)
                w = np.cross(nrm, u)
                V = V[np.argsort(np.arctan2((V - c0) @ w, (V - c0) @ u))]
                A, C, tot = np.zeros(3), np.zeros(3), 0.0
                for k in range(1, len(V) - 1):
                    t = 0.5 * np.cross(V[k] - V[0], V[k + 1] - V[0])
                    A += t
                    C += (t @ nrm) * (V[0] + V[k] + V[k + 1]) / 3
                    tot += t @ nrm
                faces[(i, j)] = (A, C / tot - pts[i])
            else:
                A = np.array([V[1, 1] - V[0, 1], -(V[1, 0] - V[0, 0])])
                faces[(i, j)] = (A if A @ nrm > 0 else -A, V.mean(0) - pts[i])
    vol = np.array([scipy_spatial.ConvexHull(vor.vertices[vor.regions[vor.point_region[base + i]]]).volume for i in range(n)])
    return faces, vol


def hollow():
    """A 10^3 lattice with a hole of radius 0.33 and one generator in it: a cell of 64 faces."""
    p = jittered_points((10, 10, 10), jitter=0.1, seed=4)
    return np.concatenate([[[0.5, 0.5, 0.5]], p[np.linalg.norm(p - 0.5, axis=1) > 0.33]])


CASES = [("jittered 8^3", lambda: jittered_points((8, 8, 8), jitter=0.1, seed=1), 3),
         ("hollow 10^3", hollow, 3),
         ("uniform random 400", lambda: np.random.default_rng(2).random((400, 3)), 3),
         ("2D jittered 16^2", lambda: jittered_points((16, 16), jitter=0.1, seed=1), 2)]


@pytest.mark.parametrize("name,points,dim", CASES, ids=[c[0] for c in CASES])
def test_builder_matches_qhull(name, points, dim):
    pts = points()
    box = np.ones(dim)
    ref, vol = periodic_qhull(pts, box)
    m = build_mesh(pts, box=tuple(box))
    ours = {(int(m.owner[f]), int(m.neighbour[f])): (m.area[f], m.face_centroid[f]) for f in range(m.n_faces)}
    amax = max(np.linalg.norm(a) for a, _ in ours.values())
    # faces of zero area (four or more generators on a sphere) are qhull's to keep or merge: compared above 1e-9
    want = {k for k, (a, _) in ref.items() if k[0] < k[1] and np.linalg.norm(a) > 1e-9 * amax}
    got = {k for k, (a, _) in ours.items() if np.linalg.norm(a) > 1e-9 * amax}
    assert want == got
    for k in got:
        assert np.abs(ref[k][0] - ours[k][0]).max() < 1e-13 * amax
        assert np.abs(ref[k][1] - ours[k][1]).max() < 1e-13
    assert np.max(np.abs(vol - m.volume) / m.volume) < 1e-13


def test_face_loop_cells_match_qhull():
    """The builder with its 3D cells kept as face loops (LUNA_MESH_DUAL=0, read once per process: a subprocess; the
    default keeps them as triangles of plane triples) against qhull and the Voronoi invariants."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys; sys.path.insert(0, 'tests')\n"
        "import numpy as np\n"
        "from conftest import voronoi_invariants\n"
        "from test_mesh_qhull import CASES, test_builder_matches_qhull\n"
        "from luna_cpp_b200.mesh import build_mesh\n"
        "for name, points, dim in CASES:\n"
        "    test_builder_matches_qhull(name, points, dim)\n"
        "    voronoi_invariants(build_mesh(points(), box=(1.0,) * dim))\n"
        "print('ok')\n"
    )
    r = subprocess.run([sys.executable, "-c", code], cwd=root, env=dict(os.environ, LUNA_MESH_DUAL="0"), capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-2000:]


def test_degenerate_lattices():
    """The exact regular lattice of the rollout server (rollout.lattice: four or more bisector planes meet at every
    vertex) gives the regular mesh: every cell a cube of the lattice's volume with 6 faces of area h^2, the invariants
    hold. Moved by ~1e-9 the near-degenerate vertices are still resolved (the invariants hold). Moved by ~1e-12 the
    builder either gives a mesh that satisfies the invariants or refuses the points with an error, never a broken mesh."""
    from conftest import voronoi_invariants
    from luna_cpp_b200.mesh import build_mesh
    from luna_cpp_b200.rollout import lattice

    for n in (5, 8):
        m = build_mesh(lattice(n, 3))
        voronoi_invariants(m)
        assert m.n_faces == 3 * n ** 3
        assert np.allclose(m.volume, 1.0 / n ** 3, rtol=1e-7)
        assert np.allclose(np.linalg.norm(m.area, axis=1), 1.0 / n ** 2, rtol=1e-7)
    m = build_mesh(lattice(6, 3) + np.random.default_rng(2).uniform(-1e-9, 1e-9, (216, 3)))
    voronoi_invariants(m)
    try:
        m = build_mesh(lattice(8, 3) + np.random.default_rng(1).uniform(-1e-12, 1e-12, (512, 3)))
    except ValueError as e:
        assert "more vertices or faces" in str(e)
    else:
        voronoi_invariants(m)
