"""The sweep's tiles (luna_mesh_tiles, host code only): every cell in exactly one tile, a tile's own cells staged
first in thread order, every list entry's staged row naming its neighbour and inside its tile's rows (the bound the
sweep's shared-memory reads rely on), entry slots unique and inside their warp's slice, the row budget kept."""
import numpy as np
import pytest

from conftest import jittered_mesh, random_mesh
from luna_cpp_b200 import hydro


def ring_mesh():
    from luna_cpp_b200.mesh import build_mesh

    th = np.linspace(0, 2 * np.pi, 600, endpoint=False)
    ring = np.stack([0.5 + 0.2 * np.cos(th), 0.5 + 0.2 * np.sin(th)], 1)
    g = (np.arange(24) + 0.5) / 24
    background = np.stack(np.meshgrid(g, g, indexing="ij"), -1).reshape(-1, 2)
    background = background[np.hypot(background[:, 0] - 0.5, background[:, 1] - 0.5) > 0.3]
    return build_mesh(np.concatenate([[[0.5, 0.5]], ring, background]), (1.0, 1.0))


def check_tiles(mesh):
    t = hydro.mesh_tiles(mesh)
    order, sb, ss, sc, local = t["order"], t["slice_base"], t["stage_start"], t["stage_cells"], t["local"]
    n, tiles = mesh.n_cells, t["tiles"]
    cells = order[order >= 0]
    assert len(cells) == n and len(np.unique(cells)) == n
    assert ss[0] == 0 and ss[-1] == len(sc) and np.all(np.diff(ss) > 0)
    rows = np.diff(ss)
    assert rows[: t["normal_tiles"]].max() == t["most_rows"] <= 416
    assert np.all(rows[t["normal_tiles"]:] > 416)
    assert len(local) == max(sb[-1] * 32, 1)
    start, lst = mesh.cell_face_start, mesh.cell_face
    seen = np.zeros(len(local), bool)
    for u in range(tiles):
        staged = sc[ss[u]: ss[u + 1]]
        assert len(np.unique(staged)) == len(staged)
        own = order[u * 128: (u + 1) * 128]
        k = int((own >= 0).sum())
        assert np.all(own[:k] >= 0) and np.all(own[k:] < 0)
        assert np.array_equal(staged[:k], own[:k])
        for lane in range(k):
            c, th = own[lane], u * 128 + lane
            length = start[c + 1] - start[c]
            assert length <= sb[(th >> 5) + 1] - sb[th >> 5]
            slots = sb[th >> 5] * 32 + (th & 31) + 32 * np.arange(length)
            assert not seen[slots].any()
            seen[slots] = True
            e = lst[start[c]: start[c + 1]]
            f = np.where(e >= 0, e, ~e)
            j = np.where(e >= 0, mesh.neighbour[f], mesh.owner[f])
            r = local[slots]
            assert np.all(r < len(staged))
            assert np.array_equal(staged[r], j)
    return t


@pytest.mark.parametrize("make", [lambda: jittered_mesh(16), lambda: jittered_mesh(64, 2), lambda: random_mesh(3000),
                                  lambda: random_mesh(2000, 2)])
def test_tile_invariants(make):
    t = check_tiles(make())
    assert t["normal_tiles"] == t["tiles"]


def test_cell_with_more_faces_than_a_tile_gets_its_own_tile():
    mesh = ring_mesh()
    t = check_tiles(mesh)
    assert t["tiles"] - t["normal_tiles"] == 1
    big = t["normal_tiles"]
    assert t["order"][big * 128] == 0 and np.all(t["order"][big * 128 + 1: (big + 1) * 128] < 0)
    assert t["most_rows_single"] == 601


def test_tiles_of_a_jittered_mesh_are_compact():
    """Morton tiles of a 16^3 jittered mesh: full tiles of 128 cells, about 2.6 staged rows a cell."""
    t = check_tiles(jittered_mesh(16))
    assert t["tiles"] == 32
    assert len(t["stage_cells"]) / 4096 < 3.0
