"""Periodic Voronoi meshes in voronoi-cpp's face layout, built on the host by ``libluna_mesh.so``.

The hydro library consumes exactly the arrays voronoi-cpp's ``voronoi::Mesh`` exposes to luna-cpp's
``FiniteVolume::refresh()`` (src/hydro/finite_volume.hpp:353-364): ``owner``/``neighbour`` per face, the CSR lists
``cell_face_start``/``cell_face`` (``~f`` marks a face the cell does not own, the owner bit read by
``Geometry::owned_at``, finite_volume.hpp:318), area vectors owner -> neighbour, face centroids relative to the owner's
generator (``Geometry::face_offset``, finite_volume.hpp:322-326), cell centroids relative to the generator, volumes and
the generators. voronoi-cpp itself is not available, so meshes come from this builder.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native


class _Arrays(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int),
        ("n_cells", ctypes.c_int64),
        ("n_faces", ctypes.c_int64),
        ("owner", ctypes.c_void_p),
        ("neighbour", ctypes.c_void_p),
        ("cell_face_start", ctypes.c_void_p),
        ("cell_face", ctypes.c_void_p),
        ("area", ctypes.c_void_p),
        ("face_centroid", ctypes.c_void_p),
        ("centroid", ctypes.c_void_p),
        ("volume", ctypes.c_void_p),
        ("positions", ctypes.c_void_p),
        ("box", ctypes.c_double * 3),
        ("inconsistent", ctypes.c_int64),
    ]


def _lib():
    lib = _native.load("mesh")
    if not getattr(lib, "_typed", False):
        lib.luna_mesh_create.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_void_p)]
        lib.luna_mesh_create.restype = ctypes.c_int
        lib.luna_mesh_arrays_of.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Arrays)]
        lib.luna_mesh_arrays_of.restype = ctypes.c_int
        lib.luna_mesh_free.argtypes = [ctypes.c_void_p]
        lib.luna_mesh_free.restype = None
        lib.luna_mesh_error.argtypes = []
        lib.luna_mesh_error.restype = ctypes.c_char_p
        lib.luna_jittered_points.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                             ctypes.c_uint64, ctypes.c_void_p]
        lib.luna_jittered_points.restype = ctypes.c_int
        lib._typed = True
    return lib


@dataclass
class Mesh:
    """A periodic Voronoi mesh (voronoi-cpp's arrays, host numpy copies)."""

    dim: int
    owner: np.ndarray  # int32 [F]
    neighbour: np.ndarray  # int32 [F]
    cell_face_start: np.ndarray  # int32 [N+1]
    cell_face: np.ndarray  # int32 [2F], ~f: not owned
    area: np.ndarray  # float64 [F, D]
    face_centroid: np.ndarray  # float64 [F, D], relative to the owner's generator
    centroid: np.ndarray  # float64 [N, D], relative to the generator
    volume: np.ndarray  # float64 [N]
    positions: np.ndarray  # float64 [N, D]
    box: tuple
    inconsistent: int = 0

    @property
    def n_cells(self) -> int:
        return int(self.volume.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.owner.shape[0])


def _copy(ptr, dtype, shape):
    count = int(np.prod(shape)) if shape else 1
    if count == 0:
        return np.zeros(shape, dtype=dtype)
    ctype = {np.int32: ctypes.c_int32, np.float64: ctypes.c_double}[dtype]
    buf = (ctype * count).from_address(ptr)
    return np.frombuffer(buf, dtype=dtype, count=count).reshape(shape).copy()


def build_mesh(points: np.ndarray, box=(1.0, 1.0, 1.0), threads: int = 0) -> Mesh:
    """The periodic Voronoi mesh of ``points`` ([N, D]) in the box [0, box_a) per axis."""
    pts = np.ascontiguousarray(points, dtype=np.float64)
    n, dim = pts.shape
    b = np.zeros(3, dtype=np.float64)
    b[: len(box)] = box
    lib = _lib()
    handle = ctypes.c_void_p()
    rc = lib.luna_mesh_create(dim, n, pts.ctypes.data, b.ctypes.data, threads, ctypes.byref(handle))
    if rc != 0:
        raise ValueError(lib.luna_mesh_error().decode())
    try:
        a = _Arrays()
        lib.luna_mesh_arrays_of(handle, ctypes.byref(a))
        N, F = a.n_cells, a.n_faces
        return Mesh(
            dim=dim,
            owner=_copy(a.owner, np.int32, (F,)),
            neighbour=_copy(a.neighbour, np.int32, (F,)),
            cell_face_start=_copy(a.cell_face_start, np.int32, (N + 1,)),
            cell_face=_copy(a.cell_face, np.int32, (2 * F,)),
            area=_copy(a.area, np.float64, (F, dim)),
            face_centroid=_copy(a.face_centroid, np.float64, (F, dim)),
            centroid=_copy(a.centroid, np.float64, (N, dim)),
            volume=_copy(a.volume, np.float64, (N,)),
            positions=_copy(a.positions, np.float64, (N, dim)),
            box=tuple(float(x) for x in b[:dim]),
            inconsistent=int(a.inconsistent),
        )
    finally:
        lib.luna_mesh_free(handle)


def _hilbert_transpose(X: np.ndarray, bits: int) -> np.ndarray:
    """Skilling's axes-to-transpose map (J. Skilling, "Programming the Hilbert curve", AIP Conf. Proc. 707, 381 (2004)),
    vectorised over rows: X [n, dim] unsigned integer coordinates of ``bits`` bits, returned in transposed form (the
    curve index's bits read across the axes, most significant level first)."""
    X = X.copy()
    dim = X.shape[1]
    q = np.uint64(1) << np.uint64(bits - 1)
    while q > 1:
        p = q - np.uint64(1)
        for i in range(dim):
            hit = (X[:, i] & q) != 0
            X[hit, 0] ^= p
            t = (X[:, 0] ^ X[:, i]) & p
            t[hit] = 0
            X[:, 0] ^= t
            X[:, i] ^= t
        q >>= np.uint64(1)
    for i in range(1, dim):
        X[:, i] ^= X[:, i - 1]
    t = np.zeros(X.shape[0], dtype=np.uint64)
    q = np.uint64(1) << np.uint64(bits - 1)
    while q > 1:
        t[(X[:, dim - 1] & q) != 0] ^= q - np.uint64(1)
        q >>= np.uint64(1)
    X ^= t[:, None]
    return X


def curve_order(points: np.ndarray, box=None, curve: str = "hilbert", bits: int = 16) -> np.ndarray:
    """The permutation that numbers ``points`` along a space-filling curve through the box: voronoi-cpp's cell
    ordering (``voronoi::Layout::curve``: hilbert, morton, ...; luna-cpp's ``--curve``, README.md:75, :94), which keeps
    a cell's neighbours close to it in memory. ``points[curve_order(points)]`` is the reordered set; "row" keeps the
    given order."""
    pts = np.asarray(points, dtype=np.float64)
    n, dim = pts.shape
    if curve == "row" or n == 0:
        return np.arange(n)
    side = np.ones(dim) if box is None else np.asarray(box, dtype=np.float64)[:dim]
    scale = float(1 << bits)
    X = np.clip(np.floor(pts / side * scale), 0, scale - 1).astype(np.uint64)
    if curve == "hilbert":
        X = _hilbert_transpose(X, bits)
    elif curve != "morton":
        raise ValueError(f"unknown curve {curve!r}")
    code = np.zeros(n, dtype=np.uint64)
    for level in range(bits - 1, -1, -1):
        for i in range(dim):
            code = (code << np.uint64(1)) | ((X[:, i] >> np.uint64(level)) & np.uint64(1))
    return np.argsort(code, kind="stable")


def jittered_points(cells, side=None, jitter: float = 0.1, seed: int = 1) -> np.ndarray:
    """problems_3d.hpp's ``jittered_points`` (src/hydro/problems_3d.hpp:37-53): the lattice point (i + 1/2) h moved by
    uniform(-jitter, jitter) spacings per axis from ``std::mt19937_64(seed)``, wrapped into [0, side); the last axis runs
    fastest. Works for 2 or 3 axes."""
    cells = [int(c) for c in cells]
    dim = len(cells)
    if side is None:
        side = [1.0] * dim
    c = np.array(cells, dtype=np.int32)
    s = np.array(side, dtype=np.float64)
    out = np.empty((int(np.prod(cells)), dim), dtype=np.float64)
    rc = _lib().luna_jittered_points(dim, c.ctypes.data, s.ctypes.data, float(jitter), int(seed), out.ctypes.data)
    if rc != 0:
        raise ValueError(_lib().luna_mesh_error().decode())
    return out
