"""Python binding of the reference's own FiniteVolume<D> built on the CPU (``oracle/_ref/libluna_ref.so``): TEST
INFRASTRUCTURE ONLY.

``oracle/Makefile`` compiles luna-cpp's src/hydro/finite_volume.hpp, euler.hpp and precision.hpp unmodified against
``ref_shim/`` (a host-only Kokkos with OpenMP, and the part of voronoi-cpp the solver reads, over this repository's mesh
arrays). The tests use it to pin the C restatement (``luna_oracle.c``) to the reference's arithmetic; bench.py may time
it as the reference's CPU path. The product never imports this module. The library needs the luna-cpp source tree to
build; where it is absent and the library was not built, ``available()`` is False.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libluna_ref.so")
PRECISIONS = {"double": 0, "riemann32": 1, "grad32": 2, "grad16": 3, "single": 4}


class _Arrays(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("n", ctypes.c_int64), ("f", ctypes.c_int64),
                ("owner", ctypes.c_void_p), ("neighbour", ctypes.c_void_p), ("start", ctypes.c_void_p),
                ("list", ctypes.c_void_p), ("area", ctypes.c_void_p), ("face_centroid", ctypes.c_void_p),
                ("centroid", ctypes.c_void_p), ("volume", ctypes.c_void_p), ("positions", ctypes.c_void_p),
                ("box", ctypes.c_double * 3)]


_REMESH = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(_Arrays))
# the caller's GeometryDerivative (mesh_derivative.hpp:10-29): tangent(dx -> dV, dc, dA, dxf), adjoint(bars -> adds to xbar)
_GEO_TANGENT = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p)
_GEO_ADJOINT = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p)
_lib = None


def build(reference: str | None = None) -> str:
    """make -C oracle REF=<luna-cpp tree>; the tree defaults to the LUNA_REFERENCE environment variable."""
    ref = reference or os.environ.get("LUNA_REFERENCE")
    cmd = ["make", "-s", "-C", HERE, "-j3"] + ([f"REF={ref}"] if ref else [])
    subprocess.run(cmd, check=True)
    return LIB


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    L = ctypes.CDLL(LIB)
    P, D, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
    sig = {
        "lr_last_error": ([], ctypes.c_char_p),
        "lr_threads": ([I], I),
        "lr_fv_create": ([ctypes.POINTER(_Arrays), D, I, I, I, I, I, I, _REMESH, P], P),
        "lr_fv_destroy": ([P], None),
        "lr_fv_state": ([P], P),
        "lr_fv_time_step": ([P, D, ctypes.POINTER(D)], I),
        "lr_fv_step": ([P, D], I),
        "lr_fv_fallbacks": ([P], ctypes.c_longlong),
        "lr_fv_step_adjoint": ([P, D, P], I),
        "lr_fv_time_step_tangent": ([P, D, P, ctypes.POINTER(D)], I),
        "lr_fv_step_tangent": ([P, D, P], I),
        "lr_fv_positions": ([P], P),
        "lr_fv_point_velocities": ([P], P),
        "lr_fv_cells": ([P], I),
        "lr_fv_faces": ([P], I),
        "lr_fv_density_gradients": ([P, P], I),
        "lr_fv_set_positions": ([P, P], I),
        "lr_fv_step_moving_tangent": ([P, D, P, P, _GEO_TANGENT, _GEO_ADJOINT, P, I], I),
        "lr_fv_step_moving_adjoint": ([P, D, P, P, _GEO_TANGENT, _GEO_ADJOINT, P, I], I),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def threads(n: int = 0) -> int:
    return int(lib().lr_threads(n))


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().lr_last_error().decode())


class ReferenceFV:
    """hydro::FiniteVolume<D> of the reference on one mesh (luna_cpp_b200.mesh.Mesh); the OracleFV interface.

    moving: Motion::moving; each mesh update calls ``remesh(positions) -> Mesh`` (default: the host builder)."""

    def __init__(self, mesh, gamma=5.0 / 3.0, order=1, per_face=True, limiter="face_centroid", riemann="hllc",
                 moving=False, precision="double", remesh=None):
        self.mesh = mesh
        self.dim = mesh.dim
        self.V = mesh.dim + 2
        self._keep = []
        self._remesh = remesh
        self._cb = _REMESH(self._on_remesh)
        arrays = self._arrays(mesh)
        self._h = lib().lr_fv_create(ctypes.byref(arrays), gamma, order, 1 if per_face else 0,
                                     1 if limiter == "none" else 0, 1 if riemann == "hll" else 0, 1 if moving else 0,
                                     PRECISIONS[precision], self._cb, None)
        if not self._h:
            raise RuntimeError(lib().lr_last_error().decode())

    def _arrays(self, mesh):
        keep = [np.ascontiguousarray(x) for x in (mesh.owner, mesh.neighbour, mesh.cell_face_start, mesh.cell_face,
                                                   mesh.area, mesh.face_centroid, mesh.centroid, mesh.volume,
                                                   mesh.positions)]
        self._keep = [keep]
        a = _Arrays()
        a.dim, a.n, a.f = mesh.dim, mesh.n_cells, mesh.n_faces
        (a.owner, a.neighbour, a.start, a.list, a.area, a.face_centroid, a.centroid, a.volume,
         a.positions) = [x.ctypes.data for x in keep]
        for k in range(3):
            a.box[k] = mesh.box[k] if k < len(mesh.box) else 0.0
        return a

    def _on_remesh(self, user, positions, out):
        try:
            x = np.ctypeslib.as_array(ctypes.cast(positions, ctypes.POINTER(ctypes.c_double)),
                                      shape=(self.mesh.n_cells, self.dim)).copy()
            if self._remesh is None:
                from luna_cpp_b200.mesh import build_mesh

                new = build_mesh(x, box=tuple(self.mesh.box[: self.dim]))
            else:
                new = self._remesh(x)
            self.mesh = new
            out[0] = self._arrays(new)
            return 0
        except Exception:  # noqa: BLE001 - reported as a failed update
            return 1

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().lr_fv_destroy(h)
            self._h = None

    @property
    def n(self):
        return self.mesh.n_cells

    def _rows(self, ptr, width):
        buf = (ctypes.c_double * (self.n * width)).from_address(ptr)
        return np.frombuffer(buf, dtype=np.float64).reshape(self.n, width)

    def state(self):
        return self._rows(lib().lr_fv_state(self._h), self.V)

    def set_state(self, q):
        self.state()[:] = q

    def get_state(self):
        return self.state().copy()

    def time_step(self, courant=0.3):
        dt = ctypes.c_double()
        _check(lib().lr_fv_time_step(self._h, courant, ctypes.byref(dt)))
        return dt.value

    def step(self, dt):
        _check(lib().lr_fv_step(self._h, dt))

    def fallbacks(self):
        return int(lib().lr_fv_fallbacks(self._h))

    def step_adjoint(self, dt, qbar):
        q = np.ascontiguousarray(qbar, dtype=np.float64).copy()
        _check(lib().lr_fv_step_adjoint(self._h, dt, q.ctypes.data))
        return q

    def time_step_tangent(self, courant, dq):
        self._dq = np.ascontiguousarray(dq, dtype=np.float64).copy()
        dt = ctypes.c_double()
        _check(lib().lr_fv_time_step_tangent(self._h, courant, self._dq.ctypes.data, ctypes.byref(dt)))
        return dt.value

    def step_tangent(self, dt, dq):
        d = np.ascontiguousarray(dq, dtype=np.float64).copy()
        _check(lib().lr_fv_step_tangent(self._h, dt, d.ctypes.data))
        return d

    def positions(self):
        return self._rows(lib().lr_fv_positions(self._h), self.dim).copy()

    def point_velocities(self):
        return self._rows(lib().lr_fv_point_velocities(self._h), self.dim).copy()

    def density_gradients(self):
        out = np.zeros((self.n, self.dim))
        _check(lib().lr_fv_density_gradients(self._h, out.ctypes.data))
        return out

    def set_positions(self, x):
        """A moving mesh's positions and their mesh (Rollout::load_positions, rollout.cpp:146-152); Q is kept."""
        a = np.ascontiguousarray(x, dtype=np.float64)
        _check(lib().lr_fv_set_positions(self._h, a.ctypes.data))

    def _geometry_callbacks(self, geometry):
        """The caller's geometry derivative as the driver's two callbacks: one derivative object, or a factory (a class
        or a function of the mesh) evaluated on the mesh as it is at each call (the order-1 derivatives ask before and
        after their step)."""
        N, D = self.n, self.dim
        make = geometry if (isinstance(geometry, type) or not hasattr(geometry, "tangent")) else (lambda mesh: geometry)

        def view(ptr, shape):
            return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)), shape=shape)

        def tangent(user, dx, dV, dc, dA, dxf):
            F = self.mesh.n_faces
            out = make(self.mesh).tangent(view(dx, (N, D)).copy())
            for arr, ptr, shape in zip(out, (dV, dc, dA, dxf), ((N,), (N, D), (F, D), (F, D))):
                view(ptr, shape)[...] = arr

        def adjoint(user, Vbar, cbar, Abar, xfbar, xbar):
            F = self.mesh.n_faces
            add = make(self.mesh).adjoint(view(Vbar, (N,)).copy(), view(cbar, (N, D)).copy(), view(Abar, (F, D)).copy(),
                                          view(xfbar, (F, D)).copy())
            view(xbar, (N, D))[...] += add

        return _GEO_TANGENT(tangent), _GEO_ADJOINT(adjoint)

    def step_moving_tangent(self, dt, dq, dx, geometry, steps_fixed=False):
        """step_moving_tangent(dt, dq, dx, geometry) (finite_volume.hpp:2431-2486): (dq, dx) -> after the step, and the
        step itself (the state advances, the mesh moves)."""
        q = np.ascontiguousarray(dq, dtype=np.float64).copy()
        x = np.ascontiguousarray(dx, dtype=np.float64).copy()
        t, a = self._geometry_callbacks(geometry)
        _check(lib().lr_fv_step_moving_tangent(self._h, dt, q.ctypes.data, x.ctypes.data, t, a, None, 1 if steps_fixed else 0))
        return q, x

    def step_moving_adjoint(self, dt, qbar, xbar, geometry, steps_fixed=False):
        """step_moving_adjoint(dt, qbar, xbar, geometry) (:2490-2604): the bars after the step -> at its start; the state
        and the mesh must be the step's start."""
        q = np.ascontiguousarray(qbar, dtype=np.float64).copy()
        x = np.ascontiguousarray(xbar, dtype=np.float64).copy()
        t, a = self._geometry_callbacks(geometry)
        _check(lib().lr_fv_step_moving_adjoint(self._h, dt, q.ctypes.data, x.ctypes.data, t, a, None, 1 if steps_fixed else 0))
        return q, x
