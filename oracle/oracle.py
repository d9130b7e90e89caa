"""Python binding of the CPU oracle (``liboracle.so``): TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this module, as the checker of the CUDA
path; the product never imports it. See ``luna_oracle.h`` for what the oracle restates and how it is pinned.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


class _Gas(ctypes.Structure):
    _fields_ = [("gamma", ctypes.c_double), ("smallr", ctypes.c_double), ("smallc", ctypes.c_double),
                ("inverse_gm1", ctypes.c_double), ("inverse_gm1_float", ctypes.c_float)]


class _Mesh(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("n", ctypes.c_int64), ("f", ctypes.c_int64),
                ("owner", ctypes.c_void_p), ("neighbour", ctypes.c_void_p), ("start", ctypes.c_void_p),
                ("list", ctypes.c_void_p), ("area", ctypes.c_void_p), ("face_centroid", ctypes.c_void_p),
                ("centroid", ctypes.c_void_p), ("volume", ctypes.c_void_p), ("positions", ctypes.c_void_p),
                ("box", ctypes.c_double * 3)]


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        from luna_cpp_b200 import build
        build.build_oracle()
    L = ctypes.CDLL(LIB)
    P, D, I, V = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, None
    sig = {
        "lo_gas_init": ([P, D], V),
        "lo_primitive": ([I, P, P, P], V),
        "lo_conserved": ([I, P, P, P], V),
        "lo_half_step": ([I, P, P, D, P, P], V),
        "lo_hllc_flux": ([I, P, P, P, P, P, P], V),
        "lo_hll_flux": ([I, P, P, P, P, P, P], V),
        "lo_hllc_flux_float": ([I, P, P, P, P, P], V),
        "lo_fv_create": ([P, P, I, I, I, I, I, I, I], P),
        "lo_fv_destroy": ([P], V),
        "lo_fv_state": ([P], P),
        "lo_fv_state_changed": ([P], V),
        "lo_fv_time_step": ([P, D], D),
        "lo_fv_step": ([P, D], V),
        "lo_fv_fallbacks": ([P], ctypes.c_int64),
        "lo_fv_threads": ([I], I),
        "lo_fv_prims": ([P], P),
        "lo_fv_gradients": ([P], P),
        "lo_fv_point_velocities": ([P], P),
        "lo_fv_step_moving_begin": ([P, D, P], V),
        "lo_fv_step_moving_end": ([P, P], V),
        "lo_grid_step": ([I, P], D),
        "lo_fv_set_half_gradients": ([P, I], V),
        "lo_fv_set_float_fluxes": ([P, I], V),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    line_sig = {
        "lo_line_create": ([ctypes.c_int, P, ctypes.c_int64, D, I, P, P, P, I, I, I], P),
        "lo_line_destroy": ([P], V),
        "lo_line_state": ([P], P),
        "lo_line_volumes": ([P], P),
        "lo_line_centroids": ([P], P),
        "lo_line_time_step": ([P, D, I], D),
        "lo_line_step": ([P, D], V),
    }
    LL = ctypes.c_longlong
    line_sig.update({
        "lo_mline_create": ([I, P, D, I, P, P, P, I, I, I, I], P),
        "lo_mline_destroy": ([P], V),
        "lo_mline_cells": ([P], I),
        "lo_mline_state": ([P], P),
        "lo_mline_positions": ([P], P),
        "lo_mline_geometry": ([P, P, P, P], V),
        "lo_mline_stats": ([P, ctypes.POINTER(LL), ctypes.POINTER(LL), ctypes.POINTER(LL)], V),
        "lo_mline_set_inflow_spacing": ([P, D], V),
        "lo_mline_supply_cells": ([P], I),
        "lo_mline_time_step": ([P, D, I], D),
        "lo_mline_step": ([P, D], V),
        "lo_mline_step_and_time_step": ([P, D, D], D),
    })
    for name, (args, res) in line_sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    if hasattr(L, "lo_fv_step_adjoint"):
        L.lo_fv_step_adjoint.argtypes = [P, D, P]
        L.lo_fv_step_adjoint.restype = None
    _lib = L
    return L


def gas(gamma: float = 5.0 / 3.0) -> _Gas:
    g = _Gas()
    lib().lo_gas_init(ctypes.byref(g), gamma)
    return g


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def riemann(L, R, n, w=None, gamma=5.0 / 3.0, solver="hllc"):
    """One flux of HLLC (or HLL) through a face of unit normal n moving with w."""
    D = len(n)
    Lr = np.ascontiguousarray(L, dtype=np.float64)
    Rr = np.ascontiguousarray(R, dtype=np.float64)
    nn = np.ascontiguousarray(n, dtype=np.float64)
    ww = np.zeros(D) if w is None else np.ascontiguousarray(w, dtype=np.float64)
    F = np.zeros(D + 2)
    g = gas(gamma)
    fn = lib().lo_hllc_flux if solver == "hllc" else lib().lo_hll_flux
    fn(D, _ptr(Lr), _ptr(Rr), _ptr(nn), _ptr(ww), ctypes.byref(g), _ptr(F))
    return F


def conserved(W, gamma=5.0 / 3.0):
    W = np.ascontiguousarray(W, dtype=np.float64)
    U = np.zeros_like(W)
    g = gas(gamma)
    D = W.shape[-1] - 2
    flat_W = W.reshape(-1, D + 2)
    flat_U = U.reshape(-1, D + 2)
    for k in range(flat_W.shape[0]):
        lib().lo_conserved(D, _ptr(flat_W[k]), ctypes.byref(g), _ptr(flat_U[k]))
    return U


class OracleFV:
    """The oracle's FiniteVolume<D> on one mesh (luna_cpp_b200.mesh.Mesh)."""

    def __init__(self, mesh, gamma=5.0 / 3.0, order=1, per_face=True, limiter="face_centroid", riemann="hllc",
                 moving=False, precision="double"):
        self._keep = []
        self.mesh = mesh
        self.dim = mesh.dim
        self.V = mesh.dim + 2
        self._gas = gas(gamma)
        m = self._desc(mesh)
        grad_float = 1 if precision in ("grad32", "riemann32", "grad16", "single") else 0
        riemann_float = 1 if precision in ("riemann32", "single") else 0
        self._h = lib().lo_fv_create(ctypes.byref(m), ctypes.byref(self._gas), order, 1 if per_face else 0,
                                      1 if limiter == "none" else 0, 1 if riemann == "hll" else 0,
                                      1 if moving else 0, grad_float, riemann_float)
        if precision == "grad16":
            lib().lo_fv_set_half_gradients(self._h, 1)
        if precision == "single":
            lib().lo_fv_set_float_fluxes(self._h, 1)

    def _desc(self, mesh):
        arrays = [np.ascontiguousarray(x) for x in (mesh.owner, mesh.neighbour, mesh.cell_face_start, mesh.cell_face,
                                                     mesh.area, mesh.face_centroid, mesh.centroid, mesh.volume,
                                                     mesh.positions)]
        self._keep.append(arrays)
        m = _Mesh()
        m.dim = mesh.dim
        m.n = mesh.n_cells
        m.f = mesh.n_faces
        (m.owner, m.neighbour, m.start, m.list, m.area, m.face_centroid, m.centroid, m.volume,
         m.positions) = [a.ctypes.data for a in arrays]
        for a in range(3):
            m.box[a] = mesh.box[a] if a < len(mesh.box) else 0.0
        self._mesh_struct = m
        return m

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().lo_fv_destroy(h)
            self._h = None

    @property
    def n(self):
        return self.mesh.n_cells

    def state(self) -> np.ndarray:
        ptr = lib().lo_fv_state(self._h)
        buf = (ctypes.c_double * (self.n * self.V)).from_address(ptr)
        return np.frombuffer(buf, dtype=np.float64).reshape(self.n, self.V)

    def set_state(self, q):
        self.state()[:] = q

    def get_state(self):
        return self.state().copy()

    def time_step(self, courant=0.3):
        return lib().lo_fv_time_step(self._h, courant)

    def step(self, dt):
        lib().lo_fv_step(self._h, dt)

    def fallbacks(self):
        return int(lib().lo_fv_fallbacks(self._h))

    def prims(self):
        ptr = lib().lo_fv_prims(self._h)
        buf = (ctypes.c_double * (self.n * (self.V + 2))).from_address(ptr)
        return np.frombuffer(buf, dtype=np.float64).reshape(self.n, self.V + 2).copy()

    def gradients(self):
        ptr = lib().lo_fv_gradients(self._h)
        buf = (ctypes.c_double * (self.n * self.V * self.dim)).from_address(ptr)
        return np.frombuffer(buf, dtype=np.float64).reshape(self.n, self.V * self.dim).copy()

    def point_velocities(self):
        ptr = lib().lo_fv_point_velocities(self._h)
        buf = (ctypes.c_double * (self.n * self.dim)).from_address(ptr)
        return np.frombuffer(buf, dtype=np.float64).reshape(self.n, self.dim).copy()

    def step_moving(self, dt, remesh):
        """One moving step; remesh(positions) -> Mesh builds the t^n+1 mesh."""
        pos = np.zeros((self.n, self.dim))
        lib().lo_fv_step_moving_begin(self._h, dt, _ptr(pos))
        new_mesh = remesh(pos)
        self.mesh = new_mesh
        m = self._desc(new_mesh)
        lib().lo_fv_step_moving_end(self._h, ctypes.byref(m))
        self._keep = self._keep[-1:]
        return new_mesh

    def step_adjoint(self, dt, qbar):
        q = np.ascontiguousarray(qbar, dtype=np.float64).copy()
        lib().lo_fv_step_adjoint(self._h, dt, _ptr(q))
        return q


def threads(n: int = 0) -> int:
    return int(lib().lo_fv_threads(n))


WALLS = {"reflective": 0, "outflow": 1, "inflow": 2}
LIMITERS = {"face_centroid": 0, "none": 1, "minmod": 2, "van_leer": 3}
RULES = {"arepo": 0, "luna": 1}


class OracleLine:
    """FiniteVolume<1> on a static line (oracle_line.c): sorted grid keys, walls or periodic; Q [n, 3] in slot order."""

    def __init__(self, keys, step, period=1 << 30, gamma=1.4, walls=("outflow", "outflow"), periodic=False, inflow=None,
                 order=1, limiter="face_centroid", riemann="hllc"):
        self.keys = np.ascontiguousarray(keys, dtype=np.int64)
        self.n = len(self.keys)
        self._gas = gas(gamma)
        w = np.array([WALLS[walls[0]], WALLS[walls[1]]], dtype=np.int32)
        inflow = np.zeros((2, 3)) if inflow is None else np.ascontiguousarray(inflow, dtype=np.float64)
        self._keep = (w, inflow)
        self._h = lib().lo_line_create(self.n, _ptr(self.keys), int(period), float(step), int(periodic), _ptr(w), _ptr(inflow),
                                       ctypes.byref(self._gas), order, LIMITERS[limiter], 0 if riemann == "hllc" else 1)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().lo_line_destroy(self._h)
            self._h = None

    def _view(self, ptr, shape):
        buf = (ctypes.c_double * int(np.prod(shape))).from_address(ptr)
        return np.frombuffer(buf, dtype=np.float64).reshape(shape)

    def set_state(self, q):
        self._view(lib().lo_line_state(self._h), (self.n, 3))[:] = q

    def get_state(self):
        return self._view(lib().lo_line_state(self._h), (self.n, 3)).copy()

    def volumes(self):
        return self._view(lib().lo_line_volumes(self._h), (self.n,)).copy()

    def centroids(self):
        return self._view(lib().lo_line_centroids(self._h), (self.n,)).copy()

    def time_step(self, courant, rule="arepo"):
        return float(lib().lo_line_time_step(self._h, courant, RULES[rule]))

    def step(self, dt):
        lib().lo_line_step(self._h, dt)


class OracleMovingLine:
    """FiniteVolume<1> on a moving line (oracle_mline.c): n generators at `positions` (cell order) on [0, length]; Q and
    x per cell in cell order, cells supplied by open walls appended."""

    def __init__(self, positions, length, gamma=1.4, walls=("outflow", "outflow"), periodic=False, inflow=None, order=1,
                 limiter="face_centroid", riemann="hllc", regularise=True):
        x = np.ascontiguousarray(positions, dtype=np.float64)
        self._gas = gas(gamma)
        w = np.array([WALLS[walls[0]], WALLS[walls[1]]], dtype=np.int32)
        inflow = np.zeros((2, 3)) if inflow is None else np.ascontiguousarray(inflow, dtype=np.float64)
        self._keep = (w, inflow)
        self._h = lib().lo_mline_create(len(x), _ptr(x), float(length), int(periodic), _ptr(w), _ptr(inflow),
                                        ctypes.byref(self._gas), order, LIMITERS[limiter], 0 if riemann == "hllc" else 1,
                                        1 if regularise else 0)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().lo_mline_destroy(self._h)
            self._h = None

    @property
    def n(self):
        return int(lib().lo_mline_cells(self._h))

    def _view(self, ptr, shape):
        buf = (ctypes.c_double * int(np.prod(shape))).from_address(ptr)
        return np.frombuffer(buf, dtype=np.float64).reshape(shape)

    def set_state(self, q):
        self._view(lib().lo_mline_state(self._h), (self.n, 3))[:] = q

    def get_state(self):
        return self._view(lib().lo_mline_state(self._h), (self.n, 3)).copy()

    def positions(self):
        return self._view(lib().lo_mline_positions(self._h), (self.n,)).copy()

    def geometry(self):
        """Per cell: the generator's grid position, the cell's length, its centroid's offset."""
        g, v, c = np.empty(self.n), np.empty(self.n), np.empty(self.n)
        lib().lo_mline_geometry(self._h, _ptr(g), _ptr(v), _ptr(c))
        return g, v, c

    def stats(self):
        a, s, u = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        lib().lo_mline_stats(self._h, ctypes.byref(a), ctypes.byref(s), ctypes.byref(u))
        return {"cells_added": a.value, "sorts": s.value, "updates": u.value}

    def set_inflow_spacing(self, spacing):
        lib().lo_mline_set_inflow_spacing(self._h, float(spacing))

    def supply_cells(self):
        return int(lib().lo_mline_supply_cells(self._h))

    def time_step(self, courant, rule="arepo"):
        return float(lib().lo_mline_time_step(self._h, courant, RULES[rule]))

    def step(self, dt):
        lib().lo_mline_step(self._h, dt)

    def step_and_time_step(self, dt, courant):
        return float(lib().lo_mline_step_and_time_step(self._h, dt, courant))
