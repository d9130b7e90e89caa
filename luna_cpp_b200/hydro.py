"""The host-side mirror of luna-cpp's ``hydro::FiniteVolume<D>`` (src/hydro/finite_volume.hpp:47-239) over the C ABI of
``libluna_b200.so`` (include/luna_b200.h).

Same call order as the reference's drivers (``dt = fv.time_step(courant); fv.step(dt)``), same constructor options
(order, update loop, limiter, motion; the Riemann solver and the precision policy as arguments), same extensive state
Q[N][D + 2]. Errors come back as ``LunaError`` carrying the library's status and message, where the reference throws
``std::invalid_argument`` / ``std::logic_error``. There is no CPU path: without the CUDA library or a GPU, construction
fails.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native

STATUS = {0: "ok", 1: "invalid argument", 2: "out of memory", 3: "CUDA error", 4: "non-finite value",
          5: "device wait timed out", 6: "call out of order"}

UPDATE = {"per_cell": 0, "per_face": 1}
LIMITER = {"face_centroid": 0, "none": 1}
MOTION = {"static_mesh": 0, "static": 0, "moving": 1}
RIEMANN = {"hllc": 0, "hll": 1}
PRECISION = {"fp64": 0, "double": 0, "fp32": 1, "riemann32": 1, "grad32": 2, "grad16": 3, "single": 4}


class LunaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


@dataclass
class Gas:
    """hydro::Gas (euler.hpp:82-101)."""

    gamma: float = 5.0 / 3.0
    smallr: float = 1e-10
    smallc: float = 1e-10


class _Gas(ctypes.Structure):
    _fields_ = [("gamma", ctypes.c_double), ("smallr", ctypes.c_double), ("smallc", ctypes.c_double)]


class MeshDesc(ctypes.Structure):
    """luna_mesh_desc (include/luna_b200.h)."""

    _fields_ = [("dim", ctypes.c_int), ("n_cells", ctypes.c_int64), ("n_faces", ctypes.c_int64),
                ("owner", ctypes.c_void_p), ("neighbour", ctypes.c_void_p), ("cell_face_start", ctypes.c_void_p),
                ("cell_face", ctypes.c_void_p), ("area", ctypes.c_void_p), ("face_centroid", ctypes.c_void_p),
                ("centroid", ctypes.c_void_p), ("volume", ctypes.c_void_p), ("positions", ctypes.c_void_p),
                ("box", ctypes.c_double * 3), ("on_device", ctypes.c_int)]


# Every entry point of include/luna_b200.h with its ctypes signature.
P, I, D64, I64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int64
SIGNATURES = {
    "luna_fv_create": ([P, P, I, I, I, I, I, I, P], I),
    "luna_fv_destroy": ([P], I),
    "luna_fv_set_stream": ([P, P], I),
    "luna_fv_state": ([P, P], I),
    "luna_fv_set_state": ([P, P, I], I),
    "luna_fv_get_state": ([P, P, I], I),
    "luna_fv_time_step": ([P, D64, P], I),
    "luna_fv_step": ([P, D64], I),
    "luna_fv_fallbacks": ([P, P], I),
    "luna_fv_error_word": ([P, P], I),
    "luna_fv_step_moving_begin": ([P, D64, P, I], I),
    "luna_fv_step_moving_end": ([P, P], I),
    "luna_fv_set_mesh": ([P, P], I),
    "luna_fv_positions": ([P, P, I], I),
    "luna_fv_point_velocities": ([P, P, I], I),
    "luna_fv_prims": ([P, P, I], I),
    "luna_fv_gradients": ([P, P, I], I),
    "luna_status_string": ([I], ctypes.c_char_p),
    "luna_last_error": ([], ctypes.c_char_p),
    "luna_fv_device_bytes": ([P, P], I),
    "luna_fv_fused_pass": ([P, P, P], I),
    "luna_fv_step_moving_tangent": ([P, D64, P, P, P, P, P, P, I], I),
    "luna_fv_step_moving_adjoint": ([P, D64, P, P, P, P, P, P, I], I),
    "luna_fv_step_moving_tangent_end": ([P, D64, P, P, P, P, P, P, I], I),
    "luna_fv_step_moving_adjoint_begin": ([P, D64], I),
    "luna_fv_set_steps_fixed": ([P, I], I),
    "luna_fv_step_moving_adjoint_new_mesh": ([P, D64, P, P, P, P, I], I),
    "luna_fv_set_timing": ([P, I], I),
    "luna_fv_step_adjoint": ([P, D64, P, I], I),
    "luna_fv_step_tangent": ([P, D64, P, I], I),
    "luna_apply_static_noalloc": ([P, P, I, I, P, P, P, D64, P, P], I),
    "luna_fv_set_limiter_mlp": ([P, P, I], I),
    "luna_fv_limiter_inputs": ([P, P, P, P], I),
    "luna_mlp_param_count": ([], I64),
    "luna_mlp_set_wait_limit": ([I], I),
    "luna_mlp_train_workspace_floats": ([I64], I64),
    "luna_mlp_forward": ([P, P, I64, P, P], I),
    "luna_mlp_train_step": ([P, P, P, P, I64, ctypes.c_float, P, P, P, I64, P], I),
    "luna_mlp_adam": ([P, P, P, P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, I, P], I),
    "luna_fv_timings": ([P, P, I], I),
    "luna_mesh_tiles": ([P, P, P, P, P, P, P], I),
    "luna_line_create": ([I64, I, P, D64, I, P, P, P, I, I, I, P], I),
    "luna_line_destroy": ([P], I),
    "luna_line_set_stream": ([P, P], I),
    "luna_line_geometry": ([P, P, P], I),
    "luna_line_set_state": ([P, P, I], I),
    "luna_line_get_state": ([P, P, I], I),
    "luna_line_time_step": ([P, D64, I, P], I),
    "luna_line_step": ([P, P], I),
    "luna_line_step_and_time_step": ([P, P, D64, P], I),
    "luna_line_step_tangent": ([P, P, P, I], I),
    "luna_line_step_adjoint": ([P, P, P, I], I),
    "luna_mline_create": ([I64, P, D64, I, P, P, P, I, I, I, I, P], I),
    "luna_mline_destroy": ([P], I),
    "luna_mline_set_stream": ([P, P], I),
    "luna_mline_cells": ([P, P], I),
    "luna_mline_set_state": ([P, P, I], I),
    "luna_mline_get_state": ([P, P, I], I),
    "luna_mline_positions": ([P, P, I], I),
    "luna_mline_geometry": ([P, P, P, P], I),
    "luna_mline_set_inflow_spacing": ([P, D64], I),
    "luna_mline_supply_cells": ([P, P], I),
    "luna_mline_time_step": ([P, D64, I, P], I),
    "luna_mline_step": ([P, D64], I),
    "luna_mline_step_and_time_step": ([P, D64, D64, P], I),
    "luna_mline_stats": ([P, P, P, P], I),
    "luna_remesh_create": ([I, P, P], I),
    "luna_remesh_destroy": ([P], I),
    "luna_remesh_set_stream": ([P, P], I),
    "luna_remesh_points": ([P, I64, P], I),
    "luna_remesh_build": ([P, I64, P, I, P, P], I),
    "luna_remesh_device_bytes": ([P, P], I),
}

PHASES = ("primitives", "sweep", "fluxes", "update", "drift")


class _Timings(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double * 5), ("launches", ctypes.c_int64 * 5)]


def lib():
    L = _native.load("hydro")
    if not getattr(L, "_typed", False):
        for name, (args, res) in SIGNATURES.items():
            if hasattr(L, name):
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = res
        L._typed = True
    return L


def check(status: int):
    if status != 0:
        raise LunaError(status, lib().luna_last_error().decode())


def mesh_desc(mesh, keep: list) -> MeshDesc:
    """A luna_mesh_desc over the host arrays of a luna_cpp_b200.mesh.Mesh (kept alive through ``keep``), or the device
    descriptor of a luna_cpp_b200.remesh.DeviceMesh."""
    if isinstance(getattr(mesh, "desc", None), MeshDesc):
        return mesh.desc
    arrays = [np.ascontiguousarray(mesh.owner, dtype=np.int32), np.ascontiguousarray(mesh.neighbour, dtype=np.int32),
              np.ascontiguousarray(mesh.cell_face_start, dtype=np.int32),
              np.ascontiguousarray(mesh.cell_face, dtype=np.int32), np.ascontiguousarray(mesh.area, dtype=np.float64),
              np.ascontiguousarray(mesh.face_centroid, dtype=np.float64),
              np.ascontiguousarray(mesh.centroid, dtype=np.float64), np.ascontiguousarray(mesh.volume, dtype=np.float64),
              np.ascontiguousarray(mesh.positions, dtype=np.float64)]
    keep.append(arrays)
    d = MeshDesc()
    d.dim = mesh.dim
    d.n_cells = mesh.n_cells
    d.n_faces = mesh.n_faces
    (d.owner, d.neighbour, d.cell_face_start, d.cell_face, d.area, d.face_centroid, d.centroid, d.volume,
     d.positions) = [a.ctypes.data for a in arrays]
    for a in range(3):
        d.box[a] = mesh.box[a] if a < len(mesh.box) else 0.0
    d.on_device = 0
    return d


def mesh_tiles(mesh) -> dict:
    """The sweep's tiles of a host mesh (luna_mesh_tiles; host work only): counts and arrays."""
    keep = []
    desc = mesh_desc(mesh, keep)
    counts = np.zeros(6, np.int64)
    check(lib().luna_mesh_tiles(ctypes.byref(desc), counts.ctypes.data, None, None, None, None, None))
    tiles, normal, staged, slots, most, most_single = (int(c) for c in counts)
    out = {"tiles": tiles, "normal_tiles": normal, "most_rows": most, "most_rows_single": most_single,
           "order": np.empty(tiles * 128, np.int32), "slice_base": np.empty(tiles * 4 + 1, np.int32),
           "stage_start": np.empty(tiles + 1, np.int32), "stage_cells": np.empty(staged, np.int32),
           "local": np.empty(slots, np.uint32)}
    check(lib().luna_mesh_tiles(ctypes.byref(desc), counts.ctypes.data, out["order"].ctypes.data, out["slice_base"].ctypes.data,
                                out["stage_start"].ctypes.data, out["stage_cells"].ctypes.data, out["local"].ctypes.data))
    return out


class FiniteVolume:
    """hydro::FiniteVolume<D, Cuda, Riemann, Precision> on one GPU (the current device)."""

    def __init__(self, mesh, gas: Gas | None = None, order: int = 1, update: str = "per_face",
                 limiter: str = "face_centroid", motion: str = "static_mesh", riemann: str = "hllc",
                 precision: str = "fp64"):
        self.mesh = mesh
        self.dim = mesh.dim
        self.V = mesh.dim + 2
        self.n = mesh.n_cells
        self.gas = gas or Gas()
        g = _Gas(self.gas.gamma, self.gas.smallr, self.gas.smallc)
        keep: list = []
        desc = mesh_desc(mesh, keep)
        h = ctypes.c_void_p()
        check(lib().luna_fv_create(ctypes.byref(desc), ctypes.byref(g), order, UPDATE[update], LIMITER[limiter],
                                   MOTION[motion], RIEMANN[riemann], PRECISION[precision], ctypes.byref(h)))
        self._h = h
        self.order, self.update, self.limiter, self.motion = order, update, limiter, motion
        self.riemann, self.precision = riemann, precision

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            lib().luna_fv_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # ---- state ----
    def state_ptr(self) -> int:
        """state(): the device pointer of Q[N][V]; the primitive rows are recomputed by the next time_step()."""
        p = ctypes.c_void_p()
        check(lib().luna_fv_state(self._h, ctypes.byref(p)))
        return int(p.value)

    def set_state(self, q) -> None:
        """Q from host (numpy) or device memory (a CUDA torch tensor, contiguous float64 [N, V])."""
        if hasattr(q, "is_cuda") and q.is_cuda:
            check(lib().luna_fv_set_state(self._h, ctypes.c_void_p(q.data_ptr()), 1))
            return
        a = np.ascontiguousarray(q, dtype=np.float64)
        if a.shape != (self.n, self.V):
            raise ValueError(f"state must be [{self.n}, {self.V}]")
        check(lib().luna_fv_set_state(self._h, a.ctypes.data, 0))

    def get_state(self, out=None):
        if out is not None and hasattr(out, "is_cuda") and out.is_cuda:
            check(lib().luna_fv_get_state(self._h, ctypes.c_void_p(out.data_ptr()), 1))
            return out
        a = np.empty((self.n, self.V), dtype=np.float64) if out is None else out
        check(lib().luna_fv_get_state(self._h, a.ctypes.data, 0))
        return a

    # ---- the step ----
    def time_step(self, courant: float = 0.3) -> float:
        dt = ctypes.c_double()
        check(lib().luna_fv_time_step(self._h, courant, ctypes.byref(dt)))
        return dt.value

    def step(self, dt: float) -> None:
        check(lib().luna_fv_step(self._h, dt))

    def step_moving(self, dt: float, remesh) -> object:
        """One moving step: the t^n fluxes, the drift, ``remesh(positions) -> Mesh`` (the mesh library's update), the
        t^n+1 fluxes. Returns the new mesh."""
        pos = np.empty((self.n, self.dim), dtype=np.float64)
        check(lib().luna_fv_step_moving_begin(self._h, dt, pos.ctypes.data, 0))
        new_mesh = remesh(pos)
        keep: list = []
        desc = mesh_desc(new_mesh, keep)
        check(lib().luna_fv_step_moving_end(self._h, ctypes.byref(desc)))
        self.mesh = new_mesh
        return new_mesh

    def step_moving_device(self, dt: float, remesher) -> object:
        """One moving step with the generators and the mesh on the device: the t^n fluxes, the drift into the
        remesher's buffer, ``remesher``'s device remesh (luna_cpp_b200.remesh.Remesher), the t^n+1 fluxes. Returns the
        new DeviceMesh."""
        ptr = remesher.points_buffer(self.n)
        check(lib().luna_fv_step_moving_begin(self._h, dt, ptr, 1))
        new_mesh = remesher.build_device(ptr, self.n)
        check(lib().luna_fv_step_moving_end(self._h, ctypes.byref(new_mesh.desc)))
        self.mesh = new_mesh
        return new_mesh

    def set_mesh(self, mesh) -> None:
        keep: list = []
        desc = mesh_desc(mesh, keep)
        check(lib().luna_fv_set_mesh(self._h, ctypes.byref(desc)))
        self.mesh = mesh

    def fallbacks(self) -> int:
        out = ctypes.c_int64()
        check(lib().luna_fv_fallbacks(self._h, ctypes.byref(out)))
        return int(out.value)

    def error_word(self) -> int:
        out = ctypes.c_uint32()
        check(lib().luna_fv_error_word(self._h, ctypes.byref(out)))
        return int(out.value)

    # ---- rows ----
    def prims(self) -> np.ndarray:
        a = np.empty((self.n, self.V + 2), dtype=np.float64)
        check(lib().luna_fv_prims(self._h, a.ctypes.data, 0))
        return a

    def gradients(self) -> np.ndarray:
        a = np.empty((self.n, self.V * self.dim), dtype=np.float64)
        check(lib().luna_fv_gradients(self._h, a.ctypes.data, 0))
        return a

    def point_velocities(self) -> np.ndarray:
        a = np.empty((self.n, self.dim), dtype=np.float64)
        check(lib().luna_fv_point_velocities(self._h, a.ctypes.data, 0))
        return a

    def positions(self) -> np.ndarray:
        a = np.empty((self.n, self.dim), dtype=np.float64)
        check(lib().luna_fv_positions(self._h, a.ctypes.data, 0))
        return a

    def step_adjoint(self, dt: float, qbar):
        """J^T qbar of one step at fixed dt from the current state (which must be the step's start); numpy in, numpy out,
        or a CUDA float64 tensor updated in place."""
        if hasattr(qbar, "is_cuda") and qbar.is_cuda:
            check(lib().luna_fv_step_adjoint(self._h, dt, ctypes.c_void_p(qbar.data_ptr()), 1))
            return qbar
        a = np.ascontiguousarray(qbar, dtype=np.float64).copy()
        check(lib().luna_fv_step_adjoint(self._h, dt, a.ctypes.data, 0))
        return a

    def step_tangent(self, dt: float, dq):
        """step(dt) with the tangent dq -> J dq beside it (fixed dt); numpy in, numpy out, or a CUDA float64 tensor
        updated in place."""
        if hasattr(dq, "is_cuda") and dq.is_cuda:
            check(lib().luna_fv_step_tangent(self._h, dt, ctypes.c_void_p(dq.data_ptr()), 1))
            return dq
        a = np.ascontiguousarray(dq, dtype=np.float64).copy()
        check(lib().luna_fv_step_tangent(self._h, dt, a.ctypes.data, 0))
        return a

    def set_steps_fixed(self, held: bool = True) -> None:
        """The order-1 moving derivatives with the grid steps held (the reference's steps_fixed)."""
        check(lib().luna_fv_set_steps_fixed(self._h, 1 if held else 0))

    @staticmethod
    def _geometry_of(geometry):
        """A GeometryDerivative factory (mesh -> derivative) from a factory or class, or from one derivative object."""
        if isinstance(geometry, type) or not hasattr(geometry, "tangent"):
            return geometry
        return lambda mesh: geometry

    def step_moving_tangent(self, dt: float, dq, dx, geometry, remesh=None):
        """The moving step's tangent at fixed topology (luna_fv_step_moving_tangent): (dq, dx) of (Q, x) at the step's
        start -> after it. ``geometry``: a GeometryDerivative (``tangent(dx) -> dV, dc, dA, dxf``) of the current mesh,
        or a factory of one from a mesh (e.g. luna_cpp_b200.geometry_derivative.Geometry2D). Order 0: nothing steps
        unless ``remesh`` (positions -> Mesh) is given, then the step follows. Order 1: ``remesh`` is required and the
        step runs between the two passes' tangents (the reference's step_moving_tangent steps too). Returns (dq, dx)."""
        make = self._geometry_of(geometry)
        q = np.ascontiguousarray(dq, dtype=np.float64).copy()
        x = np.ascontiguousarray(dx, dtype=np.float64).copy()
        dV, dc, dA, dxf = (np.ascontiguousarray(a, dtype=np.float64) for a in make(self.mesh).tangent(x))
        check(lib().luna_fv_step_moving_tangent(self._h, dt, q.ctypes.data, x.ctypes.data, dV.ctypes.data, dc.ctypes.data,
                                                dA.ctypes.data, dxf.ctypes.data, 0))
        if self.order == 1:
            if remesh is None:
                raise ValueError("the order-1 moving tangent needs remesh: its second pass is on the new mesh")
            self.step_moving(dt, remesh)
            dV, dc, dA, dxf = (np.ascontiguousarray(a, dtype=np.float64) for a in make(self.mesh).tangent(x))
            check(lib().luna_fv_step_moving_tangent_end(self._h, dt, q.ctypes.data, x.ctypes.data, dV.ctypes.data,
                                                        dc.ctypes.data, dA.ctypes.data, dxf.ctypes.data, 0))
        elif remesh is not None:
            self.step_moving(dt, remesh)
        return q, x

    def step_moving_adjoint(self, dt: float, qbar, xbar, geometry, remesh=None):
        """The moving step's adjoint (luna_fv_step_moving_adjoint), the geometry's part through ``geometry``'s
        ``adjoint(Vbar, cbar, Abar, xfbar) -> xbar`` (a derivative object or a factory from a mesh): (qbar, xbar) after
        the step -> at its start. The state and the mesh must be the step's start. Order 1: ``remesh`` is required; the
        step runs to the new mesh for the second pass and the start is restored after. Returns (qbar, xbar)."""
        make = self._geometry_of(geometry)
        q = np.ascontiguousarray(qbar, dtype=np.float64).copy()
        x = np.ascontiguousarray(xbar, dtype=np.float64).copy()
        N, D = self.n, self.dim
        start_mesh = self.mesh
        if self.order == 1:
            if remesh is None:
                raise ValueError("the order-1 moving adjoint needs remesh: its second pass is on the new mesh")
            check(lib().luna_fv_step_moving_adjoint_begin(self._h, dt))
            q_start = self.get_state()
            self.step_moving(dt, remesh)
            F2 = int(self.mesh.n_faces)
            Ab2, xfb2 = np.empty((F2, D)), np.empty((F2, D))
            check(lib().luna_fv_step_moving_adjoint_new_mesh(self._h, dt, q.ctypes.data, x.ctypes.data, Ab2.ctypes.data,
                                                             xfb2.ctypes.data, 0))
            x = x + make(self.mesh).adjoint(np.zeros(N), np.zeros((N, D)), Ab2, xfb2)
            self.set_mesh(start_mesh)
            self.set_state(q_start)
        F = int(start_mesh.n_faces)
        Vb, cb, Ab, xfb = np.empty(N), np.empty((N, D)), np.empty((F, D)), np.empty((F, D))
        check(lib().luna_fv_step_moving_adjoint(self._h, dt, q.ctypes.data, x.ctypes.data, Vb.ctypes.data, cb.ctypes.data,
                                                Ab.ctypes.data, xfb.ctypes.data, 0))
        return q, x + make(start_mesh).adjoint(Vb, cb, Ab, xfb)

    def set_limiter(self, mode: str = "plain", params=None) -> None:
        """The slope limiter of the sweep: "plain" (the reference's), "learned" (the MLP with ``params``, a CUDA float32
        tensor the caller keeps alive), or "factors" (the plain limiter in min-factor form through the learned path)."""
        code = {"plain": 0, "learned": 1, "factors": 2}[mode]
        self._limiter_params = params
        ptr = ctypes.c_void_p(params.data_ptr()) if params is not None else None
        check(lib().luna_fv_set_limiter_mlp(self._h, ptr, code))

    def limiter_inputs(self):
        """(features [N, 32] bf16, alpha [N, 5] float64, unlimited gradients [N, V*D] float64) as CUDA tensors."""
        import torch

        f = torch.empty((self.n, 32), dtype=torch.bfloat16, device="cuda")
        a = torch.empty((self.n, 5), dtype=torch.float64, device="cuda")
        g = torch.empty((self.n, self.V * self.dim), dtype=torch.float64, device="cuda")
        check(lib().luna_fv_limiter_inputs(self._h, ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(a.data_ptr()),
                                           ctypes.c_void_p(g.data_ptr())))
        return f, a, g

    def set_stream(self, stream_ptr: int) -> None:
        check(lib().luna_fv_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def set_timing(self, on: bool = True) -> None:
        check(lib().luna_fv_set_timing(self._h, 1 if on else 0))

    def timings(self, reset: bool = True) -> dict:
        """{phase: (ms, launches)} since the last reset (hydro::Timings)."""
        t = _Timings()
        check(lib().luna_fv_timings(self._h, ctypes.byref(t), 1 if reset else 0))
        return {name: (t.ms[k], int(t.launches[k])) for k, name in enumerate(PHASES)}

    def fused_pass(self) -> tuple:
        """(whether the static steps run the fused flux-and-update pass, the faces between its tiles)."""
        fused, crossing = ctypes.c_int(), ctypes.c_int64()
        check(lib().luna_fv_fused_pass(self._h, ctypes.byref(fused), ctypes.byref(crossing)))
        return bool(fused.value), int(crossing.value)

    def device_bytes(self) -> int:
        out = ctypes.c_int64()
        check(lib().luna_fv_device_bytes(self._h, ctypes.byref(out)))
        return int(out.value)
