"""The 1D solver, luna-cpp's ``hydro::FiniteVolume<1>`` (src/hydro/finite_volume_1d.hpp), through the C ABI: on a static
line (``Line``, ``luna_line_*`` in include/luna_b200.h), a batch of independent lines sharing one geometry, all stepped
by one launch; on a moving line (``MovingLine``, ``luna_mline_*``), one line whose points move with the gas and whose
open walls supply cells.

    ln = Line(positions, length, walls=("outflow", "outflow"), lines=1, gamma=1.4)
    ln.set_state(q)                      # [lines, n, 3] or [n, 3]: rho, rho v, E (extensive), caller's cell order
    t = run_to(ln, t_end, courant=0.8, rule="luna")
    W = ln.primitives()

Mirrors the reference's interface: time_step(courant, rule) -> dt (per line), step(dt), step_and_time_step(dt, courant),
step_tangent(dt, dq), step_adjoint(dt, qbar); the moving line's also positions(), cells(), cells_added(),
supply_cells(), set_inflow_spacing(spacing).
No CPU fallback: the library must be built (``python -m luna_cpp_b200.build``) and a GPU present.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .hydro import Gas, _Gas, check, lib

WALLS = {"reflective": 0, "outflow": 1, "inflow": 2}
LIMITERS = {"face_centroid": 0, "none": 1, "minmod": 2, "van_leer": 3}
RULES = {"arepo": 0, "luna": 1}


class Line:
    def __init__(self, positions, length: float, walls=("outflow", "outflow"), periodic=False, inflow=None, lines: int = 1,
                 gamma: float = 1.4, order: int = 1, limiter: str = "face_centroid", riemann: str = "hllc"):
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        self.n, self.lines, self.gamma = int(pos.shape[0]), int(lines), float(gamma)
        g = Gas(gamma)
        self._gas = _Gas(g.gamma, g.smallr, g.smallc)
        w = np.array([WALLS[walls[0]], WALLS[walls[1]]], dtype=np.int32)
        inflow_arr = None if inflow is None else np.ascontiguousarray(inflow, dtype=np.float64).reshape(2, 3)
        self._h = ctypes.c_void_p()
        check(lib().luna_line_create(self.n, self.lines, pos.ctypes.data, float(length), int(bool(periodic)), w.ctypes.data,
                                     None if inflow_arr is None else inflow_arr.ctypes.data, ctypes.byref(self._gas), int(order),
                                     LIMITERS[limiter], 0 if riemann == "hllc" else 1, ctypes.byref(self._h)))
        self.volume = np.zeros(self.n)
        self.centroid = np.zeros(self.n)
        check(lib().luna_line_geometry(self._h, self.volume.ctypes.data, self.centroid.ctypes.data))

    def close(self):
        if getattr(self, "_h", None):
            lib().luna_line_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def set_state(self, q) -> None:
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(q, dtype=np.float64), (self.lines, self.n, 3)))
        check(lib().luna_line_set_state(self._h, a.ctypes.data, 0))

    def get_state(self) -> np.ndarray:
        out = np.empty((self.lines, self.n, 3))
        check(lib().luna_line_get_state(self._h, out.ctypes.data, 0))
        return out

    def primitives(self) -> np.ndarray:
        """W = (rho, v, P) per cell from the state (without the floors)."""
        U = self.get_state() / self.volume[None, :, None]
        rho = U[..., 0]
        v = U[..., 1] / rho
        return np.stack([rho, v, (self.gamma - 1) * (U[..., 2] - 0.5 * rho * v * v)], axis=-1)

    def time_step(self, courant: float, rule: str = "arepo") -> np.ndarray:
        out = np.empty(self.lines)
        check(lib().luna_line_time_step(self._h, float(courant), RULES[rule], out.ctypes.data))
        return out

    def step(self, dt) -> None:
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (self.lines,)))
        check(lib().luna_line_step(self._h, d.ctypes.data))

    def step_and_time_step(self, dt, courant: float) -> np.ndarray:
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (self.lines,)))
        out = np.empty(self.lines)
        check(lib().luna_line_step_and_time_step(self._h, d.ctypes.data, float(courant), out.ctypes.data))
        return out

    def step_tangent(self, dt, dq) -> np.ndarray:
        """step_tangent(dt, dq) (finite_volume_1d.hpp:852-883): returns J dq (the step's Jacobian at fixed dt, extensive
        on both sides) and advances the state by the step."""
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (self.lines,)))
        x = np.ascontiguousarray(np.broadcast_to(np.asarray(dq, dtype=np.float64), (self.lines, self.n, 3))).copy()
        check(lib().luna_line_step_tangent(self._h, d.ctypes.data, x.ctypes.data, 0))
        return x

    def step_adjoint(self, dt, qbar) -> np.ndarray:
        """step_adjoint(dt, qbar) (finite_volume_1d.hpp:885-923): returns J^T qbar; the state stays the step's start."""
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (self.lines,)))
        x = np.ascontiguousarray(np.broadcast_to(np.asarray(qbar, dtype=np.float64), (self.lines, self.n, 3))).copy()
        check(lib().luna_line_step_adjoint(self._h, d.ctypes.data, x.ctypes.data, 0))
        return x


class MovingLine:
    """FiniteVolume<1> with Motion::moving (finite_volume_1d.hpp:41-56): n points at `positions` (cell order) on
    [0, length]; the state Q [cells, 3] and the positions in cell order, cells from the walls appended."""

    def __init__(self, positions, length: float, walls=("outflow", "outflow"), periodic=False, inflow=None, gamma: float = 1.4,
                 order: int = 1, limiter: str = "face_centroid", riemann: str = "hllc", regularise: bool = True):
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        self.lines, self.gamma = 1, float(gamma)
        g = Gas(gamma)
        self._gas = _Gas(g.gamma, g.smallr, g.smallc)
        w = np.array([WALLS[walls[0]], WALLS[walls[1]]], dtype=np.int32)
        inflow_arr = None if inflow is None else np.ascontiguousarray(inflow, dtype=np.float64).reshape(2, 3)
        self._h = ctypes.c_void_p()
        check(lib().luna_mline_create(int(pos.shape[0]), pos.ctypes.data, float(length), int(bool(periodic)), w.ctypes.data,
                                      None if inflow_arr is None else inflow_arr.ctypes.data, ctypes.byref(self._gas), int(order),
                                      LIMITERS[limiter], 0 if riemann == "hllc" else 1, 1 if regularise else 0, ctypes.byref(self._h)))

    def close(self):
        if getattr(self, "_h", None):
            lib().luna_mline_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def n(self) -> int:
        out = ctypes.c_int64()
        check(lib().luna_mline_cells(self._h, ctypes.byref(out)))
        return int(out.value)

    def cells(self) -> int:
        return self.n

    def set_state(self, q) -> None:
        a = np.ascontiguousarray(q, dtype=np.float64).reshape(self.n, 3)
        check(lib().luna_mline_set_state(self._h, a.ctypes.data, 0))

    def get_state(self) -> np.ndarray:
        out = np.empty((self.n, 3))
        check(lib().luna_mline_get_state(self._h, out.ctypes.data, 0))
        return out

    def positions(self) -> np.ndarray:
        out = np.empty(self.n)
        check(lib().luna_mline_positions(self._h, out.ctypes.data, 0))
        return out

    def geometry(self):
        """Per cell: the generator's grid position, the cell's length, its centroid's offset from the generator."""
        n = self.n
        g, v, c = np.empty(n), np.empty(n), np.empty(n)
        check(lib().luna_mline_geometry(self._h, g.ctypes.data, v.ctypes.data, c.ctypes.data))
        return g, v, c

    def primitives(self) -> np.ndarray:
        _, volume, _ = self.geometry()
        U = self.get_state() / volume[:, None]
        rho = U[:, 0]
        v = U[:, 1] / rho
        return np.stack([rho, v, (self.gamma - 1) * (U[:, 2] - 0.5 * rho * v * v)], axis=-1)

    def stats(self) -> dict:
        a, s, u = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(lib().luna_mline_stats(self._h, ctypes.byref(a), ctypes.byref(s), ctypes.byref(u)))
        return {"cells_added": a.value, "sorts": s.value, "updates": u.value}

    def cells_added(self) -> int:
        return self.stats()["cells_added"]

    def set_inflow_spacing(self, spacing: float) -> None:
        check(lib().luna_mline_set_inflow_spacing(self._h, float(spacing)))

    def supply_cells(self) -> int:
        out = ctypes.c_int()
        check(lib().luna_mline_supply_cells(self._h, ctypes.byref(out)))
        return int(out.value)

    def time_step(self, courant: float, rule: str = "arepo") -> np.ndarray:
        out = ctypes.c_double()
        check(lib().luna_mline_time_step(self._h, float(courant), RULES[rule], ctypes.byref(out)))
        return np.array([out.value])

    def step(self, dt) -> None:
        check(lib().luna_mline_step(self._h, float(np.asarray(dt).reshape(-1)[0])))

    def step_and_time_step(self, dt, courant: float) -> np.ndarray:
        out = ctypes.c_double()
        check(lib().luna_mline_step_and_time_step(self._h, float(np.asarray(dt).reshape(-1)[0]), float(courant), ctypes.byref(out)))
        return np.array([out.value])


def run_to(ln: Line, t_end, courant: float = 0.8, rule: str = "luna", fused: bool = False, max_steps: int = 10 ** 7):
    """Every line to t_end (scalar or per line), the last step of each shortened to land on it, as the reference's
    drivers do (hydro1d_test.cpp:100-110); lines that arrived take dt = 0. fused: step_and_time_step (LUNA's rule)
    after a first time_step. Returns the steps each line took."""
    t_end = np.broadcast_to(np.asarray(t_end, dtype=np.float64), (ln.lines,)).copy()
    t = np.zeros(ln.lines)
    steps = np.zeros(ln.lines, dtype=np.int64)
    dt_next = ln.time_step(courant, rule)
    for _ in range(max_steps):
        active = t < t_end * (1 - 1e-12)
        if not active.any():
            break
        dt = np.where(active, np.minimum(dt_next, t_end - t), 0.0)
        if fused:
            dt_next = ln.step_and_time_step(dt, courant)
        else:
            ln.step(dt)
            dt_next = ln.time_step(courant, rule)
        t += dt
        steps += active
    return steps
