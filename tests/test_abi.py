"""The C ABI: the library loads without a GPU and exports every entry point include/*.h declares."""
import ctypes
import os
import re

import pytest

from luna_cpp_b200 import _native, hydro

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"LUNA_API[^;(]*?\b(luna_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared()
    assert "luna_fv_create" in names and "luna_fv_time_step" in names and "luna_fv_step" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_native.lib_path("hydro"))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_symbol():
    assert set(declared()) <= set(hydro.SIGNATURES) | {"luna_fv_step_static"}


def test_status_strings_without_gpu():
    lib = hydro.lib()
    assert lib.luna_status_string(0) == b"ok"
    assert lib.luna_status_string(1) == b"invalid argument"


def test_create_rejects_bad_order_without_touching_the_gpu():
    """The reference throws invalid_argument on order not in {0, 1} (finite_volume.hpp:83); the C ABI returns EINVAL."""
    from conftest import jittered_mesh

    m = jittered_mesh(8)
    with pytest.raises(hydro.LunaError) as e:
        hydro.FiniteVolume(m, order=2)
    assert e.value.status == 1


def test_remesher_rejects_bad_arguments_without_touching_the_gpu():
    """luna_remesh_create checks its arguments before any CUDA call: EINVAL (1) with a message."""
    lib = hydro.lib()
    h = ctypes.c_void_p()
    box = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    assert lib.luna_remesh_create(4, box, ctypes.byref(h)) == 1
    assert b"dim" in lib.luna_last_error()
    bad = (ctypes.c_double * 3)(1.0, -1.0, 1.0)
    assert lib.luna_remesh_create(3, bad, ctypes.byref(h)) == 1
    assert lib.luna_remesh_create(3, None, ctypes.byref(h)) == 1
    assert lib.luna_remesh_build(None, 10, None, 0, None, None) == 1
    assert lib.luna_remesh_destroy(None) == 0
