"""Locating and loading the package's native libraries (built in-tree by ``luna_cpp_b200.build``).

The hydro step has no CPU fallback: if ``libluna_b200.so`` is missing the import of the hydro module fails with the
command that builds it.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))

LIBS = {
    "mesh": "libluna_mesh.so",
    "hydro": "libluna_b200.so",
}


def lib_path(name: str) -> str:
    return os.path.join(HERE, LIBS[name])


_loaded: dict[str, ctypes.CDLL] = {}


def load(name: str) -> ctypes.CDLL:
    if name in _loaded:
        return _loaded[name]
    path = lib_path(name)
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is not built; run `python -m luna_cpp_b200.build`")
    lib = ctypes.CDLL(path)
    _loaded[name] = lib
    return lib
