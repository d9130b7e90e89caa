"""In-tree build of the native libraries: ``python -m luna_cpp_b200.build [hydro|mesh|oracle|all]``.

- ``libluna_b200.so``: the hydro step, CUDA for sm_100a only (nvcc -gencode arch=compute_100a,code=sm_100a), C ABI in
  include/luna_b200.h, and the device remesher of the moving mesh (include/luna_remesh.h);
- ``libluna_mesh.so``: the periodic Voronoi mesh builder (host C++, OpenMP);
- ``oracle/liboracle.so``: the CPU oracle the tests check against (plain C, no multiply-add contraction);
- ``oracle/_ref/libluna_ref.so``: the reference's own solver compiled on the CPU (``oracle/Makefile``), which pins the
  oracle; built only where the reference's source tree is present (the Makefile names it), kept otherwise.
The libraries are built next to their sources so they travel with the tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
ORACLE = os.path.join(ROOT, "oracle")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _run(cmd, cwd=None):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=cwd)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources(directory, exts):
    out = []
    for dirpath, _, files in os.walk(directory):
        for f in files:
            if os.path.splitext(f)[1] in exts:
                out.append(os.path.join(dirpath, f))
    return sorted(out)


def build_mesh(force=False):
    target = os.path.join(PKG, "libluna_mesh.so")
    srcs = [os.path.join(CSRC, "mesh", "voronoi_build.cpp")]
    headers = [os.path.join(CSRC, "mesh", h) for h in ("luna_mesh.h", "voronoi_cell.h", "voronoi_grid.h")]
    if force or _stale(target, srcs + headers):
        # no contraction: the device remesher compiles the same cell code with -fmad=false and must match it bit for bit
        _run(["g++", "-O3", "-std=c++17", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-Wall", "-o", target] + srcs)
    return target


def build_oracle(force=False):
    target = os.path.join(ORACLE, "liboracle.so")
    srcs = [os.path.join(ORACLE, f) for f in sorted(os.listdir(ORACLE)) if f.endswith(".c")]
    if force or _stale(target, srcs + [os.path.join(ORACLE, "luna_oracle.h")]):
        _run(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared", "-Wall",
              "-Wno-maybe-uninitialized", "-o", target] + srcs + ["-lm"])
    return target


NO_CONTRACTION = {"moving_line.cu"}


def build_hydro(force=False, extra=()):
    target = os.path.join(PKG, "libluna_b200.so")
    hydro = os.path.join(CSRC, "hydro")
    mesh = os.path.join(CSRC, "mesh")
    cu = [s for s in _sources(hydro, {".cu"})]
    remesh = os.path.join(mesh, "remesh.cu")
    remesh_deps = [remesh] + [os.path.join(mesh, h) for h in ("voronoi_cell.h", "voronoi_grid.h")]
    deps = _sources(hydro, {".cu", ".cuh", ".h", ".hpp"}) + _sources(INCLUDE, {".h"}) + remesh_deps
    if not cu:
        return None
    if force or _stale(target, deps):
        # One object per source, compiled in parallel, then one link. The device remesher runs the host mesh builder's
        # cell code and must give its bits: no multiply-add contraction in that object (the hydro kernels keep it).
        from concurrent.futures import ThreadPoolExecutor

        obj_dir = os.path.join(PKG, "_build")
        os.makedirs(obj_dir, exist_ok=True)
        remesh_obj = os.path.join(obj_dir, "remesh.o")
        jobs = [[_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler",
                 "-ffp-contract=off", "-Xcompiler", "-fvisibility=hidden", "-c", "-I", INCLUDE, "-I", mesh, "-o",
                 remesh_obj, remesh]]
        objs = [remesh_obj]
        for src in cu:
            obj = os.path.join(obj_dir, os.path.splitext(os.path.basename(src))[0] + ".o")
            objs.append(obj)
            # the moving line's grid steps depend on the last bit of each point velocity: the reference's operation
            # order, no contraction
            exact = ["-fmad=false"] if os.path.basename(src) in NO_CONTRACTION else []
            jobs.append([_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler",
                         "-fPIC", "-Xcompiler", "-fvisibility=hidden", *exact, "-c", "-I", INCLUDE, "-I", hydro, *extra,
                         "-o", obj, src])
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as pool:
            for _ in pool.map(_run, jobs):
                pass
        _run([_nvcc(), *ARCH, "-shared", "-o", target, *objs, "-lcudart"])
    return target


def build_reference(force=False):
    """The reference's solver on the CPU (test infrastructure): make -C oracle. Without the reference's source tree a
    library built earlier is kept; without either, the tests that need it skip."""
    target = os.path.join(ORACLE, "_ref", "libluna_ref.so")
    cmd = ["make", "-s", "-C", ORACLE, "-j3"] + (["-B"] if force else [])
    try:
        _run(cmd)
    except subprocess.CalledProcessError:
        print("the reference's solver was not built (its source tree is not here)"
              + ("; keeping the library built earlier" if os.path.exists(target) else ""), flush=True)
    return target


def build_all(force=False):
    build_mesh(force)
    build_oracle(force)
    build_reference(force)
    build_hydro(force)


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    force = "--force" in sys.argv
    {"all": build_all, "hydro": build_hydro, "mesh": build_mesh, "oracle": build_oracle,
     "reference": build_reference}[what](force)
