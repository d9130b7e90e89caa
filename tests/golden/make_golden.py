"""Generates the golden fixtures from the reference's own test files (read as text).

- luna_riemann.json: LUNA's HLL and HLLC fluxes (jax, float64) that luna-cpp's src/test/hydro_test.cpp:48-80 pins its
  Riemann solvers to (relative max-norm difference < 1e-14, gamma 5/3, axis normals);
- luna_1d_final_states.json: LUNA's final states at N = 16 (MC limiter, HLLC, CFL 0.8) of Sod, Shu-Osher and
  Woodward-Colella, src/test/luna_1d_values.hpp, that src/test/hydro1d_test.cpp:266-296 pins FiniteVolume<1> to
  (|W - W_luna| / (1e-3 + |W_luna|) < 1e-12, the same step count);
- luna_1d_derivatives.json: LUNA's jax.jvp and jax.vjp of five fixed-dt steps of its 1D hydro (HLLC, FP64, N = 64),
  src/test/luna_derivative_values.hpp, that src/test/hydro_derivatives_test.cpp:991-1088 pins
  FiniteVolume<1>::step_tangent / step_adjoint to (forward 1e-12, J dU and J^T w 1e-8 of LUNA's largest entry; the
  flat Sod with MC reported, not gated).
Run in a tree that has the reference:
    python tests/golden/make_golden.py /path/to/luna-cpp
"""
import json
import os
import re
import sys


def parse(text, name):
    block = re.search(r"const LunaCase " + name + r"\[\] = \{(.*?)\n\};", text, re.S).group(1)
    cases = []
    for line in block.strip().splitlines():
        line = line.strip()
        if not line.startswith("{"):
            continue
        nums = [float(x) for x in re.findall(r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?", line)]
        axis, rest = int(nums[0]), nums[1:]
        cases.append({"axis": axis, "L": rest[0:5], "R": rest[5:10], "F": rest[10:15]})
    return cases


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_golden.py <luna-cpp source tree>")
    root = sys.argv[1]
    with open(os.path.join(root, "src/test/hydro_test.cpp")) as f:
        text = f.read()
    out = {
        "source": "luna-cpp src/test/hydro_test.cpp:48-80 (LUNA hll_flux_primitive / hllc_flux_primitive, jax x64)",
        "gamma": 5.0 / 3.0,
        "tolerance": 1e-14,
        "hll": parse(text, "luna_hll"),
        "hllc": parse(text, "luna_hllc"),
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "luna_riemann.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(path, len(out["hll"]), len(out["hllc"]))

    with open(os.path.join(root, "src/test/luna_1d_values.hpp")) as f:
        text = f.read()
    cases = {}
    for key, name in (("sod", "sod"), ("shu_osher", "shu-osher"), ("woodward_colella", "woodward-colella")):
        steps = int(re.search(r"const int luna_steps_" + key + r" = (\d+);", text).group(1))
        block = re.search(r"const double luna_" + key + r"\[16\]\[3\] = \{(.*?)\n\};", text, re.S).group(1)
        rows = [[float(x) for x in re.findall(r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?", line)]
                for line in block.strip().splitlines() if line.strip().startswith("{")]
        cases[name] = {"steps": steps, "W": rows}
    out = {"source": "luna-cpp src/test/luna_1d_values.hpp (LUNA's final states at N = 16, MC, HLLC, CFL 0.8, FP64)",
           "check": "src/test/hydro1d_test.cpp:266-296", "tolerance": 1e-12, "cells": 16, "courant": 0.8,
           "cases": cases}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "luna_1d_final_states.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(path, {k: len(v["W"]) for k, v in cases.items()})
    derivatives(root)


# The problems of the derivative cases (problems_1d.hpp:212, :271): Sod on [0, 1] between outflow walls, gamma 1.4;
# the right-going sound wave on the periodic [0, 1], gamma 5/3.
DERIVATIVE_PROBLEMS = {"sod": {"L": 1.0, "gamma": 1.4, "periodic": False, "walls": ["outflow", "outflow"]},
                       "sound-right": {"L": 1.0, "gamma": 5.0 / 3.0, "periodic": True, "walls": None}}
# (namespace, problem, gated) in the order of hydro_derivatives_test.cpp:1081-1087
DERIVATIVE_CASES = [("luna_d_sod_64_l1", "sod", False), ("luna_d_sod_64_l1_noisy", "sod", True),
                    ("luna_d_sod_64_l2_noisy", "sod", True), ("luna_d_sound_right_64_l2", "sound-right", True),
                    ("luna_d_sod_64_l0", "sod", True), ("luna_d_sound_right_64_l1", "sound-right", True),
                    ("luna_d_sound_right_64_l0", "sound-right", True)]


def derivatives(root):
    with open(os.path.join(root, "src/test/luna_derivative_values.hpp")) as f:
        text = f.read()
    cases = {}
    for ns, problem, gated in DERIVATIVE_CASES:
        body = re.search(r"namespace " + ns + r" \{(.*?)\n\}\n", text, re.S).group(1)
        head = re.search(r"const int n = (\d+), limiter = (\d+), steps = (\d+);", body)
        case = {"problem": problem, "gate": gated, "n": int(head.group(1)), "limiter": int(head.group(2)),
                "steps": int(head.group(3)), "dt": float(re.search(r"const double dt = ([^;]+);", body).group(1))}
        for name in ("U0", "dU", "w", "U", "JdU", "JTw"):
            block = re.search(r"const double " + name + r"\[\d+\]\[3\] = \{(.*?)\};", body, re.S).group(1)
            case[name] = [[float(x) for x in re.findall(r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?", line)]
                          for line in block.strip().splitlines() if line.strip().startswith("{")]
            assert len(case[name]) == case["n"] and all(len(r) == 3 for r in case[name]), (ns, name)
        cases[ns] = case
    out = {"source": "luna-cpp src/test/luna_derivative_values.hpp (LUNA's jax.jvp / jax.vjp of K fixed-dt steps, HLLC, "
                     "FP64; U per volume; limiter 0 minmod, 1 MC, 2 van Leer; cells at x = (i + 0.5) L / n)",
           "check": "src/test/hydro_derivatives_test.cpp:991-1088", "tolerance": {"forward": 1e-12, "derivatives": 1e-8},
           "problems": DERIVATIVE_PROBLEMS, "cases": cases}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "luna_1d_derivatives.json")
    with open(path, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(path, list(cases))


if __name__ == "__main__":
    main()
