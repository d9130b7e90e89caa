"""Generates the golden fixtures from the reference's own test files (read as text).

- luna_riemann.json: LUNA's HLL and HLLC fluxes (jax, float64) that luna-cpp's src/test/hydro_test.cpp:48-80 pins its
  Riemann solvers to (relative max-norm difference < 1e-14, gamma 5/3, axis normals);
- luna_1d_final_states.json: LUNA's final states at N = 16 (MC limiter, HLLC, CFL 0.8) of Sod, Shu-Osher and
  Woodward-Colella, src/test/luna_1d_values.hpp, that src/test/hydro1d_test.cpp:266-296 pins FiniteVolume<1> to
  (|W - W_luna| / (1e-3 + |W_luna|) < 1e-12, the same step count).
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


if __name__ == "__main__":
    main()
