"""Generates tests/golden/luna_riemann.json from the reference's own test file (read as text).

The vectors are LUNA's HLL and HLLC fluxes (jax, float64) that luna-cpp's src/test/hydro_test.cpp:48-80 pins its Riemann
solvers to (relative max-norm difference < 1e-14, gamma 5/3, axis normals). Run in a tree that has the reference:
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
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
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


if __name__ == "__main__":
    main()
