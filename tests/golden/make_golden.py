"""Generates the golden fixtures under tests/golden/ from the reference tree.

Run in a container where the reference sources are mounted (the GPU machine never runs this):

    python tests/golden/make_golden.py /path/to/keepsake

Fixtures written:
  sobol_matrices.json  columns 0..51 of generator matrices 0 and 1, read from the reference's
                       table (sobol.cpp:154+, `sobol_matrices_32`), the only two dimensions that
                       OwenScrambledSobol02Morton reads (sobol.h:160-166).
"""
import json
import os
import re
import sys


def sobol_matrices(ref_root):
    src = open(os.path.join(ref_root, "sobol.cpp")).read()
    start = src.index("sobol_matrices_32[")
    body = src[start:start + 20000]
    nums = re.findall(r"0x[0-9a-fA-F]+", body)
    vals = [int(x, 16) for x in nums[:104]]
    return {"source": "sobol.cpp sobol_matrices_32[0:104] (dimension 0 then 1, 52 columns each)",
            "dim0": vals[:52], "dim1": vals[52:104]}


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference source tree>")
    ref = sys.argv[1]
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "sobol_matrices.json"), "w") as f:
        json.dump(sobol_matrices(ref), f, indent=0)
    print("wrote sobol_matrices.json")


if __name__ == "__main__":
    main()
