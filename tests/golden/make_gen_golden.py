"""Generate tests/golden/gen/ from the REFERENCE's own instance generator.

gen_ising (reference file gpu/multibit_bias_20261008/src/gen_ising.cpp) is compiled unmodified by oracle/Makefile into
oracle/_ref/gen_ising. This script runs it for the cases in CASES and keeps its output files (PREFIX.jint8,
PREFIX.bias, PREFIX.json, and PREFIX.edges for gp) as fixtures. Run from the repository root where the reference
tree is available:

    make -C oracle && python tests/golden/make_gen_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "gen")
GEN = os.path.join(ROOT, "oracle", "_ref", "gen_ising")

# (name, gen_ising arguments without --out)
CASES = [
    ("gp16_brute", ["gp", "--n", "16", "--deg", "3", "--k", "5", "--A", "2", "--B", "1", "--seed", "7", "--brute", "1"]),
    ("gp20_brute", ["gp", "--n", "20", "--deg", "3", "--k", "8", "--A", "3", "--B", "2", "--seed", "4", "--brute", "1"]),
    ("gp64", ["gp", "--n", "64", "--deg", "4", "--k", "20", "--A", "2", "--B", "1", "--seed", "12"]),
    ("tsp4_brute", ["tsp", "--n", "4", "--wmax", "4", "--A", "9", "--B", "1", "--seed", "1", "--brute", "1"]),
    ("tsp5_brute", ["tsp", "--n", "5", "--wmax", "9", "--A", "20", "--B", "1", "--seed", "3", "--brute", "1"]),
    ("tsp8", ["tsp", "--n", "8", "--wmax", "5", "--A", "12", "--B", "2", "--seed", "11"]),
    ("rnd64_k4", ["random", "--n", "64", "--kbits", "4", "--pzero", "0.3", "--bmax", "40", "--seed", "5"]),
    ("rnd65_pbig", ["random", "--n", "65", "--kbits", "2", "--pzero", "0", "--bmax", "100", "--pbig", "0.25",
                    "--bsmall", "3", "--seed", "8"]),
]


def main():
    if not os.path.exists(GEN):
        sys.exit("oracle/_ref/gen_ising missing: run make -C oracle where the reference tree is present")
    os.makedirs(OUT, exist_ok=True)
    for name, args in CASES:
        prefix = os.path.join(OUT, name)
        for ext in (".jint8", ".bias", ".json", ".edges"):
            if os.path.exists(prefix + ext):
                os.remove(prefix + ext)
        subprocess.run([GEN, *args, "--out", prefix], check=True, stdout=subprocess.DEVNULL)
        print(name)


if __name__ == "__main__":
    main()
