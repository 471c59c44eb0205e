#!/usr/bin/env python3
"""Generates the golden fixtures that pin the oracle's sampler tables, using the reference's own
generator scripts (HamilcarR/Axomae scripts/generate_luts_sobol.py and
scripts/generate_luts_trigonometrics.py).  Only the function definitions of those scripts are
executed (their module-level code parses command-line arguments and writes files); the fixtures
are committed so the tests never need the reference checkout.

Outputs (next to this script):
  sobol_dv.npy        uint32[256, 32]  direction vectors: compute_V() of the first 255 Joe-Kuo rows
                                       (generate_luts_sobol.py:89-95, :149-175), row 255 zero.
  sobol_samples.npz   index, dim, seed, bits: sample values of the reference's sobol_sample()
                                       (generate_luts_sobol.py:128-138) for index >= 1.  That
                                       function divides by 2^32 in double; the C++ generator
                                       (math_random.h:73-86) computes float(accum) * 2^-32, which
                                       is the same value rounded to float32, stored here as bits.
                                       Index 0 is the one place the two differ (the Python
                                       returns 0 without scrambling); its C++ value is
                                       owen_scramble(0, seed) * 2^-32, taken from the reference's
                                       owen_scramble().
  acos_lut.json       sha256 of the float32 table of generate_acos(500000) plus sample entries.

Usage: python make_golden.py <reference_root>   (or set AXOMAE_REFERENCE to the reference checkout)
"""
import ast
import copy
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_functions(path: str) -> dict:
    """Executes only the imports and function definitions of a reference script."""
    src = open(path).read()
    tree = ast.parse(src)
    keep = [n for n in tree.body if isinstance(n, (ast.FunctionDef, ast.Import, ast.ImportFrom))]
    mod = ast.Module(body=keep, type_ignores=[])
    ns: dict = {}
    exec(compile(mod, path, "exec"), ns)
    return ns


def main() -> None:
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("AXOMAE_REFERENCE", "")
    if not ref or not os.path.isdir(os.path.join(ref, "scripts")):
        sys.exit("usage: make_golden.py <reference_root> (or AXOMAE_REFERENCE=<reference_root>)")
    sob = load_functions(os.path.join(ref, "scripts", "generate_luts_sobol.py"))
    trig = load_functions(os.path.join(ref, "scripts", "generate_luts_trigonometrics.py"))

    # Direction vectors exactly as the build rule invokes the script (-d 256 -s 32).
    rows = sob["to_arraylist"](sob["read_as_string"](os.path.join(ref, "scripts", "joe_kuo.txt"), 256))
    assert len(rows) == 255
    dv = np.zeros((256, 32), dtype=np.uint32)
    for d, row in enumerate(rows):
        r = copy.deepcopy(row)
        dv[d] = np.array(sob["compute_V"](r[1], r[2], r[3], 32), dtype=np.uint64).astype(np.uint32)
    np.save(os.path.join(HERE, "sobol_dv.npy"), dv)

    # Sample values.
    idx_l, dim_l, seed_l, bits_l = [], [], [], []
    for seed in (0, 0xDEADBEEF):
        for dim in range(16):
            for index in range(0, 384):
                if index == 0:
                    acc = sob["owen_scramble"](0, seed) & 0xFFFFFFFF
                    val = np.float32(np.float64(acc) / 2.0**32)
                else:
                    val = np.float32(sob["sobol_sample"](copy.deepcopy(rows[dim]), index, 32, seed))
                idx_l.append(index)
                dim_l.append(dim)
                seed_l.append(seed)
                bits_l.append(np.array(val, dtype=np.float32).view(np.uint32))
    np.savez_compressed(os.path.join(HERE, "sobol_samples.npz"), index=np.array(idx_l, np.uint32),
                        dim=np.array(dim_l, np.uint32), seed=np.array(seed_l, np.uint32),
                        bits=np.array(bits_l, np.uint32))

    # acos lookup table (PRECISION_LUT = 500000, the default AXOMAE_LUT_MEDIUMP).
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "acos_table")
        trig["generate_acos"](500000, path)
        raw = open(path, "rb").read()
    lut = np.frombuffer(raw, dtype=np.float32)
    picks = [0, 1, 2, 12345, 249999, 250000, 250001, 333333, 499998, 499999]
    json.dump({"precision": 500000, "sha256": hashlib.sha256(raw).hexdigest(),
               "samples": {str(i): float(lut[i]) for i in picks}},
              open(os.path.join(HERE, "acos_lut.json"), "w"), indent=1)
    print("golden fixtures written:", dv.shape, len(bits_l), lut.shape)


if __name__ == "__main__":
    main()
