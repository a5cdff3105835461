"""Generates tests/golden/psr_candidates_golden.json from the reference's own
host-side conversion of periodicity candidates (oracle/ref_candidates.cpp,
built by oracle/Makefile.ref into oracle/_ref/libaaref_cand.so) on the seeded
records of psr_cases.CANDIDATE_CASES.  Runs on the CPU.

    python tests/golden/make_psr_candidates_golden.py
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)

import psr_cases as P  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "psr_candidates_golden.json"))
    args = ap.parse_args()
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libaaref_cand.so"))
    Pf = ctypes.POINTER(ctypes.c_float)
    L.aaref_psr_candidates_process.argtypes = [Pf, ctypes.c_size_t, Pf, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_size_t, ctypes.c_float, ctypes.c_int]
    L.aaref_psr_candidates_process.restype = ctypes.c_int
    out = {"generator": "tests/golden/make_psr_candidates_golden.py", "reference": "AstroAccelerate v1.3.1",
           "cases": {}}
    for name, c in P.CANDIDATE_CASES.items():
        rec, msd = P.make_candidate_records(c)
        r = rec.copy()
        rc = L.aaref_psr_candidates_process(r.ctypes.data_as(Pf), c["n"], msd.ctypes.data_as(Pf), c["dm_low"],
                                            c["dm_step"], c["tsamp"], c["nt"], c["mod"], c["greedy"])
        out["cases"][name] = {"rc": rc, "sha256": hashlib.sha256(r.tobytes()).hexdigest(),
                              "head": r[:64].view(np.uint32).tolist()}
        print(name, rc, flush=True)
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
