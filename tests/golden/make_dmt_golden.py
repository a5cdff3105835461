"""Generates tests/golden/dmt_golden.json: SHA-256 of every file the
reference's own Export_DD_data (include/aa_pipeline_runner.hpp:165-216,
compiled from its sources into oracle/_ref/libaaref.so by oracle/Makefile.ref)
writes for the seeded outputs of dmt_cases.py.  Host only, no GPU.

    python tests/golden/make_dmt_golden.py
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import dmt_cases as D  # noqa: E402
import refharness as R  # noqa: E402


def main():
    L = R.load()
    PPPF = ctypes.POINTER(ctypes.POINTER(ctypes.POINTER(ctypes.c_float)))
    IP = ctypes.POINTER(ctypes.c_int)
    L.aaref_export_dd_data.argtypes = [ctypes.c_int, PPPF, ctypes.c_size_t, IP, IP, ctypes.c_char_p, IP, ctypes.c_int]
    L.aaref_export_dd_data.restype = None
    L.aaref_sd_per_file.argtypes = [ctypes.c_size_t] * 3
    L.aaref_sd_per_file.restype = ctypes.c_size_t
    rs = D.rows()
    top, keep = D.as_float3(rs)
    out = {"sd_per_file": {f"{mb},{p},{k}": L.aaref_sd_per_file(mb, p, k)
                           for mb, p, k in [(1000, 1000, 1), (1000, 2060800, 1), (1, 1000, 1), (7, 333, 3)]},
           "cases": {}}
    with tempfile.TemporaryDirectory() as td:
        for name, (per, exp) in D.CASES.items():
            base = os.path.join(td, name)
            nd = (ctypes.c_int * 3)(*D.NDMS)
            ib = (ctypes.c_int * 3)(*D.IN_BIN)
            ex = (ctypes.c_int * 3)(*exp)
            L.aaref_export_dd_data(3, ctypes.cast(top, PPPF), D.MAX_NT, nd, ib, os.fsencode(base), ex, per)
            files = sorted(f for f in os.listdir(td) if f.startswith(name + "_"))
            out["cases"][name] = {f[len(name):]: hashlib.sha256(open(os.path.join(td, f), "rb").read()).hexdigest()
                                  for f in files}
    with open(os.path.join(HERE, "dmt_golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print({k: len(v) for k, v in out["cases"].items()})


if __name__ == "__main__":
    main()
