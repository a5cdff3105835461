"""Generates tests/golden/psr_strategy_golden.json: the reference's
periodicity strategy (aa_periodicity_strategy, include/aa_periodicity_strategy.hpp,
through oracle/ref_harness.cu aaref_psr_strategy) for DDTR plans of several
sizes and a range of memory budgets, from one batch per range down to a few
DM trials per batch.  Host only, no GPU.

    python tests/golden/make_psr_strategy_golden.py
"""
from __future__ import annotations

import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import cases as C  # noqa: E402
import refharness as R  # noqa: E402

MAX_RANGES, MAX_BATCHES = 64, 4096

PLANS = {
    "survey_2e21": dict(nchans=4096, nsamp=1 << 21, tsamp=64e-6, fch1=1670.0, foff=-0.0732421875, nbits=8,
                        plan=C.SURVEY_PLAN),
    "survey_2e18": dict(nchans=4096, nsamp=1 << 18, tsamp=64e-6, fch1=1670.0, foff=-0.0732421875, nbits=8,
                        plan=C.SURVEY_PLAN),
    "binned_2e17": dict(nchans=512, nsamp=(1 << 17) + 3000, tsamp=64e-6, fch1=1670.0, foff=-0.5859375, nbits=8,
                        plan=C.BINNED_PLAN),
    "psr_cases": dict(nchans=256, nsamp=(1 << 17) + 4096, tsamp=64e-6, fch1=1550.0, foff=-1.5625, nbits=8,
                      plan=[(0, 25.5, 0.1, 1, 1), (25.6, 76.7, 0.2, 2, 1)]),
}
MEMORIES = [64 << 20, 200 << 20, 1 << 30, 3 << 30, 8 << 30, 40 << 30, 180 << 30]
SETTINGS = [(16, 1), (32, 0), (32, 2)]  # (nHarmonics, harmonic sum algorithm)


def run(L, c, mem, nh, alg):
    info = np.zeros(7, np.int64)
    rinfo = np.zeros(2 * MAX_RANGES, np.int64)
    batches = np.zeros(5 * MAX_BATCHES, np.int64)
    nb = L.aaref_psr_strategy(R._plan(c["plan"]), len(c["plan"]), c["nchans"], c["nsamp"], c["tsamp"], c["fch1"],
                              c["foff"], c["nbits"], 180 << 30, mem, 6.0, nh, alg, info.ctypes.data,
                              rinfo.ctypes.data, MAX_RANGES, batches.ctypes.data, MAX_BATCHES)
    nr = len(c["plan"])
    return {"rc": int(nb), "info": info.tolist(), "ranges": rinfo[:2 * nr].tolist(),
            "batches": batches[:5 * max(0, min(nb, MAX_BATCHES))].tolist()}


def main():
    L = R.load()
    P = ctypes.POINTER
    i, d, f, sz, ll = ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_size_t, ctypes.c_longlong
    L.aaref_psr_strategy.argtypes = [P(R.DM), i, i, i, d, d, d, i, sz, sz, f, i, i, ctypes.c_void_p,
                                     ctypes.c_void_p, i, ctypes.c_void_p, i]
    L.aaref_psr_strategy.restype = i
    out = {}
    for name, c in PLANS.items():
        for mem in MEMORIES:
            for nh, alg in SETTINGS:
                key = f"{name}/{mem}/{nh}/{alg}"
                out[key] = run(L, c, mem, nh, alg)
                print(key, out[key]["rc"], out[key]["info"], flush=True)
    with open(os.path.join(HERE, "psr_strategy_golden.json"), "w") as fh:
        json.dump({"plans": {k: dict(v, plan=[list(p) for p in v["plan"]]) for k, v in PLANS.items()},
                   "memories": MEMORIES, "settings": SETTINGS, "runs": out}, fh, indent=0)


if __name__ == "__main__":
    main()
