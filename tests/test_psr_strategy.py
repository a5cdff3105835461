"""The periodicity strategy (aa_b200_psr_strategy: FFT length, DM trials per
batch, batches of every range, input plane, cuFFT work area, MSD blocks)
against the reference's own aa_periodicity_strategy on the same DDTR plans
and memory budgets (tests/golden/psr_strategy_golden.json, made on the host
by tests/golden/make_psr_strategy_golden.py).  No GPU."""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "psr_strategy_golden.json")

with open(GOLDEN) as _fh:
    G = json.load(_fh)

MAX_RANGES, MAX_BATCHES = 64, 4096


def strategy(aa, c, mem, nh, alg):
    L = aa.lib()
    P = ctypes.POINTER
    i, d, f, sz = ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_size_t
    L.aa_b200_psr_strategy.argtypes = [P(aa.aa_b200_dm), i, i, i, d, d, d, i, sz, sz, f, i, i, ctypes.c_void_p,
                                       ctypes.c_void_p, i, ctypes.c_void_p, i]
    L.aa_b200_psr_strategy.restype = i
    plan = (aa.aa_b200_dm * len(c["plan"]))(*[aa.aa_b200_dm(*p) for p in c["plan"]])
    info = np.zeros(7, np.int64)
    rinfo = np.zeros(2 * MAX_RANGES, np.int64)
    batches = np.zeros(5 * MAX_BATCHES, np.int64)
    nb = L.aa_b200_psr_strategy(plan, len(c["plan"]), c["nchans"], c["nsamp"], c["tsamp"], c["fch1"], c["foff"],
                                c["nbits"], 180 << 30, mem, 6.0, nh, alg, info.ctypes.data, rinfo.ctypes.data,
                                MAX_RANGES, batches.ctypes.data, MAX_BATCHES)
    nr = len(c["plan"])
    return {"rc": int(nb), "info": info.tolist(), "ranges": rinfo[:2 * nr].tolist(),
            "batches": batches[:5 * max(0, min(nb, MAX_BATCHES))].tolist()}


@pytest.mark.parametrize("key", list(G["runs"]))
def test_periodicity_strategy_matches_reference(aa, key):
    name, mem, nh, alg = key.split("/")
    want = G["runs"][key]
    got = strategy(aa, G["plans"][name], int(mem), int(nh), int(alg))
    assert got["info"][6] == want["info"][6], (got["info"], want["info"])
    if want["info"][6]:
        assert got == want
