"""Generates tests/golden/strategy_golden.json from the reference's own
aa_ddtr_strategy (src/aa_ddtr_strategy.cpp:27-428), compiled from its sources
into oracle/_ref/libaaref.so (oracle/Makefile.ref).  Host only, no GPU.

Cases: the survey configurations plus seeded random plans over channel counts,
sample counts, bit depths, memory budgets (single and multi-chunk), power
law exponents and the analysis reservation.

    python tests/golden/make_strategy_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import random
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import cases as C  # noqa: E402
import refharness as R  # noqa: E402


def build_cases(n_random=160, seed=5):
    rnd = random.Random(seed)
    out = [
        dict(plan=C.SURVEY_PLAN, nchans=4096, nsamp=1 << 21, fch1=1670.0, foff=-0.0732421875, tsamp=64e-6,
             nbits=8, free_memory=180 * 2**30, power=2.0, analysis=0),
        dict(plan=[(0, 500, 0.5, 1, 1)], nchans=1024, nsamp=1 << 18, fch1=1550.0, foff=-0.390625, tsamp=64e-6,
             nbits=8, free_memory=180 * 2**30, power=2.0, analysis=0),
    ]
    for name, c in C.CASES.items():
        out.append(dict(plan=c["plan"], nchans=c["nchans"], nsamp=c["nsamp"], fch1=c["fch1"], foff=c["foff"],
                        tsamp=c["tsamp"], nbits=c["nbits"], free_memory=C.strategy_free_memory(c), power=2.0,
                        analysis=0))
    for _ in range(n_random):
        nch = rnd.choice([128, 256, 512, 1024, 2048, 3072, 4096, 2080, 8192])
        plan = C.SURVEY_PLAN[:rnd.randint(1, 8)]
        if rnd.random() < 0.3:
            plan = [(0, round(rnd.uniform(50, 400), 3), rnd.choice([0.5, 1, 0.25, 2.0]), 1, 1)]
        f1 = rnd.choice([1550.0, 1670.0, 400.0, 1400.0])
        fo = -rnd.choice([0.390625, 0.0732421875, 0.1, 1.0, 2.34375])
        if f1 + fo * nch < 0.3 * f1:
            fo = -0.5 * f1 / nch
        out.append(dict(plan=plan, nchans=nch, nsamp=rnd.choice([1 << 16, 1 << 17, 1 << 18, 1 << 20, 1 << 21, 300000]),
                        fch1=f1, foff=fo, tsamp=rnd.choice([64e-6, 64e-6, 128e-6]), nbits=rnd.choice([1, 2, 4, 8, 16, 32]),
                        free_memory=rnd.choice([180 * 2**30, 2**30, 300 * 2**20, 4 * 2**30, 16 * 2**30]),
                        power=rnd.choice([2.0, 2.0, 2.0, 1.9, 2.1]), analysis=rnd.randint(0, 1)))
    return out


def main():
    L = R.load()
    recs = []
    for c in build_cases():
        s = R.strategy(L, c["plan"], c["nchans"], c["nsamp"], c["fch1"], c["foff"], c["tsamp"], c["nbits"],
                       c["free_memory"], c["power"], c["analysis"])
        rec = dict(c, plan=[list(p) for p in c["plan"]])
        if s is None:
            rec["refused"] = True
        else:
            rec["refused"] = False
            rec["dmshifts_sha256"] = hashlib.sha256(np.asarray(s["dmshifts"], np.float32).tobytes()).hexdigest()
            rec["dmshift_last_bits"] = int(np.float32(s["dmshifts"][-1]).view(np.uint32))
            for k in ("ndms", "dm", "maxshift", "max_ndms", "num_tchunks", "t_processed"):
                rec[k] = s[k]
        recs.append(rec)
    out = os.path.join(HERE, "strategy_golden.json")
    with open(out, "w") as f:
        json.dump({"generator": "tests/golden/make_strategy_golden.py", "reference": "AstroAccelerate v1.3.1",
                   "cases": recs}, f, indent=0)
    print("wrote", out, len(recs), "cases,", sum(r["refused"] for r in recs), "refused")


if __name__ == "__main__":
    main()
