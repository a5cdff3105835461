"""Generates tests/golden/preproc_golden.json from the reference's own GPU
code: its pipeline runner with the optional input/output processing of
preproc_cases.py (oracle/ref_harness.cu aaref_run_ddtr_opts), on the seeded
inputs of cases.py.  For every DM range it stores the SHA-256 of the float32
output and a sample of values.

Needs a GPU.  Each run is a child process (the reference's aa_device_info
destructor resets the device).

    python tests/golden/make_preproc_golden.py --out <dir>/preproc_golden.json
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)

import cases as C  # noqa: E402
import preproc_cases as P  # noqa: E402
from make_ddtr_golden import digest, sample_positions  # noqa: E402


def run_one(name, q):
    import refharness as R
    cname, opts, bp = P.RUNS[name]
    case = C.CASES[cname]
    L = R.load()
    x = C.make_input(case)
    bandpass = P.custom_bandpass(case["nchans"]) if bp == "custom" else None
    s, flat = R.run_ddtr(L, x, case["plan"], case["nchans"], case["nsamp"], case["fch1"], case["foff"],
                         case["tsamp"], case["nbits"], case["free_memory"], options=opts, bandpass=bandpass)
    ranges, off = [], 0
    for r in range(len(case["plan"])):
        tot = sum(s["t_processed"][r])
        n = s["ndms"][r] * tot
        a = flat[off:off + n].reshape(s["ndms"][r], tot)
        off += n
        pos = sample_positions(a.shape, 2000 + r)
        ranges.append({"sha256": digest(a), "shape": list(a.shape),
                       "samples": [[i, j, int(np.float32(a[i, j]).view(np.uint32))] for i, j in pos]})
    q.put({"run": name, "case": cname, "options": opts, "bandpass": bp, "num_tchunks": s["num_tchunks"],
           "ranges": ranges})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "preproc_golden.json"))
    args = ap.parse_args()
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    ctx = mp.get_context("spawn")
    results = {}
    for name in P.RUNS:
        q = ctx.Queue()
        p = ctx.Process(target=run_one, args=(name, q))
        p.start()
        rec = q.get(timeout=900)
        p.join(timeout=120)
        results[name] = rec
        print(name, "ok", rec["num_tchunks"], flush=True)
    with open(args.out, "w") as f:
        json.dump({"generator": "tests/golden/make_preproc_golden.py", "reference": "AstroAccelerate v1.3.1",
                   "runs": results}, f, indent=1)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
