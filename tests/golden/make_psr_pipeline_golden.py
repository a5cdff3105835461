"""Generates tests/golden/psr_pipeline_golden.json from the reference's own
runner with the dedispersion and periodicity components (oracle/ref_harness.cu
aaref_run_pipeline_psr) on the seeded cases of psr_pipeline_cases.py: the
power and interbin candidate lists (records of DM, frequency, S/N,
harmonics) as float32 bytes.  Needs a GPU; each case runs in a child
process.

    python tests/golden/make_psr_pipeline_golden.py --out <dir>/psr_pipeline_golden.json
"""
from __future__ import annotations

import argparse
import base64
import ctypes
import hashlib
import json
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import psr_pipeline_cases as PC  # noqa: E402

CAP = 1 << 21
MAX_RECORDS = 20000  # golden lists are kept at most this long
SIGMAS = [8.0, 10.0, 12.0, 16.0, 20.0, 25.0, 30.0, 40.0, 60.0, 80.0, 120.0]


def sort_records(a):
    return a[np.lexsort((a[:, 2].view(np.uint32), a[:, 3], a[:, 1], a[:, 0]))]


def run_one(name, sigma, q):
    import refharness as R
    L = R.load()
    P, f, i, ll, sz = ctypes.POINTER, ctypes.c_float, ctypes.c_int, ctypes.c_longlong, ctypes.c_size_t
    L.aaref_run_pipeline_psr.argtypes = [ctypes.c_void_p, i, i, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         i, P(R.DM), i, sz, sz, f, i, f, i, i, i, i, ctypes.c_void_p, P(ll),
                                         ctypes.c_void_p, P(ll), ll]
    L.aaref_run_pipeline_psr.restype = i
    c = PC.PIPELINE_CASES[name]
    x = np.ascontiguousarray(PC.make_input(c))
    power = np.zeros(4 * CAP, np.float32)
    inter = np.zeros(4 * CAP, np.float32)
    npow, nint = ll(), ll()
    rc = L.aaref_run_pipeline_psr(x.ctypes.data, c["nchans"], c["nsamp"], c["tsamp"], c["fch1"], c["foff"],
                                  c["nbits"], R._plan(c["plan"]), len(c["plan"]), 0, PC.PSR_MEMORY,
                                  sigma, 1, 3.0, c["nHarmonics"], c["hs_algorithm"], c["selection"], 1,
                                  power.ctypes.data, ctypes.byref(npow), inter.ctypes.data, ctypes.byref(nint), CAP)
    out = {"rc": rc, "sigma_cutoff": sigma, "n_power": npow.value, "n_interbin": nint.value}
    if rc == 0 and max(npow.value, nint.value) <= MAX_RECORDS:
        for key, arr, n in (("power", power, npow.value), ("interbin", inter, nint.value)):
            a = arr[:4 * n].reshape(-1, 4)
            out[key] = base64.b64encode(a.tobytes()).decode()
            # candidates are appended through atomic counters: the order
            # varies, the sorted set is what repeats
            out[key + "_sorted_sha256"] = hashlib.sha256(sort_records(a).tobytes()).hexdigest()
    q.put(out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "psr_pipeline_golden.json"))
    ap.add_argument("--repeats", type=int, default=2, help="reference runs per case (their lists are compared)")
    args = ap.parse_args()
    ctx = mp.get_context("spawn")
    res = {}
    def one(name, sigma):
        q = ctx.Queue()
        p = ctx.Process(target=run_one, args=(name, sigma, q))
        p.start()
        r = q.get()
        p.join()
        return r

    for name, c in PC.PIPELINE_CASES.items():
        # the case's cutoff, raised until the lists are short enough to keep
        sigmas = [v for v in SIGMAS if v >= c["sigma_cutoff"]]
        runs = []
        for sigma in sigmas:
            r = one(name, sigma)
            print(name, sigma, r["rc"], r["n_power"], r["n_interbin"], flush=True)
            if r["rc"] == 0 and "power" in r:
                runs = [r]
                break
        if not runs:
            res[name] = {"rc": -10, "note": "no cutoff gave lists short enough"}
            continue
        for _ in range(args.repeats - 1):
            runs.append(one(name, runs[0]["sigma_cutoff"]))
        rec = dict(runs[0])
        rec["repeat_identical"] = all(r.get("power_sorted_sha256") == runs[0].get("power_sorted_sha256") and
                                      r.get("interbin_sorted_sha256") == runs[0].get("interbin_sorted_sha256")
                                      for r in runs)
        # how two runs of the reference differ: records present in one only,
        # and the largest relative S/N difference of common records
        if not rec["repeat_identical"] and len(runs) > 1:
            for key in ("power", "interbin"):
                a = np.frombuffer(base64.b64decode(runs[0][key]), np.float32).reshape(-1, 4)
                b = np.frombuffer(base64.b64decode(runs[1][key]), np.float32).reshape(-1, 4)
                ka = {tuple(v) for v in a[:, [0, 1, 3]].tolist()}
                kb = {tuple(v) for v in b[:, [0, 1, 3]].tolist()}
                rec[key + "_repeat_only_one"] = len(ka ^ kb)
        res[name] = rec
        print(name, "sigma", rec["sigma_cutoff"], rec["n_power"], rec["n_interbin"], "repeat identical:",
              rec["repeat_identical"], flush=True)
    with open(args.out, "w") as fh:
        json.dump(res, fh, indent=1)


if __name__ == "__main__":
    main()
