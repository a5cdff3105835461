"""Generates tests/golden/spd_golden.json from the reference's own GPU
single-pulse detection (oracle/ref_harness.cu aaref_spd: the interpolated MSD
profile, the boxcar S/N and width planes of src/aa_device_SPS_long.cu, and
the candidates of analysis_GPU, src/aa_device_analysis.cu:130-345) on the
seeded planes of spd_cases.py.  Needs a GPU; each run is a child process.

    python tests/golden/make_spd_golden.py --out gpurun_out/golden/spd_golden.json
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)

import spd_cases as S  # noqa: E402

MAX_CANDS = 1 << 20


def run_one(name, q):
    import refharness as R
    L = R.load()
    P, f, i = ctypes.POINTER, ctypes.c_float, ctypes.c_int
    L.aaref_spd.argtypes = [P(f), i, i, f, i, f, f, i, f, i, f, f, f, f, P(f), P(i), P(i), P(i), P(i), P(f),
                            P(ctypes.c_ushort), ctypes.c_longlong, P(ctypes.c_uint), P(ctypes.c_uint), P(f),
                            P(ctypes.c_uint), i, P(i)]
    L.aaref_spd.restype = i
    c = S.CASES[name]
    x = np.ascontiguousarray(S.make_plane(c))
    n = x.size
    msd = np.zeros(512, np.float32)
    widths = np.zeros(256, np.int32)
    nw, mwp, mit, nc = i(), i(), i(), i()
    snr = np.zeros(2 * n, np.float32)
    taps = np.zeros(2 * n, np.uint16)
    cdm = np.zeros(MAX_CANDS, np.uint32)
    cts = np.zeros(MAX_CANDS, np.uint32)
    csnr = np.zeros(MAX_CANDS, np.float32)
    cbw = np.zeros(MAX_CANDS, np.uint32)
    tsamp_r = np.float32(c["tsamp"] * c["inbin"])
    rc = L.aaref_spd(x.ctypes.data_as(P(f)), c["ndms"], c["nt"], float(tsamp_r), c["inbin"], c["max_width_s"],
                     c["sigma_constant"], c["baseline_noise"], c["cutoff"], c["algorithm"], 1.0, 0.0,
                     0.1 * c["ndms"], 0.1, msd.ctypes.data_as(P(f)), widths.ctypes.data_as(P(i)), ctypes.byref(nw),
                     ctypes.byref(mwp), ctypes.byref(mit), snr.ctypes.data_as(P(f)),
                     taps.ctypes.data_as(P(ctypes.c_ushort)), 2 * n, cdm.ctypes.data_as(P(ctypes.c_uint)),
                     cts.ctypes.data_as(P(ctypes.c_uint)), csnr.ctypes.data_as(P(f)),
                     cbw.ctypes.data_as(P(ctypes.c_uint)), MAX_CANDS, ctypes.byref(nc))
    k = nc.value
    cands = sorted((int(cdm[j]), int(cts[j]), int(csnr[j:j + 1].view(np.uint32)[0]), int(cbw[j])) for j in range(k))
    q.put({"run": name, "rc": rc, "nwidths": nw.value, "widths": widths[:nw.value].tolist(),
           "max_width_performed": mwp.value, "max_iteration": mit.value,
           "msd_bits": msd[:2 * nw.value].view(np.uint32).tolist(),
           "snr_sha256": hashlib.sha256(snr.tobytes()).hexdigest(),
           "taps_sha256": hashlib.sha256(taps.tobytes()).hexdigest(),
           "ncands": k, "cands_sha256": hashlib.sha256(json.dumps(cands).encode()).hexdigest(),
           "cands_head": cands[:64]})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "gpurun_out", "golden", "spd_golden.json"))
    args = ap.parse_args()
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    ctx = mp.get_context("spawn")
    res = {}
    for name in S.CASES:
        q = ctx.Queue()
        p = ctx.Process(target=run_one, args=(name, q))
        p.start()
        rec = q.get(timeout=900)
        p.join(timeout=120)
        res[name] = rec
        print(name, rec["rc"], rec["nwidths"], rec["max_iteration"], rec["ncands"], flush=True)
    with open(args.out, "w") as f:
        json.dump({"generator": "tests/golden/make_spd_golden.py", "reference": "AstroAccelerate v1.3.1",
                   "runs": res}, f, indent=1)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
