"""Times the reference's own analysis_GPU (AstroAccelerate v1.3.1 built from
its sources by oracle/Makefile.ref) on the single-pulse detection workload of
bench.py --config spd: the same seeded DM-time plane (1536 DM trials x 2^19
samples float32, generated on the GPU by bench.py's generator), the same
settings, CUDA events around each analysis_GPU call.  The plane size is
kept below the reference's 32-bit offset limit (nDMs * output_shift < 2^31,
src/aa_device_SPS_long.cu:69,73): at 1536 x 2^20 its analysis ended with an
illegal memory access.  Needs a GPU; prints
one JSON line.

    python tests/golden/time_reference_spd.py [--reps 5]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reps", type=int, default=5)
    args = ap.parse_args()
    import torch
    import bench
    import refharness as R
    w = bench.SPD_WORKLOAD
    plane = bench.synth_plane_device(w, w["seed"], torch.device("cuda", 0))
    torch.cuda.synchronize()
    L = R.load()
    P, f, i, ll = ctypes.POINTER, ctypes.c_float, ctypes.c_int, ctypes.c_longlong
    L.aaref_time_spd.argtypes = [ctypes.c_void_p, i, i, f, i, f, f, i, f, i, ll, i, P(f), P(ll)]
    L.aaref_time_spd.restype = i
    ms = np.zeros(args.reps, np.float32)
    nc = ll()
    tsamp = float(np.float32(w["tsamp"] * w["inbin"]))
    rc = L.aaref_time_spd(ctypes.c_void_p(plane.data_ptr()), w["ndms"], w["nt"], tsamp, w["inbin"],
                          w["max_width_s"], w["sigma_constant"], w["baseline_noise"], w["sigma_cutoff"],
                          w["algorithm"], 0, args.reps, ms.ctypes.data_as(P(f)), ctypes.byref(nc))
    n = w["ndms"] * w["nt"]
    med = float(statistics.median(ms.tolist())) if rc == 0 else None
    print(json.dumps({"impl": "reference-gpu", "rc": rc, "ms": ms.tolist(), "ms_median": med,
                      "value": (n / (med / 1e3)) if med else None, "unit": "DM-trial*samples/s",
                      "candidates": nc.value,
                      "workload": f"{w['ndms']} DM trials x {w['nt']} samples, bench.py --config spd"}))
    return 0 if rc == 0 else 1


if __name__ == "__main__":
    sys.exit(main())
