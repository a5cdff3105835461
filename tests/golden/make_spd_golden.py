"""Generates tests/golden/spd_golden.json from the reference's own GPU
single-pulse detection (oracle/ref_harness.cu aaref_spd: the interpolated MSD
profile, the boxcar S/N and width planes of src/aa_device_SPS_long.cu, and
the candidates of analysis_GPU, src/aa_device_analysis.cu:130-345) on the
seeded planes of spd_cases.py, and the reference runner with the analysis
component on DDTR cases of cases.py (oracle/ref_harness.cu
aaref_run_pipeline_spd: per-step candidates and the candidate files it
writes).  Needs a GPU; each run is a child process.

    python tests/golden/make_spd_golden.py --out <dir>/spd_golden.json
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
                            P(ctypes.c_uint), i, P(i), ctypes.c_longlong]
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
    # analysis_GPU prints the length of the list peak filtering starts from
    # ("Number of peaks: N"); the C library's stdout goes to a file meanwhile
    import re
    import tempfile
    sys.stdout.flush()
    cap = tempfile.TemporaryFile(mode="w+b")
    saved = os.dup(1)
    os.dup2(cap.fileno(), 1)
    rc = L.aaref_spd(x.ctypes.data_as(P(f)), c["ndms"], c["nt"], float(tsamp_r), c["inbin"], c["max_width_s"],
                     c["sigma_constant"], c["baseline_noise"], c["cutoff"], c["algorithm"], 1.0, 0.0,
                     0.1 * c["ndms"], 0.1, msd.ctypes.data_as(P(f)), widths.ctypes.data_as(P(i)), ctypes.byref(nw),
                     ctypes.byref(mwp), ctypes.byref(mit), snr.ctypes.data_as(P(f)),
                     taps.ctypes.data_as(P(ctypes.c_ushort)), 2 * n, cdm.ctypes.data_as(P(ctypes.c_uint)),
                     cts.ctypes.data_as(P(ctypes.c_uint)), csnr.ctypes.data_as(P(f)),
                     cbw.ctypes.data_as(P(ctypes.c_uint)), MAX_CANDS, ctypes.byref(nc), int(c.get("max_ts", 0)))
    libc = ctypes.CDLL(None)
    libc.fflush(None)
    os.dup2(saved, 1)
    os.close(saved)
    cap.seek(0)
    text = cap.read().decode(errors="replace")
    unfiltered = [int(v) for v in re.findall(r"Number of peaks: (\d+);", text)]
    k = nc.value
    cands = sorted((int(cdm[j]), int(cts[j]), int(csnr[j:j + 1].view(np.uint32)[0]), int(cbw[j])) for j in range(k))
    q.put({"run": name, "rc": rc, "nwidths": nw.value, "widths": widths[:nw.value].tolist(),
           "max_width_performed": mwp.value, "max_iteration": mit.value,
           "msd_bits": msd[:2 * nw.value].view(np.uint32).tolist(),
           "snr_sha256": hashlib.sha256(snr.tobytes()).hexdigest(),
           "taps_sha256": hashlib.sha256(taps.tobytes()).hexdigest(),
           "ncands": k, "cands_sha256": hashlib.sha256(json.dumps(cands).encode()).hexdigest(),
           "cands_head": cands[:64], "unfiltered_peaks": unfiltered})


def run_pipeline(name, q):
    """The reference runner with analysis on one DDTR case, in a scratch
    working directory that receives its candidate files."""
    import glob
    import tempfile
    import cases as C
    import refharness as R
    L = R.load()
    P, f, i, ll = ctypes.POINTER, ctypes.c_float, ctypes.c_int, ctypes.c_longlong
    pc = S.PIPELINE_CASES[name]
    case = C.CASES[pc["ddtr"]]
    x = np.ascontiguousarray(C.make_input(case))
    plan = R._plan(case["plan"])
    L.aaref_run_pipeline_spd.argtypes = [P(ctypes.c_ushort), i, i, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, i, ctypes.c_void_p, i, ctypes.c_size_t, f, f, f, i, i, i,
                                         P(i), P(i), P(ll), P(ctypes.c_uint), P(ctypes.c_uint), P(f),
                                         P(ctypes.c_uint), ll, P(ll), P(i), P(i), i]
    L.aaref_run_pipeline_spd.restype = i
    max_steps, max_chunks = 4096, 256
    sc = np.zeros(max_steps, np.int32)
    sr = np.zeros(max_steps, np.int32)
    sn = np.zeros(max_steps, np.int64)
    cdm = np.zeros(MAX_CANDS, np.uint32)
    cts = np.zeros(MAX_CANDS, np.uint32)
    csnr = np.zeros(MAX_CANDS, np.float32)
    cbw = np.zeros(MAX_CANDS, np.uint32)
    mts = ll()
    ntc = i()
    tp = np.zeros(len(case["plan"]) * max_chunks, np.int32)
    work = tempfile.mkdtemp(prefix="spdref_")
    here = os.getcwd()
    os.chdir(work)
    try:
        rc = L.aaref_run_pipeline_spd(x.ctypes.data_as(P(ctypes.c_ushort)), case["nchans"], case["nsamp"],
                                      case["tsamp"], case["fch1"], case["foff"], case["nbits"],
                                      ctypes.cast(plan, ctypes.c_void_p), len(case["plan"]),
                                      case["free_memory"], pc["sigma_cutoff"], pc["sigma_constant"],
                                      pc["max_width_s"], pc["algorithm"], pc["baseline_noise"], max_steps,
                                      sc.ctypes.data_as(P(i)), sr.ctypes.data_as(P(i)), sn.ctypes.data_as(P(ll)),
                                      cdm.ctypes.data_as(P(ctypes.c_uint)), cts.ctypes.data_as(P(ctypes.c_uint)),
                                      csnr.ctypes.data_as(P(f)), cbw.ctypes.data_as(P(ctypes.c_uint)), MAX_CANDS,
                                      ctypes.byref(mts), ctypes.byref(ntc), tp.ctypes.data_as(P(i)), max_chunks)
        files = {}
        for fn in sorted(glob.glob("*analysed*.dat")):
            rec = np.fromfile(fn, np.float32).reshape(-1, 4)
            rows = sorted(tuple(int(v) for v in r.view(np.uint32)) for r in rec)
            files[fn] = {"n": len(rows), "sha256": hashlib.sha256(json.dumps(rows).encode()).hexdigest()}
    finally:
        os.chdir(here)
    steps = []
    pos = 0
    for k in range(max(rc, 0)):
        n = int(sn[k])
        cands = sorted((int(cdm[pos + j]), int(cts[pos + j]), int(csnr[pos + j:pos + j + 1].view(np.uint32)[0]),
                        int(cbw[pos + j])) for j in range(n))
        pos += n
        steps.append({"chunk": int(sc[k]), "range": int(sr[k]), "ncands": n,
                      "cands_sha256": hashlib.sha256(json.dumps(cands).encode()).hexdigest(),
                      "cands_head": cands[:8]})
    q.put({"run": name, "rc": rc, "msd_max_ts": mts.value, "num_tchunks": ntc.value,
           "t_processed": [[int(tp[r * max_chunks + k]) for k in range(ntc.value)] for r in range(len(case["plan"]))],
           "steps": steps, "files": files})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "spd_golden.json"))
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
    pres = {}
    for name in S.PIPELINE_CASES:
        q = ctx.Queue()
        p = ctx.Process(target=run_pipeline, args=(name, q))
        p.start()
        rec = q.get(timeout=900)
        p.join(timeout=120)
        pres[name] = rec
        print(name, rec["rc"], rec["num_tchunks"], sum(s["ncands"] for s in rec["steps"]), len(rec["files"]),
              flush=True)
    with open(args.out, "w") as f:
        json.dump({"generator": "tests/golden/make_spd_golden.py", "reference": "AstroAccelerate v1.3.1",
                   "runs": res, "pipeline_runs": pres}, f, indent=1)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
