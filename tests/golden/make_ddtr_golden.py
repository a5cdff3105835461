"""Generates tests/golden/ddtr_golden.json from the reference's own GPU code.

Runs AstroAccelerate v1.3.1's pipeline runner, kernels, binning and strategy
(compiled from its sources by oracle/Makefile.ref into oracle/_ref/libaaref.so)
on the seeded cases of cases.py and on the reference's fake-signal known-answer
geometry (tests/test_ddtr_fakesignal_single.cpp:34-60, with fixed seeds instead
of srand(time(NULL))).  For every DM range it stores the SHA-256 of the float32
output and a sample of values, the strategy the reference chose, and how the
CPU oracle (oracle/aa_oracle.c) compares under each FMA-contraction variant.

Needs a GPU.  Each case runs in a child process because the reference's
aa_device_info destructor resets the device.

    python tests/golden/make_ddtr_golden.py --out <dir>/ddtr_golden.json
"""
from __future__ import annotations

import argparse
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import cases as C  # noqa: E402

N_SAMPLES = 256


def kat_cases():
    """Fake-signal geometry of tests/test_ddtr_fakesignal_single.cpp:34-60."""
    rng = np.random.Generator(np.random.PCG64(2024))
    out = {}
    for k in range(4):
        dm_position = float(int(rng.integers(0, int(0.8 * 250.0))))
        signal_start = int(rng.integers(0, 10)) * 1000 + int(rng.integers(0, 10)) * 100 + int(rng.integers(0, 10)) * 10
        out[f"kat_single_{k}"] = dict(nchans=128, nbits=8, fch1=1550.0, foff=-300.0 / 128, tsamp=6.4e-5,
                                      nsamp=int(2 / 6.4e-5), plan=[(0, 250.0, 1, 1, 1)], free_memory=0,
                                      kat=dict(dm_position=dm_position, signal_start=signal_start,
                                               width=int(1 / (6.4e-5 * 25)), sigma=0.5))
    return out


def make_case_input(name, case, strat_dmshifts=None, maxshift=None):
    if "kat" in case:
        import oracle as O
        k = case["kat"]
        x, _ = O.fake_signal(case["nchans"], case["nsamp"], case["tsamp"], strat_dmshifts, maxshift,
                             k["dm_position"], k["width"], k["signal_start"], k["sigma"])
        return x.reshape(case["nsamp"], case["nchans"])
    return C.make_input(case)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


def sample_positions(shape, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    return [(int(rng.integers(0, shape[0])), int(rng.integers(0, shape[1]))) for _ in range(N_SAMPLES)]


def run_one(name, case, q):
    import refharness as R
    import oracle as O
    L = R.load()
    fm = case["free_memory"]
    sfm = C.strategy_free_memory(case)
    # the strategy the oracle computes drives the fake-signal generator
    st_o = O.strategy(case["plan"], case["nchans"], case["nsamp"], case["fch1"], case["foff"], case["tsamp"],
                      case["nbits"], sfm)
    x = make_case_input(name, case, st_o.dmshifts, st_o.maxshift)
    t0 = time.time()
    s, flat = R.run_ddtr(L, x, case["plan"], case["nchans"], case["nsamp"], case["fch1"], case["foff"],
                         case["tsamp"], case["nbits"], fm)
    t_ref = time.time() - t0
    nr = len(case["plan"])
    ranges, off = [], 0
    outs_ref = []
    for r in range(nr):
        tot = sum(s["t_processed"][r])
        n = s["ndms"][r] * tot
        a = flat[off:off + n].reshape(s["ndms"][r], tot)
        off += n
        outs_ref.append(a)
        pos = sample_positions(a.shape, 1000 + r)
        ranges.append({"sha256": digest(a), "shape": list(a.shape),
                       "samples": [[i, j, int(np.float32(a[i, j]).view(np.uint32))] for i, j in pos],
                       "sum": float(a.astype(np.float64).sum())})
    rec = {"case": name, "strategy": {k: v for k, v in s.items() if k != "dmshifts"},
           "dmshifts_sha256": hashlib.sha256(np.asarray(s["dmshifts"], np.float32).tobytes()).hexdigest(),
           "ranges": ranges, "ref_seconds": t_ref}
    if "kat" in case:
        k = case["kat"]
        dm_idx = int(k["dm_position"]) // int(case["plan"][0][2])
        rec["kat"] = dict(k, dm_index=dm_idx, value=float(outs_ref[0][dm_idx, k["signal_start"]]))
    # oracle under each contraction variant
    if not case.get("heavy"):
        st = O.Strategy(np.asarray(s["dmshifts"], np.float32), s["ndms"], [tuple(d) for d in s["dm"]],
                        s["maxshift"], s["max_ndms"], s["num_tchunks"], s["t_processed"])
        cmp = {}
        for fma in (O.FMA_ALL, 0, O.FMA_TWO | O.FMA_CACHE, O.FMA_ONE | O.FMA_CACHE):
            outs, kern = O.run_ddtr(x, st, case["nchans"], case["nsamp"], case["tsamp"], case["nbits"], fma_mode=fma)
            cmp[str(fma)] = [{"bit_exact": bool(np.array_equal(outs[r].view(np.uint32), outs_ref[r].view(np.uint32))),
                              "n_diff": int((outs[r] != outs_ref[r]).sum()),
                              "max_abs_diff": float(np.abs(outs[r].astype(np.float64) - outs_ref[r]).max())}
                             for r in range(nr)]
            rec["kernels"] = [O.KERNEL_NAMES[kk[0]] for kk in kern]
        rec["oracle_vs_reference"] = cmp
    q.put(rec)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ddtr_golden.json"))
    ap.add_argument("--only", default="")
    ap.add_argument("--merge", default="", help="existing golden file whose other cases are kept")
    args = ap.parse_args()
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    allc = dict(C.CASES)
    allc.update(kat_cases())
    ctx = mp.get_context("spawn")
    results = {}
    if args.merge and os.path.exists(args.merge):
        with open(args.merge) as f:
            results = json.load(f)["cases"]
    for name, case in allc.items():
        if args.only and name not in args.only.split(","):
            continue
        if case.get("no_reference"):
            continue  # the reference's result is undefined for this case (see cases.py)
        q = ctx.Queue()
        p = ctx.Process(target=run_one, args=(name, case, q))
        p.start()
        rec = q.get(timeout=1800)
        p.join(timeout=120)
        results[name] = rec
        print(name, "ok", rec.get("kat", ""), {k: [r["bit_exact"] for r in v]
                                               for k, v in rec.get("oracle_vs_reference", {}).items()}, flush=True)
    with open(args.out, "w") as f:
        json.dump({"generator": "tests/golden/make_ddtr_golden.py", "reference": "AstroAccelerate v1.3.1",
                   "cases": results}, f, indent=1)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
