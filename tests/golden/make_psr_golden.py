"""Generates tests/golden/psr_golden.json from the reference's own GPU
periodicity stages (oracle/ref_harness.cu aaref_psr_blocks:
simple_power_and_interbin and periodicity_simple_harmonic_summing; the MSD
profile, peak finding and thresholding, the harmonic sums and the spectral
whitening of the other aaref_psr_* entries) on the
seeded inputs of psr_cases.py: SHA-256 of every output and its first
values.  Needs a GPU.

    python tests/golden/make_psr_golden.py --out <dir>/psr_golden.json
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)

import psr_cases as P  # noqa: E402
import refharness as R  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "psr_golden.json"))
    args = ap.parse_args()
    L = R.load()
    Pf, i = ctypes.POINTER(ctypes.c_float), ctypes.c_int
    L.aaref_psr_blocks.argtypes = [Pf, i, i, Pf, Pf, Pf, i, i, Pf, i, Pf, ctypes.POINTER(ctypes.c_ushort)]
    L.aaref_psr_blocks.restype = i
    out = {"generator": "tests/golden/make_psr_golden.py", "reference": "AstroAccelerate v1.3.1", "power": {},
           "harmonic": {}}
    hc = next(iter(P.HARMONIC_CASES.values()))
    for name, c in P.POWER_CASES.items():
        spec = P.make_spectra(c)
        pw = np.zeros(c["ndms"] * (c["nt"] >> 1), np.float32)
        ib = np.zeros(c["ndms"] * c["nt"], np.float32)
        x, msd = P.make_harmonic_input(hc)
        snr = np.zeros(x.size, np.float32)
        hm = np.zeros(x.size, np.uint16)
        rc = L.aaref_psr_blocks(spec.ctypes.data_as(Pf), c["nt"], c["ndms"], pw.ctypes.data_as(Pf),
                                ib.ctypes.data_as(Pf), x.ctypes.data_as(Pf), hc["nbins"], hc["nspectra"],
                                msd.ctypes.data_as(Pf), hc["nh"], snr.ctypes.data_as(Pf),
                                hm.ctypes.data_as(ctypes.POINTER(ctypes.c_ushort)))
        out["power"][name] = {"rc": rc, "power_sha256": hashlib.sha256(pw.tobytes()).hexdigest(),
                              "interbin_sha256": hashlib.sha256(ib.tobytes()).hexdigest(),
                              "power_head": pw[:256].view(np.uint32).tolist(),
                              "interbin_head": ib[:256].view(np.uint32).tolist()}
        print(name, rc, flush=True)
    for name, c in P.HARMONIC_CASES.items():
        cp = next(iter(P.POWER_CASES.values()))
        spec = P.make_spectra(cp)
        pw = np.zeros(cp["ndms"] * (cp["nt"] >> 1), np.float32)
        ib = np.zeros(cp["ndms"] * cp["nt"], np.float32)
        x, msd = P.make_harmonic_input(c)
        snr = np.zeros(x.size, np.float32)
        hm = np.zeros(x.size, np.uint16)
        rc = L.aaref_psr_blocks(spec.ctypes.data_as(Pf), cp["nt"], cp["ndms"], pw.ctypes.data_as(Pf),
                                ib.ctypes.data_as(Pf), x.ctypes.data_as(Pf), c["nbins"], c["nspectra"],
                                msd.ctypes.data_as(Pf), c["nh"], snr.ctypes.data_as(Pf),
                                hm.ctypes.data_as(ctypes.POINTER(ctypes.c_ushort)))
        out["harmonic"][name] = {"rc": rc, "snr_sha256": hashlib.sha256(snr.tobytes()).hexdigest(),
                                 "harmonics_sha256": hashlib.sha256(hm.tobytes()).hexdigest(),
                                 "snr_head": snr[:512].view(np.uint32).tolist(), "harmonics_head": hm[:512].tolist()}
        print(name, rc, flush=True)
    L.aaref_msd_profile.argtypes = [Pf, i, i, ctypes.POINTER(ctypes.c_int), i, i, ctypes.c_float, i, Pf]
    L.aaref_msd_profile.restype = i
    out["msd"] = {}
    for name, c in P.MSD_CASES.items():
        x = np.ascontiguousarray(P.make_power_plane(c))
        w = np.arange(1, c["nh"] + 1, dtype=np.int32)
        msd = np.zeros(2 * c["nh"], np.float32)
        rc = L.aaref_msd_profile(x.ctypes.data_as(Pf), c["nt"], c["ndms"],
                                 w.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), c["nh"], c["high_memory"],
                                 c["sigma"], c["outliers"], msd.ctypes.data_as(Pf))
        out["msd"][name] = {"rc": rc, "msd_bits": msd.view(np.uint32).tolist()}
        print(name, rc, flush=True)
    L.aaref_psr_peaks.argtypes = [Pf, ctypes.POINTER(ctypes.c_ushort), i, i, ctypes.c_float, Pf, i, i, i, i, i, Pf,
                                  i, ctypes.POINTER(ctypes.c_int), i]
    L.aaref_psr_peaks.restype = i
    out["peaks"] = {}
    out["threshold"] = {}
    for (name, c), mode in [(kv, 0) for kv in P.PEAK_CASES.items()] + [(kv, 1) for kv in P.PEAK_CASES.items()]:
        snr, harm, msd = P.make_peak_plane(c)
        max_peaks = 1 << 20
        lst = np.zeros(4 * max_peaks, np.float32)
        cnt = ctypes.c_int()
        rc = L.aaref_psr_peaks(np.ascontiguousarray(snr).ctypes.data_as(Pf),
                               np.ascontiguousarray(harm).ctypes.data_as(ctypes.POINTER(ctypes.c_ushort)), c["nt"],
                               c["ndms"], c["threshold"], msd.ctypes.data_as(Pf), c["nh"], c["dm_shift"], c["inbin"],
                               c["transposed"], c["greedy"], lst.ctypes.data_as(Pf), max_peaks, ctypes.byref(cnt),
                               mode)
        k = cnt.value
        recs = sorted(tuple(int(v) for v in r) for r in lst[:4 * k].view(np.uint32).reshape(-1, 4))
        out["threshold" if mode else "peaks"][name] = {
            "rc": rc, "count": k, "records_sha256": hashlib.sha256(json.dumps(recs).encode()).hexdigest(),
            "records_head": recs[:32]}
        print(name, "threshold" if mode else "peaks", rc, k, flush=True)
    L.aaref_psr_harmonics.argtypes = [i, Pf, i, i, Pf, i, i, i, Pf, ctypes.POINTER(ctypes.c_ushort)]
    L.aaref_psr_harmonics.restype = i
    out["harmonic_algorithms"] = {}
    for name, c in P.HS_ALGO_CASES.items():
        x, msd = P.make_hs_algo_input(c)
        snr = np.zeros(x.size, np.float32)
        hm = np.zeros(x.size, np.uint16)
        rc = L.aaref_psr_harmonics(c["algorithm"], np.ascontiguousarray(x).ctypes.data_as(Pf), c["nt"], c["ndms"],
                                   msd.ctypes.data_as(Pf), 32, c["nh"], c["scalloping"], snr.ctypes.data_as(Pf),
                                   hm.ctypes.data_as(ctypes.POINTER(ctypes.c_ushort)))
        out["harmonic_algorithms"][name] = {"rc": rc, "snr_sha256": hashlib.sha256(snr.tobytes()).hexdigest(),
                                            "harmonics_sha256": hashlib.sha256(hm.tobytes()).hexdigest(),
                                            "snr_head": snr[:256].view(np.uint32).tolist(),
                                            "harmonics_head": hm[:256].tolist()}
        print(name, rc, flush=True)
    L.aaref_psr_whitening.argtypes = [Pf, ctypes.c_longlong, i, Pf, ctypes.POINTER(ctypes.c_int), i,
                                      ctypes.POINTER(ctypes.c_int)]
    L.aaref_psr_whitening.restype = i
    out["whitening"] = {}
    for name, c in P.WHITENING_CASES.items():
        z = P.make_red_spectra(c)
        x = np.ascontiguousarray(z.view(np.float32))
        y = np.zeros_like(x)
        seg = np.zeros(1 << 16, np.int32)
        nseg = ctypes.c_int()
        rc = L.aaref_psr_whitening(x.ctypes.data_as(Pf), c["n"], c["ndms"], y.ctypes.data_as(Pf),
                                   seg.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), seg.size, ctypes.byref(nseg))
        seg = seg[:nseg.value].tolist()
        yc = y.view(np.complex64).reshape(c["ndms"], c["n"])
        shared = P.shared_bins(seg)
        stale = P.stale_bins(seg)
        masked = yc.copy()
        masked[:, shared] = 0
        masked[:, stale] = 0
        out["whitening"][name] = {
            "rc": rc, "segments": seg, "out_sha256": hashlib.sha256(y.tobytes()).hexdigest(),
            "masked_sha256": hashlib.sha256(masked.tobytes()).hexdigest(),
            "shared": [[d, b, int(yc[d, b:b + 1].view(np.uint32)[0]), int(yc[d, b:b + 1].view(np.uint32)[1])]
                       for d in range(c["ndms"]) for b in shared],
            "stale": [[d, b, int(yc[d, b:b + 1].view(np.uint32)[0]), int(yc[d, b:b + 1].view(np.uint32)[1])]
                      for d in range(c["ndms"]) for b in stale],
            "head": y.reshape(c["ndms"], -1)[0, :256].view(np.uint32).tolist(),
            "tail": y.reshape(c["ndms"], -1)[-1, -256:].view(np.uint32).tolist()}
        print(name, rc, len(seg), flush=True)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
