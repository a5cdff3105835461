"""CPU restatement of the single-pulse detection plan -- TEST INFRASTRUCTURE
ONLY (used by tests/ to check the library's plan and the golden vectors;
never by the library).

The boxcar plan of AstroAccelerate's analysis_GPU:

* BC_widths {PD_MAXTAPS, 16, 16, 16, 8, 8, 8, 8, 8, 8}, PD_MAXTAPS = 32
  (src/aa_device_analysis.cu:140-141, src/aa_params.hpp),
* Get_max_iteration (src/aa_device_analysis.cu:101-121),
* Create_PD_plan (src/aa_device_analysis.cu:44-99) with PD_NTHREADS = 512,
* Create_list_of_boxcar_widths (src/aa_device_analysis.cu:24-42),
* the widest width from the range's sampling time
  (src/aa_device_analysis.cu:131, :179): int(max_boxcar_width_in_sec / tsamp)
  in float, then integer division by inBin.

The device arithmetic (the MSD profile, the S/N planes, the candidates) is
pinned by the reference's own GPU run (tests/golden/spd_golden.json), not
restated here.
"""
from __future__ import annotations

import numpy as np

PD_MAXTAPS = 32
PD_NTHREADS = 512
BC_WIDTHS = [PD_MAXTAPS, 16, 16, 16, 8, 8, 8, 8, 8, 8]
PLAN_FIELDS = ("decimated_timesamples", "dtm", "iteration", "nBoxcars", "nBlocks", "output_shift", "shift",
               "startTaps", "unprocessed_samples", "total_ut")


def max_iteration(max_boxcar_width: int, bc=BC_WIDTHS):
    """(iterations, widest width performed) -- Get_max_iteration."""
    start_taps = 0
    it = 0
    for f, w in enumerate(bc):
        start_taps += w * (1 << f)
        if start_taps >= max_boxcar_width:
            it = f + 1
            break
    if max_boxcar_width > start_taps:
        it = len(bc)
    return it, start_taps


def boxcar_widths(max_width: int, bc=BC_WIDTHS):
    """Create_list_of_boxcar_widths: cumulative widths at 2^f steps up to max_width."""
    out, width, dit = [], 0, 1
    for w in bc:
        for _ in range(w):
            width += dit
            if width <= max_width:
                out.append(width)
        dit *= 2
    return out


def pd_plan(nt: int, bc=BC_WIDTHS):
    """Create_PD_plan: one row of PLAN_FIELDS per iteration."""
    rows = []
    prev = None
    for f, nbox in enumerate(bc):
        if f == 0:
            shift, out_shift, start_taps, it, dts, unproc = 0, 0, 0, 0, nt, nbox + 6
        else:
            shift = prev["nBoxcars"] // 2
            out_shift = prev["output_shift"] + prev["decimated_timesamples"]
            start_taps = prev["startTaps"] + prev["nBoxcars"] * (1 << prev["iteration"])
            it = prev["iteration"] + 1
            dts = prev["dtm"]
            unproc = prev["unprocessed_samples"] // 2 + nbox + 6
        dtm = nt >> (it + 1)
        dtm -= dtm & 1
        epb = PD_NTHREADS * 2 - nbox
        nblocks = dts // epb + (1 if dts - (dts // epb) * epb > 0 else 0)
        if dts < unproc:
            nblocks = 0
        total_ut = unproc * (1 << it)
        row = dict(decimated_timesamples=dts, dtm=dtm, iteration=it, nBoxcars=nbox, nBlocks=nblocks,
                   output_shift=out_shift, shift=shift, startTaps=start_taps, unprocessed_samples=unproc,
                   total_ut=total_ut)
        rows.append(row)
        prev = row
    return rows


def plan(nt: int, tsamp: float, in_bin: int, max_boxcar_width_in_sec: float) -> dict:
    """The whole plan for one range, as analysis_GPU builds it (tsamp is the
    range's sampling time, a float)."""
    mbw = int(np.float32(max_boxcar_width_in_sec) / np.float32(tsamp))
    it, mwp = max_iteration(mbw // in_bin)
    return {"widths": boxcar_widths(mwp), "max_width_performed": mwp, "max_iteration": it,
            "plan": [[r[k] for k in PLAN_FIELDS] for r in pd_plan(nt)]}


def candidate_records(dm, ts, snr, bw, dm_low, dm_step, tsamp, tstart, in_bin):
    """The float records of the candidate file (src/aa_device_analysis.cu:420-427):
    each value computed in double from the float inputs, stored as float."""
    dm = np.asarray(dm, np.float64)
    ts = np.asarray(ts, np.float64)
    rec = np.empty((dm.size, 4), np.float32)
    rec[:, 0] = dm * np.float64(np.float32(dm_step)) + np.float64(np.float32(dm_low))
    rec[:, 1] = ts * np.float64(np.float32(tsamp)) + np.float64(np.float32(tstart))
    rec[:, 2] = np.asarray(snr, np.float32)
    rec[:, 3] = np.asarray(bw, np.float64) * in_bin
    return rec
