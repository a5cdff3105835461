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
pinned bit for bit by the reference's own GPU run
(tests/golden/spd_golden.json).  Beside it, the reference's own CPU check of
the first S/N plane (tests/test_single_pulse_search_scan_1.cpp) is restated
below with its error measure, as an independent check of what the plane
means.
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


# ---------------------------------------------------------------------------
# The reference's own CPU check of the first S/N plane
# (tests/test_single_pulse_search_scan_1.cpp:8-40, :110-232), restated.
# ---------------------------------------------------------------------------
def scan_error(a, b):
    """get_error (:13-40): the absolute difference, divided by the power of
    ten of the smaller magnitude when that is above 10."""
    a, b = abs(float(a)), abs(float(b))
    if a > b:
        err = a - b
        if b > 10:
            err /= 10.0 ** int(np.log10(b))
    else:
        err = b - a
        if a > 10:
            err /= 10.0 ** int(np.log10(a))
    return min(err, 10000.0)


def scan_errors(cpu, gpu):
    """get_error over whole arrays (vectorised form of the loop above)."""
    a = np.abs(cpu.astype(np.float64))
    b = np.abs(gpu.astype(np.float64))
    lo = np.minimum(a, b)
    err = np.abs(a - b)
    scale = np.where(lo > 10, 10.0 ** np.floor(np.log10(np.maximum(lo, 1e-30))), 1.0)
    return np.minimum(err / scale, 10000.0)


def decimate_in_time(x):
    """Decimate_in_time (:110-124) with DIT_factor 2: sums of sample pairs."""
    nd, nt = x.shape
    h = nt // 2
    return (x[:, 0:2 * h:2] + x[:, 1:2 * h:2]).astype(np.float32)


def first_plane_scan(x, msd, max_taps):
    """Single_pulse_search_offcentral_1st (:126-181): per sample the best
    (FIR - mean_w) / sd_w over widths 1..max_taps (width 1 as FIR / sqrt(1)),
    the width, and the sums of max_taps samples at even samples.  float32
    arithmetic in the reference's order."""
    x = x.astype(np.float32)
    nd, nt = x.shape
    dtm = nt >> 1
    snr = np.zeros((nd, nt), np.float32)
    taps = np.zeros((nd, nt), np.uint16)
    bv = np.zeros((nd, dtm), np.float32)
    ns = nt - max_taps + 1
    m = np.asarray(msd, np.float32).reshape(-1, 2)
    snr[:, :ns] = (x[:, :ns] - m[0, 0]) / m[0, 1]
    taps[:, :ns] = 1
    fir = x[:, :ns].copy()
    s1 = fir / np.float32(np.sqrt(np.float32(1)))
    better = s1 > snr[:, :ns]
    snr[:, :ns] = np.where(better, s1, snr[:, :ns])
    for t in range(1, max_taps):
        fir = (fir + x[:, t:t + ns]).astype(np.float32)
        s = ((fir - m[t, 0]) / m[t, 1]).astype(np.float32)
        better = s > snr[:, :ns]
        snr[:, :ns] = np.where(better, s, snr[:, :ns])
        taps[:, :ns] = np.where(better, t + 1, taps[:, :ns])
    even = np.arange(0, ns, 2)
    bv[:, even // 2] = fir[:, even]
    for s0 in range(ns, nt):
        if s0 % 2 == 0:
            bv[:, s0 // 2] = x[:, s0:s0 + max_taps].sum(axis=1, dtype=np.float32)
    return snr, taps, bv


# ---------------------------------------------------------------------------
# Peak filtering (candidate algorithm 2), restated on given S/N planes
# ---------------------------------------------------------------------------
def stencil_peaks(snr_planes, taps_planes, plan_rows, ndms, cutoff, shift=0):
    """First stage (src/aa_device_peak_find.cu:9-24 with
    src/aa_device_peak_find_kernel.cu:10-70): per iteration f whose plane has
    searched columns, the interior samples (rows 3..ndms-4, columns
    3..dts-4) that no sample of their 7 x 7 neighbourhood exceeds and that
    are above the cut; records (trial + shift, x*2^f + width/2, S/N, the
    plane's first width).  snr_planes/taps_planes: the whole S/N and width
    areas of one batch; plan_rows: PLAN_FIELDS rows of pd_plan."""
    from numpy.lib.stride_tricks import sliding_window_view
    out = []
    for f, row in enumerate(plan_rows):
        r = dict(zip(PLAN_FIELDS, row))
        dts, off = r["decimated_timesamples"], r["unprocessed_samples"]
        if dts - off - 1 <= 0 or dts < 7 or ndms < 7:
            continue
        o = ndms * r["output_shift"]
        p = snr_planes[o:o + ndms * dts].reshape(ndms, dts)
        t = taps_planes[o:o + ndms * dts].reshape(ndms, dts)
        win = sliding_window_view(p, (7, 7)).max(axis=(2, 3))  # [ndms-6][dts-6], centre at +3
        c = p[3:ndms - 3, 3:dts - 3]
        ys, xs = np.nonzero((c == win) & (c > np.float32(cutoff)))
        bw0 = int(t.reshape(-1)[0])
        for y, x in zip(ys + 3, xs + 3):
            out.append((int(y) + shift, int(x) * (1 << f) + int(t[y, x]) // 2, float(p[y, x]), bw0))
    return out


def filter_peaks(peaks, tsamp):
    """Second stage (src/aa_device_peak_find_kernel.cu:391-486, radius from
    src/aa_device_analysis.cu:398): a peak is dropped when another with at
    least its S/N lies at a float squared distance fd*fd + fs*fs below
    floor(0.015 / tsamp)^2 and not 0."""
    fsz = int(15 * 0.001 / float(np.float32(tsamp)))
    maxd = np.float32(fsz * fsz)
    if not peaks:
        return []
    dm = np.array([q[0] for q in peaks], np.int64)
    ts = np.array([q[1] for q in peaks], np.int64)
    snr = np.array([q[2] for q in peaks], np.float32)
    keep = []
    for i, q in enumerate(peaks):
        fs = dm.astype(np.float32) - np.float32(q[0])
        fd = ts.astype(np.float32) - np.float32(q[1])
        dist = (fd * fd + fs * fs).astype(np.float32)
        hit = (snr >= np.float32(q[2])) & (dist < maxd) & (dist != 0)
        if not hit.any():
            keep.append(q)
    return keep


def suppressor(peak, peaks, tsamp):
    """A peak of the list that drops `peak` under filter_peaks' rule, or None."""
    fsz = int(15 * 0.001 / float(np.float32(tsamp)))
    maxd = np.float32(fsz * fsz)
    for q in peaks:
        fs = np.float32(q[0]) - np.float32(peak[0])
        fd = np.float32(q[1]) - np.float32(peak[1])
        dist = np.float32(fd * fd + fs * fs)
        if np.float32(q[2]) >= np.float32(peak[2]) and dist < maxd and dist != 0:
            return q
    return None
