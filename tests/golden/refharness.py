"""ctypes access to the reference's own DDTR code, built from its sources by
oracle/Makefile.ref into oracle/_ref/libaaref.so (see oracle/ref_harness.cu).

Used only by the scripts that generate the golden vectors in this folder.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libaaref.so")


class DM(ctypes.Structure):
    _fields_ = [("low", ctypes.c_float), ("high", ctypes.c_float), ("step", ctypes.c_float),
                ("inBin", ctypes.c_int), ("outBin", ctypes.c_int)]


def load():
    L = ctypes.CDLL(REF_LIB)
    P = ctypes.POINTER
    i, f, d, sz = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_size_t
    L.aaref_strategy.argtypes = [P(DM), i, f, i, i, d, d, d, i, sz, i, i, P(f), P(i), P(DM), P(i), P(i), P(i),
                                 P(i)]
    L.aaref_strategy.restype = i
    L.aaref_run_ddtr.argtypes = [ctypes.c_void_p, i, i, d, d, d, i, P(DM), i, sz, i, P(f), P(i), P(DM), P(i),
                                 P(i), P(i), P(i), ctypes.c_void_p, sz]
    L.aaref_run_ddtr.restype = i
    L.aaref_run_ddtr_opts.argtypes = L.aaref_run_ddtr.argtypes + [i, ctypes.c_void_p, i]
    L.aaref_run_ddtr_opts.restype = i
    return L


def _plan(plan):
    arr = (DM * len(plan))()
    for k, (lo, hi, st, ib, ob) in enumerate(plan):
        arr[k].low, arr[k].high, arr[k].step, arr[k].inBin, arr[k].outBin = lo, hi, st, ib, ob
    return arr


def _unpack(nr, nchans, sh, nd, sdm, ms, mx, nt, tp, max_chunks):
    return {
        "dmshifts": sh,
        "ndms": [int(nd[r]) for r in range(nr)],
        "dm": [[float(sdm[r].low), float(sdm[r].high), float(sdm[r].step), int(sdm[r].inBin), int(sdm[r].outBin)]
               for r in range(nr)],
        "maxshift": ms.value,
        "max_ndms": mx.value,
        "num_tchunks": nt.value,
        "t_processed": [[int(tp[r * max_chunks + k]) for k in range(nt.value)] for r in range(nr)],
    }


def strategy(L, plan, nchans, nsamp, fch1, foff, tsamp, nbits, free_memory, power=2.0, enable_analysis=0,
             max_chunks=4096):
    nr = len(plan)
    sh = np.zeros(nchans, np.float32)
    nd, sdm = (ctypes.c_int * nr)(), (DM * nr)()
    ms, mx, nt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    tp = np.zeros(nr * max_chunks, np.int32)
    rc = L.aaref_strategy(_plan(plan), nr, power, nchans, nsamp, fch1, foff, tsamp, nbits, free_memory,
                          enable_analysis, max_chunks, sh.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), nd, sdm,
                          ctypes.byref(ms), ctypes.byref(mx), ctypes.byref(nt),
                          tp.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if rc != 0:
        return None
    return _unpack(nr, nchans, sh, nd, sdm, ms, mx, nt, tp, max_chunks)


def run_ddtr(L, input_tc, plan, nchans, nsamp, fch1, foff, tsamp, nbits, free_memory, max_chunks=4096,
             out_len=None, options=0, bandpass=None):
    """Runs the reference pipeline on the GPU; returns (strategy, flat output).
    options: bit mask of the runner's processing options (oracle/ref_harness.cu
    aaref_run_ddtr_opts); bandpass: float32 values bound to the plan."""
    nr = len(plan)
    sh = np.zeros(nchans, np.float32)
    nd, sdm = (ctypes.c_int * nr)(), (DM * nr)()
    ms, mx, nt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    tp = np.zeros(nr * max_chunks, np.int32)
    if out_len is None:
        out_len = 1 << 28
    out = np.zeros(out_len, np.float32)
    x = np.ascontiguousarray(input_tc, dtype=np.uint16)
    bp = None if bandpass is None else np.ascontiguousarray(bandpass, dtype=np.float32)
    rc = L.aaref_run_ddtr_opts(x.ctypes.data, nchans, nsamp, tsamp, fch1, foff, nbits, _plan(plan), nr, free_memory,
                               max_chunks, sh.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), nd, sdm,
                               ctypes.byref(ms), ctypes.byref(mx), ctypes.byref(nt),
                               tp.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), out.ctypes.data, out_len, options,
                               None if bp is None else bp.ctypes.data, 0 if bp is None else bp.size)
    if rc != 0:
        raise RuntimeError(f"reference pipeline failed (code {rc})")
    s = _unpack(nr, nchans, sh, nd, sdm, ms, mx, nt, tp, max_chunks)
    n = sum(s["ndms"][r] * sum(s["t_processed"][r]) for r in range(nr))
    return s, out[:n].copy()
