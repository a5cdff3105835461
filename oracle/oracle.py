"""ctypes wrapper of the CPU DDTR oracle (oracle/aa_oracle.c).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()``
and by the ``cpu_baseline`` / reference leg of ``bench.py`` -- as the checker,
never as the thing measured for the product and never as a fallback for it.

The oracle restates AstroAccelerate v1.3.1's DDTR path (strategy, kernel
choice, per-kernel delay arithmetic, corner turn, x2 binning, runner loop,
fake-signal generator); see the citations in aa_oracle.c.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "libaaoracle.so")

K_SHARED8, K_SHARED16, K_SHARED4, K_CACHE = 0, 1, 2, 3
KERNEL_NAMES = {K_SHARED8: "shared8", K_SHARED16: "shared16", K_SHARED4: "shared4", K_CACHE: "cache"}
FMA_TWO, FMA_ONE, FMA_CACHE, FMA_ALL = 1, 2, 4, 7
STRIDE_REFERENCE, STRIDE_TRUE = 0, 1
MAX_CHUNKS = 4096


class DM(ctypes.Structure):
    """include/aa_ddtr_plan.hpp:28-34 struct dm."""

    _fields_ = [("low", ctypes.c_float), ("high", ctypes.c_float), ("step", ctypes.c_float),
                ("inBin", ctypes.c_int), ("outBin", ctypes.c_int)]


def build(force: bool = False) -> str:
    """Compile the oracle with OpenMP and without FMA contraction."""
    src = os.path.join(HERE, "aa_oracle.c")
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "aa_oracle.h"))):
        return LIB_PATH
    os.makedirs(BUILD_DIR, exist_ok=True)
    cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-fno-fast-math", "-o", LIB_PATH, src, "-lm"]
    subprocess.check_call(cmd)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        L.aao_strategy.argtypes = [P(DM), ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                   P(ctypes.c_float), P(ctypes.c_int), P(DM), P(ctypes.c_int),
                                   P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int)]
        L.aao_strategy.restype = ctypes.c_int
        L.aao_select_kernel.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                        ctypes.c_int]
        L.aao_select_kernel.restype = ctypes.c_int
        L.aao_delay.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                ctypes.c_float, ctypes.c_float]
        L.aao_delay.restype = ctypes.c_int
        L.aao_dedisperse.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_void_p]
        L.aao_dedisperse.restype = ctypes.c_int
        L.aao_dedisperse_window.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_longlong, ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p,
                                            ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_void_p]
        L.aao_dedisperse_window.restype = ctypes.c_int
        L.aao_corner_turn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.aao_corner_turn.restype = None
        L.aao_bin_flat.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int]
        L.aao_bin_flat.restype = ctypes.c_int
        L.aao_run_ddtr.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_int, ctypes.c_void_p, P(DM), ctypes.c_void_p, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                   ctypes.c_void_p]
        L.aao_run_ddtr.restype = ctypes.c_int
        L.aao_fake_signal.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_float, ctypes.c_int, P(ctypes.c_int)]
        L.aao_fake_signal.restype = ctypes.c_int
        L.aao_num_threads.restype = ctypes.c_int
        L.aao_set_num_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


@dataclass
class Strategy:
    """Fields of aa_ddtr_strategy (include/aa_ddtr_strategy.hpp:55-131)."""

    dmshifts: np.ndarray
    ndms: list
    dm: list  # (low, high, step, inBin, outBin) after the grid redefinition
    maxshift: int
    max_ndms: int
    num_tchunks: int
    t_processed: list  # [range][chunk]
    plan: list = field(default_factory=list)

    def total_samps(self, r: int) -> int:
        return int(sum(self.t_processed[r]))

    def output_size(self) -> int:
        return int(sum(self.ndms[r] * self.total_samps(r) for r in range(len(self.ndms))))


def plan_array(plan):
    arr = (DM * len(plan))()
    for i, (lo, hi, st, ib, ob) in enumerate(plan):
        arr[i].low, arr[i].high, arr[i].step, arr[i].inBin, arr[i].outBin = lo, hi, st, ib, ob
    return arr


def strategy(plan, nchans, nsamp, fch1, foff, tsamp, nbits, free_memory=180 * 2**30,
             power=2.0, enable_analysis=False) -> Strategy:
    """Restatement of aa_ddtr_strategy::strategy (src/aa_ddtr_strategy.cpp:27-428)."""
    L = lib()
    nr = len(plan)
    parr = plan_array(plan)
    dmshifts = np.zeros(nchans, np.float32)
    ndms = (ctypes.c_int * nr)()
    sdm = (DM * nr)()
    ms, mx, nt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    tp = np.zeros(nr * MAX_CHUNKS, np.int32)
    rc = L.aao_strategy(parr, nr, power, nchans, nsamp, fch1, foff, tsamp, nbits, free_memory,
                        int(enable_analysis), MAX_CHUNKS,
                        dmshifts.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ndms, sdm,
                        ctypes.byref(ms), ctypes.byref(mx), ctypes.byref(nt),
                        tp.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if rc != 0:
        raise ValueError(f"oracle strategy refused the plan (code {rc})")
    tpl = [[int(tp[r * MAX_CHUNKS + k]) for k in range(nt.value)] for r in range(nr)]
    dms = [(sdm[i].low, sdm[i].high, sdm[i].step, sdm[i].inBin, sdm[i].outBin) for i in range(nr)]
    return Strategy(dmshifts, [int(ndms[i]) for i in range(nr)], dms, ms.value, mx.value, nt.value, tpl,
                    list(plan))


def select_kernel(nbits, dm_step, tsamp_r, dmshift_last, failsafe=0) -> int:
    return lib().aao_select_kernel(nbits, dm_step, tsamp_r, dmshift_last, failsafe)


def delay(kernel, fma_mode, dms, dm, tx, mstartdm, mdmstep) -> int:
    return lib().aao_delay(kernel, fma_mode, dms, dm, tx, mstartdm, mdmstep)


def dedisperse(kernel, fma_mode, flat: np.ndarray, i_nsamp, nchans, t_processed, ndms, dmshifts,
               mstartdm, mdmstep, bin_, want_sums=False):
    flat = np.ascontiguousarray(flat, dtype=np.uint16)
    dmshifts = np.ascontiguousarray(dmshifts, dtype=np.float32)
    out = np.zeros((ndms, t_processed), np.float32)
    sums = np.zeros((ndms, t_processed), np.float64) if want_sums else None
    rc = lib().aao_dedisperse(kernel, fma_mode, _ptr(flat), flat.size, i_nsamp, nchans, t_processed,
                              ndms, _ptr(dmshifts), mstartdm, mdmstep, bin_, _ptr(out),
                              _ptr(sums) if want_sums else None)
    if rc != 0:
        raise ValueError(f"oracle dedisperse failed (code {rc})")
    return (out, sums) if want_sums else out


def dedisperse_window(kernel, fma_mode, flat: np.ndarray, i_nsamp, nchans, dm_first, ndm, t_first, nt,
                      dmshifts, mstartdm, mdmstep, bin_, t_shift=0, want_sums=False):
    """DM trials dm_first.. and outputs t_first.. of one (chunk, range);
    output t reads flat[c*i_nsamp + t - t_shift + delay] (a buffer that starts
    t_shift samples into the channel rows).  Returns [ndm][nt]."""
    flat = np.ascontiguousarray(flat, dtype=np.uint16)
    dmshifts = np.ascontiguousarray(dmshifts, dtype=np.float32)
    out = np.zeros((ndm, nt), np.float32)
    sums = np.zeros((ndm, nt), np.float64) if want_sums else None
    rc = lib().aao_dedisperse_window(kernel, fma_mode, _ptr(flat), flat.size, i_nsamp, nchans, dm_first, ndm,
                                     t_first, nt, t_shift, _ptr(dmshifts), mstartdm, mdmstep, bin_, _ptr(out),
                                     _ptr(sums) if want_sums else None)
    if rc != 0:
        raise ValueError(f"oracle dedisperse failed (code {rc})")
    return (out, sums) if want_sums else out


def corner_turn(in_tc: np.ndarray, nchans: int, nsamp: int) -> np.ndarray:
    in_tc = np.ascontiguousarray(in_tc, dtype=np.uint16)
    out = np.empty(nchans * nsamp, np.uint16)
    lib().aao_corner_turn(_ptr(in_tc), _ptr(out), nchans, nsamp)
    return out


def bin_flat(buf: np.ndarray, nchans: int, nsamp: int) -> np.ndarray:
    """In-place reference x2 binning (src/aa_bin_gpu.cpp:8-44) on a copy."""
    b = np.array(buf, dtype=np.uint16, copy=True)
    rc = lib().aao_bin_flat(_ptr(b), b.size, nchans, nsamp)
    if rc != 0:
        raise ValueError(f"oracle bin failed (code {rc})")
    return b


def run_ddtr(input_tc: np.ndarray, strat: Strategy, nchans, nsamp, tsamp, nbits,
             fma_mode=FMA_ALL, stride_mode=STRIDE_REFERENCE, failsafe=0):
    """Whole-run replay of the reference runner; returns the per-range output
    arrays [ndms][sum_k t_processed] and the kernel chosen per (range, chunk)."""
    L = lib()
    nr = len(strat.ndms)
    input_tc = np.ascontiguousarray(input_tc, dtype=np.uint16)
    sdm = plan_array(strat.dm)
    ndms = np.array(strat.ndms, np.int32)
    tp = np.zeros(nr * MAX_CHUNKS, np.int32)
    for r in range(nr):
        for k in range(strat.num_tchunks):
            tp[r * MAX_CHUNKS + k] = strat.t_processed[r][k]
    out = np.zeros(strat.output_size(), np.float32)
    kern = np.full(nr * MAX_CHUNKS, -1, np.int32)
    rc = L.aao_run_ddtr(_ptr(input_tc), nchans, nsamp, tsamp, nbits, _ptr(strat.dmshifts), sdm,
                        _ptr(ndms), nr, strat.maxshift, strat.num_tchunks, _ptr(tp), MAX_CHUNKS,
                        fma_mode, stride_mode, failsafe, _ptr(out), _ptr(kern))
    if rc != 0:
        raise ValueError(f"oracle run failed (code {rc})")
    outs, off = [], 0
    for r in range(nr):
        n = strat.ndms[r] * strat.total_samps(r)
        outs.append(out[off:off + n].reshape(strat.ndms[r], strat.total_samps(r)))
        off += n
    kernels = [[int(kern[r * MAX_CHUNKS + k]) for k in range(strat.num_tchunks)] for r in range(nr)]
    return outs, kernels


def fake_signal(nchans, nsamples, tsamp, dmshifts, maxshift, dm_pos, width, signal_start, sigma,
                period_ms=0):
    """src/aa_host_fake_signal_generator.cpp:13-116, time-major [t][c] ushort."""
    out = np.zeros(nsamples * nchans, np.uint16)
    dmshifts = np.ascontiguousarray(dmshifts, dtype=np.float32)
    mp = ctypes.c_int()
    rc = lib().aao_fake_signal(_ptr(out), nchans, nsamples, tsamp, _ptr(dmshifts), maxshift, dm_pos,
                               width, signal_start, sigma, period_ms, ctypes.byref(mp))
    if rc != 0:
        raise ValueError(f"fake signal refused (code {rc})")
    return out, mp.value


def num_threads() -> int:
    return lib().aao_num_threads()


def set_num_threads(n: int) -> None:
    lib().aao_set_num_threads(n)
