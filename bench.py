#!/usr/bin/env python3
"""Benchmark of the B200 dedispersion (DDTR) path.

One "step" is one full DDTR pass -- every time chunk and DM range of the
strategy -- over one synthetic filterbank of the survey-scale configuration:
4096 channels, 8-bit, fch1 1670 MHz, foff -0.0732421875 MHz, tsamp 64 us,
2^21 samples, the 8-range plan 0-150/0.1/1 ... 2000-3000/2.0/8, seeded
Gaussian noise N(127.5, 16) plus 8 dispersed boxcar pulses (DM U[50, 2900],
width log-U[0.25, 8] ms, 3-10 sigma).

  value     DM-trial.samples/s with the input resident in HBM ([t][c] uint16)
            and the output kept in HBM; corner turn, binning and dedispersion
            of all chunks and ranges are timed with CUDA events on the
            library's stream.
  parity    the timed run's output compared bit for bit with the oracle on
            windows it computes in seconds (chunk 0 range 0, the first binned
            range, every range of the last chunk); a mismatch fails the run.
  e2e       the same metric through the reference-facing C ABI
            (aa_py_pipeline_api / run loop) from a pinned host input to the
            pinned host float*** output, host<->device copies inside the timed
            region (wall clock between device synchronisations).
  roofline  the dedispersion kernel's channel adds/s against the shared-memory
            load rate measured on the same GPU (4 adds per 32-bit load), with
            the HBM figure beside it.
  batched_vs_plain  the first 8 beams of the seeded multi-beam draw, batched
            (one graph, one persistent kernel) and beam by beam, bit-exact.

`--impl reference` times the reference path's CPU restatement (the oracle;
the reference ships no CPU DDTR) on the host's cores on a bounded sample
of the same workload, and the reference's own GPU pipeline (built from its
sources) at 2^18 samples.  Under torchrun every rank runs its own beam (weak
scaling, no collective on the data path); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "astro-accelerate_b200"))

SURVEY = dict(nchans=4096, nbits=8, fch1=1670.0, foff=-0.0732421875, tsamp=64e-6, nsamp=1 << 21,
              plan=[(0, 150, 0.1, 1, 1), (150, 300, 0.2, 1, 1), (300, 500, 0.25, 1, 1), (500, 900, 0.4, 2, 1),
                    (900, 1200, 0.6, 4, 1), (1200, 1500, 0.8, 4, 1), (1500, 2000, 1.0, 4, 1),
                    (2000, 3000, 2.0, 8, 1)],
              npulses=8, seed=20)
MID = dict(SURVEY, nsamp=1 << 18)
SMALL = dict(nchans=1024, nbits=8, fch1=1550.0, foff=-0.390625, tsamp=64e-6, nsamp=1 << 18,
             plan=[(0, 500, 0.5, 1, 1)], npulses=1, seed=1)
METRIC = "DM-trial*samples/s (plain DDTR, 1 beam per GPU, bit-exact)"
METRIC_UNCHECKED = "DM-trial*samples/s (plain DDTR, 1 beam per GPU)"
# DRAM bytes per algorithmic byte of each one-byte dedispersion kernel, from
# one ncu capture each (dram__bytes_read.sum + dram__bytes_write.sum of the
# range-0 launch of the 4096 ch x 2^18 plan, 2.46 GB algorithmic); the
# roofline's traffic is each range's ratio times its algorithmic bytes,
# averaged per launch
TRAFFIC_PER_ALG_BYTE = {"k_ddtr_quad": (0.96 + 1.35) / 2.46, "k_ddtr_sub": (0.954 + 1.504) / 2.46}
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one range-0 launch of 4096 ch x 2^18 samples "
                  "per kernel (k_ddtr_quad 0.96 + 1.35 GB, k_ddtr_sub 0.95 + 1.50 GB, against 2.46 GB algorithmic), "
                  "scaled by the algorithmic bytes of each range of this workload; "
                  "profiles/k_ddtr_quad_mid_8bit_4096ch_2e18_range0.md, profiles/k_ddtr_sub_mid_8bit_4096ch_2e18_range0.md")
PUBLISHED_REALTIME = 6.28  # reference wiki, 8-range "b2" plan, unnamed GPU


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="survey",
                    choices=["survey", "mid", "small", "batched", "refine", "e2e", "spd", "whitening", "periodicity"])
    ap.add_argument("--beams", type=int, default=48, help="beams of the multi-beam draw (batched config)")
    ap.add_argument("--snippets", type=int, default=256, help="snippets per step (refine config)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle check of the timed output")
    ap.add_argument("--no-autotune", action="store_true", help="no per-range kernel timing at set-up")
    ap.add_argument("--tune-file", default="",
                    help="autotuner choices: read from this file if it exists (those ranges are not timed again) "
                         "and written to it after the warm-up (a profiling run reuses a plain run's choices)")
    ap.add_argument("--multibeam-beams", type=int, default=8,
                    help="beams of the reduced multi-beam draw timed batched vs plain in the default line (0: off)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--tile-words", type=int, default=0)
    ap.add_argument("--group-dms", type=int, default=0)
    ap.add_argument("--variant", type=int, default=0,
                    help="0 auto (autotuned per range), 1 generic kernels, 2 channel-quad, 3 subband, "
                         "4 warp-specialised channel-quad, 5 split-phase channel-quad, 6 channel-quad with the "
                         "per-byte warp switch, 7 channel-quad on 256-sample tiles, 8 channel-quad pair rows, "
                         "9 channel-quad loading every DM trial's word first, 10 as 2 without the per-byte path, "
                         "11 as 9 without the per-byte path, 12 as 11 with 32-bit shared addresses (2-12 run the "
                         "staged fp32 kernel on two-byte data)")
    ap.add_argument("--with-analysis", action="store_true",
                    help="add an e2e run through the C ABI with the analysis component after every step")
    ap.add_argument("--spd-nt", type=int, default=0, help="samples per DM trial of the spd config (default 2^19)")
    ap.add_argument("--nbits", type=int, default=0, help="bit depth of the synthetic filterbank (default: the config's)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
def synth_input_device(cfg, seed, device):
    """[nsamp][nchans] uint16 (bit pattern in an int16 tensor) on the GPU."""
    import numpy as np
    import torch
    nchans, nsamp = cfg["nchans"], cfg["nsamp"]
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    vmax = (1 << min(cfg["nbits"], 16)) - 1
    mid, sig = (vmax + 1) / 2.0 - 0.5, (vmax + 1) / 16.0
    x = torch.empty((nsamp, nchans), dtype=torch.int16, device=device)
    rows = 1 << 16
    for t0 in range(0, nsamp, rows):
        n = min(rows, nsamp - t0)
        v = torch.randn((n, nchans), generator=g, device=device) * sig + mid
        x[t0:t0 + n] = v.round_().clamp_(0, vmax).to(torch.int32).to(torch.int16)
    rng = np.random.Generator(np.random.PCG64(seed))
    f = cfg["fch1"] + cfg["foff"] * np.arange(nchans, dtype=np.float64)
    pulses = []
    for _ in range(cfg["npulses"]):
        dm = float(rng.uniform(50, 2900)) if len(cfg["plan"]) > 1 else 300.0
        width = max(1, int(round(math.exp(rng.uniform(math.log(0.25), math.log(8.0))) * 1e-3 / cfg["tsamp"])))
        amp = float(rng.uniform(3, 10)) * sig
        start = int(rng.integers(0, nsamp // 2))
        d = np.floor(4.148808e3 * dm * (f ** -2 - cfg["fch1"] ** -2) / cfg["tsamp"]).astype(np.int64)
        tt = (start + d[None, :] + np.arange(width)[:, None])
        cc = np.broadcast_to(np.arange(nchans)[None, :], tt.shape)
        ok = tt < nsamp
        ti = torch.as_tensor(tt[ok], device=device)
        ci = torch.as_tensor(cc[ok], device=device)
        vals = ((x[ti, ci].to(torch.int32) & 0xFFFF).to(torch.float32) + amp).clamp_(0, vmax)
        x[ti, ci] = vals.to(torch.int32).to(torch.int16)
        pulses.append(dict(dm=dm, width=width, amp_sigma=amp / sig, start=start))
    torch.cuda.synchronize(device)
    return x, pulses


def metadata_struct(aa, cfg):
    return aa.filterbank_metadata_struct(0.0, cfg["tsamp"], cfg["fch1"], cfg["foff"], cfg["nbits"], cfg["nsamp"],
                                         cfg["nchans"], 0.0)


def units_per_step(strat):
    return sum(strat["ndms"][r] * sum(strat["t_processed"][r]) for r in range(len(strat["ndms"])))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the first sample before the timed region starts (nvidia-smi
            # takes a moment to come up), so short regions are not unsampled
            t0 = time.perf_counter()
            while not self.rows and self.proc.poll() is None and time.perf_counter() - t0 < 5.0:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        self.n_enter = len(self.rows)
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            # one sample at or after the end of a region shorter than the period
            t0 = time.perf_counter()
            while len(self.rows) <= self.n_enter and self.proc.poll() is None and time.perf_counter() - t0 < 1.0:
                time.sleep(0.01)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[4 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------------------
def cpu_baseline(cfg, x_host_tc, seconds):
    """The oracle on a bounded sample: range 0, 64-trial DM blocks over a
    131040-sample window of chunk 0, repeated over DM blocks until `seconds`
    of CPU work (strategy from the oracle too).  Returns (DM-trial.samples/s,
    threads, description)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    ost = O.strategy(cfg["plan"], cfg["nchans"], cfg["nsamp"], cfg["fch1"], cfg["foff"], cfg["tsamp"], cfg["nbits"])
    nch = cfg["nchans"]
    tp = min(131040, ost.t_processed[0][0])
    L = tp + ost.maxshift
    flat = O.corner_turn(np.ascontiguousarray(x_host_tc[:L]), nch, L)
    d = ost.dm[0]
    kind, m0, ms = _range_delay_params(O, cfg, d, ost.dmshifts[-1])
    done, t_total, blocks = 0, 0.0, 0
    while t_total < seconds and blocks * 64 < ost.ndms[0]:
        t0 = time.perf_counter()
        O.dedisperse_window(kind, O.FMA_ALL, flat, L, nch, 64 * blocks, 64, 0, tp, ost.dmshifts, m0, ms, d[3])
        t_total += time.perf_counter() - t0
        done += 64 * tp
        blocks += 1
    return done / t_total, O.num_threads(), (f"oracle on {blocks} x 64 DM trials of range 0 over {tp} samples of "
                                             f"chunk 0 ({nch} channels), {t_total:.1f} s")


# ---------------------------------------------------------------------------
PARITY_T = 65536  # outputs per DM trial of the windowed chunk-0 checks


def _range_delay_params(O, cfg, d, dmshift_last):
    """Kernel kind, mstartdm and mdmstep of one range as the reference runner
    computes them (include/aa_permitted_pipelines_generic.hpp:778,
    src/aa_dedisperse.cpp:18-30): float arithmetic throughout."""
    import numpy as np
    tsr = np.float32(cfg["tsamp"]) * np.float32(d[3])
    kind = O.select_kernel(cfg["nbits"], d[2], tsr, dmshift_last)
    return kind, np.float32(np.float32(d[0]) / tsr), np.float32(np.float32(d[2]) / tsr)


def parity_checks(cfg, ost, host_rows, device_rows, log=None):
    """Bit-for-bit comparison of the timed run's device output with the oracle
    on windows the oracle finishes in seconds:

      * chunk 0, range 0: the last 64-trial DM block, outputs [0, PARITY_T);
      * chunk 0, the first x2-binned range: its last DM block over PARITY_T
        binned outputs (the oracle bins a window of the corner-turned chunk
        as the reference's first binning step does);
      * the last chunk (whose input starts beyond 2^31 elements for the
        survey size): a replay of the reference runner's flat buffer for that
        chunk -- corner turn, every x2 binning with the runner's lengths
        (including the mis-strided second and third steps) -- and the last
        DM block of every range over all its outputs.

    host_rows(a, b) returns input rows [a, b) as [t][c] uint16;
    device_rows(r, dm0, ndm, col0, ncol) the timed output.  Returns the
    summary dict for the bench line."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    nch, nr = cfg["nchans"], len(ost.ndms)
    last = ost.dmshifts[-1]
    checks, compared, bad = [], 0, 0
    t_start = time.perf_counter()

    def compare(label, want, r, dm0, col0):
        nonlocal compared, bad
        got = device_rows(r, dm0, want.shape[0], col0, want.shape[1])
        nbad = int(np.count_nonzero(got.view(np.uint32) != want.view(np.uint32)))
        compared += want.size
        bad += nbad
        checks.append({"check": label, "range": r, "dm_trials": [dm0, dm0 + want.shape[0]],
                       "outputs": [col0, col0 + want.shape[1]], "mismatching": nbad})
        if log:
            log(f"parity {label}: {want.size} outputs, {nbad} mismatching")

    def last_block(r):
        return 64 * (ost.ndms[r] // 64 - 1)

    # chunk 0, range 0
    d = ost.dm[0]
    kind, m0, ms = _range_delay_params(O, cfg, d, last)
    T = min(PARITY_T, ost.t_processed[0][0])
    L = T + ost.maxshift // d[3]
    flat = O.corner_turn(host_rows(0, L), nch, L)
    dm0 = last_block(0)
    want = O.dedisperse_window(kind, O.FMA_ALL, flat, L, nch, dm0, 64, 0, T, ost.dmshifts, m0, ms, d[3])
    compare("chunk 0 range 0", want, 0, dm0, 0)
    # chunk 0, first binned range (a single x2 step from unbinned data)
    r1 = next((r for r in range(1, nr) if ost.dm[r][3] == 2 and ost.dm[r - 1][3] == 1), None)
    if r1 is not None and nch % 32 == 0:
        d = ost.dm[r1]
        kind, m0, ms = _range_delay_params(O, cfg, d, last)
        msr = ost.maxshift // 2
        T = min(PARITY_T, ost.t_processed[r1][0])
        W = T + msr
        W += (-W) % 8  # the binning kernel's grid covers whole 16-sample groups
        flat = O.bin_flat(O.corner_turn(host_rows(0, 2 * W), nch, 2 * W), nch, 2 * W)
        dm0 = last_block(r1)
        want = O.dedisperse_window(kind, O.FMA_ALL, flat, W, nch, dm0, 64, 0, T, ost.dmshifts, m0, ms, 2)
        compare(f"chunk 0 range {r1} (binned x2)", want, r1, dm0, 0)
    # last chunk: replay of the runner's flat buffer
    k = ost.num_tchunks - 1
    if k > 0:
        inc = sum(ost.t_processed[0][:k])
        L = ost.t_processed[0][k] + ost.maxshift
        buf = O.corner_turn(host_rows(inc, inc + L), nch, L)
        old = 1
        for r in range(nr):
            d = ost.dm[r]
            msr = ost.maxshift // d[3]
            if d[3] > old:
                nsb = ost.t_processed[r - 1][k] + msr * d[3]
                if nsb > L:
                    # the reference would bin data of an earlier chunk left in its buffer
                    break
                buf = O.bin_flat(buf, nch, nsb)
            old = d[3]
            tp = ost.t_processed[r][k]
            kind, m0, ms = _range_delay_params(O, cfg, d, last)
            dm0 = last_block(r)
            want = O.dedisperse_window(kind, O.FMA_ALL, buf, tp + msr, nch, dm0, 64, 0, tp, ost.dmshifts, m0, ms,
                                       d[3])
            compare(f"chunk {k} range {r}", want, r, dm0, inc // d[3])
    return {"outputs_compared": compared, "mismatching": bad, "checks": checks, "oracle": "oracle/aa_oracle.c",
            "oracle_threads": O.num_threads(), "seconds": time.perf_counter() - t_start}


# ---------------------------------------------------------------------------
REF_SAMPLE_T = 16384  # outputs per DM trial of each timed reference block


def reference_gpu_mid(cfg_mid, repeats=2):
    """The reference's own GPU pipeline (AstroAccelerate built from its
    sources into oracle/_ref/libaaref.so) on the 2^18-sample configuration,
    where its 32-bit kernel indices stay in range (at 2^21 samples its chunks
    pass 2^31 elements and the harness refuses them).  Host [t][c] input,
    DM-time rows copied to the host, the runner's run(status) loop timed by
    the harness after set-up.  Returns a dict, or a dict with "unavailable"."""
    import ctypes
    import numpy as np
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libaaref.so")
    if not os.path.exists(lib_path):
        return {"unavailable": "oracle/_ref/libaaref.so is not built (the reference sources were absent at build)"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no GPU"}
        x, _ = synth_input_device(cfg_mid, cfg_mid["seed"], torch.device("cuda", 0))
        host = x.cpu().numpy().view(np.uint16)
        del x
        torch.cuda.empty_cache()
    except Exception as e:  # noqa: BLE001 - reported in the line
        return {"unavailable": f"input synthesis failed: {e}"}

    class DM(ctypes.Structure):
        _fields_ = [("low", ctypes.c_float), ("high", ctypes.c_float), ("step", ctypes.c_float),
                    ("inBin", ctypes.c_int), ("outBin", ctypes.c_int)]

    L = ctypes.CDLL(lib_path)
    L.aaref_time_ddtr.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_int, ctypes.POINTER(DM), ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    L.aaref_time_ddtr.restype = ctypes.c_int
    plan = (DM * len(cfg_mid["plan"]))()
    for k, (lo, hi, st, ib, ob) in enumerate(cfg_mid["plan"]):
        plan[k].low, plan[k].high, plan[k].step, plan[k].inBin, plan[k].outBin = lo, hi, st, ib, ob
    secs = []
    for _ in range(repeats):
        sec, nt = ctypes.c_double(), ctypes.c_int()
        rc = L.aaref_time_ddtr(host.ctypes.data, cfg_mid["nchans"], cfg_mid["nsamp"], cfg_mid["tsamp"],
                               cfg_mid["fch1"], cfg_mid["foff"], cfg_mid["nbits"], plan, len(cfg_mid["plan"]), 1,
                               ctypes.byref(sec), ctypes.byref(nt))
        if rc != 0:
            return {"unavailable": f"reference pipeline returned {rc}"}
        secs.append(sec.value)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ost = O.strategy(cfg_mid["plan"], cfg_mid["nchans"], cfg_mid["nsamp"], cfg_mid["fch1"], cfg_mid["foff"],
                     cfg_mid["tsamp"], cfg_mid["nbits"])
    units = sum(ost.ndms[r] * ost.total_samps(r) for r in range(len(ost.ndms)))
    sec = min(secs)
    return {"workload": f"{cfg_mid['nchans']} ch x {cfg_mid['nsamp']} samples, {cfg_mid['nbits']}-bit, "
                        f"{len(cfg_mid['plan'])}-range survey plan",
            "value": units / sec, "unit": "DM-trial*samples/s", "ms_per_step": sec * 1e3,
            "realtime_x": ost.total_samps(0) * cfg_mid["tsamp"] / sec, "runs": len(secs),
            "timing": "the reference runner's run(status) loop after set-up, host [t][c] input, rows copied to "
                      "the host (wall clock inside oracle/ref_harness.cu), best of the runs"}


def reference_cpu_step(O, cfg, ost, x_window, step):
    """One timed step of the reference arm: for every range, one 64-trial DM
    block (a different block each step) over REF_SAMPLE_T outputs of a
    corner-turned window of chunk 0, with that range's delay arithmetic and
    row length.  Returns the per-range outputs/s."""
    import numpy as np
    nch = cfg["nchans"]
    rates = []
    for r, d in enumerate(ost.dm):
        kind, m0, ms = _range_delay_params(O, cfg, d, ost.dmshifts[-1])
        T = min(REF_SAMPLE_T, ost.t_processed[r][0])
        nblocks = max(1, ost.ndms[r] // 64)
        dm0 = 64 * ((7 * step + 3 * r) % nblocks)
        t0 = time.perf_counter()
        # the window's row length stands in for the range's (the work per
        # output does not depend on the row length or the sample values)
        O.dedisperse_window(kind, O.FMA_ALL, x_window, x_window.shape[1], nch, dm0, 64, 0, T, ost.dmshifts, m0, ms,
                            d[3])
        rates.append(64 * T / (time.perf_counter() - t0))
    return rates


def run_reference_arm(args, cfg, rank, world):
    """The reference arm: the reference ships no CPU dedispersion, so its CPU
    path is the oracle's restatement of the reference kernels (OpenMP over all
    host threads), timed on a bounded sample of the same workload and
    extrapolated per range to a whole step; plus, on the 2^18-sample
    configuration, the reference's own GPU pipeline built from its sources."""
    import numpy as np
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    ost = O.strategy(cfg["plan"], cfg["nchans"], cfg["nsamp"], cfg["fch1"], cfg["foff"], cfg["tsamp"], cfg["nbits"])
    nch = cfg["nchans"]
    rng = np.random.Generator(np.random.PCG64(cfg["seed"]))
    Wmax = max(min(REF_SAMPLE_T, ost.t_processed[r][0]) + ost.maxshift // ost.dm[r][3] for r in range(len(ost.dm)))
    vmax = (1 << min(cfg["nbits"], 16)) - 1
    xt = np.clip(np.rint(rng.normal((vmax + 1) / 2 - 0.5, (vmax + 1) / 16.0, size=(Wmax, nch))), 0, vmax)
    x_window = O.corner_turn(xt.astype(np.uint16), nch, Wmax).reshape(nch, Wmax)
    units_r = [ost.ndms[r] * ost.total_samps(r) for r in range(len(ost.dm))]
    for w in range(args.warmup):
        reference_cpu_step(O, cfg, ost, x_window, 1000 + w)
    step_s = []
    for k in range(args.steps):
        rates = reference_cpu_step(O, cfg, ost, x_window, k)
        step_s.append(sum(u / v for u, v in zip(units_r, rates)))
    sec = statistics.median(step_s)
    value = sum(units_r) / sec
    desc = (f"oracle (OpenMP restatement of the reference kernels) per step: one 64-trial DM block of each of the "
            f"{len(ost.dm)} ranges over {REF_SAMPLE_T} outputs of chunk 0 ({nch} channels); each range's "
            f"outputs/s scaled to its whole output count, summed to the step time "
            f"{sec:.0f} s (median of {args.steps} steps); corner turn and binning not timed (<2% of the step on "
            f"the GPU)")
    line = {"metric": METRIC, "value": value, "unit": "DM-trial*samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8" if cfg["nbits"] <= 8 else "f32", "data": "synthetic",
            "config": workload_config(cfg), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "DM-trial*samples/s", "cores": O.num_threads(), "kind": "port",
                             "sample": desc},
            "e2e": {"value": value, "unit": "DM-trial*samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_gpu": reference_gpu_mid(MID) if cfg["nsamp"] >= MID["nsamp"] else None}
    print(json.dumps(line), flush=True)
    return 0


def workload_config(cfg):
    full = cfg["nsamp"] == SURVEY["nsamp"] and cfg["nchans"] == SURVEY["nchans"] and cfg["nbits"] == 8
    name = "survey-scale plain DDTR" if full else "reduced plain DDTR"
    return {"workload": f"{name}: {cfg['nchans']} ch x {cfg['nsamp']} samples, {cfg['nbits']}-bit, "
                        f"{len(cfg['plan'])}-range plan to DM {cfg['plan'][-1][1]}",
            "nchans": cfg["nchans"], "nsamp": cfg["nsamp"], "nbits": cfg["nbits"], "tsamp": cfg["tsamp"],
            "plan": [list(p) for p in cfg["plan"]], "l2_policy": "inputs larger than L2 (17 GB per step)",
            "parallelism": "one beam per GPU"}


# ---------------------------------------------------------------------------
MULTIBEAM_FREE_MEMORY = 64 << 30  # memory the beams' strategies are computed for (both arms)


def dev_rows(aa, ptr, shape):
    import torch
    return torch.as_tensor(aa._DeviceRows(ptr, shape), device="cuda")


def measure_multibeam(aa, WL, beams, steps, warmup, device, stream, clk=None):
    """Times a multi-beam draw (a) as batches -- one CUDA graph with one
    persistent dedispersion kernel per batch, batches sized to device memory
    -- and (b) beam by beam through the plain pipeline, both with the input
    resident in HBM and the output kept in HBM, both timed with CUDA events on
    the same stream (median over `steps` runs after `warmup`).  Every beam's
    batched output is compared with its plain output bit for bit."""
    import torch
    mds, plans, sizes, units_b = [], [], [], []
    for b in beams:
        md = aa.filterbank_metadata_struct(0.0, b["tsamp"], b["fch1"], b["foff"], b["nbits"], b["nsamp"],
                                           b["nchans"], 0.0)
        plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in b["plan"]])
        st = aa.strategy(b["plan"], b["nchans"], b["nsamp"], b["fch1"], b["foff"], b["tsamp"], b["nbits"],
                         MULTIBEAM_FREE_MEMORY)
        mds.append(md)
        plans.append(plan)
        units_b.append(units_per_step(st))
        sizes.append(aa.batch_estimate_bytes(md, plan, MULTIBEAM_FREE_MEMORY) + 2 * b["nsamp"] * b["nchans"])
    free, _ = torch.cuda.mem_get_info(device)
    plain_reserve = max(b["nsamp"] * b["nchans"] * 2 * 3 + u * 4 for b, u in zip(beams, units_b))
    budget = int(free * 0.9) - plain_reserve
    waves = WL.plan_waves(sizes, budget)

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tot = dict(batched_ms=0.0, plain_ms=0.0, plain_fresh_s=0.0, setup_s=0.0, units=0, launches=0, items=0)
    bit_exact, mismatches, n_cmp = True, [], 0
    wave_info = []
    for w in waves:
        xs = {i: WL.synth_beam_device(beams[i], device) for i in w}
        torch.cuda.synchronize(device)
        B = aa.batch(free_memory=MULTIBEAM_FREE_MEMORY, stream=stream.cuda_stream)
        t0 = time.perf_counter()
        for i in w:
            B.add_beam(mds[i], plans[i], xs[i])
        B.setup()
        tot["setup_s"] += time.perf_counter() - t0
        for _ in range(max(1, warmup)):
            B.run()
            B.synchronize()
        ms = []
        for _ in range(steps):
            ev0.record(stream)
            B.run()
            ev1.record(stream)
            B.synchronize()
            ms.append(ev0.elapsed_time(ev1))
        info = B.info()
        tot["batched_ms"] += statistics.median(ms)
        tot["launches"] += info["launches_per_run"]
        tot["items"] += info["work_items"]
        wave_info.append({"beams": len(w), "ms": statistics.median(ms), "work_items": info["work_items"],
                          "persistent_jobs": info["persistent_jobs"], "other_jobs": info["other_jobs"],
                          "grid": info["grid"], "smem_bytes": info["smem_bytes"]})
        # plain arm, beam by beam on the same stream
        for j, i in enumerate(w):
            b = beams[i]
            t0 = time.perf_counter()
            pipe = aa.create_pipeline(mds[i], xs[i].data_ptr(), device_input=True, device_output=True,
                                      copy_to_host=False, stream=stream.cuda_stream, card_number=device.index or 0)
            pipe.set_options(free_memory=MULTIBEAM_FREE_MEMORY)
            if not pipe.bind_ddtr_plan(plans[i]) or not (pipe.run_all() and pipe.synchronize()):
                raise RuntimeError(pipe.last_error())
            tot["plain_fresh_s"] += time.perf_counter() - t0
            for _ in range(max(0, warmup - 1)):
                pipe.rewind()
                if not (pipe.run_all() and pipe.synchronize()):
                    raise RuntimeError(pipe.last_error())
            pms = []
            for _ in range(steps):
                pipe.rewind()
                ev0.record(stream)
                if not pipe.run_all():
                    raise RuntimeError(pipe.last_error())
                ev1.record(stream)
                if not pipe.synchronize():
                    raise RuntimeError(pipe.last_error())
                pms.append(ev0.elapsed_time(ev1))
            tot["plain_ms"] += statistics.median(pms)
            for r in range(len(b["plan"])):
                ndms, total, _ = B.range_shape(j, r)
                a = B.output(j, r).view(torch.int32)
                p = dev_rows(aa, pipe.device_output(r), (ndms, total)).view(torch.int32)
                n_cmp += 1
                if not torch.equal(a, p):
                    bit_exact = False
                    mismatches.append([i, r])
            pipe.cleanUp()
            pipe.delete()
            tot["units"] += units_b[i]
        B.delete()
        del xs
        torch.cuda.synchronize(device)
        torch.cuda.empty_cache()
    for p in plans:
        p.delete()
    obs_s = sum(b["nsamp"] * b["tsamp"] for b in beams)
    return {"units": tot["units"], "batched_s": tot["batched_ms"] / 1e3, "plain_s": tot["plain_ms"] / 1e3,
            "obs_s": obs_s, "waves": wave_info, "launches": tot["launches"], "work_items": tot["items"],
            "setup_s": tot["setup_s"], "plain_fresh_s": tot["plain_fresh_s"], "bit_exact": bit_exact,
            "compared_ranges": n_cmp, "mismatches": mismatches[:10],
            "nbits_count": {n: sum(1 for b in beams if b["nbits"] == n) for n in (4, 8, 16)}}


def run_batched(args, rank, world, local):
    """Multi-beam workload: the seeded 48-beam draw (aa_b200.workloads), run
    as batches and beam by beam (measure_multibeam)."""
    import torch
    import torch.distributed as dist
    import aa_b200 as aa
    from aa_b200 import workloads as WL

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    beams = WL.multibeam_draw(seed=3 + 1000 * rank, nbeams=args.beams)
    stream = torch.cuda.Stream(device)
    stream.wait_stream(torch.cuda.current_stream(device))
    with ClockSampler(local) as clk:
        m = measure_multibeam(aa, WL, beams, args.steps, args.warmup, device, stream)
    batched_s, plain_s = m["batched_s"], m["plain_s"]
    if world > 1:
        t = torch.tensor([batched_s, plain_s], device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        batched_s, plain_s = float(t[0]), float(t[1])
    value = m["units"] * world / batched_s
    if rank == 0:
        line = {
            "metric": "DM-trial*samples/s (batched multi-beam DDTR, bit-exact vs plain per-beam launch)",
            "value": value, "unit": "DM-trial*samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(1, args.warmup), "ms_per_step": batched_s * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8+u16", "data": "synthetic",
            "config": {"workload": f"multi-beam DDTR: {len(beams)} beams, 2048-4096 ch, 4/8/16-bit, 2^16-2^21 "
                                   f"samples, 2-6-range prefixes of the survey plan cut at DM 500-3000",
                       "beams": len(beams), "nbits_count": m["nbits_count"], "seed": 3,
                       "strategy_free_memory": MULTIBEAM_FREE_MEMORY, "waves": len(m["waves"]),
                       "l2_policy": "inputs larger than L2", "parallelism": "beams per GPU, batched"},
            "realtime_x": m["obs_s"] / batched_s,
            "plain": {"value": m["units"] * world / plain_s, "ms_per_step": plain_s * 1e3,
                      "realtime_x": m["obs_s"] / plain_s,
                      "fresh_pipeline_s": m["plain_fresh_s"],
                      "note": "beam by beam through the plain pipeline (device input/output), set-up excluded; "
                              "fresh_pipeline_s = wall time of create+bind+first run per beam, summed"},
            "batched_over_plain": plain_s / batched_s,
            "bit_exact": m["bit_exact"], "compared_ranges": m["compared_ranges"], "mismatches": m["mismatches"],
            "batched": {"setup_s": m["setup_s"], "work_items": m["work_items"], "waves": m["waves"]},
            "gpu_launches": m["launches"] * args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0 if m["bit_exact"] else 1


def _search_and_refine(aa, SR, R, x, kc, outputs, strat, k=64, steps=50):
    """Candidates >= 6 sigma of every range, the k strongest events, their
    snippets and refined DMs.  outputs[r] = (rows tensor, nsamp)."""
    cands = []
    for r, (rows, nsamp) in enumerate(outputs):
        d = strat["dm"][r]
        cands.append(SR.candidates(rows, nsamp, d[0], d[2], d[3], threshold=6.0))
    top = SR.select(cands, k=k)
    if top["dm"].numel() == 0:
        return top, None, None
    snip, base = SR.cut_snippets(x, kc, top["dm"], top["t"], top["w"])
    return top, snip, base


def _match_errors(top, dm_ref, pulses, inbin_tol=512):
    """|DM error| before and after refinement for candidates that match an
    injected pulse (arrival within inbin_tol samples)."""
    before, after, found = [], [], set()
    t = top["t"].cpu().numpy()
    d0 = top["dm"].cpu().numpy()
    d1 = dm_ref.cpu().numpy()
    for i in range(len(t)):
        best = None
        for j, p in enumerate(pulses):
            dt = abs(int(t[i]) - p["start"])
            if dt <= inbin_tol + p["width"] and (best is None or dt < best[0]):
                best = (dt, j)
        if best is not None:
            p = pulses[best[1]]
            before.append(abs(float(d0[i]) - p["dm"]))
            after.append(abs(float(d1[i]) - p["dm"]))
            found.add(best[1])
    return before, after, len(found)


def run_e2e(args, rank, world, local):
    """End-to-end search: 16 beams x 4096 channels x 2^20 8-bit samples with
    4-32 injected pulses each; batched DDTR (one graph per batch), 6-sigma
    boxcar candidates, the 64 strongest events per beam cut to 1024-sample
    per-channel snippets, 50 Adam steps on DM through the adjoint kernels.
    The same search runs after the plain per-beam pipeline; wall times
    exclude data generation; set-up (buffers, tables, autotuner: the batch's
    setup(), the plain pipeline's explicit setup()) is reported apart in
    *_with_setup_s; every DDTR output is compared bit for bit."""
    import numpy as np
    import torch
    import aa_b200 as aa
    from aa_b200 import refine as R
    from aa_b200 import search as SR
    from aa_b200 import workloads as WL

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    beams = WL.e2e_beams(seed=5 + 1000 * rank, nbeams=args.beams if args.beams != 48 else 16)
    b0 = beams[0]
    kc = R.delay_per_dm(b0["nchans"], b0["fch1"], b0["foff"], b0["tsamp"])
    mds, plans, strats, sizes = [], [], [], []
    for b in beams:
        md = aa.filterbank_metadata_struct(0.0, b["tsamp"], b["fch1"], b["foff"], 8, b["nsamp"], b["nchans"], 0.0)
        plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in b["plan"]])
        mds.append(md)
        plans.append(plan)
        strats.append(aa.strategy(b["plan"], b["nchans"], b["nsamp"], b["fch1"], b["foff"], b["tsamp"], 8,
                                  MULTIBEAM_FREE_MEMORY))
        sizes.append(aa.batch_estimate_bytes(md, plan, MULTIBEAM_FREE_MEMORY) + 2 * b["nsamp"] * b["nchans"])
    free, _ = torch.cuda.mem_get_info(device)
    reserve = max(sizes) + (64 * 4096 * 1024 * 4) * 6
    waves = WL.plan_waves(sizes, int(free * 0.85) - reserve)
    T = dict(b_ddtr=0.0, b_setup=0.0, b_search=0.0, b_refine=0.0, p_ddtr=0.0, p_setup=0.0, p_search=0.0,
             p_refine=0.0)
    errs_b, errs_p, bit_exact, n_found, n_injected, n_cand = [], [], True, 0, 0, 0
    warmed = False

    def sync_time(t0):
        torch.cuda.synchronize(device)
        return time.perf_counter() - t0

    for w in waves:
        xs = {i: WL.synth_e2e_beam(beams[i], device) for i in w}
        torch.cuda.synchronize(device)
        # ---- batched path
        t0 = time.perf_counter()
        B = aa.batch(free_memory=MULTIBEAM_FREE_MEMORY)
        for i in w:
            B.add_beam(mds[i], plans[i], xs[i])
        B.setup()
        T["b_setup"] += sync_time(t0)
        t0 = time.perf_counter()
        B.run()
        B.synchronize()
        T["b_ddtr"] += sync_time(t0)
        if not warmed:
            # one untimed pass of the search and refinement (first-use set-up
            # of their kernels and of torch's allocator), so that neither arm
            # carries it
            i0 = w[0]
            outs = [(B.output(0, r), B.range_shape(0, r)[1]) for r in range(len(beams[i0]["plan"]))]
            top, snip, base = _search_and_refine(aa, SR, R, xs[i0], kc, outs, strats[i0])
            if snip is not None:
                R.refine_dm(snip, top["dm"], kc, steps=2, lr=0.05, base=base)
            torch.cuda.synchronize(device)
            warmed = True
        t0 = time.perf_counter()
        per_beam = []
        for j, i in enumerate(w):
            outs = [(B.output(j, r), B.range_shape(j, r)[1]) for r in range(len(beams[i]["plan"]))]
            per_beam.append(_search_and_refine(aa, SR, R, xs[i], kc, outs, strats[i]))
        T["b_search"] += sync_time(t0)
        t0 = time.perf_counter()
        snips = [pb for pb in per_beam if pb[1] is not None]
        if snips:
            x_all = torch.cat([s[1] for s in snips])
            base_all = torch.cat([s[2] for s in snips])
            dm0 = torch.cat([s[0]["dm"] for s in snips])
            dm_ref, _ = R.refine_dm(x_all, dm0, kc, steps=50, lr=0.05, base=base_all)
        T["b_refine"] += sync_time(t0)
        off = 0
        for (top, snip, _), i in zip(per_beam, w):
            if snip is None:
                continue
            n = top["dm"].numel()
            bf, af, nf = _match_errors(top, dm_ref[off:off + n], beams[i]["pulses"])
            off += n
            errs_b.append((bf, af))
            n_found += nf
            n_cand += n
            n_injected += len(beams[i]["pulses"])
        # ---- plain path, beam by beam
        for j, i in enumerate(w):
            t0 = time.perf_counter()
            pipe = aa.create_pipeline(mds[i], xs[i].data_ptr(), device_input=True, device_output=True,
                                      copy_to_host=False)
            pipe.set_options(free_memory=MULTIBEAM_FREE_MEMORY)
            if not (pipe.bind_ddtr_plan(plans[i]) and pipe.setup()):
                raise RuntimeError(pipe.last_error())
            T["p_setup"] += sync_time(t0)
            t0 = time.perf_counter()
            if not (pipe.run_all() and pipe.synchronize()):
                raise RuntimeError(pipe.last_error())
            T["p_ddtr"] += sync_time(t0)
            outs = []
            for r in range(len(beams[i]["plan"])):
                ndms, tot, _ = B.range_shape(j, r)
                rows = dev_rows(aa, pipe.device_output(r), (ndms, tot))
                if not torch.equal(rows.view(torch.int32), B.output(j, r).view(torch.int32)):
                    bit_exact = False
                outs.append((rows, tot))
            t0 = time.perf_counter()
            top, snip, base = _search_and_refine(aa, SR, R, xs[i], kc, outs, strats[i])
            T["p_search"] += sync_time(t0)
            t0 = time.perf_counter()
            if snip is not None:
                dm_p, _ = R.refine_dm(snip, top["dm"], kc, steps=50, lr=0.05, base=base)
                bf, af, _ = _match_errors(top, dm_p, beams[i]["pulses"])
                errs_p.append((bf, af))
            T["p_refine"] += sync_time(t0)
            pipe.cleanUp()
            pipe.delete()
        B.delete()
        del xs
        torch.cuda.empty_cache()
    for p in plans:
        p.delete()
    eb = [v for bf, _ in errs_b for v in bf]
    ea = [v for _, af in errs_b for v in af]
    batched_s = T["b_ddtr"] + T["b_search"] + T["b_refine"]
    plain_s = T["p_ddtr"] + T["p_search"] + T["p_refine"]
    line = {"metric": "end-to-end search wall time (batched DDTR + 6-sigma search + top-64 + 50 Adam DM steps)",
            "value": batched_s, "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 0, "higher_is_better": False,
            "dtype": "u8+f32", "data": "synthetic",
            "config": {"workload": f"{len(beams)} beams x 4096 ch x 2^20 8-bit samples, survey plan, 4-32 pulses each",
                       "waves": len(waves)},
            "batched_s": batched_s, "plain_s": plain_s, "plain_over_batched": plain_s / batched_s,
            "batched_with_setup_s": batched_s + T["b_setup"], "plain_with_setup_s": plain_s + T["p_setup"],
            "times": T, "ddtr_bit_exact": bit_exact,
            "candidates": n_cand, "injected": n_injected, "injected_recovered": n_found,
            "dm_error_median": {"before_refinement": float(np.median(eb)) if eb else None,
                                "after_refinement": float(np.median(ea)) if ea else None,
                                "matched_candidates": len(eb)},
            "dm_error_mean": {"before_refinement": float(np.mean(eb)) if eb else None,
                              "after_refinement": float(np.mean(ea)) if ea else None}}
    print(json.dumps(line), flush=True)
    return 0 if bit_exact else 1


def run_refine(args, rank, world, local):
    """Differentiable refinement workload: 256 snippets x 1024 channels x 8192
    samples float32 (N(0,1) + one dispersed Gaussian pulse each), one step =
    smooth peak boxcar S/N forward and its backward to the input and to DM.
    Kernel times by CUDA events; the gradient error against the FP64 host
    oracle and a central difference is measured on two snippets."""
    import numpy as np
    import torch
    from aa_b200 import refine as R
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import frac_oracle as F

    torch.cuda.set_device(local)
    S, C, T = args.snippets, 1024, 8192
    x, dm_true, dm_trial, kc = R.synth_snippets(S, nchans=C, nsamp=T, seed=4 + rank)
    widths = R.DEFAULT_WIDTHS
    mu = torch.zeros(S, device="cuda")
    sigma = torch.full((S,), float(np.sqrt(C)), device="cuda")
    xg = x.clone().requires_grad_(True)

    def step():
        d = dm_trial.clone().requires_grad_(True)
        y = R.FracDedisperse.apply(xg, d, kc)
        p = R.smooth_peak(R.BoxcarSNR.apply(y, widths, mu, sigma))
        p.sum().backward()
        return d.grad

    for _ in range(max(3, args.warmup)):
        step()
        xg.grad = None
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    fwd_ms, adj_ms, step_ms = [], [], []
    for _ in range(args.steps):
        d = dm_trial.clone()
        e[0].record()
        y = R.FracDedisperse.apply(x, d, kc)
        e[1].record()
        gy = torch.ones_like(y)
        gx = torch.empty_like(x)
        gdm = torch.empty_like(d)
        part = torch.empty((S, C), dtype=torch.float64, device="cuda")
        e[2].record()
        R.lib().aa_b200_frac_dedisperse_adj(x.data_ptr(), d.data_ptr(), kc.data_ptr(), None, gy.data_ptr(), S, C, T,
                                            gx.data_ptr(), gdm.data_ptr(), part.data_ptr(), R._stream())
        e[3].record()
        torch.cuda.synchronize()
        fwd_ms.append(e[0].elapsed_time(e[1]))
        adj_ms.append(e[2].elapsed_time(e[3]))
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        step()
        t1.record()
        torch.cuda.synchronize()
        xg.grad = None
        step_ms.append(t0.elapsed_time(t1))
    # gradient error on two snippets against FP64
    errs = []
    xh, kch = x[:2].cpu().numpy(), kc.cpu().numpy()
    d2 = dm_trial[:2].clone().requires_grad_(True)
    p2 = R.peak_snr(x[:2].contiguous(), d2, kc, widths)
    p2.sum().backward()
    for s in range(2):
        _, g64 = F.loss_and_grad_dm(xh[s], float(dm_trial[s]), kch, widths, 0.0, float(np.sqrt(C)), 0.5)
        errs.append(abs(float(d2.grad[s]) - g64) / max(1e-30, abs(g64)))
    bytes_x = S * C * T * 4
    fwd = statistics.median(fwd_ms)
    adj = statistics.median(adj_ms)
    stp = statistics.median(step_ms)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    line = {"metric": "snippets/s (refinement step: forward + adjoint to input and DM)", "value": S / (stp / 1e3),
            "unit": "snippets/s", "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": stp,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"refinement: {S} snippets x 1024 ch x 8192 samples f32, widths 1..64"},
            "kernels": {"frac_fwd_ms": fwd, "frac_adj_ms": adj,
                        "frac_fwd_gbs": bytes_x / fwd / 1e6, "frac_adj_gbs": 2 * bytes_x / adj / 1e6},
            "roofline": {"bound": "hbm", "kernel": "k_frac_fwd", "achieved": bytes_x / fwd / 1e6, "peak": hbm,
                         "unit": "GB/s", "frac": bytes_x / fwd / 1e6 / hbm},
            "grad_rel_err_vs_fp64": errs}
    print(json.dumps(line), flush=True)
    return 0


# 1536 x 2^19: the largest power-of-two plane of 1536 trials whose S/N-plane
# offsets nDMs * output_shift stay below 2^31 in the reference's int arithmetic
# (src/aa_device_SPS_long.cu:69,73; at 2^20 samples its analysis faults)
# analysis settings of the DDTR + analysis measurement (--with-analysis)
ANALYSIS = dict(sigma_cutoff=6.0, sigma_constant=3.0, max_width_s=0.01, algorithm=0, baseline_noise=1)

SPD_WORKLOAD = dict(ndms=1536, nt=1 << 19, tsamp=64e-6, inbin=1, max_width_s=0.0164, sigma_cutoff=6.0,
                    sigma_constant=3.0, baseline_noise=1, algorithm=0, npulses=16, seed=31)


def synth_plane_device(w, seed, device):
    """A DM-time plane [ndms][nt] float32 on the device: N(0, 1) noise plus
    dispersed-looking pulses (a Gaussian in time whose amplitude falls off
    and width grows with the distance from the pulse's DM trial)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    nd, nt = w["ndms"], w["nt"]
    x = torch.randn((nd, nt), generator=g, device=device, dtype=torch.float32)
    rng = torch.Generator()
    rng.manual_seed(seed)
    for _ in range(w["npulses"]):
        d0 = int(torch.randint(8, nd - 8, (1,), generator=rng))
        t0 = int(torch.randint(4096, nt - 4096, (1,), generator=rng))
        wid = float(torch.empty(1).uniform_(1.0, 64.0, generator=rng))
        amp = float(torch.empty(1).uniform_(0.5, 3.0, generator=rng))
        lo, hi = max(0, d0 - 24), min(nd, d0 + 25)
        dd = torch.arange(lo, hi, device=device, dtype=torch.float32)[:, None] - d0
        tt = torch.arange(t0 - 2048, t0 + 2048, device=device, dtype=torch.float32)[None, :] - t0
        ww = wid + 3.0 * dd.abs()
        a = amp * torch.exp(-0.5 * (dd / 6.0) ** 2) * torch.sqrt(wid / ww)
        x[lo:hi, t0 - 2048:t0 + 2048] += a * torch.exp(-0.5 * (tt / ww) ** 2)
    return x


def spd_snr_plane_bytes(aa, w):
    """Algorithmic bytes of the boxcar S/N planes, per iteration: the input
    and the running boxcar values read once (the first iteration has no
    running values), the S/N (float) and width (ushort) planes written, and
    the half-resolution sums and boxcar values written.  Returns (bytes of
    the first plane, bytes of the later planes, plan)."""
    tsamp = float(__import__("numpy").float32(w["tsamp"] * w["inbin"]))
    pl = aa.spd_plan(w["nt"], tsamp, w["inbin"], w["max_width_s"])
    first = later = 0
    for f in range(pl["max_iteration"]):
        dts, dtm, nblocks = pl["plan"][f][0], pl["plan"][f][1], pl["plan"][f][4]
        if nblocks <= 0:
            continue
        per_row = dts * 4 + (0 if f == 0 else dts * 4) + dts * (4 + 2) + dtm * 4 * 2
        if f == 0:
            first = per_row * w["ndms"]
        else:
            later += per_row * w["ndms"]
    return first, later, pl


def _ref_lib():
    """oracle/_ref/libaaref.so (the reference built from its sources), or None."""
    import ctypes
    path = os.path.join(ROOT, "oracle", "_ref", "libaaref.so")
    return ctypes.CDLL(path) if os.path.exists(path) else None


def reference_gpu_spd(plane, w, reps=3):
    """The reference's analysis_GPU (aaref_time_spd: its buffers allocated as
    its runner does, CUDA events around the call, the plane restored from a
    device copy before each run) on the same device plane.  Returns
    {"ms": [...], "candidates": n} or {"unavailable": why}."""
    import ctypes
    import numpy as np
    L = _ref_lib()
    if L is None:
        return {"unavailable": "oracle/_ref/libaaref.so is not built (the reference sources were absent at build)"}
    L.aaref_time_spd.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                 ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                 ctypes.c_longlong, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]
    L.aaref_time_spd.restype = ctypes.c_int
    ms = np.zeros(reps, np.float32)
    nc = ctypes.c_longlong()
    tsamp = float(np.float32(w["tsamp"] * w["inbin"]))
    rc = L.aaref_time_spd(plane.data_ptr(), w["ndms"], w["nt"], tsamp, w["inbin"], w["max_width_s"],
                          w["sigma_constant"], int(w["baseline_noise"]), w["sigma_cutoff"], w["algorithm"], 0, reps,
                          ms.ctypes.data, ctypes.byref(nc))
    if rc != 0:
        return {"unavailable": f"reference analysis returned {rc}"}
    return {"ms": [float(v) for v in ms], "candidates": int(nc.value)}


def reference_gpu_whitening(spec, nbins, ndms, reps=3):
    """The reference's whitening kernels (aaref_time_psr_whitening: its
    median and SGP2 kernels as spectrum_whitening_SGP2 launches them, CUDA
    events, the spectra restored from a device copy before each run) on the
    same device spectra.  Returns {"ms": [...]} or {"unavailable": why}."""
    import ctypes
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import psr_oracle as PO
    seg = PO.segment_sizes(nbins)
    if seg[-1] - seg[-2] < 3:
        # its median kernel reads past its shared array for segments of 1 or 2 bins
        return {"unavailable": "last whitening segment shorter than 3 bins"}
    L = _ref_lib()
    if L is None:
        return {"unavailable": "oracle/_ref/libaaref.so is not built (the reference sources were absent at build)"}
    L.aaref_time_psr_whitening.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_void_p]
    L.aaref_time_psr_whitening.restype = ctypes.c_int
    ms = np.zeros(reps, np.float32)
    rc = L.aaref_time_psr_whitening(spec.data_ptr(), nbins, ndms, reps, ms.ctypes.data)
    if rc != 0:
        return {"unavailable": f"reference whitening returned {rc}"}
    return {"ms": [float(v) for v in ms]}


def reference_gpu_line(args, world, metric, unit, units, config, ref, what):
    """The reference arm's line for a component the reference runs only on
    the GPU: its own kernels timed on the same device-resident workload."""
    if "unavailable" in ref:
        return {"impl": "reference", "metric": metric, "unavailable": ref["unavailable"]}
    ms = statistics.median(ref["ms"])
    value = units / (ms / 1e3)
    return {"metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": len(ref["ms"]),
            "warmup": 0, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": config, "impl": "reference",
            "cpu_baseline": {"value": value, "unit": unit, "cores": 0, "kind": "reference", "device": "gpu",
                             "sample": f"{what}, the whole workload, device-resident, CUDA events, median of "
                                       f"{len(ref['ms'])} runs (the reference has no CPU path for it)"},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


SPD_METRIC = "DM-trial*samples/s analysed (single-pulse detection, reference rules, bit-exact)"


def spd_config(w):
    n = w["ndms"] * w["nt"]
    return {"workload": f"single-pulse detection: {w['ndms']} DM trials x {w['nt']} samples f32 "
                        f"({n * 4 / 1e9:.1f} GB), boxcar widths to {int(w['max_width_s'] / w['tsamp'])} samples, "
                        f"MSD with outlier rejection, peak finding at {w['sigma_cutoff']:g} sigma",
            "l2": "inputs larger than L2"}


def run_spd(args, rank, world, local):
    """Single-pulse detection (the reference's analysis_GPU rules, bit-exact)
    on one DM-time plane of 1536 DM trials x 2^19 samples float32 (3.2 GB,
    far above L2), resident in HBM: one step = MSD profile with outlier
    rejection, boxcar S/N planes up to 256 samples and peak finding.  The
    plane is restored from a pristine copy before each step (the search
    decimates into it) outside the timed region.  e2e: the same through the
    C ABI from a pinned host plane (H2D inside the timed region) to the host
    candidate lists."""
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    w = dict(SPD_WORKLOAD, nt=args.spd_nt) if args.spd_nt else SPD_WORKLOAD
    n = w["ndms"] * w["nt"]
    pristine = synth_plane_device(w, w["seed"] + rank, device)
    if args.impl == "reference":
        if rank == 0:
            ref = reference_gpu_spd(pristine, w, max(3, args.steps))
            print(json.dumps(reference_gpu_line(args, world, SPD_METRIC, "DM-trial*samples/s", n, spd_config(w), ref,
                                                "the reference's analysis_GPU")), flush=True)
        return 0
    import aa_b200 as aa
    plane = torch.empty_like(pristine)
    spd = aa.single_pulse_detection(n, 0)
    tsamp = float(np.float32(w["tsamp"] * w["inbin"]))
    kw = dict(candidate_algorithm=w["algorithm"], enable_msd_baseline_noise=bool(w["baseline_noise"]))

    def one():
        return spd.run(plane, w["ndms"], w["nt"], tsamp, w["inbin"], w["sigma_cutoff"], w["sigma_constant"],
                       w["max_width_s"], **kw)

    for _ in range(max(3, args.warmup)):
        plane.copy_(pristine)
        one()
    torch.cuda.synchronize()
    launches0 = aa.spd_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    ncand = 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            plane.copy_(pristine)
            torch.cuda.synchronize()
            e0.record()
            r = one()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
            ncand = int(r["dm"].size)
    launches = (aa.spd_kernel_launches() - launches0) // max(1, args.steps)
    # per-family device time on one more step
    spd.time_kernels(True)
    plane.copy_(pristine)
    one()
    fam = spd.family_times()
    spd.time_kernels(False)
    step_ms = statistics.median(ms)
    # e2e: pinned host plane -> device -> analysis -> host candidates
    host = torch.empty((w["ndms"], w["nt"]), dtype=torch.float32, pin_memory=True)
    host.copy_(pristine)
    e2e_ms = []
    for _ in range(max(1, args.e2e_steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plane.copy_(host, non_blocking=True)
        r = one()
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e = statistics.median(e2e_ms)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    first_bytes, later_bytes, pl = spd_snr_plane_bytes(aa, w)
    first_ms = fam["snr_first"][0]
    achieved = first_bytes / (first_ms / 1e3) / 1e9 if first_ms > 0 else None
    # DRAM bytes of one first-plane k_boxcar_snr launch, from an ncu capture
    # of the 1536 x 65536 plane (0.4065 GB read + 0.9511 GB written) scaled
    # by the samples a launch covers
    traffic = 1.3576e9 * (n / (1536 * 65536))
    ref = reference_gpu_spd(pristine, w) if rank == 0 else None
    line = {"metric": SPD_METRIC,
            "value": n / (step_ms / 1e3), "unit": "DM-trial*samples/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": spd_config(w),
            "boxcar_plan": {"max_width_performed": pl["max_width_performed"], "iterations": pl["max_iteration"]},
            "candidates": ncand, "gpu_launches": int(launches),
            "reference_gpu": (dict(ref, ms_per_step=statistics.median(ref["ms"]),
                                   value=n / (statistics.median(ref["ms"]) / 1e3))
                              if ref and "ms" in ref else ref),
            "families_ms": {k: v[0] for k, v in fam.items()},
            "families_launches": {k: v[1] for k, v in fam.items()},
            "roofline": {"bound": "issue", "kernel": "k_boxcar_snr<32> (first boxcar S/N plane)", "achieved": achieved,
                         "peak": hbm, "unit": "GB/s", "frac": (achieved / hbm) if achieved else None,
                         "traffic": traffic, "algorithmic_bytes": first_bytes,
                         "note": "frac is of the measured HBM copy rate, which does not bind: the kernel is "
                                 "issue-bound, 32 fast divisions, compares and selects per sample"},
            "later_snr_planes_gbs": (later_bytes / (fam["snr_later"][0] / 1e3) / 1e9
                                     if fam["snr_later"][0] > 0 else None),
            "e2e": {"value": n / (e2e / 1e3), "unit": "DM-trial*samples/s", "h2d_bytes_per_step": n * 4,
                    "d2h_bytes_per_step": ncand * 16},
            "clocks": clk.summary()}
    spd.delete()
    print(json.dumps(line), flush=True)
    return 0


PERIODICITY_METRIC = "DM-trial*FFT-points/s searched (periodicity component, reference rules)"


def run_periodicity(args, rank, world, local):
    """The periodicity component after dedispersion, through the
    reference-facing C ABI: the 4096-channel x 2^18-sample 8-bit input with
    the 8-range survey plan (the reference runner's GPU size), every DM
    trial searched with a 2^17-point FFT (the processed length rounded down
    to a power of two, halved per binning): whitening, power and interbin
    spectra, MSD profile, greedy harmonic sums of 32 harmonics with
    scalloping-loss mitigation, peak finding at 10 sigma.  One step = one
    whole pipeline run (dedispersion with the rows kept on the device, then
    the periodicity search); `value` is the search's device time (CUDA
    events around each batch's stages, after its input copy), `e2e` the
    wall time of the run() call that performs the search."""
    import numpy as np
    import torch
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "metric": PERIODICITY_METRIC,
                              "unavailable": "the reference's periodicity search is not run here: its whitening "
                                             "reads one boundary and one median past its tables on every call, "
                                             "and a run of it in a shared process was followed by an illegal "
                                             "memory access"}), flush=True)
        return 0
    import aa_b200 as aa
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    cfg = MID
    x, _ = synth_input_device(cfg, cfg["seed"] + rank, device)
    host = x.cpu().numpy().view(np.uint16).reshape(-1)
    del x
    torch.cuda.empty_cache()
    md = aa.filterbank_metadata_struct(0.0, cfg["tsamp"], cfg["fch1"], cfg["foff"], cfg["nbits"], cfg["nsamp"],
                                       cfg["nchans"], 0.0)

    def one():
        comps = aa.aa_py_pipeline_components(True, False, True, False)
        o = aa.aa_py_pipeline_component_options()
        o.copy_ddtr_data_to_host = True
        pipe = aa.aa_py_pipeline(comps, o, md, host, local)
        pipe.set_device_output(True)
        plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*q) for q in cfg["plan"]])
        if not pipe.bind_ddtr_plan(plan) or not pipe.bind_periodicity_plan_full(10.0, True, 3.0, 32, 1, 0, True):
            raise RuntimeError(pipe.last_error())
        wall = None
        while True:
            comp_done = pipe.status_code() == aa.STATUS_FINISHED_COMPONENT
            t0 = time.perf_counter()
            more = pipe.run()
            dt = time.perf_counter() - t0
            if pipe.status_code() == aa.STATUS_ERROR:
                raise RuntimeError(pipe.last_error())
            if comp_done and pipe.status_code() == aa.STATUS_FINISHED_COMPONENT:
                wall = dt  # the call after dedispersion's finished_component runs the search
            if not more:
                break
        info = pipe.psr_info()
        n = (pipe.get_psr_candidates(False).shape[0], pipe.get_psr_candidates(True).shape[0])
        pipe.cleanUp()
        pipe.delete()
        plan.delete()
        return info, wall, n

    for _ in range(max(1, args.warmup)):
        one()
    launches0 = aa.lib().aa_b200_psr_kernel_launches() + aa.spd_kernel_launches()
    ms, walls = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            info, wall, ncand = one()
            ms.append(info["compute_ms"])
            walls.append(wall)
    # this library's periodicity and MSD kernels (cuFFT's own not counted)
    launches = (aa.lib().aa_b200_psr_kernel_launches() + aa.spd_kernel_launches() - launches0) // max(1, args.steps)
    strat = aa.strategy(cfg["plan"], cfg["nchans"], cfg["nsamp"], cfg["fch1"], cfg["foff"], cfg["tsamp"], cfg["nbits"])
    points = sum(strat["ndms"][r] * (info["fft_length"] // cfg["plan"][r][3]) for r in range(len(cfg["plan"])))
    step_ms = statistics.median(ms)
    wall_s = statistics.median(walls)
    line = {"metric": PERIODICITY_METRIC, "value": points / (step_ms / 1e3), "unit": "DM-trial*FFT-points/s",
            "n_gpus": 1, "steps": args.steps, "warmup": max(1, args.warmup), "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"periodicity search of the {cfg['nchans']} ch x {cfg['nsamp']} samples 8-bit "
                                   f"run, 8-range survey plan: {sum(strat['ndms'])} DM trials, FFT length "
                                   f"{info['fft_length']} (halved per binning), greedy harmonic sum of 32, "
                                   f"peak finding at 10 sigma, {info['batches']} batches",
                       "l2": "inputs larger than L2"},
            "candidates": {"power": ncand[0], "interbin": ncand[1]}, "gpu_launches": int(launches),
            "e2e": {"value": points / wall_s, "unit": "DM-trial*FFT-points/s", "wall_s": wall_s,
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 16 * (ncand[0] + ncand[1]),
                    "note": "the run() call that performs the search: rows read on the device, candidates copied "
                            "to the host"},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


WHITENING_WORKLOAD = dict(ndms=512, nbins=(1 << 20) // 2 + 1, seed=41)
WHITENING_METRIC = "spectrum bins/s whitened (periodicity spectral whitening, reference rules)"


def whitening_config(w):
    bins = w["ndms"] * w["nbins"]
    return {"workload": f"spectral whitening: {w['ndms']} spectra x {w['nbins']} complex bins f32 "
                        f"({bins * 8 / 1e9:.1f} GB), segment medians and SGP2 normalisation",
            "l2": "inputs larger than L2"}


def run_whitening(args, rank, world, local):
    """Spectral whitening of the periodicity search (the reference's
    spectrum_whitening_SGP2 with medians, bit-exact outside its raced bins)
    on 512 spectra of 2^19 + 1 complex bins (the spectra of 2^20-sample
    series, 2.1 GB, above L2), resident in HBM: one step = segment medians
    and the interpolated normalisation, in place; the spectra are restored
    from a pristine copy outside the timed region.  Algorithmic bytes: 8 per
    bin read by the median kernel, 8 read and 8 written by the
    normalisation.  e2e: pinned host spectra in, whitened spectra out,
    through aa_b200_psr_whitening."""
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    w = WHITENING_WORKLOAD
    nb, nd = w["nbins"], w["ndms"]
    bins = nd * nb
    g = torch.Generator(device=device)
    g.manual_seed(w["seed"] + rank)
    k = torch.arange(nb, device=device, dtype=torch.float32)
    amp = torch.sqrt(nb * (1.0 + 300.0 / (1.0 + k / 20.0) ** 2) / 2.0)
    pristine = (torch.randn((nd, nb, 2), device=device, generator=g) * amp[None, :, None]).contiguous()
    if args.impl == "reference":
        if rank == 0:
            ref = reference_gpu_whitening(pristine, nb, nd, max(3, args.steps))
            print(json.dumps(reference_gpu_line(args, world, WHITENING_METRIC, "bins/s", bins, whitening_config(w),
                                                ref, "the reference's segmented-median and SGP2 kernels")),
                  flush=True)
        return 0
    import aa_b200 as aa
    spec = torch.empty_like(pristine)
    L = aa.lib()
    stream = torch.cuda.current_stream(device).cuda_stream

    def one():
        if L.aa_b200_psr_whitening(spec.data_ptr(), nb, nd, stream) != 0:
            raise RuntimeError(L.aa_b200_psr_last_error().decode())

    for _ in range(max(3, args.warmup)):
        spec.copy_(pristine)
        one()
    torch.cuda.synchronize()
    launches0 = L.aa_b200_psr_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            spec.copy_(pristine)
            torch.cuda.synchronize()
            e0.record()
            one()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
    launches = (L.aa_b200_psr_kernel_launches() - launches0) // max(1, args.steps)
    step_ms = statistics.median(ms)
    host = torch.empty_like(pristine, device="cpu").pin_memory()
    host.copy_(pristine)
    out = torch.empty_like(host).pin_memory()
    e2e_ms = []
    for _ in range(max(1, args.e2e_steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        spec.copy_(host, non_blocking=True)
        one()
        out.copy_(spec, non_blocking=True)
        torch.cuda.synchronize()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e = statistics.median(e2e_ms)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    achieved = 24.0 * bins / (step_ms / 1e3) / 1e9
    cpu = None
    if rank == 0:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import psr_oracle as O
        sample = pristine[0].cpu().numpy().astype(np.float32)
        z = (sample[:, 0] + 1j * sample[:, 1]).astype(np.complex64)[None, :]
        t0 = time.perf_counter()
        O.whitening(z)
        dt = time.perf_counter() - t0
        cpu = {"value": z.size / dt, "unit": "bins/s", "cores": 1, "kind": "port",
               "sample": f"oracle on 1 spectrum of {z.size} bins, {dt:.1f} s"}
    ref = reference_gpu_whitening(pristine, nb, nd) if rank == 0 else None
    line = {"metric": WHITENING_METRIC,
            "value": bins / (step_ms / 1e3), "unit": "bins/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": whitening_config(w),
            "gpu_launches": int(launches),
            "reference_gpu": (dict(ref, ms_per_step=statistics.median(ref["ms"]),
                                   value=bins / (statistics.median(ref["ms"]) / 1e3))
                              if ref and "ms" in ref else ref),
            "roofline": {"bound": "latency", "kernel": "k_segment_medians_warp + k_sgp2_spans",
                         "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": None,
                         "algorithmic_bytes": 24 * bins,
                         "note": "frac is of the measured HBM copy rate, which does not bind: one warp sorts one "
                                 "segment of at most 79 bins in a 128-slot shuffle network (28 compare-exchange "
                                 "stages per segment), and one warp scales one interpolation span"},
            "e2e": {"value": bins / (e2e / 1e3), "unit": "bins/s", "h2d_bytes_per_step": bins * 8,
                    "d2h_bytes_per_step": bins * 8},
            "cpu_baseline": cpu, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference" and args.config not in ("survey", "mid", "small", "spd", "whitening", "periodicity"):
        # the plain DDTR configurations and the two GPU-only components have
        # a reference arm; print no line that would stand for one
        if rank == 0:
            print(json.dumps({"impl": "reference", "config": args.config,
                              "unavailable": f"no reference arm for --config {args.config}: the reference arm times "
                                             "the plain DDTR path (survey, mid, small), single-pulse detection "
                                             "(spd) and spectral whitening"}), flush=True)
        return 0
    if args.config == "batched" and args.impl != "reference":
        return run_batched(args, rank, world, local)
    if args.config == "refine" and args.impl != "reference":
        return run_refine(args, rank, world, local)
    if args.config == "e2e" and args.impl != "reference":
        return run_e2e(args, rank, world, local)
    if args.config == "spd":
        return run_spd(args, rank, world, local)
    if args.config == "whitening":
        return run_whitening(args, rank, world, local)
    if args.config == "periodicity":
        return run_periodicity(args, rank, world, local)
    cfg = {"survey": SURVEY, "mid": MID, "small": SMALL, "batched": SURVEY, "refine": SURVEY,
           "e2e": SURVEY, "spd": SURVEY, "whitening": SURVEY}[args.config]
    if args.nbits:
        cfg = dict(cfg, nbits=args.nbits)
    if args.impl == "reference":
        return run_reference_arm(args, cfg, rank, world)

    import numpy as np
    import torch
    import torch.distributed as dist
    import aa_b200 as aa

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()

    x, pulses = synth_input_device(cfg, cfg["seed"] + rank, device)
    # a stream of its own: the library launches on it and the CUDA events below
    # are recorded on it (the legacy default stream would not order them)
    stream = torch.cuda.Stream(device)
    stream.wait_stream(torch.cuda.current_stream(device))
    md = metadata_struct(aa, cfg)

    # ---------------- measured shared-memory roof of this GPU ----------------
    smem = aa.smem_load_rate(8192, stream.cuda_stream)

    # ---------------- device-resident value ----------------
    if args.tune_file and os.path.exists(args.tune_file):
        aa.load_tuned_ranges(args.tune_file)
    pipe = aa.create_pipeline(md, x.data_ptr(), device_input=True, device_output=True, copy_to_host=False,
                              stream=stream.cuda_stream, card_number=local)
    pipe.set_options(tile_words=args.tile_words, group_dms=args.group_dms)
    pipe.set_kernel_variant(args.variant)
    if args.no_autotune:
        pipe.set_autotune(False)
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in cfg["plan"]])
    if not pipe.bind_ddtr_plan(plan):
        raise RuntimeError(pipe.last_error())
    strat = aa.strategy(cfg["plan"], cfg["nchans"], cfg["nsamp"], cfg["fch1"], cfg["foff"], cfg["tsamp"],
                        cfg["nbits"])
    units = units_per_step(strat)
    for _ in range(args.warmup):
        if not (pipe.run_all() and pipe.synchronize() and pipe.rewind()):
            raise RuntimeError(pipe.last_error())
    if args.tune_file and rank == 0:
        aa.save_tuned_ranges(args.tune_file)
    pipe.time_kernels(True)
    pipe.reset_kernel_times()
    launches0 = aa.lib().aa_b200_pipeline_kernel_launches(pipe.m_obj)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize(device)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            if not (pipe.run_all() and pipe.rewind()):
                raise RuntimeError(pipe.last_error())
        ev1.record(stream)
        torch.cuda.synchronize(device)
    if not pipe.synchronize():
        raise RuntimeError(pipe.last_error())
    barrier()
    ms_total = ev0.elapsed_time(ev1)
    launches = aa.lib().aa_b200_pipeline_kernel_launches(pipe.m_obj) - launches0
    kern = {name: pipe.kernel_time(f) for f, name in enumerate(["dedisperse", "corner_turn", "bin"])}
    ranges = [pipe.range_info(r) for r in range(len(cfg["plan"]))]
    ms_step = ms_total / args.steps
    if world > 1:
        t = torch.tensor([ms_step], device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_step = float(t.item())
    value = units * world / (ms_step / 1e3)

    # ---------------- parity of the timed output (the oracle as checker) ----------------
    parity = None
    if rank == 0 and not args.no_parity:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        ost = O.strategy(cfg["plan"], cfg["nchans"], cfg["nsamp"], cfg["fch1"], cfg["foff"], cfg["tsamp"],
                         cfg["nbits"])
        same_strategy = (ost.ndms == list(strat["ndms"]) and ost.maxshift == strat["maxshift"] and
                         ost.t_processed == [list(v) for v in strat["t_processed"]])

        def host_rows(a, b):
            return x[a:b].cpu().numpy().view(np.uint16)

        def device_rows(r, dm0, ndm, col0, ncol):
            nd, tot = strat["ndms"][r], sum(strat["t_processed"][r])
            rows = dev_rows(aa, pipe.device_output(r), (nd, tot))
            return rows[dm0:dm0 + ndm, col0:col0 + ncol].cpu().numpy()

        parity = parity_checks(cfg, ost, host_rows, device_rows)
        parity["strategy_identical_to_oracle"] = same_strategy
    pipe.cleanUp()
    pipe.delete()

    # ---------------- e2e through the reference-facing C ABI ----------------
    e2e = None
    if not args.no_e2e:
        xh = torch.empty(x.shape, dtype=torch.int16, pin_memory=True)
        xh.copy_(x)
        del x
        torch.cuda.empty_cache()
        e2e = measure_e2e(aa, cfg, md, plan, xh, strat, units, args.e2e_steps, local, device, barrier, world)
        x_host = xh.numpy().view(np.uint16)
        if args.with_analysis:
            e2e["with_analysis"] = measure_e2e_analysis(aa, md, plan, xh, units, args.e2e_steps, local, device, world)
        # the same run fed the samples as a SIGPROC file stores them
        # (aa_b200_pipeline_set_packed_input): nbits/16 of the H2D bytes
        if cfg["nbits"] <= 8:
            e2e["packed_input"] = measure_e2e_packed(aa, cfg, md, plan, xh, x_host, strat, units, args.e2e_steps,
                                                     local, device, barrier, world)
        del xh
    else:
        x_host = x[:min(131040, strat["t_processed"][0][0]) + strat["maxshift"]].cpu().numpy().view(np.uint16)
        del x
    plan.delete()
    torch.cuda.empty_cache()

    # ---------------- the 2^18-sample configuration end to end ----------------
    # (the size at which the reference's own GPU pipeline runs; its arm
    # reports reference_gpu on the same input)
    mid_e2e = None
    if rank == 0 and cfg is SURVEY and not args.no_e2e:
        mid_e2e = measure_mid_e2e(aa, local, device, args.e2e_steps)

    # ---------------- batched vs plain on a reduced multi-beam draw ----------------
    multibeam = None
    if args.multibeam_beams > 0 and cfg is SURVEY:
        from aa_b200 import workloads as WL
        beams = WL.multibeam_draw(seed=3 + 1000 * rank, nbeams=48)[:args.multibeam_beams]
        m = measure_multibeam(aa, WL, beams, 2, 1, device, stream)
        bs, ps = m["batched_s"], m["plain_s"]
        if world > 1:
            t = torch.tensor([bs, ps], device=device)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            bs, ps = float(t[0]), float(t[1])
        multibeam = {
            "workload": f"the first {len(beams)} beams of the seeded 48-beam multi-beam draw (seed 3): "
                        f"2048-4096 ch, 4/8/16-bit ({m['nbits_count']}), 2^16-2^21 samples, 2-6-range prefixes of "
                        f"the survey plan; input and output resident in HBM",
            "batched": {"value": m["units"] * world / bs, "ms_per_step": bs * 1e3, "realtime_x": m["obs_s"] / bs},
            "plain": {"value": m["units"] * world / ps, "ms_per_step": ps * 1e3, "realtime_x": m["obs_s"] / ps},
            "batched_over_plain": ps / bs, "bit_exact": m["bit_exact"], "compared_ranges": m["compared_ranges"],
            "mismatches": m["mismatches"], "waves": len(m["waves"]), "steps": 2, "warmup": 1,
            "timing": "CUDA events on one stream, median of 2 runs per arm after 1 warm-up"}

    # ---------------- roofline of the dominant kernel ----------------
    dd_ms, dd_n = kern["dedisperse"]
    nch = cfg["nchans"]
    kernel_names = {"quad": "k_ddtr_quad", "phase": "k_ddtr_u8", "f32": "k_ddtr_f32", "gather": "k_ddtr_u16",
                    "sub": "k_ddtr_sub", "quadws": "k_ddtr_quadws", "quadsp": "k_ddtr_quadsp"}
    alg_bytes = alg_adds = traffic = 0
    traffic_known = True
    for r in range(len(cfg["plan"])):
        ratio = TRAFFIC_PER_ALG_BYTE.get(kernel_names[ranges[r]["kernel"]])
        traffic_known = traffic_known and ratio is not None
        for k in range(strat["num_tchunks"]):
            tp = strat["t_processed"][r][k]
            ms_r = strat["maxshift"] // cfg["plan"][r][3]
            b = nch * (tp + ms_r) * (1 if cfg["nbits"] <= 8 else 2) + strat["ndms"][r] * tp * 4
            alg_bytes += b
            traffic += (ratio or 0.0) * b
            alg_adds += strat["ndms"][r] * tp * nch
    launches_per_step = len(cfg["plan"]) * strat["num_tchunks"]
    dd_s_per_step = dd_ms / 1e3 / (dd_n / launches_per_step)
    adds_rate = alg_adds / dd_s_per_step
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    used = sorted({kernel_names[ri["kernel"]] for ri in ranges})
    hbm_achieved = alg_bytes / dd_s_per_step / 1e9
    roofline = {
        "bound": "shared-memory", "kernel": "+".join(used), "unit": "adds/s",
        "achieved": adds_rate, "peak": smem["adds_per_s"], "frac": adds_rate / smem["adds_per_s"],
        "traffic": traffic / launches_per_step if traffic_known else None,
        "algorithmic": {"adds_per_launch": alg_adds / launches_per_step,
                        "bytes_per_launch": alg_bytes / launches_per_step,
                        "per_unit": f"{nch} channel adds and, per step, the packed input once per (chunk, range) "
                                    f"plus 4 B per output"},
        "peak_source": f"measured on this GPU by aa_b200_smem_load_rate: {smem['loads_per_s']:.4g} 32-bit shared "
                       f"loads/s x 4 adds per load (the bound of the direct channel-quad sum; the subband kernel "
                       f"loads less per add and is issue-bound)",
        "traffic_source": TRAFFIC_SOURCE,
        "hbm": {"achieved": hbm_achieved, "peak": hbm, "unit": "GB/s", "frac": hbm_achieved / hbm,
                "peak_source": "MEASURED_PEAKS.json (measured)" if "hbm_gbs" in peaks else "fallback"},
    }

    result = None
    if rank == 0:
        cb_value, cb_threads, cb_desc = cpu_baseline(cfg, x_host, args.cpu_seconds) if world == 1 else (
            None, None, None)
        result = {
            "metric": METRIC if parity is not None else METRIC_UNCHECKED, "value": value,
            "unit": "DM-trial*samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8" if cfg["nbits"] <= 8 else "f32", "data": "synthetic",
            "config": workload_config(cfg),
            "realtime_x": sum(strat["t_processed"][0]) * cfg["tsamp"] / (ms_step / 1e3),
            "published_realtime_x": PUBLISHED_REALTIME,
            "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "parity": parity,
            "batched_vs_plain": multibeam, "mid_e2e": mid_e2e,
            "kernels_ms_per_step": {k: v[0] / args.steps for k, v in kern.items()},
            "kernel_share_of_step": dd_ms / max(1e-9, ms_total),
            "kernel_launches_per_step": {k: v[1] / args.steps for k, v in kern.items()},
            "ranges": ranges, "pulses": len(pulses), "clocks": clk.summary(),
            "cpu_baseline": None if cb_value is None else {"value": cb_value, "unit": "DM-trial*samples/s",
                                                            "cores": cb_threads, "kind": "port", "sample": cb_desc},
        }
        print(json.dumps(result), flush=True)
    if world > 1:
        dist.destroy_process_group()
    ok = parity is None or parity["mismatching"] == 0
    return 0 if ok else 1


def measure_e2e(aa, cfg, md, plan, xh, strat, units, e2e_steps, local, device, barrier, world):
    """The metric through aa_py_pipeline_api / run loop from the pinned host
    [t][c] input to the pinned host float*** rows (copies inside the timed
    region; wall clock between device synchronisations; the first run, which
    also allocates, is not counted)."""
    import torch
    import torch.distributed as dist
    comps = aa.aa_py_pipeline_components(True, False, False, False)
    opts = aa.aa_py_pipeline_component_options()
    opts.copy_ddtr_data_to_host = True
    api = aa.aa_py_pipeline(comps, opts, md, ctypes_ushort_ptr(xh), local)
    if not api.bind_ddtr_plan(plan):
        raise RuntimeError(api.last_error())
    walls = []
    for step in range(1 + e2e_steps):
        torch.cuda.synchronize(device)
        barrier()
        t0 = time.perf_counter()
        api.rewind()
        while api.run():
            pass
        if api.status_code() == aa.STATUS_ERROR:
            raise RuntimeError(api.last_error())
        torch.cuda.synchronize(device)
        walls.append(time.perf_counter() - t0)
    wall = statistics.median(walls[1:])
    if world > 1:
        t = torch.tensor([wall], device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        wall = float(t.item())
    h2d = sum((strat["t_processed"][0][k] + strat["maxshift"]) * cfg["nchans"] * 2
              for k in range(strat["num_tchunks"]))
    api.cleanUp()
    api.delete()
    return {"value": units * world / wall, "unit": "DM-trial*samples/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": units * 4, "ms_per_step": wall * 1e3,
            "realtime_x": sum(strat["t_processed"][0]) * cfg["tsamp"] / wall}


def measure_e2e_analysis(aa, md, plan, xh, units, e2e_steps, local, device, world):
    """The e2e run with the analysis component (single-pulse detection of
    every step's rows and its candidate files), as the reference runner does
    it."""
    import tempfile
    import torch
    a = ANALYSIS
    comps_a = aa.aa_py_pipeline_components(True, True, False, False)
    opts = aa.aa_py_pipeline_component_options()
    opts.copy_ddtr_data_to_host = True
    api = aa.aa_py_pipeline(comps_a, opts, md, ctypes_ushort_ptr(xh), local)
    if not api.bind_ddtr_plan(plan):
        raise RuntimeError(api.last_error())
    if not api.bind_analysis_plan(aa.aa_py_analysis_plan(a["sigma_cutoff"], a["sigma_constant"], a["max_width_s"],
                                                         a["algorithm"], bool(a["baseline_noise"]))):
        raise RuntimeError(api.last_error())
    api.set_candidate_output(True, tempfile.mkdtemp(prefix="spd_cands_"))
    walls, ncand = [], 0
    for step in range(1 + e2e_steps):
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        api.rewind()
        ncand = 0
        while api.run():
            if api.status_code() == aa.STATUS_HAS_MORE:
                ncand += lib_spd_count(aa, api)
        if api.status_code() == aa.STATUS_ERROR:
            raise RuntimeError(api.last_error())
        torch.cuda.synchronize(device)
        walls.append(time.perf_counter() - t0)
    wall = statistics.median(walls[1:])
    api.cleanUp()
    api.delete()
    return {"value": units * world / wall, "unit": "DM-trial*samples/s", "ms_per_step": wall * 1e3,
            "candidates": ncand, "settings": a}


def measure_e2e_packed(aa, cfg, md, plan, xh, x_host, strat, units, e2e_steps, local, device, barrier, world):
    """The e2e run fed the samples as a SIGPROC file stores them
    (aa_b200_pipeline_set_packed_input): nbits/16 of the H2D bytes."""
    import torch
    import torch.distributed as dist
    from aa_b200.sigproc import pack
    if cfg["nbits"] == 8:
        xp = torch.empty((xh.shape[0], xh.shape[1]), dtype=torch.uint8, pin_memory=True)
        xp.copy_(xh.to(torch.uint8))
    else:
        xp = torch.from_numpy(pack(x_host, cfg["nbits"])).pin_memory()
    comps = aa.aa_py_pipeline_components(True, False, False, False)
    opts = aa.aa_py_pipeline_component_options()
    opts.copy_ddtr_data_to_host = True
    api = aa.aa_py_pipeline(comps, opts, md, None, local)
    api.set_packed_input(xp.data_ptr())
    if not api.bind_ddtr_plan(plan):
        raise RuntimeError(api.last_error())
    walls = []
    for step in range(1 + e2e_steps):
        torch.cuda.synchronize(device)
        barrier()
        t0 = time.perf_counter()
        api.rewind()
        while api.run():
            pass
        if api.status_code() == aa.STATUS_ERROR:
            raise RuntimeError(api.last_error())
        torch.cuda.synchronize(device)
        walls.append(time.perf_counter() - t0)
    wall = statistics.median(walls[1:])
    if world > 1:
        t = torch.tensor([wall], device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        wall = float(t.item())
    api.cleanUp()
    api.delete()
    del xp
    return {"value": units * world / wall, "unit": "DM-trial*samples/s", "ms_per_step": wall * 1e3,
            "h2d_bytes_per_step": sum((strat["t_processed"][0][k] + strat["maxshift"]) * cfg["nchans"] *
                                      cfg["nbits"] // 8 for k in range(strat["num_tchunks"])),
            "d2h_bytes_per_step": units * 4, "api": "aa_b200_pipeline_set_packed_input"}


def measure_mid_e2e(aa, local, device, e2e_steps):
    """The 2^18-sample configuration (bench's MID: the survey plan, 4096
    channels) end to end through the C ABI, on the input the reference arm's
    reference_gpu figure uses (the same generator and seed)."""
    import torch
    cfg = MID
    x, _ = synth_input_device(cfg, cfg["seed"], device)
    xh = torch.empty(x.shape, dtype=torch.int16, pin_memory=True)
    xh.copy_(x)
    del x
    torch.cuda.empty_cache()
    md = metadata_struct(aa, cfg)
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in cfg["plan"]])
    strat = aa.strategy(cfg["plan"], cfg["nchans"], cfg["nsamp"], cfg["fch1"], cfg["foff"], cfg["tsamp"],
                        cfg["nbits"])
    units = units_per_step(strat)
    r = measure_e2e(aa, cfg, md, plan, xh, strat, units, max(3, e2e_steps), local, device, lambda: None, 1)
    plan.delete()
    r["workload"] = (f"{cfg['nchans']} ch x {cfg['nsamp']} samples, {cfg['nbits']}-bit, {len(cfg['plan'])}-range "
                     f"survey plan, host [t][c] input, rows copied to the host")
    return r


def lib_spd_count(aa, api) -> int:
    return int(aa.lib().aa_py_spd_nCandidates(api.m_obj))


def ctypes_ushort_ptr(t):
    import ctypes
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), ctypes.POINTER(ctypes.c_ushort))


if __name__ == "__main__":
    sys.exit(main())
