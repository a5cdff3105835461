"""Seeded DDTR cases shared by the golden-vector generator and the tests.

Each case is small enough for the CPU oracle to finish in seconds and
exercises one branch of the reference path: the kernel it dispatches to
(src/aa_dedisperse.cpp:5-163), the x2 binning steps of the runner
(include/aa_permitted_pipelines_generic.hpp:797-808, including the second
and later binning steps whose length the runner computes from the wrong
stride), time chunking, bit depths 2/4/8/16, and channel counts that are not
powers of two.  The inputs are synthetic (there is no public dataset for this
path): Gaussian noise at mid-scale plus dispersed boxcar pulses with the
cold-plasma delay 4.148808e3 * DM * (f^-2 - fch1^-2) s.
"""
from __future__ import annotations

import numpy as np

# the survey-scale 8-range plan (the reference's example plan,
# examples/src/filterbank_dedispersion.cpp:26-33)
SURVEY_PLAN = [(0, 150, 0.1, 1, 1), (150, 300, 0.2, 1, 1), (300, 500, 0.25, 1, 1), (500, 900, 0.4, 2, 1),
               (900, 1200, 0.6, 4, 1), (1200, 1500, 0.8, 4, 1), (1500, 2000, 1.0, 4, 1), (2000, 3000, 2.0, 8, 1)]

# binned low-DM plan: every range takes the shared kernels, inBin 1 -> 2 -> 4 -> 8
BINNED_PLAN = [(0, 6.3, 0.1, 1, 1), (6.4, 19.1, 0.2, 2, 1), (19.2, 44.7, 0.4, 4, 1), (44.8, 95.9, 0.8, 8, 1)]

CASES = {
    # cache ("failsafe") kernel, one range, 8-bit
    "cache8": dict(nchans=256, nbits=8, fch1=1550.0, foff=-1.5625, tsamp=64e-6, nsamp=1 << 15,
                   plan=[(0, 127, 0.5, 1, 1)], free_memory=0, seed=11, pulses=[(60.0, 16, 5.0)]),
    # shared 8-bit kernel through three binning steps
    "shared8_binned": dict(nchans=512, nbits=8, fch1=1670.0, foff=-0.5859375, tsamp=64e-6, nsamp=1 << 15,
                           plan=BINNED_PLAN, free_memory=0, seed=12, pulses=[(30.0, 8, 6.0), (70.0, 20, 4.0)]),
    # same, split into several time chunks by a small memory budget
    "shared8_chunked": dict(nchans=512, nbits=8, fch1=1670.0, foff=-0.5859375, tsamp=64e-6, nsamp=1 << 15,
                            plan=BINNED_PLAN, free_memory=104857600 + 9000 * 512 * 6, seed=13,
                            pulses=[(40.0, 12, 5.0)]),
    # channel count that is not a power of two (fast-math division differs
    # from IEEE in the last bit) -- no binning so nchans need not be a multiple of 32
    "shared8_nch3000": dict(nchans=3000, nbits=8, fch1=1670.0, foff=-0.1, tsamp=64e-6, nsamp=1 << 14,
                            plan=[(0, 12.7, 0.2, 1, 1)], free_memory=0, seed=14, pulses=[(8.0, 8, 5.0)]),
    # 2-bit data through the 8-bit kernel
    "shared8_2bit": dict(nchans=256, nbits=2, fch1=1400.0, foff=-1.0, tsamp=64e-6, nsamp=1 << 15,
                         plan=[(0, 12.7, 0.2, 1, 1), (12.8, 38.3, 0.4, 2, 1)], free_memory=0, seed=15,
                         pulses=[(10.0, 16, 2.0)]),
    # 4-bit shared kernel (findex 4tx+3, no /bin)
    "shared4": dict(nchans=512, nbits=4, fch1=1670.0, foff=-0.5859375, tsamp=64e-6, nsamp=1 << 15,
                    plan=[(0, 3.15, 0.05, 1, 1), (3.2, 9.5, 0.1, 2, 1)], free_memory=0, seed=16,
                    pulses=[(4.0, 12, 3.0)]),
    # 4-bit wide band: the reference sums only 4096*floor(nchans/4096) channels
    "shared4_wide": dict(nchans=4160, nbits=4, fch1=1670.0, foff=-0.0732421875, tsamp=64e-6, nsamp=1 << 13,
                         plan=[(0, 3.15, 0.05, 1, 1)], free_memory=0, seed=17, pulses=[(2.0, 8, 3.0)]),
    # 16-bit shared kernel: fp32 sums above 2^24 round, order matters
    "shared16": dict(nchans=1024, nbits=16, fch1=1670.0, foff=-0.29296875, tsamp=64e-6, nsamp=1 << 14,
                     plan=[(0, 6.3, 0.1, 1, 1), (6.4, 19.1, 0.2, 2, 1)], free_memory=0, seed=18,
                     pulses=[(10.0, 8, 3.0)]),
    # 16-bit, 1000 channels (stages end mid-row), two binning steps, three time chunks
    "shared16_ragged": dict(nchans=1000, nbits=16, fch1=1670.0, foff=-0.3, tsamp=64e-6, nsamp=1 << 15,
                            plan=[(0, 6.3, 0.1, 1, 1), (6.4, 19.1, 0.2, 2, 1), (19.2, 44.7, 0.4, 4, 1)],
                            free_memory=104857600 + 9000 * 1000 * 10, seed=22, pulses=[(12.0, 8, 3.0)]),
    # 16-bit data on the cache kernel
    "cache16": dict(nchans=512, nbits=16, fch1=1550.0, foff=-0.78125, tsamp=64e-6, nsamp=1 << 14,
                    plan=[(0, 63, 0.5, 1, 1)], free_memory=0, seed=19, pulses=[(30.0, 8, 3.0)]),
    # a band and sampling time where the reference's per-thread shift
    # shift_one*dm_shifts[c]+findex lands within one rounding of an integer:
    # fused and unfused evaluation give different delays for ~1.5% of the
    # outputs, so this case pins the contraction the reference build uses
    "fma_probe": dict(nchans=512, nbits=8, fch1=1662.862, foff=-0.526171875, tsamp=9.0443e-05, nsamp=1 << 14,
                      plan=[(10.36, 20.05, 0.0763, 1, 1)], free_memory=0, seed=21, pulses=[(14.0, 8, 5.0)]),
    # 1024 channels x 2^18 samples, 8-bit, 0-500 in steps of 0.5 (1024 trials after rounding), one pulse
    # of 1 ms at DM 300 and 5 sigma: the plain small configuration at its full size (cache kernel)
    "plain1024_full": dict(nchans=1024, nbits=8, fch1=1550.0, foff=-0.390625, tsamp=64e-6, nsamp=1 << 18,
                           plan=[(0, 500, 0.5, 1, 1)], free_memory=0, seed=1, pulses=[(300.0, 16, 5.0)], heavy=True),
    # more than 8192 channels: the reference reads the delay table from global memory
    # (shared_dedisperse_kernel_nchan8192p, src/aa_device_dedispersion_kernel.cu:243-301)
    "wide8": dict(nchans=8320, nbits=8, fch1=1670.0, foff=-300.0 / 8320, tsamp=64e-6, nsamp=1 << 13,
                  plan=[(0, 25.5, 0.1, 1, 1)], free_memory=0, seed=23, pulses=[(12.0, 8, 4.0)]),
    # the same band with 16-bit samples: above 8192 channels the reference launches its
    # constant-memory kernel without filling the table past 8192 entries
    # (src/aa_device_dedispersion_kernel.cu:540-543); this library computes the intended
    # delays, so the case is checked against the oracle only
    "wide16": dict(nchans=8320, nbits=16, fch1=1670.0, foff=-300.0 / 8320, tsamp=64e-6, nsamp=1 << 13,
                   plan=[(0, 25.5, 0.1, 1, 1)], free_memory=0, seed=24, pulses=[(12.0, 8, 3.0)],
                   no_reference=True),
    # the survey plan on a short 4096-channel block (every range is shared-kernel)
    "survey_plan": dict(nchans=4096, nbits=8, fch1=1670.0, foff=-0.0732421875, tsamp=64e-6, nsamp=45000,
                        plan=SURVEY_PLAN, free_memory=0, seed=20, pulses=[(400.0, 16, 5.0), (1700.0, 40, 4.0)],
                        heavy=True),
}

MAX_BY_BITS = {1: 1, 2: 3, 4: 15, 8: 255, 16: 65535, 32: 65535}


def cold_plasma_delays(nchans, fch1, foff, dm, tsamp):
    """Injection delay in samples: 4.148808e3 * DM * (f^-2 - fch1^-2) s."""
    f = fch1 + foff * np.arange(nchans, dtype=np.float64)
    return np.floor(4.148808e3 * dm * (f ** -2 - fch1 ** -2) / tsamp).astype(np.int64)


def make_input(case: dict) -> np.ndarray:
    """Time-major [nsamp][nchans] uint16, one value per sample (the reference's
    host input format, src/aa_sigproc_input.cpp:364-543)."""
    rng = np.random.Generator(np.random.PCG64(case["seed"]))
    nchans, nsamp, nbits = case["nchans"], case["nsamp"], case["nbits"]
    vmax = MAX_BY_BITS[nbits]
    mid, sig = (vmax + 1) / 2.0 - 0.5, (vmax + 1) / 16.0
    x = rng.normal(mid, sig, size=(nsamp, nchans))
    for (dm, width, amp) in case.get("pulses", []):
        start = int(rng.integers(nsamp // 8, nsamp // 3))
        dl = cold_plasma_delays(nchans, case["fch1"], case["foff"], dm, case["tsamp"])
        for c in range(nchans):
            t0 = start + int(dl[c])
            if t0 < nsamp:
                x[t0:min(nsamp, t0 + width), c] += amp * sig
    return np.clip(np.rint(x), 0, vmax).astype(np.uint16)


def strategy_free_memory(case: dict) -> int:
    """The device memory the strategy is computed for (0 -> a B200's)."""
    return case["free_memory"] or 180 * 2**30
