"""Seeded cases for the periodicity component end to end (the reference's
runner with dedispersion and periodicity, include/aa_permitted_pipelines_generic.hpp:570-660):
8-bit filterbanks with a dispersed periodic pulse train over Gaussian
noise, two DM ranges (the second binned x2), and the periodicity settings
each case runs (harmonic sum algorithm, candidate selection)."""
from __future__ import annotations

import numpy as np

import cases as C

# 256 channels over 1550..1150 MHz at 64 us; 2^17 + 4096 samples, so the
# processed length (nsamp - maxshift) rounds down to a 2^17-point FFT
BASE = dict(nchans=256, nbits=8, fch1=1550.0, foff=-1.5625, tsamp=64e-6, nsamp=(1 << 17) + 4096,
            plan=[(0, 25.5, 0.1, 1, 1), (25.6, 76.7, 0.2, 2, 1)], free_memory=0)

# period 48.0 ms (750 samples), duty cycle about 1 %, DM 14.3
TRAIN = dict(dm=14.3, period_samples=750.0, width=8, amp=0.12)

PSR_MEMORY = 8 << 30  # bytes the periodicity strategy plans for (both sides)

PIPELINE_CASES = {
    "psr_greedy_peaks": dict(BASE, seed=41, train=TRAIN, sigma_cutoff=8.0, nHarmonics=32, hs_algorithm=1,
                             selection=0),
    "psr_greedy_threshold": dict(BASE, seed=42, train=TRAIN, sigma_cutoff=12.0, nHarmonics=16, hs_algorithm=1,
                                 selection=1),
    "psr_simple_peaks": dict(BASE, seed=43, train=TRAIN, sigma_cutoff=8.0, nHarmonics=32, hs_algorithm=0,
                             selection=0),
    "psr_presto_plus_peaks": dict(BASE, seed=44, train=TRAIN, sigma_cutoff=8.0, nHarmonics=32, hs_algorithm=2,
                                  selection=0),
    "psr_presto_peaks": dict(BASE, seed=45, train=TRAIN, sigma_cutoff=8.0, nHarmonics=16, hs_algorithm=3,
                             selection=0),
}


def make_input(case: dict) -> np.ndarray:
    """[nsamp][nchans] uint16: noise at mid-scale plus the pulse train, each
    pulse dispersed with the cold-plasma delay of the train's DM."""
    rng = np.random.Generator(np.random.PCG64(case["seed"]))
    nchans, nsamp, nbits = case["nchans"], case["nsamp"], case["nbits"]
    vmax = C.MAX_BY_BITS[nbits]
    mid, sig = (vmax + 1) / 2.0 - 0.5, (vmax + 1) / 16.0
    x = rng.normal(mid, sig, size=(nsamp, nchans))
    tr = case["train"]
    dl = C.cold_plasma_delays(nchans, case["fch1"], case["foff"], tr["dm"], case["tsamp"]).astype(np.int64)
    t = float(rng.uniform(0, tr["period_samples"]))
    while t < nsamp:
        t0 = int(t)
        for c in range(nchans):
            a = t0 + int(dl[c])
            if a < nsamp:
                x[a:min(nsamp, a + tr["width"]), c] += tr["amp"] * sig
        t += tr["period_samples"]
    return np.clip(np.rint(x), 0, vmax).astype(np.uint16)
