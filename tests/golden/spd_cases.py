"""Seeded DM-time planes for the single-pulse detection tests: Gaussian
noise with dispersed pulses (a peak at one DM trial and sample, falling off
over neighbouring trials and widening with DM distance), and the analysis
settings of each run."""
from __future__ import annotations

import numpy as np

# name -> plane shape, plane seed, settings
CASES = {
    "small_peak": dict(ndms=64, nt=16384, seed=1, tsamp=64e-6, inbin=1, max_width_s=0.004, sigma_constant=3.0,
                       baseline_noise=0, cutoff=6.0, algorithm=0),
    "small_threshold": dict(ndms=64, nt=16384, seed=1, tsamp=64e-6, inbin=1, max_width_s=0.004, sigma_constant=3.0,
                            baseline_noise=0, cutoff=6.0, algorithm=1),
    "wide_outliers_peak": dict(ndms=128, nt=32768, seed=2, tsamp=64e-6, inbin=1, max_width_s=0.016,
                               sigma_constant=3.0, baseline_noise=1, cutoff=6.0, algorithm=0),
    "binned_outliers": dict(ndms=64, nt=16384, seed=3, tsamp=128e-6, inbin=2, max_width_s=0.02, sigma_constant=2.5,
                            baseline_noise=1, cutoff=5.5, algorithm=0),
    "very_wide_threshold": dict(ndms=64, nt=65536, seed=4, tsamp=64e-6, inbin=1, max_width_s=0.065,
                                sigma_constant=3.0, baseline_noise=0, cutoff=7.0, algorithm=1),
    # rows too short to decimate to the widest width: the MSD profile switches
    # to boxcars over the last decimation (src/aa_device_MSD_plane_profile.cu:267-338)
    "short_switch": dict(ndms=32, nt=4096, seed=5, tsamp=64e-6, inbin=1, max_width_s=0.06, sigma_constant=3.0,
                         baseline_noise=0, cutoff=6.0, algorithm=0),
    # the search in batches of 24 and 20 DM trials (analysis_GPU's maxTimeSamples
    # below the plane): peak neighbourhoods end at the batch edges
    "batched_peak": dict(ndms=64, nt=16384, seed=6, tsamp=64e-6, inbin=1, max_width_s=0.008, sigma_constant=3.0,
                         baseline_noise=0, cutoff=5.5, algorithm=0, max_ts=24 * 16384),
    "batched_threshold": dict(ndms=48, nt=8192, seed=7, tsamp=64e-6, inbin=1, max_width_s=0.004,
                              sigma_constant=3.0, baseline_noise=1, cutoff=6.0, algorithm=1, max_ts=20 * 8192),
    # 66 DM trials: batches of 64 and 2, thresholding skips rows past 4*floor(n/4)
    "ragged_dms_threshold": dict(ndms=66, nt=8192, seed=8, tsamp=64e-6, inbin=1, max_width_s=0.004,
                                 sigma_constant=3.0, baseline_noise=0, cutoff=5.0, algorithm=1),
    # peak filtering: 7 x 7 stencil peaks, then weaker peaks within 15 ms dropped
    "small_filter": dict(ndms=64, nt=16384, seed=1, tsamp=64e-6, inbin=1, max_width_s=0.004, sigma_constant=3.0,
                         baseline_noise=0, cutoff=5.0, algorithm=2),
    "wide_filter_outliers": dict(ndms=128, nt=32768, seed=9, tsamp=128e-6, inbin=2, max_width_s=0.03,
                                 sigma_constant=3.0, baseline_noise=1, cutoff=5.5, algorithm=2),
}

# The reference runner with the analysis component on the DDTR cases of
# cases.py: analysis settings per run.
PIPELINE_CASES = {
    "pipe_binned_peak": dict(ddtr="shared8_binned", sigma_cutoff=6.0, sigma_constant=3.0, max_width_s=0.01,
                             algorithm=0, baseline_noise=0),
    "pipe_chunked_threshold": dict(ddtr="shared8_chunked", sigma_cutoff=6.5, sigma_constant=3.0,
                                   max_width_s=0.005, algorithm=1, baseline_noise=1),
    "pipe_cache_peak": dict(ddtr="cache8", sigma_cutoff=5.5, sigma_constant=2.5, max_width_s=0.02, algorithm=0,
                            baseline_noise=1),
    "pipe_binned_filter": dict(ddtr="shared8_binned", sigma_cutoff=5.0, sigma_constant=3.0, max_width_s=0.01,
                               algorithm=2, baseline_noise=0),
}


def single_batch(case) -> bool:
    """The search runs the whole plane in one batch (the S/N planes of the
    reference's whole-plane stage are then comparable)."""
    n = case["ndms"] * case["nt"]
    mts = case.get("max_ts", 0) or n
    return (min(mts, n) // case["nt"]) // 4 * 4 >= case["ndms"]


def make_plane(case) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(case["seed"]))
    nd, nt = case["ndms"], case["nt"]
    x = rng.normal(100.0, 4.0, (nd, nt)).astype(np.float32)
    t_idx = np.arange(nt)
    for k in range(6):
        d0 = int(rng.integers(4, nd - 4))
        t0 = int(rng.integers(100, nt - 2000))
        w = float(rng.uniform(1.0, 60.0))
        amp = float(rng.uniform(3.0, 12.0))
        for d in range(nd):
            dd = abs(d - d0)
            ww = w + 3.0 * dd
            a = amp * np.exp(-0.5 * (dd / 3.0) ** 2) * np.sqrt(w / ww)
            if a < 0.05:
                continue
            x[d] += (a * np.exp(-0.5 * ((t_idx - t0) / ww) ** 2)).astype(np.float32)
    return x
