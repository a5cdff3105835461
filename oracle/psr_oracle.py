"""CPU restatement of two periodicity stages -- TEST INFRASTRUCTURE ONLY
(used by tests/ to check the library and the golden vectors; never by the
library).

* simple_power_and_interbin (src/aa_device_power.cu:34-52,
  src/aa_device_power_kernel.cu:19-41): bins 0 < k < nT/2 of each spectrum
  divided by sqrt(nT); power |A|^2, interbin 0.616850275 |A - B|^2 with B
  the next bin; bin 0 gives 0.
* simple harmonic sum (src/aa_device_harmonic_summing_kernel.cu:8-39): the
  running sum of bins b, 2b, 3b, ... and the best (sum - mean_f) / sd_f.

The reference divides with the fast division of its --use_fast_math build
and may fuse products into sums, so this float32 restatement agrees to about
1e-6 relative (1e-5 on the interbin values, whose differences cancel); the
bits are pinned by the reference's GPU run (tests/golden/psr_golden.json).
"""
from __future__ import annotations

import numpy as np


def power_interbin(spectra: np.ndarray, nt: int):
    """spectra [ndms][2*(nt//2+1)] float32 (interleaved complex)."""
    nd = spectra.shape[0]
    half = nt >> 1
    z = spectra.reshape(nd, -1, 2).astype(np.float32)
    norm = np.float32(np.sqrt(np.float64(nt)))
    a = np.zeros((nd, half, 2), np.float32)
    b = np.zeros((nd, half, 2), np.float32)
    a[:, 1:half] = z[:, 1:half] / norm
    b[:, 1:half] = z[:, 2:half + 1] / norm
    power = (a[..., 0] * a[..., 0] + a[..., 1] * a[..., 1]).astype(np.float32)
    d = a - b
    inter = np.zeros((nd, nt), np.float32)
    inter[:, 0:2 * half:2] = power
    inter[:, 1:2 * half:2] = np.float32(0.616850275) * (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1])
    return power, inter


def harmonic_sum_simple(x: np.ndarray, msd: np.ndarray, nh: int):
    """x [nbins][nspectra] float32 -> (snr, harmonics) of the same shape."""
    nb, ns = x.shape
    m = msd.astype(np.float32).reshape(-1, 2)
    hs = x.astype(np.float32).copy()
    snr = ((hs - m[0, 0]) / m[0, 1]).astype(np.float32)
    harm = np.zeros((nb, ns), np.uint16)
    b = np.arange(nb)
    for f in range(1, nh):
        bins = b + f * b
        ok = (b > 0) & (bins < nb)
        if not ok.any():
            continue
        idx = np.nonzero(ok)[0]
        hs[idx] = hs[idx] + x[bins[idx]]
        t = ((hs[idx] - m[f, 0]) / m[f, 1]).astype(np.float32)
        better = t > snr[idx]
        rows = idx[np.any(better, axis=1)]
        sel = better[np.isin(idx, rows)]
        snr[rows] = np.where(sel, t[np.isin(idx, rows)], snr[rows])
        harm[rows] = np.where(sel, f, harm[rows])
    return snr, harm
