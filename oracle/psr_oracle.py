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


# ---------------------------------------------------------------------------
# Spectral whitening (spectrum_whitening_SGP2 with medians)
# ---------------------------------------------------------------------------
def segment_sizes(n_samples: int, min_len: int = 6, max_len: int = 250):
    """create_dered_segment_sizes_prefix_sum (src/aa_device_spectral_whitening.cu:17-31):
    0, 1 + min_len, then steps of int(min_len * ln(position)) capped at
    max_len while the next step stays below n_samples, then n_samples."""
    import math
    s = [0]
    length = min_len
    total = 1 + length
    s.append(total)
    while total + length < n_samples:
        total += length
        length = min(int(min_len * math.log(total)), max_len)
        s.append(total)
    s.append(n_samples)
    return s


def segment_medians(power_row: np.ndarray, seg):
    """GPU_kernel_segmented_median (src/aa_device_spectral_whitening_kernel.cu:338-376):
    the segment's powers sorted among 256 zero-padded slots; odd counts take
    slot zeros + n/2, even counts the mean of slots zeros + n/2 and the one
    after (the last slot when that is past the end)."""
    out = np.empty(len(seg) - 1, np.float32)
    for b in range(len(seg) - 1):
        v = np.zeros(256, np.float32)
        r = seg[b + 1] - seg[b]
        v[256 - r:] = np.sort(power_row[seg[b]:seg[b + 1]])
        mp = 256 - r + (r >> 1)
        out[b] = (v[mp] + v[min(mp + 1, 255)]) * np.float32(0.5) if r % 2 == 0 else v[mp]
    return out


def whitening(spectra: np.ndarray):
    """GPU_kernel_spectrum_whitening_SGP2 (src/aa_device_spectral_whitening_kernel.cu:378-427)
    restated on [ndms][n] complex64 spectra: bins divided by the square root
    of median / ln 2 interpolated linearly between segment middles (the first
    half segment by its own median, bin 0 set to 1; the bins after the middle
    of the last segment by the last block's thread norms, index range - t).
    A bin the reference scales in two blocks (even segment then odd one) is
    scaled once, by the later block.  Exact float sqrt and division stand in
    for the reference's fast-math forms: equal to about 1e-6 relative."""
    x = spectra.astype(np.complex64).copy()
    ndms, n = x.shape
    seg = segment_sizes(n)
    ns = len(seg)
    ln2inv = 1.44269504088896
    for d in range(ndms):
        p = (x[d].real * x[d].real + x[d].imag * x[d].imag).astype(np.float32)
        med = segment_medians(p, seg)
        scale = np.ones(n, np.float32)
        cm = np.float32(np.float64(med[0]) * ln2inv)
        scale[:(seg[1] - seg[0]) >> 1] = np.float32(1.0 / np.float64(np.sqrt(cm)))
        for b in range(1, ns - 1):
            fm1, f0, fp1 = seg[b - 1], seg[b], seg[b + 1]
            pr, cr = f0 - fm1, fp1 - f0
            pm = np.float32(np.float64(med[b - 1]) * ln2inv)
            cm = np.float32(np.float64(med[b]) * ln2inv)
            rng = (pr + cr + 1) >> 1
            slope = np.float32(np.float32(cm - pm) / np.float32(rng))
            last = b == ns - 2
            shared = not last and pr % 2 == 0 and cr % 2 == 1
            for t in range(256):
                i = rng - t
                with np.errstate(invalid="ignore", divide="ignore"):
                    norm = np.float32(1.0 / np.float64(np.sqrt(np.float32(pm + np.float32(slope * np.float32(i))))))
                lp = fm1 + (pr >> 1) + i
                if 0 <= i < rng - (1 if shared else 0) and lp < n:
                    scale[lp] = norm
                if last:
                    tp = fm1 + (pr >> 1) + rng + t
                    if tp < n:
                        scale[tp] = norm
        x[d] = (x[d].real * scale) + 1j * (x[d].imag * scale)
        x[d, 0] = 1.0 + 0.0j
    return x


def shared_norms(spectrum: np.ndarray):
    """For one spectrum ([n] complex64): per bin that two neighbouring
    blocks of the reference's whitening both scale (an even segment followed
    by an odd one), the pair (norm of the earlier block's last index, norm of
    the later block's first index), as whitening() computes norms."""
    n = spectrum.size
    seg = segment_sizes(n)
    p = (spectrum.real * spectrum.real + spectrum.imag * spectrum.imag).astype(np.float32)
    med = segment_medians(p, seg)
    ln2inv = 1.44269504088896

    def norm(b, i):
        pr, cr = seg[b] - seg[b - 1], seg[b + 1] - seg[b]
        pm = np.float32(np.float64(med[b - 1]) * ln2inv)
        cm = np.float32(np.float64(med[b]) * ln2inv)
        rng = (pr + cr + 1) >> 1
        slope = np.float32(np.float32(cm - pm) / np.float32(rng))
        return np.float32(1.0 / np.float64(np.sqrt(np.float32(pm + np.float32(slope * np.float32(i))))))

    out = {}
    for b in range(1, len(seg) - 2):
        pr, cr = seg[b] - seg[b - 1], seg[b + 1] - seg[b]
        if pr % 2 == 0 and cr % 2 == 1:
            rng = (pr + cr + 1) >> 1
            out[seg[b] + (cr >> 1)] = (norm(b, rng - 1), norm(b + 1, 0))
    return out


def candidates_process(rec, msd, dm_low, dm_step, tsamp, nt, mod, greedy):
    """aa_periodicity_candidates_data::Process (include/aa_periodicity_candidates.hpp:81-105)
    on records [n][4] float32, in its float/double expressions: the bin width
    (1/tsamp) / float(nt * mod) with nt rounded to float, fraction offset/h
    in double stored as float, DM and frequency in double stored as float,
    S/N in float."""
    r = np.array(rec, np.float32).reshape(-1, 4).copy()
    h = r[:, 3].astype(np.int64)
    fc = np.zeros(len(r), np.float32)
    if greedy:
        ds = (r[:, 3].astype(np.float64) / 100.0).astype(np.int64)
        h = h - ds * 100
        bw = np.float32((1.0 / tsamp) / np.float64(np.float32(np.float32(nt) * np.float32(mod))))
        pos = h > 0
        frac = (ds[pos].astype(np.float64) / h[pos].astype(np.float64)).astype(np.float32)
        fc[pos] = (bw * frac).astype(np.float32)
    m = np.asarray(msd, np.float32)
    r[:, 0] = (r[:, 0].astype(np.float64) * dm_step + dm_low).astype(np.float32)
    r[:, 1] = (r[:, 1].astype(np.float64) * (1.0 / (tsamp * np.float64(nt) * np.float64(np.float32(mod))))
               + fc.astype(np.float64)).astype(np.float32)
    r[:, 2] = ((r[:, 2] - m[2 * h]) / m[2 * h + 1]).astype(np.float32)
    r[:, 3] = h.astype(np.float32)
    return r
