"""Seeded inputs for the periodicity building blocks: complex spectra as
cufftExecR2C writes them (nT/2+1 bins per DM trial) and corner-turned power
spectra [bins][spectra] with a (mean, deviation) per harmonic count."""
from __future__ import annotations

import numpy as np

POWER_CASES = {
    "pow_8192x24": dict(nt=8192, ndms=24, seed=1),
    "pow_6000x7": dict(nt=6000, ndms=7, seed=2),
    "pow_4097x3": dict(nt=4097, ndms=3, seed=3),
}
HARMONIC_CASES = {
    "hs_4097x100_h32": dict(nbins=4097, nspectra=100, nh=32, seed=4),
    "hs_1000x64_h8": dict(nbins=1000, nspectra=64, nh=8, seed=5),
    "hs_513x7_h16": dict(nbins=513, nspectra=7, nh=16, seed=6),
}


def make_spectra(c) -> np.ndarray:
    """[ndms][nt/2+1] complex64 as interleaved float32 pairs: noise spectra of
    N(0, sqrt(nt)) with a few strong periodic lines."""
    rng = np.random.Generator(np.random.PCG64(c["seed"]))
    nb = (c["nt"] >> 1) + 1
    z = (rng.normal(0, 1, (c["ndms"], nb)) + 1j * rng.normal(0, 1, (c["ndms"], nb))) * np.sqrt(c["nt"] / 2)
    for d in range(c["ndms"]):
        k = int(rng.integers(5, nb // 8))
        for h in range(1, 6):
            if h * k < nb:
                z[d, h * k] += (8.0 / h) * np.sqrt(c["nt"]) * np.exp(1j * rng.uniform(0, 2 * np.pi))
    return np.ascontiguousarray(z.astype(np.complex64)).view(np.float32).reshape(c["ndms"], 2 * nb)


def make_harmonic_input(c):
    """(input [nbins][nspectra] float32, msd [2*nh] float32)."""
    rng = np.random.Generator(np.random.PCG64(c["seed"]))
    x = rng.exponential(1.0, (c["nbins"], c["nspectra"])).astype(np.float32)
    for s in range(c["nspectra"]):
        k = int(rng.integers(3, max(4, c["nbins"] // 16)))
        for h in range(1, 9):
            if h * k < c["nbins"]:
                x[h * k, s] += np.float32(6.0 / h)
    f = np.arange(c["nh"], dtype=np.float32)
    msd = np.empty(2 * c["nh"], np.float32)
    msd[0::2] = f + 1
    msd[1::2] = np.sqrt(f + 1)
    return x, msd


# MSD plane profiles of power-spectrum planes, as the periodicity search runs
# them (high_memory, widths 1..nHarmonics), and in the analysis' form
MSD_CASES = {
    "msd_power_h32_or": dict(nt=16384, ndms=32, seed=7, nh=32, high_memory=1, sigma=3.0, outliers=1),
    "msd_power_h16": dict(nt=8192, ndms=48, seed=8, nh=16, high_memory=1, sigma=3.0, outliers=0),
    "msd_power_h8_low": dict(nt=8192, ndms=20, seed=9, nh=8, high_memory=0, sigma=2.5, outliers=1),
    "msd_power_h32_odd": dict(nt=10000, ndms=13, seed=10, nh=32, high_memory=1, sigma=3.0, outliers=1),
}


def make_power_plane(c) -> np.ndarray:
    """[ndms][nt] float32 power-like values (exponential) with a few lines."""
    rng = np.random.Generator(np.random.PCG64(c["seed"]))
    x = rng.exponential(1.0, (c["ndms"], c["nt"])).astype(np.float32)
    for d in range(c["ndms"]):
        k = int(rng.integers(10, c["nt"] // 16))
        for h in range(1, 8):
            if h * k < c["nt"]:
                x[d, h * k] += np.float32(20.0 / h)
    return x


# Peak finding on harmonic-sum S/N planes (with their harmonic counts)
PEAK_CASES = {
    "peaks_transposed": dict(nt=4096, ndms=48, seed=11, nh=16, threshold=3.0, dm_shift=100, inbin=1, transposed=1,
                             greedy=0),
    "peaks_normal": dict(nt=3000, ndms=33, seed=12, nh=16, threshold=3.0, dm_shift=0, inbin=1, transposed=0,
                         greedy=0),
    "peaks_normal_greedy": dict(nt=2048, ndms=20, seed=13, nh=8, threshold=2.5, dm_shift=7, inbin=1, transposed=0,
                                greedy=1),
}


def make_peak_plane(c):
    """(S/N plane, harmonic counts, msd[2*nh]) in the case's layout."""
    rng = np.random.Generator(np.random.PCG64(c["seed"]))
    shape = (c["nt"], c["ndms"]) if c["transposed"] else (c["ndms"], c["nt"])
    snr = rng.normal(0, 1, shape).astype(np.float32)
    harm = rng.integers(0, c["nh"], shape).astype(np.uint16)
    if c["greedy"]:
        harm = (harm + 100 * rng.integers(0, 3, shape)).astype(np.uint16)
    f = np.arange(c["nh"], dtype=np.float32)
    msd = np.empty(2 * c["nh"], np.float32)
    msd[0::2] = 2.0 * (f + 1)
    msd[1::2] = np.sqrt(f + 1) * np.float32(1.5)
    return snr, harm, msd


# Greedy (1), PRESTO plus (2) and PRESTO (3) harmonic sums on normal power
# planes [ndms][nt]; nh is the reference's nHarmonics argument; the msd table
# always has 32 entries.
HS_ALGO_CASES = {
    "greedy_h16": dict(algorithm=1, nt=8192, ndms=6, seed=14, nh=16, scalloping=0),
    "greedy_h8_scal": dict(algorithm=1, nt=5000, ndms=5, seed=15, nh=8, scalloping=1),
    "presto_plus_h8": dict(algorithm=2, nt=4096, ndms=4, seed=16, nh=8, scalloping=0),
    "presto_plus_h6_scal": dict(algorithm=2, nt=3001, ndms=3, seed=17, nh=6, scalloping=1),
    "presto_h5": dict(algorithm=3, nt=8192, ndms=4, seed=18, nh=5, scalloping=0),
    "presto_h4_scal": dict(algorithm=3, nt=6000, ndms=3, seed=19, nh=4, scalloping=1),
    "presto_h32": dict(algorithm=3, nt=8192, ndms=3, seed=20, nh=32, scalloping=0),
}


def make_hs_algo_input(c):
    """(plane [ndms][nt] float32 power with harmonic combs, msd [64] float32)."""
    x = make_power_plane(dict(nt=c["nt"], ndms=c["ndms"], seed=c["seed"]))
    f = np.arange(32, dtype=np.float32)
    msd = np.empty(64, np.float32)
    msd[0::2] = f + 1
    msd[1::2] = np.sqrt(f + 1)
    return x, msd


# Spectral whitening (SGP2 with medians) on red-noise spectra of n complex
# bins: the periodicity search's nT/2 + 1 bins, an odd and an even size
WHITENING_CASES = {
    "white_4097x8": dict(n=4097, ndms=8, seed=21),
    "white_65537x3": dict(n=65537, ndms=3, seed=22),
    "white_16384x4": dict(n=16384, ndms=4, seed=23),
    "white_1000x5": dict(n=1000, ndms=5, seed=24),
}

# Whitening cases whose last segment is 1 bin (n = a boundary + 1) and 2 bins
# (a boundary + 2): median and interpolation branches the cases above never
# take.  No reference golden run covers them (for a 2-bin segment the
# reference's median kernel reads one slot past its shared array); the
# oracle pins them.
WHITENING_EDGE_CASES = {
    "white_3968x3_last1": dict(n=3968, ndms=3, seed=25),
    "white_8954x2_last2": dict(n=8954, ndms=2, seed=26),
}

# Segment lengths for the medians alone, around every register-width switch
# of the median kernel (32, 64, 128 bins) and at both ends (1 and 256 bins).
MEDIAN_SEGMENT_LENGTHS = [1, 2, 3, 4, 5, 31, 32, 33, 63, 64, 65, 127, 128, 129, 130, 200, 255, 256, 6, 250, 17, 1, 2]


def make_red_spectra(c) -> np.ndarray:
    """[ndms][n] complex64: complex Gaussian bins whose power falls as a red
    spectrum 1 + 300 / (1 + k / 20)^2 over a floor of n, with a few lines."""
    rng = np.random.Generator(np.random.PCG64(c["seed"]))
    k = np.arange(c["n"], dtype=np.float64)
    amp = np.sqrt(c["n"] * (1.0 + 300.0 / (1.0 + k / 20.0) ** 2) / 2.0)
    z = (rng.normal(0, 1, (c["ndms"], c["n"])) + 1j * rng.normal(0, 1, (c["ndms"], c["n"]))) * amp
    for d in range(c["ndms"]):
        f = int(rng.integers(30, c["n"] // 10))
        for h in range(1, 5):
            if h * f < c["n"]:
                z[d, h * f] += 10.0 * np.sqrt(c["n"]) / h
    return np.ascontiguousarray(z.astype(np.complex64))


def shared_bins(seg):
    """Bins the reference's whitening scales in two neighbouring blocks:
    where an even segment is followed by an odd one (not the last pair),
    the middle of the odd one."""
    out = []
    for b in range(1, len(seg) - 2):
        pr, cr = seg[b] - seg[b - 1], seg[b + 1] - seg[b]
        if pr % 2 == 0 and cr % 2 == 1:
            out.append(seg[b] + (cr >> 1))
    return out


def stale_bins(seg):
    """Bins from the middle of the last segment to the end: the reference's
    whitening launches one block past its segments, which reads the boundary
    after its table (device memory it never wrote) and, when that word holds
    a boundary a little past the end, scales these bins a second time."""
    return list(range(seg[-2] + ((seg[-1] - seg[-2]) >> 1), seg[-1]))


# Periodicity candidate records (DM trial, bin, power, harmonic count) as the
# peak finding writes them, converted by the host lists: power lists (mod 1),
# interbin lists (mod 2), greedy lists (bin offsets in the hundreds)
CANDIDATE_CASES = {
    "cands_power": dict(n=3000, ndms=512, nt=1 << 20, nh=32, mod=1.0, greedy=0, dm_low=0.0, dm_step=0.1,
                        tsamp=6.4e-5, seed=31),
    "cands_interbin": dict(n=2500, ndms=1024, nt=1 << 18, nh=16, mod=2.0, greedy=0, dm_low=150.0, dm_step=0.25,
                           tsamp=1.28e-4, seed=32),
    "cands_greedy": dict(n=4000, ndms=300, nt=(1 << 19) + 3, nh=8, mod=1.0, greedy=1, dm_low=12.5, dm_step=0.05,
                         tsamp=6.5536e-5, seed=33),
    "cands_greedy_interbin": dict(n=1500, ndms=77, nt=1 << 16, nh=32, mod=2.0, greedy=1, dm_low=1000.0,
                                  dm_step=3.0, tsamp=2.56e-4, seed=34),
}


def make_candidate_records(c):
    """(records [n][4] float32, msd [2*nh] float32)."""
    rng = np.random.Generator(np.random.PCG64(c["seed"]))
    n = c["n"]
    rec = np.empty((n, 4), np.float32)
    rec[:, 0] = rng.integers(0, c["ndms"], n)
    rec[:, 1] = rng.integers(1, c["nt"] // 2 * (2 if c["mod"] == 2.0 else 1), n)
    rec[:, 2] = rng.uniform(5.0, 200.0, n).astype(np.float32)
    h = rng.integers(0, c["nh"], n)
    if c["greedy"]:
        h = h + 100 * rng.integers(0, 4, n)
    rec[:, 3] = h
    f = np.arange(c["nh"], dtype=np.float32)
    msd = np.empty(2 * c["nh"], np.float32)
    msd[0::2] = np.float32(1.7) * (f + 1)
    msd[1::2] = np.sqrt(f + 1) * np.float32(1.3)
    return np.ascontiguousarray(rec), msd
