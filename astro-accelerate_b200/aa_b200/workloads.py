"""Seeded synthetic workloads for the multi-beam configuration.

There is no public dataset for this path; the multi-beam benchmark draws its
beams from a seed:

  * channels uniform in 2048..4096, over the survey band (fch1 1670 MHz,
    300 MHz wide, so foff = -300/nchans MHz), tsamp 64 us;
  * bit depth uniform in {4, 8, 16};
  * length log-uniform in 2^16..2^21 samples;
  * a DM plan made of the first 2-6 ranges (uniform) of the survey plan
    (0-150/0.1/1 ... 2000-3000/2.0/8), truncated at a maximum DM uniform in
    500..3000 (ranges starting above it are dropped, the last one is cut);
  * noise N(mid-scale, range/16) clipped to the integer range of the depth.
"""
from __future__ import annotations

import numpy as np

SURVEY_PLAN = [(0, 150, 0.1, 1, 1), (150, 300, 0.2, 1, 1), (300, 500, 0.25, 1, 1), (500, 900, 0.4, 2, 1),
               (900, 1200, 0.6, 4, 1), (1200, 1500, 0.8, 4, 1), (1500, 2000, 1.0, 4, 1), (2000, 3000, 2.0, 8, 1)]


def multibeam_draw(seed: int = 3, nbeams: int = 48) -> list:
    """Beam descriptions (dicts with nchans, nbits, nsamp, fch1, foff, tsamp,
    plan, seed)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    beams = []
    for b in range(nbeams):
        nch = int(rng.integers(2048, 4097))
        nbits = int(rng.choice([4, 8, 16]))
        nsamp = int(round(2 ** rng.uniform(16, 21)))
        maxdm = float(rng.uniform(500, 3000))
        nr = int(rng.integers(2, 7))
        plan = [list(p) for p in SURVEY_PLAN[:nr] if p[0] < maxdm]
        plan[-1][1] = min(plan[-1][1], maxdm)
        beams.append(dict(nchans=nch, nbits=nbits, nsamp=nsamp, fch1=1670.0, foff=-300.0 / nch, tsamp=64e-6,
                          plan=[tuple(p) for p in plan], seed=seed * 1000 + b))
    return beams


def synth_beam_device(beam: dict, device):
    """[nsamp][nchans] samples as a uint16 bit pattern in an int16 CUDA tensor:
    N(mid, range/16) clipped to [0, 2^nbits - 1]."""
    import torch
    vmax = (1 << min(beam["nbits"], 16)) - 1
    mid, sig = (vmax + 1) / 2.0 - 0.5, (vmax + 1) / 16.0
    g = torch.Generator(device=device)
    g.manual_seed(beam["seed"])
    x = torch.empty((beam["nsamp"], beam["nchans"]), dtype=torch.int16, device=device)
    rows = max(1, (1 << 28) // (4 * beam["nchans"]))
    for t0 in range(0, beam["nsamp"], rows):
        n = min(rows, beam["nsamp"] - t0)
        v = torch.randn((n, beam["nchans"]), generator=g, device=device) * sig + mid
        x[t0:t0 + n] = v.round_().clamp_(0, vmax).to(torch.int32).to(torch.int16)
    return x


def plan_waves(sizes: list, budget: int) -> list:
    """Greedy split of beams (in order) into groups whose byte sizes fit the
    budget; a beam larger than the budget gets a group of its own."""
    waves, cur, used = [], [], 0
    for i, s in enumerate(sizes):
        if cur and used + s > budget:
            waves.append(cur)
            cur, used = [], 0
        cur.append(i)
        used += s
    if cur:
        waves.append(cur)
    return waves

