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



# End-to-end search workload: 16 beams of 4096 channels, 8-bit, 2^20 samples,
# the survey band and plan, 4-32 dispersed boxcar pulses per beam (DM U[50,
# 2900], width log-U[0.25, 8] ms, 3-10 sigma per channel, cold-plasma delay
# 4.148808e3 DM (f^-2 - fch1^-2) s), placed so that every sweep ends inside
# the beam.
def e2e_beams(seed: int = 5, nbeams: int = 16, nsamp: int = 1 << 20) -> list:
    rng = np.random.Generator(np.random.PCG64(seed))
    beams = []
    nch, fch1, foff, tsamp = 4096, 1670.0, -0.0732421875, 64e-6
    f = fch1 + foff * np.arange(nch, dtype=np.float64)
    kc = 4.148808e3 * (f ** -2 - fch1 ** -2) / tsamp
    for b in range(nbeams):
        pulses = []
        for _ in range(int(rng.integers(4, 33))):
            dm = float(rng.uniform(50, 2900))
            width = max(1, int(round(np.exp(rng.uniform(np.log(0.25), np.log(8.0))) * 1e-3 / tsamp)))
            amp = float(rng.uniform(3, 10))
            sweep = int(np.ceil(dm * kc[-1])) + width
            start = int(rng.integers(0, nsamp - sweep))
            pulses.append(dict(dm=dm, width=width, amp_sigma=amp, start=start))
        beams.append(dict(nchans=nch, nbits=8, nsamp=nsamp, fch1=fch1, foff=foff, tsamp=tsamp, plan=list(SURVEY_PLAN),
                          seed=seed * 1000 + b, pulses=pulses))
    return beams


def synth_e2e_beam(beam: dict, device):
    """The beam's noise (synth_beam_device) plus its pulses."""
    import torch
    x = synth_beam_device(beam, device)
    nch = beam["nchans"]
    f = beam["fch1"] + beam["foff"] * np.arange(nch, dtype=np.float64)
    sig = 16.0
    c = torch.arange(nch, device=device)
    for p in beam["pulses"]:
        d = torch.as_tensor(np.floor(4.148808e3 * p["dm"] * (f ** -2 - beam["fch1"] ** -2) / beam["tsamp"]),
                            dtype=torch.int64, device=device)
        for k in range(p["width"]):
            tt = p["start"] + d + k
            v = (x[tt, c].to(torch.int32) & 0xFFFF).to(torch.float32) + p["amp_sigma"] * sig
            x[tt, c] = v.clamp_(0, 255).to(torch.int32).to(torch.int16)
    return x


def partition(costs: list, nranks: int) -> list:
    """Beams to ranks, heaviest first onto the least loaded rank (longest
    processing time first); returns one list of beam indices per rank, each in
    ascending order.  Beams are independent, so no data moves between ranks."""
    loads = [0.0] * nranks
    parts = [[] for _ in range(nranks)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(nranks), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += costs[i]
    return [sorted(p) for p in parts]


def beam_cost(beam: dict, strategy: dict) -> float:
    """Channel-adds of one beam's dedispersion (fp32 work counted 3x)."""
    units = sum(strategy["ndms"][r] * sum(strategy["t_processed"][r]) for r in range(len(strategy["ndms"])))
    return float(units) * beam["nchans"] * (3.0 if beam["nbits"] > 8 else 1.0)
