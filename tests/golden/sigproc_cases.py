"""Seeded SIGPROC filterbank files for the reader and packed-input tests:
every bit depth the reference's reader handles, header keywords it skips, a
partial record at the end of the data, NaN samples in a 32-bit file."""
from __future__ import annotations

import numpy as np

CASES = {
    "u8_256": dict(nbits=8, nchans=256, nsamp=1000, seed=1),
    "u4_512": dict(nbits=4, nchans=512, nsamp=777, seed=2),
    "u2_256": dict(nbits=2, nchans=256, nsamp=513, seed=3),
    "u1_1024": dict(nbits=1, nchans=1024, nsamp=300, seed=4),
    "u16_128": dict(nbits=16, nchans=128, nsamp=999, seed=5),
    "f32_64": dict(nbits=32, nchans=64, nsamp=400, seed=6),
    "f32_nan": dict(nbits=32, nchans=64, nsamp=100, seed=7, nan=True),
    "u8_extra_keywords": dict(nbits=8, nchans=64, nsamp=100, seed=8, source_name="J0534+2200",
                              extra_ints={"ibeam": 1}),
    "u8_partial_record": dict(nbits=8, nchans=64, nsamp=100, seed=9, trailing=37),
    "u16_partial_record": dict(nbits=16, nchans=32, nsamp=64, seed=10, trailing=3),
}


def make_data(case) -> np.ndarray:
    """[nsamp][nchans] samples: uniform over the bit depth's range (float32
    N(100, 15) for 32-bit)."""
    rng = np.random.Generator(np.random.PCG64(case["seed"]))
    n, c, nb = case["nsamp"], case["nchans"], case["nbits"]
    if nb == 32:
        x = rng.normal(100.0, 15.0, (n, c)).astype(np.float32)
        if case.get("nan"):
            x.reshape(-1)[rng.choice(n * c, 17, replace=False)] = np.nan
        return x
    return rng.integers(0, 1 << nb, (n, c), dtype=np.uint32).astype(np.uint16)


def write_case(case, path, writer) -> None:
    """writer: aa_b200.sigproc.write_filterbank."""
    data = make_data(case)
    writer(path, data, case["nbits"], tsamp=64e-6 * (1 + case["seed"] % 3), fch1=1400.0 + case["seed"],
           foff=-0.5 / (1 + case["seed"] % 4), tstart=58000.5 + case["seed"], source_name=case.get("source_name"),
           extra_ints=case.get("extra_ints"))
    if case.get("trailing"):
        rng = np.random.Generator(np.random.PCG64(1000 + case["seed"]))
        with open(path, "ab") as f:
            f.write(rng.integers(0, 256, case["trailing"], dtype=np.uint8).tobytes())
