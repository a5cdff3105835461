"""Seeded DM-time outputs for the output_dmt writer tests."""
from __future__ import annotations

import numpy as np

NDMS = [64, 128, 32]
IN_BIN = [1, 2, 4]
MAX_NT = 1000

# name -> (DMs per file, ranges to export)
CASES = {
    "per48_all": (48, [1, 1, 1]),
    "whole_from_range1": (-1, [0, 1, 1]),
    "per5_range0": (5, [1, 0, 0]),
    "per262_all": (262, [1, 1, 1]),
}


def rows(seed: int = 11):
    """rows[r]: [NDMS[r]][MAX_NT/IN_BIN[r] + 7] float32 (longer than exported)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return [rng.normal(0.0, 1.0, (n, MAX_NT // b + 7)).astype(np.float32) for n, b in zip(NDMS, IN_BIN)]


def as_float3(rs):
    """float*** view of rows (ctypes), with the arrays kept alive."""
    import ctypes
    PF = ctypes.POINTER(ctypes.c_float)
    row_ptrs = [(PF * r.shape[0])(*[r[d].ctypes.data_as(PF) for d in range(r.shape[0])]) for r in rs]
    top = (ctypes.POINTER(PF) * len(rs))(*[ctypes.cast(p, ctypes.POINTER(PF)) for p in row_ptrs])
    return top, (rs, row_ptrs)
