"""CPU restatement of the reference's DM-time export (AstroAccelerate v1.3.1,
include/aa_pipeline_runner.hpp:165-223, Export_DD_data and
Calculate_sd_per_file_from_file_size), in numpy.

TEST INFRASTRUCTURE ONLY: used by tests/ to check the library's output_dmt
writer; nothing in the product imports it.  Pinned against the reference's
own routine (oracle/ref_harness.cu aaref_export_dd_data) through
tests/golden/dmt_golden.json.
"""
from __future__ import annotations

import numpy as np


def sd_per_file(size_in_mb: int, primary_dimension: int, floats_per_element: int) -> int:
    """:219-223"""
    return ((size_in_mb * 1024 * 1024) // 4 * floats_per_element) // primary_dimension


def export(rows, max_nt: int, ndms, in_bin, base: str, ranges_to_export, dms_per_file: int) -> list:
    """:165-216.  rows[r]: [ndms[r]][>= max_nt/inBin[r]] float32.  Returns the
    paths written, in order."""
    written = []
    for r in range(len(rows)):
        if not ranges_to_export[r]:
            continue
        nt = max_nt // in_bin[r]
        ndm = ndms[r]
        if dms_per_file < 0:
            dms_per_file = ndm          # the parameter itself changes, for later ranges too
        runs = [dms_per_file] * (ndm // dms_per_file)
        if ndm % dms_per_file:
            runs.append(ndm % dms_per_file)
        txt = f"{base}_{r}.txt"
        with open(txt, "w") as f:
            f.write(f"{nt}\n{ndm}\n{dms_per_file}\n{len(runs)}\n")
        written.append(txt)
        d0 = 0
        for i, n in enumerate(runs):
            dat = f"{base}_{r}_{i}.dat"
            np.ascontiguousarray(np.asarray(rows[r], dtype=np.float32)[d0:d0 + n, :nt]).tofile(dat)
            written.append(dat)
            d0 += n
    return written
