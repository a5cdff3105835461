"""Runs of the reference's optional input/output processing
(include/aa_permitted_pipelines_generic.hpp:525-560, :704-760, :821-831) on
seeded cases of cases.py: name -> (case name, option bits, bandpass).

Option bits as oracle/ref_harness.cu aaref_run_ddtr_opts: 1 zero_dm, 2
zero_dm_with_outliers, 4 input_DDTR_normalization, 8
output_DDTR_normalization, 16 old_rfi, 32 set_bandpass_average."""
from __future__ import annotations

import numpy as np

ZDM, ZDM_OUT, IN_NORM, OUT_NORM, OLD_RFI, BP_AVG = 1, 2, 4, 8, 16, 32


def custom_bandpass(nchans, seed=21):
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.uniform(100.0, 150.0, nchans).astype(np.float32)


RUNS = {
    "s8_zdm": ("shared8_binned", ZDM, None),
    "s8_zdm_outliers": ("shared8_binned", ZDM_OUT, None),
    "s8_in_norm": ("shared8_binned", IN_NORM, None),
    "s8_out_norm": ("shared8_binned", OUT_NORM, None),
    "s8_old_rfi": ("shared8_binned", OLD_RFI, None),
    "s8_zdm_bp_average": ("shared8_binned", ZDM | BP_AVG, None),
    "s8_zdm_custom_bp": ("shared8_binned", ZDM, "custom"),
    "s8_all": ("shared8_binned", ZDM | IN_NORM | OUT_NORM | OLD_RFI, None),
    "s8_chunked_zdm_in_norm": ("shared8_chunked", ZDM | IN_NORM, None),
    "s8_chunked_out_norm_rfi": ("shared8_chunked", OUT_NORM | OLD_RFI, None),
    "s4_zdm": ("shared4", ZDM, None),
    "s4_zdm_outliers": ("shared4", ZDM_OUT, None),
    "s4_in_norm": ("shared4", IN_NORM, None),
    "s16_zdm": ("shared16", ZDM, None),
    "s16_zdm_outliers": ("shared16", ZDM_OUT, None),
    "s16_in_norm_out_norm": ("shared16", IN_NORM | OUT_NORM, None),
    "s16_old_rfi": ("shared16", OLD_RFI, None),
    "c8_zdm_out_norm": ("cache8", ZDM | OUT_NORM, None),
}
