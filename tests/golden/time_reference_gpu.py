"""Times the reference's own GPU pipeline (AstroAccelerate v1.3.1 built from
its sources by oracle/Makefile.ref) on the survey-scale configuration of
bench.py: 4096 channels x 2^21 samples, 8-bit, the 8-range plan, seeded
Gaussian noise plus 8 dispersed pulses.  Needs a GPU; prints one JSON line.

    python tests/golden/time_reference_gpu.py [--copy-to-host] [--config mid|survey]

The survey configuration is refused: its 4096 x 1 048 544-element chunks
overflow the reference kernels' 32-bit indices (an illegal memory access when
it was run); the reduced configuration (2^18 samples) stays below 2^31.

The data are generated on the GPU with bench.py's generator, copied to host
memory (the reference takes a host [t][c] unsigned short buffer), and the
runner's run(status) loop is timed with the wall clock after setup.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--copy-to-host", action="store_true")
    ap.add_argument("--config", default="mid", choices=["survey", "mid"])
    ap.add_argument("--analysis", action="store_true",
                    help="with the analysis component (bench.py's ANALYSIS settings); candidate files go to a "
                         "scratch directory")
    args = ap.parse_args()
    import torch
    import bench
    import refharness as R
    cfg = bench.SURVEY if args.config == "survey" else bench.MID
    x, _ = bench.synth_input_device(cfg, cfg["seed"], torch.device("cuda", 0))
    host = x.cpu().numpy().view(np.uint16)
    del x
    torch.cuda.empty_cache()
    L = R.load()
    L.aaref_time_ddtr.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_int, ctypes.POINTER(R.DM), ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    L.aaref_time_ddtr.restype = ctypes.c_int
    sec, nt = ctypes.c_double(), ctypes.c_int()
    if args.analysis:
        import tempfile
        a = bench.ANALYSIS
        L.aaref_time_pipeline_spd.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.POINTER(R.DM),
                                              ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                              ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_longlong)]
        L.aaref_time_pipeline_spd.restype = ctypes.c_int
        nc = ctypes.c_longlong()
        here = os.getcwd()
        os.chdir(tempfile.mkdtemp(prefix="spdtime_"))
        try:
            rc = L.aaref_time_pipeline_spd(host.ctypes.data, cfg["nchans"], cfg["nsamp"], cfg["tsamp"], cfg["fch1"],
                                           cfg["foff"], cfg["nbits"], R._plan(cfg["plan"]), len(cfg["plan"]),
                                           int(args.copy_to_host), a["sigma_cutoff"], a["sigma_constant"],
                                           a["max_width_s"], a["algorithm"], a["baseline_noise"],
                                           ctypes.byref(sec), ctypes.byref(nt), ctypes.byref(nc))
        finally:
            os.chdir(here)
        if rc != 0:
            raise SystemExit(f"reference run failed ({rc})")
        import aa_b200 as aa
        s = aa.strategy(cfg["plan"], cfg["nchans"], cfg["nsamp"], cfg["fch1"], cfg["foff"], cfg["tsamp"],
                        cfg["nbits"])
        units = sum(s["ndms"][r] * sum(s["t_processed"][r]) for r in range(len(s["ndms"])))
        print(json.dumps({"impl": "reference-gpu", "config": args.config, "analysis": a,
                          "copy_to_host": args.copy_to_host, "seconds": sec.value, "num_tchunks": nt.value,
                          "candidates": nc.value, "units": units, "dm_trial_samples_per_s": units / sec.value}),
              flush=True)
        return
    rc = L.aaref_time_ddtr(host.ctypes.data, cfg["nchans"], cfg["nsamp"], cfg["tsamp"], cfg["fch1"], cfg["foff"],
                           cfg["nbits"], R._plan(cfg["plan"]), len(cfg["plan"]), int(args.copy_to_host),
                           ctypes.byref(sec), ctypes.byref(nt))
    if rc == -4:
        raise SystemExit("refused: a chunk exceeds 2^31 elements, where the reference's 32-bit kernel indices "
                         "overflow (src/aa_device_dedispersion_kernel.cu:194,214)")
    if rc != 0:
        raise SystemExit(f"reference run failed ({rc})")
    import aa_b200 as aa  # planner only (host), for the unit count
    s = aa.strategy(cfg["plan"], cfg["nchans"], cfg["nsamp"], cfg["fch1"], cfg["foff"], cfg["tsamp"], cfg["nbits"])
    units = sum(s["ndms"][r] * sum(s["t_processed"][r]) for r in range(len(s["ndms"])))
    print(json.dumps({"impl": "reference-gpu", "config": args.config, "copy_to_host": args.copy_to_host,
                      "seconds": sec.value, "num_tchunks": nt.value, "units": units,
                      "dm_trial_samples_per_s": units / sec.value,
                      "realtime_x": sum(s["t_processed"][0]) * cfg["tsamp"] / sec.value}), flush=True)


if __name__ == "__main__":
    main()
