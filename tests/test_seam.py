"""The reference's own dedispersion seam (namespace astroaccelerate:
load_chunk_data, corner_turn_SM_inplace, bin_gpu, set_dedispersion_constants,
dedisperse, save_data_offset_stream) as libaa_b200.so exports it.

A caller written against the reference's declarations (tests/seam_caller.cpp,
which follows the reference runner's DDTR loop) compiles against
include/aa_b200_seam.hpp and links with the library alone; on the GPU its
output equals the oracle's for every DM range, chunk and binning step."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import cases as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "astro-accelerate_b200", "aa_b200")
CUDA = "/usr/local/cuda"

# the reference's declarations (include/aa_dedisperse.hpp:20,
# include/aa_device_load_data.hpp:15-17, include/aa_corner_turn.hpp:28,
# include/aa_bin_gpu.hpp:17, include/aa_device_save_data.hpp:12), demangled
REFERENCE_SEAM = [
    "astroaccelerate::dedisperse(int, int, int*, float*, unsigned short*, float*, float*, int, float*, float*, "
    "float*, int const*, int, int)",
    "astroaccelerate::load_chunk_data(unsigned short*, unsigned short const*, int, int, int, float*, float*, int)",
    "astroaccelerate::set_dedispersion_constants(int, int)",
    "astroaccelerate::corner_turn_SM_inplace(unsigned short*, unsigned short*, unsigned long, unsigned long)",
    "astroaccelerate::bin_gpu(unsigned short*, float*, int, int)",
    "astroaccelerate::save_data_offset_stream(int, int, int**, long, int*, int const*, float*, float***)",
]


def build_caller(aa, out_dir):
    exe = os.path.join(out_dir, "seam_caller")
    cmd = ["g++", "-std=c++17", "-O1", os.path.join(ROOT, "tests", "seam_caller.cpp"), "-I",
           os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"), "-L", LIBDIR, "-laa_b200",
           f"-Wl,-rpath,{LIBDIR}", "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-o", exe]
    subprocess.check_call(cmd)
    return exe


def test_library_exports_the_reference_seam(aa):
    out = subprocess.run(["nm", "-DC", "--defined-only", aa.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split(" ", 2)[2] for line in out.splitlines() if " T " in line}
    missing = [s for s in REFERENCE_SEAM if s not in exported]
    assert not missing, missing


def test_reference_style_caller_links_unchanged(aa, tmp_path):
    exe = build_caller(aa, str(tmp_path))
    assert os.path.exists(exe)


def write_plan(path, case, s):
    with open(path, "w") as f:
        f.write(f"{case['nchans']} {case['nsamp']} {case['nbits']} {case['tsamp']!r} {s.maxshift} {len(s.ndms)} "
                f"{s.num_tchunks}\n")
        for r, d in enumerate(s.dm):
            f.write(f"{float(np.float32(d[0]))!r} {float(np.float32(d[2]))!r} {d[3]} {s.ndms[r]}\n")
        for r in range(len(s.ndms)):
            f.write(" ".join(str(v) for v in s.t_processed[r]) + "\n")
        f.write(" ".join(repr(float(v)) for v in s.dmshifts) + "\n")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["shared8_binned", "shared8_chunked", "shared16", "shared4", "cache16"])
def test_reference_style_caller_matches_oracle(aa, oracle_mod, cuda_device, tmp_path, name):
    case = C.CASES[name]
    x = C.make_input(case)
    s = oracle_mod.strategy(case["plan"], case["nchans"], case["nsamp"], case["fch1"], case["foff"], case["tsamp"],
                            case["nbits"], C.strategy_free_memory(case))
    want, _ = oracle_mod.run_ddtr(x, s, case["nchans"], case["nsamp"], case["tsamp"], case["nbits"])
    plan, inp, outp = (str(tmp_path / n) for n in ("plan.txt", "input.bin", "output.bin"))
    write_plan(plan, case, s)
    np.ascontiguousarray(x, dtype=np.uint16).tofile(inp)
    exe = build_caller(aa, str(tmp_path))
    r = subprocess.run([exe, plan, inp, outp], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr, aa.last_error())
    got = np.fromfile(outp, np.float32)
    off = 0
    for rr, w in enumerate(want):
        g = got[off:off + w.size].reshape(w.shape)
        off += w.size
        div = case["nchans"] * (1 if case["nbits"] == 4 else s.dm[rr][3])
        if div & (div - 1) == 0:
            bad = np.flatnonzero(g.view(np.uint32) != w.view(np.uint32))
            assert bad.size == 0, f"range {rr}: {bad.size} outputs differ"
        else:
            ulp = np.abs(g.view(np.int32).astype(np.int64) - w.view(np.int32).astype(np.int64))
            assert ulp.max() <= 2, f"range {rr}: {ulp.max()} ulp"
    assert off == got.size
