"""The C-ABI library loads and exports every entry point include/aa_b200.h
declares; the host-side logic behind it works without a GPU."""
from __future__ import annotations

import ctypes
import subprocess

import numpy as np
import pytest


def test_library_exports_every_declared_symbol(aa):
    L = aa.lib()
    names = aa.declared_symbols()
    assert len(names) >= 45
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", aa.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(names) <= exported


def test_library_build_targets_sm100a():
    """The library's device code is compiled for sm_100a only."""
    import os
    mk = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "astro-accelerate_b200",
                           "Makefile")).read()
    gencode = [ln for ln in mk.splitlines() if ln.startswith("GENCODE")]
    assert gencode == ["GENCODE   := -gencode arch=compute_100a,code=sm_100a"]


@pytest.mark.gpu
def test_library_runs_sm100_code(aa, cuda_device):
    """The CUDA runtime reports the library's kernels as sm_100 binaries."""
    v = ctypes.c_int()
    assert aa.lib().aa_b200_binary_version(ctypes.byref(v)) == 0
    assert v.value == 100


def test_plan_objects_roundtrip(aa):
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(0, 150, 0.1, 1, 1), aa.aa_py_dm(150, 300, 0.2, 1, 1)])
    assert plan.range() == 2
    assert plan.power() == 2.0
    assert plan.set_power(2.1) and abs(plan.power() - 2.1) < 1e-6
    assert plan.set_enable_msd_baseline_noise(True) and plan.enable_msd_baseline_noise()
    assert plan.bind_bandpass_normalization(np.ones(8, np.float32), 8)
    plan.delete()
    md = aa.aa_py_filterbank_metadata(50000.0, 64e-6, 8, 1024, 1550.0, -0.39, 1024)
    assert md.tstart() == 50000.0


def test_out_of_scope_components_are_refused(aa):
    md = aa.filterbank_metadata_struct(0.0, 64e-6, 1550.0, -0.39, 8, 1 << 16, 256, 0.0)
    # FDAS is out of scope (dedispersion, analysis and periodicity are implemented)
    comps = aa.aa_py_pipeline_components(True, False, False, True)
    opts = aa.aa_py_pipeline_component_options()
    x = np.zeros(256 * (1 << 16), np.uint16)
    p = aa.aa_py_pipeline(comps, opts, md, x, 0)
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(0, 100, 1, 1, 1)])
    assert not p.bind_ddtr_plan(plan)
    assert "periodicity" in p.last_error()
    assert not p.run() and p.status_code() == aa.STATUS_ERROR
    assert not p.bind_fdas_plan(None)
    p.delete()
    plan.delete()


def test_periodicity_plan_needs_its_component_and_a_ddtr_plan(aa):
    """Host-side refusals (no GPU call): a periodicity plan on a pipeline
    without the periodicity component, or before the DDTR plan is bound."""
    md = aa.filterbank_metadata_struct(0.0, 64e-6, 1550.0, -0.39, 8, 1 << 16, 256, 0.0)
    x = np.zeros(256 * (1 << 16), np.uint16)
    pp = aa.aa_py_periodicity_plan(6.0, 3.0, 32, 0, 0, True)
    for comps, needle in ((aa.aa_py_pipeline_components(True, False, False, False), "periodicity component"),
                          (aa.aa_py_pipeline_components(True, False, True, False), "DDTR plan")):
        p = aa.aa_py_pipeline(comps, aa.aa_py_pipeline_component_options(), md, x, 0)
        assert not p.bind_periodicity_plan(pp)
        assert needle in p.last_error(), p.last_error()
        assert aa.lib().aa_b200_pipeline_psr_count(p.m_obj, 0) == 0
        p.delete()


def test_setup_needs_a_bound_plan(aa):
    """Explicit set-up before a DDTR plan is bound is refused with a message
    (host only: no device call is made)."""
    md = aa.filterbank_metadata_struct(0.0, 64e-6, 1550.0, -0.39, 8, 1 << 16, 256, 0.0)
    p = aa.aa_py_pipeline(aa.aa_py_pipeline_components(True, False, False, False),
                          aa.aa_py_pipeline_component_options(), md, np.zeros(256 * (1 << 16), np.uint16), 0)
    assert not p.setup()
    assert "no DDTR plan bound" in p.last_error()
    p.delete()


def test_strategy_refusal_codes(aa):
    import pytest
    with pytest.raises(ValueError):
        aa.strategy([(0, 3000, 1.0, 1, 1)], 4096, 1 << 12, 1670.0, -0.0732421875, 64e-6, 8)  # maxshift >= nsamp
    with pytest.raises(ValueError):
        aa.strategy([], 4096, 1 << 20, 1670.0, -0.0732421875, 64e-6, 8)


def test_tuned_range_store_is_host_only(aa):
    """The autotuner's kept choices can be counted and dropped without a GPU."""
    assert aa.tuned_ranges(clear=True) == 0
    assert aa.tuned_ranges() == 0


def test_tuned_range_file_roundtrip(aa, tmp_path):
    """The autotuner's kept choices go to a text file and back (host only):
    an entry read from a file is written out unchanged; a file that is not
    one, or a malformed entry, is refused."""
    aa.tuned_ranges(clear=True)
    line = "3 0 4096 8 2 16 1072 1096 4 37 1028 120304 7 0"
    src = tmp_path / "in.txt"
    src.write_text("aa_b200 tuned ranges 1\n" + line + "\n")
    assert aa.load_tuned_ranges(str(src)) == 1
    assert aa.tuned_ranges() == 1
    out = tmp_path / "out.txt"
    assert aa.save_tuned_ranges(str(out)) == 1
    assert out.read_text().splitlines() == ["aa_b200 tuned ranges 1", line]
    bad = tmp_path / "bad.txt"
    bad.write_text("something else\n")
    with pytest.raises(OSError, match="not a tuned-range file"):
        aa.load_tuned_ranges(str(bad))
    bad.write_text("aa_b200 tuned ranges 1\n3 0 1\n")
    with pytest.raises(OSError, match="malformed"):
        aa.load_tuned_ranges(str(bad))
    with pytest.raises(OSError, match="cannot open"):
        aa.load_tuned_ranges(str(tmp_path / "missing.txt"))
    assert aa.tuned_ranges(clear=True) == 0
    assert aa.tuned_ranges_used() == 0  # no pipeline has been set up here


def test_batch_kernel_choice_is_checked(aa):
    """The batch's kernel choice takes 0, 1 or 2 before setup (host only)."""
    b = aa.batch()
    try:
        with pytest.raises(RuntimeError, match="kernel choice"):
            b.set_kernel_choice(3)
        assert b.set_kernel_choice(2) and b.set_kernel_choice(0)
        assert b.sub_jobs() == 0
    finally:
        b.delete()


def test_failure_injection_counter(aa):
    """aa_b200_debug_fail_after arms a host-side countdown (no GPU needed to set it)."""
    L = aa.lib()
    L.aa_b200_debug_fail_after(7)
    assert L.aa_b200_debug_fail_countdown() == 7
    L.aa_b200_debug_fail_after(-1)
    assert L.aa_b200_debug_fail_countdown() == 0
