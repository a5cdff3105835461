"""Single-pulse detection host logic without a GPU: the plan against the
oracle's restatement and the reference's golden runs, the candidate file,
and the analysis plan's refusals through the pipeline C ABI."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import spd_cases as S
import spd_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "spd_golden.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)["runs"]


@pytest.mark.parametrize("name", list(S.CASES))
def test_oracle_plan_matches_reference_runs(golden, name):
    """The restated plan gives the widths, widest width and iterations the
    reference reported on its own GPU run."""
    c = S.CASES[name]
    g = golden[name]
    p = O.plan(c["nt"], np.float32(c["tsamp"] * c["inbin"]), c["inbin"], c["max_width_s"])
    assert p["widths"] == g["widths"]
    assert p["max_width_performed"] == g["max_width_performed"]
    assert p["max_iteration"] == g["max_iteration"]


@pytest.mark.parametrize("nt", [128, 777, 4096, 16384, 65536, 262143, 1 << 20])
@pytest.mark.parametrize("tsamp,in_bin,width", [(64e-6, 1, 0.004), (128e-6, 2, 0.02), (64e-6, 1, 0.5),
                                                (256e-6, 4, 0.001), (64e-6, 8, 1.0)])
def test_library_plan_matches_oracle(aa, nt, tsamp, in_bin, width):
    ts = float(np.float32(tsamp * in_bin))
    got = aa.spd_plan(nt, ts, in_bin, width)
    want = O.plan(nt, np.float32(ts), in_bin, width)
    assert got == want


@pytest.mark.parametrize("name", list(S.CASES))
def test_golden_candidates_are_consistent(golden, name):
    """Candidates of the reference's run: above the cut, inside the plane,
    with a width of the plan; peak finding keeps fewer than thresholding."""
    c = S.CASES[name]
    g = golden[name]
    assert g["ncands"] > 0
    mwp = g["max_width_performed"]
    for dm, ts, snr_bits, bw in g["cands_head"]:
        snr = np.array([snr_bits], np.uint32).view(np.float32)[0]
        assert snr > c["cutoff"]
        assert 0 <= dm < c["ndms"]
        assert 0 <= ts < c["nt"]
        assert 1 <= bw <= mwp
        if c["algorithm"] == 1:
            assert dm < (c["ndms"] // 4) * 4 or not S.single_batch(c)


def test_candidate_file(aa, tmp_path):
    dm = np.array([0, 3, 17], np.uint32)
    ts = np.array([5, 1000, 65535], np.uint32)
    snr = np.array([6.5, 7.25, 12.0], np.float32)
    bw = np.array([1, 32, 96], np.uint32)
    aa.write_candidates(str(tmp_path), 0, 1.5, 10.0, 16.4, 0.1, np.float32(64e-6 * 2), 2,
                        {"dm": dm, "ts": ts, "snr": snr, "bw": bw})
    aa.write_candidates(str(tmp_path), 1, 0.0, 0.0, 6.4, 0.1, np.float32(64e-6), 1,
                        {"dm": dm, "ts": ts, "snr": snr, "bw": bw})
    aa.write_candidates(str(tmp_path), 0, 9.0, 0.0, 6.4, 0.1, np.float32(64e-6), 1,
                        {"dm": dm[:0], "ts": ts[:0], "snr": snr[:0], "bw": bw[:0]})
    names = sorted(os.listdir(tmp_path))
    assert names == ["analysed-t_0.00-dm_0.00-6.40.dat", "peak_analysed-t_1.50-dm_10.00-16.40.dat"]
    got = np.fromfile(tmp_path / names[1], np.float32).reshape(-1, 4)
    want = O.candidate_records(dm, ts, snr, bw, 10.0, 0.1, np.float32(64e-6 * 2), 1.5, 2)
    assert got.view(np.uint32).tolist() == want.view(np.uint32).tolist()


def test_analysis_plan_refusals(aa):
    md = aa.filterbank_metadata_struct(0.0, 64e-6, 1500.0, -1.0, 8, 1 << 15, 256, 0.0)
    o = aa.aa_py_pipeline_component_options()
    ap = aa.aa_py_analysis_plan(6.0, 3.0, 0.01, 0, False)
    # the analysis component not requested
    pipe = aa.aa_py_pipeline(aa.aa_py_pipeline_components(True, False, False, False), o, md,
                             np.zeros(256 * (1 << 15), np.uint16), 0)
    assert not pipe.bind_analysis_plan(ap)
    assert "not requested" in pipe.last_error()
    pipe.delete()
    # requested, but no DDTR strategy behind the plan
    pipe = aa.aa_py_pipeline(aa.aa_py_pipeline_components(True, True, False, False), o, md,
                             np.zeros(256 * (1 << 15), np.uint16), 0)
    assert not pipe.bind_analysis_plan(ap)
    assert "not ready" in pipe.last_error()
    pipe.delete()
    L = aa.lib()
    p = L.aa_py_analysis_plan(None, 6.0, 3.0, 0.01, 7, True)
    assert abs(L.aa_py_analysis_plan_sigma_cutoff(p) - 6.0) < 1e-6
    assert abs(L.aa_py_analysis_plan_sigma_constant(p) - 3.0) < 1e-6
    assert abs(L.aa_py_analysis_plan_max_boxcar_width_in_sec(p) - 0.01) < 1e-6
    assert L.aa_py_analysis_plan_enable_msd_baseline_noise(p)
    L.aa_analysis_plan_delete(p)


def test_fdas_still_refused(aa):
    md = aa.filterbank_metadata_struct(0.0, 64e-6, 1500.0, -1.0, 8, 1 << 15, 256, 0.0)
    o = aa.aa_py_pipeline_component_options()
    pipe = aa.aa_py_pipeline(aa.aa_py_pipeline_components(True, True, True, True), o, md,
                             np.zeros(256 * (1 << 15), np.uint16), 0)
    assert "the dedispersion, analysis and periodicity components" in pipe.last_error()
    pipe.delete()
    # dedispersion, analysis and periodicity together are accepted
    pipe = aa.aa_py_pipeline(aa.aa_py_pipeline_components(True, True, True, False), o, md,
                             np.zeros(256 * (1 << 15), np.uint16), 0)
    assert pipe.last_error() == ""
    pipe.delete()


def test_analysis_strategy_and_psr_entries(aa):
    """aa_py_pipeline_api_analysis_strategy gives the bound settings (none
    before bind); the periodicity candidate entries exist and return nothing
    before a periodicity search has run."""
    md = aa.filterbank_metadata_struct(0.0, 64e-6, 1500.0, -1.0, 8, 1 << 15, 256, 0.0)
    o = aa.aa_py_pipeline_component_options()
    pipe = aa.aa_py_pipeline(aa.aa_py_pipeline_components(True, True, False, False), o, md,
                             np.zeros(256 * (1 << 15), np.uint16), 0)
    L = aa.lib()
    assert not L.aa_py_pipeline_api_analysis_strategy(pipe.m_obj)
    assert not L.aa_py_get_psr_nCandidates(pipe.m_obj)
    assert not L.aa_py_get_psr_interbin_nCandidates(pipe.m_obj)
    L.aa_py_write_to_disk_psr_candidates(pipe.m_obj, b"unused")
    assert "periodicity" in pipe.last_error()
    pipe.delete()
