"""The periodicity component end to end through the reference-facing C ABI
(aa_py_pipeline_api with the dedispersion and periodicity components,
aa_py_pipeline_api_bind_periodicity_plan and the ten-argument form, the run
loop to the end, aa_py_get_psr_nCandidates / _interbin_) against the
reference's own runner on the same filterbanks (golden lists from
oracle/ref_harness.cu aaref_run_pipeline_psr, tests/golden/psr_pipeline_golden.json).

Both pipelines append candidates with atomic counters, so a list's order
varies from run to run; the lists are compared as sorted record sets: the
same records (DM, frequency, harmonic count equal) up to as many as differed
between two runs of the reference itself, and S/N within 1e-4 relative for
95 % of them and within 2 % for all (the reference's whitening scales some
bins in two unordered blocks, the library scales them once, and the
reference's own repeated runs give different S/N bits).  The golden lists were made by the reference in fresh processes;
the test does not run the reference (its whitening reads one boundary and
one median past its tables on every call)."""
from __future__ import annotations

import base64
import json
import os

import numpy as np
import pytest

import psr_pipeline_cases as PC

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "psr_pipeline_golden.json")


@pytest.fixture(scope="module")
def golden():
    if not os.path.exists(GOLDEN):
        pytest.skip("periodicity pipeline golden lists not generated (tests/golden/make_psr_pipeline_golden.py)")
    with open(GOLDEN) as fh:
        return json.load(fh)


def run_pipeline(aa, case, x, device_output=False, simple_bind=False, sigma=None, psr_memory=PC.PSR_MEMORY):
    md = aa.filterbank_metadata_struct(0.0, case["tsamp"], case["fch1"], case["foff"], case["nbits"],
                                       case["nsamp"], case["nchans"], 0.0)
    comps = aa.aa_py_pipeline_components(True, False, True, False)
    o = aa.aa_py_pipeline_component_options()
    o.copy_ddtr_data_to_host = True
    pipe = aa.aa_py_pipeline(comps, o, md, np.ascontiguousarray(x.reshape(-1)), 0)
    pipe.set_options(free_memory=180 * 2**30)
    if device_output:
        pipe.set_device_output(True)
    pipe.set_periodicity_memory(psr_memory)
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in case["plan"]])
    assert pipe.bind_ddtr_plan(plan), pipe.last_error()
    if simple_bind:
        pp = aa.aa_py_periodicity_plan(sigma or case["sigma_cutoff"], 3.0, case["nHarmonics"], 0, case["selection"],
                                       True)
        assert pipe.bind_periodicity_plan(pp), pipe.last_error()
    else:
        assert pipe.bind_periodicity_plan_full(sigma or case["sigma_cutoff"], True, 3.0, case["nHarmonics"],
                                               case["hs_algorithm"], case["selection"], True), pipe.last_error()
    statuses = []
    while pipe.run():
        statuses.append(pipe.status_code())
        assert pipe.status_code() != aa.STATUS_ERROR, pipe.last_error()
    assert pipe.status_code() == aa.STATUS_FINISHED, pipe.last_error()
    power = pipe.get_psr_candidates(False)
    inter = pipe.get_psr_candidates(True)
    info = pipe.psr_info()
    pipe.cleanUp()
    pipe.delete()
    plan.delete()
    return power, inter, statuses, info


def decode(g, key):
    return np.frombuffer(base64.b64decode(g[key]), np.float32).reshape(-1, 4)


def sort_records(a):
    """Records in (DM, frequency, harmonics, S/N bits) order."""
    a = np.ascontiguousarray(a, np.float32)
    return a[np.lexsort((a[:, 2].view(np.uint32), a[:, 3], a[:, 1], a[:, 0]))]


def keyed(a):
    return {tuple(v[[0, 1, 3]]): float(v[2]) for v in sort_records(a)}


def compare(got, want, what, allow=0, rtol=1e-5, share=1.0, rtol_all=None):
    """True when the sorted lists are the same bits; otherwise asserts that
    at most `allow` records are in one list only (by DM, frequency and
    harmonic count), that at least `share` of the others have S/N within
    rtol and all within rtol_all, and returns False."""
    gs, ws = sort_records(got), sort_records(want)
    if gs.tobytes() == ws.tobytes():
        return True
    kg = {tuple(v[[0, 1, 3]]): v[2] for v in gs}
    kw = {tuple(v[[0, 1, 3]]): v[2] for v in ws}
    only = set(kg) ^ set(kw)
    assert len(only) <= allow, f"{what}: {len(only)} records in one list only (allowed {allow})"
    common = sorted(set(kg) & set(kw))
    a = np.array([kg[k] for k in common], np.float64)
    b = np.array([kw[k] for k in common], np.float64)
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-30)
    bad = rel > rtol
    assert bad.sum() <= (1.0 - share) * len(a), \
        f"{what}: {int(bad.sum())} of {len(a)} S/N differ beyond {rtol} (worst {rel.max():.2e})"
    if rtol_all is not None:
        assert rel.max() <= rtol_all, f"{what}: S/N differ by {rel.max():.2e} relative"
    return False


@pytest.mark.parametrize("name", list(PC.PIPELINE_CASES))
def test_periodicity_matches_reference_runner(aa, golden, cuda_device, name):
    case = PC.PIPELINE_CASES[name]
    g = golden[name]
    assert g["rc"] == 0
    x = PC.make_input(case)
    # the golden run's cutoff (raised from the case's until its lists were short)
    power, inter, statuses, info = run_pipeline(aa, case, x, sigma=g["sigma_cutoff"])
    # dedispersion steps, its finished_component, then the periodicity's
    assert statuses[-1] == aa.STATUS_FINISHED_COMPONENT and statuses[-2] == aa.STATUS_FINISHED_COMPONENT
    assert info["batches"] >= 2 and info["fft_length"] == 1 << 17
    assert power.shape[0] > 0, "no power candidates: the pulse train was not found"
    # The same records up to the reference's own run-to-run differences.
    # S/N: its whitening scales the bins where an even segment meets an odd
    # one (19 of the 65537 bins here) by one of two neighbouring norms, or
    # both, in unordered blocks, and its own two golden runs gave different
    # S/N bits for the same records.  A record whose harmonics or interbin
    # pair meet such a bin moves by up to ~1 %; the MSD over the plane, and
    # so every S/N, by much less.  So: 95 % of the records within 1e-4 (also
    # covering the cuFFT build this process loaded), every record within 2 %.
    for key, got in (("power", power), ("interbin", inter)):
        compare(got, decode(g, key), key, allow=2 * g.get(key + "_repeat_only_one", 0) + 2, rtol=1e-4,
                share=0.95, rtol_all=2e-2)


def test_periodicity_train_found(aa, cuda_device):
    """The strongest power candidate is the injected train: its DM and a
    harmonic of its frequency."""
    case = PC.PIPELINE_CASES["psr_greedy_peaks"]
    power, _, _, _ = run_pipeline(aa, case, PC.make_input(case))
    best = power[np.argmax(power[:, 2])]
    f0 = 1.0 / (case["train"]["period_samples"] * case["tsamp"])
    assert abs(best[0] - case["train"]["dm"]) < 1.0, best
    ratio = best[1] / f0
    assert abs(ratio - round(ratio)) < 0.02 and round(ratio) >= 1, best


def test_periodicity_from_device_rows_and_reference_binding(aa, cuda_device):
    """Rows kept on the device give the lists the host rows give; the
    reference wrapper's six-argument binding equals the ten-argument one
    with the greedy sum."""
    case = PC.PIPELINE_CASES["psr_greedy_peaks"]
    x = PC.make_input(case)
    p0, i0, _, _ = run_pipeline(aa, case, x)
    p1, i1, _, _ = run_pipeline(aa, case, x, device_output=True)
    p2, i2, _, _ = run_pipeline(aa, case, x, simple_bind=True)
    for a, b in ((p0, p1), (i0, i1), (p0, p2), (i0, i2)):
        assert sort_records(a).tobytes() == sort_records(b).tobytes()


def test_periodicity_in_batches(aa, cuda_device):
    """A budget of 300 MB splits each range into batches of 64 DM trials
    (the strategy the reference computes for it, tests/test_psr_strategy.py):
    every batch runs (its own MSD), the train is still found and the
    candidates' DMs come from several batches."""
    case = PC.PIPELINE_CASES["psr_greedy_peaks"]
    power, inter, _, info = run_pipeline(aa, case, PC.make_input(case), psr_memory=300 << 20)
    assert info["batches"] == 6 and info["dms_per_batch"] == 64
    best = power[np.argmax(power[:, 2])]
    assert abs(best[0] - case["train"]["dm"]) < 1.0, best
    assert len(np.unique(np.floor(power[:, 0] / 6.4))) >= 2
