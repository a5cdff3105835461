"""The reference runner's optional input/output processing on the GPU (zero
DM, zero DM with outliers, input and output normalisation, old RFI, bandpass
average, a custom bandpass), called through the C ABI: every range's output
bit-identical to the reference's own GPU run with the same options
(tests/golden/preproc_golden.json, tests/golden/make_preproc_golden.py)."""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import pytest

import cases as C
import preproc_cases as P

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "preproc_golden.json")


@pytest.fixture(scope="module")
def golden():
    if not os.path.exists(GOLDEN):
        pytest.skip("processing golden vectors not generated (tests/golden/make_preproc_golden.py)")
    with open(GOLDEN) as f:
        return json.load(f)["runs"]


def run_with_options(aa, case, opts, bandpass=None, variant=0, packed=None, device=None):
    md = aa.filterbank_metadata_struct(0.0, case["tsamp"], case["fch1"], case["foff"], case["nbits"],
                                       case["nsamp"], case["nchans"], 0.0)
    comps = aa.aa_py_pipeline_components(True, False, False, False)
    o = aa.aa_py_pipeline_component_options()
    o.copy_ddtr_data_to_host = True
    o.zero_dm = bool(opts & P.ZDM)
    o.zero_dm_with_outliers = bool(opts & P.ZDM_OUT)
    o.input_DDTR_normalization = bool(opts & P.IN_NORM)
    o.output_DDTR_normalization = bool(opts & P.OUT_NORM)
    o.old_rfi = bool(opts & P.OLD_RFI)
    o.set_bandpass_average = bool(opts & P.BP_AVG)
    x = C.make_input(case)
    pipe = aa.aa_py_pipeline(comps, o, md, np.ascontiguousarray(x.reshape(-1)), 0)
    if packed is not None:
        pipe.set_packed_input(packed)
    pipe.set_options(free_memory=C.strategy_free_memory(case))
    pipe.set_kernel_variant(variant)
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in case["plan"]])
    if bandpass is not None:
        assert plan.bind_bandpass_normalization(bandpass, bandpass.size)
    assert pipe.bind_ddtr_plan(plan), pipe.last_error()
    while pipe.run():
        assert pipe.status_code() != aa.STATUS_ERROR, pipe.last_error()
    assert pipe.status_code() == aa.STATUS_FINISHED, pipe.last_error()
    outs = [a.copy() for a in pipe.output_arrays()]
    pipe.cleanUp()
    pipe.delete()
    plan.delete()
    return outs


def check(got, rec):
    for r, rr in enumerate(rec["ranges"]):
        g = got[r]
        assert list(g.shape) == rr["shape"]
        if hashlib.sha256(g.tobytes()).hexdigest() != rr["sha256"]:
            bad = [(i, j) for i, j, bits in rr["samples"] if int(g[i, j].view(np.uint32)) != bits]
            pytest.fail(f"range {r}: differs from the reference GPU ({len(bad)}/{len(rr['samples'])} sampled values "
                        f"differ, e.g. {bad[:3]})")


@pytest.mark.parametrize("run", list(P.RUNS))
def test_processing_matches_reference_gpu(aa, golden, cuda_device, run):
    cname, opts, bp = P.RUNS[run]
    case = C.CASES[cname]
    bandpass = P.custom_bandpass(case["nchans"]) if bp == "custom" else None
    check(run_with_options(aa, case, opts, bandpass), golden[run])


@pytest.mark.parametrize("run", ["s8_all", "s16_zdm_outliers"])
def test_processing_with_generic_kernels(aa, golden, cuda_device, run):
    cname, opts, _ = P.RUNS[run]
    check(run_with_options(aa, C.CASES[cname], opts, variant=1), golden[run])


def test_processing_on_packed_input(aa, golden, cuda_device):
    """Packed input is unpacked into a writable chunk before zero DM."""
    from aa_b200.sigproc import pack
    cname, opts, _ = P.RUNS["s8_all"]
    case = C.CASES[cname]
    packed = pack(C.make_input(case), 8)
    check(run_with_options(aa, case, opts, packed=packed), golden["s8_all"])


def test_zero_dm_needs_4_8_or_16_bits(aa, cuda_device):
    case = dict(C.CASES["shared8_2bit"])
    with pytest.raises(AssertionError, match="4, 8 or 16-bit"):
        run_with_options(aa, case, P.ZDM)
