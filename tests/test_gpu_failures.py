"""Failure handling without a GPU fault (the library's own checks).

* A bounded mbarrier wait that is made to run out (an expected arrival never
  comes) returns the timeout flag to the host, and the context stays usable.
* Host-side failure injection: the n-th checked CUDA result of a pipeline
  (or batch engine) reads as a failure; every such run ends with the error
  status and message, releases what it allocated, and a following run is
  bit-identical to the oracle.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import cases as C

pytestmark = pytest.mark.gpu


def _run(aa, case, x):
    from test_gpu_parity import run_pipeline
    return run_pipeline(aa, case, x)


def _oracle(oracle_mod, case, x):
    s = oracle_mod.strategy(case["plan"], case["nchans"], case["nsamp"], case["fch1"], case["foff"], case["tsamp"],
                            case["nbits"], C.strategy_free_memory(case))
    outs, _ = oracle_mod.run_ddtr(x, s, case["nchans"], case["nsamp"], case["tsamp"], case["nbits"])
    return outs


def test_bounded_wait_runs_out_and_context_survives(aa, oracle_mod, cuda_device):
    st = ctypes.c_int(-1)
    assert aa.lib().aa_b200_selftest_bounded_wait(2000, ctypes.byref(st)) == 0
    assert st.value == 8
    case = C.CASES["shared8_binned"]
    x = C.make_input(case)
    got, _, _, _ = _run(aa, case, x)
    want = _oracle(oracle_mod, case, x)
    for g, w in zip(got, want):
        assert np.array_equal(g.view(np.uint32), w.view(np.uint32))


def _attempt(aa, case, x, n):
    """One pipeline run with the n-th checked CUDA result failing; returns the
    error message, or None when the run finished before the n-th check."""
    md = aa.filterbank_metadata_struct(0.0, case["tsamp"], case["fch1"], case["foff"], case["nbits"], case["nsamp"],
                                       case["nchans"], 0.0)
    comps = aa.aa_py_pipeline_components(True, False, False, False)
    o = aa.aa_py_pipeline_component_options()
    o.copy_ddtr_data_to_host = True
    pipe = aa.aa_py_pipeline(comps, o, md, np.ascontiguousarray(x.reshape(-1)), 0)
    pipe.set_options(free_memory=C.strategy_free_memory(case))
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in case["plan"]])
    aa.lib().aa_b200_debug_fail_after(n)
    msg = None
    try:
        if not pipe.bind_ddtr_plan(plan):
            msg = pipe.last_error()
        else:
            while pipe.run():
                pass
            if pipe.status_code() == aa.STATUS_ERROR:
                msg = pipe.last_error()
    finally:
        aa.lib().aa_b200_debug_fail_after(0)
        pipe.cleanUp()
        pipe.delete()
        plan.delete()
    return msg


def test_injected_failures_end_cleanly(aa, oracle_mod, cuda_device):
    import torch
    case = C.CASES["shared8_binned"]
    x = C.make_input(case)
    # how many checked CUDA results a whole run has
    big = 1 << 40
    aa.lib().aa_b200_debug_fail_after(big)
    _run(aa, case, x)
    used = big - aa.lib().aa_b200_debug_fail_countdown()
    aa.lib().aa_b200_debug_fail_after(0)
    assert used > 20
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    ns = sorted(set(list(range(1, 25)) + list(range(25, used + 1, max(1, used // 40))) + [used]))
    failed = 0
    for n in ns:
        msg = _attempt(aa, case, x, n)
        if msg is not None:
            assert "injected failure" in msg, (n, msg)
            failed += 1
    assert failed >= len(ns) - 2
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 < 64 << 20, f"{(free0 - free1) >> 20} MiB not released after {len(ns)} failed runs"
    got, _, _, _ = _run(aa, case, x)
    want = _oracle(oracle_mod, case, x)
    for g, w in zip(got, want):
        assert np.array_equal(g.view(np.uint32), w.view(np.uint32))


def test_injected_failure_in_batch_engine(aa, cuda_device):
    import torch
    case = C.CASES["shared8_binned"]
    x = torch.from_numpy(C.make_input(case).astype(np.int16)).to(cuda_device)
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in case["plan"]])
    md = aa.filterbank_metadata_struct(0.0, case["tsamp"], case["fch1"], case["foff"], case["nbits"], case["nsamp"],
                                       case["nchans"], 0.0)
    for n in (3, 9, 40):
        aa.lib().aa_b200_debug_fail_after(n)
        try:
            with pytest.raises(RuntimeError, match="injected failure"):
                b = aa.batch(free_memory=C.strategy_free_memory(case))
                b.add_beam(md, plan, x)
                b.setup()
                b.run()
                b.synchronize()
        finally:
            aa.lib().aa_b200_debug_fail_after(0)
    plan.delete()
