"""Multi-beam batch (aa_b200_batch_*) against the plain per-beam pipeline.

Seven beams of different channel counts (256-3000, not all multiples of 32),
bit depths (2/4/8/16), DM plans (one to four ranges, binned, shared and cache
delay kernels) and lengths run in one batch; with a memory budget small
enough that the longer beams are split into several time chunks.  Each beam's
output must be bit-identical to the same beam run alone through the
reference-facing pipeline with the same memory budget, for the persistent
kernel and for one launch per job, with and without the CUDA graph and the
autotuner, and on a replay of the graph.
"""
from __future__ import annotations

import numpy as np
import pytest

import cases as C

pytestmark = pytest.mark.gpu

BEAMS = ["shared8_binned", "shared16_ragged", "shared4", "shared8_nch3000", "shared8_2bit", "cache8", "cache16"]
FREE_MEMORY = 104857600 + 9000 * 1000 * 10


def md_of(aa, case):
    return aa.filterbank_metadata_struct(0.0, case["tsamp"], case["fch1"], case["foff"], case["nbits"],
                                         case["nsamp"], case["nchans"], 0.0)


def plain_outputs(aa, case, x):
    comps = aa.aa_py_pipeline_components(True, False, False, False)
    o = aa.aa_py_pipeline_component_options()
    o.copy_ddtr_data_to_host = True
    pipe = aa.aa_py_pipeline(comps, o, md_of(aa, case), np.ascontiguousarray(x.reshape(-1)), 0)
    pipe.set_options(free_memory=FREE_MEMORY)
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in case["plan"]])
    assert pipe.bind_ddtr_plan(plan), pipe.last_error()
    while pipe.run():
        assert pipe.status_code() != aa.STATUS_ERROR, pipe.last_error()
    assert pipe.status_code() == aa.STATUS_FINISHED, pipe.last_error()
    outs = [a.copy() for a in pipe.output_arrays()]
    nchunks = pipe.num_tchunks()
    pipe.cleanUp()
    pipe.delete()
    plan.delete()
    return outs, nchunks


@pytest.fixture(scope="module")
def beams(aa, cuda_device):
    import torch
    data = []
    for name in BEAMS:
        case = C.CASES[name]
        x = C.make_input(case)
        want, nchunks = plain_outputs(aa, case, x)
        d_x = torch.from_numpy(x.view(np.int16).copy()).cuda()
        data.append((name, case, d_x, want, nchunks))
    assert max(d[4] for d in data) > 1, "the memory budget should split some beam into chunks"
    return data


def run_batch(aa, beams, kernel_choice=None, **opts):
    b = aa.batch(free_memory=FREE_MEMORY, **opts)
    plans = []
    try:
        for name, case, d_x, _, _ in beams:
            plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in case["plan"]])
            plans.append(plan)
            b.add_beam(md_of(aa, case), plan, d_x)
        if kernel_choice is not None:
            b.set_kernel_choice(kernel_choice)
        b.setup()
        results = []
        for _ in range(2):
            b.run()
            b.synchronize()
            results.append([[b.output(i, r).cpu().numpy() for r in range(len(case["plan"]))]
                            for i, (_, case, _, _, _) in enumerate(beams)])
        return results, {**b.info(), "sub_jobs": b.sub_jobs()}
    finally:
        b.delete()
        for p in plans:
            p.delete()


def assert_matches_plain(beams, results):
    for rep, res in enumerate(results):
        for bi, (name, case, _, want, _) in enumerate(beams):
            for r, w in enumerate(want):
                g = res[bi][r]
                assert g.shape == w.shape, (name, r)
                bad = np.flatnonzero(g.view(np.uint32) != w.view(np.uint32))
                assert bad.size == 0, (f"run {rep}, beam {name}, range {r}: {bad.size} outputs differ from the "
                                       f"plain pipeline, first at {np.unravel_index(bad[0], g.shape)}")


@pytest.mark.parametrize("persistent,use_graph,autotune", [(True, True, True), (True, False, False),
                                                           (False, True, True), (False, False, False)])
def test_batch_matches_plain_pipeline(aa, beams, persistent, use_graph, autotune):
    results, info = run_batch(aa, beams, persistent=persistent, use_graph=use_graph, autotune=autotune)
    if persistent:
        assert info["persistent_jobs"] > 0 and info["work_items"] > 0
    assert_matches_plain(beams, results)


@pytest.mark.parametrize("choice", [1, 2])
def test_batch_kernel_choice_matches_plain_pipeline(aa, beams, choice):
    """The channel-quad (1) or the subband (2) body forced on the one-byte
    ranges both can run: the subband jobs run in a persistent launch of their
    own after the others, and every beam stays bit-identical to its plain
    run, on the first run and on the graph's replay."""
    results, info = run_batch(aa, beams, persistent=True, use_graph=True, autotune=True, kernel_choice=choice)
    if choice == 2:
        assert 0 < info["sub_jobs"] < info["persistent_jobs"]
    else:
        assert info["sub_jobs"] == 0
    assert_matches_plain(beams, results)


def test_batch_one_persistent_launch(aa, beams):
    """All staged dedispersion steps of all beams go into one kernel launch."""
    _, info = run_batch(aa, beams, persistent=True, use_graph=True, autotune=False)
    n_ops = info["launches_per_run"] - 1 - info["other_jobs"]
    assert info["persistent_jobs"] > len(BEAMS)  # several (chunk, range) jobs per beam
    assert n_ops > 0  # the rest are corner turns and binning steps


def test_batch_refuses_bad_plan(aa, cuda_device):
    import torch
    case = C.CASES["shared8_binned"]
    b = aa.batch(free_memory=FREE_MEMORY)
    d = torch.zeros((case["nsamp"], case["nchans"]), dtype=torch.int16, device="cuda")
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(0.0, 10.0, 0.1, 2, 1)])  # first range binned: refused like the runner
    try:
        b.add_beam(md_of(aa, case), plan, d)
        with pytest.raises(RuntimeError, match="inBin 1"):
            b.setup()
    finally:
        b.delete()
        plan.delete()
