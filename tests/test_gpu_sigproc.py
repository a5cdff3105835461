"""Packed SIGPROC input on the GPU: a pipeline fed the data section as stored
(aa_b200_pipeline_set_packed_input; unpacked in the corner-turn kernel)
gives outputs bit-identical to the same pipeline fed the reference reader's
unsigned-short buffer, for every bit depth, from host and from device memory;
the 8-bit case also against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

import cases as C
import sigproc_cases as S

pytestmark = pytest.mark.gpu

# bit depth -> (nchans, nsamp, plan)
SHAPES = {
    1: (512, 16384, [(0, 30, 0.25, 1, 1), (30, 60, 0.5, 2, 1)]),
    2: (256, 16384, [(0, 12.7, 0.2, 1, 1), (12.8, 38.3, 0.4, 2, 1)]),
    4: (512, 16384, [(0, 3.15, 0.05, 1, 1), (3.2, 9.5, 0.1, 2, 1)]),
    8: (512, 32768, [(0, 6.3, 0.1, 1, 1), (6.4, 19.1, 0.2, 2, 1), (19.2, 44.7, 0.4, 4, 1)]),
    16: (256, 16384, [(0, 6.3, 0.1, 1, 1), (6.4, 19.1, 0.2, 2, 1)]),
    32: (128, 16384, [(0, 20, 0.25, 1, 1)]),
}


def _write(tmp_path, nbits):
    from aa_b200.sigproc import write_filterbank
    nchans, nsamp, plan = SHAPES[nbits]
    case = dict(nbits=nbits, nchans=nchans, nsamp=nsamp, seed=40 + nbits)
    path = str(tmp_path / f"b{nbits}.fil")
    data = S.make_data(case)
    write_filterbank(path, data, nbits, tsamp=64e-6, fch1=1550.0, foff=-300.0 / nchans)
    return path, plan


def _run(aa, meta, plan_rows, input_data=None, packed=None, device=False):
    if device:
        pipe = aa.create_pipeline(meta, input_data, True, False, True)
    else:
        comps = aa.aa_py_pipeline_components(True, False, False, False)
        o = aa.aa_py_pipeline_component_options()
        o.copy_ddtr_data_to_host = True
        pipe = aa.aa_py_pipeline(comps, o, meta, input_data, 0)
    if packed is not None:
        pipe.set_packed_input(packed)
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in plan_rows])
    assert pipe.bind_ddtr_plan(plan), pipe.last_error()
    while pipe.run():
        assert pipe.status_code() != aa.STATUS_ERROR, pipe.last_error()
    assert pipe.status_code() == aa.STATUS_FINISHED, pipe.last_error()
    outs = [a.copy() for a in pipe.output_arrays()]
    pipe.cleanUp()
    pipe.delete()
    plan.delete()
    return outs


@pytest.mark.parametrize("nbits", [1, 2, 4, 8, 16, 32])
def test_packed_input_matches_unsigned_short_input(aa, cuda_device, tmp_path, nbits):
    path, plan = _write(tmp_path, nbits)
    r = aa.aa_py_sigproc_input(path)
    meta = r.read_metadata()
    assert r.read_signal() and r.read_packed(), r.last_error()
    u16 = np.ascontiguousarray(r.input_array())
    packed = np.ascontiguousarray(r.packed_array())
    want = _run(aa, meta, plan, input_data=u16)
    got = _run(aa, meta, plan, packed=packed)
    assert len(got) == len(want) == len(plan)
    for g, w in zip(got, want):
        assert g.shape == w.shape
        assert np.array_equal(g.view(np.uint32), w.view(np.uint32))
    r.delete()


@pytest.mark.parametrize("nbits", [4, 8])
def test_packed_device_input(aa, cuda_device, tmp_path, nbits):
    import torch
    path, plan = _write(tmp_path, nbits)
    r = aa.aa_py_sigproc_input(path)
    meta = r.read_metadata()
    assert r.read_signal() and r.read_packed()
    want = _run(aa, meta, plan, input_data=np.ascontiguousarray(r.input_array()))
    d = torch.from_numpy(np.ascontiguousarray(r.packed_array())).to(cuda_device)
    got = _run(aa, meta, plan, input_data=d.data_ptr(), packed=d.data_ptr(), device=True)
    for g, w in zip(got, want):
        assert np.array_equal(g.view(np.uint32), w.view(np.uint32))
    r.delete()


def test_packed_8bit_matches_oracle(aa, oracle_mod, cuda_device, tmp_path):
    path, plan = _write(tmp_path, 8)
    r = aa.aa_py_sigproc_input(path)
    meta = r.read_metadata()
    assert r.read_packed()
    got = _run(aa, meta, plan, packed=np.ascontiguousarray(r.packed_array()))
    nchans, nsamp = meta.m_nchans, meta.m_nsamples
    case = dict(nbits=8, nchans=nchans, nsamp=nsamp, fch1=1550.0, foff=-300.0 / nchans, tsamp=64e-6, plan=plan,
                free_memory=0)
    s = oracle_mod.strategy(plan, nchans, nsamp, 1550.0, -300.0 / nchans, 64e-6, 8, C.strategy_free_memory(case))
    x = S.make_data(dict(nbits=8, nchans=nchans, nsamp=nsamp, seed=48))
    want, _ = oracle_mod.run_ddtr(x, s, nchans, nsamp, 64e-6, 8)
    for g, w in zip(got, want):
        assert np.array_equal(g.view(np.uint32), w.view(np.uint32))
    r.delete()


def test_packed_input_set_after_bind_is_refused(aa, cuda_device, tmp_path):
    path, plan = _write(tmp_path, 8)
    r = aa.aa_py_sigproc_input(path)
    meta = r.read_metadata()
    assert r.read_packed()
    comps = aa.aa_py_pipeline_components(True, False, False, False)
    o = aa.aa_py_pipeline_component_options()
    o.copy_ddtr_data_to_host = True
    pipe = aa.aa_py_pipeline(comps, o, meta, None, 0)
    pipe.set_packed_input(np.ascontiguousarray(r.packed_array()))
    p = aa.aa_py_ddtr_plan([aa.aa_py_dm(*x) for x in plan])
    assert pipe.bind_ddtr_plan(p)
    with pytest.raises(ValueError, match="before the plan is bound"):
        pipe.set_packed_input(np.ascontiguousarray(r.packed_array()))
    pipe.delete()
    p.delete()
    r.delete()


def test_output_dmt_writes_export_files(aa, cuda_device, tmp_path):
    """output_dmt: when the run finishes, every range's output is written in
    the reference's Export_DD_data files (include/aa_pipeline_runner.hpp:165-216)
    with the DM rows per file of include/aa_permitted_pipelines_1.hpp:312-323."""
    import os

    import dmt_oracle as O

    case = C.CASES["shared8_binned"]
    x = C.make_input(case)
    md = aa.filterbank_metadata_struct(0.0, case["tsamp"], case["fch1"], case["foff"], case["nbits"], case["nsamp"],
                                       case["nchans"], 0.0)
    comps = aa.aa_py_pipeline_components(True, False, False, False)
    o = aa.aa_py_pipeline_component_options()
    o.copy_ddtr_data_to_host = True
    o.output_dmt = True
    pipe = aa.aa_py_pipeline(comps, o, md, np.ascontiguousarray(x.reshape(-1)), 0)
    pipe.set_export_base(str(tmp_path / "lib" / "DD_data"))
    os.makedirs(tmp_path / "lib")
    plan = aa.aa_py_ddtr_plan([aa.aa_py_dm(*p) for p in case["plan"]])
    assert pipe.bind_ddtr_plan(plan), pipe.last_error()
    while pipe.run():
        pass
    assert pipe.status_code() == aa.STATUS_FINISHED, pipe.last_error()
    outs = [a.copy() for a in pipe.output_arrays()]
    inc = aa.lib().aa_py_total_computed_samples(pipe.m_obj)
    ndms = [a.shape[0] for a in outs]
    in_bin = [p[3] for p in case["plan"]]
    os.makedirs(tmp_path / "oracle")
    want = O.export(outs, inc, ndms, in_bin, str(tmp_path / "oracle" / "DD_data"), [1] * len(outs),
                    O.sd_per_file(1000, inc, 1))
    for w in want:
        g = tmp_path / "lib" / os.path.basename(w)
        assert g.read_bytes() == open(w, "rb").read(), os.path.basename(w)
    assert sorted(os.listdir(tmp_path / "lib")) == sorted(os.path.basename(w) for w in want)
    pipe.cleanUp()
    pipe.delete()
    plan.delete()
