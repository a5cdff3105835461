"""aa_b200_dedisperse_noalloc: dedispersion for callers that cannot allocate
device memory.

Callers running inside a memory pool or arena that owns the GPU's memory, in
real-time loops that must not synchronise with the allocator, or on hosts that
reserve all device memory at start-up cannot let the library call cudaMalloc.
The entry point keeps its delay, window and offset tables in a fixed array of
the library's device image instead.  This test calls it through the C ABI
twice in a row and checks both results against aa_b200_dedisperse (which
allocates its scratch) and against the CPU oracle, bit for bit -- the
tolerance of every other parity test here -- and that the second call changes
nothing in the device's free memory.
The file is named to be collected last, so a run that stops at the first
failure has run every other test before it.
"""
from __future__ import annotations

import numpy as np
import pytest

import cases as C

pytestmark = pytest.mark.gpu

PAD = 1 << 16


def _inputs(aa, name):
    import torch
    case = C.CASES[name]
    x = C.make_input(case)
    s = aa.strategy(case["plan"], case["nchans"], case["nsamp"], case["fch1"], case["foff"], case["tsamp"],
                    case["nbits"], C.strategy_free_memory(case))
    L = s["t_processed"][0][0] + s["maxshift"]
    nch, nbits = case["nchans"], case["nbits"]
    d_raw = torch.from_numpy(x[:L].view(np.int16).copy()).cuda()
    dt = torch.uint8 if nbits <= 8 else torch.int16
    d_ct = torch.zeros(nch * L + PAD, dtype=dt, device="cuda")
    aa.corner_turn(d_raw, d_ct, nbits, nch, L, L)
    tp = s["t_processed"][0][0]
    tsr = float(np.float32(case["tsamp"]) * np.float32(s["dm"][0][3]))
    args = dict(i=0, t_processed=tp, inBin=[d[3] for d in s["dm"]], dmshifts=s["dmshifts"], d_input=d_ct,
                i_nsamp=L, d_input_elems=d_ct.numel(), out_pitch=tp, nchans=nch, tsamp=tsr,
                dm_low=[d[0] for d in s["dm"]], dm_step=[d[2] for d in s["dm"]], ndms=s["ndms"], nbits=nbits)
    return torch, s, tp, args, case, x


@pytest.mark.parametrize("name", ["shared8_binned", "fma_probe", "cache16"])
def test_noalloc_matches_allocating_entry_point(aa, oracle_mod, cuda_device, name):
    torch, s, tp, args, case, x = _inputs(aa, name)
    n = s["ndms"][0] * tp
    ref = torch.zeros(n, dtype=torch.float32, device="cuda")
    aa.dedisperse(d_output=ref, **args)
    outs = []
    for call in range(2):
        out = torch.full((n,), -1.0, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        aa.dedisperse_noalloc(d_output=out, **args)
        torch.cuda.synchronize()
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before
        outs.append(out.cpu().numpy())
    want = ref.cpu().numpy()
    for got in outs:
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # and directly against the oracle: range 0 of chunk 0 on the corner-turned input
    O = oracle_mod
    L = args["i_nsamp"]
    d = s["dm"][0]
    tsr = np.float32(case["tsamp"]) * np.float32(d[3])
    kind = O.select_kernel(case["nbits"], d[2], tsr, s["dmshifts"][-1])
    flat = O.corner_turn(x[:L], case["nchans"], L)
    m0, ms = np.float32(np.float32(d[0]) / tsr), np.float32(np.float32(d[2]) / tsr)
    oracle_out = O.dedisperse(kind, O.FMA_ALL, flat, L, case["nchans"], tp, s["ndms"][0], s["dmshifts"], m0, ms, d[3])
    for got in outs:
        assert np.array_equal(got.view(np.uint32), oracle_out.reshape(-1).view(np.uint32))


def test_noalloc_refuses_sizes_beyond_its_scratch(aa, cuda_device):
    import torch
    d_in = torch.zeros(1 << 16, dtype=torch.uint8, device="cuda")
    out = torch.zeros(1 << 10, dtype=torch.float32, device="cuda")
    nch = 4096
    with pytest.raises(RuntimeError, match="exceeds the fixed scratch limits"):
        aa.dedisperse_noalloc(0, 224, [1], np.zeros(nch, np.float32), d_in, 1000, d_in.numel(), out, 224, nch,
                              64e-6, [0.0], [0.1], [1024], 8)
