"""GPU parity of the stateless seam (aa_b200_corner_turn, aa_b200_bin_gpu,
aa_b200_dedisperse) against the oracle, through the C ABI."""
from __future__ import annotations

import numpy as np
import pytest

import cases as C

pytestmark = pytest.mark.gpu

PAD = 1 << 16


def _setup(aa, oracle_mod, name):
    import torch
    case = C.CASES[name]
    x = C.make_input(case)
    s = aa.strategy(case["plan"], case["nchans"], case["nsamp"], case["fch1"], case["foff"], case["tsamp"],
                    case["nbits"], C.strategy_free_memory(case))
    L = s["t_processed"][0][0] + s["maxshift"]
    d_raw = torch.from_numpy(x[:L].view(np.int16).copy()).cuda()
    return torch, case, x, s, L, d_raw


def test_corner_turn_and_bin(aa, oracle_mod, cuda_device):
    torch, case, x, s, L, d_raw = _setup(aa, oracle_mod, "shared8_binned")
    nch = case["nchans"]
    d_ct = torch.zeros(nch * L + PAD, dtype=torch.uint8, device="cuda")
    aa.corner_turn(d_raw, d_ct, 8, nch, L, L)
    torch.cuda.synchronize()
    want = oracle_mod.corner_turn(x[:L], nch, L)
    assert np.array_equal(d_ct[:nch * L].cpu().numpy(), want.astype(np.uint8))
    d_b = torch.zeros_like(d_ct)
    aa.bin_gpu(d_ct, d_b, 8, nch, L)
    torch.cuda.synchronize()
    wb = oracle_mod.bin_flat(want, nch, L)
    assert np.array_equal(d_b[:nch * L].cpu().numpy(), wb.astype(np.uint8))


def test_corner_turn_rejects_out_of_range_samples(aa, cuda_device):
    import torch
    x = torch.full((64, 32), 300, dtype=torch.int16, device="cuda")
    out = torch.zeros(64 * 32, dtype=torch.uint8, device="cuda")
    with pytest.raises(RuntimeError, match="range"):
        aa.corner_turn(x, out, 8, 32, 64, 64)


@pytest.mark.parametrize("name", ["shared8_binned", "cache8", "shared4", "shared16", "fma_probe"])
def test_dedisperse_seam_matches_oracle(aa, oracle_mod, cuda_device, name):
    torch, case, x, s, L, d_raw = _setup(aa, oracle_mod, name)
    nch, nbits = case["nchans"], case["nbits"]
    eb = 1 if nbits <= 8 else 2
    dt = torch.uint8 if eb == 1 else torch.int16
    d_ct = torch.zeros(nch * L + PAD, dtype=dt, device="cuda")
    aa.corner_turn(d_raw, d_ct, nbits, nch, L, L)
    tp = s["t_processed"][0][0]
    nd = s["ndms"]
    out = torch.zeros(nd[0] * tp, dtype=torch.float32, device="cuda")
    tsr = float(np.float32(case["tsamp"]) * np.float32(s["dm"][0][3]))
    aa.dedisperse(0, tp, [d[3] for d in s["dm"]], s["dmshifts"], d_ct, L, d_ct.numel(), out, tp, nch, tsr,
                  [d[0] for d in s["dm"]], [d[2] for d in s["dm"]], nd, nbits)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(nd[0], tp)
    flat = oracle_mod.corner_turn(x[:L], nch, L)
    kern = oracle_mod.select_kernel(nbits, s["dm"][0][2], np.float32(tsr), s["dmshifts"][-1])
    m0 = np.float32(np.float32(s["dm"][0][0]) / np.float32(tsr))
    ms = np.float32(np.float32(s["dm"][0][2]) / np.float32(tsr))
    want = oracle_mod.dedisperse(kern, oracle_mod.FMA_ALL, flat, L, nch, tp, nd[0], s["dmshifts"], m0, ms,
                                 s["dm"][0][3])
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_dedisperse_refuses_short_allocation(aa, oracle_mod, cuda_device):
    torch, case, x, s, L, d_raw = _setup(aa, oracle_mod, "shared8_binned")
    nch = case["nchans"]
    d_ct = torch.zeros(nch * L, dtype=torch.uint8, device="cuda")
    tp = s["t_processed"][0][0]
    out = torch.zeros(s["ndms"][0] * tp, dtype=torch.float32, device="cuda")
    with pytest.raises(RuntimeError, match="padding|elements"):
        aa.dedisperse(0, tp, [1, 2, 4, 8], s["dmshifts"], d_ct, L, nch * L // 2, out, tp, nch, 64e-6,
                      [d[0] for d in s["dm"]], [d[2] for d in s["dm"]], s["ndms"], 8)
