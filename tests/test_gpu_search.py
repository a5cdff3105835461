"""Single-pulse search kernels (csrc/sps.cu) and snippet cutting against
float64 numpy restatements of the same definitions."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WIDTHS = (1, 2, 4, 8, 16, 32, 64)


def _np_peaks(rows, widths, block):
    ndms, T = rows.shape
    nb = (T + block - 1) // block
    best = np.full((ndms, nb), -np.inf)
    for r in range(ndms):
        m, sd = rows[r].mean(), rows[r].std()
        c = np.concatenate([[0.0], np.cumsum(rows[r])])
        for w in widths:
            t = np.arange(T - w + 1)
            snr = (c[t + w] - c[t] - w * m) / (sd * np.sqrt(w))
            for b in range(nb):
                seg = snr[b * block:(b + 1) * block]
                if seg.size:
                    best[r, b] = max(best[r, b], seg.max())
    return best


def test_block_peaks_match_numpy(cuda_device):
    import torch
    from aa_b200 import search as S
    from aa_b200 import lib
    rng = np.random.default_rng(3)
    rows = rng.normal(size=(5, 5000))
    rows[2, 3000:3008] += 3.0
    pitch = 5008
    buf = torch.zeros((5, pitch), dtype=torch.float32, device="cuda")
    buf[:, :5000] = torch.as_tensor(rows, dtype=torch.float32)
    snr, t, w = S.range_peaks(buf, 5000, WIDTHS)
    block = lib().aa_b200_sps_block_samples()
    want = _np_peaks(rows.astype(np.float32).astype(np.float64), WIDTHS, block)
    assert np.allclose(snr.cpu().numpy(), want, rtol=1e-4, atol=1e-4)
    b = 3000 // block
    assert abs(int(t[2, b]) - 3000) <= 2 and int(w[2, b]) == 8
    c = S.candidates(buf, 5000, 10.0, 0.5, 2, threshold=6.0, widths=WIDTHS)
    assert c["snr"].numel() >= 1
    i = int(torch.argmax(c["snr"]))
    assert abs(float(c["dm"][i]) - 11.0) < 1e-6 and abs(int(c["t"][i]) - 6000) <= 4


def test_select_keeps_one_candidate_per_event(cuda_device):
    import torch
    from aa_b200 import search as S
    dev = "cuda"
    c1 = {"snr": torch.tensor([9.0, 8.0, 7.0], device=dev), "dm": torch.tensor([10.0, 10.5, 30.0], device=dev),
          "t": torch.tensor([1000, 1100, 90000], device=dev), "w": torch.tensor([4, 4, 8], device=dev)}
    out = S.select([c1], k=64, separation=4096)
    assert out["t"].tolist() == [1000, 90000]


def test_cut_snippets_aligns_channels(cuda_device):
    import torch
    from aa_b200 import search as S
    nsamp, nch = 4000, 16
    x = torch.arange(nsamp * nch, device="cuda", dtype=torch.int32).reshape(nsamp, nch).remainder(251).to(torch.int16)
    kc = torch.linspace(0, 30, nch, dtype=torch.float64, device="cuda")
    dm = torch.tensor([10.3], device="cuda")
    t = torch.tensor([1500], device="cuda")
    w = torch.tensor([8], device="cuda")
    snip, base = S.cut_snippets(x, kc, dm, t, w, nwin=64, offset=0.0, scale=1.0)
    xh = x.cpu().numpy().astype(np.int64)
    b = np.floor(float(dm[0]) * kc.cpu().numpy()).astype(np.int64)
    s0 = 1500 + 4 - 32
    for c in (0, 7, 15):
        assert int(base[0, c]) == b[c]
        assert np.array_equal(snip[0, c].cpu().numpy(), xh[s0 + b[c]:s0 + b[c] + 64, c].astype(np.float32))
