"""Differentiable refinement kernels (csrc/frac.cu) through torch.autograd,
against the FP64 host oracle (oracle/frac_oracle.py) and FP64 central
differences (h = 1e-3 in DM).

Tolerances: forward outputs within 1e-5 of the FP64 result relative to the
largest magnitude; gradients (to the input and to DM) within 1e-5 relative
to the FP64 analytic gradient and to the central difference (the series and
S/N are FP64 on the device; only the snippets are float32).  The central
difference is taken at trial DMs where no channel's delay crosses a whole
sample inside dm +- h, where the interpolated function is smooth in DM.
"""
from __future__ import annotations

import numpy as np
import pytest

import frac_oracle as F

pytestmark = pytest.mark.gpu

WIDTHS = (1, 2, 4, 8, 16, 32, 64)
TOL = 1e-5


def _setup(S=3, C=256, T=4096, seed=11):
    import torch
    from aa_b200 import refine as R
    x, dm_true, dm_trial, kc = R.synth_snippets(S, nchans=C, nsamp=T, seed=seed, amp=0.6,
                                                band=dict(tsamp=512e-6))
    return torch, R, x, dm_true, dm_trial, kc


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1e-30, np.max(np.abs(b))))


def test_forward_matches_fp64(cuda_device):
    torch, R, x, _, dm, kc = _setup()
    y = R.FracDedisperse.apply(x, dm, kc).cpu().numpy()
    xh, kch = x.cpu().numpy(), kc.cpu().numpy()
    for s in range(x.shape[0]):
        assert _rel(y[s], F.frac_forward(xh[s], float(dm[s]), kch)) <= TOL


def test_adjoint_matches_fp64(cuda_device):
    torch, R, x, _, dm, kc = _setup(seed=12)
    x = x.clone().requires_grad_(True)
    d = dm.clone().requires_grad_(True)
    y = R.FracDedisperse.apply(x, d, kc)
    g = torch.randn(y.shape, generator=torch.Generator(device="cuda").manual_seed(3), device="cuda",
                    dtype=torch.float64)
    y.backward(g)
    xh, kch, gh = x.detach().cpu().numpy(), kc.cpu().numpy(), g.cpu().numpy()
    for s in range(x.shape[0]):
        gx, gdm = F.frac_adjoint(xh[s], float(dm[s]), kch, gh[s])
        assert _rel(x.grad[s].cpu().numpy(), gx) <= TOL
        assert abs(float(d.grad[s]) - gdm) <= TOL * abs(gdm)


def test_row_shifts_match_fp64(cuda_device):
    """Snippets cut per channel (integer row shifts base[s][c])."""
    torch, R, x, _, dm, kc = _setup(seed=15)
    gen = torch.Generator(device="cuda").manual_seed(9)
    base = torch.randint(-40, 40, (x.shape[0], x.shape[1]), generator=gen, device="cuda", dtype=torch.int32)
    xg = x.clone().requires_grad_(True)
    d = dm.clone().requires_grad_(True)
    y = R.FracDedisperse.apply(xg, d, kc, base)
    g = torch.randn(y.shape, generator=gen, device="cuda", dtype=torch.float64)
    y.backward(g)
    xh, kch, gh, bh = x.cpu().numpy(), kc.cpu().numpy(), g.cpu().numpy(), base.cpu().numpy()
    for s in range(x.shape[0]):
        assert _rel(y[s].detach().cpu().numpy(), F.frac_forward(xh[s], float(dm[s]), kch, bh[s])) <= TOL
        gx, gdm = F.frac_adjoint(xh[s], float(dm[s]), kch, gh[s], bh[s])
        assert _rel(xg.grad[s].cpu().numpy(), gx) <= TOL
        assert abs(float(d.grad[s]) - gdm) <= TOL * abs(gdm)


def test_boxcar_matches_fp64(cuda_device):
    import torch
    from aa_b200 import refine as R
    gen = torch.Generator(device="cuda").manual_seed(5)
    y = torch.randn((2, 3000), generator=gen, device="cuda", dtype=torch.float64).requires_grad_(True)
    mu = torch.tensor([0.1, -0.2], device="cuda")
    sigma = torch.tensor([1.5, 2.0], device="cuda")
    snr = R.BoxcarSNR.apply(y, WIDTHS, mu, sigma)
    g = torch.randn(snr.shape, generator=gen, device="cuda", dtype=torch.float64)
    snr.backward(g)
    for s in range(2):
        want = F.boxcar_forward(y[s].detach().cpu().numpy(), WIDTHS, float(mu[s]), float(sigma[s]))
        assert _rel(snr[s].detach().cpu().numpy(), want) <= TOL
        gw = F.boxcar_adjoint(g[s].cpu().numpy(), WIDTHS, float(sigma[s]))
        assert _rel(y.grad[s].cpu().numpy(), gw) <= TOL


def test_peak_snr_gradient_matches_fp64_and_central_difference(cuda_device):
    torch, R, x, _, dm, kc = _setup(S=2, C=256, T=4096, seed=13)
    kch, xh = kc.cpu().numpy(), x.cpu().numpy()
    # trial DMs near the drawn ones where the FP64 stencil crosses no sample boundary
    trial = []
    for s in range(x.shape[0]):
        d0 = float(dm[s])
        for k in range(20000):
            d = float(np.float32(d0 + 0.000713 * k))
            if F.no_cell_crossing(d, kch, 1e-3):
                trial.append(d)
                break
        else:
            pytest.skip("no trial DM without a cell crossing found")
    d = torch.tensor(trial, dtype=torch.float32, device="cuda", requires_grad=True)
    sigma = float(np.sqrt(x.shape[1]))
    p = R.peak_snr(x, d, kc, WIDTHS, temperature=0.5)
    p.sum().backward()
    for s in range(x.shape[0]):
        L, g64 = F.loss_and_grad_dm(xh[s], trial[s], kch, WIDTHS, 0.0, sigma, 0.5)
        fd = F.central_difference_dm(xh[s], trial[s], kch, WIDTHS, 0.0, sigma, 0.5, h=1e-3)
        assert abs(float(p[s].detach()) - L) <= TOL * abs(L)
        assert abs(float(d.grad[s]) - g64) <= TOL * abs(g64), (float(d.grad[s]), g64)
        assert abs(float(d.grad[s]) - fd) <= TOL * abs(fd), (float(d.grad[s]), fd)


def test_refinement_moves_towards_the_true_dm(cuda_device):
    torch, R, x, dm_true, dm_trial, kc = _setup(S=8, C=256, T=4096, seed=14)
    dm, hist = R.refine_dm(x, dm_trial, kc, steps=50, lr=0.05, widths=WIDTHS)
    before = (dm_trial - dm_true).abs()
    after = (dm - dm_true).abs()
    assert float(hist[-1].mean()) >= float(hist[0].mean())
    assert float(after.median()) < float(before.median())


def test_refinement_rejects_bad_inputs(cuda_device):
    import torch
    from aa_b200 import refine as R
    x = torch.zeros((2, 8, 64), device="cuda")
    kc = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(TypeError):
        R.FracDedisperse.apply(x.double(), torch.zeros(2, device="cuda"), kc)
    with pytest.raises(RuntimeError, match="widths"):
        R.BoxcarSNR.apply(torch.zeros((2, 64), device="cuda", dtype=torch.float64), tuple(range(1, 20)),
                          torch.zeros(2, device="cuda"),
                          torch.ones(2, device="cuda"))
