"""Differentiable candidate refinement on the B200 kernels.

FracDedisperse and BoxcarSNR are torch.autograd.Functions whose forward and
backward passes are the hand-written kernels of csrc/frac.cu, called through
the C ABI (aa_b200_frac_*, aa_b200_boxcar_*); there is no PyTorch fallback.

    y   = FracDedisperse.apply(x, dm, kc, base)  x [S][C][T] f32, dm [S] f32, kc [C] f64,
                                                 base [S][C] int32 row shifts or None; y [S][T] f64
    snr = BoxcarSNR.apply(y, widths, mu, sigma)  snr [S][len(widths)][T] f64

The snippets stay float32; the channel sums, the series y and the S/N and
their gradients are FP64, so that a smooth maximum of the S/N at a low
temperature (which amplifies rounding) keeps an FP64-accurate DM gradient.

The delays are recomputed from (dm, kc) in the backward pass.  mu and sigma
(per snippet) are constants of the S/N: by default the noise level of the
dedispersed series of unit-variance channels (mu 0, sigma sqrt(C)).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import lib

DISPERSION_CONSTANT = 4.148808e3  # s MHz^2 / (pc cm^-3)
DEFAULT_WIDTHS = (1, 2, 4, 8, 16, 32, 64)


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _err() -> str:
    return lib().aa_b200_frac_last_error().decode()


def delay_per_dm(nchans: int, fch1: float, foff: float, tsamp: float, device="cuda") -> torch.Tensor:
    """kc[c]: delay of channel c relative to fch1, samples per unit DM (float64)."""
    f = fch1 + foff * np.arange(nchans, dtype=np.float64)
    kc = DISPERSION_CONSTANT * (f ** -2 - fch1 ** -2) / tsamp
    return torch.as_tensor(kc, dtype=torch.float64, device=device)


def _check_cuda(*ts):
    for t in ts:
        if not (t.is_cuda and t.is_contiguous()):
            raise ValueError("refinement tensors must be contiguous CUDA tensors")


class FracDedisperse(torch.autograd.Function):
    """Fractional-delay (linearly interpolated) dedispersion; gradients to x and dm."""

    @staticmethod
    def forward(ctx, x, dm, kc, base=None):
        if x.dtype != torch.float32 or dm.dtype != torch.float32 or kc.dtype != torch.float64:
            raise TypeError("x, dm must be float32 and kc float64")
        x, dm, kc = x.contiguous(), dm.contiguous(), kc.contiguous()
        _check_cuda(x, dm, kc)
        S, C, T = x.shape
        if dm.shape != (S,) or kc.shape != (C,):
            raise ValueError("dm must be [S] and kc [C]")
        if base is not None:
            base = base.to(torch.int32).contiguous()
            _check_cuda(base)
            if base.shape != (S, C):
                raise ValueError("base must be [S][C]")
        y = torch.empty((S, T), dtype=torch.float64, device=x.device)
        if lib().aa_b200_frac_dedisperse_fwd(x.data_ptr(), dm.data_ptr(), kc.data_ptr(),
                                             base.data_ptr() if base is not None else None, S, C, T, y.data_ptr(),
                                             _stream()):
            raise RuntimeError(_err())
        ctx.save_for_backward(x, dm, kc, base)
        return y

    @staticmethod
    def backward(ctx, gy):
        x, dm, kc, base = ctx.saved_tensors
        gy = gy.to(torch.float64).contiguous()
        S, C, T = x.shape
        need_x, need_dm = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        gx = torch.empty_like(x) if need_x else None
        gdm = torch.empty_like(dm) if need_dm else None
        partial = torch.empty((S, C), dtype=torch.float64, device=x.device) if need_dm else None
        if need_x or need_dm:
            if lib().aa_b200_frac_dedisperse_adj(x.data_ptr(), dm.data_ptr(), kc.data_ptr(),
                                                 base.data_ptr() if base is not None else None, gy.data_ptr(), S, C, T,
                                                 gx.data_ptr() if need_x else None,
                                                 gdm.data_ptr() if need_dm else None,
                                                 partial.data_ptr() if need_dm else None, _stream()):
                raise RuntimeError(_err())
        return gx, gdm, None, None


class BoxcarSNR(torch.autograd.Function):
    """Boxcar S/N of dedispersed series for ascending widths; gradient to y."""

    @staticmethod
    def forward(ctx, y, widths, mu, sigma):
        y = y.to(torch.float64).contiguous()
        _check_cuda(y, mu, sigma)
        S, T = y.shape
        w = (ctypes.c_int * len(widths))(*widths)
        snr = torch.empty((S, len(widths), T), dtype=torch.float64, device=y.device)
        if lib().aa_b200_boxcar_snr_fwd(y.data_ptr(), S, T, w, len(widths), mu.data_ptr(), sigma.data_ptr(),
                                        snr.data_ptr(), _stream()):
            raise RuntimeError(_err())
        ctx.widths = tuple(widths)
        ctx.save_for_backward(sigma)
        ctx.T = T
        return snr

    @staticmethod
    def backward(ctx, gsnr):
        (sigma,) = ctx.saved_tensors
        gsnr = gsnr.to(torch.float64).contiguous()
        S = gsnr.shape[0]
        w = (ctypes.c_int * len(ctx.widths))(*ctx.widths)
        gy = torch.empty((S, ctx.T), dtype=torch.float64, device=gsnr.device)
        if lib().aa_b200_boxcar_snr_adj(gsnr.data_ptr(), S, ctx.T, w, len(ctx.widths), sigma.data_ptr(),
                                        gy.data_ptr(), _stream()):
            raise RuntimeError(_err())
        return gy, None, None, None


def smooth_peak(snr: torch.Tensor, temperature: float = 0.5) -> torch.Tensor:
    """Per-snippet smooth maximum of the S/N over widths and time."""
    return temperature * torch.logsumexp(snr.flatten(1) / temperature, dim=1)


def peak_snr(x, dm, kc, widths=DEFAULT_WIDTHS, mu=None, sigma=None, temperature: float = 0.5, base=None):
    """Smooth peak S/N [S] of snippets x at trial DMs dm (differentiable)."""
    S, C, _ = x.shape
    if mu is None:
        mu = torch.zeros(S, dtype=torch.float32, device=x.device)
    if sigma is None:
        sigma = torch.full((S,), float(np.sqrt(C)), dtype=torch.float32, device=x.device)
    y = FracDedisperse.apply(x, dm, kc, base)
    return smooth_peak(BoxcarSNR.apply(y, tuple(widths), mu, sigma), temperature)


def refine_dm(x, dm0, kc, steps: int = 50, lr: float = 0.05, widths=DEFAULT_WIDTHS, mu=None, sigma=None,
              temperature: float = 0.5, base=None):
    """Adam ascent of the smooth peak S/N in DM, one trial DM per snippet.
    Returns (refined dm [S], peak S/N history [steps+1][S])."""
    dm = dm0.detach().clone().to(torch.float32).contiguous().requires_grad_(True)
    if mu is not None:
        mu = mu.to(torch.float32).contiguous()
    if sigma is not None:
        sigma = sigma.to(torch.float32).contiguous()
    opt = torch.optim.Adam([dm], lr=lr)
    hist = []
    for _ in range(steps):
        opt.zero_grad(set_to_none=True)
        p = peak_snr(x, dm, kc, widths, mu, sigma, temperature, base)
        hist.append(p.detach())
        (-p.sum()).backward()
        opt.step()
    with torch.no_grad():
        hist.append(peak_snr(x, dm, kc, widths, mu, sigma, temperature, base))
    return dm.detach(), torch.stack(hist)


# Synthetic candidate snippets: N(0,1) channels plus one dispersed Gaussian
# pulse.  Band 1670 MHz down 300 MHz, tsamp 128 us, so a pulse at DM 1000
# sweeps about 5650 of the 8192 samples.
SNIPPET_BAND = dict(fch1=1670.0, foff=-300.0 / 1024, tsamp=128e-6)


def synth_snippets(nsnip: int, nchans: int = 1024, nsamp: int = 8192, seed: int = 4, amp: float = 0.35,
                   band=None, device="cuda"):
    """(x [S][C][T] float32, true DM [S], trial DM [S], kc [C]): DM true
    U[100, 1000], width sigma U[0.5, 4] ms, trial DM = true + N(0, 0.5)."""
    band = dict(SNIPPET_BAND, **(band or {}))
    foff = band["foff"] * 1024 / nchans
    kc = delay_per_dm(nchans, band["fch1"], foff, band["tsamp"], device=device)
    rng = np.random.Generator(np.random.PCG64(seed))
    dm_true = rng.uniform(100.0, 1000.0, nsnip)
    width = rng.uniform(0.5e-3, 4e-3, nsnip) / band["tsamp"]
    dm_trial = dm_true + rng.normal(0.0, 0.5, nsnip)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    x = torch.randn((nsnip, nchans, nsamp), generator=g, device=device, dtype=torch.float32)
    t = torch.arange(nsamp, device=device, dtype=torch.float64)
    for s in range(nsnip):
        sweep = float(dm_true[s] * kc[-1])
        t0 = 256.0 + rng.uniform(0.0, max(1.0, nsamp - 512.0 - sweep))
        arrival = t0 + dm_true[s] * kc  # [C]
        pulse = amp * torch.exp(-0.5 * ((t[None, :] - arrival[:, None]) / width[s]) ** 2)
        x[s] += pulse.to(torch.float32)
    return (x, torch.as_tensor(dm_true, dtype=torch.float32, device=device),
            torch.as_tensor(dm_trial, dtype=torch.float32, device=device), kc)
