"""Single-pulse candidates from the DM-time output and snippets for refinement.

The S/N kernels are csrc/sps.cu (through the C ABI); the selection of the
strongest candidates and the cutting of per-channel snippets run on the GPU
with torch indexing.  A candidate is (S/N, DM, arrival sample at the top of
the band in native samples, boxcar width in native samples).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import lib

DEFAULT_WIDTHS = (1, 2, 4, 8, 16, 32, 64)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _err():
    return lib().aa_b200_frac_last_error().decode()


def range_peaks(rows: torch.Tensor, nsamp: int, widths=DEFAULT_WIDTHS):
    """Per (DM row, block) peak S/N, start sample and width of a [ndms][pitch]
    float32 CUDA tensor whose first nsamp columns are valid."""
    if rows.dtype != torch.float32 or not rows.is_cuda or rows.stride(1) != 1:
        raise ValueError("rows must be a float32 CUDA tensor with unit column stride")
    ndms, pitch = rows.shape[0], rows.stride(0)
    mean = torch.empty(ndms, device=rows.device)
    std = torch.empty(ndms, device=rows.device)
    if lib().aa_b200_sps_row_stats(rows.data_ptr(), ndms, pitch, nsamp, mean.data_ptr(), std.data_ptr(), _stream()):
        raise RuntimeError(_err())
    nb = (nsamp + lib().aa_b200_sps_block_samples() - 1) // lib().aa_b200_sps_block_samples()
    snr = torch.empty((ndms, nb), device=rows.device)
    t = torch.empty((ndms, nb), dtype=torch.int32, device=rows.device)
    w = torch.empty((ndms, nb), dtype=torch.int32, device=rows.device)
    wa = (ctypes.c_int * len(widths))(*widths)
    if lib().aa_b200_sps_block_peaks(rows.data_ptr(), ndms, pitch, nsamp, mean.data_ptr(), std.data_ptr(), wa,
                                     len(widths), snr.data_ptr(), t.data_ptr(), w.data_ptr(), _stream()):
        raise RuntimeError(_err())
    return snr, t, w


def candidates(rows, nsamp, dm_low, dm_step, inbin, threshold=6.0, widths=DEFAULT_WIDTHS):
    """Block peaks of one range at or above the threshold, in native samples:
    dict of tensors snr, dm, t, w."""
    snr, t, w = range_peaks(rows, nsamp, widths)
    keep = snr >= threshold
    idx = keep.nonzero()
    dm = dm_low + idx[:, 0].to(torch.float64) * dm_step
    return {"snr": snr[keep], "dm": dm.to(torch.float32), "t": t[keep].to(torch.int64) * inbin,
            "w": w[keep].to(torch.int64) * inbin}


def select(cands: list, k: int = 64, separation: int = 4096) -> dict:
    """The k strongest events among the candidates of several ranges.  The
    same pulse is seen at many neighbouring DMs, so candidates are first
    reduced to the strongest per time bin of `separation` native samples (on
    the GPU); the bin winners are then taken strongest first, skipping one
    that arrives within `separation` samples of a stronger one already kept."""
    if not cands:
        return {"snr": torch.empty(0), "dm": torch.empty(0), "t": torch.empty(0, dtype=torch.int64),
                "w": torch.empty(0, dtype=torch.int64)}
    allc = {key: torch.cat([c[key] for c in cands]) for key in ("snr", "dm", "t", "w")}
    if allc["snr"].numel() == 0:
        return allc
    dev = allc["snr"].device
    # strongest candidate per time bin: sort by S/N, then a stable sort by bin
    # leaves each bin's strongest first
    order = torch.argsort(allc["snr"], descending=True, stable=True)
    bins = torch.div(allc["t"][order], separation, rounding_mode="floor")
    by_bin = torch.argsort(bins, stable=True)
    sb = bins[by_bin]
    first = torch.ones_like(sb, dtype=torch.bool)
    first[1:] = sb[1:] != sb[:-1]
    winners = order[by_bin[first]]
    winners = winners[torch.argsort(allc["snr"][winners], descending=True, stable=True)]
    t = allc["t"][winners].cpu().numpy()
    kept = []
    for i in range(len(winners)):
        if len(kept) == k:
            break
        if all(abs(int(t[i]) - int(t[j])) >= separation for j in kept):
            kept.append(i)
    sel = winners[torch.as_tensor(np.array(kept, dtype=np.int64), device=dev)]
    return {key: v[sel] for key, v in allc.items()}


def cut_snippets(x_tc: torch.Tensor, kc: torch.Tensor, dm: torch.Tensor, t: torch.Tensor, w: torch.Tensor,
                 nwin: int = 1024, offset: float = 127.5, scale: float = 16.0):
    """Per-channel windows of the raw input x_tc [nsamp][nchans] (uint16 bit
    patterns in int16) around each candidate, aligned at its DM:
    snippet[k][c][i] = (x[s0_k + base_kc + i][c] - offset) / scale with
    s0 = t + w/2 - nwin/2 and base_kc = floor(dm_k * kc_c); samples outside the
    input read as offset.  Returns (snippets [K][C][nwin] float32, base [K][C] int32)."""
    nsamp, nch = x_tc.shape
    K = int(dm.shape[0])
    base = torch.floor(dm.to(torch.float64)[:, None] * kc[None, :]).to(torch.int64)  # [K][C]
    s0 = (t + w // 2 - nwin // 2).to(torch.int64)
    out = torch.empty((K, nch, nwin), dtype=torch.float32, device=x_tc.device)
    ar = torch.arange(nwin, device=x_tc.device, dtype=torch.int64)
    cidx = torch.arange(nch, device=x_tc.device, dtype=torch.int64)
    for k in range(K):
        rows = s0[k] + base[k][:, None] + ar[None, :]  # [C][nwin]
        ok = (rows >= 0) & (rows < nsamp)
        v = x_tc[rows.clamp(0, nsamp - 1), cidx[:, None]].to(torch.int32) & 0xFFFF
        out[k] = torch.where(ok, (v.to(torch.float32) - offset) / scale, torch.zeros((), device=x_tc.device))
    return out, base.to(torch.int32)
