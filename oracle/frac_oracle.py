"""FP64 host oracle of the differentiable refinement path (test infrastructure).

The reference has no fractional-delay dedisperser and no differentiable S/N,
so there is nothing of it to replay: this file restates the functions the
B200 kernels compute (astro-accelerate_b200/csrc/frac.cu) in float64 numpy,
with their analytic gradients, and the central finite differences that pin
those gradients.  Only tests/, __graft_entry__.smoke() and bench.py's
baseline leg use it.

    tau_c = dm * kc_c, n_c = floor(tau_c) - base_c, w_c = tau_c - floor(tau_c)
    y[t]  = sum_c x[c][t+n_c] + w_c (x[c][t+n_c+1] - x[c][t+n_c])   (0 outside [0, T))
    snr[i][t] = (sum_{k<w_i} y'[t+k] - w_i mu) / (sigma sqrt(w_i)),  y' = mu beyond T
"""
from __future__ import annotations

import numpy as np

DISPERSION_CONSTANT = 4.148808e3  # s MHz^2 / (pc cm^-3)


def delay_per_dm(nchans: int, fch1: float, foff: float, tsamp: float) -> np.ndarray:
    """kc_c: delay of channel c relative to fch1, in samples per unit DM (float64)."""
    f = fch1 + foff * np.arange(nchans, dtype=np.float64)
    return DISPERSION_CONSTANT * (f ** -2 - fch1 ** -2) / tsamp


def _shift(row: np.ndarray, n: int) -> np.ndarray:
    """out[t] = row[t + n], 0 outside the row."""
    T = row.shape[-1]
    out = np.zeros(T, dtype=np.float64)
    lo, hi = max(0, -n), min(T, T - n)
    if hi > lo:
        out[lo:hi] = row[lo + n:hi + n]
    return out


def frac_forward(x: np.ndarray, dm: float, kc: np.ndarray, base=None) -> np.ndarray:
    """y[T] for one snippet x[C][T]; base[C]: integer row shifts (or None)."""
    x = np.asarray(x, dtype=np.float64)
    tau = float(np.float32(dm)) * kc
    w = tau - np.floor(tau)
    n = np.floor(tau).astype(np.int64) - (0 if base is None else np.asarray(base, np.int64))
    y = np.zeros(x.shape[1], dtype=np.float64)
    for c in range(x.shape[0]):
        a0 = _shift(x[c], int(n[c]))
        a1 = _shift(x[c], int(n[c]) + 1)
        y += a0 + w[c] * (a1 - a0)
    return y


def frac_adjoint(x: np.ndarray, dm: float, kc: np.ndarray, gy: np.ndarray, base=None):
    """(gx[C][T], gdm) for one snippet."""
    x = np.asarray(x, dtype=np.float64)
    gy = np.asarray(gy, dtype=np.float64)
    tau = float(np.float32(dm)) * kc
    w = tau - np.floor(tau)
    n = np.floor(tau).astype(np.int64) - (0 if base is None else np.asarray(base, np.int64))
    gx = np.zeros_like(x)
    gdm = 0.0
    for c in range(x.shape[0]):
        gx[c] = (1.0 - w[c]) * _shift(gy, -int(n[c])) + w[c] * _shift(gy, -int(n[c]) - 1)
        a0 = _shift(x[c], int(n[c]))
        a1 = _shift(x[c], int(n[c]) + 1)
        gdm += kc[c] * float(np.dot(gy, a1 - a0))
    return gx, gdm


def boxcar_forward(y: np.ndarray, widths, mu: float, sigma: float) -> np.ndarray:
    y = np.asarray(y, dtype=np.float64)
    T = y.shape[0]
    wmax = max(widths)
    yp = np.concatenate([y, np.full(wmax, mu)])
    c = np.concatenate([[0.0], np.cumsum(yp)])
    t = np.arange(T)
    return np.stack([(c[t + w] - c[t] - w * mu) / (sigma * np.sqrt(w)) for w in widths])


def boxcar_adjoint(gsnr: np.ndarray, widths, sigma: float) -> np.ndarray:
    gsnr = np.asarray(gsnr, dtype=np.float64)
    T = gsnr.shape[1]
    gy = np.zeros(T)
    for i, w in enumerate(widths):
        g = gsnr[i] / (sigma * np.sqrt(w))
        c = np.concatenate([[0.0], np.cumsum(g)])
        t = np.arange(T)
        gy += c[t + 1] - c[np.maximum(t + 1 - w, 0)]
    return gy


def smooth_peak(snr: np.ndarray, temperature: float) -> float:
    """temperature * logsumexp(snr / temperature): a smooth maximum."""
    z = np.asarray(snr, dtype=np.float64).ravel() / temperature
    m = z.max()
    return temperature * (m + np.log(np.exp(z - m).sum()))


def smooth_peak_grad(snr: np.ndarray, temperature: float) -> np.ndarray:
    z = np.asarray(snr, dtype=np.float64) / temperature
    e = np.exp(z - z.max())
    return e / e.sum()


def loss_and_grad_dm(x, dm, kc, widths, mu, sigma, temperature):
    """Smooth peak S/N of one snippet and its derivative in DM (analytic, FP64)."""
    y = frac_forward(x, dm, kc)
    snr = boxcar_forward(y, widths, mu, sigma)
    L = smooth_peak(snr, temperature)
    gy = boxcar_adjoint(smooth_peak_grad(snr, temperature), widths, sigma)
    _, gdm = frac_adjoint(x, dm, kc, gy)
    return L, gdm


def central_difference_dm(x, dm, kc, widths, mu, sigma, temperature, h=1e-3):
    """Central finite difference of the smooth peak S/N in DM, in FP64 with
    delays evaluated at dm +- h (no float32 rounding of the trial DM)."""
    def L_at(d):
        x64 = np.asarray(x, dtype=np.float64)
        tau = d * kc
        n = np.floor(tau).astype(np.int64)
        w = tau - n
        y = np.zeros(x64.shape[1])
        for c in range(x64.shape[0]):
            a0 = _shift(x64[c], int(n[c]))
            a1 = _shift(x64[c], int(n[c]) + 1)
            y += a0 + w[c] * (a1 - a0)
        return smooth_peak(boxcar_forward(y, widths, mu, sigma), temperature)
    d0 = float(np.float32(dm))
    return (L_at(d0 + h) - L_at(d0 - h)) / (2 * h)


def no_cell_crossing(dm, kc, h=1e-3) -> bool:
    """True when no channel's delay crosses an integer within dm +- h (the
    interpolated function is then linear in DM on the whole stencil)."""
    d0 = float(np.float32(dm))
    return bool(np.all(np.floor((d0 - h) * kc) == np.floor((d0 + h) * kc)))
