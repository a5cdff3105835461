"""The FP64 host oracle of the refinement path pinned by finite differences
(no GPU): the analytic adjoints must agree with central differences."""
from __future__ import annotations

import numpy as np
import pytest

import frac_oracle as F

WIDTHS = (1, 2, 4, 8, 16)


def _snippet(C=16, T=256, seed=0):
    rng = np.random.default_rng(seed)
    kc = F.delay_per_dm(C, 1670.0, -300.0 / C, 128e-6)
    x = rng.normal(size=(C, T))
    return x, kc


def _dm_without_crossing(kc, start, h=1e-3):
    for k in range(10000):
        d = start + 0.00731 * k
        if F.no_cell_crossing(d, kc, h):
            return float(np.float32(d))
    pytest.skip("no trial DM without a cell crossing found")


def test_forward_integer_delays_are_plain_shifts():
    x, kc = _snippet()
    kc = np.round(kc * 0) + np.arange(len(kc), dtype=np.float64)  # delay c samples at DM 1
    y = F.frac_forward(x, 1.0, kc)
    want = sum(np.concatenate([x[c, c:], np.zeros(c)]) for c in range(x.shape[0]))
    assert np.allclose(y, want, rtol=0, atol=1e-12)


def test_adjoint_is_the_transpose():
    x, kc = _snippet(seed=1)
    dm = 3.7
    rng = np.random.default_rng(2)
    gy = rng.normal(size=x.shape[1])
    gx, _ = F.frac_adjoint(x, dm, kc, gy)
    u = rng.normal(size=x.shape)
    # <gy, A u> == <A^T gy, u>
    assert np.isclose(np.dot(gy, F.frac_forward(u, dm, kc)), np.sum(gx * u), rtol=1e-12)


def test_dm_gradient_matches_central_difference():
    x, kc = _snippet(seed=3)
    dm = _dm_without_crossing(kc, 7.3)
    rng = np.random.default_rng(4)
    gy = rng.normal(size=x.shape[1])
    _, gdm = F.frac_adjoint(x, dm, kc, gy)
    h = 1e-3
    # frac_forward rounds its DM to float32: evaluate the stencil in FP64
    def y64(d):
        tau = d * kc
        n = np.floor(tau).astype(int)
        w = tau - n
        return sum(F._shift(x[c], n[c]) + w[c] * (F._shift(x[c], n[c] + 1) - F._shift(x[c], n[c]))
                   for c in range(x.shape[0]))
    fd = (np.dot(gy, y64(dm + h)) - np.dot(gy, y64(dm - h))) / (2 * h)
    assert abs(gdm - fd) <= 1e-9 * max(1.0, abs(fd))


def test_boxcar_adjoint_is_the_transpose():
    rng = np.random.default_rng(5)
    y = rng.normal(size=300)
    g = rng.normal(size=(len(WIDTHS), 300))
    u = rng.normal(size=300)
    lhs = np.sum(g * (F.boxcar_forward(u, WIDTHS, 0.0, 2.0) - F.boxcar_forward(np.zeros(300), WIDTHS, 0.0, 2.0)))
    rhs = np.dot(F.boxcar_adjoint(g, WIDTHS, 2.0), u)
    assert np.isclose(lhs, rhs, rtol=1e-12)
    assert F.boxcar_forward(y, WIDTHS, 0.3, 2.0).shape == (len(WIDTHS), 300)


def test_full_loss_gradient_matches_central_difference():
    x, kc = _snippet(C=32, T=512, seed=6)
    x[:, 200:210] += 1.5  # a bright feature so the smooth peak is well defined
    dm = _dm_without_crossing(kc, 2.1)
    L, g = F.loss_and_grad_dm(x, dm, kc, WIDTHS, 0.0, np.sqrt(32), 0.5)
    fd = F.central_difference_dm(x, dm, kc, WIDTHS, 0.0, np.sqrt(32), 0.5, h=1e-3)
    assert np.isfinite(L)
    assert abs(g - fd) <= 1e-5 * max(1e-3, abs(fd))
