"""The CPU oracle on its own: the reference's known-answer tests, its pieces
against direct numpy restatements, and its agreement with the reference GPU
output (golden vectors).  Host only."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

import cases as C


def test_fake_signal_known_answer(oracle_mod):
    """tests/test_ddtr_fakesignal_single.cpp:109-117: the dedispersed pulse of
    the fake-signal generator is exactly 255 at (DM, start); fixed seeds."""
    rng = np.random.Generator(np.random.PCG64(31))
    s = oracle_mod.strategy([(0, 250.0, 1, 1, 1)], 128, 31250, 1550.0, -300 / 128, 6.4e-5, 8, 180 * 2**30)
    for _ in range(6):
        dm = float(int(rng.integers(0, 200)))
        st = int(rng.integers(0, 10)) * 1000 + int(rng.integers(0, 10)) * 100 + int(rng.integers(0, 10)) * 10
        x, _ = oracle_mod.fake_signal(128, 31250, 6.4e-5, s.dmshifts, s.maxshift, dm, 625, st, 0.5)
        outs, kern = oracle_mod.run_ddtr(x, s, 128, 31250, 6.4e-5, 8)
        assert kern[0][0] == oracle_mod.K_CACHE
        assert outs[0][int(dm), st] == 255.0


def test_fake_signal_periodic_known_answer(oracle_mod):
    """tests/test_ddtr_fakesignal_period.cpp:88-131: every pulse of a periodic
    train is exactly 255 at its (DM, start)."""
    tsamp = 6.4e-5
    nsamp = int(1.5 / tsamp)
    s = oracle_mod.strategy([(0, 120, 1, 1, 1)], 128, nsamp, 1550.0, -300 / 128, tsamp, 8, 180 * 2**30)
    period, dm = 137, 42.0
    x, mp = oracle_mod.fake_signal(128, nsamp, tsamp, s.dmshifts, s.maxshift, dm, int(1 / (tsamp * 25)), 0, 0.5,
                                   period_ms=period)
    outs, _ = oracle_mod.run_ddtr(x, s, 128, nsamp, tsamp, 8)
    start = -mp - 2 * s.maxshift
    step = int(period / 1000.0 / tsamp)
    while start < 0:
        start += step
    n = 0
    while start + s.maxshift < nsamp and start < outs[0].shape[1]:
        assert outs[0][int(dm), start] == 255.0
        start += step
        n += 1
    assert n >= 3


def test_corner_turn(oracle_mod):
    x = np.random.default_rng(0).integers(0, 65535, size=(300, 37), dtype=np.uint16)
    ct = oracle_mod.corner_turn(x, 37, 300)
    assert np.array_equal(ct.reshape(37, 300), x.T)


def test_binning_flat_semantics(oracle_mod):
    """src/aa_bin_gpu.cpp:8-44 on the flat buffer: first nchans*nsamp/2
    elements are (a+b)>>1 of [c][nsamp] pairs, the rest of nchans*nsamp is
    zero, everything beyond is untouched."""
    rng = np.random.default_rng(1)
    nch, ns = 64, 96
    buf = rng.integers(0, 255, size=nch * ns + 50, dtype=np.uint16)
    out = oracle_mod.bin_flat(buf, nch, ns)
    a = buf[:nch * ns].reshape(nch, ns).astype(np.uint32)
    want = ((a[:, 0::2] + a[:, 1::2]) >> 1).astype(np.uint16).reshape(-1)
    assert np.array_equal(out[:nch * ns // 2], want)
    assert not out[nch * ns // 2:nch * ns].any()
    assert np.array_equal(out[nch * ns:], buf[nch * ns:])


def test_cache_kernel_is_plain_shift_and_sum(oracle_mod):
    """Cache-kernel semantics against a direct numpy shift-and-sum."""
    rng = np.random.default_rng(2)
    nch, ns, tp, ndms = 16, 400, 256, 8
    flat = rng.integers(0, 255, size=nch * ns, dtype=np.uint16)
    shifts = np.linspace(0, 0.01, nch).astype(np.float32)
    ms, st = np.float32(0.0), np.float32(100.0)
    out, sums = oracle_mod.dedisperse(oracle_mod.K_CACHE, oracle_mod.FMA_ALL, flat, ns, nch, tp, ndms, shifts, ms, st,
                                      1, want_sums=True)
    x = flat.reshape(nch, ns).astype(np.int64)
    for d in range(ndms):
        delays = [oracle_mod.delay(oracle_mod.K_CACHE, oracle_mod.FMA_ALL, float(shifts[c]), d, 0, ms, st)
                  for c in range(nch)]
        want = sum(x[c, delays[c]:delays[c] + tp] for c in range(nch))
        assert np.array_equal(sums[d], want)


def test_shared_kernel_delay_classes(oracle_mod):
    """Shared-kernel delay: per-block base plus a per-thread shift that can
    differ between thread classes by one sample, never more."""
    rng = np.random.default_rng(3)
    for _ in range(2000):
        dms = np.float32(rng.uniform(0, 2e-3))
        m0, st = np.float32(rng.uniform(0, 2000)), np.float32(rng.uniform(100, 5000))
        dm = int(rng.integers(0, 512))
        for kern in (oracle_mod.K_SHARED8, oracle_mod.K_SHARED16, oracle_mod.K_SHARED4):
            d = [oracle_mod.delay(kern, oracle_mod.FMA_ALL, float(dms), dm, tx, float(m0), float(st)) for tx in range(8)]
            assert max(d) - min(d) <= 1 and min(d) >= 0


@pytest.mark.parametrize("name", [n for n, c in C.CASES.items() if not c.get("heavy")])
def test_oracle_matches_reference_gpu(oracle_mod, golden_ddtr, name):
    """The oracle reproduces the reference's own GPU output bit for bit when
    nchans*bin is a power of two (fast-math division is exact there)."""
    if name not in golden_ddtr:
        pytest.skip("case not in the golden file")
    case = C.CASES[name]
    rec = golden_ddtr[name]
    x = C.make_input(case)
    s = oracle_mod.strategy(case["plan"], case["nchans"], case["nsamp"], case["fch1"], case["foff"], case["tsamp"],
                            case["nbits"], C.strategy_free_memory(case))
    assert s.t_processed == rec["strategy"]["t_processed"]
    outs, kern = oracle_mod.run_ddtr(x, s, case["nchans"], case["nsamp"], case["tsamp"], case["nbits"])
    for r, rr in enumerate(rec["ranges"]):
        div = case["nchans"] * (1 if kern[r][0] == oracle_mod.K_SHARED4 else s.dm[r][3])
        if div & (div - 1) == 0:
            assert hashlib.sha256(outs[r].tobytes()).hexdigest() == rr["sha256"], f"range {r}"
        else:
            for i, j, bits in rr["samples"]:
                ref = np.uint32(bits).view(np.float32)
                if abs(float(ref) * div) < 2**24:  # integer sums; fp32 sums of 16-bit data above 2^24 are rounded
                    assert np.rint(float(outs[r][i, j]) * div) == np.rint(float(ref) * div)
                assert abs(int(outs[r][i, j].view(np.int32)) - int(np.int32(bits))) <= 2


@pytest.mark.parametrize("name", ["shared8_binned", "shared4", "cache16"])
def test_windowed_dedispersion_equals_whole_range(oracle_mod, name):
    """aao_dedisperse_window (the bench's in-run parity check) gives the same
    bits as the whole-range oracle for a DM block and a time window, on the
    whole buffer and on a buffer that starts inside the channel rows."""
    O = oracle_mod
    case = C.CASES[name]
    x = C.make_input(case)
    s = O.strategy(case["plan"], case["nchans"], case["nsamp"], case["fch1"], case["foff"], case["tsamp"],
                   case["nbits"], C.strategy_free_memory(case))
    d = s.dm[0]
    tsr = np.float32(case["tsamp"]) * np.float32(d[3])
    kind = O.select_kernel(case["nbits"], d[2], tsr, s.dmshifts[-1])
    m0, ms = np.float32(np.float32(d[0]) / tsr), np.float32(np.float32(d[2]) / tsr)
    tp = s.t_processed[0][0]
    L = tp + s.maxshift
    nch = case["nchans"]
    full = O.dedisperse(kind, O.FMA_ALL, O.corner_turn(x[:L], nch, L), L, nch, tp, s.ndms[0], s.dmshifts, m0, ms,
                        d[3])
    dm0 = 64 * (s.ndms[0] // 64 - 1)
    t0, nt = 96, tp - 96 - 64
    w = O.dedisperse_window(kind, O.FMA_ALL, O.corner_turn(x[:L], nch, L), L, nch, dm0, 64, t0, nt, s.dmshifts, m0,
                            ms, d[3])
    assert np.array_equal(w.view(np.uint32), full[dm0:dm0 + 64, t0:t0 + nt].view(np.uint32))
    sh = 64
    w2 = O.dedisperse_window(kind, O.FMA_ALL, O.corner_turn(x[sh:L], nch, L - sh), L - sh, nch, dm0, 64, t0, nt,
                             s.dmshifts, m0, ms, d[3], t_shift=sh)
    assert np.array_equal(w2.view(np.uint32), full[dm0:dm0 + 64, t0:t0 + nt].view(np.uint32))


@pytest.mark.parametrize("name", [n for n, c in C.CASES.items() if c.get("heavy")])
def test_oracle_matches_reference_gpu_samples_of_heavy_cases(oracle_mod, golden_ddtr, name):
    """The cases too large for a whole oracle run here: the oracle's value at
    each of the golden file's sampled outputs (DM trial, sample) of the
    single-chunk, unbinned ranges equals the reference GPU's bit for bit."""
    if name not in golden_ddtr:
        pytest.skip("case not in the golden file")
    case = C.CASES[name]
    rec = golden_ddtr[name]
    x = C.make_input(case)
    s = oracle_mod.strategy(case["plan"], case["nchans"], case["nsamp"], case["fch1"], case["foff"], case["tsamp"],
                            case["nbits"], C.strategy_free_memory(case))
    assert s.t_processed == rec["strategy"]["t_processed"]
    if s.num_tchunks != 1:
        pytest.skip("sampled check covers single-chunk cases")
    L = s.t_processed[0][0] + s.maxshift
    flat = oracle_mod.corner_turn(x[:L], case["nchans"], L)
    checked = 0
    for r, rr in enumerate(rec["ranges"]):
        d = s.dm[r]
        if d[3] != 1:
            continue
        tsr = np.float32(case["tsamp"]) * np.float32(d[3])
        kind = oracle_mod.select_kernel(case["nbits"], d[2], tsr, s.dmshifts[-1])
        m0, ms = np.float32(np.float32(d[0]) / tsr), np.float32(np.float32(d[2]) / tsr)
        for i, j, bits in rr["samples"]:
            v = oracle_mod.dedisperse_window(kind, oracle_mod.FMA_ALL, flat, L, case["nchans"], i, 1, j, 1,
                                             s.dmshifts, m0, ms, d[3])
            assert int(v[0, 0].view(np.uint32)) == bits, (r, i, j)
            checked += 1
    assert checked > 0
