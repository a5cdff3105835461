"""Strategy parity: the CPU oracle and this library's planner against the
reference's own aa_ddtr_strategy (golden vectors from
tests/golden/make_strategy_golden.py).  Host only."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest


def _cases(golden_strategy):
    return golden_strategy["cases"]


def _check(rec, got):
    if rec["refused"]:
        assert got is None, "the reference refused this plan"
        return
    assert got is not None, "the reference accepted this plan"
    assert hashlib.sha256(np.asarray(got["dmshifts"], np.float32).tobytes()).hexdigest() == rec["dmshifts_sha256"]
    assert got["ndms"] == rec["ndms"]
    assert [list(map(float, d[:3])) + [int(d[3]), int(d[4])] for d in got["dm"]] == \
        [list(map(float, d[:3])) + [int(d[3]), int(d[4])] for d in rec["dm"]]
    assert got["maxshift"] == rec["maxshift"]
    assert got["max_ndms"] == rec["max_ndms"]
    assert got["num_tchunks"] == rec["num_tchunks"]
    assert got["t_processed"] == rec["t_processed"]


def test_oracle_strategy_matches_reference(oracle_mod, golden_strategy):
    n = 0
    for rec in _cases(golden_strategy):
        try:
            s = oracle_mod.strategy([tuple(p) for p in rec["plan"]], rec["nchans"], rec["nsamp"], rec["fch1"],
                                    rec["foff"], rec["tsamp"], rec["nbits"], rec["free_memory"], rec["power"],
                                    bool(rec["analysis"]))
            got = dict(dmshifts=s.dmshifts, ndms=s.ndms, dm=[list(d) for d in s.dm], maxshift=s.maxshift,
                       max_ndms=s.max_ndms, num_tchunks=s.num_tchunks, t_processed=s.t_processed)
        except ValueError:
            got = None
        _check(rec, got)
        n += 1
    assert n >= 100


def test_planner_matches_reference(aa, golden_strategy):
    for rec in _cases(golden_strategy):
        try:
            got = aa.strategy([tuple(p) for p in rec["plan"]], rec["nchans"], rec["nsamp"], rec["fch1"], rec["foff"],
                              rec["tsamp"], rec["nbits"], rec["free_memory"], rec["power"], bool(rec["analysis"]))
        except ValueError:
            got = None
        _check(rec, got)


def test_survey_configs_strategy(aa):
    """The survey-scale plan on 4096 channels x 2^21 samples: 8 ranges,
    maxshift 36064, three chunks (the values the reference computes)."""
    import cases as C
    s = aa.strategy(C.SURVEY_PLAN, 4096, 1 << 21, 1670.0, -0.0732421875, 64e-6, 8)
    assert s["ndms"] == [1536, 768, 832, 1024, 512, 384, 512, 512]
    assert s["maxshift"] == 36064
    assert s["num_tchunks"] == 3
    assert s["t_processed"][0] == [1012480, 1012480, 35840]
    s1 = aa.strategy([(0, 500, 0.5, 1, 1)], 1024, 1 << 18, 1550.0, -0.390625, 64e-6, 8)
    assert s1["ndms"] == [1024] and s1["maxshift"] == 11489 and s1["t_processed"] == [[250432]]


@pytest.mark.parametrize("nbits,step,expect", [(8, 0.1, 0), (8, 0.5, 3), (16, 0.1, 1), (4, 0.05, 2), (4, 0.2, 3),
                                               (8, 0.1, 3)])
def test_kernel_selection(aa, oracle_mod, nbits, step, expect):
    """src/aa_dedisperse.cpp lineshift rule, 4096-channel survey band."""
    s = aa.strategy([(0, 50, step, 1, 1)], 4096, 1 << 20, 1670.0, -0.0732421875, 64e-6, nbits)
    failsafe = 1 if (nbits, step, expect) == (8, 0.1, 3) else 0
    ts = np.float32(64e-6)
    k = aa.select_kernel(nbits, step, ts, s["dmshifts"][-1], failsafe)
    assert k == oracle_mod.select_kernel(nbits, step, ts, s["dmshifts"][-1], failsafe) == expect
