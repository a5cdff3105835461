"""The seeded multi-beam draw and the wave split (host only)."""
from __future__ import annotations

import math

from aa_b200 import workloads as WL


def test_multibeam_draw_follows_its_definition():
    beams = WL.multibeam_draw(seed=3, nbeams=48)
    assert len(beams) == 48
    assert beams == WL.multibeam_draw(seed=3, nbeams=48)  # seeded
    for b in beams:
        assert 2048 <= b["nchans"] <= 4096
        assert b["nbits"] in (4, 8, 16)
        assert 2 ** 16 - 1 <= b["nsamp"] <= 2 ** 21 + 1
        assert abs(b["foff"] * b["nchans"] + 300.0) < 1e-9
        assert 1 <= len(b["plan"]) <= 6
        for p, q in zip(b["plan"], WL.SURVEY_PLAN):
            assert (p[0], p[2], p[3]) == (q[0], q[2], q[3])
            assert p[1] <= q[1]
        assert b["plan"][-1][0] < b["plan"][-1][1] <= 3000
    assert {b["nbits"] for b in beams} == {4, 8, 16}
    mean_log = sum(math.log2(b["nsamp"]) for b in beams) / len(beams)
    assert 17.5 < mean_log < 19.5


def test_plan_waves_respects_budget():
    sizes = [5, 3, 8, 2, 9, 1, 4]
    waves = WL.plan_waves(sizes, 10)
    assert sorted(i for w in waves for i in w) == list(range(len(sizes)))
    for w in waves:
        assert sum(sizes[i] for i in w) <= 10 or len(w) == 1
    assert WL.plan_waves([20], 10) == [[0]]
