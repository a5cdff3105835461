"""Periodicity candidate lists (the reference's aa_periodicity_candidates):
the library's conversion and the restatement bit for bit against the
reference's own host code on seeded records
(tests/golden/psr_candidates_golden.json), and the list's order, copy and
export."""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import pytest

import psr_cases as P
import psr_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "psr_candidates_golden.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)["cases"]


def _args(c):
    return c["dm_low"], c["dm_step"], c["tsamp"], c["nt"], c["mod"], c["greedy"]


@pytest.mark.parametrize("name", list(P.CANDIDATE_CASES))
def test_library_conversion_matches_reference(aa, golden, name):
    c = P.CANDIDATE_CASES[name]
    g = golden[name]
    assert g["rc"] == 0
    rec, msd = P.make_candidate_records(c)
    assert aa.lib().aa_b200_psr_candidates_process(rec.ctypes.data, c["n"], msd.ctypes.data, *_args(c)) == 0
    assert rec[:64].view(np.uint32).tolist() == g["head"]
    assert hashlib.sha256(rec.tobytes()).hexdigest() == g["sha256"]


@pytest.mark.parametrize("name", list(P.CANDIDATE_CASES))
def test_oracle_conversion_matches_reference(golden, name):
    c = P.CANDIDATE_CASES[name]
    rec, msd = P.make_candidate_records(c)
    r = O.candidates_process(rec, msd, *_args(c))
    assert hashlib.sha256(np.ascontiguousarray(r).tobytes()).hexdigest() == golden[name]["sha256"]


def test_greedy_offsets_become_frequency_corrections():
    """A greedy count 3 + 100 * 2 is 3 harmonics with a correction of 2/3 of
    a bin width; the non-greedy reading keeps the count as it is."""
    msd = np.array([0, 1] * 8, np.float32)
    rec = np.array([[4, 1000, 10, 203]], np.float32)
    g = O.candidates_process(rec, msd, 0.0, 1.0, 1e-3, 1000, 1.0, 1)
    assert g[0, 3] == 3
    assert np.isclose(g[0, 1], 1000 / (1e-3 * 1000) + (2 / 3) * (1 / 1e-3) / 1000, rtol=1e-6)


def test_list_accumulates_copies_and_exports(aa, tmp_path):
    L = aa.lib()
    lst = L.aa_b200_psr_candidates_create()
    parts = []
    try:
        for name in ["cands_power", "cands_greedy", "cands_interbin"]:
            c = P.CANDIDATE_CASES[name]
            rec, msd = P.make_candidate_records(c)
            assert L.aa_b200_psr_candidates_add(lst, rec.ctypes.data, c["n"], 0, len(parts), msd.ctypes.data,
                                                *_args(c)) == 0
            parts.append(O.candidates_process(rec, msd, *_args(c)))
        assert L.aa_b200_psr_candidates_add(lst, None, 0, 0, 9, None, 0.0, 1.0, 1e-3, 8, 1.0, 0) == 0
        want = np.concatenate(parts)
        assert L.aa_b200_psr_candidates_count(lst) == len(want)
        got = np.zeros_like(want)
        assert L.aa_b200_psr_candidates_copy(lst, got.ctypes.data) == 0
        assert got.view(np.uint32).tolist() == want.view(np.uint32).tolist()
        path = tmp_path / "psr_candidates.dat"
        assert L.aa_b200_psr_candidates_export(lst, str(path).encode()) == 0
        assert np.fromfile(path, np.float32).reshape(-1, 4).view(np.uint32).tolist() == want.view(np.uint32).tolist()
        assert L.aa_b200_psr_candidates_export(lst, str(tmp_path / "missing" / "x.dat").encode()) == 1
        assert b"cannot open" in L.aa_b200_psr_candidates_last_error()
        assert L.aa_b200_psr_candidates_add(lst, None, 5, 0, 0, None, 0.0, 1.0, 1e-3, 8, 1.0, 0) == 1
    finally:
        L.aa_b200_psr_candidates_destroy(lst)


@pytest.mark.gpu
def test_list_adds_device_records(aa, golden):
    """Records in device memory (as the periodicity peak finding leaves
    them) give the reference's conversion."""
    import torch
    c = P.CANDIDATE_CASES["cands_greedy_interbin"]
    rec, msd = P.make_candidate_records(c)
    d = torch.from_numpy(rec.copy()).cuda()
    L = aa.lib()
    lst = L.aa_b200_psr_candidates_create()
    try:
        assert L.aa_b200_psr_candidates_add(lst, d.data_ptr(), c["n"], 1, 0, msd.ctypes.data, *_args(c)) == 0
        got = np.zeros_like(rec)
        assert L.aa_b200_psr_candidates_copy(lst, got.ctypes.data) == 0
        assert hashlib.sha256(got.tobytes()).hexdigest() == golden["cands_greedy_interbin"]["sha256"]
    finally:
        L.aa_b200_psr_candidates_destroy(lst)
