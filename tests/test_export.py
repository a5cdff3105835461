"""DM-time output files in the reference's Export_DD_data format
(include/aa_pipeline_runner.hpp:165-223): the library's writer
(aa_b200_export_dd_data) and the oracle restatement against the SHA-256 of
the files the reference's own routine writes for the same outputs
(tests/golden/dmt_golden.json, tests/golden/make_dmt_golden.py)."""
from __future__ import annotations

import ctypes
import hashlib
import json
import os

import pytest

import dmt_cases as D
import dmt_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dmt_golden.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _digests(folder, name):
    return {f[len(name):]: hashlib.sha256(open(os.path.join(folder, f), "rb").read()).hexdigest()
            for f in sorted(os.listdir(folder)) if f.startswith(name + "_")}


@pytest.mark.parametrize("name", list(D.CASES))
def test_writer_matches_reference_export(aa, golden, tmp_path, name):
    per, exp = D.CASES[name]
    rs = D.rows()
    top, keep = D.as_float3(rs)
    L = aa.lib()
    rc = L.aa_b200_export_dd_data(3, ctypes.cast(top, aa.PPPFLOAT), D.MAX_NT, (ctypes.c_int * 3)(*D.NDMS),
                                  (ctypes.c_int * 3)(*D.IN_BIN), os.fsencode(str(tmp_path / name)),
                                  (ctypes.c_int * 3)(*exp), per)
    assert rc == 0, aa.last_error()
    assert _digests(str(tmp_path), name) == golden["cases"][name]


@pytest.mark.parametrize("name", list(D.CASES))
def test_oracle_matches_reference_export(golden, tmp_path, name):
    per, exp = D.CASES[name]
    O.export(D.rows(), D.MAX_NT, D.NDMS, D.IN_BIN, str(tmp_path / name), exp, per)
    assert _digests(str(tmp_path), name) == golden["cases"][name]


def test_files_per_range(aa, golden):
    """per5_range0: 64 DM trials in runs of 5 -> 13 data files and a text file."""
    files = golden["cases"]["per5_range0"]
    assert sum(f.endswith(".dat") for f in files) == 13 and "_0.txt" in files


def test_sd_per_file(aa, golden):
    for key, want in golden["sd_per_file"].items():
        mb, p, k = (int(v) for v in key.split(","))
        assert aa.lib().aa_b200_sd_per_file_from_file_size(mb, p, k) == want == O.sd_per_file(mb, p, k)


def test_zero_rows_per_file_is_refused(aa, tmp_path):
    rs = D.rows()
    top, keep = D.as_float3(rs)
    rc = aa.lib().aa_b200_export_dd_data(3, ctypes.cast(top, aa.PPPFLOAT), D.MAX_NT, (ctypes.c_int * 3)(*D.NDMS),
                                         (ctypes.c_int * 3)(*D.IN_BIN), os.fsencode(str(tmp_path / "z")),
                                         (ctypes.c_int * 3)(1, 1, 1), 0)
    assert rc == 1 and "0" in aa.last_error()


def test_unwritable_folder_is_an_error(aa, tmp_path):
    rs = D.rows()
    top, keep = D.as_float3(rs)
    rc = aa.lib().aa_b200_export_dd_data(3, ctypes.cast(top, aa.PPPFLOAT), D.MAX_NT, (ctypes.c_int * 3)(*D.NDMS),
                                         (ctypes.c_int * 3)(*D.IN_BIN),
                                         os.fsencode(str(tmp_path / "missing" / "x")), (ctypes.c_int * 3)(1, 1, 1), 48)
    assert rc == 1 and "cannot write" in aa.last_error()
