"""SIGPROC filterbank reader (include/aa_b200.h aa_py_sigproc_input*,
aa_b200_sigproc_*) on the host: metadata and unpacked samples against what
the reference's own reader returns (tests/golden/sigproc_golden.json, made by
tests/golden/make_sigproc_golden.py from src/aa_sigproc_input.cpp), the
oracle restatement against the same vectors, the packed read, and the files
the library refuses."""
from __future__ import annotations

import hashlib
import json
import os
import struct

import numpy as np
import pytest

import sigproc_cases as S
import sigproc_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sigproc_golden.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def writer(aa):
    from aa_b200.sigproc import write_filterbank
    return write_filterbank


def _file(tmp_path, name, writer):
    path = str(tmp_path / (name + ".fil"))
    S.write_case(S.CASES[name], path, writer)
    return path


@pytest.mark.parametrize("name", list(S.CASES))
def test_reader_matches_reference_reader(aa, golden, writer, tmp_path, name):
    path = _file(tmp_path, name, writer)
    g = golden[name]
    r = aa.aa_py_sigproc_input(path)
    m = r.read_metadata()
    assert (m.m_nbits, m.m_nsamples, m.m_nchans) == (g["meta"]["nbits"], g["meta"]["nsamples"], g["meta"]["nchans"])
    assert (m.m_tstart, m.m_tsamp, m.m_fch1, m.m_foff) == (g["meta"]["tstart"], g["meta"]["tsamp"],
                                                            g["meta"]["fch1"], g["meta"]["foff"])
    assert r.read_signal(), r.last_error()
    assert not r.read_signal()  # once, as aa_sigproc_input::read_signal
    buf = r.input_array()
    assert buf.size == g["elements"]
    assert hashlib.sha256(buf.tobytes()).hexdigest() == g["sha256"]
    r.delete()


@pytest.mark.parametrize("name", list(S.CASES))
def test_oracle_matches_reference_reader(golden, writer, tmp_path, name):
    path = _file(tmp_path, name, writer)
    meta, buf = O.read(path)
    g = golden[name]
    for k in ("nbits", "nsamples", "nchans", "tsamp", "fch1", "foff", "tstart"):
        assert meta[k] == g["meta"][k], k
    assert hashlib.sha256(buf.tobytes()).hexdigest() == g["sha256"]


@pytest.mark.parametrize("name", list(S.CASES))
def test_packed_read_is_the_stored_data(aa, writer, tmp_path, name):
    case = S.CASES[name]
    path = _file(tmp_path, name, writer)
    r = aa.aa_py_sigproc_input(path)
    m = r.read_metadata()
    h = r.header()
    assert r.read_packed(), r.last_error()
    p = r.packed_array()
    blob = open(path, "rb").read()
    assert h["data_start"] == O.parse_header(blob)[1]
    assert h["nsamp"] == m.m_nsamples == case["nsamp"]
    if case["nbits"] == 32:
        assert p.dtype == np.uint16 and p.shape == (case["nsamp"], case["nchans"])
        assert np.array_equal(p, O.read(path)[1])  # the 16-bit rescaled samples
    else:
        nrec = case["nchans"] * case["nbits"] // 8
        stored = np.frombuffer(blob, np.uint8, offset=h["data_start"])[:case["nsamp"] * nrec]
        assert np.array_equal(p.view(np.uint8).reshape(-1), stored)
        assert np.array_equal(O.unpack(p.view(np.uint8).reshape(-1), case["nbits"], case["nchans"], case["nsamp"]),
                              S.make_data(case))


def test_header_values(aa, writer, tmp_path):
    path = _file(tmp_path, "u8_extra_keywords", writer)
    r = aa.aa_py_sigproc_input(path)
    r.read_metadata()
    h = r.header()
    assert h["nifs"] == 1 and h["nbits"] == 8 and h["nchans"] == 64 and h["data_type"] == 1
    assert h["data_bytes"] == 64 * 100


def _raw_header(items):
    out = b""
    for k, fmt, v in items:
        out += struct.pack("<i", len(k)) + k.encode()
        if fmt:
            out += struct.pack("<" + fmt, v)
    return out


@pytest.mark.parametrize("items,why", [
    ([("HEADER_START", None, 0), ("nbits", "i", 8), ("nchans", "i", 16), ("nifs", "i", 2), ("HEADER_END", None, 0)],
     "IF"),
    ([("HEADER_START", None, 0), ("nbits", "i", 4), ("nchans", "i", 7), ("nifs", "i", 1), ("HEADER_END", None, 0)],
     "multiple of 8"),
    ([("HEADER_START", None, 0), ("nbits", "i", 3), ("nchans", "i", 16), ("nifs", "i", 1), ("HEADER_END", None, 0)],
     "bit"),
    ([("HEADER_START", None, 0), ("nbits", "i", 8), ("nchans", "i", 16)], "HEADER_END"),
])
def test_refused_files(aa, tmp_path, items, why):
    path = str(tmp_path / "bad.fil")
    with open(path, "wb") as f:
        f.write(_raw_header(items) + bytes(64))
    r = aa.aa_py_sigproc_input(path)
    m = r.read_metadata()
    assert m.m_nbits == 0
    assert why in r.last_error()
    assert not r.read_signal()
    assert O.read(path) is None


def test_missing_file(aa, tmp_path):
    r = aa.aa_py_sigproc_input(str(tmp_path / "none.fil"))
    assert r.read_metadata().m_nbits == 0
    assert "cannot open" in r.last_error()


def test_pack_roundtrip(aa):
    from aa_b200.sigproc import pack
    for name, case in S.CASES.items():
        if case["nbits"] == 32:
            continue
        x = S.make_data(case)
        p = pack(x, case["nbits"]).reshape(-1)
        assert np.array_equal(O.unpack(p, case["nbits"], case["nchans"], case["nsamp"]), x), name
