"""CPU restatement of the reference's SIGPROC filterbank reader
(AstroAccelerate v1.3.1, src/aa_sigproc_input.cpp:85-543), in numpy.

TEST INFRASTRUCTURE ONLY: used by tests/ to check the library's reader and
its packed-input path; nothing in the product imports it.  Pinned against the
reference's own reader (oracle/ref_harness.cu aaref_sigproc_read) through
tests/golden/sigproc_golden.json.
"""
from __future__ import annotations

import struct

import numpy as np

# src/aa_sigproc_input.cpp:127-263: keyword -> struct format of its value
KEYWORDS = {
    "telescope_id": "i", "machine_id": "i", "data_type": "i", "barycentric": "i", "pulsarcentric": "i",
    "az_start": "d", "za_start": "d", "src_raj": "d", "src_dej": "d", "tstart": "d", "tsamp": "d",
    "nbits": "i", "nsamples": "i", "fch1": "d", "foff": "d", "fchannel": "d", "nchans": "i", "nifs": "i",
    "refdm": "d", "period": "d",
}


def parse_header(blob: bytes):
    """(values, data_start) following the keyword loop of :110-269: a
    length-prefixed string; lengths <= 1 or >= 80 are passed over; a known
    keyword is followed by its binary value, an unknown one consumes nothing
    more; HEADER_END ends the header.  None when the header is cut short."""
    vals = {k: 0 for k in KEYWORDS}
    pos = 0
    while True:
        if pos + 4 > len(blob):
            return None
        (nchar,) = struct.unpack_from("<i", blob, pos)
        pos += 4
        if not 1 < nchar < 80:
            continue
        if pos + nchar > len(blob):
            return None
        s = blob[pos:pos + nchar].decode("latin-1")
        pos += nchar
        if s == "HEADER_END":
            return vals, pos
        fmt = KEYWORDS.get(s)
        if fmt is not None:
            n = struct.calcsize("<" + fmt)
            if pos + n > len(blob):
                return None
            (vals[s],) = struct.unpack_from("<" + fmt, blob, pos)
            pos += n


def nsamples_of(data_bytes: int, nbits: int, nchans: int) -> int:
    """:296-319, integer division as there."""
    return {32: data_bytes // (nchans * 4), 16: data_bytes // (nchans * 2), 8: data_bytes // nchans,
            4: 2 * data_bytes // nchans, 2: 4 * data_bytes // nchans, 1: 8 * data_bytes // nchans}[nbits]


def unpack(raw: np.ndarray, nbits: int, nchans: int, nsamp: int) -> np.ndarray:
    """:389-521 -> [nsamp][nchans] uint16."""
    if nbits == 16:
        return raw[:nsamp * nchans * 2].view("<u2").reshape(nsamp, nchans).astype(np.uint16)
    if nbits == 8:
        return raw[:nsamp * nchans].reshape(nsamp, nchans).astype(np.uint16)
    per = 8 // nbits
    b = raw[:nsamp * nchans // per].reshape(nsamp, nchans // per, 1).astype(np.uint16)
    if nbits == 1:
        shifts = np.arange(per, dtype=np.uint16)                       # :505-510, bit i -> channel 8c+i
    else:
        shifts = (8 - nbits * (np.arange(per, dtype=np.uint16) + 1))   # :441-495, high bits first
    return ((b >> shifts) & ((1 << nbits) - 1)).reshape(nsamp, nchans).astype(np.uint16)


def rescale32(x: np.ndarray) -> np.ndarray:
    """:332-386: min/max over the file (initial +-1e10, NaN never compares),
    bin = (max - min) / 65535, (unsigned short)((x - min) / bin) in float32,
    the float -> unsigned short conversion as x86-64 performs it (truncation
    to int32, INT_MIN for NaN or out of range, then the low 16 bits)."""
    x = x.astype(np.float32, copy=False)
    fin = x[~np.isnan(x)]
    mx = np.float32(max(np.float32(-1e10), fin.max())) if fin.size else np.float32(-1e10)
    mn = np.float32(min(np.float32(1e10), fin.min())) if fin.size else np.float32(1e10)
    with np.errstate(invalid="ignore", divide="ignore"):
        bin_ = np.float32(np.float32(mx - mn) / np.float32(65535.0))
        q = (x - mn) / bin_
    ok = ~np.isnan(q) & (q < np.float32(2147483648.0)) & (q >= np.float32(-2147483648.0))
    v = np.full(x.shape, -(2**31), dtype=np.int64)
    v[ok] = np.trunc(q[ok]).astype(np.int64)
    return (v & 0xFFFF).astype(np.uint16)


def read(path: str):
    """(metadata dict, [nsamp][nchans] uint16) as aa_sigproc_input's
    read_metadata + read_signal produce them; None for files the library
    refuses (no HEADER_END, nifs != 1, unsupported nbits, channels not filling
    whole bytes)."""
    blob = open(path, "rb").read()
    h = parse_header(blob)
    if h is None:
        return None
    vals, start = h
    nbits, nchans = vals["nbits"], vals["nchans"]
    if vals["nifs"] != 1 or nchans <= 0 or nbits not in (1, 2, 4, 8, 16, 32) or (nchans * nbits) % 8:
        return None
    data = np.frombuffer(blob, dtype=np.uint8, offset=start)
    nsamp = nsamples_of(len(data), nbits, nchans)
    meta = dict(tstart=vals["tstart"], tsamp=vals["tsamp"], fch1=vals["fch1"], foff=vals["foff"], nbits=nbits,
                nsamples=nsamp, nchans=nchans)
    if nbits == 32:
        buf = rescale32(data[:nsamp * nchans * 4].view("<f4").reshape(nsamp, nchans))
    else:
        buf = unpack(data, nbits, nchans, nsamp)
    return meta, buf
