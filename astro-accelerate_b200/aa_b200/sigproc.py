"""SIGPROC filterbank files: packing of samples in the order the reference's
reader unpacks them (src/aa_sigproc_input.cpp:441-521) and a writer, for
producing test and survey files; reading goes through the library
(aa_b200.aa_py_sigproc_input).

Channel order inside a byte: 4-bit high nibble first, 2-bit most significant
pair first, 1-bit least significant bit first.
"""
from __future__ import annotations

import struct

import numpy as np

__all__ = ["pack", "write_filterbank", "record_bytes"]


def record_bytes(nbits: int, nchans: int) -> int:
    """Bytes of one stored time sample (all channels)."""
    if nbits not in (1, 2, 4, 8, 16, 32):
        raise ValueError("nbits must be 1, 2, 4, 8, 16 or 32")
    if (nchans * nbits) % 8:
        raise ValueError("nchans * nbits must be a multiple of 8")
    return nchans * nbits // 8


def pack(data_tc: np.ndarray, nbits: int) -> np.ndarray:
    """[nsamples][nchans] samples -> the stored records, [nsamples][record
    bytes] uint8 (float32 values for nbits 32, little-endian uint16 for 16)."""
    data_tc = np.asarray(data_tc)
    nsamp, nchans = data_tc.shape
    record_bytes(nbits, nchans)
    if nbits == 32:
        return np.ascontiguousarray(data_tc, dtype="<f4").view(np.uint8).reshape(nsamp, nchans * 4)
    if nbits == 16:
        return np.ascontiguousarray(data_tc, dtype="<u2").view(np.uint8).reshape(nsamp, nchans * 2)
    x = data_tc.astype(np.uint8)
    if x.max(initial=0) >= (1 << nbits):
        raise ValueError(f"sample above the {nbits}-bit range")
    per = 8 // nbits
    g = x.reshape(nsamp, nchans // per, per).astype(np.uint32)
    if nbits == 1:
        shifts = np.arange(per, dtype=np.uint32)               # channel 8b+i -> bit i
    else:
        shifts = (8 - nbits * (np.arange(per, dtype=np.uint32) + 1))  # first channel in the top bits
    return (g << shifts).sum(axis=2).astype(np.uint8)


def _string(s: str) -> bytes:
    b = s.encode()
    return struct.pack("<i", len(b)) + b


def write_filterbank(path: str, data_tc: np.ndarray, nbits: int, tsamp: float, fch1: float, foff: float,
                     tstart: float = 60000.0, telescope_id: int = 0, machine_id: int = 0, data_type: int = 1,
                     source_name: str | None = None, src_raj: float = 0.0, src_dej: float = 0.0,
                     extra_ints: dict | None = None) -> int:
    """Writes a single-IF SIGPROC filterbank; returns the header length in bytes.
    extra_ints adds integer keywords (e.g. ibeam) after the standard ones."""
    data_tc = np.asarray(data_tc)
    nchans = data_tc.shape[1]
    h = _string("HEADER_START")
    h += _string("telescope_id") + struct.pack("<i", telescope_id)
    h += _string("machine_id") + struct.pack("<i", machine_id)
    h += _string("data_type") + struct.pack("<i", data_type)
    if source_name is not None:
        h += _string("source_name") + _string(source_name)
    h += _string("src_raj") + struct.pack("<d", src_raj)
    h += _string("src_dej") + struct.pack("<d", src_dej)
    h += _string("tstart") + struct.pack("<d", tstart)
    h += _string("tsamp") + struct.pack("<d", tsamp)
    h += _string("nbits") + struct.pack("<i", nbits)
    h += _string("fch1") + struct.pack("<d", fch1)
    h += _string("foff") + struct.pack("<d", foff)
    h += _string("nchans") + struct.pack("<i", nchans)
    h += _string("nifs") + struct.pack("<i", 1)
    for k, v in (extra_ints or {}).items():
        h += _string(k) + struct.pack("<i", v)
    h += _string("HEADER_END")
    with open(path, "wb") as f:
        f.write(h)
        f.write(pack(data_tc, nbits).tobytes())
    return len(h)
