"""Generates tests/golden/sigproc_golden.json: what the reference's own
SIGPROC reader (aa_sigproc_input, src/aa_sigproc_input.cpp:85-543, compiled
from its sources into oracle/_ref/libaaref.so by oracle/Makefile.ref) returns
for the seeded files of sigproc_cases.py (written by aa_b200.sigproc).
Host only, no GPU.

    python tests/golden/make_sigproc_golden.py
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "astro-accelerate_b200"))
import refharness as R  # noqa: E402
import sigproc_cases as S  # noqa: E402
from aa_b200.sigproc import write_filterbank  # noqa: E402


def reference_read(L, path, cap=1 << 26):
    meta = (ctypes.c_double * 4)()
    imeta = (ctypes.c_int * 4)()
    buf = np.zeros(cap, np.uint16)
    n = L.aaref_sigproc_read(os.fsencode(path), meta, imeta, buf.ctypes.data, cap)
    m = dict(tstart=meta[0], tsamp=meta[1], fch1=meta[2], foff=meta[3], nbits=imeta[0], nsamples=imeta[1],
             nchans=imeta[2], nifs=imeta[3])
    return m, (buf[:n].copy() if n >= 0 else None)


def load():
    L = R.load()
    L.aaref_sigproc_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                                     ctypes.c_void_p, ctypes.c_longlong]
    L.aaref_sigproc_read.restype = ctypes.c_longlong
    return L


def main():
    L = load()
    out = {}
    with tempfile.TemporaryDirectory() as td:
        for name, case in S.CASES.items():
            path = os.path.join(td, name + ".fil")
            S.write_case(case, path, write_filterbank)
            m, buf = reference_read(L, path)
            out[name] = dict(meta=m, elements=int(buf.size), sha256=hashlib.sha256(buf.tobytes()).hexdigest(),
                             first=[int(v) for v in buf[:16]])
    with open(os.path.join(HERE, "sigproc_golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(f"{len(out)} cases")


if __name__ == "__main__":
    main()
