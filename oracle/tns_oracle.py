"""Test infrastructure only: a CPU restatement of the reference's .tns loader
(SymtensLoader::SymtensLoader, src/utils/loader.cpp:8-36), used as the
checker of the device parser (symprop_tensor_load_tns).

The loader reads `order dim`, then repeatedly `order` unsigned ids and one
double with an std::istream, sorts the ids and keeps the record while the
stream is good().  For well-formed tokens that means:
  * tokens are maximal runs of non-whitespace (C isspace);
  * a trailing partial record is dropped (a read fails);
  * a record whose value token ends the file is dropped too: the extraction
    of that value hits end-of-file, which clears good() (loader.cpp:28-29);
  * values convert as strtod does (correctly rounded), as Python's float().
Tokens the stream would read only in part (for instance `1.5x` or `inf`) are
rejected here with ValueError, as the device parser rejects them.
Pinned against the reference binary's own loader (oracle/_ref/ref_probe load)
by tests/test_tns.py.
"""
import re

import numpy as np

_TOKEN = re.compile(rb"[^ \t\n\v\f\r]+")
_UINT = re.compile(rb"\+?[0-9]+\Z")
_DOUBLE = re.compile(rb"[+-]?([0-9]+\.?[0-9]*|\.[0-9]+)([eE][+-]?[0-9]+)?\Z")


def load_tns(data: bytes):
    """(order, dim, inds nnz x order uint32 sorted per row, vals float64)."""
    toks = [(m.group(0), m.end()) for m in _TOKEN.finditer(data)]
    if len(toks) < 2 or not _UINT.match(toks[0][0]) or not _UINT.match(toks[1][0]):
        raise ValueError("header: expected 'order dim'")
    order, dim = int(toks[0][0]), int(toks[1][0])
    body = toks[2:]
    nrec = len(body) // (order + 1)
    if nrec and len(body) % (order + 1) == 0 and body[-1][1] == len(data):
        nrec -= 1  # the last value ends the file: end-of-file clears good()
    inds = np.zeros((nrec, order), dtype=np.uint32)
    vals = np.zeros(nrec, dtype=np.float64)
    for k in range(nrec):
        rec = body[k * (order + 1):(k + 1) * (order + 1)]
        ids = []
        for tok, _ in rec[:order]:
            if not _UINT.match(tok) or int(tok) > 0xFFFFFFFF:
                raise ValueError(f"record {k + 1}: bad id token {tok!r}")
            ids.append(int(tok))
        tok = rec[order][0]
        if not _DOUBLE.match(tok):
            raise ValueError(f"record {k + 1}: bad value token {tok!r}")
        inds[k] = sorted(ids)
        vals[k] = float(tok)
    return order, dim, inds, vals
