"""Order-independent digests of row sets (test helper).

A set of int64 rows is summarised by (count, sum of a 64-bit mix of each row
mod 2^64, xor of the same); equal multisets give equal digests whatever the
row order, so full-size outputs can be compared without sorting.
"""
import numpy as np

from oracle.ref import canon_ee

_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix(x):
    x = x ^ (x >> np.uint64(30))
    x = x * _M1
    x = x ^ (x >> np.uint64(27))
    x = x * _M2
    return x ^ (x >> np.uint64(31))


def row_hash(rows):
    r = np.ascontiguousarray(rows, dtype=np.int64)
    if r.ndim == 1:
        r = r[:, None]
    h = np.zeros(len(r), np.uint64)
    with np.errstate(over="ignore"):
        for c in range(r.shape[1]):
            h = _mix(h ^ (r[:, c].astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15) * np.uint64(c + 1)))
    return h


def set_digest(rows):
    h = row_hash(rows)
    with np.errstate(over="ignore"):
        s = int(np.sum(h, dtype=np.uint64))
    x = int(np.bitwise_xor.reduce(h)) if len(h) else 0
    return [int(len(h)), s, x]


def set_rows(sten, is_vf):
    """(is_vf, s0..s3) int64 rows of a stencil set, EE stencils in
    lexicographic orientation ([a,b,c,d] vs [c,d,a,b]: the smaller)."""
    s = np.asarray(sten, np.int64).reshape(-1, 4).copy()
    v = np.asarray(is_vf).astype(np.int64).reshape(-1)
    ee = v == 0
    if ee.any():
        s[ee] = canon_ee(s[ee])
    return np.concatenate([v[:, None], s], axis=1)


def hit_rows(sten, is_vf, toi):
    """(is_vf, s0..s3, toi bits) rows: a hit and its exact toi, in the
    orientation given (lower primitive index first for EE stencils, as the
    device emits them and the oracle restatement enumerates them)."""
    s = np.asarray(sten, np.int64).reshape(-1, 4)
    v = np.asarray(is_vf).astype(np.int64).reshape(-1, 1)
    t = np.ascontiguousarray(toi, np.float64).view(np.int64).reshape(-1, 1)
    return np.concatenate([v, s, t], axis=1)
