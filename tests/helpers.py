"""Shared helpers of the test suite: seeded inputs and bitwise comparisons of device and oracle records."""
from __future__ import annotations

import numpy as np

TWO_PI = 2 * np.pi


def uniform_starts(n, s, seed, lo=0.0, hi=TWO_PI):
    return np.random.default_rng(seed).uniform(lo, hi, size=(n, s))


def identity_frames(n, d, k):
    return np.broadcast_to(np.eye(d)[:, :k], (n, d, k)).copy()


def haar_frames(n, d, k, seed):
    rng = np.random.default_rng(seed)
    out = np.empty((n, d, k))
    for i in range(n):
        q, r = np.linalg.qr(rng.standard_normal((d, d)))
        out[i] = (q * np.sign(np.diag(r)))[:, :k]
    return out


def same_bits(a, b):
    """Bitwise equality of float arrays, with every NaN equal to every NaN."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "f":
        na, nb = np.isnan(a), np.isnan(b)
        return bool(np.array_equal(na, nb) and np.array_equal(a.view(np.uint64 if a.itemsize == 8 else np.uint32)[~na],
                                                              b.view(np.uint64 if b.itemsize == 8 else np.uint32)[~nb]))
    return bool(np.array_equal(a, b))


def states_equal(sa, sb):
    """Bitwise equality of two structured state arrays, field by field (padding ignored, NaNs equal)."""
    if sa is None or sb is None:
        return sa is None and sb is None
    for name in sa.dtype.names:
        fa, fb = sa[name], sb[name]
        if fa.dtype.names:
            if not states_equal(fa, fb):
                return False
            continue
        if name.startswith("_p"):
            continue
        if not same_bits(fa, fb):
            return False
    return True
