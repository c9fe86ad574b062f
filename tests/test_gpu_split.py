"""The split-precision kernel of the coupled-maps ensemble (precision "mixed-ind64": Float64 orbit and GALI/SALI frame,
Float32 QRSpectrum(Householder) frame) against the plain Float64 kernel, which is bit for bit the oracle: every output
of the benched configuration -- the orbit, the four exponents, the QR records and status, GALI_2..4, SALI and the
indicator frame's log sums -- with the tolerance written in each assertion; relaunch carry and failure records."""
import numpy as np
import pytest

from chaos_b200 import GALI, SALI, FroeschleMap, HouseholderQR, QRSpectrum
from chaos_b200.propagate import FrameSpec, propagate_frames
from helpers import identity_frames, same_bits, uniform_starts

pytestmark = pytest.mark.gpu

SYS = FroeschleMap(1.5, 1.5, 0.05)


def _frames(n):
    W0 = identity_frames(n, 4, 4)
    return [FrameSpec(4, (QRSpectrum(HouseholderQR()),), W0), FrameSpec(4, (GALI(), SALI()), W0)]


def _run(x0, N, precision, **kw):
    return propagate_frames(SYS, x0, N, _frames(len(x0)), tau=10, precision=precision, finals=False, throw=False, **kw)


def _lam(r):
    q = r[0].states["r0"]
    return (q["sums"][:, :, 0] + q["sums"][:, :, 1]) / np.maximum(q["n"][:, None], 1)


def test_froeschle_fused_mixed():
    """8192 orbits uniform in [0, 2 pi)^4, N = 1e5, tau = 10, W0 = I (the benched workload's map, frames and
    horizon): the orbit bit for bit; |d lambda_i| <= 1e-3 for i = 1..4; the QR frame's status and step equal on
    every orbit and its orthogonality loss within the Float32 threshold; G_max within 1e-3 relative where the Float64
    window is well conditioned (G_max < 1e6); the indicator frame (Float64) gives the same class at the rounding-noise
    bounds (SALI and GALI_2 1e-8, GALI_3 1e-14, GALI_4 1e-16) on every orbit and, above them, the same values within
    |d log10| <= 0.05; its log sums within 1e-8 relative; every orbit completes N steps in both."""
    n, N = 8192, 100_000
    x0 = uniform_starts(n, 4, seed=1)
    a = _run(x0, N, "fp64")
    b = _run(x0, N, "mixed-ind64")
    assert same_bits(a[0].x, b[0].x)
    for f in range(2):
        assert np.array_equal(a[f].code, b[f].code), np.flatnonzero(a[f].code != b[f].code)[:20]
        assert np.array_equal(a[f].hstep, b[f].hstep)
    ok = (a[0].code == 0) & (b[0].code == 0)
    assert ok.all() and np.all(a[0].hstep == N)
    dl = np.abs(_lam(a) - _lam(b))
    assert np.max(dl) <= 1e-3, np.max(dl, axis=0)
    qa, qb = a[0].states["r0"], b[0].states["r0"]
    assert np.array_equal(qa["n"], qb["n"]) and np.array_equal(qa["count_max"], qb["count_max"])
    assert np.all(qb["orth_max"] <= 8 * 2.0 ** -23 * 4)
    well = qa["G_max"] < 1e6
    assert np.max(np.abs(qb["G_max"][well] / qa["G_max"][well] - 1.0), initial=0.0) <= 1e-3
    ga, gb = a[1].states, b[1].states
    sa, sb = ga["r1"]["sali"], gb["r1"]["sali"]
    assert np.array_equal(sa < 1e-8, sb < 1e-8)
    big = sa >= 1e-8
    assert np.max(np.abs(np.log10(sa[big]) - np.log10(sb[big])), initial=0.0) <= 0.05
    for k, bound in enumerate((1e-8, 1e-14, 1e-16)):
        va, vb = ga["r0"]["gali"][:, k], gb["r0"]["gali"][:, k]
        assert np.array_equal(va < bound, vb < bound), k
        big = va >= bound
        assert np.max(np.abs(np.log10(va[big]) - np.log10(vb[big])), initial=0.0) <= 0.05, k
    ta = ga["r0"]["s"] + ga["r0"]["c"]
    tb = gb["r0"]["s"] + gb["r0"]["c"]
    assert np.max(np.abs(ta - tb) / np.maximum(np.abs(ta), 1.0)) <= 1e-8
    assert np.array_equal(ga["r1"]["n"], gb["r1"]["n"]) and np.array_equal(ga["r0"]["n"], gb["r0"]["n"])


def test_split_relaunch_and_layouts():
    """A run split into launches of 700 steps carries the state: the orbit, both frames, GALI and SALI bit for bit
    the one-launch run, the exponent sums (flushed at every launch end) within 1e-13 relative."""
    n, N = 3000, 7000
    x0 = uniform_starts(n, 4, seed=5)
    one = _run(x0, N, "mixed-ind64")
    many = _run(x0, N, "mixed-ind64", launch_steps=700)
    assert same_bits(one[0].x, many[0].x)
    for f in range(2):
        assert same_bits(one[f].W, many[f].W)
        assert np.array_equal(one[f].code, many[f].code)
    assert same_bits(one[1].states["r0"]["gali"], many[1].states["r0"]["gali"])
    assert same_bits(one[1].states["r1"]["sali"], many[1].states["r1"]["sali"])
    la, lb = _lam(one), _lam(many)
    assert np.max(np.abs(la - lb)) <= 1e-13


def test_split_failures():
    """Failure records equal the plain kernel's: a non-finite start stops both frames at the first handoff with the
    state status; a zero column stops the QR frame (pivot) and the GALI frame (column norm) with the reducer status
    at that handoff, the SALI record naming column 1."""
    n, N = 256, 2000
    x0 = uniform_starts(n, 4, seed=7)
    x0[3, 2] = np.nan
    W0 = identity_frames(n, 4, 4)
    W0[10, :, 0] = 0.0
    fr = [FrameSpec(4, (QRSpectrum(HouseholderQR()),), W0), FrameSpec(4, (GALI(), SALI()), W0)]
    a = propagate_frames(SYS, x0, N, fr, tau=10, finals=False, throw=False)
    b = propagate_frames(SYS, x0, N, fr, tau=10, precision="mixed-ind64", finals=False, throw=False)
    for f in range(2):
        assert np.array_equal(a[f].code, b[f].code) and np.array_equal(a[f].hstep, b[f].hstep)
    assert a[0].code[3] == 1 and a[0].hstep[3] == 10
    assert b[0].code[10] == 3 and b[1].code[10] == 3
    qa, qb = a[0].states["r0"], b[0].states["r0"]
    assert int(qb["code"][10]) == int(qa["code"][10]) == 1 and int(qb["column"][10]) == 1
    sa, sb = a[1].states["r1"], b[1].states["r1"]
    assert int(sb["code"][10]) == int(sa["code"][10]) and int(sb["column"][10]) == int(sa["column"][10])
    assert same_bits(a[0].x, b[0].x)
    # a failing handoff leaves the frame as it was (the factorisation runs in the frame's registers)
    assert np.allclose(b[0].W[10], a[0].W[10], rtol=1e-4, atol=1e-6) and np.all(b[0].W[10][:, 0] == 0)


def test_split_values_of_last_successful_handoff():
    """GALI's and SALI's values are formed once, from the unit columns of a launch's last successful handoff. Orbits
    whose state (p1 = 4e16, 9e15, 6e15: the trigonometry of x1 turns non-finite) or frame (p1 = 1e16) fails at a
    later handoff keep, bit for bit, the values of the same kernel run that ends at their last successful step, in
    one launch and in launches of one window each. Status and step equal the Float64 kernel's for the indicator
    frame (Float64 in both) on every orbit whose state fails or survives, and for the Float32 QR frame on the
    ordinary orbits (on the late ones the huge trigonometric values of x1 overflow it earlier than Float64)."""
    n, N = 32, 400
    x0 = uniform_starts(n, 4, seed=11)
    late = {3: (4e16, 1, 20), 5: (9e15, 1, 60), 7: (6e15, 1, 90), 9: (1e16, 2, 60)}
    for i, (p1, _, _) in late.items():
        x0[i] = [0.5, 0.2, p1, 0.1]
    a = _run(x0, N, "fp64")
    for kw in ({}, {"launch_steps": 10}):
        b = _run(x0, N, "mixed-ind64", **kw)
        plain = np.setdiff1d(np.arange(n), list(late))
        assert np.array_equal(a[0].code[plain], b[0].code[plain]) and np.array_equal(a[0].hstep[plain], b[0].hstep[plain])
        same = np.setdiff1d(np.arange(n), [9])
        assert np.array_equal(a[1].code[same], b[1].code[same]) and np.array_equal(a[1].hstep[same], b[1].hstep[same])
        g = b[1].states
        for i, (_, code, step) in late.items():
            assert int(b[1].code[i]) == code, (i, b[1].code[i])
            if i != 9:
                assert int(b[1].hstep[i]) == step, (i, b[1].hstep[i])
            last = int(g["r0"]["n"][i])
            assert last == int(b[1].hstep[i]) - 10 and last >= 10
            c = _run(x0[i:i + 1], last, "mixed-ind64")[1].states
            assert same_bits(g["r0"]["gali"][i], c["r0"]["gali"][0]), (i, g["r0"]["gali"][i], c["r0"]["gali"][0])
            assert same_bits(g["r1"]["sali"][i], c["r1"]["sali"][0]), i
