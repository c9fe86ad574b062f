"""The linear symplectic maps built from blocks (src/Systems/linear_symplectic.jl:39-91: rotation_block,
hyperbolic_block, block_diagonal, conjugated) and the exact exponent test that uses them, test/lyap-householder-qr/
hh_exact.jl:74-126 (AC6, Y5 in higher dimension): A = block_diagonal of hyperbolic blocks, normal or conjugated
into a non-normal A_S; k = d, tau = 1, n = 500, start 0, QRSpectrum(HouseholderQR). With the Gram determinants of
Y = A^n Q0 in 4096-bit arithmetic, the cumulative exponent sums C_i satisfy (a) |C_i - ln vol_i| <= i n theta,
(b) for normal A |C_i / n - Lambda_i - B_i / n| <= i theta, (c) |sum lambda| <= theta, with the reference's
theta = 16 eps (G_max / tau + M_max) (hh_helpers.jl:124). Run on the oracle (the GPU parity of LinearSymplecticMap
d = 4, 6 is in test_gpu_parity.py)."""
from __future__ import annotations

import math

import mpmath
import numpy as np
import pytest

from chaos_b200 import (HouseholderQR, LinearSymplecticMap, QRSpectrum, block_diagonal, conjugated, hyperbolic_block,
                        rotation_block)
from chaos_b200.propagate import FrameSpec
from helpers import haar_frames

EPS = 2.0 ** -52


def test_blocks():
    R = rotation_block(0.3)
    assert R[0, 0] == math.cos(0.3) and R[0, 1] == math.sin(0.3) and R[1, 0] == -math.sin(0.3)
    H = hyperbolic_block(0.5)
    assert H[0, 0] == math.cosh(0.5) and H[0, 1] == H[1, 0] == math.sinh(0.5)
    A = block_diagonal(R, H)
    # (q1, q2, p1, p2): block j acts on (q_j, p_j)
    assert A[0, 0] == R[0, 0] and A[0, 2] == R[0, 1] and A[2, 0] == R[1, 0] and A[1, 3] == H[0, 1]
    assert A[0, 1] == 0 and A[0, 3] == 0
    J = np.block([[np.zeros((2, 2)), np.eye(2)], [-np.eye(2), np.zeros((2, 2))]])
    for M in (A, conjugated(A, np.array([[1.0, 2.0], [2.0, 1.0]]))):
        assert np.max(np.abs(M.T @ J @ M - J)) <= 64 * EPS      # symplectic
    with pytest.raises(ValueError):
        conjugated(A, np.array([[1.0, 2.0], [3.0, 1.0]]))


def _logvol(A, Q0, n, i):
    with mpmath.workprec(4096):
        Am = mpmath.matrix([[mpmath.mpf(float(v)) for v in row] for row in A])
        Y = (Am ** n) * mpmath.matrix([[mpmath.mpf(float(v)) for v in row] for row in Q0])
        Yi = Y[:, :i]
        return mpmath.log(mpmath.det(Yi.T * Yi)) / 2


@pytest.mark.parametrize("mus", [(0.45, 0.2), (0.45, 0.3, 0.1)])
@pytest.mark.parametrize("nonnormal", [False, True])
def test_exact_exponents_of_hyperbolic_blocks(oracle, mus, nonnormal):
    N = len(mus)
    d = 2 * N
    A0 = block_diagonal(*[hyperbolic_block(m) for m in mus])
    B = np.array([[1.0, 2.0], [2.0, 1.0]]) if N == 2 else np.array([[1.0, 2.0, 0.0], [2.0, 1.0, 1.0], [0.0, 1.0, 1.0]])
    A = conjugated(A0, B) if nonnormal else A0
    n = 500
    Q0 = haar_frames(1, d, d, 60 + d + nonnormal)
    r = oracle.oracle_frames(LinearSymplecticMap(A), np.zeros((1, d)), n, [FrameSpec(d, (QRSpectrum(HouseholderQR()),), Q0)],
                             tau=1, math="portable")[0]
    assert r["code"][0] == 0
    sums = r["states"]["r0"]["sums"][0]
    C = np.cumsum(sums[:, 0] + sums[:, 1])
    sv = np.linalg.svd(A, compute_uv=False)
    theta = 16 * EPS * (sv[0] / sv[-1] + np.max(np.abs(A)))
    lam = sorted([m for m in mus] + [-m for m in mus], reverse=True)
    Lam = np.cumsum(lam)
    # eigenvectors (e_q_j +- e_p_j) / sqrt 2 in the order of the exponents, for the B_i term of the normal case
    V = np.zeros((d, d))
    order = sorted([(m, j, 1) for j, m in enumerate(mus)] + [(-m, j, -1) for j, m in enumerate(mus)], key=lambda t: -t[0])
    for c, (_, j, sg) in enumerate(order):
        V[j, c] = 1 / math.sqrt(2)
        V[N + j, c] = sg / math.sqrt(2)
    for i in range(1, d + 1):
        lv = _logvol(A, Q0[0], n, i)
        assert abs(float(mpmath.mpf(C[i - 1]) - lv)) <= i * n * theta                                 # (a)
        if not nonnormal:
            Bi = math.log(abs(np.linalg.det(V[:, :i].T @ Q0[0][:, :i])))
            # (b); B_i is evaluated in binary64 here (the reference: 2048 bits), whence the 1e-14 on top
            assert abs(C[i - 1] / n - Lam[i - 1] - Bi / n) <= i * theta + 1e-14
    lam_final = (sums[:, 0] + sums[:, 1]) / n
    assert abs(np.sum(lam_final)) <= theta                                                          # (c)
