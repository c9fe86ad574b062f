"""Residual records of a spectrum (src/Diagnostics/residuals.jl), evaluated on the host from the reducers' finals.

`eps_sum` (:26) and `eps_pair` (:29-32) are the residual record the reference keeps with every QR spectrum;
`sum_threshold` (:55) is its bound. Float64 arithmetic in the reference's order.
"""
from __future__ import annotations

import numpy as np

from .foundation import EPS


def eps_sum(lam) -> float:
    """|sum_i lambda_i| (spec D5), the sum a left fold."""
    s = np.float64(0.0)
    for i, v in enumerate(np.asarray(lam, dtype=np.float64)):
        s = np.float64(v) if i == 0 else s + np.float64(v)
    return float(abs(s))


def eps_pair(lam) -> float:
    """max_i |lambda_i + lambda_{2N+1-i}| over i = 1..M/2, estimator order, no sorting (spec D1)."""
    lam = np.asarray(lam, dtype=np.float64)
    M = lam.size
    return float(max(abs(lam[i] + lam[M - 1 - i]) for i in range(M // 2)))


def sum_threshold(tol: float, G_max: float, tau: int, M_max: float) -> float:
    """tol eps (G_max / tau + M_max), independent of the run length (residuals.jl:55)."""
    return float(np.float64(tol) * EPS * (np.float64(G_max) / tau + np.float64(M_max)))


def orth_loss(Q) -> float:
    """eps_orth: max |Q'Q - I| (spec D4)."""
    Q = np.asarray(Q, dtype=np.float64)
    return float(np.max(np.abs(Q.T @ Q - np.eye(Q.shape[1]))))
