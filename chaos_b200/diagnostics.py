"""Residual records of a Lyapunov spectrum (src/Diagnostics/residuals.jl), evaluated on the host from the QRSpectrum
finals a propagation returns.

* `eps_sum(lambda)` (residuals.jl:13): |sum_i lambda_i| (spec D5);
* `eps_pair(lambda)` (residuals.jl:16-18): max_i |lambda_i + lambda_{M+1-i}| over i = 1..M/2, estimator order, no
  sorting (spec D1);
* `sum_threshold(tol, T, G_max, tau, M_max)` (residuals.jl:32): tol eps(T) (G_max / tau + M_max), the bound of both
  residuals that `monitor_exponents` (src/Diagnostics/monitor.jl:79-88) and the study recorder's thresholds
  (src/Experiments/run_record.jl:189-197) apply, with the default multiplier `pairing_residual_tol = 16`
  (_config/numerics-defaults.toml:10).

`spectrum_residuals(result, tau=...)` gives the three per orbit for a QRSpectrum result (k = d: the whole spectrum),
with G_max from the QR state itself and M_max, the largest entry of a one-step tangent, from the system's bound
`tangent_bound()` unless the caller passes the observed maximum (the reference's caller passes its monitor's
running maximum, which the bound dominates).
"""
from __future__ import annotations

import numpy as np

from .foundation import EPS

PAIRING_RESIDUAL_TOL = 16.0
EPS32 = float(np.finfo(np.float32).eps)


def effective_eps(T: str = "Float64") -> float:
    """effective_eps(T) (src/Foundation/Foundation.jl:44): eps of the element type."""
    if T in ("Float64", np.float64, "f64"):
        return EPS
    if T in ("Float32", np.float32, "f32"):
        return EPS32
    raise ValueError(f"unknown element type {T!r}")


def eps_sum(lam) -> float:
    """|sum_i lambda_i| (spec D5); the sum is the left fold of StaticArrays' `sum`."""
    lam = np.asarray(lam, dtype=np.float64).ravel()
    s = lam[0]
    for v in lam[1:]:
        s = s + v
    return float(abs(s))


def eps_pair(lam) -> float:
    """max_i |lambda_i + lambda_{M+1-i}| over i = 1..M/2, estimator order, no sorting (spec D1)."""
    lam = np.asarray(lam, dtype=np.float64).ravel()
    M = lam.size
    if M < 2:
        raise ValueError("pairing needs at least two exponents")
    return float(max(abs(lam[i] + lam[M - 1 - i]) for i in range(M // 2)))


def sum_threshold(tol: float, T, G_max, tau, M_max):
    """T(tol) effective_eps(T) (T(G_max) / tau + T(M_max)), independent of the run length (residuals.jl:32).
    Arrays of G_max broadcast."""
    return np.float64(tol) * effective_eps(T) * (np.asarray(G_max, dtype=np.float64) / tau + np.float64(M_max))


def _lambdas(states) -> np.ndarray:
    """lambda_i = (s_i + c_i) / n per orbit from QRState records (qr_spectrum.jl:85-91); 0 before any handoff."""
    sums = states["sums"]
    n = states["n"].astype(np.float64)
    tot = sums[..., 0] + sums[..., 1]
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(n[:, None] > 0, tot / n[:, None], 0.0)


def spectrum_residuals(result, *, tau: int, tol: float = PAIRING_RESIDUAL_TOL, M_max=None, T="Float64",
                       system=None) -> dict:
    """Per-orbit residual records of a QRSpectrum result with k = d: `eps_sum`, `eps_pair`, their common
    `threshold` = sum_threshold(tol, T, G_max, tau, M_max) and `sum_ok` = eps_sum <= threshold (the check
    `monitor_exponents` raises on). `result` is a PropagationResult whose chain's first reducer is QRSpectrum;
    `T` is the element type of the frame ("Float32" for the mixed kernels' frames). M_max defaults to
    `system.tangent_bound()`."""
    from .reducers import QRSpectrum

    if not result.reducers or not isinstance(result.reducers[0], QRSpectrum):
        raise ValueError("the residual records need a QRSpectrum frame")
    st = result.states["r0"]
    lam = _lambdas(st)
    n, k = lam.shape
    if M_max is None:
        if system is None or getattr(system, "tangent_bound", lambda: None)() is None:
            raise ValueError("M_max is needed (no tangent bound for this system)")
        M_max = system.tangent_bound()
    # eps_sum as the left fold (cumsum adds left to right)
    es = np.abs(np.cumsum(lam, axis=1)[:, -1]) if k else np.zeros(n)
    ep = np.max(np.abs(lam[:, : k // 2] + lam[:, ::-1][:, : k // 2]), axis=1) if k >= 2 else np.zeros(n)
    thr = sum_threshold(tol, T, st["G_max"], tau, M_max)
    return dict(lam=lam, eps_sum=es, eps_pair=ep, threshold=thr, sum_ok=es <= thr)


def orth_loss(Q) -> float:
    """eps_orth: max |Q'Q - I| (spec D4, residuals.jl:10)."""
    Q = np.asarray(Q, dtype=np.float64)
    return float(np.max(np.abs(Q.T @ Q - np.eye(Q.shape[1]))))


# The bounds below which SALI and GALI_k sit in their rounding noise at 1e5 steps of the coupled maps (two Float64
# frames with different roundings agree within 0.02 decades above them and scatter below; measured on 65536 orbits):
# SALI and GALI_2 1e-8, GALI_3 1e-14, GALI_4 and higher 1e-16.
SALI_BOUND = 1e-8
GALI_BOUNDS = {2: 1e-8, 3: 1e-14}
GALI_BOUND_HIGH = 1e-16


def precision_errors(ref, got, N: int) -> list[dict]:
    """Per frame, how a run in reduced precision (`got`) differs from the Float64 run (`ref`) on the same orbits and
    frames: the status agreement and completed fractions, then per reducer -- QRSpectrum: max and 99th percentile
    |d lambda_i| over the orbits both completed, and G_max's ratio on the windows the Float64 run finds well
    conditioned (G_max < 1e6) with the fraction beyond 1e7 (where a Float32 frame cannot resolve the window:
    G eps(Float32) > 1); SALI and GALI_k: agreement of the class at the noise bounds above (SALI_BOUND, GALI_BOUNDS)
    and the largest |d log10| above them. `ref` and `got` are lists of PropagationResult (or records with .states,
    .code, .hstep, .reducers)."""
    from .reducers import GALI, QRSpectrum, SALI

    out = []
    for a, b in zip(ref, got):
        ok = (a.code == 0) & (b.code == 0)
        rec = dict(code_agree=float(np.mean(a.code == b.code)), hstep_agree=float(np.mean(a.hstep == b.hstep)),
                   completed_ref=float(np.mean((a.code == 0) & (a.hstep == N))),
                   completed_got=float(np.mean((b.code == 0) & (b.hstep == N))),
                   code_disagreements=[int(i) for i in np.flatnonzero(a.code != b.code)[:20]])
        for i, r in enumerate(a.reducers):
            sa, sb = a.states[f"r{i}"], b.states[f"r{i}"]
            if isinstance(r, QRSpectrum):
                d = np.abs(_lambdas(sa) - _lambdas(sb))[ok]
                rec["dlambda_max"] = [float(v) for v in (d.max(axis=0) if len(d) else np.zeros(d.shape[1]))]
                rec["dlambda_p99"] = [float(v) for v in (np.percentile(d, 99, axis=0) if len(d) else np.zeros(d.shape[1]))]
                ga, gb = sa["G_max"][ok], sb["G_max"][ok]
                well = ga < 1e6
                ratio = gb[well] / ga[well] if well.any() else np.ones(1)
                rec["G_max"] = dict(ratio_well_conditioned=[float(ratio.min()), float(ratio.max())],
                                    well_conditioned=float(np.mean(well)) if len(ga) else 0.0,
                                    beyond_1e7=float(np.mean(ga >= 1e7)) if len(ga) else 0.0)
            elif isinstance(r, SALI):
                va, vb = sa["sali"][ok], sb["sali"][ok]
                ca, cb = va < SALI_BOUND, vb < SALI_BOUND
                big = ~ca & ~cb
                rec["sali"] = dict(class_agree=float(np.mean(ca == cb)) if len(va) else 1.0, aligned_ref=float(np.mean(ca)) if len(va) else 0.0,
                                   dlog10_max=float(np.max(np.abs(np.log10(va[big]) - np.log10(vb[big])), initial=0.0)))
            elif isinstance(r, GALI):
                g = []
                for k in range(sa["gali"].shape[1]):
                    va, vb = sa["gali"][ok, k], sb["gali"][ok, k]
                    fl = GALI_BOUNDS.get(k + 2, GALI_BOUND_HIGH)
                    ca, cb = va < fl, vb < fl
                    big = ~ca & ~cb
                    g.append(dict(k=k + 2, class_agree=float(np.mean(ca == cb)) if len(va) else 1.0,
                                  dlog10_max=float(np.max(np.abs(np.log10(va[big]) - np.log10(vb[big])), initial=0.0))))
                rec["gali"] = g
        out.append(rec)
    return out
