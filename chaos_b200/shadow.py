"""The two-trajectory estimator, `propagate_shadow` (src/Lyapunov/two_trajectory.jl:181-259), on the B200.

Per orbit a shadow starts at `displaced(x0, d0 u0)` and both orbits are advanced by the map; every tau steps the
separation d is measured, log(d / d_prev) is added to a Neumaier sum and the shadow is put back at distance d0 along
the separation. X2 = (sum + comp) / N estimates the largest exponent. The device work is `cl_b200_shadow` /
`cl_b200_shadow_device` (chaos_b200/csrc/cl_shadow.cu); this module is the host side: the argument checks, the
directions (`U0` normalised by `safe_norm`, else the seeded frame's first column), the start check of Algorithm 1,
launch windows, the finals and the errors of the lowest failing orbit.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi
from ._lib import last_error, lib
from .foundation import DeviceError, DimensionMismatch, NumericalHealthError
from .propagate import FrameSpec, PropagationResult, build_run
from .systems import WrappedStandardMap, _reduce

_PI = 3.141592653589793 + 1.2246467991473532e-16   # `_pi(Float64)` of src/Systems/standard_map.jl:46


def end_dtype(s: int) -> np.dtype:
    """ShadowEnd{s, Float64} (two_trajectory.jl:12-20) as a numpy structured type (isbits layout)."""
    return np.dtype([("x", "<f8", (s,)), ("y", "<f8", (s,)), ("sum_s", "<f8"), ("sum_c", "<f8"), ("dprev", "<f8"),
                     ("code", "i1"), ("_p0", "V7"), ("step", "<i8"), ("value", "<f8")])


def _safe_norm(v) -> float:
    """safe_norm (src/Foundation/norm.jl:8-12): m = maximum(abs, v); m sqrt(sum((v / m)^2)), left folds."""
    v = [float(a) for a in v]
    m = abs(v[0])
    for a in v[1:]:
        b = abs(a)
        m = b if (b > m or math.isnan(b)) and not math.isnan(m) else m
    if m == 0.0 or not math.isfinite(m):
        return m
    q = v[0] / m
    s = q * q
    for a in v[1:]:
        q = a / m
        s = s + q * q
    return m * math.sqrt(s)


def _separation(sys, x, y):
    if isinstance(sys, WrappedStandardMap):
        tp = 2 * _PI
        h = tp / 2
        out = []
        for i in range(2):
            u = float(y[i]) - float(x[i])
            out.append(u - tp if u > h else (u + tp if u <= -h else u))
        return out
    return [float(b) - float(a) for a, b in zip(x[: sys.d], y[: sys.d])]


def _displaced(sys, x, delta):
    if isinstance(sys, WrappedStandardMap):
        tp = 2 * _PI
        xr, a = _reduce(float(x[0]) + delta[0], tp)
        pr, b = _reduce(float(x[1]) + delta[1], tp)
        return [xr, pr, float(x[2]) + a, float(x[3]) + b]
    return [float(a) + b for a, b in zip(x, delta)]


def _error(code: int, value: float, step: int, d0: float, orbit: int, backend: str) -> NumericalHealthError:
    """_shadow_error (two_trajectory.jl:84-89)."""
    if code == 1:
        return NumericalHealthError("state", value, math.inf, step, orbit, backend)
    thr = d0 if code == 3 else (0.0 if math.isfinite(value) else math.inf)
    return NumericalHealthError("separation", value, thr, step, orbit, backend)


def propagate_shadow(sys, x0, N: int, *, d0: float, tau: int = 1, seed: int = 0, U0=None, chunk: int | None = None,
                     launch_steps: int | None = None) -> PropagationResult:
    """Two-trajectory estimates for every orbit of `x0` (n x s). Returns a PropagationResult with `x` the final
    reference states, `W` the final shadow states, `finals[i] = ({n, sum, comp, X2, d_prev},)` and the raw end
    records in `states`. Raises NumericalHealthError ("state" or "separation") for the lowest failing orbit, and
    the reference's ArgumentErrors (ValueError here) for bad arguments."""
    x0 = np.ascontiguousarray(np.asarray(x0, dtype=np.float64))
    if x0.ndim != 2:
        raise ValueError("x0 must be an (orbits x state) array")
    n, s = x0.shape
    d = sys.d
    N, tau = int(N), int(tau)
    if not (tau >= 1 and N >= 1 and N % tau == 0):
        raise ValueError(f"N must be a positive multiple of tau, got N = {N}, tau = {tau}")
    if s < d:
        raise ValueError(f"state length {s} is below the system dimension {d}")
    if chunk is not None and chunk < 1:
        raise ValueError(f"chunk must be positive, got {chunk}")
    d0 = float(d0)
    if not (math.isfinite(d0) and d0 > 0):
        raise ValueError(f"d0 must be finite and positive, got {d0}")
    if s != d and not isinstance(sys, WrappedStandardMap) and n:
        # Algorithm 1's start check runs on the host for every orbit before any launch (_check_starts,
        # two_trajectory.jl:158-162, called at :190): `displaced(sys, x, d0 u0)` falls back to `x + d0 u0`
        # (separation.jl:17) for every system but WrappedStandardMap, an SVector{s} plus an SVector{d}, which
        # StaticArrays rejects when s != d (the wrapped Froeschle map, s = 8, and the wrapped chain, s = 4N).
        raise DimensionMismatch(f"Sizes ({s},) and ({d},) of input arrays do not match")
    u = None
    if U0 is not None:
        U0 = np.asarray(U0, dtype=np.float64)
        if len(U0) != n:
            raise ValueError("U0 needs one vector per orbit")
        u = np.empty((n, d))
        for j in range(n):
            nrm = _safe_norm(U0[j])
            u[j] = [float(v) / nrm for v in U0[j]]
        # Algorithm 1 on the host, before any launch: every realised d_0^+ must lie in [d0/2, 2 d0]
        for j in range(n):
            y = _displaced(sys, x0[j], [d0 * float(v) for v in u[j]])
            dp = _safe_norm(_separation(sys, x0[j], y))
            code = 2 if not (math.isfinite(dp) and dp > 0) else (3 if (dp < d0 / 2 or dp > 2 * d0) else 0)
            if code:
                raise _error(code, dp, 0, d0, j + 1, "cpu")
    L = int(launch_steps) if launch_steps else N
    if L % tau:
        raise ValueError("launch_steps must be a multiple of tau")
    size = n if chunk is None else int(chunk)
    ends = np.zeros(n, dtype=end_dtype(s))
    prov_gpu_ms, launches = 0.0, 0
    for lo in range(0, n, size):
        hi = min(n, lo + size)
        run = build_run(sys, N, tau, [FrameSpec(1, ())], "fp64", seed, orbit_base=lo, steps=L)
        xs = np.ascontiguousarray(x0[lo:hi])
        us = None if u is None else np.ascontiguousarray(u[lo:hi])
        e = np.zeros(hi - lo, dtype=end_dtype(s))
        prov = _abi.cl_prov()
        rc = lib().cl_b200_shadow(C.byref(run), hi - lo, xs.ctypes.data_as(C.POINTER(C.c_double)),
                                  None if us is None else us.ctypes.data_as(C.POINTER(C.c_double)),
                                  e.ctypes.data, d0, C.byref(prov))
        if rc != 0:
            msg = last_error()
            if rc == _abi.EINVAL:
                raise ValueError(msg)
            raise DeviceError(rc, msg)
        bad = np.flatnonzero(e["code"] != 0)
        if len(bad):
            j = int(bad[0])
            raise _error(int(e["code"][j]), float(e["value"][j]), int(e["step"][j]), d0, lo + j + 1, "gpu")
        ends[lo:hi] = e
        prov_gpu_ms += prov.gpu_ms
        launches += prov.launches
    finals = [({"n": N, "sum": float(r["sum_s"]), "comp": float(r["sum_c"]), "X2": (float(r["sum_s"]) + float(r["sum_c"])) / N,
                "d_prev": float(r["dprev"])},) for r in ends]
    provenance = {"backend": "gpu", "estimator": "two-trajectory", "d0": d0, "tau": tau, "seed": seed, "k": 0,
                  "chunk_size": size, "launch_steps": L, "launches": launches, "gpu_ms": prov_gpu_ms,
                  "state_mode": "wrapped" if isinstance(sys, WrappedStandardMap) else "lifted"}
    return PropagationResult(x=np.array([r["x"] for r in ends]), W=np.array([r["y"] for r in ends]), finals=finals,
                             provenance=provenance, states=ends, code=ends["code"].copy(), hstep=ends["step"].copy())
