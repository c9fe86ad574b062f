"""Systems of the fixed menu the B200 kernels cover (src/Systems), as host-side parameter records.

Each system fills a `cl_system` and knows its tangent dimension `d` and state length `s`. The arithmetic of
`forward` / `tangent` runs only on the device; the host-side helpers here are the start-point constructions of the
reference (`torus_state`, `lift`, the Henon-Heiles energy-shell starts), which the reference also runs on the host.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi

_PI = 3.141592653589793 + 1.2246467991473532e-16  # `_pi` in Float64, src/Systems/standard_map.jl:46


class System:
    d: int
    s: int
    name: str

    def to_cl(self) -> _abi.cl_system:
        raise NotImplementedError

    def dimension(self) -> int:
        return self.d


@dataclass(frozen=True)
class StandardMap(System):
    """StandardMap(K), src/Systems/standard_map.jl:8-44: p' = p + K sin x, x' = x + p' (lifted)."""
    K: float
    d: int = field(default=2, init=False)
    s: int = field(default=2, init=False)
    name: str = field(default="StandardMap", init=False)

    def to_cl(self):
        c = _abi.cl_system(kind=_abi.SYS_STANDARD, K=float(self.K))
        return c


@dataclass(frozen=True)
class WrappedStandardMap(System):
    """WrappedStandardMap(K), src/Systems/wrapped_standard_map.jl:12-57: the torus map with exact winding counts,
    state (x, p, m, n)."""
    K: float
    d: int = field(default=2, init=False)
    s: int = field(default=4, init=False)
    name: str = field(default="WrappedStandardMap", init=False)

    def to_cl(self):
        return _abi.cl_system(kind=_abi.SYS_WRAPPED_STANDARD, K=float(self.K))


@dataclass(frozen=True)
class FroeschleMap(System):
    """FroeschleMap(nu, kappa, mu), src/Systems/froeschle_map.jl:9-58, state (x1, x2, p1, p2)."""
    nu: float
    kappa: float
    mu: float
    d: int = field(default=4, init=False)
    s: int = field(default=4, init=False)
    name: str = field(default="FroeschleMap", init=False)

    def to_cl(self):
        return _abi.cl_system(kind=_abi.SYS_FROESCHLE, nu=float(self.nu), kappa=float(self.kappa), mu=float(self.mu))


class StandardMapChain(System):
    """StandardMapChain(N, K, eps; boundary=:open), src/Systems/standard_map_chain.jl:11-31, state
    (q_1..q_N, p_1..p_N), banded tangent (chain_tangent.jl). The compiled menu covers N in 2..8."""

    def __init__(self, N: int, K: float, eps: float, boundary: str = "open"):
        if not 2 <= N <= 100:
            raise ValueError(f"number of sites N must be in 2:100, got {N}")
        if boundary not in ("open", "ring"):
            raise ValueError(f"boundary must be :open or :ring, got :{boundary}")
        if boundary == "ring" and N < 3:
            raise ValueError(f"a ring needs N >= 3, got {N}")
        self.N, self.K, self.eps, self.ring = int(N), float(K), float(eps), boundary == "ring"
        self.d = self.s = 2 * self.N
        self.name = "StandardMapChain"

    def to_cl(self):
        return _abi.cl_system(kind=_abi.SYS_CHAIN, n_sites=self.N, ring=int(self.ring), K=self.K, eps=self.eps)

    def __repr__(self):
        return f"StandardMapChain({self.N}, {self.K}, {self.eps}, boundary={'ring' if self.ring else 'open'})"


class LinearSymplecticMap(System):
    """LinearSymplecticMap(A), src/Systems/linear_symplectic.jl: z' = A z, tangent A (d even, d <= 16)."""

    def __init__(self, A):
        A = np.asarray(A, dtype=np.float64)
        if A.ndim != 2 or A.shape[0] != A.shape[1] or A.shape[0] % 2:
            raise ValueError("symplectic map needs an even square matrix")
        if A.shape[0] > _abi.MAX_DIM:
            raise ValueError(f"dimension above {_abi.MAX_DIM} is not in the compiled menu")
        self.A = A
        self.d = self.s = A.shape[0]
        self.name = "LinearSymplecticMap"

    def to_cl(self):
        c = _abi.cl_system(kind=_abi.SYS_LINEAR)
        flat = np.zeros(_abi.MAX_DIM * _abi.MAX_DIM)
        flat[: self.d * self.d] = self.A.ravel(order="F")
        c.A[:] = flat.tolist()
        return c


@dataclass(frozen=True)
class HenonHeilesFlow:
    """HenonHeilesFlow(), src/Systems/flow_models.jl:30,101-103: H = |p|^2/2 + |q|^2/2 + q1^2 q2 - q2^3/3."""
    name: str = "HenonHeilesFlow"

    @staticmethod
    def hamiltonian(z) -> float:
        q1, q2, p1, p2 = (float(v) for v in z)
        return (p1 * p1 + p2 * p2) / 2 + (q1 * q1 + q2 * q2) / 2 + q1 * q1 * q2 - q2 ** 3 / 3


@dataclass(frozen=True)
class Gauss:
    """Gauss(Float64, s; maxiter, tol), src/Integrators/gauss.jl:49-69; the compiled menu has s = 3 (order 6).
    `tol=None` is the reference's relative acceptance bound 8 eps max(1, |Y|)."""
    stages: int = 3
    tol: float | None = None
    maxiter: int = 50

    def __post_init__(self):
        if self.stages != 3:
            raise ValueError("the compiled menu covers the 3-stage Gauss method only")
        if self.maxiter < 2:
            raise ValueError("maxiter must be at least 2")


class SplittingMethod:
    """A table method (src/Integrators/splitting.jl:16-36): drift weights c, kick weights d, k stages, one step =
    drift(c_1 tau), kick(d_1 tau), ..., first stage first. Construction checks the reference's conditions: k >= 1,
    as many kick as drift weights, finite weights, |sum c - 1| and |sum d - 1| at most 4 k max(eps, 10^-digits),
    and for a palindromic table c_i = c_(k+1-i), d_i = d_(k-i), d_k = 0."""

    def __init__(self, c, d, *, order: int, palindromic: bool, name: str, digits: float = math.inf):
        c = [float(v) for v in c]
        d = [float(v) for v in d]
        k = len(c)
        if not (k >= 1 and len(d) == k):
            raise ValueError(f"a splitting table needs k >= 1 stages and as many kick as drift weights, got {k} and {len(d)}")
        if not all(math.isfinite(v) for v in c + d):
            raise ValueError(f"table {name} has a non-finite weight")
        tol = 4 * k * max(2.0 ** -52, 10.0 ** (-digits))
        if not (abs(_jl_sum(c) - 1.0) <= tol and abs(_jl_sum(d) - 1.0) <= tol):
            raise ValueError(f"table {name} violates the sum conditions sum c = sum d = 1 (bound {tol})")
        if palindromic and not (all(c[i] == c[k - 1 - i] for i in range(k)) and
                                all(d[i] == d[k - 2 - i] for i in range(k - 1)) and d[k - 1] == 0.0):
            raise ValueError(f"table {name} is declared palindromic but is not (c_i = c_(k+1-i), d_i = d_(k-i), d_k = 0)")
        self.c, self.d, self.order, self.palindromic, self.name, self.digits = tuple(c), tuple(d), order, palindromic, name, digits

    @property
    def stages(self) -> int:
        return len(self.c)

    def __repr__(self):
        return f"SplittingMethod({self.name}, {self.stages} stages, order {self.order})"


def _jl_sum(v):
    """Julia's `sum` of a short Float64 vector: pairwise blocks of 1024 degenerate to a left fold below 1024."""
    s = 0.0
    for x in v:
        s = s + x
    return s


def _normalize(cs, ds, trailing: bool):
    """Merge the drifts between consecutive kicks and drop empty stages (splitting.jl:109-120)."""
    c, d, acc = [], [], 0.0
    for ci, di in zip(cs, ds):
        acc = acc + ci
        if di != 0.0:
            c.append(acc)
            d.append(di)
            acc = 0.0
    if acc != 0.0:
        c.append(acc)
        d.append(0.0)
    if trailing and d[-1] != 0.0:
        c.append(0.0)
        d.append(0.0)
    return c, d


def Leapfrog(order: str = "DKD") -> SplittingMethod:
    """Leapfrog(Float64, order), src/Integrators/tables.jl:15-20: DKD (c = (1/2, 1/2), d = (1, 0)) or KDK."""
    if order == "DKD":
        c, d = [0.5, 0.5], [1.0, 0.0]
    elif order == "KDK":
        c, d = [0.0, 1.0, 0.0], [0.5, 0.5, 0.0]
    else:
        raise ValueError(f"Leapfrog order must be :DKD or :KDK, got :{order}")
    return SplittingMethod(c, d, order=2, palindromic=True, name=f"leapfrog {order}")


# Kahan and Li (1997), Appendix A: the step fractions gamma_1.. of the palindromic compositions of leapfrogs
# (the middle one last), 20 digits as published; scheme 6 is s9odr6a, 8 is s17odr8a.
_KAHANLI_GAMMA = {
    "s7odr6": (6, ("0.78451361047755726382", "0.23557321335935813368", "-1.1776799841788710069",
                   "1.3151863206839112189")),
    "s9odr6a": (6, ("0.39216144400731413928", "0.33259913678935943860", "-0.70624617255763935981",
                    "0.082213596293550800230", "0.79854399093482996340")),
    "s17odr8a": (8, ("0.13020248308889008088", "0.56116298177510838456", "-0.38947496264484728641",
                     "0.15884190655515560090", "-0.39590389413323757734", "0.18453964097831570709",
                     "0.25837438768632204729", "0.29501172360931029887", "-0.60550853383003451170")),
}


def KahanLi(scheme=6) -> SplittingMethod:
    """KahanLi(Float64, scheme), src/Integrators/tables.jl:74-86: the leapfrog (DKD) composed with the step fractions
    gamma_1..gamma_m..gamma_1 (splitting.jl:174-177, 126-134); the decimal constants are rounded to Float64 once
    (Julia's `parse`, correctly rounded, as Python's `float`)."""
    key = scheme if isinstance(scheme, str) else {6: "s9odr6a", 8: "s17odr8a"}.get(scheme)
    if key not in _KAHANLI_GAMMA:
        raise ValueError("KahanLi: scheme 6, 8 or 's7odr6'")
    order, g = _KAHANLI_GAMMA[key]
    half = [float(v) for v in g]
    gammas = half + half[-2::-1]
    lf = Leapfrog("DKD")
    cs, ds = [], []
    for gm in gammas:
        for ci, di in zip(lf.c, lf.d):
            cs.append(gm * ci)
            ds.append(gm * di)
    c, d = _normalize(cs, ds, lf.palindromic)
    return SplittingMethod(c, d, order=order, palindromic=True, name=f"Kahan-Li {key}", digits=20)


class IntegratorMap(System):
    """IntegratorMap(method, flow, tau), src/Integrators/integrator_map.jl:12-23: one step of the flow as a map, by
    Gauss (gauss.jl:49-192) or a table method (stepper.jl:27-48); the tangent is the exact Jacobian of the step
    (gauss.jl:176-192; stepper.jl:108-118, the product of the stage Jacobians)."""

    def __init__(self, method, flow: HenonHeilesFlow, tau: float):
        if not isinstance(flow, HenonHeilesFlow):
            raise TypeError("the compiled menu integrates HenonHeilesFlow")
        if not isinstance(method, (Gauss, SplittingMethod)):
            raise TypeError("the compiled menu integrates with Gauss(3) or a SplittingMethod table")
        if isinstance(method, SplittingMethod) and method.stages > _abi.MAX_STAGES:
            raise ValueError(f"a table of {method.stages} stages is above the compiled limit ({_abi.MAX_STAGES})")
        self.method, self.flow, self.tau = method, flow, float(tau)
        self.d = self.s = 4
        kind = "Gauss3" if isinstance(method, Gauss) else "SplittingMethod"
        self.name = f"IntegratorMap{{{kind},HenonHeilesFlow}}"

    def to_cl(self):
        if isinstance(self.method, SplittingMethod):
            k = self.method.stages
            cs = _abi.cl_system(kind=_abi.SYS_HH_SPLIT, dt=self.tau, n_stages=k, gauss_tol=math.nan)
            for i in range(k):
                cs.stage_c[i] = self.method.c[i]
                cs.stage_d[i] = self.method.d[i]
            return cs
        tol = math.nan if self.method.tol is None else float(self.method.tol)
        return _abi.cl_system(kind=_abi.SYS_HH_GAUSS, gauss_maxiter=self.method.maxiter, gauss_tol=tol, dt=self.tau)


# ---- host-side start-point helpers ------------------------------------------------------------------------------------
def _reduce(u: float, tp: float):
    """_reduce, src/Systems/wrapped_standard_map.jl:15-28."""
    a = math.floor(u / tp)
    r = u - tp * a
    if r < 0:
        r += tp
        a -= 1
    if r >= tp:
        r -= tp
        a += 1
    return float(r), float(a)


def torus_state(z) -> np.ndarray:
    """torus_state((X, P)) -> (x, p, m, n), src/Systems/wrapped_standard_map.jl:63-69."""
    tp = 2 * _PI
    x, m = _reduce(float(z[0]), tp)
    p, n = _reduce(float(z[1]), tp)
    return np.array([x, p, m, n])


def lift(s) -> np.ndarray:
    """lift((x, p, m, n)) -> (x + 2 pi m, p + 2 pi n), src/Systems/wrapped_standard_map.jl:77-80."""
    tp = 2 * _PI
    return np.array([s[0] + tp * s[2], s[1] + tp * s[3]])


def _hh_u(q2: float) -> float:  # Equation 7: V(0, q2), src/Systems/henon_heiles.jl:4
    return q2 ** 2 / 2 - q2 ** 3 / 3


def section_interval(E: float):
    """section_interval(HenonHeilesFlow(), E) -> (a, b), src/Systems/henon_heiles.jl:48-52 (bisection :32-40)."""
    E = float(E)
    if not (math.isfinite(E) and 0 < E <= 1 / 6):
        raise ValueError(f"section_interval needs 0 < E <= 1/6, got {E}")
    if E == 1 / 6:
        return (-0.5, 1.0)

    def bisect(lo, hi):
        sgn = _hh_u(lo) - E > 0
        for _ in range(4096):
            mid = (lo + hi) / 2
            if mid == lo or mid == hi:
                break
            if (_hh_u(mid) - E > 0) == sgn:
                lo = mid
            else:
                hi = mid
        return (lo + hi) / 2

    return (bisect(-1.0, 0.0), bisect(0.0, 1.0))


def energy_start(E: float, q2: float, p2: float):
    """energy_start(HenonHeilesFlow(), E, q2, p2) -> (z, status), src/Systems/henon_heiles.jl:62-68."""
    if not (math.isfinite(E) and math.isfinite(q2) and math.isfinite(p2)):
        return None, "nonfinite"
    r = 2 * (E - p2 ** 2 / 2 - _hh_u(q2))
    if not (r > 0 and abs(q2) <= 1):
        return None, "outside"
    return np.array([0.0, q2, math.sqrt(r), p2]), "ok"


def random_energy_starts(E: float, n: int, seed: int, maxtries: int = 10_000) -> np.ndarray:
    """n rejection draws of src/Systems/henon_heiles.jl:76-85 (`random_energy_start`) on the windows
    `section_interval(E)` x [-sqrt(2E), sqrt(2E)], from numpy's PCG64 stream (the reference draws from
    StableRNGs.jl, which is absent; the distribution is the same)."""
    a, b = section_interval(E)
    pm = math.sqrt(2 * E)
    rng = np.random.Generator(np.random.PCG64(seed))
    out = np.empty((n, 4))
    for i in range(n):
        for _ in range(maxtries):
            q2 = a + (b - a) * rng.random()
            p2 = -pm + (pm - -pm) * rng.random()
            z, st = energy_start(E, q2, p2)
            if st == "ok":
                out[i] = z
                break
        else:
            raise RuntimeError("no admissible point")
    return out
