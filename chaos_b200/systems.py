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


class IntegratorMap(System):
    """IntegratorMap(method, flow, tau), src/Integrators/integrator_map.jl:12-23: one Gauss step of the flow as
    a map; the tangent is the exact Jacobian of the step (gauss.jl:176-192)."""

    def __init__(self, method: Gauss, flow: HenonHeilesFlow, tau: float):
        if not isinstance(flow, HenonHeilesFlow):
            raise TypeError("the compiled menu integrates HenonHeilesFlow")
        self.method, self.flow, self.tau = method, flow, float(tau)
        self.d = self.s = 4
        self.name = "IntegratorMap{Gauss3,HenonHeilesFlow}"

    def to_cl(self):
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
