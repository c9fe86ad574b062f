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

    def tangent_bound(self) -> float:
        """Largest |entry| a one-step tangent [[1 + c, 1], [c, 1]], c = K cos x, can have: 1 + |K|."""
        return 1.0 + abs(self.K)


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

    def tangent_bound(self) -> float:
        """Largest |entry| of a one-step tangent (the standard map's): 1 + |K|."""
        return 1.0 + abs(self.K)

    def torus_state(self, z) -> np.ndarray:
        """torus_state((X, P)) (wrapped_standard_map.jl:63-69) of the lifted point z = (X, P)."""
        return _torus(z, 2)


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

    def tangent_bound(self) -> float:
        """Largest |entry| a tangent [[I, I], [A, I + A]] can have (|a| <= |nu| + |mu|, |c| <= |kappa| + |mu|)."""
        return 1.0 + max(abs(self.nu), abs(self.kappa)) + abs(self.mu)


@dataclass(frozen=True)
class WrappedFroeschleMap(System):
    """WrappedFroeschleMap(nu, kappa, mu), src/Systems/froeschle_map.jl:60-126: the Froeschle map on the torus with
    winding counts, state (x1, x2, p1, p2, c1, c2, c3, c4), coordinates in [0, 2 pi) and exact integer counts; the
    tangent is evaluated at the unreduced sums x + p."""
    nu: float
    kappa: float
    mu: float
    d: int = field(default=4, init=False)
    s: int = field(default=8, init=False)
    name: str = field(default="WrappedFroeschleMap", init=False)

    def to_cl(self):
        return _abi.cl_system(kind=_abi.SYS_WRAPPED_FROESCHLE, nu=float(self.nu), kappa=float(self.kappa),
                              mu=float(self.mu))

    def tangent_bound(self) -> float:
        """Largest |entry| of a one-step tangent (the lifted map's bound)."""
        return 1.0 + max(abs(self.nu), abs(self.kappa)) + abs(self.mu)

    def torus_state(self, z) -> np.ndarray:
        """torus_state(sys, z) (:110-114): each coordinate of the lifted z reduced into [0, 2 pi) with its count."""
        return _torus(z, 4)

    def lift(self, s) -> np.ndarray:
        """lift(sys, s) (:121-124): z_j + 2 pi c_j."""
        return _lift(s, 4)


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

    def tangent_bound(self) -> float:
        """Largest |entry| of a one-step tangent: the band's diagonal 1 + K cos q_j + eps (two neighbours' cos)."""
        return 1.0 + abs(self.K) + 2.0 * abs(self.eps)

    def __repr__(self):
        return f"StandardMapChain({self.N}, {self.K}, {self.eps}, boundary={'ring' if self.ring else 'open'})"


class WrappedStandardMapChain(StandardMapChain):
    """WrappedStandardMapChain(N, K, eps; boundary=:open), src/Systems/wrapped_standard_map_chain.jl: the chain on
    the torus with winding counts, state (q_1..q_N, p_1..p_N, counts of q, counts of p), d = 2N, s = 4N."""

    def __init__(self, N: int, K: float, eps: float, boundary: str = "open"):
        super().__init__(N, K, eps, boundary)
        self.s = 4 * self.N
        self.name = "WrappedStandardMapChain"

    def to_cl(self):
        return _abi.cl_system(kind=_abi.SYS_WRAPPED_CHAIN, n_sites=self.N, ring=int(self.ring), K=self.K,
                              eps=self.eps)

    def torus_state(self, z) -> np.ndarray:
        """torus_state(sys, z) (:75-83): (reduced coordinates, counts)."""
        if len(z) != self.d:
            raise ValueError("lifted state length is not 2N for this chain")
        return _torus(z, self.d)

    def lift(self, s) -> np.ndarray:
        """lift(sys, s) (:90-94)."""
        if len(s) != self.s:
            raise ValueError("wrapped state length is not 4N for this chain")
        return _lift(s, self.d)

    def __repr__(self):
        return f"WrappedStandardMapChain({self.N}, {self.K}, {self.eps}, boundary={'ring' if self.ring else 'open'})"


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

    def tangent_bound(self) -> float:
        """The tangent is A: max |A_ij|."""
        return float(np.max(np.abs(self.A)))

    def to_cl(self):
        c = _abi.cl_system(kind=_abi.SYS_LINEAR)
        flat = np.zeros(_abi.MAX_DIM * _abi.MAX_DIM)
        flat[: self.d * self.d] = self.A.ravel(order="F")
        c.A[:] = flat.tolist()
        return c


def _fma(a: float, b: float, c: float) -> float:
    """fma(a, b, c) rounded once (the exact value of a b + c in rational arithmetic, correctly rounded), with the
    IEEE sign of a zero result; finite arguments."""
    from fractions import Fraction
    p = Fraction(a) * Fraction(b)
    t = p + Fraction(c)
    if t != 0:
        return float(t)
    if p == 0 and c == 0:
        neg_p = (math.copysign(1.0, a) * math.copysign(1.0, b)) < 0
        return -0.0 if (neg_p and math.copysign(1.0, c) < 0) else 0.0
    return 0.0


def _smatmul(A, B):
    """StaticArrays' unrolled SMatrix product: C[i, j] = A[i, 1] B[1, j], then muladd(A[i, q], B[q, j], C[i, j]) for
    q = 2..n, the muladd fused (the chain `fused_product` restates, src/Foundation/product.jl:9-20)."""
    A, B = np.asarray(A, dtype=np.float64), np.asarray(B, dtype=np.float64)
    n, m, p = A.shape[0], A.shape[1], B.shape[1]
    C = np.empty((n, p))
    for i in range(n):
        for j in range(p):
            acc = float(A[i, 0]) * float(B[0, j])
            for q in range(1, m):
                acc = _fma(float(A[i, q]), float(B[q, j]), acc)
            C[i, j] = acc
    return C


def rotation_block(theta: float) -> np.ndarray:
    """rotation_block(Float64, theta), src/Systems/linear_symplectic.jl:43-46: [[cos, sin], [-sin, cos]]; the
    sine and cosine are the host libm's (Julia's own libm may differ in the last bit)."""
    s, c = math.sin(float(theta)), math.cos(float(theta))
    return np.array([[c, s], [-s, c]])


def hyperbolic_block(mu: float) -> np.ndarray:
    """hyperbolic_block(Float64, mu), linear_symplectic.jl:53-56: [[cosh, sinh], [sinh, cosh]], eigenvalues
    exp(+-mu)."""
    m = float(mu)
    ch, sh = math.cosh(m), math.sinh(m)
    return np.array([[ch, sh], [sh, ch]])


def block_diagonal(*blocks) -> np.ndarray:
    """block_diagonal(blocks...), linear_symplectic.jl:58-77: the direct sum of 2 x 2 blocks on the pairs
    (q_j, p_j), reordered to (q_1..q_N, p_1..p_N)."""
    N = len(blocks)
    D = 2 * N
    A = np.zeros((D, D))
    for j, b in enumerate(blocks):
        b = np.asarray(b, dtype=np.float64)
        for r in range(2):
            for c in range(2):
                A[j + r * N, j + c * N] = b[r, c]
    return A


def conjugated(A, B) -> np.ndarray:
    """conjugated(A, B), linear_symplectic.jl:79-91: the non-normal S^-1 A S with S = [I B; 0 I], B symmetric
    N x N, evaluated as (S(-1) A) S(1) with the SMatrix product."""
    A, B = np.asarray(A, dtype=np.float64), np.asarray(B, dtype=np.float64)
    D, N = A.shape[0], B.shape[0]
    if D != 2 * N:
        raise ValueError(f"A is {D} x {D} but B is {N} x {N}")
    if not np.array_equal(B, B.T):
        raise ValueError("B must be symmetric")

    def S(sgn):
        M = np.eye(D)
        M[:N, N:] = sgn * B
        return M
    return _smatmul(_smatmul(S(-1.0), A), S(1.0))


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

    def __init__(self, c, d, *, order: int, palindromic: bool, name: str, digits: float = math.inf, source: str = ""):
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
        self.source = source

    @property
    def stages(self) -> int:
        return len(self.c)

    def isolated_force_evaluations(self) -> int:
        """Force evaluations of one step alone: kicks of consecutive stages with no drift between them share one
        (splitting.jl:86-97)."""
        n, open_ = 0, False
        for ci, di in zip(self.c, self.d):
            if ci != 0.0:
                open_ = False
            if di != 0.0:
                if not open_:
                    n += 1
                open_ = True
        return n

    def force_evaluations(self) -> int:
        """Force evaluations per step of a long run: the last kick of a step merges with the first kick of the next
        when the table starts and ends with a kick and drifts somewhere (splitting.jl:62-83)."""
        iso = self.isolated_force_evaluations()
        any_drift = any(ci != 0.0 for ci in self.c)
        first_kick = self.c[0] == 0.0 and self.d[0] != 0.0
        last_kick = False
        for ci, di in zip(reversed(self.c), reversed(self.d)):
            if di != 0.0 or ci != 0.0:
                last_kick = di != 0.0
                break
        return iso - 1 if (first_kick and last_kick and any_drift) else iso

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


def SymplecticEuler(order: str = "DK") -> SplittingMethod:
    """SymplecticEuler(Float64, order), src/Integrators/tables.jl:8-12: one stage, drift then kick (DK) or the adjoint
    kick then drift (KD); first order."""
    if order == "DK":
        c, d = [1.0], [1.0]
    elif order == "KD":
        c, d = [0.0, 1.0], [1.0, 0.0]
    else:
        raise ValueError(f"SymplecticEuler order must be :DK or :KD, got :{order}")
    return SplittingMethod(c, d, order=1, palindromic=False, name=f"symplectic Euler {order}",
                           source="Yoshida1990,Ruth1983")


def Leapfrog(order: str = "DKD") -> SplittingMethod:
    """Leapfrog(Float64, order), src/Integrators/tables.jl:15-20: DKD (c = (1/2, 1/2), d = (1, 0)) or KDK."""
    if order == "DKD":
        c, d = [0.5, 0.5], [1.0, 0.0]
    elif order == "KDK":
        c, d = [0.0, 1.0, 0.0], [0.5, 0.5, 0.0]
    else:
        raise ValueError(f"Leapfrog order must be :DKD or :KDK, got :{order}")
    return SplittingMethod(c, d, order=2, palindromic=True, name=f"leapfrog {order}",
                           source="Yoshida1990,Ruth1983,ForestRuth1990")


def _compose(m: SplittingMethod, gammas, order: int, name: str, *, source=None, digits=None) -> SplittingMethod:
    """The pieces m(gamma_1 tau) m(gamma_2 tau) ... (the first applied first), neighbouring drifts merged and the
    stage (0, 0) appended after a final kick of a symmetric table (splitting.jl:137-145)."""
    cs, ds = [], []
    for g in gammas:
        for ci, di in zip(m.c, m.d):
            cs.append(g * ci)
            ds.append(g * di)
    c, d = _normalize(cs, ds, m.palindromic)
    return SplittingMethod(c, d, order=order, palindromic=m.palindromic, name=name,
                           source=m.source if source is None else source,
                           digits=m.digits if digits is None else digits)


def _check_raise(m: SplittingMethod, order: int):
    if not m.palindromic:
        raise ValueError("composition raises the order of a symmetric table only")
    if not (order > m.order and (order - m.order) % 2 == 0):
        raise ValueError(f"target order {order} must exceed {m.order} by an even number")


def _pow(x: float, y: float) -> float:
    """x^y of two binary64 numbers, x > 0, rounded once from a 200-bit evaluation (the value a correctly rounded
    pow returns; Julia's Float64 `^` evaluates in double-double and agrees except within ~2^-16 ulp of a tie)."""
    import mpmath as mpm
    with mpm.workprec(200):
        return float(mpm.power(mpm.mpf(x), mpm.mpf(y)))


def triple_jump(m: SplittingMethod, order: int) -> SplittingMethod:
    """Raise the symmetric table m to `order`, 2 per level, with S(z1 tau) S(z0 tau) S(z1 tau),
    z1 = 1 / (2 - 2^(1/(p+1))), z0 = 1 - 2 z1 (Yoshida 1990 Eqs. (4.12)-(4.14); splitting.jl:153-161)."""
    _check_raise(m, order)
    name = f"triple jump {order} of {m.name}"
    while m.order < order:
        z1 = 1.0 / (2.0 - _pow(2.0, 1.0 / float(m.order + 1)))
        z0 = 1.0 - 2.0 * z1
        m = _compose(m, (z1, z0, z1), m.order + 2, name)
    return m


def suzuki_jump(m: SplittingMethod, order: int) -> SplittingMethod:
    """Raise the symmetric table m to `order` with Suzuki's five pieces S(s)^2 S(1 - 4 s) S(s)^2,
    s = 1 / (4 - 4^(1/(p+1))) (Kahan and Li 1997 Sect. 3; splitting.jl:169-177)."""
    _check_raise(m, order)
    name = f"Suzuki {order} of {m.name}"
    while m.order < order:
        s = 1.0 / (4.0 - _pow(4.0, 1.0 / float(m.order + 1)))
        m = _compose(m, (s, s, 1.0 - 4.0 * s, s, s), m.order + 2, name)
    return m


def adjoint_method(m):
    """The adjoint table, the stages in reverse order, so that inverse(S(tau)) = S*(-tau); a symmetric (or
    corrected) method is its own adjoint (splitting.jl:125-133)."""
    if isinstance(m, CorrectedMethod) or m.palindromic:
        return m
    k = m.stages
    cs = [0.0] + [m.c[k + 1 - i] for i in range(2, k + 1)] + [m.c[0]]
    ds = [m.d[k - 1]] + [m.d[k - i] for i in range(2, k + 1)] + [0.0]
    c, d = _normalize(cs, ds, False)
    return SplittingMethod(c, d, order=m.order, palindromic=False, name=f"{m.name} (adjoint)", source=m.source,
                           digits=m.digits)


def _palindromic_leapfrog(half, order, name, source, digits) -> SplittingMethod:
    """The leapfrog (DKD) composed with the step fractions half + reversed(half[:-1]) (splitting.jl:176-178)."""
    half = list(half)
    return _compose(Leapfrog("DKD"), half + half[-2::-1], order, name, source=source, digits=digits)


def McLachlan2() -> SplittingMethod:
    """McLachlan's optimized second-order method, tables.jl:24-28 (McLachlan 1995 Eq. (4.2)): drifts z, 1 - 2 z, z
    with z = (y^2 + 6 y - 2) / (12 y), y = (2 sqrt(326) - 36)^(1/3), in binary64 in the reference's order."""
    y = _pow(2.0 * math.sqrt(326.0) - 36.0, 1.0 / 3.0)
    z = ((y * y + 6.0 * y) - 2.0) / (12.0 * y)
    return SplittingMethod([z, 1.0 - 2.0 * z, z], [0.5, 0.5, 0.0], order=2, palindromic=True,
                           name="McLachlan optimized second order", source="McLachlan1995")


def Ruth3() -> SplittingMethod:
    """Ruth's third-order method, tables.jl:32-35 (Ruth 1983 Eq. (31)), stored kick first."""
    return SplittingMethod([0.0, 2.0 / 3.0, -2.0 / 3.0, 1.0], [7.0 / 24.0, 3.0 / 4.0, -1.0 / 24.0, 0.0], order=3,
                           palindromic=False, name="Ruth third order", source="Ruth1983,ForestRuth1990")


def ForestRuth() -> SplittingMethod:
    """Forest-Ruth, the triple jump of the DKD leapfrog to order 4 (tables.jl:39-42)."""
    m = triple_jump(Leapfrog("DKD"), 4)
    return SplittingMethod(m.c, m.d, order=4, palindromic=True, name="Forest-Ruth",
                           source="ForestRuth1990,Omelyan2002,Yoshida1990")


def PEFRL() -> SplittingMethod:
    """PEFRL, the position-extended Forest-Ruth-like method of Omelyan et al. 2002 Eqs. (20), (22), 16 digits
    (tables.jl:45-50)."""
    xi, lam, chi = float("0.1786178958448091"), float("-0.2123418310626054"), float("-0.06626458266981849")
    kd = (1.0 - 2.0 * lam) / 2.0
    return SplittingMethod([xi, chi, 1.0 - 2.0 * (chi + xi), chi, xi], [kd, lam, lam, kd, 0.0], order=4,
                           palindromic=True, name="PEFRL", source="Omelyan2002", digits=16)


# Calvo and Sanz-Serna (1993) Eq. (2.8): the nodes gamma_i and weights b_i of the five-stage fourth-order FSAL RKN
# method, 18 digits as published.
_CSS4_GAMMA = ("0", "0.205177661542286386", "0.608198943146500973", "0.487278066807586965", "1")
_CSS4_B = ("0.061758858135626325", "0.338978026553643355", "0.614791307175577566", "-0.140548014659373380",
           "0.125019822794526133")


def CalvoSanzSerna4() -> SplittingMethod:
    """The Calvo-Sanz-Serna fourth-order RKN method as a splitting (tables.jl:54-60): kick b_i, then drift to the next
    node; stored drift first, c_1 = gamma_1 = 0, c_i = gamma_i - gamma_(i-1)."""
    g = [float(v) for v in _CSS4_GAMMA]
    b = [float(v) for v in _CSS4_B]
    c = [g[0]] + [g[i] - g[i - 1] for i in range(1, 5)]
    return SplittingMethod(c, b, order=4, palindromic=False, name="Calvo-Sanz-Serna fourth order",
                           source="CalvoSanzSerna1993a", digits=18)


# Yoshida (1990) Tables 1 and 2: w_1..w_m of the symmetric composition of leapfrogs, 15 digits as printed.
_YOSHIDA_W = {
    (6, "A"): ("-0.117767998417887E1", "0.235573213359357E0", "0.784513610477560E0"),
    (8, "A"): ("-0.161582374150097E1", "-0.244699182370524E1", "-0.716989419708120E-2", "0.244002732616735E1",
               "0.157739928123617E0", "0.182020630970714E1", "0.104242620869991E1"),
    (8, "D"): ("0.102799849391985E0", "-0.196061023297549E1", "0.193813913762276E1", "-0.158240635368243E0",
               "-0.144485223686048E1", "0.253693336566229E0", "0.914844246229740E0"),
}


def Yoshida(order: int, solution: str = "A") -> SplittingMethod:
    """Yoshida(Float64, order, solution), tables.jl:68-73: the leapfrogs w_m .. w_1, w_0, w_1 .. w_m with
    w_0 = 1 - 2 sum w_i (Yoshida 1990 Eq. (5.18)); 6 :A, 8 :A, 8 :D."""
    key = (int(order), str(solution))
    if key not in _YOSHIDA_W:
        raise ValueError(f"Yoshida: no solution {solution} of order {order} (6 :A, 8 :A, 8 :D)")
    w = [float(v) for v in _YOSHIDA_W[key]]
    half = w[::-1] + [1.0 - 2.0 * _jl_sum(w)]
    return _palindromic_leapfrog(half, key[0], f"Yoshida {key[0]}{key[1]}", "Yoshida1990", 15)


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
    return _palindromic_leapfrog([float(v) for v in g], order, f"Kahan-Li {key}", "KahanLi1997", 20)


# Sofroniou and Spaletta (2005) Eq. (17): gamma_1..gamma_18 of the 35-stage tenth-order composition
# (gamma_i = gamma_(36-i)), 32 digits as printed.
_SOFSPA_GAMMA = (
    "0.078795722521686419263907679337684", "0.31309610341510852776481247192647", "0.027918383235078066109520273275299",
    "-0.22959284159390709415121339679655", "0.13096206107716486317465685927961", "-0.26973340565451071434460973222411",
    "0.074973343155891435666137105641410", "0.11199342399981020488957508073640", "0.36613344954622675119314812353150",
    "-0.39910563013603589787862981058340", "0.10308739852747107731580277001372", "0.41143087395589023782070411897608",
    "-0.0048663605831352617621956593099771", "-0.39203335370863990644808193642610",
    "0.051942502962449647037182904015976", "0.050665090759924496335874344156866", "0.049674370639729879054568800279461",
    "0.049317735759594537917680008339338")


def SofroniouSpaletta10() -> SplittingMethod:
    """The Sofroniou-Spaletta tenth-order composition of 35 leapfrogs (tables.jl:89-95): 36 stages."""
    return _palindromic_leapfrog([float(v) for v in _SOFSPA_GAMMA], 10, "Sofroniou-Spaletta 10",
                                 "SofroniouSpaletta2005", 32)


def _legendre_rule(n: int, lobatto: bool, bits: int = 330):
    """Nodes and weights on [-1, 1] of the n-point Gauss-Legendre rule (nodes the roots of P_n), or of the
    (n + 1)-point Gauss-Lobatto rule (the ends and the roots of P_n'), by Newton's method on the Legendre recurrence
    in `bits`-bit arithmetic (src/Integrators/tables_near.jl:8-44 restated with mpmath)."""
    import mpmath as mpm
    with mpm.workprec(bits):
        def pp(x):   # (P_n(x), P_n'(x)); the derivative formula is not used at the ends x = -1, 1
            a, b = mpm.mpf(1), x
            for k in range(2, n + 1):
                a, b = b, ((2 * k - 1) * x * b - (k - 1) * a) / k
            return b, (n * (a - x * b) / (1 - x * x) if x * x != 1 else mpm.inf)
        tiny = mpm.ldexp(1, -(bits - 30))
        if lobatto:
            xs = [mpm.mpf(-1)]
            for i in range(n - 1, 0, -1):
                x = mpm.cospi(mpm.mpf(i) / n)
                for _ in range(80):
                    p, dp = pp(x)
                    ddp = (2 * x * dp - n * (n + 1) * p) / (1 - x * x)
                    dx = dp / ddp
                    x -= dx
                    if abs(dx) < tiny:
                        break
                xs.append(x)
            xs.append(mpm.mpf(1))
            xs.sort()
            ws = [mpm.mpf(2) / (n * (n + 1) * pp(x)[0] ** 2) for x in xs]
            return xs, ws
        xs = []
        for i in range(1, n + 1):
            x = mpm.cospi((i - mpm.mpf(1) / 4) / (n + mpm.mpf(1) / 2))
            for _ in range(80):
                p, dp = pp(x)
                dx = p / dp
                x -= dx
                if abs(dx) < tiny:
                    break
            xs.append(x)
        xs.sort()
        return xs, [mpm.mpf(2) / ((1 - x * x) * pp(x)[1] ** 2) for x in xs]


def _quadrature_table(n: int, lobatto: bool):
    """The table of SABA_n (kicks at the n Gauss nodes) or SBAB_n (kicks at the n + 1 Lobatto nodes) on [0, 1]: the
    drifts before each kick and after the last, the kick weights, the first half mirrored onto the second so the
    table is bitwise symmetric, each value rounded to Float64 once (tables_near.jl:47-61)."""
    import mpmath as mpm
    if n < 1:
        raise ValueError(f"SABA/SBAB need n >= 1, got {n}")
    xs, ws = _legendre_rule(n, lobatto)
    with mpm.workprec(330):
        xs = [(x + 1) / 2 for x in xs]
        ws = [w / 2 for w in ws]
        m = len(xs)
        cb = [xs[0]] + [xs[j] - xs[j - 1] for j in range(1, m)] + [1 - xs[-1]]
        k = m + 1
        c = [float(cb[(i if i <= (k + 1) // 2 else k + 1 - i) - 1]) for i in range(1, k + 1)]
        d = [0.0 if i == k else float(ws[(i if i <= (m + 1) // 2 else m + 1 - i) - 1]) for i in range(1, k + 1)]
    return c, d


def SABA(n: int) -> SplittingMethod:
    """SABA_n (Laskar and Robutel 2001): the symmetric splitting A B A ... with kicks at the n Gauss-Legendre nodes,
    order (2n, 2) in (tau, eps) for H = A + eps B (src/Integrators/tables_near.jl:63-67)."""
    c, d = _quadrature_table(int(n), False)
    return SplittingMethod(c, d, order=2, palindromic=True, name=f"SABA{n}", digits=40, source="LaskarRobutel2001")


def SBAB(n: int) -> SplittingMethod:
    """SBAB_n (Laskar and Robutel 2001): kicks at the n + 1 Gauss-Lobatto nodes, the first and last drifts exactly 0
    (src/Integrators/tables_near.jl:69-73)."""
    c, d = _quadrature_table(int(n), True)
    return SplittingMethod(c, d, order=2, palindromic=True, name=f"SBAB{n}", digits=40, source="LaskarRobutel2001")


# Blanes et al. (2013) Table 3 (ABA864) and Table 4 (ABAH864): a_1.. and b_1.. of a1 b1 a2 b2 ... b2 a2 b1 a1,
# 40 digits as published.
_ABA864_A = ("0.0711334264982231177779387300061549964174", "0.241153427956640098736487795326289649618",
             "0.521411761772814789212136078067994229991", "-0.333698616227678005726562603400438876027")
_ABA864_B = ("0.183083687472197221961703757166430291072", "0.310782859898574869507522291054262796375",
             "-0.0265646185119588006972121379164987592663", "0.0653961422823734184559721793911134363710")
_ABAH864_A = ("0.06810235651658372084723976682061164571212", "0.2511360387221033233072829580455350680082",
              "-0.07507264957216562516006821767601620052338", "-0.009544719701745007811488218957217113269121",
              "0.5307579480704471776340674235341732001443")
_ABAH864_B = ("0.1684432593618954534310382697756917558148", "0.4243177173742677224300351657407231801453",
              "-0.5858109694681756812309015355404036521923", "0.4930499927320125053698281000239887162321")


def ABA864() -> SplittingMethod:
    """ABA864 (Blanes et al. 2013 Table 3), 8 stages, generalized order (8, 6, 4) (tables_near.jl:80-88): the
    central kick b_4 is recomputed as 1 - 2 (b_1 + b_2 + b_3) in binary64, since the printed b_i sum to 1 only to
    5e-31."""
    a = [float(v) for v in _ABA864_A]
    b = [float(v) for v in _ABA864_B]
    b[3] = 1.0 - 2.0 * (b[0] + b[1] + b[2])
    c = [a[0], a[1], a[2], a[3], a[3], a[2], a[1], a[0]]
    d = [b[0], b[1], b[2], b[3], b[2], b[1], b[0], 0.0]
    return SplittingMethod(c, d, order=4, palindromic=True, name="ABA864", source="Blanes2013", digits=40)


def ABAH864() -> SplittingMethod:
    """ABAH864 (Blanes et al. 2013 Table 4), 9 stages (tables_near.jl:91-97)."""
    a = [float(v) for v in _ABAH864_A]
    b = [float(v) for v in _ABAH864_B]
    c = [a[0], a[1], a[2], a[3], a[4], a[3], a[2], a[1], a[0]]
    d = [b[0], b[1], b[2], b[3], b[3], b[2], b[1], b[0], 0.0]
    return SplittingMethod(c, d, order=4, palindromic=True, name="ABAH864", source="Blanes2013", digits=40)


# Laskar and Robutel (2001) Table II: the coefficient c of {{A,B},B} in the modified Hamiltonian, 40 digits as
# published, for the n that have no closed form.
_CORR_SABA = {4: "0.003396775048208601331532157783492144", 5: "0.002270543121419264819434955050039130",
              6: "0.001624459841624282521452258512463608", 7: "0.001219643912760418472579211822331645",
              8: "0.000949308177745602234792177503535054", 9: "0.000759846022860436646358196674176815",
              10: "0.000621934331486166426497049845358646"}
_CORR_SBAB = {5: "0.002381486672953634187470386232181453", 6: "0.001681346512091906326563693215296434",
              7: "0.001251765616039400003072516100251191", 8: "0.000968797968073688571654684208462982",
              9: "0.000772349023999952078227686810260323", 10: "0.000630320044163167840798638762665112"}


def _corrector_c(n: int, sbab: bool) -> float:
    """The corrector coefficient of SABA_n / SBAB_n (tables_near.jl:107-111): the closed forms of Table II for the
    small n, evaluated in binary64, else the tabulated value."""
    if not 1 <= n <= 10:
        raise ValueError(f"the corrector coefficient is tabulated for n = 1 to 10 (Laskar and Robutel 2001 Table II), got {n}")
    if sbab:
        closed = {1: lambda: -1.0 / 24.0, 2: lambda: 1.0 / 72.0, 3: lambda: (13.0 - 5.0 * math.sqrt(5.0)) / 288.0,
                  4: lambda: (3861.0 - 791.0 * math.sqrt(21.0)) / 64800.0}
        return closed[n]() if n in closed else float(_CORR_SBAB[n])
    closed = {1: lambda: 1.0 / 12.0, 2: lambda: (2.0 - math.sqrt(3.0)) / 24.0,
              3: lambda: (54.0 - 13.0 * math.sqrt(15.0)) / 648.0}
    return closed[n]() if n in closed else float(_CORR_SABA[n])


@dataclass(frozen=True)
class CorrectedMethod:
    """CorrectedMethod(base, c), tables_near.jl:113-123 and stepper.jl:131-172: the corrector kick
    exp(-kappa L_F), F = |grad V|^2, kappa = tau^3 eps^2 c / 2, before and after the symmetric table `base`
    (for the Henon-Heiles flow eps = perturbation_scale = 1 and grad F = 2 Hs grad V, flow_models.jl:106-112)."""
    base: SplittingMethod
    c: float
    order: int

    @property
    def name(self) -> str:
        return self.base.name[:4] + "C" + self.base.name[4:]

    @property
    def palindromic(self) -> bool:
        return True

    @property
    def stages(self) -> int:
        return self.base.stages

    def force_evaluations(self) -> int:
        return self.base.isolated_force_evaluations() + 2

    def isolated_force_evaluations(self) -> int:
        return self.base.isolated_force_evaluations() + 2


def SABAC(n: int) -> CorrectedMethod:
    """SABA_n with the corrector kick before and after; order 4 in eps for n >= 2 (tables_near.jl:125-126)."""
    return CorrectedMethod(SABA(n), _corrector_c(int(n), False), 4 if n >= 2 else 2)


def SBABC(n: int) -> CorrectedMethod:
    """SBAB_n with the corrector (tables_near.jl:127-128)."""
    return CorrectedMethod(SBAB(n), _corrector_c(int(n), True), 4 if n >= 2 else 2)


def coefficients(m):
    """(c, d), the drift and kick weights of a table method (of the base table of a corrected method)."""
    m = m.base if isinstance(m, CorrectedMethod) else m
    return m.c, m.d


def stage_count(m) -> int:
    return m.stages


def nominal_order(m) -> int:
    return m.order


def is_palindromic(m) -> bool:
    return m.palindromic


def table_digits(m) -> float:
    return (m.base if isinstance(m, CorrectedMethod) else m).digits


def method_name(m) -> str:
    return m.name


def method_source(m) -> str:
    return (m.base if isinstance(m, CorrectedMethod) else m).source


def force_evaluations(m) -> int:
    return m.force_evaluations()


def isolated_force_evaluations(m) -> int:
    return m.isolated_force_evaluations()


class IntegratorMap(System):
    """IntegratorMap(method, flow, tau), src/Integrators/integrator_map.jl:12-23: one step of the flow as a map, by
    Gauss (gauss.jl:49-192) or a table method (stepper.jl:27-48); the tangent is the exact Jacobian of the step
    (gauss.jl:176-192; stepper.jl:108-118, the product of the stage Jacobians)."""

    def __init__(self, method, flow: HenonHeilesFlow, tau: float):
        if not isinstance(flow, HenonHeilesFlow):
            raise TypeError("the compiled menu integrates HenonHeilesFlow")
        if not isinstance(method, (Gauss, SplittingMethod, CorrectedMethod)):
            raise TypeError("the compiled menu integrates with Gauss(3) or a SplittingMethod table")
        if isinstance(method, (SplittingMethod, CorrectedMethod)) and method.stages > _abi.MAX_STAGES:
            raise ValueError(f"a table of {method.stages} stages is above the compiled limit ({_abi.MAX_STAGES})")
        self.method, self.flow, self.tau = method, flow, float(tau)
        self.d = self.s = 4
        kind = "Gauss3" if isinstance(method, Gauss) else type(method).__name__
        self.name = f"IntegratorMap{{{kind},HenonHeilesFlow}}"

    def to_cl(self):
        if isinstance(self.method, (SplittingMethod, CorrectedMethod)):
            corrected = isinstance(self.method, CorrectedMethod)
            table = self.method.base if corrected else self.method
            k = table.stages
            cs = _abi.cl_system(kind=_abi.SYS_HH_SPLIT, dt=self.tau, n_stages=k, gauss_tol=math.nan,
                                corrector=int(corrected), eps=float(self.method.c) if corrected else 0.0)
            for i in range(k):
                cs.stage_c[i] = table.c[i]
                cs.stage_d[i] = table.d[i]
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


def _torus(z, d: int) -> np.ndarray:
    """The d coordinates of z each reduced into [0, 2 pi) (_reduce), followed by their d counts."""
    tp = 2 * _PI
    r = [_reduce(float(v), tp) for v in z[:d]]
    return np.array([v for v, _ in r] + [c for _, c in r])


def _lift(s, d: int) -> np.ndarray:
    tp = 2 * _PI
    return np.array([s[j] + tp * s[d + j] for j in range(d)])


def torus_state(*args) -> np.ndarray:
    """torus_state((X, P)) -> (x, p, m, n), src/Systems/wrapped_standard_map.jl:63-69; torus_state(sys, z) for the
    wrapped Froeschle map and the wrapped chain."""
    if len(args) == 2:
        return args[0].torus_state(args[1])
    return _torus(args[0], 2)


def lift(*args) -> np.ndarray:
    """lift((x, p, m, n)) -> (x + 2 pi m, p + 2 pi n), src/Systems/wrapped_standard_map.jl:77-80; lift(sys, s) for
    the wrapped Froeschle map and the wrapped chain."""
    if len(args) == 2:
        return args[0].lift(args[1])
    return _lift(args[0], 2)


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
