"""The study recorder on the B200: `record` runs the variational methods with grid records, the device form of
`_variational_batch!` (src/Experiments/run_device.jl:167-189) over the library's `cl_b200_record`
(chaos_b200/csrc/cl_record.cu); `record_shadow` the two-trajectory method; `record_indicators` the indicator
recorder's tangent kind (src/Experiments/run_indicator_device.jl:31-60) over `cl_b200_indicator`
(chaos_b200/csrc/cl_indicator.cu).

At every grid step the record holds the estimator's exponents, the monitor's running maxima of the determinant and
symplecticity residuals of the tangent and of max|M|, the orthogonality loss, the running maxima of the sum and
pairing residuals (k = 2), G_max and the state (run_device.jl:10-35). An orbit that fails stops; its failing grid
index (1-based) is in `fail` and, as `_unpack!` does (run_device.jl:126-139), only the rows before it are
meaningful.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._lib import last_error, lib
from .foundation import DeviceError
from .propagate import FrameSpec, build_run
from .reducers import FLI, MEGNO, SALI, Benettin, QRSpectrum

COLUMNS = ("lambda", "det", "symp", "orth", "sum", "pair", "G_max", "M_max", "state")


@dataclass
class RecordResult:
    R: np.ndarray          # (n, n_grid, k + 7 + s): R[i, g] is the row of orbit i at grid step g
    grid: np.ndarray
    fail: np.ndarray       # 1-based failing grid index per orbit, 0 = none
    x: np.ndarray
    W: np.ndarray          # (n, d, k)
    states: np.ndarray     # the estimator's state then MonState, per orbit (raw bytes)
    code: np.ndarray
    hstep: np.ndarray
    k: int
    gpu_ms: float = 0.0

    def column(self, name: str) -> np.ndarray:
        """A named field of every row: "lambda" (n, n_grid, k), "state" (n, n_grid, s), else (n, n_grid)."""
        k = self.k
        if name == "lambda":
            return self.R[:, :, :k]
        if name == "state":
            return self.R[:, :, k + 7:]
        return self.R[:, :, k + COLUMNS.index(name) - 1]


def record(sys, x0, N: int, tau: int, estimator, grid, *, W0=None, launch_steps: int | None = None,
           precision: str = "fp64") -> RecordResult:
    """Record n orbits of `sys` (StandardMap, WrappedStandardMap or a 2 x 2 LinearSymplecticMap) with `estimator`
    (Benettin() with k = 1, or QRSpectrum(CGS / MGS / RGS / HouseholderQR / AugmentedQR) with k = 2) at the step
    counts `grid` (increasing multiples of tau, at most N). W0 defaults to I[:, 1:k]; `launch_steps` splits the run
    into launches that carry everything (the grid rows of a launch are written by it). `precision` "mixed" keeps the
    orbit, the monitor and the log sums in Float64 and the frame and its QR in Float32."""
    x0 = np.ascontiguousarray(np.asarray(x0, dtype=np.float64))
    n, s = x0.shape
    d = sys.d
    k = 1 if isinstance(estimator, Benettin) else 2
    if not isinstance(estimator, (Benettin, QRSpectrum)):
        raise ValueError("the recorder's estimators are Benettin and QRSpectrum")
    grid = np.ascontiguousarray(np.asarray(grid, dtype=np.int64))
    if grid.ndim != 1 or len(grid) < 1 or np.any(np.diff(grid) <= 0) or grid[0] < tau or grid[-1] > N or \
            np.any(grid % tau):
        raise ValueError("grid: increasing multiples of tau in tau..N")
    L = int(launch_steps) if launch_steps else int(N)
    if L % tau:
        raise ValueError("launch_steps must be a multiple of tau")
    run = build_run(sys, N, tau, [FrameSpec(k, (estimator,))], precision, 0, steps=L)
    Lb = lib()
    ncol = Lb.cl_b200_record_columns(C.byref(run))
    sb = Lb.cl_b200_record_state_bytes(C.byref(run))
    if W0 is None:
        W0 = np.broadcast_to(np.eye(d)[:, :k], (n, d, k))
    Wc = np.ascontiguousarray(np.asarray(W0, dtype=np.float64).transpose(0, 2, 1))   # columns of d contiguous
    x = x0.copy()
    states = np.zeros((n, sb), np.uint8)
    code = np.zeros(n, np.int8)
    hstep = np.zeros(n, np.int64)
    R = np.zeros((n, len(grid), ncol))
    fail = np.zeros(n, np.int64)
    prov = _abi.cl_prov()
    rc = Lb.cl_b200_record(C.byref(run), n, x.ctypes.data, Wc.ctypes.data, states.ctypes.data, code.ctypes.data,
                           hstep.ctypes.data, grid.ctypes.data, len(grid), R.ctypes.data, fail.ctypes.data,
                           C.byref(prov))
    if rc != 0:
        msg = last_error()
        if rc == _abi.EINVAL:
            raise ValueError(msg)
        raise DeviceError(rc, msg)
    return RecordResult(R=R, grid=grid, fail=fail, x=x, W=Wc.transpose(0, 2, 1), states=states, code=code,
                        hstep=hstep, k=k, gpu_ms=prov.gpu_ms)


def record_shadow(sys, x0, N: int, tau: int, grid, *, d0: float, seed: int = 0, U0=None,
                  launch_steps: int | None = None):
    """The recorder's two-trajectory method (`_shadow_batch!`, run_device.jl:191-214): at the grid steps, X2 so far
    and the reference state (R (n, n_grid, 8 + s): column 0 and columns 8..), the 1-based failing grid index per
    orbit (`fail`), and the end records (ShadowEnd layout). U0 rows are normalised by safe_norm as
    `propagate_shadow` does; without U0 the directions are the seeded frames' first columns."""
    from .shadow import _safe_norm, end_dtype
    x0 = np.ascontiguousarray(np.asarray(x0, dtype=np.float64))
    n, s = x0.shape
    grid = np.ascontiguousarray(np.asarray(grid, dtype=np.int64))
    if grid.ndim != 1 or len(grid) < 1 or np.any(np.diff(grid) <= 0) or grid[0] < tau or grid[-1] > N or \
            np.any(grid % tau):
        raise ValueError("grid: increasing multiples of tau in tau..N")
    L = int(launch_steps) if launch_steps else int(N)
    u = None
    if U0 is not None:
        U0 = np.asarray(U0, dtype=np.float64)
        u = np.ascontiguousarray([[float(v) / _safe_norm(row) for v in row] for row in U0])
    run = build_run(sys, N, tau, [FrameSpec(1, ())], "fp64", seed, steps=L)
    ends = np.zeros(n, dtype=end_dtype(s))
    R = np.zeros((n, len(grid), 8 + s))
    fail = np.zeros(n, np.int64)
    prov = _abi.cl_prov()
    rc = lib().cl_b200_shadow_record(C.byref(run), n, x0.ctypes.data, None if u is None else u.ctypes.data,
                                     ends.ctypes.data, float(d0), grid.ctypes.data, len(grid), R.ctypes.data,
                                     fail.ctypes.data, C.byref(prov))
    if rc != 0:
        msg = last_error()
        if rc == _abi.EINVAL:
            raise ValueError(msg)
        raise DeviceError(rc, msg)
    return R, fail, ends


# The columns of each member (IND_MEMBER_COLUMNS, src/Experiments/run_indicator_chain.jl:16-17)
MEMBER_COLUMNS = {"SALI": ("SALI.sali", "SALI.L"), "FLI": ("FLI.fli", "FLI.fli1"),
                  "MEGNO": ("MEGNO.Y1", "MEGNO.Ybar1", "MEGNO.Ybar20_1", "MEGNO.Y2", "MEGNO.Ybar2", "MEGNO.Ybar20_2")}


def indicator_chain(members) -> tuple:
    """`chain_members` (run_indicator_chain.jl:27-28): the reducers in order, every member but the last
    non-replacing, the last replacing (SALI has one form)."""
    members = [str(m) for m in members]
    if not members or any(m not in MEMBER_COLUMNS for m in members):
        raise ValueError(f"members must be a non-empty list of SALI, FLI, MEGNO, got {members}")
    out = []
    for i, m in enumerate(members):
        last = i == len(members) - 1
        out.append(SALI() if m == "SALI" else FLI(replace=last) if m == "FLI" else MEGNO(replace=last))
    return tuple(out)


@dataclass
class IndicatorRecord:
    R: np.ndarray          # (n, n_grid, ncol): the members' columns, det_max, symp_max, M_max, x[:ns]
    columns: tuple
    grid: np.ndarray
    fail: np.ndarray       # 1-based failing grid index per orbit, 0 = none
    x: np.ndarray
    W: np.ndarray          # (n, d, 2)
    states: np.ndarray     # the members' states then the monitor's maxima, per orbit (raw bytes)
    code: np.ndarray
    hstep: np.ndarray
    gpu_ms: float = 0.0

    def column(self, name: str) -> np.ndarray:
        return self.R[:, :, self.columns.index(name)]


def record_indicators(sys, x0, N: int, tau: int, members, grid, *, ns: int = 2, W0=None,
                      launch_steps: int | None = None) -> IndicatorRecord:
    """The indicator recorder's tangent kind for n orbits of `sys` (StandardMap, WrappedStandardMap or a 2 x 2
    LinearSymplecticMap): the chain of `members` (names, e.g. ["MEGNO", "SALI"]) on the frame W0 (default I) with
    the non-raising monitor after it; at the step counts `grid` (increasing multiples of tau, at most N) one row of
    the members' series columns (E24 order), det_max, symp_max, M_max and the first `ns` coordinates. An orbit that
    fails stops; its failing grid index (1-based) is in `fail` and only the rows before it are meaningful."""
    x0 = np.ascontiguousarray(np.asarray(x0, dtype=np.float64))
    n, s = x0.shape
    d = sys.d
    chain = indicator_chain(members)
    grid = np.ascontiguousarray(np.asarray(grid, dtype=np.int64))
    if grid.ndim != 1 or len(grid) < 1 or np.any(np.diff(grid) <= 0) or grid[0] < tau or grid[-1] > N or \
            np.any(grid % tau):
        raise ValueError("grid: increasing multiples of tau in tau..N")
    if not 0 <= ns <= s:
        raise ValueError(f"ns must lie in 0..{s}")
    L = int(launch_steps) if launch_steps else int(N)
    if L % tau:
        raise ValueError("launch_steps must be a multiple of tau")
    run = build_run(sys, N, tau, [FrameSpec(2, chain)], "fp64", 0, steps=L)
    Lb = lib()
    ncol = Lb.cl_b200_indicator_columns(C.byref(run), ns)
    if ncol < 0:
        raise ValueError(f"member chain {members} is outside the compiled menu")
    sb = Lb.cl_b200_indicator_state_bytes(C.byref(run))
    if W0 is None:
        W0 = np.broadcast_to(np.eye(d)[:, :2], (n, d, 2))
    Wc = np.ascontiguousarray(np.asarray(W0, dtype=np.float64).transpose(0, 2, 1))
    x = x0.copy()
    states = np.zeros((n, sb), np.uint8)
    code = np.zeros(n, np.int8)
    hstep = np.zeros(n, np.int64)
    R = np.zeros((n, len(grid), ncol))
    fail = np.zeros(n, np.int64)
    prov = _abi.cl_prov()
    rc = Lb.cl_b200_indicator(C.byref(run), n, ns, x.ctypes.data, Wc.ctypes.data, states.ctypes.data,
                              code.ctypes.data, hstep.ctypes.data, grid.ctypes.data, len(grid), R.ctypes.data,
                              fail.ctypes.data, C.byref(prov))
    if rc != 0:
        msg = last_error()
        if rc == _abi.EINVAL:
            raise ValueError(msg)
        raise DeviceError(rc, msg)
    cols = tuple(c for m in members for c in MEMBER_COLUMNS[m]) + ("det_max", "symp_max", "M_max") + \
        tuple(f"x{j + 1}" for j in range(ns))
    return IndicatorRecord(R=R, columns=cols, grid=grid, fail=fail, x=x, W=Wc.transpose(0, 2, 1), states=states,
                           code=code, hstep=hstep, gpu_ms=prov.gpu_ms)


# ---- the pair kind ------------------------------------------------------------------------------------------------
PAIR_MEMBER_COLUMNS = {"RLI": ("RLI.DL", "RLI.RLI"), "MEGNO": MEMBER_COLUMNS["MEGNO"]}


def pair_chain(members) -> tuple:
    """The reducers of a pair chain (RLI, MEGNO; run_indicator_chain.jl:26-28): the last member replacing."""
    from .reducers import RLI
    members = [str(m) for m in members]
    if not members or any(m not in PAIR_MEMBER_COLUMNS for m in members):
        raise ValueError(f"pair members must be a non-empty list of RLI, MEGNO, got {members}")
    return tuple(RLI(replace=i == len(members) - 1) if m == "RLI" else MEGNO(replace=i == len(members) - 1)
                 for i, m in enumerate(members))


def _wrap_diff(u: float, tp: float) -> float:
    """_wrap_diff (rli.jl:135): u - tp round(u / tp), round half to even as Julia's `round`."""
    return u - tp * float(round(u / tp))


def pair_distance(sys, z) -> float:
    """pair_distance (rli.jl:150): safe_norm of the minimal-image separation of the halves of a pair state for the
    standard maps (each coordinate difference reduced modulo 2 pi), the plain difference otherwise."""
    from .shadow import _PI, _safe_norm
    from .systems import StandardMap, WrappedStandardMap
    z = [float(v) for v in z]
    h = len(z) // 2
    if isinstance(sys, (StandardMap, WrappedStandardMap)):
        tp = 2 * _PI
        return _safe_norm([_wrap_diff(z[h] - z[0], tp), _wrap_diff(z[h + 1] - z[1], tp)])
    return _safe_norm([z[h + i] - z[i] for i in range(h)])


def pair_start(sys, x0, u, Dx: float, *, orbit: int = 0):
    """pair_start (rli.jl:182-193): (z, Dx, Dx_r, mode) with z = (A; B), A = x0 (torus_state(x0) for the wrapped map)
    and B = A + Dx u (reduced with A's counts in wrapped mode); a Dx that is not finite and positive, or a realised
    separation that is zero, not finite or outside [Dx / 2, 2 Dx], raises NumericalHealthError("separation") at
    step 0 for `orbit`."""
    import math
    from .foundation import NumericalHealthError
    from .shadow import _displaced
    from .systems import WrappedStandardMap, torus_state
    dx = float(Dx)
    if not (math.isfinite(dx) and dx > 0):
        raise NumericalHealthError("separation", dx, 0.0 if math.isfinite(dx) else math.inf, 0, orbit, "cpu")
    zA = np.asarray(torus_state(x0) if isinstance(sys, WrappedStandardMap) else x0, dtype=np.float64)
    zB = np.asarray(_displaced(sys, zA, [dx * float(v) for v in u]), dtype=np.float64)
    z = np.concatenate([zA, zB])
    dr = pair_distance(sys, z)
    if not (math.isfinite(dr) and dr > 0):
        raise NumericalHealthError("separation", dr, 0.0 if math.isfinite(dr) else math.inf, 0, orbit, "cpu")
    if not (dr >= dx / 2 and dr <= 2 * dx):
        raise NumericalHealthError("separation", dr, dx, 0, orbit, "cpu")
    return z, dx, dr, "wrapped" if isinstance(sys, WrappedStandardMap) else "lifted"


def pair_frame(xi) -> np.ndarray:
    """The block frame of a pair, (xi; 0) and (0; xi) (run_indicator_record.jl:230-231), as a (2 d, 2) array."""
    xi = np.asarray(xi, dtype=np.float64)
    d = len(xi)
    W = np.zeros((2 * d, 2))
    W[:d, 0] = xi
    W[d:, 1] = xi
    return W


def record_indicator_pairs(sys, z0, W0, N: int, tau: int, members, grid, *, ns: int = 2,
                           launch_steps: int | None = None) -> IndicatorRecord:
    """The indicator recorder's pair kind: the chain of `members` (RLI, MEGNO) and the monitor on PairMap(sys) from
    the pair states z0 (n, 2 s; `pair_start`) and block frames W0 (n, 2 d, 2; `pair_frame`), rows at the step
    counts `grid` as `record_indicators` writes them (RLI's columns DL, RLI; the monitor reads orbit A; the first
    `ns` coordinates of the pair state)."""
    from .systems import LinearSymplecticMap, StandardMap, WrappedStandardMap
    if not isinstance(sys, (StandardMap, WrappedStandardMap, LinearSymplecticMap)):
        raise TypeError("the pair kind covers the standard maps and 2 x 2 linear maps")
    z0 = np.ascontiguousarray(np.asarray(z0, dtype=np.float64))
    n, s2 = z0.shape
    if s2 != 2 * sys.s:
        raise ValueError(f"a pair state has {2 * sys.s} entries, got {s2}")
    d = sys.d
    W0 = np.asarray(W0, dtype=np.float64)
    if W0.shape != (n, 2 * d, 2):
        raise ValueError(f"W0 must be (orbits, {2 * d}, 2)")
    chain = pair_chain(members)
    grid = np.ascontiguousarray(np.asarray(grid, dtype=np.int64))
    if grid.ndim != 1 or len(grid) < 1 or np.any(np.diff(grid) <= 0) or grid[0] < tau or grid[-1] > N or \
            np.any(grid % tau):
        raise ValueError("grid: increasing multiples of tau in tau..N")
    if not 0 <= ns <= s2:
        raise ValueError(f"ns must lie in 0..{s2}")
    L = int(launch_steps) if launch_steps else int(N)
    if L % tau:
        raise ValueError("launch_steps must be a multiple of tau")
    run = build_run(sys, N, tau, [FrameSpec(2, chain)], "fp64", 0, steps=L)
    Lb = lib()
    ncol = Lb.cl_b200_indicator_pair_columns(C.byref(run), ns)
    if ncol < 0:
        raise ValueError(f"pair chain {members} is outside the compiled menu")
    sb = Lb.cl_b200_indicator_state_bytes(C.byref(run))
    Wc = np.ascontiguousarray(W0.transpose(0, 2, 1))
    x = z0.copy()
    states = np.zeros((n, sb), np.uint8)
    code = np.zeros(n, np.int8)
    hstep = np.zeros(n, np.int64)
    R = np.zeros((n, len(grid), ncol))
    fail = np.zeros(n, np.int64)
    prov = _abi.cl_prov()
    rc = Lb.cl_b200_indicator_pair(C.byref(run), n, ns, x.ctypes.data, Wc.ctypes.data, states.ctypes.data,
                                   code.ctypes.data, hstep.ctypes.data, grid.ctypes.data, len(grid), R.ctypes.data,
                                   fail.ctypes.data, C.byref(prov))
    if rc != 0:
        msg = last_error()
        if rc == _abi.EINVAL:
            raise ValueError(msg)
        raise DeviceError(rc, msg)
    cols = tuple(c for m in members for c in PAIR_MEMBER_COLUMNS[m]) + ("det_max", "symp_max", "M_max") + \
        tuple(f"z{j + 1}" for j in range(ns))
    return IndicatorRecord(R=R, columns=cols, grid=grid, fail=fail, x=x, W=Wc.transpose(0, 2, 1), states=states,
                           code=code, hstep=hstep, gpu_ms=prov.gpu_ms)
