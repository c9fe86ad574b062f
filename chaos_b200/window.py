"""The indicator recorder's window kinds on the B200 (src/Experiments/run_indicator_device.jl:62-91): the weighted
phase advance (src/Indicators/naff_reducer.jl:122-243) and the weighted Birkhoff averages
(src/Indicators/wbirkhoff_reducer.jl:18-137) as reader reducers of the orbit point, run after the non-raising
monitor with the deviation column reset at each handoff, rows of the monitor and the orbit point at the grid steps,
and the readers' finals (`reducer_final`, with `frequency_index`, `circle_distance` and `birkhoff_index`) computed on
the host from the carried states. The device work is `cl_b200_indicator_window` (chaos_b200/csrc/cl_window.cu).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._lib import last_error, lib
from .foundation import DeviceError
from .propagate import FrameSpec, build_run

MIN_WINDOW = 16          # NF_E2_MIN_WINDOW = WB_MIN_WINDOW (naff_reducer.jl:5, wbirkhoff.jl:5)
FLOOR_MULTIPLIER = 32    # WB_FLOOR_MULTIPLIER and frequency_index's default (wbirkhoff.jl:6, naff_map.jl:26)
_EPS = 2.0 ** -52
_TINY = 2.2250738585072014e-308
_TWO_PI = 2 * 3.141592653589793


# ---- observables (naff_reducer.jl:89-117, wbirkhoff.jl:12-56, run_indicator_chain.jl:20-23); indices are 1-based
@dataclass(frozen=True)
class PlanarObservable:
    iq: int
    ip: int
    kind = _abi.OBS_PLANAR

    def cl(self):
        return self.iq, self.ip


@dataclass(frozen=True)
class LiftedAngleObservable:
    iq: int
    im: int = 0
    kind = _abi.OBS_LIFTED_ANGLE

    def cl(self):
        return self.iq, self.im


@dataclass(frozen=True)
class CosObservable:
    i: int
    k: int = 1
    kind = _abi.OBS_COS

    def cl(self):
        return self.i, self.k


@dataclass(frozen=True)
class SinObservable:
    i: int
    k: int = 1
    kind = _abi.OBS_SIN

    def cl(self):
        return self.i, self.k


@dataclass(frozen=True)
class LiftedObservable:
    iq: int
    im: int
    kind = _abi.OBS_LIFTED

    def cl(self):
        return self.iq, self.im


@dataclass(frozen=True)
class IndCoordinate:
    i: int
    kind = _abi.OBS_COORDINATE

    def cl(self):
        return self.i, 0


def _windows(window) -> tuple:
    ws = (int(window),) if isinstance(window, (int, np.integer)) else tuple(int(w) for w in window)
    if not ws or any(w < MIN_WINDOW for w in ws) or len(ws) > _abi.MAX_WINDOWS:
        raise ValueError(f"window must be at least {MIN_WINDOW} (1 to {_abi.MAX_WINDOWS} horizons), got {window}")
    return ws


def _order(p) -> int:
    if not (isinstance(p, (int, np.integer)) and 1 <= p <= 4):
        raise ValueError(f"birkhoff_order must be an integer from 1 to 4 (the centre weight exp(-4^p) underflows "
                         f"above), got {p}")
    return int(p)


def circle_distance(a: float, b: float) -> float:
    """circle_distance (naff_map.jl:9): |d - round(d)|, d = a - b."""
    d = a - b
    return abs(d - round(d)) if math.isfinite(d) else math.nan


def frequency_index(delta: float, floor_multiplier: float = FLOOR_MULTIPLIER):
    """frequency_index (naff_map.jl:26-29): (D, below_floor, delta_floor)."""
    fl = floor_multiplier * _EPS
    return math.log10(max(delta, fl)), delta <= fl, fl


def birkhoff_index(avg1: float, avg2: float, S: float, floor_multiplier: float = FLOOR_MULTIPLIER) -> dict:
    """birkhoff_index (wbirkhoff.jl:156-171)."""
    delta = avg1 - avg2
    phi = max(floor_multiplier * _EPS * S, _TINY)
    a = abs(delta)
    below = a <= phi
    nan = math.nan
    if S == 0:
        return dict(delta=delta, absdig=nan, reldig=nan, dig=nan, below_floor=below, zero=True)
    if not math.isfinite(a):
        return dict(delta=delta, absdig=nan, reldig=nan, dig=nan, below_floor=False, zero=False)
    e = max(a, phi)
    m = abs(avg1) / 2 + abs(avg2) / 2
    absdig = -math.log10(e)
    reldig = -math.log10(e / m) if m > phi else nan
    return dict(delta=delta, absdig=absdig, reldig=reldig, dig=absdig if math.isnan(reldig) else max(absdig, reldig),
                below_floor=below, zero=False)


class WeightedPhaseAdvance:
    """WeightedPhaseAdvance(; window, observable, birkhoff_order = 1) (naff_reducer.jl:122-154)."""

    kind = _abi.WIN_PHASE_ADVANCE

    def __init__(self, *, window, observable, birkhoff_order: int = 1):
        if not isinstance(observable, (PlanarObservable, LiftedAngleObservable)):
            raise ValueError("the phase advance reads a PlanarObservable or a LiftedAngleObservable")
        self.window, self.observables, self.birkhoff_order = _windows(window), (observable,), _order(birkhoff_order)

    def handoffs(self) -> int:
        return 2 * max(self.window) + 1

    def check_run(self, tau: int, N: int) -> None:
        """check_run (naff_reducer.jl:236-243): N / tau = 2 max(window) + 1 handoffs."""
        need = self.handoffs()
        if not (N % tau == 0 and N // tau == need):
            raise ValueError(f"the run of {N} steps at tau = {tau} does not have the {need} handoffs (2 window + 1) "
                             f"that window = {self.window} needs")

    def state_bytes(self) -> int:
        return 64 * len(self.window) + 32

    def final(self, raw: bytes) -> dict:
        """reducer_final (naff_reducer.jl:222-232) from the WPAState{Float64, H} bytes."""
        H = len(self.window)
        f = np.frombuffer(raw[:64 * H], dtype="<f8").reshape(H, 8)
        tail = raw[64 * H:]
        n = int(np.frombuffer(tail[16:24], "<i8")[0])
        s = int(np.frombuffer(tail[24:28], "<i4")[0])
        nwrap = int(np.frombuffer(tail[28:30], "<i2")[0])
        nu1, nu2, delta, D, below = [], [], [], [], []
        for h, N in enumerate(self.window):
            A1, B1, A2, B2 = f[h, 0] + f[h, 1], f[h, 2] + f[h, 3], f[h, 4] + f[h, 5], f[h, 6] + f[h, 7]
            v1 = float(A1 / (_TWO_PI * B1)) if s >= N + 1 else math.nan
            v2 = float(A2 / (_TWO_PI * B2)) if s >= 2 * N + 1 else math.nan
            dl = circle_distance(v1, v2)
            nu1.append(v1); nu2.append(v2); delta.append(dl)
            if math.isnan(dl):
                D.append(math.nan); below.append(False)
            else:
                ix = frequency_index(dl)
                D.append(ix[0]); below.append(ix[1])
        return dict(n=n, handoffs=s, complete=s >= 2 * max(self.window) + 1, near_pi=nwrap, nu1=np.array(nu1),
                    nu2=np.array(nu2), delta=np.array(delta), D=np.array(D), below_floor=np.array(below))


class WeightedBirkhoff:
    """WeightedBirkhoff(; window, observables, birkhoff_order = 1) (wbirkhoff_reducer.jl:18-33)."""

    kind = _abi.WIN_BIRKHOFF

    def __init__(self, *, window, observables, birkhoff_order: int = 1):
        obs = tuple(observables)
        ok = (CosObservable, SinObservable, LiftedObservable, IndCoordinate)
        if not (1 <= len(obs) <= _abi.MAX_OBSERVABLES and all(isinstance(o, ok) for o in obs)):
            raise ValueError(f"observables must be a nonempty tuple of at most {_abi.MAX_OBSERVABLES} of the cos, "
                             "sin, lifted and coordinate observables")
        self.window, self.observables, self.birkhoff_order = _windows(window), obs, _order(birkhoff_order)

    def handoffs(self) -> int:
        return 2 * max(self.window)

    def check_run(self, tau: int, N: int) -> None:
        """check_run (wbirkhoff_reducer.jl:118-135): N / tau = 2 max(window) handoffs."""
        need = self.handoffs()
        if not (N % tau == 0 and N // tau == need):
            raise ValueError(f"the run of {N} steps at tau = {tau} does not have the {need} handoffs (2 window) that "
                             f"window = {self.window} needs")

    def state_bytes(self) -> int:
        return 16 + len(self.window) * (16 + 40 * len(self.observables))

    def final(self, raw: bytes) -> dict:
        """reducer_final (wbirkhoff_reducer.jl:100-110) from the WBState{Float64, H, K} bytes."""
        H, K = len(self.window), len(self.observables)
        hb = 16 + 40 * K
        tail = raw[H * hb:]
        n = int(np.frombuffer(tail[0:8], "<i8")[0])
        s = int(np.frombuffer(tail[8:12], "<i4")[0])
        shape = (K, H)
        out = {k: np.full(shape, math.nan) for k in ("avg1", "avg2", "S", "delta", "absdig", "reldig", "dig")}
        out["below_floor"] = np.zeros(shape, bool)
        out["zero"] = np.zeros(shape, bool)
        Bs = []
        for h, N in enumerate(self.window):
            hv = np.frombuffer(raw[h * hb:(h + 1) * hb], "<f8")
            B = float(hv[0] + hv[1])
            Bs.append(B)
            for k in range(K):
                c = hv[2 + 5 * k: 7 + 5 * k]
                S = float(c[4])
                a1 = float((c[0] + c[1]) / B) if s >= N else math.nan
                out["avg1"][k, h], out["S"][k, h] = a1, S
                if s < 2 * N:
                    continue
                a2 = float((c[2] + c[3]) / B)
                out["avg2"][k, h] = a2
                for key, v in birkhoff_index(a1, a2, S).items():
                    out[key][k, h] = v
        return dict(n=n, handoffs=s, complete=s >= 2 * max(self.window), B=np.array(Bs), **out)


def to_cl(reader) -> _abi.cl_window:
    w = _abi.cl_window(kind=reader.kind, n_windows=len(reader.window), n_observables=len(reader.observables),
                       birkhoff_order=reader.birkhoff_order)
    for h, N in enumerate(reader.window):
        w.window[h] = N
    for k, o in enumerate(reader.observables):
        w.obs_kind[k] = o.kind
        w.obs_a[k], w.obs_b[k] = o.cl()
    return w


@dataclass
class WindowRecord:
    R: np.ndarray          # (n, n_grid, 3 + ns): det_max, symp_max, M_max, x[:ns]
    grid: np.ndarray
    fail: np.ndarray       # 1-based failing grid index per orbit, 0 = none
    x: np.ndarray
    states: np.ndarray     # MonState then the reader's state, per orbit (raw bytes)
    code: np.ndarray
    hstep: np.ndarray
    finals: list           # the reader's reducer_final per orbit
    gpu_ms: float = 0.0


def record_indicator_window(sys, x0, N: int, tau: int, reader, grid, *, ns: int = 2, launch_steps: int | None = None,
                            check: bool = True) -> WindowRecord:
    """The window kinds of the indicator recorder for n orbits of `sys` (StandardMap, WrappedStandardMap or a 2 x 2
    LinearSymplecticMap) with `reader` (WeightedPhaseAdvance or WeightedBirkhoff): the orbit run N steps (`check`:
    the reader's check_run, N / tau handoffs), rows of the monitor and the first `ns` coordinates at `grid`, the
    reader's finals per orbit."""
    x0 = np.ascontiguousarray(np.asarray(x0, dtype=np.float64))
    n, s = x0.shape
    if not isinstance(reader, (WeightedPhaseAdvance, WeightedBirkhoff)):
        raise ValueError("the window kinds read a WeightedPhaseAdvance or a WeightedBirkhoff")
    if check:
        reader.check_run(tau, N)
    grid = np.ascontiguousarray(np.asarray(grid, dtype=np.int64))
    if grid.ndim != 1 or len(grid) < 1 or np.any(np.diff(grid) <= 0) or grid[0] < tau or grid[-1] > N or \
            np.any(grid % tau):
        raise ValueError("grid: increasing multiples of tau in tau..N")
    if not 0 <= ns <= s:
        raise ValueError(f"ns must lie in 0..{s}")
    L = int(launch_steps) if launch_steps else int(N)
    if L % tau:
        raise ValueError("launch_steps must be a multiple of tau")
    run = build_run(sys, N, tau, [FrameSpec(1, ())], "fp64", 0, steps=L)
    win = to_cl(reader)
    Lb = lib()
    sb = 24 + Lb.cl_b200_window_state_bytes(C.byref(win))
    x = x0.copy()
    states = np.zeros((n, sb), np.uint8)
    code = np.zeros(n, np.int8)
    hstep = np.zeros(n, np.int64)
    R = np.zeros((n, len(grid), 3 + ns))
    fail = np.zeros(n, np.int64)
    prov = _abi.cl_prov()
    rc = Lb.cl_b200_indicator_window(C.byref(run), C.byref(win), n, ns, x.ctypes.data, states.ctypes.data,
                                     code.ctypes.data, hstep.ctypes.data, grid.ctypes.data, len(grid), R.ctypes.data,
                                     fail.ctypes.data, C.byref(prov))
    if rc != 0:
        msg = last_error()
        if rc == _abi.EINVAL:
            raise ValueError(msg)
        raise DeviceError(rc, msg)
    finals = [reader.final(states[i, 24:].tobytes()) for i in range(n)]
    return WindowRecord(R=R, grid=grid, fail=fail, x=x, states=states, code=code, hstep=hstep, finals=finals,
                        gpu_ms=prov.gpu_ms)
