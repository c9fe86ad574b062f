"""The device launch plan of `propagate` (src/Tangent/propagate.jl:146-190) and its test hooks (:82-88, :169-177).

One launch must stay within a budget of LAUNCH_BUDGET_S seconds: a launch of L steps over m orbits takes about
ns 1e-9 L max(m, LAUNCH_WAVE) seconds, ns the device's measured nanoseconds per orbit-step for one wave of
LAUNCH_WAVE resident orbits. `budget_steps(ns, tau)` is the largest multiple of tau within the budget for one wave
(0 when even L = tau exceeds it), `budget_orbits(ns, L)` the orbits a launch of L steps may carry, and
`device_plan(forced, N, tau, ns)` gives (L, orbit cap): a forced L (the test hook `LAUNCH_STEPS`) keeps the wave
floor. A run of N steps is then ceil(N / L) launches per chunk that carry the state (D44).

`gpu_step_ns(precision)` is the per-machine record of the one-wave value: the reference keeps it in a git-ignored
benchmark file per device and precision (ext/ChaoslabCUDAExt.jl:42-62) and falls back to DEFAULT_GPU_NS without it;
here the record lives in chaos_b200/data/gpu-benchmark.toml (git-ignored; the reference's table layout
`[<device name>."<precision label>"]`, so the Julia extension reads the same file) and is measured on first use on a
device that has none (`record_step_ns`: the standard map K = 2 pi, k = 2, tau = 1, QRSpectrum(MGS), the reference's
record workload, timed on the device). The wave is the device's: LAUNCH_WAVE = 1024 is the orbits the reference's
card runs concurrently (its D29 measurement); a B200 runs 148 SMs x 512 threads = 75776 orbit threads at once, so
its record keeps `launch_wave` = SMs x 512 beside the value measured on that many orbits, and the plan uses both.

`BEFORE_LAUNCH` is the `_before_launch(device, chunk_index, launch, carried)` hook: when set, `propagate` runs its
launches one by one from the host and calls it before each with the live carried buffers.
"""
from __future__ import annotations

import math
import os
import threading

LAUNCH_BUDGET_S = 1.0   # seconds per launch (propagate.jl:147)
LAUNCH_WAVE = 1024      # orbits of one wave (propagate.jl:148)
DEFAULT_GPU_NS = 100.0  # ns per orbit-step without a record (propagate.jl:149)
INT_MAX = (1 << 63) - 1

LAUNCH_STEPS: int | None = None   # forced steps per launch (tests; propagate.jl:169-170)
BEFORE_LAUNCH = None              # callable(device, chunk_index, launch, carried) or None (propagate.jl:88)

_HERE = os.path.dirname(os.path.abspath(__file__))
RECORD_PATH = os.path.join(_HERE, "data", "gpu-benchmark.toml")
_lock = threading.Lock()
_cache: dict = {}


def budget_orbits(ns: float, L: int) -> int:
    """floor(min(budget / (ns 1e-9 L), typemax(Int) / 4)) (propagate.jl:152)."""
    return int(math.floor(min(LAUNCH_BUDGET_S / (ns * 1e-9 * L), INT_MAX // 4)))


def budget_steps(ns: float, tau: int, wave: int = LAUNCH_WAVE) -> int:
    """The largest multiple of tau with ns 1e-9 L wave <= budget; 0 when L = tau exceeds it (propagate.jl:154-167)."""
    def fits(m):
        return ns * 1e-9 * (m * tau) * wave <= LAUNCH_BUDGET_S
    cap = INT_MAX // (4 * tau)
    m = int(math.floor(min(LAUNCH_BUDGET_S / (ns * 1e-9 * wave * tau), cap)))
    while m > 0 and not fits(m):
        m -= 1
    while m < cap and fits(m + 1):
        m += 1
    return m * tau


def forced_launch(tau: int) -> int | None:
    """The forced launch length, checked against tau (propagate.jl:173-178)."""
    L = LAUNCH_STEPS
    if L is not None and not (L >= 1 and L % tau == 0):
        raise ValueError(f"forced steps per launch must be a positive multiple of tau, got L = {L}, tau = {tau}")
    return L


def device_plan(forced: int | None, N: int, tau: int, ns: float, wave: int = LAUNCH_WAVE) -> tuple[int, int]:
    """(steps per launch, orbit cap) (propagate.jl:183-190): (0, 0) when even L = tau exceeds the budget."""
    L = min(budget_steps(ns, tau, wave), N) if forced is None else min(forced, N)
    return (0, 0) if L == 0 else (L, max(wave, budget_orbits(ns, L)))


def launches(N: int, L: int) -> int:
    """ceil(N / L), 0 when L is 0 (propagate.jl:193)."""
    return 0 if L == 0 else -(-N // L)


def _label(precision: str) -> str:
    return "Float64" if precision == "fp64" else "Float64 orbit / Float32 tangent"


def _read() -> dict:
    import tomllib
    try:
        with open(RECORD_PATH, "rb") as f:
            rec = tomllib.load(f)
        return rec if isinstance(rec, dict) else {}
    except (OSError, ValueError):
        return {}


def _write(rec: dict) -> None:
    lines = []
    for dev, per in rec.items():
        for label, entry in per.items():
            if not isinstance(entry, dict):
                continue
            lines.append(f'["{dev}"."{label}"]')
            lines += [f"{k} = {float(v)!r}" for k, v in entry.items() if isinstance(v, (int, float))]
            lines.append("")
    os.makedirs(os.path.dirname(RECORD_PATH), exist_ok=True)
    tmp = RECORD_PATH + f".{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        f.write("\n".join(lines))
    os.replace(tmp, RECORD_PATH)


def record_step_ns(precision: str = "fp64", device: str | None = None) -> float:
    """Measure the one-wave ns per orbit-step on the current device (the standard map's kernel of the precision's
    class: Float64, or Float32 tangent frames) and store it in the record with the device's wave."""
    import ctypes as C

    import numpy as np

    from . import _abi
    from ._lib import last_error, lib
    from .propagate import FrameSpec, build_run, probe
    from .reducers import MGS, QRSpectrum, chain_dtype
    from .systems import StandardMap

    pr = probe()
    device = device or pr["device"]
    wave = int(pr["sm_count"]) * 512 if pr.get("sm_count") else LAUNCH_WAVE
    n, N = wave, 2000
    sysm = StandardMap(2 * math.pi)
    x0 = np.random.default_rng(1).uniform(0, 2 * math.pi, (n, 2))
    W0 = np.ascontiguousarray(np.broadcast_to(np.eye(2), (n, 2, 2)))
    reds = (QRSpectrum(MGS()),)
    run = build_run(sysm, N, 1, [FrameSpec(2, reds)], "fp64" if precision == "fp64" else "mixed", 1)
    x, W = np.empty((n, 2)), np.empty((n, 2, 2))
    st = np.zeros(n, dtype=chain_dtype(reds, 2, 2))
    code, hs = np.zeros(n, dtype=np.int8), np.zeros(n, dtype=np.int64)
    b = _abi.cl_buffers()
    b.x0, b.x = x0.ctypes.data, x.ctypes.data
    b.W0[0], b.W[0], b.states[0], b.code[0], b.hstep[0] = W0.ctypes.data, W.ctypes.data, st.ctypes.data, \
        code.ctypes.data, hs.ctypes.data
    prov = _abi.cl_prov()
    best = math.inf
    for _ in range(3):
        rc = lib().cl_b200_propagate(C.byref(run), n, C.byref(b), C.byref(prov))
        if rc != 0:
            raise RuntimeError(f"record run failed: {rc} {last_error()}")
        best = min(best, prov.gpu_ms)
    ns = best * 1e6 / (n * N)
    with _lock:
        rec = _read()
        rec.setdefault(device, {})[_label(precision)] = {"gpu_ns_per_step_wave": ns, "launch_wave": wave}
        _write(rec)
        _cache[(device, _label(precision))] = (ns, wave)
    return ns


def device_record(precision: str = "fp64", device: str | None = None, measure: bool = True) -> tuple[float, int] | None:
    """(ns per orbit-step for one wave, the wave) of (device, precision) from the record, measured and stored on
    first use when `measure`; None when absent and not measured."""
    if device is None:
        device = _device_name()
    key = (device, _label(precision))
    if key in _cache:
        return _cache[key]
    e = _read().get(device, {}).get(_label(precision), {})
    v, w = e.get("gpu_ns_per_step_wave"), e.get("launch_wave", LAUNCH_WAVE)
    if isinstance(v, (int, float)) and math.isfinite(v) and v > 0 and isinstance(w, (int, float)) and w >= 1:
        _cache[key] = (float(v), int(w))
        return _cache[key]
    if not measure:
        return None
    record_step_ns(precision, device)
    return _cache[key]


def gpu_step_ns(precision: str = "fp64", device: str | None = None, measure: bool = True) -> float | None:
    """`gpu_step_ns(device, T)`: the record's one-wave ns per orbit-step (None without a record when not measuring;
    the plan then uses DEFAULT_GPU_NS)."""
    r = device_record(precision, device, measure)
    return None if r is None else r[0]


_names: dict = {}


def _device_name() -> str:
    from .propagate import probe
    if "current" not in _names:
        _names["current"] = probe()["device"]
    return _names["current"]
