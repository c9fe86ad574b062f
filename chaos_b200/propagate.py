"""`propagate` on the B200: the host side of the drop-in boundary.

Mirrors `propagate(sys, x0, N; k, tau, seed, reducers, backend, chunk, W0)` of src/Tangent/propagate.jl:267-290
and its record `PropagationResult` (:20-26): the same argument checks and ArgumentErrors (ValueError here), the
same chunking rule (`chunk_size`, :10-18), the same per-orbit failure handling (the lowest failing orbit id throws
its `NumericalHealthError`, :111-113) and the same host-side `reducer_final` summaries (:116-118), with the device
chunk running in libchaoslab_b200 through its C ABI. There is no CPU path in this package: the reference keeps its
own CPU backend; a device failure is raised as `DeviceError` with the reference's fallback reason index.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import platform
from dataclasses import dataclass, field

import numpy as np

from . import _abi, launch_plan
from ._lib import last_error, lib
from .foundation import DeviceError, NumericalHealthError
from .reducers import GALI, SALI, Finals, Reducer, chain_dtype
from .systems import System

STATUS_OK, STATUS_STATE, STATUS_W, STATUS_REDUCER = 0, 1, 2, 3
CHUNK_HEADROOM = 0.5
PRECISIONS = {"fp64": _abi.PREC_FP64, "mixed": _abi.PREC_MIXED, "mixed-ind64": _abi.PREC_MIXED_IND64}
PRECISION_LABELS = {"fp64": "Float64", "mixed": "Float64 orbit / Float32 tangent",
                    "mixed-ind64": "Float64 orbit and indicator frames / Float32 Lyapunov frames"}


@dataclass
class FrameSpec:
    """One tangent frame of a run: k deviation vectors, its reducer chain, optional initial frames (n, d, k)."""
    k: int
    reducers: tuple = ()
    W0: np.ndarray | None = None


@dataclass
class PropagationResult:
    """`PropagationResult(x, W, finals, provenance)` (propagate.jl:20-26) plus the raw device records."""
    x: np.ndarray                # (n, s)
    W: np.ndarray                # (n, d, k)
    finals: list | None          # per orbit, a tuple of reducer_final dicts (None when not requested)
    provenance: dict
    states: np.ndarray | None = None   # structured array in the Julia isbits layout
    code: np.ndarray | None = None
    hstep: np.ndarray | None = None
    reducers: tuple = field(default=())

    def spectrum_residuals(self, system=None, *, tol: float = 16.0, M_max=None) -> dict:
        """The residual records of a QRSpectrum frame with k = d (src/Diagnostics/residuals.jl:13-32): per orbit
        eps_sum, eps_pair and their threshold sum_threshold(tol, T, G_max, tau, M_max), T the frame's element type
        (Float32 for a mixed-precision frame), M_max from `system.tangent_bound()` unless given."""
        from .diagnostics import spectrum_residuals
        T = "Float32" if self.provenance.get("precision", "Float64") != "Float64" else "Float64"
        return spectrum_residuals(self, tau=int(self.provenance["tau"]), tol=tol, M_max=M_max, T=T, system=system)


def bytes_per_orbit(d: int, k: int, s: int | None = None) -> int:
    """sizeof(T)(s + d k + 2k) + 16 (propagate.jl:1-6)."""
    s = d if s is None else s
    return 8 * (s + d * k + 2 * k) + 16


def chunk_size(free_bytes: int, d: int, k: int, f: float = CHUNK_HEADROOM, reducer_bytes: int = 0,
               s: int | None = None) -> int:
    """floor(f free / (bytes_per_orbit + reducer_bytes)), at least 1 (propagate.jl:10-18)."""
    return max(1, math.floor(f * free_bytes / (bytes_per_orbit(d, k, s) + reducer_bytes)))


def _check_steps(N: int, tau: int) -> None:
    if not (tau >= 1 and N >= 1 and N % tau == 0):
        raise ValueError(f"N must be a positive multiple of tau, got N = {N}, tau = {tau}")


def _check_frame(sys: System, fr: FrameSpec) -> None:
    d = sys.d
    if not 1 <= fr.k <= d:
        raise ValueError(f"k must be in 1:{d}, got {fr.k}")
    rs = tuple(fr.reducers)
    for i, r in enumerate(rs):
        if not isinstance(r, Reducer):
            raise TypeError(f"{r!r} is not a reducer of the compiled menu")
        if isinstance(r, SALI) and i > 0 and isinstance(rs[i - 1], GALI):
            continue   # SALI of the GALI frame's columns 1-2
        r.check(d, fr.k)


def build_run(sys: System, N: int, tau: int, frames: list[FrameSpec], precision: str = "fp64", seed: int = 0,
              n0: int = 0, steps: int = 0, orbit_base: int = 0) -> _abi.cl_run:
    run = _abi.cl_run()
    run.abi_version = _abi.ABI_VERSION
    run.d, run.s, run.tau = sys.d, sys.s, int(tau)
    run.N, run.n0, run.steps = int(N), int(n0), int(steps)
    run.n_frames = len(frames)
    run.precision = PRECISIONS[precision]
    run.seed = int(seed) % (1 << 64)
    run.orbit_base = int(orbit_base)
    run.sys = sys.to_cl()
    for f, fr in enumerate(frames):
        run.frames[f].k = fr.k
        run.frames[f].n_reducers = len(fr.reducers)
        for i, r in enumerate(fr.reducers):
            run.frames[f].reducers[i] = r.to_cl()
    return run


def _first_bad(v: np.ndarray) -> float:
    flat = np.asarray(v, dtype=np.float64).ravel(order="F")
    bad = np.flatnonzero(~np.isfinite(flat))
    return float(flat[bad[0]])


def _health_error(code, x, W, step, orbit, backend):   # orbit.jl:63-68
    if code == STATUS_STATE:
        return NumericalHealthError("state", _first_bad(x), math.inf, step, orbit, backend)
    return NumericalHealthError("deviation matrix", _first_bad(W), math.inf, step, orbit, backend)


def _reducer_error(reducers, st, orbit, backend):   # orbit.jl:34-37: the first failed reducer of the chain
    for i, r in enumerate(reducers):
        sub = st[f"r{i}"]
        if isinstance(r, GALI) and i + 1 < len(reducers) and isinstance(reducers[i + 1], SALI):
            pass
        if r.failed(sub):
            return r.error(sub, orbit, backend)
    raise AssertionError("STATUS_REDUCER without a failed reducer")


def probe() -> dict:
    """`Foundation.probe` record of the device (loadable, functional, device, compiles) plus memory."""
    p = _abi.cl_probe()
    rc = lib().cl_b200_probe(C.byref(p))
    return dict(loadable=bool(p.loadable), functional=bool(p.functional), compiles=bool(p.compiles) and rc == 0,
                device=p.device.decode(), sm=p.sm, sm_count=p.sm_count, free_bytes=p.free_bytes,
                total_bytes=p.total_bytes)


def release_cache() -> None:
    """Return the device memory the library's pools keep between host-buffer calls to the driver
    (`cl_b200_release_cache`, the counterpart of CUDA.jl's `CUDA.reclaim()`)."""
    rc = lib().cl_b200_release_cache()
    if rc != 0:
        raise DeviceError(rc, last_error())


def _ptr(a):
    return None if a is None else a.ctypes.data


def propagate_frames(sys: System, x0, N: int, frames: list[FrameSpec], *, tau: int = 1, seed: int = 0,
                     precision: str = "fp64", chunk: int | None = None, launch_steps: int | None = None,
                     finals: bool = True, throw: bool = True) -> list[PropagationResult]:
    """Integrate every orbit of x0 once and carry each frame of `frames` along it; frame f's result is the
    reference's `propagate(sys, x0, N; k = frames[f].k, tau, seed, reducers = frames[f].reducers,
    W0 = frames[f].W0)`."""
    x0 = np.ascontiguousarray(np.asarray(x0, dtype=np.float64))
    if x0.ndim != 2:
        raise ValueError("x0 must be an (n, s) array")
    n, s = x0.shape
    N, tau = int(N), int(tau)
    _check_steps(N, tau)
    d = sys.d
    if s < d:
        raise ValueError(f"state length {s} is below the system dimension {d}")
    if s != sys.s:
        raise ValueError(f"state length {s} does not match {sys.name} (s = {sys.s})")
    if chunk is not None and chunk < 1:
        raise ValueError(f"chunk must be positive, got {chunk}")
    if not 1 <= len(frames) <= _abi.MAX_FRAMES:
        raise ValueError("one to three frames")
    if launch_steps is not None and (launch_steps < 1 or launch_steps % tau):
        raise ValueError(f"forced steps per launch must be a positive multiple of tau, got L = {launch_steps}, tau = {tau}")
    W0s = []
    for f, fr in enumerate(frames):
        _check_frame(sys, fr)
        if fr.W0 is not None:
            W0 = np.asarray(fr.W0, dtype=np.float64)
            if W0.shape[0] != n:
                raise ValueError("W0 needs one matrix per orbit")
            if W0.shape[1:] != (d, fr.k):
                raise ValueError(f"W0 matrices must be {d} x {fr.k}")
            same = [g for g in range(f) if frames[g].W0 is fr.W0]   # one frame's W0 given again: one copy
            W0s.append(W0s[same[0]] if same else np.ascontiguousarray(W0.transpose(0, 2, 1)))   # column-major per orbit
        else:
            W0s.append(None)
    run = build_run(sys, N, tau, frames, precision, seed)
    L = lib()
    rc = L.cl_b200_check(C.byref(run))
    if rc != 0:
        msg = last_error()
        if rc == _abi.EINVAL:
            raise ValueError(msg)
        raise DeviceError(rc, msg)
    # the launch plan (propagate.jl:183-190): steps per launch within the budget for one wave, and the orbit cap
    forced = launch_steps if launch_steps is not None else launch_plan.forced_launch(tau)
    ns, wave = launch_plan.device_record(precision)
    Lsteps, cap = launch_plan.device_plan(forced, N, tau, ns, wave)
    if Lsteps == 0:
        raise DeviceError(-8, f"a launch of tau = {tau} steps exceeds the launch budget for one wave")
    run.steps = Lsteps
    dtypes = [chain_dtype(fr.reducers, d, fr.k) for fr in frames]
    rbytes = sum(dt.itemsize for dt in dtypes)
    if chunk is None:
        pr = probe()
        kk = max(fr.k for fr in frames)
        csize = chunk_size(pr["free_bytes"], d, kk, reducer_bytes=rbytes, s=s) if pr["free_bytes"] else n
    else:
        csize = chunk
    csize = min(csize, cap, n) if n else 1
    x = np.empty((n, s))
    Wout = [np.empty((n, fr.k, d)) for fr in frames]
    states = [np.zeros(n, dtype=dt) if dt.itemsize else None for dt in dtypes]
    codes = [np.zeros(n, dtype=np.int8) for _ in frames]
    hsteps = [np.zeros(n, dtype=np.int64) for _ in frames]
    prov_dev = _abi.cl_prov()
    gpu_ms, chunks = 0.0, 0
    errors: list = [None] * len(frames)
    for lo in range(0, n, csize):
        hi = min(lo + csize, n)
        run.orbit_base = lo
        bufs = _abi.cl_buffers()
        bufs.x0 = x0[lo:hi].ctypes.data
        bufs.x = x[lo:hi].ctypes.data
        for f in range(len(frames)):
            bufs.W0[f] = None if W0s[f] is None else W0s[f][lo:hi].ctypes.data
            bufs.W[f] = Wout[f][lo:hi].ctypes.data
            bufs.states[f] = None if states[f] is None else states[f][lo:hi].ctypes.data
            bufs.code[f] = codes[f][lo:hi].ctypes.data
            bufs.hstep[f] = hsteps[f][lo:hi].ctypes.data
        hook = launch_plan.BEFORE_LAUNCH
        if hook is None:   # every launch of the chunk inside one library call
            rc = L.cl_b200_propagate(C.byref(run), hi - lo, C.byref(bufs), C.byref(prov_dev))
            if rc != 0:
                raise DeviceError(rc, last_error())
            gpu_ms += prov_dev.gpu_ms
        else:   # launch by launch, the hook before each with the live carried device buffers (propagate.jl:101-104)
            w, launch = _hooked_chunk(L, run, hi - lo, bufs, frames, d, s, N, Lsteps, hook, prov_dev, chunks + 1)
            prov_dev.launch_steps, prov_dev.launches = Lsteps, launch
            gpu_ms += w
        chunks += 1
        for f, fr in enumerate(frames):   # lowest failing orbit id first (propagate.jl:111-113)
            if errors[f] is not None:
                continue
            bad = np.flatnonzero(codes[f][lo:hi] != STATUS_OK)
            if bad.size:
                i = lo + int(bad[0])
                c = int(codes[f][i])
                if c == STATUS_REDUCER:
                    errors[f] = _reducer_error(tuple(fr.reducers), states[f][i], i + 1, "gpu")
                else:
                    errors[f] = _health_error(c, x[i], Wout[f][i].T, int(hsteps[f][i]), i + 1, "gpu")
    if throw:
        for e in errors:
            if e is not None:
                raise e
    results = []
    # the frames' vectorised finals, on host threads when there are several frames of many orbits (numpy releases
    # the interpreter lock in the column arithmetic)
    fins: list = [None] * len(frames)
    todo = [f for f, fr in enumerate(frames) if finals and states[f] is not None]
    if len(todo) > 1 and n >= 8192:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=len(todo)) as ex:
            futs = {f: ex.submit(Finals, tuple(frames[f].reducers), states[f], d) for f in todo}
            for f, fu in futs.items():
                fins[f] = fu.result()
    else:
        for f in todo:
            fins[f] = Finals(tuple(frames[f].reducers), states[f], d)
    for f, fr in enumerate(frames):
        prov = dict(backend="gpu", device=prov_dev.device.decode(), backend_fallback_reason="",
                    precision=PRECISION_LABELS[precision],
                    threads=os.cpu_count(), cpu=platform.processor() or platform.machine(), seed=seed, tau=tau,
                    k=fr.k, chunk_size=csize, headroom=CHUNK_HEADROOM, gpu_chunks=chunks, gpu_chunk_size=csize,
                    launch_steps=int(prov_dev.launch_steps), launches_per_chunk=int(prov_dev.launches),
                    kernel=prov_dev.variant.decode(), gpu_ms=gpu_ms, registers=int(prov_dev.regs))
        for r in fr.reducers:
            prov.update(r.provenance())
        W = Wout[f].transpose(0, 2, 1)
        fin = fins[f]
        if finals and states[f] is None:
            fin = [() for _ in range(n)]
        results.append(PropagationResult(x=x, W=W, finals=fin, provenance=prov, states=states[f], code=codes[f],
                                         hstep=hsteps[f], reducers=tuple(fr.reducers)))
    return results



def _hooked_chunk(L, run, n, hbufs, frames, d, s, N, Lsteps, hook, prov_dev, chunk_index):
    """One chunk launch by launch on device buffers: the host inputs are staged once, `hook(device, chunk, launch,
    carried)` runs before every launch with the live device buffers (torch tensors: x, W, states as bytes), each
    launch is one window [n0, n0 + L) of `cl_b200_propagate_device`, and the outputs are copied back into the host
    buffers at the end. Returns (device milliseconds, launches)."""
    import torch

    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)

    def up(ptr, nbytes):
        buf = torch.empty(nbytes, dtype=torch.uint8)
        C.memmove(buf.data_ptr(), ptr, nbytes)
        return buf.to(dev)

    tx0 = up(hbufs.x0, 8 * n * s)
    tx = torch.empty_like(tx0)
    dbufs = _abi.cl_buffers()
    dbufs.x0, dbufs.x = tx0.data_ptr(), tx.data_ptr()
    keep, tW, tst = [tx0, tx], [], []
    for f, fr in enumerate(frames):
        wb = 8 * n * fr.k * d
        W0 = up(hbufs.W0[f], wb) if hbufs.W0[f] else None
        W = torch.empty(wb, dtype=torch.uint8, device=dev)
        sb = _abi.frame_state_bytes(run.frames[f]) * n if hbufs.states[f] else 0
        st = torch.zeros(max(sb, 1), dtype=torch.uint8, device=dev)
        code = torch.zeros(n, dtype=torch.int8, device=dev)
        hs = torch.zeros(n, dtype=torch.int64, device=dev)
        dbufs.W0[f] = None if W0 is None else W0.data_ptr()
        dbufs.W[f], dbufs.code[f], dbufs.hstep[f] = W.data_ptr(), code.data_ptr(), hs.data_ptr()
        dbufs.states[f] = st.data_ptr() if sb else None
        keep += [W0, W, st, code, hs]
        tW.append(W.view(torch.float64).view(n, fr.k, d))
        tst.append(st if sb else None)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launch, n0, ms = 0, 0, 0.0
    while n0 < N:
        launch += 1
        hook(prov_dev.device.decode() or "B200", chunk_index, launch,
             dict(x=tx.view(torch.float64).view(n, s), W=tW, states=tst, workspace=None))
        run.n0, run.steps = n0, min(Lsteps, N - n0)
        e0.record(stream)
        rc = L.cl_b200_propagate_device(C.byref(run), n, C.byref(dbufs), 0, C.c_void_p(stream.cuda_stream))
        e1.record(stream)
        if rc != 0:
            raise DeviceError(rc, last_error())
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        n0 += run.steps
    run.n0, run.steps = 0, Lsteps
    torch.cuda.synchronize(dev)

    def down(t, ptr, nbytes):
        hb = t.reshape(-1).view(torch.uint8)[:nbytes].cpu()
        C.memmove(ptr, hb.data_ptr(), nbytes)

    down(tx, hbufs.x, 8 * n * s)
    for f, fr in enumerate(frames):
        down(tW[f], hbufs.W[f], 8 * n * fr.k * d)
        if tst[f] is not None:
            down(tst[f], hbufs.states[f], tst[f].numel())
        down(keep[2 + 5 * f + 3], hbufs.code[f], n)
        down(keep[2 + 5 * f + 4], hbufs.hstep[f], 8 * n)
    return ms, launch

def propagate(sys: System, x0, N: int, *, k: int, tau: int = 1, seed: int = 0, reducers=(), backend: str = "gpu",
              chunk: int | None = None, W0=None, precision: str = "fp64", launch_steps: int | None = None,
              finals: bool = True) -> PropagationResult:
    """propagate(sys, x0, N; k, tau=1, seed, reducers=(), backend=:gpu, chunk=nothing, W0=nothing) on the B200
    (src/Tangent/propagate.jl:267-290). `x0` is (n, s); `W0` (n, d, k) or None for the seeded frames;
    `precision` is "fp64" (the reference's arithmetic) or "mixed" (Float32 tangent frames)."""
    if backend not in ("gpu", "auto"):
        raise ValueError("backend must be :gpu or :auto here; the CPU path is the reference's own")
    return propagate_frames(sys, x0, N, [FrameSpec(int(k), tuple(reducers), W0)], tau=tau, seed=seed,
                            precision=precision, chunk=chunk, launch_steps=launch_steps, finals=finals)[0]


def propagate_orbit(sys: System, x0, W0, N: int, tau: int, reducers, *, orbit: int = 1, precision: str = "fp64"):
    """propagate_orbit(sys, x0, W0, N, tau, reducers; orbit = 1) -> (x, W, states), src/Tangent/orbit.jl:77-99: one
    orbit from `x0` (length s) with the deviation matrix `W0` (d x k) through the same kernel, the reducer states in
    the Julia layout; a reducer failure raises that reducer's NumericalHealthError and a non-finite state or frame
    at a handoff the health error, each naming `orbit`."""
    x0 = np.asarray(x0, dtype=np.float64).reshape(1, -1)
    W0 = np.asarray(W0, dtype=np.float64)
    if W0.ndim != 2:
        raise ValueError("W0 must be a d x k matrix")
    _check_steps(int(N), int(tau))
    fr = FrameSpec(W0.shape[1], tuple(reducers), W0[None])
    r = propagate_frames(sys, x0, N, [fr], tau=tau, precision=precision, finals=False, throw=False)[0]
    code = int(r.code[0])
    if code == STATUS_REDUCER:
        raise _reducer_error(tuple(reducers), r.states[0], int(orbit), "gpu")
    if code != STATUS_OK:
        raise _health_error(code, r.x[0], r.W[0], int(r.hstep[0]), int(orbit), "gpu")
    return r.x[0], r.W[0], (r.states[0] if r.states is not None else None)
