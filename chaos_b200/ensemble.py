"""Batched uneven ensembles: classes of orbits with per-orbit map parameter K, per-orbit length and an escape stop,
run by persistent kernels from a device work queue (include/chaoslab_b200.h, `cl_b200_ensemble*`).

The reference has one N and one system per `propagate` call and no escape stop; each orbit of an ensemble equals
the reference call `propagate_orbit(sys(K_i), x0_i, W0_i, N_i', tau, reducers)` (src/Tangent/orbit.jl:85-99) with
N_i' its length, or the first handoff at which max_j |p_j| exceeds the escape bound (code 4 then).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._lib import last_error, lib
from .foundation import DeviceError
from .propagate import FrameSpec, _check_frame, build_run
from .reducers import chain_dtype
from .systems import StandardMap, StandardMapChain, System

STATUS_ESCAPED = 4


@dataclass
class EnsembleClass:
    """Orbits of one system kind and dimension: x0 (n, s), one frame, per-orbit K / lengths (optional)."""
    sys: System
    x0: np.ndarray
    frame: FrameSpec
    tau: int
    N: int
    K: np.ndarray | None = None
    lengths: np.ndarray | None = None
    escape: float = 0.0
    precision: str = "fp64"
    seed: int = 0
    minb: int = 0
    unroll: int = 0
    lanes: int = 0       # lanes per orbit: 1, or the lattice's site count (cooperative kernel); 0 = tuned/default


@dataclass
class EnsembleResult:
    x: np.ndarray
    W: np.ndarray
    states: np.ndarray | None
    code: np.ndarray
    hstep: np.ndarray
    gpu_ms: float = 0.0


def queue_order(lengths: np.ndarray) -> np.ndarray:
    """Longest orbit first (a stable argsort of -N): the persistent kernels take orbits in this order, 32 per warp."""
    return np.argsort(-np.asarray(lengths, dtype=np.int64), kind="stable").astype(np.int64)


def _check(c: EnsembleClass) -> None:
    _check_frame(c.sys, c.frame)
    if c.lengths is not None:
        L = np.asarray(c.lengths)
        if L.shape != (len(c.x0),):
            raise ValueError("one length per orbit")
        if np.any(L < c.tau) or np.any(L % c.tau) or np.any(L > c.N):
            raise ValueError("lengths must be positive multiples of tau, at most N")


def make_class_struct(c: EnsembleClass, keep: list) -> _abi.cl_ensemble_class:
    _check(c)
    x0 = np.ascontiguousarray(np.asarray(c.x0, dtype=np.float64))
    n = len(x0)
    d, k = c.sys.d, c.frame.k
    run = build_run(c.sys, c.N, c.tau, [c.frame], c.precision, c.seed)
    cs = _abi.cl_ensemble_class()
    cs.run = run
    cs.n_orbits = n
    cs.escape = float(c.escape)
    cs.minb, cs.unroll, cs.lanes = c.minb, c.unroll, c.lanes
    W0 = None if c.frame.W0 is None else np.ascontiguousarray(np.asarray(c.frame.W0, dtype=np.float64).transpose(0, 2, 1))
    lengths = None if c.lengths is None else np.ascontiguousarray(c.lengths, dtype=np.int64)
    order = queue_order(lengths if lengths is not None else np.full(n, c.N))
    K = None if c.K is None else np.ascontiguousarray(c.K, dtype=np.float64)
    out = dict(x=np.empty((n, c.sys.s)), W=np.empty((n, k, d)), code=np.zeros(n, np.int8), hstep=np.zeros(n, np.int64))
    dt = chain_dtype(tuple(c.frame.reducers), d, k)
    out["states"] = np.zeros(n, dtype=dt) if dt.itemsize else None
    keep += [x0, W0, lengths, order, K, out]
    cs.order = order.ctypes.data
    cs.K = None if K is None else K.ctypes.data
    cs.N = None if lengths is None else lengths.ctypes.data
    cs.buf.x0 = x0.ctypes.data
    cs.buf.x = out["x"].ctypes.data
    cs.buf.W0[0] = None if W0 is None else W0.ctypes.data
    cs.buf.W[0] = out["W"].ctypes.data
    cs.buf.states[0] = None if out["states"] is None else out["states"].ctypes.data
    cs.buf.code[0] = out["code"].ctypes.data
    cs.buf.hstep[0] = out["hstep"].ctypes.data
    return cs


def propagate_ensemble(classes: list[EnsembleClass]) -> list[EnsembleResult]:
    """Run every class (host buffers: copies in, concurrent persistent launches, copies out)."""
    keep: list = []
    arr = (_abi.cl_ensemble_class * len(classes))(*[make_class_struct(c, keep) for c in classes])
    prov = _abi.cl_prov()
    rc = lib().cl_b200_ensemble(arr, len(classes), C.byref(prov))
    if rc != 0:
        msg = last_error()
        if rc == _abi.EINVAL:
            raise ValueError(msg)
        raise DeviceError(rc, msg)
    res = []
    for j in range(len(classes)):
        out = keep[6 * j + 5]
        res.append(EnsembleResult(x=out["x"], W=out["W"].transpose(0, 2, 1), states=out["states"], code=out["code"],
                                  hstep=out["hstep"], gpu_ms=prov.gpu_ms))
    return res


def lattice_workload(n_total: int, seed: int = 1, n_max: int = 10 ** 6, n_min: int = 10 ** 3,
                     dims=(2, 4, 8, 16), taus=(5, 10, 10, 20), eps: float = 0.05, escape: float = 1e3,
                     precision: str = "mixed"):
    """The uneven lattice ensemble: n_total orbits in equal shares of d in `dims` (d = 2 the standard map, else a
    chain of d/2 coupled standard maps with coupling eps), K uniform in [0.5, 3], coordinates uniform in [0, 2 pi),
    lengths log-uniform in [n_min, n_max] rounded down to a multiple of the class's tau, k = min(d, 8),
    QRSpectrum(HouseholderQR) from W0 = I[:, 1:k], escape at |p| > `escape`."""
    from .reducers import HouseholderQR, QRSpectrum
    rng = np.random.default_rng(seed)
    per = n_total // len(dims)
    classes = []
    for d, tau in zip(dims, taus):
        k = min(d, 8)
        sysm = StandardMap(1.0) if d == 2 else StandardMapChain(d // 2, 1.0, eps)
        x0 = rng.uniform(0, 2 * math.pi, (per, d))
        K = rng.uniform(0.5, 3.0, per)
        L = np.exp(rng.uniform(math.log(n_min), math.log(n_max), per))
        L = np.maximum(tau, (L // tau).astype(np.int64) * tau)
        Nmax = int(n_max // tau * tau)
        W0 = np.broadcast_to(np.eye(d)[:, :k], (per, d, k)).copy()
        classes.append(EnsembleClass(sysm, x0, FrameSpec(k, (QRSpectrum(HouseholderQR()),), W0), tau, Nmax, K=K,
                                     lengths=L, escape=escape, precision=precision, seed=seed))
    return classes


class DeviceClass:
    """One class's buffers resident on a CUDA device (torch tensors) and its `cl_ensemble_class` pointing at them,
    for `cl_b200_ensemble_device`, `cl_b200_ensemble_tune` and the graph entry points. x and W come back
    orbit-major (W as k columns of d, the C side's layout)."""

    def __init__(self, c: EnsembleClass, torch, device):
        keep: list = []
        self.c = c
        self.cls = make_class_struct(c, keep)
        n, s, d, k = len(c.x0), c.sys.s, c.sys.d, c.frame.k
        t = torch
        W0 = keep[1]
        if W0 is None:
            raise ValueError("a device class needs an explicit W0")
        sb = keep[5]["states"].dtype.itemsize if keep[5]["states"] is not None else 0
        self.t = dict(x0=t.tensor(keep[0], device=device), x=t.empty((n, s), dtype=t.float64, device=device),
                      W0=t.tensor(W0, device=device), W=t.empty((n, d * k), dtype=t.float64, device=device),
                      st=t.zeros(max(1, n * sb // 8), dtype=t.int64, device=device),
                      code=t.zeros(n, dtype=t.int8, device=device), hs=t.zeros(n, dtype=t.int64, device=device),
                      order=t.tensor(keep[3], device=device))
        if keep[4] is not None:
            self.t["K"] = t.tensor(keep[4], device=device)
        if keep[2] is not None:
            self.t["N"] = t.tensor(keep[2], device=device)
        self.state_dtype = keep[5]["states"].dtype if sb else None
        b = self.cls.buf
        b.x0, b.x = self.t["x0"].data_ptr(), self.t["x"].data_ptr()
        b.W0[0], b.W[0] = self.t["W0"].data_ptr(), self.t["W"].data_ptr()
        b.states[0] = self.t["st"].data_ptr() if sb else None
        b.code[0], b.hstep[0] = self.t["code"].data_ptr(), self.t["hs"].data_ptr()
        self.cls.order = self.t["order"].data_ptr()
        self.cls.K = self.t["K"].data_ptr() if "K" in self.t else None
        self.cls.N = self.t["N"].data_ptr() if "N" in self.t else None
        self.orbit_steps = int(np.sum(c.lengths)) if c.lengths is not None else len(c.x0) * int(c.N)

    def states(self) -> np.ndarray | None:
        if self.state_dtype is None:
            return None
        return self.t["st"].cpu().numpy().view(self.state_dtype)[: len(self.c.x0)]


def device_classes_array(dcs: list[DeviceClass]):
    return (_abi.cl_ensemble_class * len(dcs))(*[dc.cls for dc in dcs])
