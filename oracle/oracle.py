"""TEST INFRASTRUCTURE: Python binding of the CPU oracle (liboracle.so). Only tests/, __graft_entry__.smoke() and
the cpu_baseline / reference legs of bench.py import this module; the product never does.

`oracle_frames` runs the serial restatement of the reference's per-orbit body on the same cl_run the B200 library
takes and returns the same records (x, W, states, code, hstep per frame).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from chaos_b200 import _abi
from chaos_b200.propagate import FrameSpec, build_run
from chaos_b200.reducers import chain_dtype

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
MATH = {"portable": 0, "libm": 1}
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        dp = P(C.c_double)
        L.oracle_propagate.argtypes = [P(_abi.cl_run), C.c_int64, P(_abi.cl_buffers), C.c_int32, C.c_int32]
        L.oracle_static_supported.argtypes = [P(_abi.cl_run)]
        L.oracle_static_propagate.argtypes = [P(_abi.cl_run), C.c_int64, P(_abi.cl_buffers), C.c_int32]
        L.oracle_propagate.restype = C.c_int
        L.oracle_sincos.argtypes = [C.c_int32, dp, dp, dp, C.c_int64]
        L.oracle_log.argtypes = [C.c_int32, dp, dp, C.c_int64]
        L.oracle_exp.argtypes = [C.c_int32, dp, dp, C.c_int64]
        L.oracle_atan2.argtypes = [C.c_int32, dp, dp, dp, C.c_int64]
        L.oracle_fused_product.argtypes = [dp, dp, dp, C.c_int32, C.c_int32, C.c_int32]
        L.oracle_safe_norm.argtypes = [dp, C.c_int32]
        L.oracle_safe_norm.restype = C.c_double
        ip = P(C.c_int32)
        L.oracle_orthonormalize.argtypes = [C.c_int32, dp, C.c_int32, C.c_int32, dp, dp, ip, ip, ip]
        L.oracle_window_Gw.argtypes = [dp, C.c_int32]
        L.oracle_window_Gw.restype = C.c_double
        L.oracle_orth_loss.argtypes = [dp, C.c_int32, C.c_int32]
        L.oracle_orth_loss.restype = C.c_double
        L.oracle_seeded_frame.argtypes = [C.c_uint64, C.c_int64, C.c_int32, C.c_int32, dp]
        L.oracle_gauss3_step.argtypes = [dp, C.c_double, C.c_int32, C.c_double, dp]
        L.oracle_split_step.argtypes = [dp, C.c_double, C.c_int32, dp, dp, dp]
        L.oracle_record.argtypes = [P(_abi.cl_run), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32]
        L.oracle_advance.argtypes = [P(_abi.cl_system), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                     C.c_int32]
        L.oracle_indicator_window.argtypes = [P(_abi.cl_run), P(_abi.cl_window), C.c_int64, C.c_int32, C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                              C.c_void_p, C.c_int32, C.c_int32]
        L.oracle_state_bytes.argtypes = [P(_abi.cl_run), C.c_int32]
        L.oracle_state_bytes.restype = C.c_int64
        L.oracle_indicator.argtypes = [P(_abi.cl_run), C.c_int32, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                       C.c_void_p, C.c_int32, C.c_int32]
        L.oracle_shadow.argtypes = [P(_abi.cl_run), C.c_int64, dp, C.c_void_p, C.c_void_p, C.c_double, C.c_int32,
                                    C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        L.oracle_max_threads.restype = C.c_int32
        L.oracle_ensemble.argtypes = [P(_abi.cl_run), C.c_int64, P(_abi.cl_buffers), dp, P(C.c_int64), C.c_double,
                                      C.c_int32, C.c_int32]
        L.oracle_ensemble.restype = C.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def sincos(x, math="portable"):
    x = np.ascontiguousarray(x, dtype=np.float64)
    s, c = np.empty_like(x), np.empty_like(x)
    lib().oracle_sincos(MATH[math], _dp(x), _dp(s), _dp(c), x.size)
    return s, c


def log(x, math="portable"):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    lib().oracle_log(MATH[math], _dp(x), _dp(y), x.size)
    return y


def fused_product(A, B):
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    m, p = A.shape
    n = B.shape[1]
    Cm = np.zeros((m, n), order="F")
    lib().oracle_fused_product(_dp(A), _dp(B), _dp(Cm), m, p, n)
    return Cm


def orthonormalize(alg: int, W):
    W = np.asfortranarray(W, dtype=np.float64)
    d, k = W.shape
    Q, R = np.zeros((d, k), order="F"), np.zeros((k, k), order="F")
    cnt, st, col = C.c_int32(), C.c_int32(), C.c_int32()
    lib().oracle_orthonormalize(alg, _dp(W), d, k, _dp(Q), _dp(R), C.byref(cnt), C.byref(st), C.byref(col))
    return Q, R, cnt.value, st.value, col.value


def window_Gw(R):
    R = np.asfortranarray(R, dtype=np.float64)
    return lib().oracle_window_Gw(_dp(R), R.shape[0])


def seeded_frame(seed, orbit, d, k):
    W = np.zeros((d, k), order="F")
    lib().oracle_seeded_frame(seed % (1 << 64), orbit, d, k, _dp(W))
    return W


def gauss3_step(z, h, maxiter=50, tol=float("nan")):
    z = np.ascontiguousarray(z, dtype=np.float64).copy()
    T = np.zeros((4, 4), order="F")
    lib().oracle_gauss3_step(_dp(z), h, maxiter, tol, _dp(T))
    return z, T


def split_step(z, h, method):
    """One step of the table method `method` (a SplittingMethod) on the Henon-Heiles flow: (z', 4 x 4 tangent)."""
    z = np.ascontiguousarray(z, dtype=np.float64).copy()
    T = np.zeros((4, 4), order="F")
    c = np.ascontiguousarray(method.c, dtype=np.float64)
    d = np.ascontiguousarray(method.d, dtype=np.float64)
    lib().oracle_split_step(_dp(z), h, len(c), _dp(c), _dp(d), _dp(T))
    return z, T


def oracle_record(sys, x0, N, tau, estimator, grid, *, W0=None, launch_steps=None, math="portable", threads=0):
    """The recorder on the oracle: dict R (n, n_grid, ncol), fail, x, W (n, d, k), states (raw), code, hstep."""
    from chaos_b200.reducers import Benettin
    x = np.ascontiguousarray(np.asarray(x0, dtype=np.float64)).copy()
    n, s = x.shape
    d = sys.d
    k = 1 if isinstance(estimator, Benettin) else 2
    run = build_run(sys, N, tau, [FrameSpec(k, (estimator,))], "fp64", 0)
    ncol = k + 7 + s
    sb = (48 if k == 1 else 16 * k + 72) + 24
    if W0 is None:
        W0 = np.broadcast_to(np.eye(d)[:, :k], (n, d, k))
    W = np.ascontiguousarray(np.asarray(W0, dtype=np.float64).transpose(0, 2, 1))
    grid = np.ascontiguousarray(np.asarray(grid, dtype=np.int64))
    states = np.zeros((n, sb), np.uint8)
    code = np.zeros(n, np.int8)
    hstep = np.zeros(n, np.int64)
    R = np.zeros((n, len(grid), ncol))
    fail = np.zeros(n, np.int64)
    total, L, done = int(N), int(launch_steps) if launch_steps else int(N), 0
    while done < total:
        run.n0, run.steps = done, min(L, total - done)
        rc = lib().oracle_record(C.byref(run), n, x.ctypes.data, W.ctypes.data, states.ctypes.data, code.ctypes.data,
                                 hstep.ctypes.data, grid.ctypes.data, len(grid), R.ctypes.data, fail.ctypes.data,
                                 MATH[math], threads)
        if rc != 0:
            raise ValueError(f"oracle_record returned {rc}")
        done += run.steps
    return dict(R=R, fail=fail, x=x, W=W.transpose(0, 2, 1), states=states, code=code, hstep=hstep)


def oracle_advance(m, flow, x0, tau, n, threads=0):
    """advance_ensemble on the oracle: (states (len, 4), ok (len,) bool) of `n` steps of size tau of IntegratorMap's
    integrator `m` (a SplittingMethod or Gauss) on the Henon-Heiles flow."""
    from chaos_b200.systems import IntegratorMap
    x0 = np.ascontiguousarray(np.asarray(x0, dtype=np.float64).reshape(-1, 4))
    out = np.empty_like(x0)
    ok = np.zeros(len(x0), np.uint8)
    cs = IntegratorMap(m, flow, tau).to_cl()
    rc = lib().oracle_advance(C.byref(cs), len(x0), x0.ctypes.data, out.ctypes.data, ok.ctypes.data, int(n), threads)
    if rc != 0:
        raise ValueError(f"oracle_advance returned {rc}")
    return out, ok.astype(bool)


def oracle_indicators(sys, x0, N, tau, members, grid, *, ns=2, W0=None, launch_steps=None, math="portable",
                      threads=0):
    """The indicator recorder (tangent kind) on the oracle: dict R (n, n_grid, cols + 3 + ns), fail, x, W (n, d, 2),
    states (raw: the members' states then the monitor's three maxima), code, hstep."""
    from chaos_b200.record import indicator_chain
    x = np.ascontiguousarray(np.asarray(x0, dtype=np.float64)).copy()
    n, s = x.shape
    d = sys.d
    chain = indicator_chain(members)
    run = build_run(sys, N, tau, [FrameSpec(2, chain)], "fp64", 0)
    cols = sum(6 if m == "MEGNO" else 2 for m in members)
    ncol = cols + 3 + ns
    sb = lib().oracle_state_bytes(C.byref(run), 0) + 24
    if W0 is None:
        W0 = np.broadcast_to(np.eye(d)[:, :2], (n, d, 2))
    W = np.ascontiguousarray(np.asarray(W0, dtype=np.float64).transpose(0, 2, 1))
    grid = np.ascontiguousarray(np.asarray(grid, dtype=np.int64))
    states = np.zeros((n, sb), np.uint8)
    code = np.zeros(n, np.int8)
    hstep = np.zeros(n, np.int64)
    R = np.zeros((n, len(grid), ncol))
    fail = np.zeros(n, np.int64)
    total, L, done = int(N), int(launch_steps) if launch_steps else int(N), 0
    while done < total:
        run.n0, run.steps = done, min(L, total - done)
        rc = lib().oracle_indicator(C.byref(run), 0, n, ns, x.ctypes.data, W.ctypes.data, states.ctypes.data,
                                    code.ctypes.data, hstep.ctypes.data, grid.ctypes.data, len(grid), R.ctypes.data,
                                    fail.ctypes.data, MATH[math], threads)
        if rc != 0:
            raise ValueError(f"oracle_indicator returned {rc}")
        done += run.steps
    return dict(R=R, fail=fail, x=x, W=W.transpose(0, 2, 1), states=states, code=code, hstep=hstep)


def oracle_indicator_pairs(sys, z0, W0, N, tau, members, grid, *, ns=2, launch_steps=None, math="portable",
                           threads=0):
    """The indicator recorder's pair kind on the oracle: the stream PairMap(sys) from the pair states z0 (n, 2 s) and
    block frames W0 (n, 2 d, 2); dict R (n, n_grid, cols + 3 + ns), fail, x, W, states, code, hstep."""
    from chaos_b200.record import pair_chain
    x = np.ascontiguousarray(np.asarray(z0, dtype=np.float64)).copy()
    n = len(x)
    d = sys.d
    chain = pair_chain(members)
    run = build_run(sys, N, tau, [FrameSpec(2, chain)], "fp64", 0)
    ncol = sum(6 if m == "MEGNO" else 2 for m in members) + 3 + ns
    sb = lib().oracle_state_bytes(C.byref(run), 0) + 24
    W = np.ascontiguousarray(np.asarray(W0, dtype=np.float64).transpose(0, 2, 1))
    assert W.shape == (n, 2, 2 * d)
    grid = np.ascontiguousarray(np.asarray(grid, dtype=np.int64))
    states = np.zeros((n, sb), np.uint8)
    code = np.zeros(n, np.int8)
    hstep = np.zeros(n, np.int64)
    R = np.zeros((n, len(grid), ncol))
    fail = np.zeros(n, np.int64)
    total, L, done = int(N), int(launch_steps) if launch_steps else int(N), 0
    while done < total:
        run.n0, run.steps = done, min(L, total - done)
        rc = lib().oracle_indicator(C.byref(run), 1, n, ns, x.ctypes.data, W.ctypes.data, states.ctypes.data,
                                    code.ctypes.data, hstep.ctypes.data, grid.ctypes.data, len(grid), R.ctypes.data,
                                    fail.ctypes.data, MATH[math], threads)
        if rc != 0:
            raise ValueError(f"oracle_indicator returned {rc}")
        done += run.steps
    return dict(R=R, fail=fail, x=x, W=W.transpose(0, 2, 1), states=states, code=code, hstep=hstep)


def oracle_indicator_window(sys, x0, N, tau, reader, grid, *, ns=2, launch_steps=None, math="portable", threads=0):
    """The indicator recorder's window kinds on the oracle: dict R (n, n_grid, 3 + ns), fail, x, states (MonState
    then the reader's state), code, hstep, finals (the reader's reducer_final per orbit)."""
    from chaos_b200.window import to_cl
    x = np.ascontiguousarray(np.asarray(x0, dtype=np.float64)).copy()
    n = len(x)
    run = build_run(sys, N, tau, [FrameSpec(1, ())], "fp64", 0)
    win = to_cl(reader)
    sb = 24 + reader.state_bytes()
    grid = np.ascontiguousarray(np.asarray(grid, dtype=np.int64))
    states = np.zeros((n, sb), np.uint8)
    code = np.zeros(n, np.int8)
    hstep = np.zeros(n, np.int64)
    R = np.zeros((n, len(grid), 3 + ns))
    fail = np.zeros(n, np.int64)
    total, L, done = int(N), int(launch_steps) if launch_steps else int(N), 0
    while done < total:
        run.n0, run.steps = done, min(L, total - done)
        rc = lib().oracle_indicator_window(C.byref(run), C.byref(win), n, ns, x.ctypes.data, states.ctypes.data,
                                           code.ctypes.data, hstep.ctypes.data, grid.ctypes.data, len(grid),
                                           R.ctypes.data, fail.ctypes.data, MATH[math], threads)
        if rc != 0:
            raise ValueError(f"oracle_indicator_window returned {rc}")
        done += run.steps
    finals = [reader.final(states[i, 24:].tobytes()) for i in range(n)]
    return dict(R=R, fail=fail, x=x, states=states, code=code, hstep=hstep, finals=finals)


def oracle_shadow(sys, x0, N, *, d0, tau=1, seed=0, U0=None, math="portable", threads=0, launch_steps=None,
                  orbit_base=0, grid=None):
    """The two-trajectory estimator on the oracle: the end records (structured array, ShadowEnd layout); with
    `grid`, (ends, R (n, n_grid, 8 + s), fail) of the recorder's two-trajectory method."""
    from chaos_b200.shadow import end_dtype
    x0 = np.ascontiguousarray(np.asarray(x0, dtype=np.float64))
    n, s = x0.shape
    run = build_run(sys, N, tau, [FrameSpec(1, ())], "fp64", seed, orbit_base=orbit_base)
    ends = np.zeros(n, dtype=end_dtype(s))
    u = None if U0 is None else np.ascontiguousarray(np.asarray(U0, dtype=np.float64))
    g = None if grid is None else np.ascontiguousarray(np.asarray(grid, dtype=np.int64))
    R = None if g is None else np.zeros((n, len(g), 8 + s))
    fail = None if g is None else np.zeros(n, np.int64)
    total, L, done = int(N), int(launch_steps) if launch_steps else int(N), 0
    while done < total:
        run.n0, run.steps = done, min(L, total - done)
        rc = lib().oracle_shadow(C.byref(run), n, _dp(x0), None if u is None else u.ctypes.data, ends.ctypes.data,
                                 float(d0), MATH[math], threads, None if g is None else g.ctypes.data,
                                 0 if g is None else len(g), None if R is None else R.ctypes.data,
                                 None if fail is None else fail.ctypes.data)
        if rc != 0:
            raise ValueError(f"oracle_shadow returned {rc}")
        done += run.steps
    return ends if g is None else (ends, R, fail)


def oracle_frames(sys, x0, N, frames: list[FrameSpec], *, tau=1, seed=0, math="portable", threads=0,
                  launch_steps=None, orbit_base=0, engine="runtime"):
    """Run the oracle; returns a list (per frame) of dicts x (n, s), W (n, d, k), states, code, hstep.
    engine "static": the statically sized drivers of static_leg.cpp (map systems, one K for every frame, portable
    math), bit for bit the runtime-sized oracle's records at the reference CPU algorithm's own speed."""
    x0 = np.ascontiguousarray(np.asarray(x0, dtype=np.float64))
    n, s = x0.shape
    d = sys.d
    run = build_run(sys, N, tau, frames, "fp64", seed, orbit_base=orbit_base)
    x = np.empty((n, s))
    W0s, Ws, sts, codes, hs = [], [], [], [], []
    for fr in frames:
        W0s.append(None if fr.W0 is None else np.ascontiguousarray(np.asarray(fr.W0, dtype=np.float64).transpose(0, 2, 1)))
        Ws.append(np.empty((n, fr.k, d)))
        dt = chain_dtype(tuple(fr.reducers), d, fr.k)
        sts.append(np.zeros(n, dtype=dt) if dt.itemsize else None)
        codes.append(np.zeros(n, dtype=np.int8))
        hs.append(np.zeros(n, dtype=np.int64))
    total = int(N)
    L = int(launch_steps) if launch_steps else total
    done = 0
    while done < total:
        run.n0 = done
        run.steps = min(L, total - done)
        b = _abi.cl_buffers()
        b.x0 = x0.ctypes.data
        b.x = x.ctypes.data
        for f in range(len(frames)):
            b.W0[f] = None if W0s[f] is None else W0s[f].ctypes.data
            b.W[f] = Ws[f].ctypes.data
            b.states[f] = None if sts[f] is None else sts[f].ctypes.data
            b.code[f] = codes[f].ctypes.data
            b.hstep[f] = hs[f].ctypes.data
        if engine == "static":
            if math != "portable" or lib().oracle_static_supported(C.byref(run)) != 0:
                raise ValueError("the static oracle covers map systems with one K per run and portable math")
            rc = lib().oracle_static_propagate(C.byref(run), n, C.byref(b), threads)
        else:
            rc = lib().oracle_propagate(C.byref(run), n, C.byref(b), MATH[math], threads)
        if rc != 0:
            raise ValueError(f"oracle_propagate returned {rc}")
        done += run.steps
    return [dict(x=x, W=Ws[f].transpose(0, 2, 1), states=sts[f], code=codes[f], hstep=hs[f])
            for f in range(len(frames))]


def oracle_ensemble(sys, x0, N, frame: FrameSpec, *, tau, K=None, lengths=None, escape=0.0, seed=0,
                    math="portable", threads=0):
    """One ensemble class on the oracle: per-orbit K and lengths, escape bound (see oracle_capi.cpp)."""
    x0 = np.ascontiguousarray(np.asarray(x0, dtype=np.float64))
    n, s = x0.shape
    d = sys.d
    run = build_run(sys, N, tau, [frame], "fp64", seed)
    x = np.empty((n, s))
    W0 = None if frame.W0 is None else np.ascontiguousarray(np.asarray(frame.W0, dtype=np.float64).transpose(0, 2, 1))
    W = np.empty((n, frame.k, d))
    dt = chain_dtype(tuple(frame.reducers), d, frame.k)
    st = np.zeros(n, dtype=dt) if dt.itemsize else None
    code = np.zeros(n, dtype=np.int8)
    hs = np.zeros(n, dtype=np.int64)
    b = _abi.cl_buffers()
    b.x0, b.x = x0.ctypes.data, x.ctypes.data
    b.W0[0] = None if W0 is None else W0.ctypes.data
    b.W[0] = W.ctypes.data
    b.states[0] = None if st is None else st.ctypes.data
    b.code[0], b.hstep[0] = code.ctypes.data, hs.ctypes.data
    Kc = None if K is None else np.ascontiguousarray(K, dtype=np.float64)
    Nc = None if lengths is None else np.ascontiguousarray(lengths, dtype=np.int64)
    rc = lib().oracle_ensemble(C.byref(run), n, C.byref(b), None if Kc is None else _dp(Kc),
                               None if Nc is None else Nc.ctypes.data_as(C.POINTER(C.c_int64)), float(escape),
                               MATH[math], threads)
    if rc != 0:
        raise ValueError(f"oracle_ensemble returned {rc}")
    return dict(x=x, W=W.transpose(0, 2, 1), states=st, code=code, hstep=hs)
