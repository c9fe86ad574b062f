"""The learned screen: classify orbits as chaotic or regular from their first 2000 steps, and integrate in full only
the orbits the network is unsure about (plus a random audit). No reference counterpart: the reference classifies
by full integration only (its screening loop, src/Experiments/screening.jl:26-52, runs every orbit to the end).

The map is the 4D coupled standard map (FroeschleMap), one k = 2 frame with the chain (MEGNO(replace = false),
SALI()) and tau = 10, on the Float64 kernels by default (`precision="fp64"`: the training labels, the full
integrations of the unsure and audited orbits and the plain full run that the screen is judged against all come
from the reference's Float64 arithmetic; `precision="mixed"` runs the same pipeline on the mixed kernels). The
training set is the coupled-maps ensemble: coordinates uniform in [0, 2 pi)^4. Features: every 100 steps up to 2000, the column-1 log-stretch
rate, log10 SALI and the running MEGNO Y (cl_b200_screen_features reads them off the reducer states between
relaunch windows, which carry the state bit for bit). Label: the final mean MEGNO Ybar of column 1 > 2.2 at
N = 1e5; regression target: the final lambda_1 estimate. The orbits kept for full integration continue from their
2000-step state, so the screen never redoes work.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._lib import last_error, lib
from .mlp import MLP, _declare
from .propagate import FrameSpec, build_run
from .reducers import MEGNO, SALI
from .systems import FroeschleMap

TAU = 10
WINDOW = 100
FEATURE_STEPS = 2000
N_FULL = 100_000
STATE_WORDS = 34        # MEGNOState (200 B) + SALIState (72 B)
THRESHOLD = 2.2         # final MEGNO above which an orbit is labelled chaotic


def _ck(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: {rc} {last_error()}")


@dataclass
class Carried:
    """Device buffers of a batch of orbits between relaunches (orbit-major)."""
    x0: object
    x: object
    W0: object
    W: object
    st: object
    code: object
    hstep: object
    n: int


class Screen:
    def __init__(self, torch, device, sysm=None, precision: str = "fp64", seed: int = 1):
        self.t, self.dev = torch, device
        self.sys = sysm or FroeschleMap(1.5, 1.5, 0.05)
        self.precision = precision
        self.seed = seed
        self.frame = FrameSpec(2, (MEGNO(replace=False), SALI()))
        self.L = _declare(lib())

    def stream(self):
        return self.t.cuda.current_stream(self.dev).cuda_stream

    def buffers(self, x0_np) -> Carried:
        t, d = self.t, self.dev
        n = len(x0_np)
        x0 = t.tensor(np.ascontiguousarray(x0_np, dtype=np.float64), device=d)
        W0 = t.zeros((n, 8), dtype=t.float64, device=d)
        W0[:, 0] = 1.0
        W0[:, 5] = 1.0
        return Carried(x0=x0, x=t.empty_like(x0), W0=W0, W=t.empty_like(W0),
                       st=t.zeros(n * STATE_WORDS, dtype=t.float64, device=d),
                       code=t.zeros(n, dtype=t.int8, device=d), hstep=t.zeros(n, dtype=t.int64, device=d), n=n)

    def _launch(self, b: Carried, n0: int, steps: int, N: int):
        run = build_run(self.sys, N, TAU, [self.frame], self.precision, self.seed, n0=n0, steps=steps)
        cb = _abi.cl_buffers()
        cb.x0, cb.x = b.x0.data_ptr(), b.x.data_ptr()
        cb.W0[0], cb.W[0] = b.W0.data_ptr(), b.W.data_ptr()
        cb.states[0], cb.code[0], cb.hstep[0] = b.st.data_ptr(), b.code.data_ptr(), b.hstep.data_ptr()
        _ck(self.L.cl_b200_propagate_device(C.byref(run), b.n, C.byref(cb), 0, C.c_void_p(self.stream())), "propagate")

    def features(self, b: Carried, N: int = N_FULL):
        """Run the first FEATURE_STEPS steps in windows, filling the (n, 64) features (BF16 and FP32)."""
        t = self.t
        fb = t.zeros((b.n, 64), dtype=t.bfloat16, device=self.dev)
        f32 = t.zeros((b.n, 64), dtype=t.float32, device=self.dev)
        windows = FEATURE_STEPS // WINDOW
        for w in range(windows):
            self._launch(b, w * WINDOW, WINDOW, N)
            _ck(self.L.cl_b200_screen_features(b.st.data_ptr(), b.n, (w + 1) * WINDOW, w, windows, f32.data_ptr(),
                                               fb.data_ptr(), self.stream()), "features")
        return fb, f32

    def finish(self, b: Carried, N: int = N_FULL):
        """Continue carried orbits from FEATURE_STEPS to N; returns (label, lambda_1, code) on the host."""
        if b.n:
            self._launch(b, FEATURE_STEPS, N - FEATURE_STEPS, N)
        st = b.st.view(-1, STATE_WORDS).cpu().numpy()
        K = st[:, 22].view(np.int64)
        Ybar = np.where(K > 0, (st[:, 6] + st[:, 7]) / np.maximum(K, 1), 0.0)
        nn = st[:, 21].view(np.int64)
        lam = np.where(nn > 0, (st[:, 0] + st[:, 1]) / np.maximum(nn, 1), 0.0)
        return (Ybar > THRESHOLD).astype(np.float32), lam, b.code.cpu().numpy()

    def subset(self, b: Carried, idx) -> Carried:
        t = self.t
        ii = t.tensor(np.asarray(idx, dtype=np.int64), device=self.dev)
        return Carried(x0=b.x0.index_select(0, ii), x=b.x.index_select(0, ii), W0=b.W0.index_select(0, ii),
                       W=b.W.index_select(0, ii), st=b.st.view(-1, STATE_WORDS).index_select(0, ii).reshape(-1),
                       code=b.code.index_select(0, ii), hstep=b.hstep.index_select(0, ii), n=len(idx))

    # ---- the pipeline -----------------------------------------------------------------------------------------------
    def training_set(self, n: int, N: int = N_FULL, seed: int = 11, plane: bool = False):
        """n labelled orbits of the coupled-maps ensemble: all four coordinates uniform in [0, 2 pi) (~97 % chaotic:
        the coupling's mu (1 - cos) term leaves few regular orbits in the full torus), or, with plane = True,
        (x1, p1) uniform on [0, 2 pi)^2 with x2 = p2 = 0.1 (the plane the grid screens; ~85 % chaotic). Returns the
        BF16 features of the orbits that finished without a failure, their labels and their final lambda_1."""
        rng = np.random.default_rng(seed)
        if plane:
            x0 = np.stack([rng.uniform(0, 2 * math.pi, n), np.full(n, 0.1), rng.uniform(0, 2 * math.pi, n),
                           np.full(n, 0.1)], axis=1)
        else:
            x0 = rng.uniform(0, 2 * math.pi, (n, 4))
        b = self.buffers(x0)
        fb, f32 = self.features(b, N)
        label, lam, code = self.finish(b, N)
        ok = code == 0
        return fb[self.t.tensor(np.flatnonzero(ok), device=self.dev)], label[ok], lam[ok].astype(np.float32)

    def train(self, X, label, lam, epochs=8, batch=4096, lr=2e-3, w_reg=1.0, seed=0, val_frac=0.1,
              balance: float = 0.1):
        """Train the network on (features, label, lambda_1). `balance` in (0, 1): every epoch draws its rows with
        replacement so that a row is regular with that probability (the coupled-maps ensemble is ~98 % chaotic;
        0.5 weighs both classes equally); 0 keeps the natural mix. The default 0.1 was chosen on a 1024^2 grid of the
        screened plane at the configured band (0.05, 0.95) and 5 % audit: 0 left 16.8 % of the grid unsure (4.5x
        fewer orbit-steps), 0.5 misclassified 1.16 %, 0.1 gave 8.97x at 0.63 %."""
        t = self.t
        n = X.shape[0]
        rng = np.random.default_rng(seed)
        perm = rng.permutation(n)
        nv = int(n * val_frac) // 128 * 128
        vi, ti = perm[:nv], perm[nv:]
        net = MLP(t, self.dev, seed=seed)
        lt = t.tensor(label, device=self.dev)
        tt = t.tensor(lam, device=self.dev)
        hist = []
        if balance and len(ti):
            pos = label[ti] > 0.5
            fp = max(pos.mean(), 1e-12)
            w = np.where(pos, (1.0 - balance) / fp, balance / max(1.0 - fp, 1e-12))
            w = w / w.sum()
        for ep in range(epochs):
            order = rng.choice(ti, size=len(ti), replace=True, p=w) if balance and len(ti) else rng.permutation(ti)
            for lo in range(0, len(order) - batch + 1, batch):
                idx = t.tensor(order[lo:lo + batch], device=self.dev)
                rl = net.train_step(X.index_select(0, idx), lt.index_select(0, idx), tt.index_select(0, idx),
                                    w_reg=w_reg, lr=lr)
            hist.append(float(rl.mean().item()))
        out = net.predict(X.index_select(0, t.tensor(vi, device=self.dev))).cpu().numpy()
        acc = float(((out[:, 0] > 0) == (label[vi] > 0.5)).mean()) if nv else float("nan")
        return net, dict(loss=hist, val_accuracy=acc, n_train=len(ti), n_val=nv)

    def screen_grid(self, net, G: int, N: int = N_FULL, lo=0.05, hi=0.95, audit=0.05, seed=3):
        """Classify a G x G grid of (x1, p1) starts in [0, 2 pi)^2 with x2 = p2 = 0.1: features for all, full
        integration for the uncertain ones (lo < P < hi) and a random audit fraction of the rest."""
        t = self.t
        g = (np.arange(G) + 0.5) * (2 * math.pi / G)
        x1, p1 = np.meshgrid(g, g, indexing="ij")
        x0 = np.stack([x1.ravel(), np.full(G * G, 0.1), p1.ravel(), np.full(G * G, 0.1)], axis=1)
        t.cuda.synchronize(self.dev)
        t0 = time.perf_counter()
        b = self.buffers(x0)
        fb, _ = self.features(b, N)
        out = net.predict(fb)
        z = out[:, 0].cpu().numpy()
        P = 1.0 / (1.0 + np.exp(-z.astype(np.float64)))
        unsure = np.flatnonzero((P > lo) & (P < hi))
        sure = np.flatnonzero(~((P > lo) & (P < hi)))
        rng = np.random.default_rng(seed)
        aud = np.sort(rng.choice(sure, size=int(round(audit * len(sure))), replace=False)) if len(sure) else sure
        full_idx = np.union1d(unsure, aud)
        sub = self.subset(b, full_idx)
        lab_full, lam_full, code_full = self.finish(sub, N)
        t.cuda.synchronize(self.dev)
        t_screen = time.perf_counter() - t0
        pred = (P > 0.5).astype(np.float32)
        final = pred.copy()
        final[full_idx] = lab_full
        pos = {int(k): i for i, k in enumerate(full_idx)}
        aud_lab = np.array([lab_full[pos[int(k)]] for k in aud], dtype=np.float32)
        mis = float((pred[aud] != aud_lab).mean()) if len(aud) else float("nan")
        steps_screen = len(x0) * FEATURE_STEPS + len(full_idx) * (N - FEATURE_STEPS)
        return dict(n=len(x0), labels=final, P=P, unsure=len(unsure), audited=len(aud), audit_misclassification=mis,
                    seconds=t_screen, orbit_steps=steps_screen, full_orbit_steps=len(x0) * N)

    def full_grid(self, G: int, N: int = N_FULL):
        """The plain method: every grid orbit integrated to N; returns the labels and the time."""
        t = self.t
        g = (np.arange(G) + 0.5) * (2 * math.pi / G)
        x1, p1 = np.meshgrid(g, g, indexing="ij")
        x0 = np.stack([x1.ravel(), np.full(G * G, 0.1), p1.ravel(), np.full(G * G, 0.1)], axis=1)
        t.cuda.synchronize(self.dev)
        t0 = time.perf_counter()
        b = self.buffers(x0)
        self._launch(b, 0, N, N)
        st = b.st.view(-1, STATE_WORDS).cpu().numpy()
        t.cuda.synchronize(self.dev)
        dt = time.perf_counter() - t0
        K = st[:, 22].view(np.int64)
        Ybar = np.where(K > 0, (st[:, 6] + st[:, 7]) / np.maximum(K, 1), 0.0)
        return (Ybar > THRESHOLD).astype(np.float32), dt
