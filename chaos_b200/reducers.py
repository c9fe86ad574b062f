"""Reducers of the fixed menu (src/Lyapunov, src/Indicators) with their host-side protocol.

The device runs `reducer_step` for every handoff (fused into the orbit kernel) and hands back each state in the
isbits layout of the Julia struct (T = Float64). Here each reducer knows that layout as a numpy structured dtype
and runs the host half of the reducer protocol (src/Tangent/Tangent.jl:21-111) on it: `final` (`reducer_final`),
`failed` (`reducer_failed`), `error` (`reducer_error`) and `provenance` (`reducer_provenance`), with the same
arithmetic as the reference.
"""
from __future__ import annotations

import math

import numpy as np

from . import _abi
from .foundation import EPS, NumericalHealthError


def _cs(name):
    return [(name + "_s", "<f8"), (name + "_c", "<f8")]


def _tot(s, c):
    return float(np.float64(s) + np.float64(c))


class Orthonormalizer:
    code: int
    name: str
    gs_family = False

    def __repr__(self):
        return type(self).__name__ + "()"

    def __eq__(self, other):
        return type(self) is type(other)

    def __hash__(self):
        return hash(type(self).__name__)


class CGS(Orthonormalizer):
    code, name, gs_family = _abi.QR_CGS, "CGS", True


class MGS(Orthonormalizer):
    code, name, gs_family = _abi.QR_MGS, "MGS", True


class RGS(Orthonormalizer):
    code, name, gs_family = _abi.QR_RGS, "RGS", True


class HouseholderQR(Orthonormalizer):
    code, name = _abi.QR_HOUSEHOLDER, "V-H"


class AugmentedQR(Orthonormalizer):
    code, name = _abi.QR_AUGMENTED, "V-A"


class GivensQR(Orthonormalizer):
    code, name = _abi.QR_GIVENS, "V-G"


class Reducer:
    kind: int
    replaces = True

    def to_cl(self) -> _abi.cl_reducer:
        return _abi.cl_reducer(kind=self.kind)

    def dtype(self, d: int, k: int) -> np.dtype:
        raise NotImplementedError

    def check(self, d: int, k: int) -> None:
        """`reducer_init` argument checks (ArgumentError in the reference)."""

    def failed(self, st) -> bool:
        return int(st["code"]) != 0

    def finals(self, st, d=None) -> dict | None:
        """Columns of `final` over every orbit at once (arrays with the orbit as the first axis), the same values as
        `final` per orbit; None where only the per-orbit form exists."""
        return None

    def provenance(self) -> dict:
        return {}

    def __repr__(self):
        return type(self).__name__ + "()"


class QRSpectrum(Reducer):
    """QRSpectrum(alg; orthogonality_tol=8.0), src/Lyapunov/qr_spectrum.jl:14-96."""
    kind = _abi.RED_QR

    def __init__(self, alg: Orthonormalizer, orthogonality_tol: float = 8.0):
        self.alg, self.orthogonality_tol = alg, float(orthogonality_tol)

    def __repr__(self):
        return f"QRSpectrum({self.alg!r})"

    def to_cl(self):
        return _abi.cl_reducer(kind=self.kind, alg=self.alg.code, orthogonality_tol=self.orthogonality_tol)

    def dtype(self, d, k):   # QRState{Float64,K}, qr_spectrum.jl:22-33
        return np.dtype([("sums", "<f8", (k, 2)), ("n", "<i8"), ("G_max", "<f8"), ("orth_max", "<f8"),
                         ("count_max", "<i8"), ("code", "i1"), ("_p0", "V7"), ("column", "<i8"),
                         ("value", "<f8"), ("threshold", "<f8"), ("step", "<i8")])

    def final(self, st):   # qr_spectrum.jl:85-91
        k = st["sums"].shape[0]
        n = int(st["n"])
        s = st["sums"][:, 0].astype(np.float64)
        c = st["sums"][:, 1].astype(np.float64)
        lam = np.array([0.0 if n == 0 else _tot(s[i], c[i]) / n for i in range(k)])
        return dict(n=n, sum=s.copy(), comp=c.copy(), **{"lambda": lam}, G_max=float(st["G_max"]),
                    orth_max=float(st["orth_max"]), count_max=int(st["count_max"]))

    def finals(self, st, d=None):
        n = st["n"].astype(np.int64, copy=False)
        s = st["sums"][:, :, 0].astype(np.float64, copy=False)
        c = st["sums"][:, :, 1].astype(np.float64, copy=False)
        with np.errstate(invalid="ignore", divide="ignore"):
            lam = np.where(n[:, None] == 0, 0.0, (s + c) / n[:, None].astype(np.float64, copy=False))
        return dict(n=n, sum=s, comp=c, **{"lambda": lam}, G_max=st["G_max"].astype(np.float64, copy=False),
                    orth_max=st["orth_max"].astype(np.float64, copy=False), count_max=st["count_max"].astype(np.int64, copy=False))

    def error(self, st, orbit, backend):   # qr_spectrum.jl:80-83
        kind = "orthogonality" if int(st["code"]) == 4 else "orthonormalisation breakdown"
        return NumericalHealthError(kind, float(st["value"]), float(st["threshold"]), int(st["step"]), orbit,
                                    backend, int(st["column"]))

    def provenance(self):
        return dict(estimator="qr", orthonormalizer=self.alg.name, orthogonality_tol=self.orthogonality_tol)


class Benettin(Reducer):
    """Benettin(), src/Lyapunov/benettin.jl:11-53 (k = 1)."""
    kind = _abi.RED_BENETTIN

    def check(self, d, k):
        if k != 1:
            raise ValueError(f"Benettin needs k = 1, got k = {k}")

    def dtype(self, d, k):
        return np.dtype(_cs("sum") + [("n", "<i8"), ("code", "i1"), ("_p0", "V7"), ("value", "<f8"),
                                      ("step", "<i8")])

    def final(self, st):
        n = int(st["n"])
        lam = 0.0 if n == 0 else _tot(st["sum_s"], st["sum_c"]) / n
        return dict(n=n, sum=np.array([st["sum_s"]]), comp=np.array([st["sum_c"]]), **{"lambda": np.array([lam])})

    def finals(self, st, d=None):
        n = st["n"].astype(np.int64, copy=False)
        s, c = st["sum_s"].astype(np.float64, copy=False), st["sum_c"].astype(np.float64, copy=False)
        with np.errstate(invalid="ignore", divide="ignore"):
            lam = np.where(n == 0, 0.0, (s + c) / n.astype(np.float64, copy=False))
        return dict(n=n, sum=s[:, None], comp=c[:, None], **{"lambda": lam[:, None]})

    def error(self, st, orbit, backend):
        v = float(st["value"])
        return NumericalHealthError("deviation matrix", v, 0.0 if math.isfinite(v) else math.inf, int(st["step"]),
                                    orbit, backend, 1)

    def provenance(self):
        return dict(estimator="benettin")


class SALI(Reducer):
    """SALI(), src/Indicators/sali.jl:14-68 (k = 2)."""
    kind = _abi.RED_SALI

    def check(self, d, k):
        if k != 2:
            raise ValueError(f"SALI needs k = 2, got k = {k}")

    def dtype(self, d, k):
        return np.dtype(_cs("s1") + _cs("s2") + [("sali", "<f8"), ("value", "<f8"), ("n", "<i8"), ("step", "<i8"),
                                                 ("code", "i1"), ("column", "i1"), ("_p0", "V6")])

    def final(self, st):   # sali.jl:55-59
        s = np.array([st["s1_s"], st["s2_s"]], dtype=np.float64)
        c = np.array([st["s1_c"], st["s2_c"]], dtype=np.float64)
        n = int(st["n"])
        L = 0.0 if n == 0 else -((s[0] + s[1]) + (c[0] + c[1]))
        return dict(n=n, sali=float(st["sali"]), L=float(L), sum=s, comp=c, floor=4 * EPS)

    def finals(self, st, d=None):
        n = st["n"].astype(np.int64, copy=False)
        s = np.stack([st["s1_s"], st["s2_s"]], axis=1).astype(np.float64, copy=False)
        c = np.stack([st["s1_c"], st["s2_c"]], axis=1).astype(np.float64, copy=False)
        L = np.where(n == 0, 0.0, -((s[:, 0] + s[:, 1]) + (c[:, 0] + c[:, 1])))
        return dict(n=n, sali=st["sali"].astype(np.float64, copy=False), L=L, sum=s, comp=c, floor=np.full(len(n), 4 * EPS))

    def error(self, st, orbit, backend):
        v = float(st["value"])
        return NumericalHealthError("deviation matrix", v, 0.0 if math.isfinite(v) else math.inf, int(st["step"]),
                                    orbit, backend, int(st["column"]))

    def provenance(self):
        return dict(indicator="sali")


class GALI(Reducer):
    """GALI(), src/Indicators/gali.jl:17-201 (2 <= k <= d)."""
    kind = _abi.RED_GALI

    def check(self, d, k):
        if not 2 <= k <= d:
            raise ValueError("GALI needs 2 <= k <= d")

    def dtype(self, d, k):   # GALIState{Float64, D, K, K-1}
        return np.dtype([("s", "<f8", (k,)), ("c", "<f8", (k,)), ("gali", "<f8", (k - 1,)), ("value", "<f8"),
                         ("n", "<i8"), ("step", "<i8"), ("code", "i1"), ("_p0", "V7"), ("column", "<i8")])

    def final(self, st, d=None):   # gali.jl:186-199
        k = st["s"].shape[0]
        n = int(st["n"])
        L = None
        if d is not None and k == d:
            if n == 0:
                L = 0.0
            else:
                s, c = np.float64(st["s"][0]), np.float64(st["c"][0])
                for i in range(1, k):
                    s = s + np.float64(st["s"][i])
                    c = c + np.float64(st["c"][i])
                L = float(-(s + c))
        floors = np.array([2 * (i + 1) * EPS for i in range(1, k)])
        return dict(n=n, gali=st["gali"].astype(np.float64).copy(), L=L, sum=st["s"].astype(np.float64).copy(),
                    comp=st["c"].astype(np.float64).copy(), floor=floors)

    def finals(self, st, d=None):
        k = st["s"].shape[1]
        n = st["n"].astype(np.int64, copy=False)
        S = st["s"].astype(np.float64, copy=False)
        Cc = st["c"].astype(np.float64, copy=False)
        L = None
        if d is not None and k == d:
            s, c = S[:, 0].copy(), Cc[:, 0].copy()
            for i in range(1, k):   # left folds, as _log_form (gali.jl:186-193)
                s = s + S[:, i]
                c = c + Cc[:, i]
            L = np.where(n == 0, 0.0, -(s + c))
        floors = np.broadcast_to(np.array([2 * (i + 1) * EPS for i in range(1, k)]), (len(n), k - 1))
        return dict(n=n, gali=st["gali"].astype(np.float64, copy=False), L=L, sum=S, comp=Cc, floor=floors)

    def error(self, st, orbit, backend):
        v = float(st["value"])
        thr = math.inf if not math.isfinite(v) else (0.0 if v == 0 else float(np.finfo(np.float64).tiny))
        return NumericalHealthError("deviation matrix", v, thr, int(st["step"]), orbit, backend, int(st["column"]))

    def provenance(self):
        return dict(indicator="gali")


_MEGNO_SUMS = ["s", "R1", "R2", "Q", "Q2"]


class MEGNO(Reducer):
    """MEGNO(; replace=True), src/Indicators/megno.jl:29-113 (k = 2)."""
    kind = _abi.RED_MEGNO

    def __init__(self, replace: bool = True):
        self.replace = bool(replace)
        self.replaces = self.replace

    def __repr__(self):
        return f"MEGNO(replace={self.replace})"

    def to_cl(self):
        return _abi.cl_reducer(kind=self.kind, replace=int(self.replace))

    def check(self, d, k):
        if k != 2:
            raise ValueError(f"MEGNO needs k = 2, got k = {k}")

    def dtype(self, d, k):
        f = []
        for col in ("c1", "c2"):
            for nm in _MEGNO_SUMS:
                f += _cs(f"{col}_{nm}")
        return np.dtype(f + [("value", "<f8"), ("n", "<i8"), ("K", "<i8"), ("step", "<i8"), ("code", "i1"),
                             ("column", "i1"), ("_p0", "V6")])

    @staticmethod
    def series(st, col, n, K):   # megno.jl:97-102
        if K == 0:
            return 0.0, 0.0, 0.0
        f = np.float64
        tn = f(n)
        R1 = f(st[f"{col}_R1_s"]) + f(st[f"{col}_R1_c"])
        Q = f(st[f"{col}_Q_s"]) + f(st[f"{col}_Q_c"])
        Q2 = f(st[f"{col}_Q2_s"]) + f(st[f"{col}_Q2_c"])
        return float(2 * R1 / tn), float(Q / f(K)), float(f(n // K) * Q2 / (tn * tn * tn))

    def final(self, st):   # megno.jl:104-111
        n, K = int(st["n"]), int(st["K"])
        y1, b1, e1 = self.series(st, "c1", n, K)
        y2, b2, e2 = self.series(st, "c2", n, K)
        pair = lambda nm, comp: np.array([st[f"c1_{nm}_{comp}"], st[f"c2_{nm}_{comp}"]], dtype=np.float64)  # noqa
        tot = lambda nm: np.array([_tot(st[f"c1_{nm}_s"], st[f"c1_{nm}_c"]), _tot(st[f"c2_{nm}_s"], st[f"c2_{nm}_c"])])  # noqa
        return dict(n=n, handoffs=K, Y=np.array([y1, y2]), Ybar=np.array([b1, b2]), Ybar20=np.array([e1, e2]),
                    sum=pair("s", "s"), comp=pair("s", "c"), R1=tot("R1"), R2=tot("R2"), Q=tot("Q"), Q2=tot("Q2"))

    def finals(self, st, d=None):
        n, K = st["n"].astype(np.int64, copy=False), st["K"].astype(np.int64, copy=False)
        f = np.float64
        tn = n.astype(f, copy=False)
        cols = {nm: np.zeros((len(n), 2)) for nm in ("Y", "Ybar", "Ybar20")}
        with np.errstate(invalid="ignore", divide="ignore"):
            nk = np.where(K == 0, 0, n // np.where(K == 0, 1, K)).astype(f, copy=False)
            for j, col in enumerate(("c1", "c2")):
                R1 = st[f"{col}_R1_s"].astype(f, copy=False) + st[f"{col}_R1_c"].astype(f, copy=False)
                Q = st[f"{col}_Q_s"].astype(f, copy=False) + st[f"{col}_Q_c"].astype(f, copy=False)
                Q2 = st[f"{col}_Q2_s"].astype(f, copy=False) + st[f"{col}_Q2_c"].astype(f, copy=False)
                cols["Y"][:, j] = np.where(K == 0, 0.0, 2 * R1 / tn)
                cols["Ybar"][:, j] = np.where(K == 0, 0.0, Q / K.astype(f, copy=False))
                cols["Ybar20"][:, j] = np.where(K == 0, 0.0, nk * Q2 / (tn * tn * tn))
        pair = lambda nm, comp: np.stack([st[f"c1_{nm}_{comp}"], st[f"c2_{nm}_{comp}"]], axis=1).astype(f, copy=False)  # noqa
        tot = lambda nm: np.stack([st[f"c1_{nm}_s"].astype(f, copy=False) + st[f"c1_{nm}_c"].astype(f, copy=False),  # noqa
                                   st[f"c2_{nm}_s"].astype(f, copy=False) + st[f"c2_{nm}_c"].astype(f, copy=False)], axis=1)
        return dict(n=n, handoffs=K, Y=cols["Y"], Ybar=cols["Ybar"], Ybar20=cols["Ybar20"], sum=pair("s", "s"),
                    comp=pair("s", "c"), R1=tot("R1"), R2=tot("R2"), Q=tot("Q"), Q2=tot("Q2"))

    def error(self, st, orbit, backend):
        v = float(st["value"])
        return NumericalHealthError("deviation matrix", v, 0.0 if math.isfinite(v) else math.inf, int(st["step"]),
                                    orbit, backend, int(st["column"]))

    def provenance(self):
        return dict(indicator="megno", convention="weights at the end of the window, mean over the handoffs 1..K")


class FLI(Reducer):
    """FLI(; replace=True), src/Indicators/fli.jl:26-96 (k = 2)."""
    kind = _abi.RED_FLI

    def __init__(self, replace: bool = True):
        self.replace = bool(replace)
        self.replaces = self.replace

    def __repr__(self):
        return f"FLI(replace={self.replace})"

    def to_cl(self):
        return _abi.cl_reducer(kind=self.kind, replace=int(self.replace))

    def check(self, d, k):
        if k != 2:
            raise ValueError(f"FLI needs k = 2, got k = {k}")

    def dtype(self, d, k):
        return np.dtype(_cs("s1") + _cs("s2") + [("f1", "<f8"), ("fB", "<f8"), ("value", "<f8"), ("n", "<i8"),
                                                 ("step", "<i8"), ("step1", "<i8"), ("stepB", "<i8"), ("code", "i1"),
                                                 ("column", "i1"), ("colB", "i1"), ("_p0", "V5")])

    def final(self, st):   # fli.jl:91-94
        return dict(n=int(st["n"]), fli=float(st["fB"]), fli1=float(st["f1"]),
                    sum=np.array([st["s1_s"], st["s2_s"]], dtype=np.float64),
                    comp=np.array([st["s1_c"], st["s2_c"]], dtype=np.float64),
                    stepB=int(st["stepB"]), colB=int(st["colB"]), step1=int(st["step1"]))

    def finals(self, st, d=None):
        return dict(n=st["n"].astype(np.int64, copy=False), fli=st["fB"].astype(np.float64, copy=False), fli1=st["f1"].astype(np.float64, copy=False),
                    sum=np.stack([st["s1_s"], st["s2_s"]], axis=1).astype(np.float64, copy=False),
                    comp=np.stack([st["s1_c"], st["s2_c"]], axis=1).astype(np.float64, copy=False),
                    stepB=st["stepB"].astype(np.int64, copy=False), colB=st["colB"].astype(np.int64, copy=False),
                    step1=st["step1"].astype(np.int64, copy=False))

    def error(self, st, orbit, backend):
        v = float(st["value"])
        return NumericalHealthError("deviation matrix", v, 0.0 if math.isfinite(v) else math.inf, int(st["step"]),
                                    orbit, backend, int(st["column"]))

    def provenance(self):
        return dict(indicator="fli")


class RLI(Reducer):
    """RLI(; replace=True), src/Indicators/rli.jl:24-114 (k = 2, on a pair stream of even dimension)."""
    kind = _abi.RED_RLI

    def __init__(self, replace: bool = True):
        self.replace = bool(replace)
        self.replaces = self.replace

    def __repr__(self):
        return f"RLI(replace={self.replace})"

    def to_cl(self):
        return _abi.cl_reducer(kind=self.kind, replace=int(self.replace))

    def check(self, d, k):
        if k != 2:
            raise ValueError(f"RLI needs k = 2, got k = {k}")
        if d % 2:
            raise ValueError(f"RLI needs an even dimension, got d = {d}")

    def dtype(self, d, k):
        return np.dtype(_cs("sA") + _cs("sB") + _cs("Q") + [("value", "<f8"), ("n", "<i8"), ("K", "<i8"),
                                                            ("step", "<i8"), ("code", "i1"), ("column", "i1"),
                                                            ("_p0", "V6")])

    def final(self, st):   # rli.jl:98-101
        n, K = int(st["n"]), int(st["K"])
        f = np.float64
        if K == 0:
            dl = rli = 0.0
        else:
            dl = float(abs((f(st["sB_s"]) - f(st["sA_s"])) + (f(st["sB_c"]) - f(st["sA_c"]))) / f(n))
            rli = float((f(st["Q_s"]) + f(st["Q_c"])) / f(K))
        return dict(n=n, handoffs=K, DL=dl, RLI=rli, sum=np.array([st["sA_s"], st["sB_s"]], dtype=np.float64),
                    comp=np.array([st["sA_c"], st["sB_c"]], dtype=np.float64), Q=_tot(st["Q_s"], st["Q_c"]))

    def error(self, st, orbit, backend):   # rli.jl:92-96
        v = float(st["value"])
        what = "pairing" if int(st["code"]) == 2 else "deviation matrix"
        return NumericalHealthError(what, v, 0.0 if math.isfinite(v) else math.inf, int(st["step"]), orbit, backend,
                                    int(st["column"]))

    def provenance(self):
        return dict(indicator="rli", convention="same xi_0, shadow along xi_0, mean over the handoffs 1..K")


def chain_dtype(reducers, d: int, k: int) -> np.dtype:
    """The isbits layout of the Julia tuple of the chain's states (each field 8-byte aligned, sizes multiples of 8)."""
    fields, off = [], 0
    names, formats, offsets = [], [], []
    for i, r in enumerate(reducers):
        dt = r.dtype(d, k)
        assert dt.itemsize == _abi.state_bytes(r.kind, k), (r, dt.itemsize)
        names.append(f"r{i}")
        formats.append(dt)
        offsets.append(off)
        off += dt.itemsize
    del fields
    if not reducers:
        return np.dtype([])
    return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": off})


class Finals:
    """`finals` of a result: one tuple of `reducer_final` records per orbit (src/Tangent/propagate.jl:116-118),
    computed for every orbit at once from the state columns (the same Float64 arithmetic as `final`, vectorised) and
    handed out per orbit on access: `finals[i]` is the tuple of dicts `final` gives for orbit i."""

    def __init__(self, reducers, states, d: int):
        self.reducers = tuple(reducers)
        self.n = 0 if states is None else len(states)
        self.d = d
        self._states = states
        self.columns = [r.finals(states[f"r{i}"], d) if isinstance(r, GALI) else r.finals(states[f"r{i}"])
                        for i, r in enumerate(self.reducers)]

    def __len__(self):
        return self.n

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[j] for j in range(*i.indices(self.n))]
        if i < 0:
            i += self.n
        if not 0 <= i < self.n:
            raise IndexError(i)
        out = []
        for j, (r, cols) in enumerate(zip(self.reducers, self.columns)):
            if cols is None:
                st = self._states[f"r{j}"][i]
                out.append(r.final(st, self.d) if isinstance(r, GALI) else r.final(st))
                continue
            rec = {}
            for key, v in cols.items():
                if v is None:
                    rec[key] = None
                elif v.ndim == 1:
                    rec[key] = int(v[i]) if v.dtype.kind in "iu" else float(v[i])
                else:
                    rec[key] = np.array(v[i])
            out.append(rec)
        return tuple(out)

    def __iter__(self):
        for i in range(self.n):
            yield self[i]
