"""The run store: one HDF5 file per chunk of a study (src/Experiments/run_store.jl:1-240 with
run_indicator_store.jl:1-120; layout version 2: root attributes, `/orbits/<id>/` groups, `/provenance/<member>/`,
`/pooled/<id>/`), written through this package's own HDF5 writer (chaos_b200/h5.py).

`write_chunk(path, attrs, orbits)` follows run_store.jl:138-186: the file is written under `path + ".tmp"` with
`complete = false`, read back and compared bit for bit (orbit data, pooled counts, provenance, root attributes), its
`complete` attribute set to true in place and read back, the file flushed to the disk, a file already holding the
final name moved to `<path>.old<k>`, and the temporary file renamed (retried while another process holds it).
`read_chunk`, `read_chunk_attrs`, `chunk_layout` and `pooled_of` mirror the reference's readers (run_store.jl:192-240,
run_indicator_store.jl:41-100).

Axis order (the layout's rule): an array of Julia shape (n, k) is stored with file extents (k, n); the records here
hold the Julia shapes (`state` (n, 2), `lyap[m]` (n, k), `series` (n, c), `final` (rows, columns), `counts`
(bins + 2, 2)) and the store transposes on write and read.

`orbit_records(rec, items, ...)` turns the device recorder's result (chaos_b200.record.record) into the orbit records
of a chunk as run_device.jl:127-140 and run_record.jl:186-238 do: rows before the failing grid row, NaN from it on,
the thresholds from the last good row's G_max and M_max, the first exceedance step of every diagnostic.
"""
from __future__ import annotations

import errno
import os
import time
from collections import namedtuple
from dataclasses import dataclass, field

import numpy as np

from . import h5
from .diagnostics import effective_eps, sum_threshold

SCHEMA_VERSION = 2
RETRY_CODES = (errno.EBUSY, errno.EACCES, errno.EPERM)
RETRY_TRIES = 12
RETRY_PAUSE = 0.1

Chunk = namedtuple("Chunk", "attrs orbits pooled")


@dataclass
class IndicatorTable:
    """The stored tables of one indicator spec of one orbit (run_indicator_store.jl:13-27); `pool` is in memory only
    (the counts pooled over the chunk)."""
    series: np.ndarray | None = None
    columns: list = field(default_factory=list)
    final: np.ndarray | None = None
    rows: list = field(default_factory=list)
    fcolumns: list = field(default_factory=list)
    flags: np.ndarray | None = None
    bits: list = field(default_factory=list)
    scalars: np.ndarray | None = None
    scolumns: list = field(default_factory=list)
    range: np.ndarray | None = None
    counts: np.ndarray | None = None
    pool: np.ndarray | None = None


@dataclass
class OrbitRecord:
    """One orbit of a chunk (run_record.jl:6-19)."""
    id: int
    attrs: dict
    t: np.ndarray
    state: np.ndarray
    winding: np.ndarray | None
    lyap: dict
    diagnostics: dict
    thresholds: dict
    first_exceedance: dict
    cost: dict
    failure: str = ""
    indicators: dict = field(default_factory=dict)


def diagnostic_names(method: str) -> list[str]:
    """run_record.jl:56-61: none for L2; det and symp for L1; no orth for L9; else det, symp, orth, sum, pair."""
    if method == "L2":
        return []
    if method == "L1":
        return ["det", "symp"]
    if method == "L9":
        return ["det", "symp", "sum", "pair"]
    return ["det", "symp", "orth", "sum", "pair"]


# ---------------------------------------------------------------- equality (bit for bit, as the reference's _same)
def _bits(a):
    a = np.asarray(a)
    return a.view(np.uint64) if a.dtype == np.float64 else a


def _same_array(a, b) -> bool:
    if a is None or b is None:
        return a is None and b is None
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(_bits(a), _bits(b))


def _isequal(a, b) -> bool:
    """Julia's isequal over the attribute values: NaN equals NaN, -0.0 differs from 0.0, arrays element-wise."""
    if a is None or b is None:
        return a is None and b is None
    if isinstance(a, (bool, np.bool_)) or isinstance(b, (bool, np.bool_)):
        return isinstance(a, (bool, np.bool_)) and isinstance(b, (bool, np.bool_)) and bool(a) == bool(b)
    if isinstance(a, str) or isinstance(b, str):
        return a == b
    if isinstance(a, (list, tuple)) and all(isinstance(s, str) for s in a) and isinstance(b, (list, tuple)) and \
            all(isinstance(s, str) for s in b):
        return list(a) == list(b)
    if isinstance(a, dict) or isinstance(b, dict):
        return isinstance(a, dict) and isinstance(b, dict) and a.keys() == b.keys() and \
            all(_isequal(a[k], b[k]) for k in a)
    x, y = np.asarray(a), np.asarray(b)
    if x.dtype.kind == "f" or y.dtype.kind == "f":
        x, y = x.astype(np.float64), y.astype(np.float64)
    elif x.dtype.kind in "iu" and y.dtype.kind in "iu":
        return x.shape == y.shape and np.array_equal(x, y)
    return x.shape == y.shape and x.dtype == y.dtype and np.array_equal(_bits(x), _bits(y))


def _same_indicators(a: dict, b: dict) -> bool:
    if a.keys() != b.keys():
        return False
    for k in a:
        for f in ("series", "final", "flags", "scalars", "range", "counts"):
            if not _same_array(getattr(a[k], f), getattr(b[k], f)):
                return False
        for f in ("columns", "rows", "fcolumns", "bits", "scolumns"):
            if list(getattr(a[k], f)) != list(getattr(b[k], f)):
                return False
    return True


def same_orbit(a: OrbitRecord, b: OrbitRecord) -> bool:
    """run_store.jl:106-113: every stored field of two orbit records equal bit for bit."""
    return (a.id == b.id and _isequal(a.attrs, b.attrs) and _same_array(a.t, b.t) and _same_array(a.state, b.state)
            and _same_array(a.winding, b.winding) and a.lyap.keys() == b.lyap.keys()
            and all(_same_array(a.lyap[m], b.lyap[m]) for m in a.lyap)
            and _same_indicators(a.indicators, b.indicators) and a.diagnostics.keys() == b.diagnostics.keys()
            and all(_same_array(a.diagnostics[m], b.diagnostics[m])
                    and _isequal(float(a.thresholds[m]), float(b.thresholds[m]))
                    and int(a.first_exceedance[m]) == int(b.first_exceedance[m]) for m in a.diagnostics)
            and a.cost.keys() == b.cost.keys() and all(_same_array(a.cost[m], b.cost[m]) for m in a.cost))


# ---------------------------------------------------------------- the tree of a chunk
def _file(a, dtype=None) -> np.ndarray:
    """A Julia-shaped array in file order (dimensions reversed): the transpose, C-contiguous."""
    a = np.asarray(a) if dtype is None else np.asarray(a, dtype=dtype)
    return np.ascontiguousarray(a.T)


def _julia(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a).T)


def _put_orbit(root: h5.Group, o: OrbitRecord) -> None:
    """run_store.jl:87-100 and run_indicator_store.jl:15-27."""
    g = root.require(f"orbits/{int(o.id)}")
    g.attrs.update(o.attrs)
    g.put("t", h5.Dataset(_file(o.t, np.int64)))
    g.put("state", h5.Dataset(_file(o.state, np.float64)))
    if o.winding is not None:
        g.put("winding", h5.Dataset(_file(o.winding, np.int64)))
    for m, v in o.lyap.items():
        g.put("lyap/" + m, h5.Dataset(_file(v, np.float64)))
    for nm, v in o.diagnostics.items():
        g.put("diagnostics/" + nm, h5.Dataset(_file(v, np.float64), attrs={
            "threshold": float(o.thresholds[nm]), "first_exceedance_step": int(o.first_exceedance[nm])}))
    for m, c in o.cost.items():
        g.put("cost/" + m, h5.Dataset(_file(c, np.float64)))
    for sid, t in o.indicators.items():
        base = f"indicators/{sid}/"
        if t.series is not None:
            g.put(base + "series", h5.Dataset(_file(t.series, np.float64), attrs={"columns": list(t.columns)}))
        if t.final is not None:
            g.put(base + "final", h5.Dataset(_file(t.final, np.float64),
                                             attrs={"columns": list(t.fcolumns), "rows": list(t.rows)}))
            g.put(base + "flags", h5.Dataset(_file(t.flags, np.int64), attrs={"bits": list(t.bits)}))
        if t.scalars is not None:
            at = {"columns": list(t.scolumns)}
            if t.range is not None:
                at["range"] = np.asarray(t.range, dtype=np.float64)
            g.put(base + "scalars", h5.Dataset(_file(t.scalars, np.float64), attrs=at))
        if t.counts is not None:
            g.put(base + "counts", h5.Dataset(_file(t.counts, np.uint32)))


def pooled_of(orbits) -> dict:
    """run_indicator_store.jl:41-50: per spec id, the number of orbits with pooled counts and, when they share one
    range bitwise, the exact int64 sum of their counts and that range."""
    out = {}
    ids = sorted({sid for o in orbits for sid, t in o.indicators.items() if t.pool is not None})
    for sid in ids:
        ts = [o.indicators[sid] for o in orbits if sid in o.indicators and o.indicators[sid].pool is not None]
        shared = all(_isequal(t.range, ts[0].range) for t in ts)
        counts = None
        if shared:
            counts = np.zeros(np.shape(ts[0].pool), np.int64)
            for t in ts:
                counts += np.asarray(t.pool, dtype=np.int64)
        out[sid] = {"orbits": len(ts), "counts": counts,
                    "range": None if not shared or ts[0].range is None else np.asarray(ts[0].range, np.float64)}
    return out


def _tree(attrs: dict, prov: dict, orbits, hook) -> h5.Group:
    root = h5.Group(attrs=dict(attrs))
    for m, d in prov.items():
        root.require(f"provenance/{m}").attrs.update(d)
    root.require("orbits")
    hook("before_data")
    half = -(-len(orbits) // 2)
    for j, o in enumerate(orbits, 1):
        _put_orbit(root, o)
        if j == half:
            hook("during_data")
    for sid, p in sorted(pooled_of(orbits).items()):
        g = root.require(f"pooled/{sid}")
        g.attrs["orbits"] = int(p["orbits"])
        if p["counts"] is None:
            continue
        g.put("counts", h5.Dataset(_file(p["counts"], np.int64)))
        g.attrs["range"] = p["range"]
    return root


# ---------------------------------------------------------------- files
def _nohook(_point) -> None:
    return None


def _retry(f, tries: int = RETRY_TRIES, pause: float | None = None):
    """run_store.jl:26-35: call f(), again while another process holds a file (EBUSY / EACCES / EPERM)."""
    pause = RETRY_PAUSE if pause is None else pause
    for k in range(1, tries + 1):
        try:
            return f()
        except OSError as e:
            if e.errno not in RETRY_CODES or k >= tries:
                raise
            time.sleep(pause * k)


def _move_retry(src: str, dst: str, mover=os.replace, tries: int = RETRY_TRIES, pause: float | None = None):
    return _retry(lambda: mover(src, dst), tries=tries, pause=pause)


def _take_name(path: str) -> None:
    """run_store.jl:129-136: a final name that is taken is moved to `<name>.old<k>` first."""
    if not os.path.lexists(path):
        return
    k = 1
    while os.path.lexists(f"{path}.old{k}"):
        k += 1
    os.rename(path, f"{path}.old{k}")


def _fsync(path: str) -> None:
    fd = os.open(path, os.O_RDWR)
    try:
        os.fsync(fd)
    finally:
        os.close(fd)


def _attr_diff(want: dict, got: dict) -> list[str]:
    return sorted(k for k in set(want) | set(got) if not (k in want and k in got and _isequal(want[k], got[k])))


def write_chunk(path: str, attrs: dict, orbits, *, hook=_nohook, onread=_nohook, mover=os.replace) -> str:
    """Write a chunk file atomically (run_store.jl:138-186); `hook(point)` is called at "before_data",
    "during_data" (after half the orbits), "after_data", "before_rename" and "after_rename"; `onread(kind)` before
    each read-back of the temporary file ("datasets", "attrs")."""
    tmp = path + ".tmp"
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    want = dict(attrs)
    want["complete"] = False
    prov = want.pop("provenance", {})
    h5.write(tmp, _tree(want, prov, list(orbits), hook))
    onread("datasets")
    back = read_chunk(tmp)
    if len(back.orbits) != len(orbits) or not all(same_orbit(a, b) for a, b in zip(sorted(orbits, key=lambda o: o.id),
                                                                                  back.orbits)):
        raise RuntimeError(f"write_chunk: {tmp} differs from the buffers after the write")
    if not _isequal(pooled_of(orbits), back.pooled):
        raise RuntimeError(f"write_chunk: pooled counts of {tmp} differ from the buffers after the write")
    if not _isequal(prov, back.attrs.get("provenance", {})):
        raise RuntimeError(f"write_chunk: provenance of {tmp} differs from the buffers after the write")
    bad = _attr_diff(want, {k: v for k, v in back.attrs.items() if k != "provenance"})
    if bad:
        raise RuntimeError(f"write_chunk: root attributes of {tmp} differ from the buffers after the write: "
                           + ", ".join(bad))
    hook("after_data")
    h5.patch_attr(tmp, "/", "complete", True)
    onread("attrs")
    if read_chunk_attrs(tmp).get("complete") is not True:
        raise RuntimeError(f"write_chunk: {tmp} does not read back complete")
    _fsync(tmp)
    hook("before_rename")
    _take_name(path)
    _move_retry(tmp, path, mover=mover)
    hook("after_rename")
    return path


# ---------------------------------------------------------------- reading
def _ds(g: h5.Group, name: str):
    m = g.members.get(name)
    if m is None:
        return None, {}
    if not isinstance(m, h5.Dataset):
        raise h5.H5FormatError(f"{name!r} is not a dataset")
    return _julia(m.data), m.attrs


def _read_indicators(g: h5.Group) -> dict:
    """run_indicator_store.jl:82-100."""
    out = {}
    ig = g.members.get("indicators")
    if ig is None:
        return out
    for sid, s in ig.members.items():
        series, sa = _ds(s, "series")
        final, fa = _ds(s, "final")
        flags, ga = _ds(s, "flags")
        scalars, ca = _ds(s, "scalars")
        counts, _ = _ds(s, "counts")
        out[sid] = IndicatorTable(series=series, columns=list(sa.get("columns", [])), final=final,
                                  rows=list(fa.get("rows", [])), fcolumns=list(fa.get("columns", [])), flags=flags,
                                  bits=list(ga.get("bits", [])), scalars=scalars,
                                  scolumns=list(ca.get("columns", [])), range=ca.get("range"), counts=counts)
    return out


def _read_orbit(g: h5.Group, oid: int) -> OrbitRecord:
    """run_store.jl:201-210."""
    cg = g.members["cost"]
    lyap = {m: _julia(d.data) for m, d in g.members["lyap"].members.items()} if "lyap" in g.members else {}
    diag, thr, fe = {}, {}, {}
    if "diagnostics" in g.members:
        for nm, d in g.members["diagnostics"].members.items():
            diag[nm] = _julia(d.data)
            thr[nm] = float(d.attrs["threshold"])
            fe[nm] = int(d.attrs["first_exceedance_step"])
    cost = {m: _julia(d.data) for m, d in cg.members.items()}
    wind = _julia(g.members["winding"].data) if "winding" in g.members else None
    return OrbitRecord(oid, dict(g.attrs), _julia(g.members["t"].data), _julia(g.members["state"].data), wind, lyap,
                       diag, thr, fe, cost, "", _read_indicators(g))


def _read_pooled(root: h5.Group) -> dict:
    out = {}
    pg = root.members.get("pooled")
    if pg is None:
        return out
    for sid, g in pg.members.items():
        out[sid] = {"orbits": int(g.attrs["orbits"]),
                    "counts": _julia(g.members["counts"].data) if "counts" in g.members else None,
                    "range": g.attrs.get("range")}
    return out


def read_chunk(path: str) -> Chunk:
    """run_store.jl:213-223: `(attrs, orbits, pooled)`, the orbits in id order; the provenance groups under
    attrs["provenance"]."""
    if not os.path.isfile(path):
        raise FileNotFoundError(f"no chunk file {path}")
    root = h5.read(path)
    og = root.members["orbits"]
    attrs = dict(root.attrs)
    if "provenance" in root.members:
        attrs["provenance"] = {m: dict(g.attrs) for m, g in root.members["provenance"].members.items()}
    orbits = [_read_orbit(og.members[str(i)], i) for i in sorted(int(k) for k in og.members)]
    return Chunk(attrs, orbits, _read_pooled(root))


def read_chunk_attrs(path: str) -> dict:
    """The root attributes only (run_store.jl:226)."""
    return dict(h5.read(path).attrs)


_JULIA_TYPES = {"<i8": "Int64", "<i4": "Int32", "<u4": "UInt32", "|u1": "UInt8", "<f8": "Float64", "<f4": "Float32"}


def chunk_layout(path: str) -> dict:
    """run_store.jl:228-240: dataset path => (element type name, Julia dimensions) of every dataset of a chunk."""
    out = {}

    def walk(g: h5.Group, prefix: str) -> None:
        for k, m in g.members.items():
            if isinstance(m, h5.Dataset):
                out[f"{prefix}/{k}"] = (_JULIA_TYPES[m.data.dtype.str], tuple(reversed(m.data.shape)))
            else:
                walk(m, f"{prefix}/{k}")
    walk(h5.read(path), "")
    return out


# ---------------------------------------------------------------- device records to orbit records
_ALG_G = ("L3", "L4")     # CGS and MGS: the orthogonality threshold scales with the window's G_w (orthonormalize.jl:141-151)


def thresholds(method: str, tol: dict, *, tau: int, G_max: float, M_max: float, k: int, T: str = "Float64") -> dict:
    """run_record.jl:189-200 for a 2 x 2 tangent: det `tol eps (1 + M_max)`, symp `tol eps N^2 (1 + M_max)^2`
    (N = 1), with k = 2 sum and pair `sum_threshold(pairing tol, T, G_max, tau, M_max)` and, except L9, orth
    `tol eps k g`, g = G_max + 1 / G_max for CGS / MGS (L3, L4), else 1 (residuals.jl:22-32)."""
    eps = effective_eps(T)
    m = abs(float(M_max))
    out = {"det": float(np.float64(tol["det_residual_tol"]) * eps * (1 + m)),
           "symp": float(np.float64(tol["det_residual_tol"]) * eps * 1 * (1 + m) ** 2)}
    if k == 2:
        s = float(sum_threshold(tol["pairing_residual_tol"], T, G_max, tau, M_max))
        out["sum"] = s
        out["pair"] = s
        if method != "L9":
            g = (G_max + 1 / G_max) if method in _ALG_G else 1.0
            out["orth"] = float(np.float64(tol["orthogonality_tol"]) * eps * k * g)
    return out


def _first_exceedance(v: np.ndarray, thr: float, t: np.ndarray) -> int:
    """run_record.jl:203-206: the step count of the first row above the threshold, 0 when none (NaN is not above)."""
    hit = np.flatnonzero(v > thr)
    return int(t[hit[0]]) if hit.size else 0


def orbit_records(rec, items, tol: dict, *, T: str = "Float64") -> list[OrbitRecord]:
    """The orbit records of a chunk from the device recorder's result `rec` (chaos_b200.record.RecordResult): orbit j
    of the record belongs to `items[j]`, a dict with the item's `orbit` (the id), `system`, `param`, `x0`, `p0`,
    `design_class`, `orbit_seed`, `hash`, `method`, `horizon`, `tau`, `vectors` and `coordinate_mode`; `tol` holds
    `det_residual_tol`, `pairing_residual_tol` and `orthogonality_tol`. Rows before the failing grid row come from
    the record (run_device.jl:127-140); from it on `t` is 0 and the state, exponents and diagnostics NaN
    (run_record.jl:226-238); the thresholds use the last good row's G_max and M_max (1 and 1 when there is none)."""
    k, grid = rec.k, np.asarray(rec.grid, np.int64)
    n = len(grid)
    s = rec.R.shape[2] - (k + 7)
    out = []
    for j, it in enumerate(items):
        fail = int(rec.fail[j])
        last = n if fail == 0 else fail - 1
        rows = rec.R[j, :last]
        t = np.zeros(n, np.int64)
        t[:last] = grid[:last]
        state = np.zeros((n, 2))
        lyap = np.zeros((n, k))
        ser = np.zeros((5, n))
        state[:last] = rows[:, k + 7:k + 9]
        lyap[:last] = rows[:, :k]
        ser[:, :last] = rows[:, k:k + 5].T
        wrapped = it["coordinate_mode"] == "wrapped"
        wind = np.zeros((n, 2), np.int64) if wrapped else None
        if wrapped and s == 4:
            wind[:last] = rows[:, k + 9:k + 11].astype(np.int64)
        gmax, mmax = (float(rows[-1, k + 5]), float(rows[-1, k + 6])) if last >= 1 else (1.0, 1.0)
        if fail:
            state[fail - 1:] = np.nan
            lyap[fail - 1:] = np.nan
            ser[:, fail - 1:] = np.nan
        method = it["method"]
        names = diagnostic_names(method)
        thr = {} if method == "L2" else thresholds(method, tol, tau=int(it["tau"]), G_max=gmax, M_max=mmax, k=k, T=T)
        col = {"det": 0, "symp": 1, "orth": 2, "sum": 3, "pair": 4}
        diag = {nm: ser[col[nm]].copy() for nm in names}
        fe = {nm: _first_exceedance(diag[nm], thr[nm], t) for nm in names}
        nser = 1 + 2 + (2 if wrapped else 0) + int(it["vectors"]) + len(names)
        resident = 8 * (s + 2 * k + 2 * k) + 16 + rec.states.shape[1] + 8 * nser * n
        attrs = {"system": it["system"], "params": it["param"], "ic": f"{it['x0']},{it['p0']}",
                 "class_label": it["design_class"], "seed": it["orbit_seed"], "item_hash": it["hash"],
                 "design_class": it["design_class"], "flags": [], "steps_recorded": n}
        failure = "" if not fail else f"orbit {it['orbit']}: status {int(rec.code[j])} at step {int(rec.hstep[j])}"
        out.append(OrbitRecord(int(it["orbit"]), attrs, t, state, wind, {method: lyap}, diag, thr, fe,
                               {method: np.array([it["horizon"], it["vectors"], 0.0, 0.0, resident], np.float64)},
                               failure))
    return out
