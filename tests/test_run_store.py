"""The run store (chaos_b200/run_store.py over chaos_b200/h5.py): HDF5 chunk files with the layout of
src/Experiments/run_store.jl and run_indicator_store.jl, tested as the reference's test/experiments/ex_store.jl and
ex_d86_store.jl test it -- the layout and element types, bit-for-bit read-back with special values, the atomic write
(temporary name, `complete`, `.old<k>`, retried rename, hook points), pooled counts -- and the file bytes against the
HDF5 format's fixed fields."""
from __future__ import annotations

import errno
import os
import struct

import numpy as np
import pytest

from chaos_b200 import h5
from chaos_b200 import run_store as RS

TOL = {"det_residual_tol": 16.0, "pairing_residual_tol": 16.0, "orthogonality_tol": 16.0}


def _orbit(oid: int, n: int = 6, k: int = 2, wrapped: bool = False, rng=None, indicators=None) -> RS.OrbitRecord:
    rng = rng or np.random.default_rng(oid)
    names = RS.diagnostic_names("L4")
    diag = {nm: rng.random(n) for nm in names}
    return RS.OrbitRecord(
        oid, {"system": "standard", "params": "0.971635", "ic": "0.1,0.2", "class_label": "chaotic", "seed": 17 + oid,
              "item_hash": "ab" * 32, "design_class": "chaotic", "flags": [], "steps_recorded": n},
        np.arange(1, n + 1, dtype=np.int64) * 10, rng.random((n, 2)),
        rng.integers(-5, 5, (n, 2)).astype(np.int64) if wrapped else None, {"L4": rng.standard_normal((n, k))},
        diag, {nm: 1e-12 * (i + 1) for i, nm in enumerate(names)}, {nm: 0 for nm in names},
        {"L4": np.array([1e4, k, 0.25, 1.0, 4096.0])}, "", indicators or {})


def _attrs(**kw) -> dict:
    a = {"schema_version": 2, "study": "p1-le-benchmark", "chunk": 17, "chunk_key": "k1:chaotic", "status": "ok",
         "attempt": 1, "pilot": False, "arms": ["a", "bb"], "first_attempt_reasons": [], "failure_reasons": [],
         "created_utc": "2026-10-12T14:03:00Z", "tau": 10, "horizon": 10000, "vectors": 2, "dirty": False,
         "backend": "gpu", "device": "NVIDIA B200", "backend_fallback_reason": ""}
    a.update(kw)
    return a


# ---------------------------------------------------------------- the HDF5 layer
def test_h5_fixed_fields(tmp_path):
    """Superblock version 0 (signature, sizes 8 / 8, K = 4 / 16, base 0, end of file = file size, the root's symbol
    table entry with cache type 1 pointing at a version 1 object header whose Symbol Table message names a TREE node
    and a HEAP) and the Float64 datatype message bytes of the specification."""
    p = tmp_path / "f.h5"
    root = h5.Group(attrs={"x": 1.5})
    root.put("d", h5.Dataset(np.arange(3, dtype=np.float64)))
    h5.write(str(p), root)
    b = p.read_bytes()
    assert b[:8] == b"\x89HDF\r\n\x1a\n" and b[8:16] == bytes([0, 0, 0, 0, 0, 8, 8, 0])
    assert struct.unpack_from("<HHI", b, 16) == (4, 16, 0)
    base, free, eof, drv = struct.unpack_from("<QQQQ", b, 24)
    assert (base, free, eof, drv) == (0, h5.UNDEF, len(b), h5.UNDEF)
    name_off, hdr, cache = struct.unpack_from("<QQI", b, 56)
    bt, heap = struct.unpack_from("<QQ", b, 80)
    assert name_off == 0 and cache == 1 and hdr % 8 == 0
    assert b[hdr] == 1 and struct.unpack_from("<HH", b, hdr + 16) == (0x11, 16)
    assert struct.unpack_from("<QQ", b, hdr + 24) == (bt, heap)
    assert b[bt:bt + 4] == b"TREE" and b[heap:heap + 4] == b"HEAP"
    f64 = bytes([0x11, 0x20, 63, 0, 8, 0, 0, 0, 0, 0, 64, 0, 52, 11, 0, 52]) + struct.pack("<I", 1023)
    assert f64 in b


@pytest.mark.parametrize("members", [0, 1, 8, 9, 256, 257, 1100])
def test_h5_group_sizes(members):
    """Groups whose members fill no, one, several symbol table nodes and one, two or three B-tree levels: every
    member back, in byte order of the names."""
    root = h5.Group()
    g = root.require("orbits")
    for i in range(members):
        g.put(str(i), h5.Group(attrs={"i": i}))
    back = h5.read_image(h5.image(root))
    names = list(back.members["orbits"].members)
    assert names == sorted((str(i) for i in range(members)), key=str.encode)
    assert all(back.members["orbits"].members[str(i)].attrs == {"i": i} for i in range(members))
    # the leaf level read the way older readers iterate it -- down the left-most children, then along the right
    # sibling links -- gives the same symbol table nodes as the recursive walk
    img = h5.image(root)
    bt = struct.unpack_from("<Q", img, 80)[0]
    obt = None
    for off, hdr in _snod_entries(img, bt):
        obt = struct.unpack_from("<Q", img, hdr + 24)[0]
    node, level = obt, img[obt + 5]
    while level:
        node = struct.unpack_from("<Q", img, node + 32)[0]
        level = img[node + 5]
    chain = []
    while node != h5.UNDEF:
        used = struct.unpack_from("<H", img, node + 6)[0]
        chain += [struct.unpack_from("<Q", img, node + 32 + 16 * i)[0] for i in range(used)]
        node = struct.unpack_from("<Q", img, node + 16)[0]
    assert len(chain) == -(-members // 8)
    assert sum(struct.unpack_from("<H", img, a + 6)[0] for a in chain) == members


def _snod_entries(img, node):
    """(name offset, header address) of every entry under a group B-tree node, recursively."""
    level, used = img[node + 5], struct.unpack_from("<H", img, node + 6)[0]
    for i in range(used):
        child = struct.unpack_from("<Q", img, node + 32 + 16 * i)[0]
        if level:
            yield from _snod_entries(img, child)
        else:
            for j in range(struct.unpack_from("<H", img, child + 6)[0]):
                yield struct.unpack_from("<QQ", img, child + 8 + 40 * j)


def test_h5_values():
    vals = {"t": True, "f": False, "i": -(2 ** 62), "x": -0.0, "nan": float("nan"), "sub": 5e-324, "s": "",
            "u": "Gram–Schmidt", "l": ["", "a", "ccc"], "e": [], "r": [0.25, float("inf")], "w": np.uint32(7),
            "ia": np.arange(4, dtype=np.int64)}
    back = h5.read_image(h5.image(h5.Group(attrs=vals))).attrs
    assert back.keys() == vals.keys()
    for k, v in vals.items():
        assert RS._isequal(v, back[k]), k
    assert type(back["t"]) is bool and type(back["i"]) is int and type(back["s"]) is str and back["l"] == vals["l"]
    assert np.signbit(back["x"]) and back["w"].dtype == np.uint32
    with pytest.raises(h5.H5FormatError):
        h5.image(h5.Group(attrs={"bad": "a\0b"}))
    with pytest.raises(h5.H5FormatError):
        h5.image(h5.Group(attrs={"big": "x" * 70000}))


def test_h5_datasets_bitwise():
    rng = np.random.default_rng(1)
    a = rng.standard_normal((3, 5))
    a[0, 0], a[1, 1], a[2, 2] = np.nan, -0.0, 5e-324
    arrs = {"f": a, "i": rng.integers(-9, 9, 7).astype(np.int64), "u": rng.integers(0, 99, (2, 4)).astype(np.uint32),
            "z": np.zeros((0, 2)), "s": np.array(3.5)}
    root = h5.Group()
    for k, v in arrs.items():
        root.put(k, h5.Dataset(v, attrs={"columns": ["a", "b"]}))
    back = h5.read_image(h5.image(root))
    for k, v in arrs.items():
        d = back.members[k].data
        assert d.dtype == v.dtype and d.shape == v.shape and RS._same_array(d, v), k
        assert back.members[k].attrs == {"columns": ["a", "b"]}


def test_h5_rejects_foreign_bytes(tmp_path):
    with pytest.raises(h5.H5FormatError):
        h5.read_image(b"not an hdf5 file at all" * 8)
    img = h5.image(h5.Group(attrs={"a": 1}))
    with pytest.raises(h5.H5FormatError):
        h5.read_image(img[:-8])


# ---------------------------------------------------------------- chunk files
def test_chunk_layout_and_read_back(tmp_path):
    """ex_store.jl "D53m store layout" / "write and read back bit for bit": Julia shapes and element types of every
    dataset, the special values stored as written, complete true, no temporary file left."""
    p = str(tmp_path / "s" / "chunk-00017.h5")
    orbs = [_orbit(i, wrapped=(i % 2 == 0)) for i in (3, 1, 2, 10)]
    m = orbs[0].lyap["L4"]
    m[0, 0], m[1, 0], m[2, 0], m[3, 0] = np.nan, np.inf, -0.0, 5e-324
    RS.write_chunk(p, _attrs(), orbs)
    ch = RS.read_chunk(p)
    assert [o.id for o in ch.orbits] == [1, 2, 3, 10]
    want = {o.id: o for o in orbs}
    assert all(RS.same_orbit(want[o.id], o) for o in ch.orbits)
    assert ch.attrs["complete"] is True and ch.attrs["pilot"] is False and ch.attrs["arms"] == ["a", "bb"]
    assert os.listdir(os.path.dirname(p)) == ["chunk-00017.h5"]
    lay = RS.chunk_layout(p)
    for o in orbs:
        b = f"/orbits/{o.id}"
        assert lay[f"{b}/t"] == ("Int64", (6,)) and lay[f"{b}/state"] == ("Float64", (6, 2))
        assert lay[f"{b}/lyap/L4"] == ("Float64", (6, 2)) and lay[f"{b}/cost/L4"] == ("Float64", (5,))
        assert all(lay[f"{b}/diagnostics/{d}"] == ("Float64", (6,)) for d in RS.diagnostic_names("L4"))
        assert (f"{b}/winding" in lay) == (o.winding is not None)
    raw = h5.read(p).members["orbits"].members["1"].members["state"].data
    assert raw.shape == (2, 6) and np.array_equal(raw, orbs[1].state.T)
    with pytest.raises(FileNotFoundError):
        RS.read_chunk(str(tmp_path / "missing.h5"))


def test_indicators_provenance_pooled(tmp_path):
    """ex_d86_store.jl: the indicator tables with their attributes, the provenance groups, and pooled counts -- the
    exact int64 sum when the orbits share a range, the orbit count alone when they do not."""
    def tab(seed, rng_lo):
        r = np.random.default_rng(seed)
        return RS.IndicatorTable(series=r.random((6, 3)), columns=["MEGNO", "Ybar", "FLI"], final=r.random((2, 4)),
                                 rows=["w1", "w2"], fcolumns=["a", "b", "c", "d"], flags=np.array([128, 1538]),
                                 bits=["mirror1", "degenerate"], scalars=r.random(3), scolumns=["x", "y", "z"],
                                 range=np.array([rng_lo, 2.0]), counts=r.integers(0, 50, (5, 2)).astype(np.uint32),
                                 pool=r.integers(0, 50, (5, 2)))
    orbs = [_orbit(i, indicators={"s1": tab(i, 0.5)}) for i in range(1, 4)]
    for o in orbs:
        o.lyap = {}
    prov = {"MEGNO": {"key": "v", "replace": True}, "stretching": {"bins": 3}}
    p = str(tmp_path / "c.h5")
    RS.write_chunk(p, _attrs(kind="tangent", provenance=prov), orbs)
    ch = RS.read_chunk(p)
    assert all(RS.same_orbit(a, b) for a, b in zip(orbs, ch.orbits))
    assert RS._isequal(ch.attrs["provenance"], prov)
    assert ch.pooled["s1"]["orbits"] == 3 and np.array_equal(ch.pooled["s1"]["counts"],
                                                             sum(o.indicators["s1"].pool for o in orbs))
    assert RS.chunk_layout(p)["/orbits/1/indicators/s1/counts"] == ("UInt32", (5, 2))
    orbs[2].indicators["s1"].range = np.array([0.25, 2.0])
    RS.write_chunk(p, _attrs(), orbs)
    ch = RS.read_chunk(p)
    assert ch.pooled["s1"] == {"orbits": 3, "counts": None, "range": None}
    assert os.path.exists(p + ".old1")


def test_atomic_write_hooks_and_names(tmp_path):
    """run_store.jl:138-186: the hook points in order; a taken final name moves to .old1, .old2; the rename is
    retried while another process holds the file (EBUSY), other errors are raised; a read-back that differs
    raises and leaves the final name untouched."""
    p = str(tmp_path / "c.h5")
    seen = []
    RS.write_chunk(p, _attrs(), [_orbit(1)], hook=seen.append, onread=lambda k: seen.append("read:" + k))
    assert seen == ["before_data", "during_data", "read:datasets", "after_data", "read:attrs", "before_rename",
                    "after_rename"]
    RS.write_chunk(p, _attrs(chunk=18), [_orbit(1)])
    RS.write_chunk(p, _attrs(chunk=19), [_orbit(1)])
    assert RS.read_chunk_attrs(p + ".old1")["chunk"] == 17 and RS.read_chunk_attrs(p + ".old2")["chunk"] == 18
    tries = []

    def busy(src, dst):
        tries.append(1)
        if len(tries) < 3:
            raise OSError(errno.EBUSY, "busy")
        os.replace(src, dst)
    RS.RETRY_PAUSE, old = 0.0, RS.RETRY_PAUSE
    try:
        RS.write_chunk(p, _attrs(chunk=20), [_orbit(1)], mover=busy)
        assert len(tries) == 3 and RS.read_chunk_attrs(p)["chunk"] == 20

        def denied(src, dst):
            raise OSError(errno.ENOSPC, "no space")
        with pytest.raises(OSError):
            RS.write_chunk(p, _attrs(chunk=21), [_orbit(1)], mover=denied)
    finally:
        RS.RETRY_PAUSE = old


def test_read_back_mismatch_is_caught(tmp_path):
    q = str(tmp_path / "d.h5")

    def corrupt(kind):
        if kind == "datasets":
            b = bytearray(open(q + ".tmp", "rb").read())
            i = b.rfind(np.float64(1e4).tobytes())
            b[i:i + 8] = np.float64(2e4).tobytes()
            open(q + ".tmp", "wb").write(bytes(b))
    with pytest.raises(RuntimeError, match="differs from the buffers"):
        RS.write_chunk(q, _attrs(), [_orbit(1)], onread=corrupt)
    assert not os.path.exists(q)


# ---------------------------------------------------------------- device records to orbit records
class _Rec:
    def __init__(self, R, grid, fail, k, wrapped):
        self.R, self.grid, self.fail, self.k = R, np.asarray(grid), np.asarray(fail), k
        self.states = np.zeros((R.shape[0], 48), np.uint8)
        self.code = np.where(self.fail > 0, 1, 0)
        self.hstep = np.zeros(R.shape[0], np.int64)


def _item(i, method="L4", wrapped=False):
    return {"orbit": i + 1, "system": "standard", "param": "1.2", "x0": "0.1", "p0": "0.2", "design_class": "chaotic",
            "orbit_seed": "5", "hash": "h%d" % i, "method": method, "horizon": 40, "tau": 10, "vectors": 2,
            "coordinate_mode": "wrapped" if wrapped else "lifted"}


def test_orbit_records_rows_and_thresholds(tmp_path):
    """run_device.jl:127-140 and run_record.jl:186-238: rows before the failing grid row, NaN (and t = 0) from it
    on, windings as integers, the thresholds from the last good row's G_max and M_max, first exceedance steps."""
    k, grid = 2, [10, 20, 30, 40]
    rng = np.random.default_rng(3)
    R = rng.random((2, 4, k + 7 + 4))
    R[:, :, k + 9:k + 11] = rng.integers(-3, 3, (2, 4, 2))
    R[0, :, k] = [1e-20, 1e-20, 1.0, 1e-20]                   # det above its threshold at step 30
    rec = _Rec(R, grid, [0, 3], k, True)
    orbs = RS.orbit_records(rec, [_item(0, wrapped=True), _item(1, wrapped=True)], TOL)
    a, b = orbs
    assert np.array_equal(a.t, grid) and np.array_equal(b.t, [10, 20, 0, 0])
    assert np.array_equal(a.state, R[0, :, k + 7:k + 9]) and np.all(np.isnan(b.state[2:]))
    assert np.array_equal(b.lyap["L4"][:2], R[1, :2, :k]) and np.all(np.isnan(b.lyap["L4"][2:]))
    assert np.array_equal(a.winding, R[0, :, k + 9:k + 11].astype(np.int64)) and np.all(b.winding[2:] == 0)
    eps = np.finfo(np.float64).eps
    gmax, mmax = R[0, 3, k + 5], R[0, 3, k + 6]
    assert a.thresholds["det"] == 16.0 * eps * (1 + mmax)
    assert a.thresholds["symp"] == 16.0 * eps * (1 + mmax) ** 2
    assert a.thresholds["sum"] == 16.0 * eps * (gmax / 10 + mmax) == a.thresholds["pair"]
    assert a.thresholds["orth"] == 16.0 * eps * 2 * (gmax + 1 / gmax)
    assert a.first_exceedance["det"] == 30 and b.first_exceedance["det"] in (0, 10, 20)
    assert b.thresholds["det"] == 16.0 * eps * (1 + R[1, 1, k + 6])
    assert a.cost["L4"][4] == 8 * (4 + 4 + 4) + 16 + 48 + 8 * (1 + 2 + 2 + 2 + 5) * 4
    p = str(tmp_path / "r.h5")
    RS.write_chunk(p, _attrs(), orbs)
    assert all(RS.same_orbit(x, y) for x, y in zip(orbs, RS.read_chunk(p).orbits))


@pytest.mark.parametrize("name", ["standard", "wrapped"])
def test_oracle_record_chunk(oracle, tmp_path, name):
    """A chunk from the oracle's study recorder (MGS, k = 2, a failing orbit): the records, the file and its
    read-back agree bit for bit; the failing orbit's rows are NaN from its failing grid row on."""
    from types import SimpleNamespace

    from chaos_b200 import MGS, QRSpectrum, StandardMap, WrappedStandardMap, torus_state
    z = np.random.default_rng(31).uniform(0, 2 * np.pi, (12, 2))
    sysm = StandardMap(2.5) if name == "standard" else WrappedStandardMap(6.0)
    x = z if name == "standard" else np.array([torus_state(v) for v in z])
    x[3, 0] = np.nan
    grid = [5, 20, 100]
    ref = oracle.oracle_record(sysm, x, 100, 5, QRSpectrum(MGS()), grid)
    rec = SimpleNamespace(R=ref["R"], grid=np.asarray(grid), fail=ref["fail"], k=2, states=ref["states"],
                          code=ref["code"], hstep=ref["hstep"])
    items = [_item(i, wrapped=name == "wrapped") for i in range(len(x))]
    orbs = RS.orbit_records(rec, items, TOL)
    assert ref["fail"][3] == 1 and np.all(np.isnan(orbs[3].state)) and orbs[3].t.sum() == 0
    assert (orbs[0].winding is not None) == (name == "wrapped")
    p = str(tmp_path / "chunk-00001.h5")
    RS.write_chunk(p, _attrs(coordinate_mode="wrapped" if name == "wrapped" else "lifted"), orbs)
    back = RS.read_chunk(p)
    assert all(RS.same_orbit(u, v) for u, v in zip(orbs, back.orbits))


def test_h5_dataset_header_by_hand():
    """A dataset's version 1 object header walked by hand (not through the package's reader): Dataspace, Datatype
    (constant), Fill Value and Data Layout messages in that order, then an Attribute message; the layout's address and
    size point at the array's little-endian bytes; the bool and string attribute types carry the format's class bits."""
    data = np.array([[1.5, -2.0, 3.25], [0.0, 7.0, -0.5]])
    root = h5.Group()
    root.put("d", h5.Dataset(data, attrs={"ok": True, "name": "ab"}))
    b = h5.image(root)
    # the root group's only member: its symbol table node entry gives the dataset's header
    bt = struct.unpack_from("<Q", b, 80)[0]
    snod = struct.unpack_from("<Q", b, bt + 32)[0]
    assert b[snod:snod + 4] == b"SNOD" and struct.unpack_from("<H", b, snod + 6)[0] == 1
    hdr = struct.unpack_from("<Q", b, snod + 8 + 8)[0]
    ver, _, nmsg, refc, size = struct.unpack_from("<BBHII", b, hdr)
    assert (ver, nmsg, refc) == (1, 6, 1)
    p, end, kinds = hdr + 16, hdr + 16 + size, []
    while p < end:
        mtype, msize, flags = struct.unpack_from("<HHB", b, p)
        kinds.append((mtype, flags))
        body = p + 8
        if mtype == 0x1:
            assert b[body] == 1 and b[body + 1] == 2 and struct.unpack_from("<QQ", b, body + 8) == (2, 3)
        if mtype == 0x8:
            assert b[body] == 3 and b[body + 1] == 1
            addr, nbytes = struct.unpack_from("<QQ", b, body + 2)
            assert nbytes == 48 and b[addr:addr + nbytes] == data.astype("<f8").tobytes()
        if mtype == 0xC:
            nlen, dlen = struct.unpack_from("<HH", b, body + 2)
            name = b[body + 8:body + 8 + nlen - 1].decode()
            dt = body + 8 + ((nlen + 7) & ~7)
            if name == "ok":
                assert b[dt] == 0x18 and b[dt + 1] == 2 and b[dt + 8] == 0x10   # enum of 2 members, int8 base
            else:
                assert b[dt] == 0x13 and b[dt + 1] == 0x10 and struct.unpack_from("<I", b, dt + 4)[0] == 2
        p = body + msize
    assert [k for k, _ in kinds] == [0x1, 0x3, 0x5, 0x8, 0xC, 0xC]
    assert dict(kinds)[0x3] == 1
