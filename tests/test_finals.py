"""The finals records of a result (`reducer_final` per orbit, src/Tangent/propagate.jl:116-118) computed for all
orbits at once: every record equals the per-orbit `final` of the reducer, field by field and bit for bit."""
import numpy as np
import pytest

from chaos_b200 import FLI, GALI, MEGNO, SALI, Benettin, FroeschleMap, GivensQR, HouseholderQR, QRSpectrum, StandardMap
from chaos_b200.propagate import FrameSpec
from chaos_b200.reducers import Finals
from helpers import haar_frames, identity_frames, uniform_starts


def _eq(a, b):
    assert a.keys() == b.keys()
    for key in a:
        va, vb = a[key], b[key]
        if va is None or vb is None:
            assert va is None and vb is None
            continue
        assert type(va) is type(vb), key
        va, vb = np.asarray(va), np.asarray(vb)
        assert va.shape == vb.shape, key
        assert np.array_equal(va.view(np.uint64) if va.dtype.kind == "f" else va,
                              vb.view(np.uint64) if vb.dtype.kind == "f" else vb), key


CASES = [
    (lambda: FroeschleMap(1.5, 1.5, 0.05), 4, lambda n: FrameSpec(4, (QRSpectrum(HouseholderQR()),), identity_frames(n, 4, 4))),
    (lambda: FroeschleMap(1.5, 1.5, 0.05), 4, lambda n: FrameSpec(4, (GALI(), SALI()), identity_frames(n, 4, 4))),
    (lambda: FroeschleMap(1.5, 1.5, 0.05), 4, lambda n: FrameSpec(3, (GALI(),), identity_frames(n, 4, 3))),
    (lambda: StandardMap(1.1), 2, lambda n: FrameSpec(2, (MEGNO(replace=False), FLI(replace=False), QRSpectrum(GivensQR())), haar_frames(n, 2, 2, 1))),
    (lambda: StandardMap(0.0), 2, lambda n: FrameSpec(1, (Benettin(),), identity_frames(n, 2, 1))),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_columns_equal_per_orbit(oracle, case):
    mk, d, frame = CASES[case]
    n = 40
    sysm = mk()
    x0 = uniform_starts(n, d, seed=case)
    fr = frame(n)
    st = oracle.oracle_frames(sysm, x0, 300, [fr], tau=5, math="portable")[0]["states"]
    fin = Finals(fr.reducers, st, d)
    assert len(fin) == n
    for i in range(n):
        for j, r in enumerate(fr.reducers):
            ref = r.final(st[f"r{j}"][i], d) if isinstance(r, GALI) else r.final(st[f"r{j}"][i])
            _eq(fin[i][j], ref)
    st0 = np.zeros(3, dtype=st.dtype)   # before any handoff: n = 0 records
    f0 = Finals(fr.reducers, st0, d)
    for j, r in enumerate(fr.reducers):
        ref = r.final(st0[f"r{j}"][0], d) if isinstance(r, GALI) else r.final(st0[f"r{j}"][0])
        _eq(f0[0][j], ref)
