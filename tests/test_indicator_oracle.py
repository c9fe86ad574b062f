"""The indicator recorder's oracle (CPU), tangent kind (src/Experiments/run_indicator_device.jl:31-60): a row at a
grid step holds the members' reducer finals of the same chain run directly to that step (run_indicator_record.jl:
40-56), the monitor's maxima of the same orbit as the study recorder's, the orbit point; a member of the correct chain
is bitwise the stand-alone member and a replacing member first changes the later members (the mutation check of
test/experiments/ex_d86_chains.jl:75-88); launch windows change no bit; a failure stops the orbit at its grid index."""
from __future__ import annotations

import numpy as np
import pytest

from chaos_b200 import (FLI, MEGNO, MGS, SALI, LinearSymplecticMap, QRSpectrum, StandardMap, WrappedStandardMap,
                        torus_state)
from chaos_b200.propagate import FrameSpec
from chaos_b200.record import MEMBER_COLUMNS, indicator_chain

CHAINS = [["SALI"], ["FLI", "SALI"], ["MEGNO", "SALI"], ["FLI", "MEGNO", "SALI"], ["FLI"], ["MEGNO"], ["FLI", "MEGNO"]]


def _system(name, n=24, seed=5):
    z = np.random.default_rng(seed).uniform(0, 2 * np.pi, (n, 2))
    if name == "standard":
        return StandardMap(1.3), z
    if name == "wrapped":
        return WrappedStandardMap(2.5), np.array([torus_state(v) for v in z])
    return LinearSymplecticMap([[2.0, 1.0], [1.0, 1.0]]), z * 1e-6


def _member_columns(red, st):
    f = red.final(st)
    if isinstance(red, SALI):
        return np.stack([np.atleast_1d(f["sali"]), np.atleast_1d(f["L"])], axis=-1)
    if isinstance(red, FLI):
        return np.stack([np.atleast_1d(f["fli"]), np.atleast_1d(f["fli1"])], axis=-1)
    return np.concatenate([[f["Y"][c], f["Ybar"][c], f["Ybar20"][c]] for c in range(2)])[None, :]


@pytest.mark.parametrize("members", CHAINS, ids=",".join)
@pytest.mark.parametrize("name", ["standard", "wrapped", "linear"])
def test_rows_are_the_direct_runs_finals(oracle, members, name):
    sys, x0 = _system(name)
    N = 200 if name != "linear" else 40
    tau, grid = 2, [g for g in (2, 10, 40, 120, 200) if g <= N]
    rec = oracle.oracle_indicators(sys, x0, N, tau, members, grid, ns=2)
    chain = indicator_chain(members)
    assert (rec["fail"] == 0).all() and (rec["code"] == 0).all()
    W0 = np.broadcast_to(np.eye(2), (len(x0), 2, 2)).copy()
    for g, n in enumerate(grid):
        ref = oracle.oracle_frames(sys, x0, n, [FrameSpec(2, chain, W0)], tau=tau)[0]
        for i in range(len(x0)):
            want = np.concatenate([_member_columns(r, ref["states"][f"r{j}"][i]).ravel()
                                   for j, r in enumerate(chain)])
            got = rec["R"][i, g, :len(want)]
            assert got.tobytes() == want.tobytes(), (g, i)
        assert np.array_equal(rec["R"][:, g, -2:], ref["x"][:, :2])
    ref = oracle.oracle_frames(sys, x0, N, [FrameSpec(2, chain, W0)], tau=tau)[0]
    cb = ref["states"].dtype.itemsize
    assert rec["states"][:, :cb].tobytes() == ref["states"].tobytes()
    assert rec["W"].tobytes() == ref["W"].tobytes()


@pytest.mark.parametrize("name", ["standard", "wrapped", "linear"])
def test_monitor_columns_are_the_recorders(oracle, name):
    sys, x0 = _system(name, 32, 6)
    N, tau, grid = 60, 3, [3, 30, 60]
    ind = oracle.oracle_indicators(sys, x0, N, tau, ["MEGNO", "SALI"], grid, ns=2)
    rec = oracle.oracle_record(sys, x0, N, tau, QRSpectrum(MGS()), grid)
    # indicator row: 8 member columns, det, symp, M_max, x, p; recorder row: l1, l2, det, symp, orth, sum, pair, G, M
    assert np.array_equal(ind["R"][:, :, 8], rec["R"][:, :, 2])
    assert np.array_equal(ind["R"][:, :, 9], rec["R"][:, :, 3])
    assert np.array_equal(ind["R"][:, :, 10], rec["R"][:, :, 8])
    assert np.array_equal(ind["R"][:, :, 11:], rec["R"][:, :, 9:11])
    for c in (8, 9, 10):
        assert np.all(np.diff(ind["R"][:, :, c], axis=1) >= 0)


def test_chain_member_is_the_stand_alone_member(oracle):
    """The correct chain FLI, MEGNO, SALI (forms false, false, true): its FLI and MEGNO columns are bitwise the
    stand-alone members'; SALI first and replacing changes the FLI after it."""
    sys, x0 = _system("standard", 16, 9)
    N, tau, grid = 100, 1, [10, 50, 100]
    good = oracle.oracle_indicators(sys, x0, N, tau, ["FLI", "MEGNO", "SALI"], grid)["R"]
    fli = oracle.oracle_indicators(sys, x0, N, tau, ["FLI"], grid)["R"]
    megno = oracle.oracle_indicators(sys, x0, N, tau, ["MEGNO"], grid)["R"]
    assert good[:, :, 0:2].tobytes() == fli[:, :, 0:2].tobytes()
    assert good[:, :, 2:8].tobytes() == megno[:, :, 0:6].tobytes()
    bad = oracle.oracle_indicators(sys, x0, N, tau, ["SALI", "FLI"], grid)["R"]
    assert not np.array_equal(bad[:, :, 2:4], fli[:, :, 0:2])


@pytest.mark.parametrize("L", [4, 20, 140])
def test_launch_windows_change_no_bit(oracle, L):
    sys, x0 = _system("wrapped", 20, 7)
    a = oracle.oracle_indicators(sys, x0, 140, 2, ["FLI", "MEGNO", "SALI"], [20, 22, 100, 140], ns=4)
    b = oracle.oracle_indicators(sys, x0, 140, 2, ["FLI", "MEGNO", "SALI"], [20, 22, 100, 140], ns=4,
                                 launch_steps=L)
    for key in a:
        assert np.asarray(a[key]).tobytes() == np.asarray(b[key]).tobytes(), key


def test_failure_stops_at_its_grid_index(oracle):
    sys = StandardMap(1.0)
    x0 = np.array([[0.3, 0.2], [0.5, 1e308], [1.0, 0.5]])
    grid = [2, 4, 8]
    rec = oracle.oracle_indicators(sys, x0, 8, 2, ["MEGNO", "SALI"], grid)
    assert rec["fail"].tolist() == [0, 1, 0]
    assert rec["code"][1] != 0 and rec["code"][0] == 0 and rec["code"][2] == 0
    assert np.all(rec["R"][1] == 0)            # no row of the failed orbit was written
    ok = oracle.oracle_indicators(sys, x0[[0, 2]], 8, 2, ["MEGNO", "SALI"], grid)
    assert rec["R"][[0, 2]].tobytes() == ok["R"].tobytes()


def test_member_columns_names():
    assert sum(len(MEMBER_COLUMNS[m]) for m in ["FLI", "MEGNO", "SALI"]) == 10
    with pytest.raises(ValueError):
        indicator_chain(["RLI"])
    forms = [getattr(r, "replaces", True) for r in indicator_chain(["FLI", "MEGNO", "SALI"])]
    assert forms == [False, False, True]


def test_chain_outside_the_menu_is_refused_before_any_launch():
    from chaos_b200 import record_indicators
    sys, x0 = _system("standard", 4)
    with pytest.raises(ValueError, match="outside the compiled menu"):
        record_indicators(sys, x0, 10, 1, ["SALI", "SALI"], [10])
    with pytest.raises(ValueError):
        record_indicators(sys, x0, 10, 2, ["MEGNO"], [3])      # grid not a multiple of tau
