"""The batched uneven ensemble on the B200 against the oracle, bit for bit (FP64 classes): per-orbit K, per-orbit
lengths, the escape stop, the work-queue order, every tuned kernel variant and the CUDA-graph replay."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from chaos_b200 import HouseholderQR, QRSpectrum, StandardMap, StandardMapChain
from chaos_b200._lib import lib
from chaos_b200.ensemble import EnsembleClass, make_class_struct, propagate_ensemble
from chaos_b200.propagate import FrameSpec
from helpers import same_bits, states_equal, uniform_starts

pytestmark = pytest.mark.gpu


def _class(d, n, tau, seed, precision="fp64", escape=1e3, nmax=4000):
    rng = np.random.default_rng(seed)
    k = min(d, 8)
    sysm = StandardMap(1.0) if d == 2 else StandardMapChain(d // 2, 1.0, 0.05)
    x0 = uniform_starts(n, d, seed)
    K = rng.uniform(0.5, 3.0, n)
    L = np.maximum(tau, (np.exp(rng.uniform(np.log(50), np.log(nmax), n)) // tau).astype(np.int64) * tau)
    W0 = np.broadcast_to(np.eye(d)[:, :k], (n, d, k)).copy()
    return EnsembleClass(sysm, x0, FrameSpec(k, (QRSpectrum(HouseholderQR()),), W0), tau, int(nmax // tau * tau), K=K,
                         lengths=L, escape=escape, precision=precision)


def _oracle(oracle, c):
    return oracle.oracle_ensemble(c.sys, c.x0, c.N, c.frame, tau=c.tau, K=c.K, lengths=c.lengths, escape=c.escape)


@pytest.mark.parametrize("d,tau", [(2, 5), (4, 10), (8, 10), (16, 20)])
@pytest.mark.parametrize("escape", [1e3, 25.0])
def test_ensemble_class_bitwise(oracle, d, tau, escape):
    c = _class(d, 300, tau, 100 + d, escape=escape)
    dev = propagate_ensemble([c])[0]
    ref = _oracle(oracle, c)
    assert np.array_equal(dev.code, ref["code"]) and np.array_equal(dev.hstep, ref["hstep"])
    assert same_bits(dev.x, ref["x"]) and same_bits(dev.W, ref["W"]) and states_equal(dev.states, ref["states"])
    if escape == 25.0 and d == 2:
        assert (dev.code == 4).any()   # a low bound: some standard-map orbits escape within a few thousand steps


def test_ensemble_all_classes_concurrently(oracle):
    cs = [_class(d, 200, tau, 7 + d) for d, tau in [(2, 5), (4, 10), (8, 10), (16, 20)]]
    devs = propagate_ensemble(cs)
    for c, dev in zip(cs, devs):
        ref = _oracle(oracle, c)
        assert same_bits(dev.W, ref["W"]) and states_equal(dev.states, ref["states"])


@pytest.mark.parametrize("minb", [1, 2, 4])
@pytest.mark.parametrize("unroll", [1, 10])
def test_every_variant_same_bits(oracle, minb, unroll):
    c = _class(4, 257, 10, 55)
    c.minb, c.unroll = minb, unroll
    dev = propagate_ensemble([c])[0]
    ref = _oracle(oracle, c)
    assert same_bits(dev.W, ref["W"]) and states_equal(dev.states, ref["states"])


def test_mixed_ensemble_close_to_fp64():
    c64 = _class(8, 512, 10, 77, nmax=3000)
    cmx = _class(8, 512, 10, 77, precision="mixed", nmax=3000)
    a, b = propagate_ensemble([c64])[0], propagate_ensemble([cmx])[0]
    ok = (a.code == 0) & (b.code == 0)
    n = a.states["r0"]["n"][ok]
    l64 = (a.states["r0"]["sums"][ok, 0, 0] + a.states["r0"]["sums"][ok, 0, 1]) / n
    lmx = (b.states["r0"]["sums"][ok, 0, 0] + b.states["r0"]["sums"][ok, 0, 1]) / n
    assert np.max(np.abs(l64 - lmx)) <= 1e-3


def test_graph_replay_and_tuner(oracle):
    """cl_b200_ensemble_tune picks a variant; a captured CUDA graph replays the ensemble with the same bits."""
    import torch
    c = _class(4, 300, 10, 91)
    ref = _oracle(oracle, c)
    keep = []
    cs = make_class_struct(c, keep)
    dev = torch.device("cuda", 0)
    n, s, dk = c.x0.shape[0], c.sys.s, c.sys.d * c.frame.k
    t = dict(x0=torch.tensor(np.ascontiguousarray(c.x0), device=dev), x=torch.empty((n, s), dtype=torch.float64, device=dev),
             W0=torch.tensor(np.ascontiguousarray(c.frame.W0.transpose(0, 2, 1)), device=dev),
             W=torch.empty((n, dk), dtype=torch.float64, device=dev),
             st=torch.empty(n * keep[5]["states"].dtype.itemsize // 8, dtype=torch.int64, device=dev),
             code=torch.empty(n, dtype=torch.int8, device=dev), hs=torch.empty(n, dtype=torch.int64, device=dev),
             order=torch.tensor(keep[3], device=dev), K=torch.tensor(keep[4], device=dev),
             N=torch.tensor(keep[2], device=dev))
    cs.buf.x0, cs.buf.x = t["x0"].data_ptr(), t["x"].data_ptr()
    cs.buf.W0[0], cs.buf.W[0] = t["W0"].data_ptr(), t["W"].data_ptr()
    cs.buf.states[0], cs.buf.code[0], cs.buf.hstep[0] = t["st"].data_ptr(), t["code"].data_ptr(), t["hs"].data_ptr()
    cs.order, cs.K, cs.N = t["order"].data_ptr(), t["K"].data_ptr(), t["N"].data_ptr()
    L = lib()
    stream = torch.cuda.current_stream(dev).cuda_stream
    assert L.cl_b200_ensemble_tune(C.byref(cs), 256, 200, C.c_void_p(stream)) == 0
    assert cs.minb in (1, 2, 4) and cs.unroll in (1, 10)
    arr = (type(cs) * 1)(cs)
    g = C.c_void_p()
    assert L.cl_b200_ensemble_graph_create(arr, 1, C.byref(g)) == 0
    try:
        for _ in range(2):
            assert L.cl_b200_ensemble_graph_launch(g, C.c_void_p(stream)) == 0
            torch.cuda.synchronize(dev)
            W = t["W"].cpu().numpy().reshape(n, c.frame.k, c.sys.d).transpose(0, 2, 1)
            assert same_bits(W, ref["W"])
            assert np.array_equal(t["code"].cpu().numpy(), ref["code"])
    finally:
        L.cl_b200_ensemble_graph_destroy(g)
