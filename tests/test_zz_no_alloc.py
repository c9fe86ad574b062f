"""The ensemble entry point that allocates nothing (`cl_b200_ensemble_device_noalloc`), for callers that cannot
allocate GPU memory while they call in: its queue heads live in a fixed array inside the library instead of a
buffer it would allocate. Called twice in a row through the C ABI, it must give bit for bit what the allocating
entry point (`cl_b200_ensemble_device`) gives on the same classes -- the tolerance of every FP64 test here.

This file is collected last, so a run that stops at the first failure has run every other test before it; it
also passes on its own in a fresh process (the first call sets the fixed array up)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from chaos_b200 import _abi
from chaos_b200._lib import last_error, lib
from chaos_b200.ensemble import EnsembleClass, make_class_struct
from chaos_b200 import HouseholderQR, QRSpectrum, StandardMap, StandardMapChain
from chaos_b200.propagate import FrameSpec

pytestmark = pytest.mark.gpu


def _classes():
    out = []
    for d, tau, seed in ((2, 5, 3), (8, 10, 4)):
        rng = np.random.default_rng(seed)
        n, k = 700, min(d, 8)
        sysm = StandardMap(1.0) if d == 2 else StandardMapChain(d // 2, 1.0, 0.05)
        x0 = rng.uniform(0, 2 * np.pi, (n, d))
        K = rng.uniform(0.5, 3.0, n)
        L = np.maximum(tau, (np.exp(rng.uniform(np.log(50), np.log(3000), n)) // tau).astype(np.int64) * tau)
        W0 = np.broadcast_to(np.eye(d)[:, :k], (n, d, k)).copy()
        out.append(EnsembleClass(sysm, x0, FrameSpec(k, (QRSpectrum(HouseholderQR()),), W0), tau, 3000 // tau * tau,
                                 K=K, lengths=L, escape=25.0, precision="fp64"))
    return out


def _on_device(classes, torch, dev):
    """Class structs whose buffers are device tensors (kept alive in the returned list)."""
    keep, structs, outs = [], [], []
    for c in classes:
        host_keep = []
        cs = make_class_struct(c, host_keep)
        n, s, dk = len(c.x0), c.sys.s, c.sys.d * c.frame.k
        sb = host_keep[5]["states"].dtype.itemsize
        t = dict(x0=torch.tensor(np.ascontiguousarray(c.x0), device=dev),
                 x=torch.zeros((n, s), dtype=torch.float64, device=dev),
                 W0=torch.tensor(np.ascontiguousarray(c.frame.W0.transpose(0, 2, 1)), device=dev),
                 W=torch.zeros((n, dk), dtype=torch.float64, device=dev),
                 st=torch.zeros(n * sb // 8, dtype=torch.int64, device=dev),
                 code=torch.zeros(n, dtype=torch.int8, device=dev),
                 hs=torch.zeros(n, dtype=torch.int64, device=dev),
                 order=torch.tensor(host_keep[3], device=dev), K=torch.tensor(host_keep[4], device=dev),
                 N=torch.tensor(host_keep[2], device=dev))
        cs.buf.x0, cs.buf.x = t["x0"].data_ptr(), t["x"].data_ptr()
        cs.buf.W0[0], cs.buf.W[0] = t["W0"].data_ptr(), t["W"].data_ptr()
        cs.buf.states[0], cs.buf.code[0], cs.buf.hstep[0] = t["st"].data_ptr(), t["code"].data_ptr(), t["hs"].data_ptr()
        cs.order, cs.K, cs.N = t["order"].data_ptr(), t["K"].data_ptr(), t["N"].data_ptr()
        keep.append((host_keep, t))
        structs.append(cs)
        outs.append(t)
    arr = (_abi.cl_ensemble_class * len(structs))(*structs)
    return arr, outs, keep


def _records(outs):
    return [{k: outs[i][k].cpu().numpy().copy() for k in ("x", "W", "st", "code", "hs")} for i in range(len(outs))]


def test_noalloc_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    L = lib()
    classes = _classes()

    arr, outs, keep = _on_device(classes, torch, dev)
    assert L.cl_b200_ensemble_device(arr, len(classes), C.c_void_p(stream)) == 0, last_error()
    torch.cuda.synchronize(dev)
    want = _records(outs)
    assert any((w["code"] == 4).any() for w in want)     # the escape stop is exercised

    for call in range(2):   # two calls in a row on fresh output buffers: same bits each time
        arr2, outs2, keep2 = _on_device(classes, torch, dev)
        rc = L.cl_b200_ensemble_device_noalloc(arr2, len(classes), C.c_void_p(stream))
        assert rc == 0, last_error()
        torch.cuda.synchronize(dev)
        got = _records(outs2)
        for w, g in zip(want, got):
            for k in w:
                assert np.array_equal(w[k].view(np.uint8), g[k].view(np.uint8)), (call, k)


def test_noalloc_rejects_too_many_classes():
    torch = pytest.importorskip("torch")
    L = lib()
    arr = (_abi.cl_ensemble_class * (_abi.NOALLOC_MAX_CLASSES + 1))()
    rc = L.cl_b200_ensemble_device_noalloc(arr, _abi.NOALLOC_MAX_CLASSES + 1, None)
    assert rc == _abi.EINVAL and "at most 64 classes" in last_error()


def test_noalloc_captures_into_a_graph_of_memsets_and_kernels():
    """The call captured on a stream in global capture mode (where an allocation call from any thread would end the
    capture with an error) gives a graph whose nodes are memsets and kernels only -- no allocation node -- and the
    graph, replayed, gives the allocating entry point's bits."""
    torch = pytest.importorskip("torch")
    rt = pytest.importorskip("cuda.bindings.runtime")
    dev = torch.device("cuda", 0)
    L = lib()
    classes = _classes()
    arr, outs, keep = _on_device(classes, torch, dev)
    assert L.cl_b200_ensemble_device(arr, len(classes), C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)) == 0
    torch.cuda.synchronize(dev)
    want = _records(outs)

    arr2, outs2, keep2 = _on_device(classes, torch, dev)
    torch.cuda.synchronize(dev)
    err, s = rt.cudaStreamCreate()
    assert err == rt.cudaError_t.cudaSuccess
    graph = gexec = None
    try:
        err, = rt.cudaStreamBeginCapture(s, rt.cudaStreamCaptureMode.cudaStreamCaptureModeGlobal)
        assert err == rt.cudaError_t.cudaSuccess
        rc = L.cl_b200_ensemble_device_noalloc(arr2, len(classes), C.c_void_p(int(s)))
        err, graph = rt.cudaStreamEndCapture(s)
        assert rc == 0, last_error()
        assert err == rt.cudaError_t.cudaSuccess
        err, _, count = rt.cudaGraphGetNodes(graph, 0)
        err, nodes, count = rt.cudaGraphGetNodes(graph, count)
        assert err == rt.cudaError_t.cudaSuccess and count >= 2
        kinds = {rt.cudaGraphNodeGetType(nd)[1] for nd in nodes[:count]}
        assert kinds <= {rt.cudaGraphNodeType.cudaGraphNodeTypeKernel, rt.cudaGraphNodeType.cudaGraphNodeTypeMemset}, kinds
        assert rt.cudaGraphNodeType.cudaGraphNodeTypeKernel in kinds
        err, gexec = rt.cudaGraphInstantiate(graph, 0)
        assert err == rt.cudaError_t.cudaSuccess
        assert rt.cudaGraphLaunch(gexec, s)[0] == rt.cudaError_t.cudaSuccess
        assert rt.cudaStreamSynchronize(s)[0] == rt.cudaError_t.cudaSuccess
    finally:
        if gexec is not None:
            rt.cudaGraphExecDestroy(gexec)
        if graph is not None:
            rt.cudaGraphDestroy(graph)
        rt.cudaStreamDestroy(s)
    got = _records(outs2)
    for w, g in zip(want, got):
        for k in w:
            assert np.array_equal(w[k].view(np.uint8), g[k].view(np.uint8)), k
