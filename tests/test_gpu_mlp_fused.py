"""The screen network's fused inference pass (one persistent tcgen05 kernel, cl_b200_mlp_forward_fused) against the
per-layer GEMM chain -- bit for bit, the same MMAs in the same order and the same epilogue arithmetic -- and against
the CPU oracle (oracle/mlp_oracle.py); the weight packing against a numpy restatement of the MMA layout."""
from __future__ import annotations

import numpy as np
import pytest

import mlp_oracle as MO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_dev():
    torch = pytest.importorskip("torch")
    return torch, torch.device("cuda", 0)


def _pack_numpy(W, R):
    """Tiles of R rows x 64 columns, K-major core matrices of 8 rows x 8 columns: element (r, k) of tile (rt, kb) at
    element offset (rt * nkb + kb) * R * 64 + ((r // 8) * 8 + k // 8) * 64 + (r % 8) * 8 + k % 8."""
    rows, cols = W.shape
    nrt, nkb = -(-rows // R), -(-cols // 64)
    P = np.zeros((nrt * R, nkb * 64), W.dtype)
    P[:rows, :cols] = W
    out = np.zeros(nrt * nkb * R * 64, W.dtype)
    r, k = np.meshgrid(np.arange(nrt * R), np.arange(nkb * 64), indexing="ij")
    rt, rr, kb, kk = r // R, r % R, k // 64, k % 64
    off = (rt * nkb + kb) * R * 64 + ((rr // 8) * 8 + kk // 8) * 64 + (rr % 8) * 8 + kk % 8
    out[off.ravel()] = P.ravel()
    return out


@pytest.mark.parametrize("rows,cols,ld,R", [(256, 256, 256, 256), (16, 256, 256, 16), (300, 200, 208, 16),
                                            (131, 64, 64, 128)])
def test_pack_layout(torch_dev, rows, cols, ld, R):
    torch, dev = torch_dev
    from chaos_b200._lib import lib
    from chaos_b200.mlp import _declare
    L = _declare(lib())
    rng = np.random.default_rng(rows + cols)
    W = rng.standard_normal((rows, ld)).astype(np.float32)
    Wt = torch.tensor(W, device=dev).to(torch.bfloat16)
    nrt, nkb = -(-rows // R), -(-cols // 64)
    dst = torch.full((nrt * R * nkb * 64,), 7.0, dtype=torch.bfloat16, device=dev)
    rc = L.cl_b200_mlp_pack_kmajor(Wt.data_ptr(), rows, cols, ld, R, dst.data_ptr(),
                                   torch.cuda.current_stream(dev).cuda_stream)
    assert rc == 0
    want = _pack_numpy(Wt.float().cpu().numpy()[:, :cols], R)
    assert np.array_equal(dst.float().cpu().numpy(), want)


def _net(torch, dev, seed):
    from chaos_b200.mlp import MLP
    net = MLP(torch, dev, seed=seed)
    rng = np.random.default_rng(seed + 100)
    for lay in net.layers:
        lay["b"].copy_(torch.tensor(rng.standard_normal(lay["b"].numel()).astype(np.float32) * 0.3, device=dev))
    return net


@pytest.mark.parametrize("B", [1, 127, 128, 1000, 148 * 128 + 77, 65536 + 300])
def test_fused_equals_layered(torch_dev, B):
    """Every output bit equal to the per-layer chain (ragged last tile, fewer tiles than SMs, several tiles per CTA)."""
    torch, dev = torch_dev
    from chaos_b200._lib import lib
    from chaos_b200.mlp import _declare
    net = _net(torch, dev, 3)
    rng = np.random.default_rng(B)
    X = torch.tensor(rng.standard_normal((B, 64)).astype(np.float32) * 0.7, device=dev).to(torch.bfloat16)
    a = net.forward(X)
    b = net.forward_fused(X)
    torch.cuda.synchronize(dev)
    assert _declare(lib()).cl_b200_mlp_status() == 0
    assert torch.equal(a, b), float((a - b).abs().max())


def test_fused_persistent_tiles(torch_dev):
    """A grid capped at 3 CTAs walks 40 tiles each (the rings' phases wrap many times): the same bits as one tile per
    CTA."""
    torch, dev = torch_dev
    net = _net(torch, dev, 5)
    rng = np.random.default_rng(2)
    B = 120 * 128 - 5
    X = torch.tensor(rng.standard_normal((B, 64)).astype(np.float32), device=dev).to(torch.bfloat16)
    a = net.forward_fused(X)
    b = net.forward_fused(X, max_ctas=3)
    c = net.forward_fused(X, max_ctas=1)
    torch.cuda.synchronize(dev)
    assert torch.equal(a, b) and torch.equal(a, c)


def test_fused_matches_oracle(torch_dev):
    """Against the oracle (BF16 operands rounded as the device rounds them, everything else FP64): outputs within
    2e-3 of their scale -- FP32 accumulation order and the activation's special-function rounding (relative 1e-6)
    can move a BF16 rounding of an activation by one unit."""
    torch, dev = torch_dev
    net = _net(torch, dev, 7)
    rng = np.random.default_rng(4)
    B = 1000
    X = rng.standard_normal((B, 64)).astype(np.float32)
    out = net.forward_fused(torch.tensor(X, device=dev).to(torch.bfloat16)).cpu().numpy()
    want, _, _ = MO.forward(net.weights_numpy(), X)
    scale = np.max(np.abs(want))
    assert np.max(np.abs(out - want)) <= 2e-3 * scale


def test_fused_rejects_bad_arguments(torch_dev):
    torch, dev = torch_dev
    from chaos_b200._lib import lib
    from chaos_b200.mlp import _declare
    L = _declare(lib())
    net = _net(torch, dev, 1)
    P = net.packed()
    X = torch.zeros((128, 64), dtype=torch.bfloat16, device=dev)
    out = torch.empty((128, 16), dtype=torch.float32, device=dev)
    b = [lay["b"].data_ptr() for lay in net.layers]
    before = L.cl_b200_launch_count()
    assert L.cl_b200_mlp_forward_fused(X.data_ptr() + 2, 128, *[p.data_ptr() for p in P], *b, out.data_ptr(), 0,
                                       None) != 0
    assert L.cl_b200_mlp_forward_fused(X.data_ptr(), 0, *[p.data_ptr() for p in P], *b, out.data_ptr(), 0, None) != 0
    assert L.cl_b200_launch_count() == before


def test_fused_from_host_memory(torch_dev):
    """The host-data call (chunks over two streams, copies overlapping the passes) gives the device pass's outputs bit
    for bit, with a ragged last chunk."""
    torch, dev = torch_dev
    net = _net(torch, dev, 9)
    rng = np.random.default_rng(6)
    B = 3 * 4096 + 777
    X = torch.tensor(rng.standard_normal((B, 64)).astype(np.float32), device=dev).to(torch.bfloat16)
    want = net.forward_fused(X)
    Xh = X.cpu().pin_memory()
    oh = torch.full((B, 16), 7.0, dtype=torch.float32).pin_memory()
    net.forward_fused_host(Xh, oh, chunk_rows=4096)
    torch.cuda.synchronize(dev)
    assert torch.equal(oh, want.cpu())
