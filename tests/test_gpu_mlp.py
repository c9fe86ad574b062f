"""The learned screen's tensor-core kernels against the CPU oracle (oracle/mlp_oracle.py): the tcgen05 GEMM on
BF16 operands with FP32 accumulation, the forward pass and every gradient of the backward pass."""
from __future__ import annotations

import numpy as np
import pytest

import mlp_oracle as MO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_dev():
    torch = pytest.importorskip("torch")
    return torch, torch.device("cuda", 0)


@pytest.mark.parametrize("M,N,K,gelu,bias", [(256, 256, 64, False, False), (384, 16, 256, True, True),
                                             (128, 256, 296, True, True), (200, 64, 40, False, True),
                                             (1024, 128, 256, False, False)])
def test_gemm_matches_fp64(torch_dev, M, N, K, gelu, bias):
    torch, dev = torch_dev
    from chaos_b200.mlp import gemm
    rng = np.random.default_rng(M + N + K)
    A = MO.bf16_round(rng.standard_normal((M, K)))
    B = MO.bf16_round(rng.standard_normal((N, K)))
    b = rng.standard_normal(N).astype(np.float32) if bias else None
    At = torch.tensor(A.astype(np.float32), device=dev).to(torch.bfloat16)
    Bt = torch.tensor(B.astype(np.float32), device=dev).to(torch.bfloat16)
    bt = None if b is None else torch.tensor(b, device=dev)
    C32 = torch.empty((M, N), dtype=torch.float32, device=dev)
    pre = torch.empty((M, N), dtype=torch.float32, device=dev)
    gemm(At, Bt, M, N, K, bias=bt, gelu=gelu, C32=C32, pre=pre, stream=torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize(dev)
    Z = A @ B.T + (0 if b is None else b.astype(np.float64))
    want = MO.gelu(Z) if gelu else Z
    scale = np.max(np.abs(Z))
    assert np.max(np.abs(pre.cpu().numpy() - Z)) <= 2e-5 * scale
    assert np.max(np.abs(C32.cpu().numpy() - want)) <= 2e-5 * scale


@pytest.mark.parametrize("M,N,K,accumulate", [(256, 64, 8192, False), (16, 256, 4096, True), (256, 256, 20000, False)])
def test_gemm_split_k_matches_fp64(torch_dev, M, N, K, accumulate):
    """Weight-gradient shapes (few output tiles, K = the batch): K is split over CTAs whose partial tiles are added
    into the FP32 result (zeroed first, or added to C when accumulating)."""
    torch, dev = torch_dev
    from chaos_b200.mlp import gemm
    rng = np.random.default_rng(M * 7 + K)
    A = MO.bf16_round(rng.standard_normal((M, K)))
    B = MO.bf16_round(rng.standard_normal((N, K)))
    C0 = rng.standard_normal((M, N)).astype(np.float32)
    At = torch.tensor(A.astype(np.float32), device=dev).to(torch.bfloat16)
    Bt = torch.tensor(B.astype(np.float32), device=dev).to(torch.bfloat16)
    C32 = torch.tensor(C0, device=dev) if accumulate else torch.full((M, N), 7.0, dtype=torch.float32, device=dev)
    gemm(At, Bt, M, N, K, C32=C32, accumulate=accumulate, stream=torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize(dev)
    Z = A @ B.T + (C0.astype(np.float64) if accumulate else 0.0)
    scale = np.max(np.abs(A @ B.T))
    assert np.max(np.abs(C32.cpu().numpy() - Z)) <= 2e-5 * scale


def test_forward_backward_match_oracle(torch_dev):
    torch, dev = torch_dev
    from chaos_b200.mlp import MLP
    rng = np.random.default_rng(5)
    B = 256
    net = MLP(torch, dev, seed=3)
    X = rng.standard_normal((B, 64)).astype(np.float32) * 0.5
    label = (rng.random(B) < 0.4).astype(np.float32)
    target = rng.standard_normal(B).astype(np.float32) * 0.2
    Xb = torch.tensor(X, device=dev).to(torch.bfloat16)
    out = net.forward(Xb, keep=True)
    rl, g32, gb = net.loss_and_grad(out, torch.tensor(label, device=dev), torch.tensor(target, device=dev), 1.0)
    net.backward(g32, gb)
    torch.cuda.synchronize(dev)
    W = net.weights_numpy()
    o_out, pres, acts = MO.forward(W, X)
    o_loss, o_g = MO.head(o_out, label, target, 1.0)
    grads = MO.backward(W, pres, acts, o_g)
    rel = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))  # noqa: E731
    assert rel(out.cpu().numpy()[:, :2], o_out[:, :2]) <= 1e-2
    assert rel(rl.cpu().numpy(), o_loss) <= 1e-2
    for li, lay in enumerate(net.layers):
        assert rel(lay["gW"].cpu().numpy(), grads[li][0]) <= 2e-2, li
        assert rel(lay["gb"].cpu().numpy(), grads[li][1]) <= 2e-2, li


def test_training_reduces_loss(torch_dev):
    torch, dev = torch_dev
    from chaos_b200.mlp import MLP
    rng = np.random.default_rng(9)
    B = 1024
    X = rng.standard_normal((B, 64)).astype(np.float32)
    w = rng.standard_normal(64)
    label = (X @ w > 0).astype(np.float32)
    target = (0.1 * np.tanh(X[:, :4].sum(axis=1))).astype(np.float32)
    net = MLP(torch, dev, seed=1)
    Xb = torch.tensor(X, device=dev).to(torch.bfloat16)
    lt, tt = torch.tensor(label, device=dev), torch.tensor(target, device=dev)
    first = None
    for it in range(200):
        rl = net.train_step(Xb, lt, tt, w_reg=1.0, lr=2e-3)
        if it == 0:
            first = float(rl.mean().item())
    last = float(rl.mean().item())
    out = net.predict(Xb)
    acc = float(((out[:, 0].cpu().numpy() > 0) == (label > 0.5)).mean())
    assert last < 0.3 * first and acc > 0.95
