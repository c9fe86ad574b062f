"""The learned screen end to end on the B200 (small sizes): features from the first 2000 steps, the network trained
on the GPU by the library's tensor-core kernels, the screened grid against the plain full integration. It shows
what the network gains: the same classification from a fraction of the orbit-steps."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_screen_small_grid():
    torch = pytest.importorskip("torch")
    from chaos_b200.screen import Screen
    dev = torch.device("cuda", 0)
    N = 20_000
    sc = Screen(torch, dev)
    X, label, lam = sc.training_set(24_576, N=N)
    assert 0.05 < label.mean() < 0.95          # both classes present
    net, info = sc.train(X, label, lam, epochs=10, batch=2048)
    assert info["val_accuracy"] > 0.9, info
    G = 96
    res = sc.screen_grid(net, G, N=N)
    plain, _ = sc.full_grid(G, N=N)
    agree = float((res["labels"] == plain).mean())
    gain = res["full_orbit_steps"] / res["orbit_steps"]
    assert agree >= 0.99, (agree, res["unsure"])
    assert gain > 2.0, gain
