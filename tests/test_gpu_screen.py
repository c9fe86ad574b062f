"""The learned screen end to end on the B200 (small sizes): features from the first 2000 steps, the network trained
on the GPU by the library's tensor-core kernels on the coupled-maps ensemble (coordinates uniform in [0, 2 pi)^4,
Float64 labels), the screened grid against the plain full integration in Float64. It shows what the network gains:
the same classification (at most 1 % of the grid differs) from at most a fifth of the orbit-steps, at the full
horizon N = 1e5. The mixed kernels' MEGNO class agrees with the Float64 class on the grid."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_screen_small_grid():
    torch = pytest.importorskip("torch")
    from chaos_b200.screen import Screen
    dev = torch.device("cuda", 0)
    from chaos_b200.screen import N_FULL
    N = N_FULL
    sc = Screen(torch, dev)
    assert sc.precision == "fp64"
    X, label, lam = sc.training_set(24_576, N=N)
    assert 0.005 < label.mean() < 0.995          # both classes present
    net, info = sc.train(X, label, lam, epochs=10, batch=2048)
    assert info["val_accuracy"] > 0.9, info
    G = 96
    res = sc.screen_grid(net, G, N=N)
    plain, _ = sc.full_grid(G, N=N)
    mis = float((res["labels"] != plain).mean())
    gain = res["full_orbit_steps"] / res["orbit_steps"]
    assert mis <= 0.01, (mis, res["unsure"])
    assert gain >= 5.0, gain


def test_mixed_megno_class_agrees():
    """The same grid integrated in full by the mixed kernels: the MEGNO class (final Ybar > 2.2) equals the Float64
    class on at least 99 % of the orbits."""
    torch = pytest.importorskip("torch")
    from chaos_b200.screen import Screen
    dev = torch.device("cuda", 0)
    G, N = 96, 20_000
    a, _ = Screen(torch, dev, precision="fp64").full_grid(G, N=N)
    b, _ = Screen(torch, dev, precision="mixed").full_grid(G, N=N)
    assert float((a == b).mean()) >= 0.99
