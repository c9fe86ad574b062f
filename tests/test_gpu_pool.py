"""The device pool of the host-buffer entry points: a second call of the same sizes allocates nothing from the
driver and gives the same bits, the probe counts the pool's idle memory as free, and `release_cache` returns it."""
from __future__ import annotations

import numpy as np
import pytest

from chaos_b200 import FroeschleMap, GALI, HouseholderQR, QRSpectrum, SALI, probe, propagate_frames, release_cache
from chaos_b200.propagate import FrameSpec
from helpers import same_bits, states_equal

pytestmark = pytest.mark.gpu


def test_pool_keeps_memory_between_calls():
    import torch
    n = 1 << 16
    x0 = np.random.default_rng(3).uniform(0, 2 * np.pi, (n, 4))
    W0 = np.broadcast_to(np.eye(4), (n, 4, 4)).copy()
    frames = [FrameSpec(4, (QRSpectrum(HouseholderQR()),), W0), FrameSpec(4, (GALI(), SALI()), W0)]
    sysm = FroeschleMap(1.5, 1.5, 0.05)
    release_cache()
    free0, _ = torch.cuda.mem_get_info()
    a = propagate_frames(sysm, x0, 200, frames, tau=10, finals=False, throw=False)
    free1, _ = torch.cuda.mem_get_info()
    b = propagate_frames(sysm, x0, 200, frames, tau=10, finals=False, throw=False)
    free2, _ = torch.cuda.mem_get_info()
    buffers = n * (8 * 4 + 2 * (8 * 16 + 8 * 16 + 1 + 8))   # x, W0 and W per frame, code, hstep (states on top)
    assert free0 - free1 >= buffers            # the first call's buffers stay in the pool
    assert abs(free2 - free1) < buffers // 10  # the second call takes them from the pool
    for f in range(2):
        assert same_bits(a[f].x, b[f].x) and same_bits(a[f].W, b[f].W) and states_equal(a[f].states, b[f].states)
    idle = probe()["free_bytes"] - torch.cuda.mem_get_info()[0]
    assert idle >= buffers                     # the probe counts the pool's idle memory as free
    release_cache()
    free3, _ = torch.cuda.mem_get_info()
    assert free3 - free2 >= buffers
