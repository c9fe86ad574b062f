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


def test_pinned_host_buffers_give_the_same_bits():
    """The host-buffer call with page-locked arrays (whose copies to the device run asynchronously, so the library
    must not touch them while in flight) gives the bits of the same call on pageable arrays."""
    import ctypes as C
    import torch
    from chaos_b200 import _abi
    from chaos_b200._lib import last_error, lib
    from chaos_b200.propagate import build_run
    n, N = 4096, 400
    sysm = FroeschleMap(1.5, 1.5, 0.05)
    frames = [FrameSpec(4, (QRSpectrum(HouseholderQR()),))]
    r = build_run(sysm, N, 10, frames, "fp64", 0)
    sb = lib().cl_b200_state_bytes(C.byref(r), 0)
    x0 = np.random.default_rng(9).uniform(0, 2 * np.pi, (n, 4))
    W0 = np.ascontiguousarray(np.broadcast_to(np.eye(4), (n, 4, 4)))

    def call(pinned):
        def arr(shape, dtype, init=None):
            t = torch.empty(shape, dtype=dtype, pin_memory=pinned)
            a = t.numpy()
            if init is not None:
                a[...] = init
            return t, a
        keep = [arr((n, 4), torch.float64, x0), arr((n, 4, 4), torch.float64, W0), arr((n, 4), torch.float64),
                arr((n, 16), torch.float64), arr((n * sb,), torch.uint8), arr((n,), torch.int8), arr((n,), torch.int64)]
        b = _abi.cl_buffers()
        b.x0, b.W0[0], b.x, b.W[0] = (keep[i][1].ctypes.data for i in range(4))
        b.states[0], b.code[0], b.hstep[0] = (keep[i][1].ctypes.data for i in range(4, 7))
        prov = _abi.cl_prov()
        assert lib().cl_b200_propagate(C.byref(r), n, C.byref(b), C.byref(prov)) == 0, last_error()
        return [k[1].copy() for k in keep[2:]]
    a, b = call(False), call(True)
    for u, v in zip(a, b):
        assert same_bits(u, v) if u.dtype.kind == "f" else np.array_equal(u, v)
