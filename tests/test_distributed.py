"""Multi-rank host logic on the CPU (gloo, world size 2): orbit shards, global orbit ids and the gather of records
that `bench.py --gpus N` and multi-GPU callers use. No GPU: each rank stands in for its device run with the oracle
(the same per-orbit records a device shard returns)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from chaos_b200.distributed import gather_records, lowest_failure, shard


def test_shards_partition():
    for n in (0, 1, 7, 64, 1001):
        for w in (1, 2, 3, 8):
            parts = [shard(n, r, w) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle"), os.path.join(root, "tests")]
    import oracle as O
    from chaos_b200 import QRSpectrum, MGS, StandardMap
    from chaos_b200.propagate import FrameSpec
    from helpers import haar_frames, uniform_starts
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 101
        x0 = uniform_starts(n, 2, 3)
        x0[57, 1] = np.nan   # orbit 58 fails; it lives on rank 1
        W0 = haar_frames(n, 2, 2, 4)
        lo, hi = shard(n, rank, world)
        r = O.oracle_frames(StandardMap(2.0), x0[lo:hi], 200, [FrameSpec(2, (QRSpectrum(MGS()),), W0[lo:hi])], tau=5,
                            orbit_base=lo)[0]
        full = gather_records(dict(x=r["x"], W=r["W"], code=r["code"], hstep=r["hstep"]), n, rank, world)
        if rank == 0:
            one = O.oracle_frames(StandardMap(2.0), x0, 200, [FrameSpec(2, (QRSpectrum(MGS()),), W0)], tau=5)[0]
            same = all(np.array_equal(np.nan_to_num(full[k]), np.nan_to_num(one[k])) for k in ("x", "W", "code", "hstep"))
            q.put((same, lowest_failure(full["code"])))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_matches_one_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    same, low = q.get(timeout=5)
    assert same
    assert low == 57
