"""Orbit sharding across ranks (one process per GPU) and the host-side gather of the per-orbit records.

Orbits are independent (src/Tangent/propagate.jl:32-50 runs one work item per orbit with no exchange), so N GPUs
run N disjoint contiguous shards of the orbit ids with no collective in the data path; the only communication is
the final gather of records (and, in the bench, a barrier and the max over ranks of the device time). Orbit ids stay
global (`orbit_base`), so seeded frames and error records are the same as in a one-GPU run, and the error raised
is that of the lowest failing orbit id over all shards, as in the reference (propagate.jl:111-113).
"""
from __future__ import annotations

import numpy as np


def shard(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous balanced shard [lo, hi) of n orbits for `rank` of `world` (sizes differ by at most one)."""
    if not (0 <= rank < world):
        raise ValueError("rank outside the world")
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def gather_records(records: dict, n: int, rank: int, world: int, group=None) -> dict | None:
    """Gather each rank's per-orbit arrays (keys -> arrays with the shard's orbits on axis 0) to rank 0 and
    concatenate them in orbit order; returns the full dict on rank 0, None elsewhere. Uses torch.distributed
    object collectives (any backend: gloo on CPU, NCCL on GPUs)."""
    import torch.distributed as dist
    lo, hi = shard(n, rank, world)
    payload = (lo, hi, {k: np.asarray(v) for k, v in records.items()})
    out = [None] * world if rank == 0 else None
    dist.gather_object(payload, out, dst=0, group=group)
    if rank != 0:
        return None
    out.sort(key=lambda t: t[0])
    assert out[0][0] == 0 and out[-1][1] == n and all(a[1] == b[0] for a, b in zip(out, out[1:]))
    return {k: np.concatenate([p[2][k] for p in out], axis=0) for k in records}


def lowest_failure(codes: np.ndarray) -> int | None:
    """0-based id of the lowest orbit whose code is not 0 (None if every orbit finished)."""
    bad = np.flatnonzero(np.asarray(codes) != 0)
    return int(bad[0]) if bad.size else None
