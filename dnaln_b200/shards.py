"""Read-sharded mapping over several GPUs (one process per GPU).

Reads are independent, so a batch splits into contiguous shards, one per rank, each
mapped against that rank's resident index replica with no exchange on the data path;
records are gathered back in read order. The transport is torch.distributed (NCCL on
GPUs, gloo for the CPU tests); only host objects (records, CIGARs) move, once per batch.
"""
from __future__ import annotations

from typing import Callable

import numpy as np

from . import MAP_RECORD_DTYPE, MapResult, ReadBatch


def shard_bounds(n: int, world: int) -> list[tuple[int, int]]:
    """Contiguous, near-equal [a, b) read ranges, one per rank, covering [0, n)."""
    base, extra = divmod(n, world)
    out, a = [], 0
    for r in range(world):
        b = a + base + (1 if r < extra else 0)
        out.append((a, b))
        a = b
    return out


def concat_results(parts: list[MapResult]) -> MapResult:
    """Concatenates per-shard results in order, rebasing CIGAR offsets."""
    recs, cigs, base = [], [], 0
    for p in parts:
        r = p.records.copy()
        r["cigar_off"] += base
        recs.append(r)
        cigs.append(p.cigar)
        base += len(p.cigar)
    rec = np.concatenate(recs) if recs else np.zeros(0, dtype=MAP_RECORD_DTYPE)
    cig = np.concatenate(cigs) if cigs else np.zeros(0, np.uint32)
    return MapResult(rec, cig)


def map_sharded(map_fn: Callable[[ReadBatch], MapResult], reads: ReadBatch, rank: int, world: int,
                group=None) -> MapResult | None:
    """Maps this rank's shard with map_fn and gathers every shard on rank 0 (None elsewhere).
    Every rank must call it with the same batch (collective)."""
    import torch.distributed as dist
    a, b = shard_bounds(len(reads), world)[rank]
    mine = map_fn(reads.slice(a, b))
    payload = (mine.records.tobytes(), mine.cigar.tobytes())
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(payload, gathered, dst=0, group=group)
    if rank != 0:
        return None
    parts = [MapResult(np.frombuffer(r, dtype=MAP_RECORD_DTYPE).copy(), np.frombuffer(c, np.uint32).copy())
             for r, c in gathered]
    return concat_results(parts)
