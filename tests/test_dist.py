"""Multi-process host logic on CPU (gloo, world size 2): read shards mapped independently
and gathered in read order equal the single-process result; the bench's timing reduce is
the max over ranks. The per-shard mapper here is the oracle (the GPU mapper has the same
signature), so no GPU is needed."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import dnaln_b200 as D
from dnaln_b200 import shards, synth


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def port_mapper(g, params):
    import oracle
    port = oracle.Port()
    idx = port.index(g)

    def fn(reads):
        rec, cig, co = port.map(idx, reads, params)
        out = np.zeros(len(rec), dtype=D.MAP_RECORD_DTYPE)
        for j, f in enumerate(("contig", "pos", "rev", "mapq", "score", "nm", "n_cand")):
            out[f] = rec[:, j]
        out["cigar_off"], out["cigar_len"] = co[:-1], np.diff(co)
        return D.MapResult(out, cig)
    return fn


def worker(rank, world, port_no, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port_no))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        g, reads, _ = synth.workload("repeat-2Mbp-20k-150bp", seed=5, n_reads=1201)
        fn = port_mapper(g, D.default_map_params())
        res = shards.map_sharded(fn, reads, rank, world)
        import torch
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            full = fn(reads)
            q.put((np.array_equal(res.records, full.records), np.array_equal(res.cigar, full.cigar), float(t.item())))
    finally:
        dist.destroy_process_group()


def test_shard_bounds_cover_and_balance():
    for n in (0, 1, 7, 262_144, 1_000_000):
        for world in (1, 2, 3, 8):
            b = shards.shard_bounds(n, world)
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
            sizes = [y - x for x, y in b]
            assert max(sizes) - min(sizes) <= 1


@pytest.mark.timeout(300)
def test_two_rank_gloo_sharded_mapping_equals_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port_no = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port_no, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(240)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    same_rec, same_cig, tmax = q.get(timeout=5)
    assert same_rec and same_cig
    assert tmax == 2.0
