"""The measured workloads at their stated sizes, every record against the reference's own
Mapper::map (src/mapper.cpp:75-223, compiled from its sources into oracle/_ref) and, for the
served stream, every request's SAM against the reference's append_sam
(src/mapper.cpp:231-270):

* mixed-4.6Mbp-1M-50to1000bp — all 1,000,000 reads (log-uniform 50-1000 bp, 2% with an
  8-15 bp deletion) at band width 16 and again at 64, in batches of 262,144;
* repeat-120Mbp-10M-150bp — all 10,000,000 reads on the 120 Mbp repeat-rich genome
  (1.28 GB index resident), in batches of 262,144;
* serve — a Poisson stream of 300 requests over both resident indexes (4.6 Mbp and
  120 Mbp), log-uniform 1-50,000 reads of U[100, 300] bp each, through the continuously
  batching server while other requests are on the GPU.

Minutes of CPU work for the reference on all host threads; marked slow."""
import os
import threading
import time

import numpy as np
import pytest

import dnaln_b200 as D
from dnaln_b200 import synth
from dnaln_b200.serve import Server

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

NTHREADS = max(1, min(32, os.cpu_count() or 1))
BATCH = 262_144


def records(res: D.MapResult) -> np.ndarray:
    r = res.records
    return np.stack([r["contig"], r["pos"], r["rev"], r["mapq"], r["score"], r["nm"], r["n_cand"]], 1).astype(np.int64)


def assert_same(exp, res: D.MapResult, what: str):
    rec, cig, co = exp[:3]
    got = records(res)
    bad = np.nonzero((got != rec).any(1))[0]
    assert len(bad) == 0, f"{what}: {len(bad)} records differ, first {bad[:5]}: gpu {got[bad[:3]]} vs ref {rec[bad[:3]]}"
    assert np.array_equal(res.records["cigar_len"], np.diff(co).astype(np.int32)), what
    assert np.array_equal(res.cigar, cig), what


def map_in_batches(ctx, ref, g, reads, p):
    iid = ctx.index_build(g)
    rg = ref.genome(g)
    multi = 0
    try:
        for a in range(0, len(reads), BATCH):
            part = reads.slice(a, min(len(reads), a + BATCH))
            exp = ref.map(rg, part, p, nthreads=NTHREADS)
            multi += int((exp[0][:, 6] > 1).sum())
            assert_same(exp, ctx.map_batch(iid, part, p), f"reads {a}..{a + len(part)}")
    finally:
        ctx.index_free(iid)
    return multi


@pytest.mark.parametrize("bw", [16, 64])
def test_mixed_lengths_1m_reads_against_reference(ctx, ref, bw):
    g, reads, _ = synth.workload("mixed-4.6Mbp-1M-50to1000bp", seed=5)
    assert len(reads) == 1_000_000 and reads.seq_len.max() > 900 and reads.seq_len.min() < 60
    ctx.reset_stats()
    map_in_batches(ctx, ref, g, reads, D.default_map_params(bw=bw))
    assert ctx.stats()["long_reads"] > 100_000  # the long-read kernel carried its share


def test_repeat_120mbp_10m_reads_against_reference(ctx, ref):
    g, reads, _ = synth.workload("repeat-120Mbp-10M-150bp", seed=2)
    assert len(reads) == 10_000_000
    multi = map_in_batches(ctx, ref, g, reads, D.default_map_params())
    assert multi > 200_000  # multi-candidate ranking, ties and MAPQ < 60 at scale


def test_served_poisson_stream_against_reference(ctx, ref):
    genomes = [synth.make_genome(synth.GENOME_4M6, 31), synth.make_genome(synth.GENOME_120M, 32)]
    spec = synth.ReadsSpec(n_reads=300_000, len_min=100, len_max=300, len_dist=2)
    pools = [synth.make_reads(g, spec, 40 + i, with_qual=True)[0] for i, g in enumerate(genomes)]
    rng = np.random.default_rng(33)
    n_req = 300
    reqs = []
    for _ in range(n_req):
        gi = int(rng.integers(2))
        size = int(min(50_000, max(1, np.floor(np.exp(rng.uniform(0, np.log(50_001)))))))
        a = int(rng.integers(0, len(pools[gi]) - size + 1))
        reqs.append((gi, pools[gi].slice(a, a + size)))
    p = D.default_map_params()
    iids = [ctx.index_build(g) for g in genomes]
    handles = [None] * n_req
    try:
        with Server(ctx, lanes=3) as srv:
            arrivals = np.cumsum(rng.exponential(1 / 5000.0, n_req))  # ~5,000 requests/s offered: a queue forms

            def produce():
                t0 = time.perf_counter()
                for i, (gi, rb) in enumerate(reqs):
                    dt = arrivals[i] - (time.perf_counter() - t0)
                    if dt > 0:
                        time.sleep(dt)
                    handles[i] = srv.submit(iids[gi], rb, p)

            th = threading.Thread(target=produce)
            th.start()
            th.join()
            got = [srv.wait(h) for h in handles]
            st = srv.stats()
    finally:
        for i in iids:
            ctx.index_free(i)
    assert st["requests"] == n_req and st["reads"] == sum(len(rb) for _, rb in reqs)
    assert st["batches"] < n_req  # requests shared batches
    rgs = [ref.genome(g) for g in genomes]
    for i, ((gi, rb), res) in enumerate(zip(reqs, got)):
        rec, cig, co, sam = ref.map(rgs[gi], rb, p, nthreads=NTHREADS, want_sam=True)
        assert_same((rec, cig, co), res, f"request {i}")
        assert D.sam_format(rb, res, genomes[gi]) == sam, f"request {i}: SAM differs"
