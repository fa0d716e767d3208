"""The request server (dnaln_serve_*): continuous batching over two resident indexes.

A request's records and CIGARs must be exactly those of mapping it alone
(Context.map_batch), whatever it was batched with: requests for two genomes, of 0 to a few
thousand reads and mixed lengths, submitted from several producer threads while others
are on the GPU, split across batches by the batch-size and HBM-budget limits."""
import threading
import time

import numpy as np
import pytest

import dnaln_b200 as D
from dnaln_b200 import synth
from dnaln_b200.serve import Server

pytestmark = pytest.mark.gpu


def recs(res: D.MapResult) -> np.ndarray:
    r = res.records
    return np.stack([r["contig"], r["pos"], r["rev"], r["mapq"], r["score"], r["nm"], r["n_cand"], r["cigar_off"],
                     r["cigar_len"]], 1).astype(np.int64)


@pytest.fixture(scope="module")
def two_genomes(ctx):
    ga, ra, _ = synth.workload("mixed-1Mbp-5k-50to1000bp", seed=21)
    gb, rb, _ = synth.workload("repeat-2Mbp-20k-150bp", seed=22)
    ia, ib = ctx.index_build(ga), ctx.index_build(gb)
    yield (ia, ra), (ib, rb)
    ctx.index_free(ia)
    ctx.index_free(ib)


def make_requests(two_genomes, n_req, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_req):
        iid, reads = two_genomes[int(rng.integers(2))]
        size = int(np.exp(rng.uniform(0, np.log(3000)))) if rng.random() > 0.05 else 0
        a = int(rng.integers(0, len(reads) - size + 1))
        out.append((iid, reads.slice(a, a + size)))
    return out


def serve_all(srv, reqs, p, producers=3, jitter_s=0.002, seed=0):
    """Submits reqs from `producers` threads with random gaps; returns results in order."""
    handles = [None] * len(reqs)

    def produce(k):
        rng = np.random.default_rng(seed + k)
        for i in range(k, len(reqs), producers):
            time.sleep(float(rng.uniform(0, jitter_s)))
            iid, reads = reqs[i]
            handles[i] = srv.submit(iid, reads, p)

    th = [threading.Thread(target=produce, args=(k,)) for k in range(producers)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return [srv.wait(h) for h in handles]


@pytest.mark.parametrize("coalesce,lanes,max_batch", [(True, 2, 2500), (True, 3, 100_000), (False, 1, 1500)])
def test_each_request_same_alone_and_in_the_mix(ctx, two_genomes, coalesce, lanes, max_batch):
    p = D.default_map_params()
    reqs = make_requests(two_genomes, 36, seed=lanes)
    alone = [ctx.map_batch(iid, reads, p) for iid, reads in reqs]
    with Server(ctx, lanes=lanes, coalesce=coalesce, max_batch_reads=max_batch) as srv:
        got = serve_all(srv, reqs, p, seed=lanes)
        st = srv.stats()
    for i, (g, a) in enumerate(zip(got, alone)):
        assert np.array_equal(recs(g), recs(a)), f"request {i} differs from its result alone"
        assert np.array_equal(g.cigar, a.cigar), f"request {i}: CIGARs differ from its result alone"
    assert st["requests"] == len(reqs)
    assert st["reads"] == sum(len(r) for _, r in reqs)
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    if not coalesce:  # one request per batch: at least one batch per non-empty request
        assert st["batches"] >= sum(1 for _, r in reqs if len(r))


def test_budget_limited_batches_and_bw64(ctx, two_genomes):
    # a small HBM budget: batches of a few hundred reads, requests split across many of them
    p = D.default_map_params(bw=64)
    reqs = make_requests(two_genomes, 12, seed=9)
    alone = [ctx.map_batch(iid, reads, p) for iid, reads in reqs]
    with Server(ctx, lanes=2, hbm_budget_bytes=40 << 20) as srv:
        got = serve_all(srv, reqs, p, producers=2, seed=5)
        st = srv.stats()
    for g, a in zip(got, alone):
        assert np.array_equal(recs(g), recs(a))
        assert np.array_equal(g.cigar, a.cigar)
    assert st["lane_budget_bytes"] < (20 << 20)
    assert st["mean_batch_reads"] < 1500


def test_errors_and_empty_requests(ctx, two_genomes):
    (ia, ra), _ = two_genomes
    p = D.default_map_params()
    with Server(ctx, lanes=1, hbm_budget_bytes=32 << 20) as srv:
        empty = srv.submit(ia, ra.slice(0, 0), p)
        assert len(srv.wait(empty).records) == 0
        with pytest.raises(D.DnalnError) as e:
            srv.submit(12345, ra.slice(0, 5), p)
        assert e.value.code == D.N.ERR_NOT_FOUND
        huge = D.ReadBatch.from_lists([b"ACGT" * 150_000], [b"huge"])  # over a lane's share of the budget
        with pytest.raises(D.DnalnError) as e:
            srv.submit(ia, huge, p)
        assert e.value.code == D.N.ERR_OOM
        ok = srv.submit(ia, ra.slice(0, 50), p)  # the server still serves after refusals
        assert np.array_equal(recs(srv.wait(ok)), recs(ctx.map_batch(ia, ra.slice(0, 50), p)))


def test_index_attach_shares_one_copy(ctx, two_genomes):
    (ia, ra), _ = two_genomes
    p = D.default_map_params()
    with D.Context(ctx.device) as other:
        j = other.index_attach(ctx, ia)
        assert other.index_stats(j) == ctx.index_stats(ia)
        a = other.map_batch(j, ra.slice(0, 400), p)
        other.index_free(j)  # drops the other context's reference only
    b = ctx.map_batch(ia, ra.slice(0, 400), p)
    assert np.array_equal(recs(a), recs(b)) and np.array_equal(a.cigar, b.cigar)
