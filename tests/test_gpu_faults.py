"""Recovery paths and host-side faults, none of which faults, traps or hangs the GPU:

* the chaining pool (scratch of reads seeded one warp each) made too small, so a batch
  outgrows it: the host grows the pool and maps the batch again, same records;
* the traceback direction-code scratch capped at 1 MiB, so every traceback launch is split
  into chunks (launch bases > 0): same records;
* a device allocation made to fail on the host (option fail_alloc_after): the call returns
  DNALN_ERR_OOM and the context maps the next batch correctly;
* a served request cancelled while it waits and while parts of it are on the GPU: its wait
  returns DNALN_ERR_CANCELLED, every other request stays bit-exact.

The reference stops the process on any such failure (die(), src/common.cpp:55-64); the
library reports a status instead and stays usable."""
import time

import numpy as np
import pytest

import dnaln_b200 as D
from dnaln_b200 import _native as N
from dnaln_b200 import synth
from dnaln_b200.serve import Server

pytestmark = pytest.mark.gpu


def recs(res: D.MapResult) -> np.ndarray:
    r = res.records
    return np.stack([r["contig"], r["pos"], r["rev"], r["mapq"], r["score"], r["nm"], r["n_cand"], r["cigar_off"],
                     r["cigar_len"]], 1).astype(np.int64)


def same(a: D.MapResult, b: D.MapResult) -> bool:
    return np.array_equal(recs(a), recs(b)) and np.array_equal(a.cigar, b.cigar)


@pytest.fixture(scope="module")
def repeat():
    return synth.workload("repeat-2Mbp-20k-150bp", seed=3)


@pytest.fixture(scope="module")
def mixed():
    return synth.workload("mixed-1Mbp-5k-50to1000bp", seed=4)


def test_chaining_pool_regrow_maps_the_batch_again(ctx, repeat):
    g, reads, _ = repeat
    p = D.default_map_params()
    iid = ctx.index_build(g)
    try:
        want = ctx.map_batch(iid, reads, p)
    finally:
        ctx.index_free(iid)
    with D.Context(ctx.device) as c2:
        c2.set_option("chain_pool", 64)
        j = c2.index_build(g)
        got = c2.map_batch(j, reads, p)
        assert c2.stats()["batch_retries"] >= 1  # the batch outgrew the pool and was mapped again
        assert same(got, want)
        again = c2.map_batch(j, reads, p)        # the grown pool holds it now
        assert c2.stats()["batch_retries"] == 1
        assert same(again, want)


@pytest.mark.parametrize("bw", [16, 64])
def test_traceback_scratch_chunking(ctx, mixed, bw):
    g, reads, _ = mixed
    p = D.default_map_params(bw=bw)
    iid = ctx.index_build(g)
    try:
        want = ctx.map_batch(iid, reads, p)
    finally:
        ctx.index_free(iid)
    with D.Context(ctx.device) as c2:
        c2.set_option("dir_cap_bytes", 1 << 20)
        c2.set_option("graphs", 0)
        j = c2.index_build(g)
        c2.reset_stats()
        c2.set_kernel_trace(True)
        got = c2.map_batch(j, reads, p)
        kt = c2.kernel_times()
        walks = kt.get("k_sw_walk", (0, 0.0))[0]
        assert walks > 4, kt  # the traceback tasks went through many chunked launches
        assert same(got, want)


def test_injected_allocation_failure_leaves_the_context_usable(ctx, repeat):
    g, reads, _ = repeat
    sub = reads.slice(0, 5000)
    p = D.default_map_params()
    iid = ctx.index_build(g)
    try:
        want = ctx.map_batch(iid, sub, p)
    finally:
        ctx.index_free(iid)
    with D.Context(ctx.device) as c2:
        c2.set_option("fail_alloc_after", 0)  # the index's first allocation fails
        with pytest.raises(D.DnalnError) as e:
            c2.index_build(g)
        assert e.value.code == N.ERR_OOM
        c2.set_option("fail_alloc_after", -1)
        j = c2.index_build(g)
        for after in (0, 7, 20):  # failures at different points of a first batch's buffer growth
            c3 = D.Context(ctx.device)
            try:
                k = c3.index_attach(c2, j)
                c3.set_option("fail_alloc_after", after)
                with pytest.raises(D.DnalnError) as e:
                    c3.map_batch(k, sub, p)
                assert e.value.code == N.ERR_OOM
                c3.set_option("fail_alloc_after", -1)
                assert same(c3.map_batch(k, sub, p), want)  # the same context maps the next batch
            finally:
                c3.close()
        assert same(c2.map_batch(j, sub, p), want)


def test_cancelled_request_and_the_others(ctx, repeat):
    g, reads, _ = repeat
    p = D.default_map_params()
    iid = ctx.index_build(g)
    try:
        big = synth.make_reads(g, synth.ReadsSpec(n_reads=60_000), 77)[0]
        a, c = reads.slice(0, 3000), reads.slice(5000, 7000)
        want_a, want_c = ctx.map_batch(iid, a, p), ctx.map_batch(iid, c, p)
        with Server(ctx, lanes=1, max_batch_reads=500) as srv:
            ra = srv.submit(iid, a, p)
            rb = srv.submit(iid, big, p)      # 120 batches of 500 reads: still running when cancelled
            rc = srv.submit(iid, c, p)
            srv.cancel(rb)
            with pytest.raises(D.DnalnError) as e:
                srv.wait(rb)
            assert e.value.code == N.ERR_CANCELLED
            assert same(srv.wait(ra), want_a)
            assert same(srv.wait(rc), want_c)
            done = srv.submit(iid, a, p)
            first = srv.wait(done)
            assert same(first, want_a)
            st = srv.stats()
            assert st["requests"] == 3  # the cancelled request is not counted as served
            with pytest.raises(D.DnalnError) as e:
                srv.cancel(rb)                # already waited for: unknown
            assert e.value.code == N.ERR_INVALID_ARG
            # a request cancelled after it completed keeps its result
            late = srv.submit(iid, c, p)
            time.sleep(0.5)  # long enough for 2,000 reads to be mapped
            srv.cancel(late)
            assert same(srv.wait(late), want_c)
    finally:
        ctx.index_free(iid)
