"""Per-stage GPU entry points against the oracle: sketch (src/minimizer.cpp), the resident
index layout and lookups (src/index.hpp/.cpp), and chaining (src/chain.cpp)."""
import numpy as np
import pytest

import dnaln_b200 as D
from dnaln_b200 import synth
from helpers import known_answer_anchors, random_anchor_set, random_codes

pytestmark = pytest.mark.gpu


def test_sketch_matches_reference_random(ctx, ref):
    # the reference's brute-force case: k in [5, 24], w in [1, 20], 50..449 bp, Ns in a third
    rng = np.random.default_rng(7)
    for trial in range(200):
        k = 5 + int(rng.integers(20))
        w = 1 + int(rng.integers(20))
        s = random_codes(rng, 50 + int(rng.integers(400)), 0.01 if trial % 3 == 0 else 0.0)
        (h, p, st), = ctx.sketch([s], k, w, [1000])
        eh, ep, es = ref.sketch(s, k, w, 1000)
        assert np.array_equal(h, eh) and np.array_equal(p, ep) and np.array_equal(st, es), (trial, k, w)


def test_sketch_batch_and_edges(ctx, port):
    rng = np.random.default_rng(11)
    seqs = [random_codes(rng, n, r) for n, r in [(0, 0), (5, 0), (14, 0), (15, 0), (24, 0), (25, 0), (150, 0),
                                                 (150, 0.05), (1000, 0.01), (3000, 0.0), (300, 0.3)]]
    seqs.append(np.full(200, 4, np.uint8))
    seqs.append(np.tile(np.array([0, 3], np.uint8), 100))  # palindromic k-mers everywhere
    seqs.append(np.zeros(200, np.uint8))                   # poly-A
    for k, w in [(15, 10), (4, 1), (28, 255), (31, 3)]:
        got = ctx.sketch(seqs, k, w)
        for s, (h, p, st) in zip(seqs, got):
            eh, ep, es = port.sketch(s, k, w)
            assert np.array_equal(h, eh) and np.array_equal(p, ep) and np.array_equal(st, es), (len(s), k, w)


def test_strand_symmetry(ctx):
    rng = np.random.default_rng(11)
    s = random_codes(rng, 5000)
    rc = np.where(s[::-1] < 4, 3 - s[::-1], 4).astype(np.uint8)
    (ha, _, _), (hb, _, _) = ctx.sketch([s, rc], 15, 10)
    common = len(np.intersect1d(ha, hb))
    assert common >= 0.95 * len(np.unique(ha))


@pytest.fixture(scope="module")
def small_genome():
    return synth.make_genome(synth.GENOME_REPEAT_2M, 5)


def test_index_layout_matches_port(ctx, port, small_genome):
    g = small_genome
    iid = ctx.index_build(g, 15, 10)
    try:
        keys, offs, cnts, pos = ctx.index_export(iid)
        pk, po, pc, pp = port.index(g, 15, 10).export()
        assert np.array_equal(keys, pk) and np.array_equal(offs, po) and np.array_equal(cnts, pc)
        assert np.array_equal(pos, pp)
        st = ctx.index_stats(iid)
        ps = port.index(g, 15, 10).stats()
        for kk in ("n_keys", "n_positions", "max_count", "memory_bytes"):
            assert st[kk] == ps[kk]
    finally:
        ctx.index_free(iid)


def _ragged_genome(rng):
    # contigs of 0, 3, 40, 2,000, 30,000 and 120,000 bases, N runs inside and at the contig
    # edges, one contig all N
    lens = [0, 3, 40, 2000, 30000, 500, 120000]
    parts = []
    for i, n in enumerate(lens):
        c = random_codes(rng, n, 0.002)
        if n >= 40:
            c[:7] = 4
            c[-5:] = 4
        if i == 5:
            c[:] = 4
        parts.append(c)
    off = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
    return D.Genome(np.concatenate(parts).astype(np.uint8), off, np.array(lens, np.uint32))


@pytest.mark.parametrize("k,w", [(15, 10), (4, 1), (28, 255), (12, 5), (21, 40)])
def test_index_build_on_device_matches_port(ctx, port, k, w):
    # the device build (sketch of every contig, stable sort, rank-ordered bucket placement)
    # must give the reference's table bucket for bucket, for ragged contigs, N runs and the
    # extreme k / w (even k: palindromic k-mers)
    g = _ragged_genome(np.random.default_rng(k * 1000 + w))
    iid = ctx.index_build(g, k, w)
    try:
        keys, offs, cnts, pos = ctx.index_export(iid)
        pk, po, pc, pp = port.index(g, k, w).export()
        assert np.array_equal(keys, pk) and np.array_equal(offs, po) and np.array_equal(cnts, pc)
        assert np.array_equal(pos, pp)
        st = ctx.index_stats(iid)
        ps = port.index(g, k, w).stats()
        for kk in ("n_keys", "n_positions", "max_count", "memory_bytes"):
            assert st[kk] == ps[kk], kk
    finally:
        ctx.index_free(iid)


def test_index_build_all_n_and_tiny(ctx, port):
    for codes, lens in [(np.full(1000, 4, np.uint8), [1000]), (np.array([0, 1, 2], np.uint8), [3])]:
        g = D.Genome(codes, np.array([0], np.uint64), np.array(lens, np.uint32))
        iid = ctx.index_build(g, 15, 10)
        try:
            keys, offs, cnts, pos = ctx.index_export(iid)
            assert ctx.index_stats(iid)["n_keys"] == 0 and len(pos) == 0
            assert np.array_equal(keys, port.index(g, 15, 10).export()[0])
        finally:
            ctx.index_free(iid)


def test_lookup_every_minimizer_and_absent(ctx, ref, small_genome):
    g = small_genome
    iid = ctx.index_build(g, 15, 10)
    rg = ref.genome(g, 15, 10)
    try:
        keys, offs, cnts, pos = ctx.index_export(iid)
        present = keys[keys != np.uint64(2**64 - 1)]
        rng = np.random.default_rng(1)
        probe = np.concatenate([present[rng.permutation(len(present))[:20000]],
                                rng.integers(0, 2**30, 5000, dtype=np.uint64), np.array([1 << 40], np.uint64)])
        off, cnt = ctx.lookup(iid, probe)
        for i in range(0, len(probe), 97):
            exp = rg.lookup(int(probe[i]))
            assert cnt[i] == len(exp)
            assert np.array_equal(pos[off[i]:off[i] + cnt[i]], exp)
        assert cnt[-1] == 0  # k=15 hashes are < 2^30
    finally:
        ctx.index_free(iid)


def test_chain_known_answer(ctx):
    (srt, ch), = ctx.chain([known_answer_anchors()], 15)
    assert len(ch["score"]) >= 1
    assert ch["n_anchors"][0] == 10 and ch["dmin"][0] == 1000 and ch["dmax"][0] == 1003


def test_chain_random_sets_match_reference(ctx, ref):
    rng = np.random.default_rng(3)
    sets = [random_anchor_set(rng, int(rng.integers(0, 60)), int(rng.integers(0, 40))) for _ in range(400)]
    sets += [random_anchor_set(rng, 400, 300), random_anchor_set(rng, 5, 2000)]  # large sets (global scratch)
    sets.append(known_answer_anchors())
    for cp in [(5000, 16, 50, 20, 2), (200, 5, 10, 0, 1), (100000, 64, 80, 30, 3)]:
        got = ctx.chain(sets, 15, D.ChainParams(*cp))
        for i, ((sr, sq, ss), ch) in enumerate(got):
            (er, eq, es), ech = ref.chain(*sets[i], 15, cp)
            assert np.array_equal(sr, er) and np.array_equal(sq, eq) and np.array_equal(ss, es), i
            for key in ech:
                assert np.array_equal(ch[key], ech[key]), (i, key, cp)
