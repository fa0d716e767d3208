"""Whole-batch mapping on the GPU (dnaln_gpu_map_batch, the Mapper::map drop-in) against
the reference compiled from its own sources and the C port: identical records
(RNAME/POS/FLAG/MAPQ/CIGAR/NM/AS and candidate counts) and byte-identical SAM bodies."""
import os

import numpy as np
import pytest

import dnaln_b200 as D
from dnaln_b200 import synth

pytestmark = pytest.mark.gpu

NTHREADS = max(1, min(16, os.cpu_count() or 1))


def gpu_records(res: D.MapResult) -> np.ndarray:
    r = res.records
    return np.stack([r["contig"], r["pos"], r["rev"], r["mapq"], r["score"], r["nm"], r["n_cand"]], 1).astype(np.int64)


def assert_same_as(expected, res: D.MapResult, n: int):
    rec, cig, co = expected
    got = gpu_records(res)
    bad = np.nonzero((got != rec).any(1))[0]
    assert len(bad) == 0, f"{len(bad)} records differ, first {bad[:5]}: gpu {got[bad[:3]]} vs ref {rec[bad[:3]]}"
    assert np.array_equal(res.records["cigar_len"], np.diff(co).astype(np.int32))
    assert np.array_equal(res.cigar, cig)


@pytest.fixture(scope="module")
def small():
    return synth.workload("small-1Mbp-10k-150bp", seed=7, with_qual=True)


@pytest.fixture(scope="module")
def repeat():
    return synth.workload("repeat-2Mbp-20k-150bp", seed=3, with_qual=True)


@pytest.fixture(scope="module")
def mixed():
    return synth.workload("mixed-1Mbp-5k-50to1000bp", seed=4, with_qual=True)


def test_small_workload_sam_identical(ctx, ref, small):
    g, reads, truth = small
    p = D.default_map_params()
    iid = ctx.index_build(g)
    try:
        res = ctx.map_batch(iid, reads, p)
        rg = ref.genome(g)
        rec, cig, co, sam = ref.map(rg, reads, p, nthreads=NTHREADS, want_sam=True)
        assert_same_as((rec, cig, co), res, len(reads))
        assert D.sam_format(reads, res, g) == sam
        mapped = res.records["contig"] >= 0
        near = mapped & (res.records["rev"] == truth.rev) & (np.abs(res.records["pos"] - truth.start) <= 10)
        assert near.mean() > 0.98
    finally:
        ctx.index_free(iid)


@pytest.mark.parametrize("bw", [16, 64])
def test_repeat_workload_multi_candidate_parity(ctx, ref, repeat, bw):
    g, reads, _ = repeat
    p = D.default_map_params(bw=bw)
    iid = ctx.index_build(g)
    try:
        res = ctx.map_batch(iid, reads, p)
        rec, cig, co, sam = ref.map(ref.genome(g), reads, p, nthreads=NTHREADS, want_sam=True)
        assert (rec[:, 6] > 1).sum() > 500  # ranking, ties and MAPQ < 60 are exercised
        assert_same_as((rec, cig, co), res, len(reads))
        assert D.sam_format(reads, res, g) == sam
    finally:
        ctx.index_free(iid)


@pytest.mark.parametrize("bw", [16, 64])
def test_mixed_lengths_parity(ctx, ref, mixed, bw):
    g, reads, _ = mixed
    p = D.default_map_params(bw=bw)
    iid = ctx.index_build(g)
    try:
        res = ctx.map_batch(iid, reads, p)
        rec, cig, co = ref.map(ref.genome(g), reads, p, nthreads=NTHREADS)
        assert_same_as((rec, cig, co), res, len(reads))
    finally:
        ctx.index_free(iid)


def test_port_agrees_with_gpu_on_parameter_variants(ctx, port, repeat):
    g, reads, _ = repeat
    sub = reads.slice(0, 3000)
    iid = ctx.index_build(g)
    pi = port.index(g)
    try:
        for kw in [dict(max_cand=1), dict(max_cand=3, pri_ratio=0.9), dict(min_aln_score=0), dict(max_occ=3),
                   dict(match=1, mismatch=4, gap_open=6, gap_ext=1, bw=8), dict(match=3, mismatch=2, gap_open=0,
                                                                                 gap_ext=3, bw=21)]:
            p = D.default_map_params(**kw)
            assert_same_as(port.map(pi, sub, p), ctx.map_batch(iid, sub, p), len(sub))
    finally:
        ctx.index_free(iid)


def test_batch_invariance(ctx, repeat):
    # every read's record is the same alone, in a small batch and in the full batch
    g, reads, _ = repeat
    p = D.default_map_params()
    iid = ctx.index_build(g)
    try:
        full = ctx.map_batch(iid, reads, p)
        rng = np.random.default_rng(0)
        for i in rng.choice(len(reads), 40, replace=False):
            alone = ctx.map_batch(iid, reads.slice(int(i), int(i) + 1), p)
            assert np.array_equal(gpu_records(alone)[0], gpu_records(full)[i])
            assert np.array_equal(alone.cigar_of(0), full.cigar_of(int(i)))
        part = ctx.map_batch(iid, reads.slice(100, 1100), p)
        assert np.array_equal(gpu_records(part), gpu_records(full)[100:1100])
    finally:
        ctx.index_free(iid)


def test_empty_and_degenerate_reads(ctx, port, small):
    g, _, _ = small
    exact = np.frombuffer(b"ACGTN", np.uint8)[g.codes[5000:5150]].tobytes()  # an exact genome substring
    seqs = [b"", b"A", b"ACGT" * 3, b"N" * 200, b"ACGTNNNNACGT" * 20, exact, b"acgtu" * 30]
    names = [f"r{i}".encode() for i in range(len(seqs))]
    reads = D.ReadBatch.from_lists(seqs, names)
    iid = ctx.index_build(g)
    try:
        p = D.default_map_params()
        res = ctx.map_batch(iid, reads, p)
        assert_same_as(port.map(port.index(g), reads, p), res, len(reads))
        assert res.records["contig"][5] == 0 and res.records["score"][5] == 300
        assert len(ctx.map_batch(iid, reads.slice(0, 0), p).records) == 0
    finally:
        ctx.index_free(iid)


@pytest.mark.slow
def test_full_size_workload_against_reference(ctx, ref):
    # the 4.6 Mbp / 1,000,000-read workload, in its batches of 262,144 reads
    g, reads, truth = synth.workload("ecoli-4.6Mbp-1M-150bp", seed=1)
    p = D.default_map_params()
    iid = ctx.index_build(g)
    try:
        rg = ref.genome(g)
        for a in range(0, len(reads), 262_144):
            b = min(len(reads), a + 262_144)
            part = reads.slice(a, b)
            res = ctx.map_batch(iid, part, p)
            assert_same_as(ref.map(rg, part, p, nthreads=NTHREADS), res, len(part))
    finally:
        ctx.index_free(iid)
