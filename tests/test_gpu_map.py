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


@pytest.mark.parametrize("bw", [16, 32])
def test_sw_forms_give_the_same_records(ctx, repeat, bw):
    # the inter- and intra-sequence SW kernels (and whichever the tuner picks) map alike
    g, reads, _ = repeat
    p = D.default_map_params(bw=bw)
    iid = ctx.index_build(g)
    try:
        got = []
        for form in (1, 2, 3, 0):
            ctx.set_option("sw_form", form)
            got.append(ctx.map_batch(iid, reads, p))
    finally:
        ctx.set_option("sw_form", 0)
        ctx.index_free(iid)
    for other in got[1:]:
        assert np.array_equal(gpu_records(got[0]), gpu_records(other))
        assert np.array_equal(got[0].cigar, other.cigar)


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


@pytest.mark.parametrize("wl", ["repeat", "mixed", "small"])
def test_thread_and_warp_seed_paths_identical(ctx, request, wl):
    # short reads are seeded and chained one thread per read, long ones one thread per read
    # with state in global memory, the rest (past either kernel's bounds) one warp per
    # read; turning the long-read kernel off, or forcing every read through the warp
    # kernels, must give the same records and CIGARs
    g, reads, _ = request.getfixturevalue(wl)
    p = D.default_map_params()
    iid = ctx.index_build(g)
    try:
        ctx.reset_stats()
        mixed_path = ctx.map_batch(iid, reads, p)
        st = ctx.stats()
        ctx.set_option("long_thread", 0)
        no_long = ctx.map_batch(iid, reads, p)
        ctx.set_option("long_thread", 1)
        ctx.set_option("warp_seed_only", 1)
        warp_path = ctx.map_batch(iid, reads, p)
    finally:
        ctx.set_option("warp_seed_only", 0)
        ctx.set_option("long_thread", 1)
        ctx.index_free(iid)
    if wl == "mixed":  # long reads took the long-read thread kernel
        assert st["long_reads"] > 0
    for other in (no_long, warp_path):
        assert np.array_equal(gpu_records(mixed_path), gpu_records(other))
        assert np.array_equal(mixed_path.records["cigar_len"], other.records["cigar_len"])
        assert np.array_equal(mixed_path.cigar, other.cigar)


def test_graph_replays_give_the_same_results(ctx, repeat, mixed):
    # a batch whose launches repeat is captured as a CUDA graph on its second run and
    # replayed from the third on; every run must give what kernel-by-kernel launches give
    for g, reads, bw in [(repeat[0], repeat[1], 16), (mixed[0], mixed[1], 64)]:
        p = D.default_map_params(bw=bw)
        iid = ctx.index_build(g)
        try:
            ctx.set_option("graphs", 0)
            want = ctx.map_batch(iid, reads, p)
            ctx.set_option("graphs", 1)
            g0 = ctx.stats()["graph_launches"]
            for _ in range(4):
                got = ctx.map_batch(iid, reads, p)
                assert np.array_equal(gpu_records(got), gpu_records(want))
                assert np.array_equal(got.cigar, want.cigar)
            assert ctx.stats()["graph_launches"] >= g0 + 2
        finally:
            ctx.set_option("graphs", 1)
            ctx.index_free(iid)


@pytest.mark.parametrize("sub_batch", [0, 3000])
def test_submit_wait_matches_map_batch(ctx, repeat, sub_batch):
    # several batches in flight through the worker (reads copied in while the previous batch
    # computes), waited for out of order; each must equal the synchronous call
    g, reads, _ = repeat
    p = D.default_map_params()
    iid = ctx.index_build(g)
    try:
        ctx.set_sub_batch(0)
        spans = [(0, 7000), (7000, 7001), (7001, 7001), (7001, 20000), (3000, 9000)]
        want = [ctx.map_batch(iid, reads.slice(a, b), p) for a, b in spans]
        ctx.set_sub_batch(sub_batch)
        tickets = [ctx.map_submit(iid, reads.slice(a, b), p) for a, b in spans]
        for t, w in reversed(list(zip(tickets, want))):
            got = ctx.map_wait(t)
            assert np.array_equal(gpu_records(got), gpu_records(w))
            assert np.array_equal(got.records["cigar_off"], w.records["cigar_off"])
            assert np.array_equal(got.cigar, w.cigar)
    finally:
        ctx.set_sub_batch(0)
        ctx.index_free(iid)


@pytest.mark.parametrize("sub_batch", [0, 997, 4096])
def test_sub_batch_pipeline_identical(ctx, repeat, sub_batch):
    # the host-buffer call streams sub-batches through two device slots; records and
    # CIGARs must not depend on the split, also when reads sit out of order in the buffer
    from dnaln_b200 import _native as N
    g, reads, _ = repeat
    p = D.default_map_params()
    iid = ctx.index_build(g)
    try:
        ctx.set_sub_batch(0)
        whole = ctx.map_batch(iid, reads, p)
        n = len(reads)
        lens = np.ascontiguousarray(reads.seq_len)
        order = np.random.default_rng(5).permutation(n)  # buffer layout: reads stored in this order
        chunks = [reads.read(int(i)) for i in order]
        buf = np.frombuffer(b"".join(chunks), np.uint8).copy()
        pos = np.zeros(n, np.int64)
        pos[order] = np.concatenate([[0], np.cumsum([len(x) for x in chunks])[:-1]])
        nh = reads.name_hash()
        rec = np.zeros(n, dtype=D.MAP_RECORD_DTYPE)
        cap = int(np.sum(2 * lens.astype(np.int64) + 3))
        cig = np.zeros(cap, np.uint32)
        used = D.C.c_int64()
        ctx.set_sub_batch(sub_batch)
        rc = N.lib().dnaln_gpu_map_batch(ctx.handle, iid, N.ptr(buf), N.ptr(pos), N.ptr(lens), N.ptr(nh), n,
                                         D.C.byref(p), N.ptr(rec), N.ptr(cig), cap, D.C.byref(used))
        assert rc == 0, N.lib().dnaln_gpu_last_error(ctx.handle).decode()
        got = D.MapResult(rec, cig[:used.value])
        assert np.array_equal(gpu_records(got), gpu_records(whole))
        for i in range(0, n, 97):
            assert np.array_equal(got.cigar_of(i), whole.cigar_of(i))
        assert used.value == len(whole.cigar)
    finally:
        ctx.set_sub_batch(0)
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


@pytest.mark.slow
def test_repeat_120mbp_workload_against_reference(ctx, ref):
    # the 120 Mbp genome (8 contigs, repeat families, N runs; 1.28 GB index resident in HBM),
    # 500,000 of its 150 bp reads in batches of 262,144: multi-candidate ranking, ties, MAPQ
    g, reads, _ = synth.workload("repeat-120Mbp-10M-150bp", seed=2, n_reads=500_000)
    p = D.default_map_params()
    iid = ctx.index_build(g)
    try:
        assert ctx.index_stats(iid)["device_bytes"] > 1 << 30
        rg = ref.genome(g)
        multi = 0
        for a in range(0, len(reads), 262_144):
            part = reads.slice(a, min(len(reads), a + 262_144))
            exp = ref.map(rg, part, p, nthreads=NTHREADS)
            multi += int((exp[0][:, 6] > 1).sum())
            assert_same_as(exp, ctx.map_batch(iid, part, p), len(part))
        assert multi > 10_000
    finally:
        ctx.index_free(iid)


def test_seed_block_tuner_and_pinned_sizes_agree(ctx):
    # the reads-per-block tuner times 64 and 128 reads per block on the first large batch;
    # every size gives the same records
    g, reads, _ = synth.workload("small-1Mbp-10k-150bp", seed=9, n_reads=40_000)
    p = D.default_map_params()
    got = []
    for size in (0, 64, 128):
        with D.Context(ctx.device) as c2:
            c2.set_option("seed_block", size)
            j = c2.index_build(g)
            got.append(c2.map_batch(j, reads, p))
            t = c2.seed_tuning()
            if size == 0:
                assert t["tuned"] == 1 and t["reads_per_block"] in (64, 128) and t["reads"] == len(reads)
                assert t["ms_64"] > 0 and t["ms_128"] > 0
                assert t["reads_per_block"] == (64 if t["ms_64"] < t["ms_128"] else 128)
            else:
                assert t["tuned"] == 0
    for other in got[1:]:
        assert np.array_equal(gpu_records(got[0]), gpu_records(other))
        assert np.array_equal(got[0].cigar, other.cigar)


@pytest.mark.parametrize("wl", ["repeat", "mixed"])
def test_work_stealing_and_fixed_grids_agree(ctx, request, wl):
    # the warp-per-read chaining kernel either takes reads by atomic claims on resident
    # blocks or strides over a fixed grid: same records
    g, reads, _ = request.getfixturevalue(wl)
    p = D.default_map_params()
    iid = ctx.index_build(g)
    try:
        got = []
        for mode in (1, 0):
            ctx.set_option("work_stealing", mode)
            got.append(ctx.map_batch(iid, reads, p))
    finally:
        ctx.set_option("work_stealing", 1)
        ctx.index_free(iid)
    for other in got[1:]:
        assert np.array_equal(gpu_records(got[0]), gpu_records(other))
        assert np.array_equal(got[0].cigar, other.cigar)


def test_bulk_encode_and_per_read_encode_agree(ctx, mixed, small):
    # the codes of both strands come from shared-memory tiles moved by bulk copies when a
    # tile's reads are back to back, read by read otherwise; records must not depend on it,
    # for packed reads and for reads stored out of order (every tile not back to back)
    from dnaln_b200 import _native as N
    for g, reads in ((mixed[0], mixed[1]), (small[0], small[1].slice(0, 4000))):
        p = D.default_map_params()
        iid = ctx.index_build(g)
        try:
            got = []
            for bulk in (1, 0):
                ctx.set_option("encode_bulk", bulk)
                got.append(ctx.map_batch(iid, reads, p))
            # reads stored in a permuted order in the buffer (offsets still per read)
            n = len(reads)
            order = np.random.default_rng(3).permutation(n)
            chunks = [reads.read(int(i)) for i in order]
            buf = np.frombuffer(b"".join(chunks), np.uint8).copy()
            pos = np.zeros(n, np.int64)
            pos[order] = np.concatenate([[0], np.cumsum([len(x) for x in chunks])[:-1]])
            lens = np.ascontiguousarray(reads.seq_len)
            nh = reads.name_hash()
            rec = np.zeros(n, dtype=D.MAP_RECORD_DTYPE)
            cap = int(np.sum(2 * lens.astype(np.int64) + 3))
            cig = np.zeros(cap, np.uint32)
            used = D.C.c_int64()
            ctx.set_option("encode_bulk", 1)
            rc = N.lib().dnaln_gpu_map_batch(ctx.handle, iid, N.ptr(buf), N.ptr(pos), N.ptr(lens), N.ptr(nh), n,
                                             D.C.byref(p), N.ptr(rec), N.ptr(cig), cap, D.C.byref(used))
            assert rc == 0, N.lib().dnaln_gpu_last_error(ctx.handle).decode()
            got.append(D.MapResult(rec, cig[:used.value]))
        finally:
            ctx.set_option("encode_bulk", 0)
            ctx.index_free(iid)
        for other in got[1:]:
            assert np.array_equal(gpu_records(got[0]), gpu_records(other))
            assert np.array_equal(got[0].cigar, other.cigar)
