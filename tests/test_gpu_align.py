"""Banded SW on the GPU (dnaln_gpu_align, the Aligner::align drop-in) against the oracle:
bit-exact score, coordinates, NM and CIGAR, both modes, the reference's four scoring
schemes, plus edge cases (empty/one-base queries, all-N, short targets, long reads,
wide bands handled by the generic kernel)."""
import numpy as np
import pytest

import dnaln_b200 as D
from helpers import SCHEMES, mutate, random_codes, random_tasks

pytestmark = pytest.mark.gpu


def check_same(gpu: D.AlignOut, exp, traceback: bool):
    assert len(gpu.results) == len(exp)
    for i, e in enumerate(exp):
        r = gpu.results[i]
        got = (int(r["score"]), int(r["qb"]), int(r["qe"]), int(r["tb"]), int(r["te"]), int(r["nm"]))
        assert got[0] == e[0], f"task {i}: score {got[0]} != {e[0]}"
        if traceback:
            assert got == tuple(e[:6]), f"task {i}: {got} != {tuple(e[:6])}"
            assert np.array_equal(gpu.cigar_of(i), e[6]), f"task {i}: cigar {gpu.cigar_of(i)} != {e[6]}"


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("traceback", [False, True])
def test_random_tasks_match_port(ctx, port, scheme, traceback):
    rng = np.random.default_rng(13 + scheme[5] + 100 * traceback)
    qs, ts = random_tasks(rng, 600, scheme[5])
    sp = D.ScoreParams(*scheme)
    check_same(ctx.align(qs, ts, traceback, sp), port.align(qs, ts, traceback, scheme), traceback)


@pytest.mark.parametrize("scheme", SCHEMES + [(2, 0, 4, 2, 0, 16), (1, 3, 5, 2, 2, 12)])
def test_walk_diagonal_blocks_against_reference(ctx, ref, scheme):
    """Long diagonal runs, the case the walk takes eight steps at a time: queries with
    scattered Ns and sparse substitutions against N-free targets (so the 16-bit DP kernels
    take them), local starts and ends at every offset within a block (random junk on
    either end of the query), and a scheme where mismatches and Ns cost nothing."""
    rng = np.random.default_rng(31 + scheme[1] + 7 * scheme[4])
    bw = scheme[5]
    qs, ts = [], []
    for i in range(400):
        core = random_codes(rng, 40 + int(rng.integers(600)), 0.01)
        head, tail = random_codes(rng, i % 9), random_codes(rng, (i // 9) % 9)
        q = np.concatenate([head, core, tail])
        m = mutate(rng, np.where(core > 3, rng.integers(0, 4, core.shape), core).astype(np.uint8), 0.005, 0.0)
        shift = int(rng.integers(2 * bw + 1))
        t = np.concatenate([random_codes(rng, shift + len(head)), m, random_codes(rng, 2 * bw + len(tail))])
        qs.append(q)
        ts.append(t.astype(np.uint8))
    sp = D.ScoreParams(*scheme)
    check_same(ctx.align(qs, ts, True, sp), ref.align(qs, ts, True, scheme), True)


@pytest.mark.parametrize("n", [1, 5, 32, 33, 1003])
def test_batch_sizes_match_reference(ctx, ref, n):
    rng = np.random.default_rng(n)
    qs, ts = random_tasks(rng, n, 16)
    for tb in (False, True):
        check_same(ctx.align(qs, ts, tb), ref.align(qs, ts, tb, SCHEMES[0], simd=True), tb)


def test_perfect_match(ctx):
    # 150 bp query inside a target with bw random flanking bases: 150M, score 300, tb = bw
    rng = np.random.default_rng(17)
    q = random_codes(rng, 150)
    t = np.concatenate([random_codes(rng, 16), q, random_codes(rng, 16)])
    out = ctx.align([q], [t], True)
    r = out.results[0]
    assert (r["score"], r["qb"], r["qe"], r["tb"], r["nm"]) == (300, 0, 150, 16, 0)
    assert D.cigar_to_string(out.cigar_of(0)) == "150M"


def test_edge_cases(ctx, port):
    rng = np.random.default_rng(5)
    qs = [np.zeros(0, np.uint8), random_codes(rng, 1), np.full(40, 4, np.uint8), random_codes(rng, 100),
          random_codes(rng, 100), random_codes(rng, 1000, 0.01), random_codes(rng, 64)]
    ts = [random_codes(rng, 33), qs[1].copy(), np.full(72, 4, np.uint8), np.zeros(0, np.uint8),
          random_codes(rng, 10), np.concatenate([random_codes(rng, 7), qs[5], random_codes(rng, 25)]),
          np.concatenate([qs[6], qs[6]])]
    for tb in (False, True):
        check_same(ctx.align(qs, ts, tb), port.align(qs, ts, tb), tb)


@pytest.mark.parametrize("bw", [0, 1, 3, 32, 64, 100])
def test_other_band_widths(ctx, port, bw):
    # widths without a register-resident kernel go through the generic band kernel
    rng = np.random.default_rng(bw + 1)
    qs, ts = random_tasks(rng, 120, bw, max_len=400)
    sc = (2, 4, 4, 2, 1, bw)
    for tb in (False, True):
        check_same(ctx.align(qs, ts, tb, D.ScoreParams(*sc)), port.align(qs, ts, tb, sc), tb)


@pytest.mark.parametrize("scheme", SCHEMES)
def test_wide_band_lanes(ctx, port, scheme):
    # bw 64 (W = 129) runs four lanes per pair of alignments; odd task counts, mixed lengths
    # up to 1000 and N bases (the int32 list) included
    sc = scheme[:5] + (64,)
    rng = np.random.default_rng(sum(scheme))
    qs, ts = random_tasks(rng, 1001, 64, max_len=1000)
    for q in qs[::37]:
        q[rng.integers(len(q))] = 4 if len(q) else 0
    for t in ts[::53]:
        if len(t):
            t[rng.integers(len(t))] = 4
    for tb in (False, True):
        check_same(ctx.align(qs, ts, tb, D.ScoreParams(*sc)), port.align(qs, ts, tb, sc), tb)


def test_large_scores_outside_byte_profile(ctx, port):
    # scores that do not fit the signed-byte substitution profile use the generic path
    sc = (200, 300, 5, 2, 150, 16)
    rng = np.random.default_rng(9)
    qs, ts = random_tasks(rng, 100, 16)
    for tb in (False, True):
        check_same(ctx.align(qs, ts, tb, D.ScoreParams(*sc)), port.align(qs, ts, tb, sc), tb)


def test_traceback_consistency(ctx):
    # CIGAR re-scores to the score; query/target spans match; starts and ends with M
    rng = np.random.default_rng(21)
    for sc in SCHEMES:
        qs, ts = random_tasks(rng, 300, sc[5])
        out = ctx.align(qs, ts, True, D.ScoreParams(*sc))
        so = ctx.align(qs, ts, False, D.ScoreParams(*sc))
        A, B, O, E, amb, bw = sc
        W = 2 * bw + 1
        for i, (q, t) in enumerate(zip(qs, ts)):
            r = out.results[i]
            assert r["score"] == so.results[i]["score"]
            if r["score"] == 0:
                continue
            tt = np.full(len(q) + W - 1, 4, np.uint8)
            tt[:min(len(t), len(tt))] = t[:len(tt)]
            s, qi, tj, qspan, tspan = 0, int(r["qb"]), int(r["tb"]), 0, 0
            cig = out.cigar_of(i)
            for c in cig:
                op, ln = int(c) & 0xF, int(c) >> 4
                if op == 0:
                    for _ in range(ln):
                        a, b = q[qi], tt[tj]
                        s += -amb if (a > 3 or b > 3) else (A if a == b else -B)
                        qi += 1
                        tj += 1
                    qspan += ln
                    tspan += ln
                elif op == 1:
                    s -= O + ln * E
                    qi += ln
                    qspan += ln
                else:
                    s -= O + ln * E
                    tj += ln
                    tspan += ln
            assert s == r["score"]
            assert qspan == r["qe"] - r["qb"] and tspan == r["te"] - r["tb"]
            assert int(cig[0]) & 0xF == 0 and int(cig[-1]) & 0xF == 0


@pytest.mark.parametrize("bw", [16, 32, 64])
def test_sw_forms_identical_and_tuned(ctx, port, bw):
    # W = 33 and 65 have an inter-sequence kernel and two intra-sequence ones (32 or 16
    # cells per lane), W = 129 the two intra-sequence ones; every form must give the
    # oracle's results, and the tuner (sw_form 0) times them all on the first batch
    rng = np.random.default_rng(100 + bw)
    qs, ts = random_tasks(rng, 9000 if bw < 64 else 3000, bw, max_len=300)
    sc = (2, 4, 4, 2, 1, bw)
    W = 2 * bw + 1
    try:
        for tb in (False, True):
            exp = port.align(qs, ts, tb, sc)
            for form in (1, 2, 3, 0):
                ctx.set_option("sw_form", form)
                check_same(ctx.align(qs, ts, tb, D.ScoreParams(*sc)), exp, tb)
    finally:
        ctx.set_option("sw_form", 0)
    tuned = [t for t in ctx.sw_tuning() if t["W"] == W]
    assert tuned
    for t in tuned:
        assert t["ms_intra"] > 0 and t["ms_narrow"] > 0
        assert (t["ms_inter"] > 0) == (W != 129)
        timed = {f: ms for f, ms in enumerate((t["ms_inter"], t["ms_intra"], t["ms_narrow"])) if ms > 0}
        if t["tasks"] >= 4096:
            assert t["form"] == min(timed, key=timed.get)  # the fastest form was chosen
        else:  # too small a sample to time: the width's first form
            assert t["form"] == min(timed)
        assert t["lanes_per_pair"] == {0: 1, 1: (W - 1) // 32, 2: (W - 1) // 16}[t["form"]]
