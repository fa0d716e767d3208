"""The allocation-free SW entry point, dnaln_gpu_align_noalloc, for callers that cannot call
cudaMalloc (a host framework that owns all device memory, a serving loop that must not
allocate per request). Called through the C ABI with device buffers the test owns, twice
in a row, and compared bit for bit with dnaln_gpu_align, the existing entry point.

Kept in a file of its own that is collected last, so that a run stopping at the first
failure has run every other test before it; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import dnaln_b200 as D
from dnaln_b200 import _native as N
from helpers import random_tasks

pytestmark = pytest.mark.gpu


def concat(seqs):
    lens = np.array([len(s) for s in seqs], np.int32)
    off = np.zeros(len(seqs), np.int64)
    off[1:] = np.cumsum(lens[:-1])
    buf = np.concatenate(seqs) if lens.sum() else np.zeros(1, np.uint8)
    return buf.astype(np.uint8), off, lens


def run_noalloc(qs, ts, sp, traceback=True, max_qlen=None, q_off_fix=None, expect=N.OK):
    """Calls the entry point on device copies of the tasks; q_off_fix (index, value)
    overwrites one query offset, to describe a task wrongly on purpose."""
    import torch
    qb, qo, ql = concat(qs)
    tb, to, tl = concat(ts)
    if q_off_fix is not None:
        qo[q_off_fix[0]] = q_off_fix[1]
    n = len(qs)
    max_qlen = int(ql.max()) if max_qlen is None else max_qlen
    stride = 2 * max_qlen + 1
    dev = {k: torch.from_numpy(v).cuda() for k, v in dict(qb=qb, qo=qo, ql=ql, tb=tb, to=to, tl=tl).items()}
    out = torch.zeros(n * 40, dtype=torch.uint8, device="cuda")
    cig = torch.zeros(n * stride, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = N.lib().dnaln_gpu_align_noalloc(dev["qb"].data_ptr(), dev["qo"].data_ptr(), dev["ql"].data_ptr(),
                                         dev["tb"].data_ptr(), dev["to"].data_ptr(), dev["tl"].data_ptr(), n, max_qlen,
                                         int(traceback), C.byref(sp), out.data_ptr(), cig.data_ptr(), stride,
                                         stream.cuda_stream)
    assert rc == expect, f"dnaln_gpu_align_noalloc returned {N.ERR_NAMES.get(rc, rc)}"
    torch.cuda.synchronize()
    res = out.cpu().numpy().view(D.ALIGN_RESULT_DTYPE)
    return res, cig.cpu().numpy().view(np.uint32)


def assert_same(qs, ts, sp, ctx, rows=None, **kw):
    """rows: the tasks to compare (default all)."""
    exp = ctx.align(qs, ts, True, sp)
    res, cig = run_noalloc(qs, ts, sp, **kw)
    rows = np.arange(len(qs)) if rows is None else np.asarray(rows)
    for f in ("score", "qb", "qe", "tb", "te", "nm", "cigar_len"):
        assert np.array_equal(res[f][rows], exp.results[f][rows]), f
    for i in rows:
        o, m = int(res["cigar_off"][i]), int(res["cigar_len"][i])
        assert np.array_equal(cig[o:o + m], exp.cigar_of(i)), i
    return res


@pytest.mark.parametrize("scheme", [(2, 4, 4, 2, 1, 16), (2, 4, 4, 2, 1, 64), (1, 4, 6, 1, 1, 8)])
def test_noalloc_matches_align_on_two_calls_in_a_row(ctx, scheme):
    sp = D.ScoreParams(*scheme)
    rng = np.random.default_rng(scheme[5])
    qs1, ts1 = random_tasks(rng, 700, scheme[5])
    # longer queries need more scratch per warp: at bw 64 this call runs as two launches
    qs2, ts2 = random_tasks(rng, 1000, scheme[5], max_len=1000)
    assert_same(qs1, ts1, sp, ctx)
    assert_same(qs2, ts2, sp, ctx)  # second call reuses the static scratch left by the first


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    sp = D.ScoreParams(2, 4, 4, 2, 1, 1000)
    z = torch.zeros(64, dtype=torch.uint8, device="cuda")
    rc = N.lib().dnaln_gpu_align_noalloc(z.data_ptr(), z.data_ptr(), z.data_ptr(), z.data_ptr(), z.data_ptr(),
                                         z.data_ptr(), 1, 2_000_000, 1, C.byref(sp), z.data_ptr(), z.data_ptr(),
                                         4_000_001, None)
    assert rc == N.ERR_INVALID_ARG


def test_noalloc_score_only_matches_align(ctx):
    # without traceback only the score is computed; no CIGAR is written (cigar_len 0)
    sp = D.ScoreParams(2, 4, 4, 2, 1, 16)
    qs, ts = random_tasks(np.random.default_rng(5), 500, 16)
    exp = ctx.align(qs, ts, False, sp)
    res, _ = run_noalloc(qs, ts, sp, traceback=False)
    assert np.array_equal(res["score"], exp.results["score"])
    assert not res["cigar_len"].any()


def test_noalloc_refuses_a_task_described_wrongly_and_keeps_the_others(ctx):
    # a query longer than the stated maximum, then a negative query offset: the call
    # returns DNALN_ERR_INVALID_ARG, the task is aligned as empty, the others stand
    sp = D.ScoreParams(2, 4, 4, 2, 1, 16)
    qs, ts = random_tasks(np.random.default_rng(6), 300, 16, max_len=200)
    lens = np.array([len(q) for q in qs])
    long_one = int(np.argmax(lens))
    limit = int(lens[long_one]) - 1
    others = [i for i in range(len(qs)) if lens[i] <= limit]
    res = assert_same(qs, ts, sp, ctx, rows=others, max_qlen=limit, expect=N.ERR_INVALID_ARG)
    assert res["score"][long_one] == 0 and res["cigar_len"][long_one] == 0
    rest = [i for i in range(len(qs)) if i != 7]
    res = assert_same(qs, ts, sp, ctx, rows=rest, q_off_fix=(7, -5), expect=N.ERR_INVALID_ARG)
    assert res["score"][7] == 0
