"""Index image files (dnaln_gpu_index_save / _load) and the upload of a host-built table
(dnaln_gpu_index_upload): an index that comes back from a file, or from the reference's
MinimizerIndex layout built on the host, maps every read exactly as the index built on the
device; files and tables that do not check out are refused before anything uses them."""
import numpy as np
import pytest

import dnaln_b200 as D
from dnaln_b200 import _native as N
from dnaln_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    g, reads, _ = synth.workload("small-1Mbp-10k-150bp", seed=3, n_reads=3000)
    return g, reads


def _same_index(ctx, a, b):
    ea, eb = ctx.index_export(a), ctx.index_export(b)
    for x, y in zip(ea, eb):
        assert np.array_equal(x, y)
    sa, sb = ctx.index_stats(a), ctx.index_stats(b)
    for kk in ("n_keys", "n_positions", "max_count", "memory_bytes", "n_buckets"):
        assert sa[kk] == sb[kk], kk


def _same_mapping(ctx, a, b, reads):
    p = D.default_map_params()
    ra, rb = ctx.map_batch(a, reads, p), ctx.map_batch(b, reads, p)
    assert np.array_equal(ra.records, rb.records)
    assert np.array_equal(ra.cigar, rb.cigar)


def test_image_round_trip(ctx, small, tmp_path):
    g, reads = small
    a = ctx.index_build(g, 15, 10)
    path = tmp_path / "small.dnbidx"
    try:
        ctx.index_save(a, path)
        assert not (tmp_path / "small.dnbidx.tmp").exists()
        b = ctx.index_load(path)
        try:
            _same_index(ctx, a, b)
            _same_mapping(ctx, a, b, reads)
        finally:
            ctx.index_free(b)
    finally:
        ctx.index_free(a)


def test_image_ragged_and_all_n(ctx, tmp_path):
    # contigs of 0, 3 and 40 bases, a contig of N only, N runs at the edges: the N runs
    # and the contig table come back as they were
    rng = np.random.default_rng(5)
    lens = [0, 3, 40, 2000, 500, 30000]
    parts = []
    for i, n in enumerate(lens):
        c = rng.integers(0, 4, n).astype(np.uint8)
        if n >= 40:
            c[:6] = 4
            c[-4:] = 4
        if i == 4:
            c[:] = 4
        parts.append(c)
    off = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
    g = D.Genome(np.concatenate(parts), off, np.array(lens, np.uint32))
    a = ctx.index_build(g, 12, 5)
    try:
        ctx.index_save(a, tmp_path / "r.img")
        b = ctx.index_load(tmp_path / "r.img")
        try:
            _same_index(ctx, a, b)
        finally:
            ctx.index_free(b)
    finally:
        ctx.index_free(a)


def _expect(code, fn, *args):
    with pytest.raises(D.DnalnError) as e:
        fn(*args)
    assert e.value.code == code, e.value


def test_image_refuses_damaged_files(ctx, small, tmp_path):
    g, _ = small
    a = ctx.index_build(g, 15, 10)
    good = tmp_path / "good.img"
    try:
        ctx.index_save(a, good)
    finally:
        ctx.index_free(a)
    blob = good.read_bytes()
    cases = {
        "flipped": bytearray(blob),
        "truncated": bytearray(blob[:-5]),
        "longer": bytearray(blob + b"\0"),
        "magic": bytearray(blob),
        "header": bytearray(blob),
    }
    cases["flipped"][len(blob) // 2] ^= 0x10           # a byte of the genome / table
    cases["magic"][0] ^= 0xFF
    cases["header"][16] = 99                           # k outside [4, 28]
    for name, data in cases.items():
        f = tmp_path / f"{name}.img"
        f.write_bytes(bytes(data))
        _expect(N.ERR_IO, ctx.index_load, f)
    _expect(N.ERR_IO, ctx.index_load, tmp_path / "absent.img")
    b = ctx.index_load(good)  # the context is still usable
    ctx.index_free(b)


def test_upload_of_host_table_maps_like_device_build(ctx, port, small):
    # the table the reference's build makes on the host (the oracle's restatement of
    # src/index.cpp:10-45), uploaded, against the one built on the device
    g, reads = small
    keys, offs, cnts, pos = port.index(g, 15, 10).export()
    a = ctx.index_build(g, 15, 10)
    b = ctx.index_upload(g, keys, offs, cnts, pos, 15, 10)
    try:
        _same_index(ctx, a, b)
        _same_mapping(ctx, a, b, reads)
    finally:
        ctx.index_free(a)
        ctx.index_free(b)


def test_upload_refuses_bad_tables(ctx, port, small):
    g, _ = small
    keys, offs, cnts, pos = port.index(g, 15, 10).export()
    full = np.nonzero(keys != np.uint64(2**64 - 1))[0]
    bad_off = offs.copy()
    bad_off[full[0]] = len(pos)                         # positions past the array
    bad_pos = pos.copy()
    bad_pos[0] = np.uint32(2 * len(g.codes) + 1)        # a position past the genome
    no_empty = np.arange(16, dtype=np.uint64)           # every bucket holds a key
    z16 = np.zeros(16, np.uint32)
    _expect(N.ERR_INVALID_ARG, ctx.index_upload, g, keys[:-1], offs[:-1], cnts[:-1], pos)  # not a power of two
    _expect(N.ERR_INVALID_ARG, ctx.index_upload, g, keys, bad_off, cnts, pos)
    _expect(N.ERR_INVALID_ARG, ctx.index_upload, g, keys, offs, cnts, bad_pos)
    _expect(N.ERR_INVALID_ARG, ctx.index_upload, g, no_empty, z16, z16, pos)
    _expect(N.ERR_INVALID_ARG, ctx.index_upload, g, keys, offs, cnts, pos, 3, 10)  # k below 4
