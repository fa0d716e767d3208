"""dnaln_b200 — B200-native (sm_100a) read-mapping path of dnaln behind a C ABI.

Python mirror of the reference's interfaces for this path (names and argument meaning
follow dnaln's C++ API):

* :meth:`Context.sketch`      — ``sketch`` (src/minimizer.hpp:34), batched over sequences
* :meth:`Context.index_build` — ``MinimizerIndex::build`` (src/index.cpp:10-45), HBM-resident
* :meth:`Context.lookup`      — ``MinimizerIndex::lookup`` (src/index.hpp:24-38), batched
* :meth:`Context.chain`       — ``Chainer::run`` (src/chain.hpp:41), batched over anchor sets
* :meth:`Context.align`       — ``Aligner::align`` (src/align.hpp:62-68)
* :meth:`Context.map_batch`   — ``Mapper::map`` (src/mapper.cpp:75-223)
* :func:`sam_format`          — ``Mapper::append_sam`` (src/mapper.cpp:231-270)
* :class:`dnaln_b200.serve.Server` — request server with continuous batching (no
  reference counterpart)

Every call goes to the CUDA library; there is no CPU fallback. Errors raise
:class:`DnalnError` carrying the C status code and message.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from ._native import (ALIGN_RESULT_DTYPE, MAP_RECORD_DTYPE, ChainParams, MapParams, ScoreParams, Stats, lib, ptr)

__all__ = ["Context", "Genome", "ReadBatch", "DnalnError", "ScoreParams", "ChainParams", "MapParams",
           "default_map_params", "sam_format", "parse_reads", "evaluate", "fnv1a", "lib", "MAP_RECORD_DTYPE", "ALIGN_RESULT_DTYPE",
           "cigar_to_string"]

CIGAR_OPS = "MIDNSHP=X"


class DnalnError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dnaln_b200 error {N.ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


def cigar_to_string(ops) -> str:
    """BAM-encoded ops -> CIGAR text ("*" when empty), src/common.cpp:21-29."""
    if len(ops) == 0:
        return "*"
    return "".join(f"{int(c) >> 4}{CIGAR_OPS[int(c) & 0xF]}" for c in ops)


def default_map_params(bw: int = 16, **kw) -> MapParams:
    """The reference's defaults (src/mapper.hpp:25-35, src/align.hpp:34-40, src/chain.hpp:30-36)."""
    p = MapParams()
    p.k, p.w, p.max_occ, p.max_cand, p.pri_ratio, p.min_aln_score = 15, 10, 500, 10, 0.5, 40
    p.sc = ScoreParams(2, 4, 4, 2, 1, bw)
    p.ch = ChainParams(5000, 16, 50, 20, 2)
    for k, v in kw.items():
        if hasattr(p.sc, k) and k in {f[0] for f in ScoreParams._fields_}:
            setattr(p.sc, k, v)
        else:
            setattr(p, k, v)
    return p


def fnv1a(name: bytes) -> int:
    return int(lib().dnaln_fnv1a(name, len(name)))


@dataclass
class Genome:
    """Concatenated base codes (A0 C1 G2 T3 N4) with a contig table (src/reference.hpp:16-30)."""
    codes: np.ndarray
    contig_off: np.ndarray
    contig_len: np.ndarray
    names: list[str] = field(default_factory=list)

    def __post_init__(self):
        self.codes = np.ascontiguousarray(self.codes, dtype=np.uint8)
        self.contig_off = np.ascontiguousarray(self.contig_off, dtype=np.uint64)
        self.contig_len = np.ascontiguousarray(self.contig_len, dtype=np.uint32)
        if not self.names:
            self.names = [f"chr{i + 1}" for i in range(len(self.contig_off))]

    @property
    def n_contigs(self) -> int:
        return len(self.contig_off)

    def name_buffers(self) -> tuple[np.ndarray, np.ndarray]:
        raw = [n.encode() for n in self.names]
        off = np.zeros(len(raw) + 1, dtype=np.int64)
        off[1:] = np.cumsum([len(r) for r in raw])
        return np.frombuffer(b"".join(raw) or b"\0", dtype=np.uint8).copy(), off


@dataclass
class ReadBatch:
    """Reads as concatenated ASCII with offsets (n+1 entries), like a SeqRecord batch."""
    seq: np.ndarray       # uint8 ASCII
    seq_off: np.ndarray   # int64, n+1
    names: np.ndarray     # uint8
    name_off: np.ndarray  # int64, n+1
    qual: np.ndarray | None = None  # uint8, same offsets as seq (None = '*')
    qual_off: np.ndarray | None = None  # int64, n+1: qualities with offsets of their own (mixed FASTA/FASTQ)

    def __post_init__(self):
        self.seq = np.ascontiguousarray(self.seq, dtype=np.uint8)
        self.seq_off = np.ascontiguousarray(self.seq_off, dtype=np.int64)
        self.names = np.ascontiguousarray(self.names, dtype=np.uint8)
        self.name_off = np.ascontiguousarray(self.name_off, dtype=np.int64)
        self._hash = None

    @classmethod
    def from_lists(cls, seqs: list[bytes], names: list[bytes], qual: list[bytes] | None = None) -> "ReadBatch":
        so = np.zeros(len(seqs) + 1, dtype=np.int64)
        so[1:] = np.cumsum([len(s) for s in seqs])
        no = np.zeros(len(names) + 1, dtype=np.int64)
        no[1:] = np.cumsum([len(s) for s in names])
        q = np.frombuffer(b"".join(qual), dtype=np.uint8).copy() if qual else None
        return cls(np.frombuffer(b"".join(seqs) or b"\0", dtype=np.uint8).copy(), so,
                   np.frombuffer(b"".join(names) or b"\0", dtype=np.uint8).copy(), no, q)

    def __len__(self) -> int:
        return len(self.seq_off) - 1

    @property
    def seq_len(self) -> np.ndarray:
        return np.diff(self.seq_off).astype(np.int32)

    def name(self, i: int) -> bytes:
        return self.names[self.name_off[i]:self.name_off[i + 1]].tobytes()

    def read(self, i: int) -> bytes:
        return self.seq[self.seq_off[i]:self.seq_off[i + 1]].tobytes()

    def name_hash(self) -> np.ndarray:
        if self._hash is None:
            h = np.zeros(len(self), dtype=np.uint32)
            if len(self):
                lib().dnaln_fnv1a_batch(ptr(self.names), ptr(self.name_off), len(self), ptr(h))
            self._hash = h
        return self._hash

    def slice(self, a: int, b: int) -> "ReadBatch":
        so = self.seq_off[a:b + 1] - self.seq_off[a]
        no = self.name_off[a:b + 1] - self.name_off[a]
        qo = self.seq_off if self.qual_off is None else self.qual_off
        q = None if self.qual is None else self.qual[qo[a]:qo[b]].copy()
        qn = None if self.qual_off is None else self.qual_off[a:b + 1] - self.qual_off[a]
        return ReadBatch(self.seq[self.seq_off[a]:self.seq_off[b]].copy(), so,
                         self.names[self.name_off[a]:self.name_off[b]].copy(), no, q, qn)


@dataclass
class MapResult:
    records: np.ndarray  # MAP_RECORD_DTYPE
    cigar: np.ndarray    # uint32 BAM ops

    def cigar_of(self, i: int) -> np.ndarray:
        r = self.records[i]
        return self.cigar[r["cigar_off"]:r["cigar_off"] + r["cigar_len"]]


@dataclass
class AlignOut:
    results: np.ndarray  # ALIGN_RESULT_DTYPE
    cigar: np.ndarray

    def cigar_of(self, i: int) -> np.ndarray:
        r = self.results[i]
        return self.cigar[r["cigar_off"]:r["cigar_off"] + r["cigar_len"]]


def _concat(seqs: list[np.ndarray]) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    lens = np.array([len(s) for s in seqs], dtype=np.int32)
    off = np.zeros(len(seqs), dtype=np.int64)
    if len(seqs) > 1:
        off[1:] = np.cumsum(lens[:-1], dtype=np.int64)
    buf = np.concatenate([np.asarray(s, dtype=np.uint8) for s in seqs]) if seqs and lens.sum() else np.zeros(1, np.uint8)
    return np.ascontiguousarray(buf), off, lens


class Context:
    """One CUDA context + stream on `device` (dnaln_gpu_ctx_create); not thread-safe."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        h = C.c_void_p()
        rc = self._lib.dnaln_gpu_ctx_create(device, C.byref(h))
        if rc != N.OK:
            raise DnalnError(rc, "cannot create a context (no CUDA device?)")
        self._h = h
        self.device = device

    # -- plumbing -----------------------------------------------------------------------
    def _check(self, rc: int) -> None:
        if rc != N.OK:
            raise DnalnError(rc, self._lib.dnaln_gpu_last_error(self._h).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.dnaln_gpu_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def set_stream(self, stream_ptr: int | None) -> None:
        self._check(self._lib.dnaln_gpu_set_stream(self._h, stream_ptr))

    def stats(self) -> dict:
        s = Stats()
        self._check(self._lib.dnaln_gpu_get_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in Stats._fields_}

    def reset_stats(self) -> None:
        self._check(self._lib.dnaln_gpu_reset_stats(self._h))

    def set_kernel_trace(self, on: bool, only: str | None = None) -> None:
        """Times every kernel launch (or only those of kernel `only`) with a CUDA event pair
        on its stream."""
        self._check(self._lib.dnaln_gpu_set_kernel_trace(self._h, 1 if on else 0,
                                                         only.encode() if only else None))

    def kernel_times(self) -> dict:
        """{kernel name: (launches, total ms)} since the last reset_stats()."""
        n = C.c_int32()
        self._check(self._lib.dnaln_gpu_kernel_times(self._h, None, 0, C.byref(n)))
        arr = (N.KernelTime * max(n.value, 1))()
        self._check(self._lib.dnaln_gpu_kernel_times(self._h, arr, n.value, C.byref(n)))
        return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].ms)) for i in range(n.value)}

    def set_option(self, name: str, value: int) -> None:
        """Tuning switch (sub_batch, warp_seed_only, dir_cap_bytes); results do not change."""
        self._check(self._lib.dnaln_gpu_set_option(self._h, name.encode(), int(value)))

    def seed_tuning(self) -> dict:
        """The reads-per-block choice of the thread-per-read seeding kernel (dnaln_gpu_seed_tuning)."""
        t = N.SeedTuning()
        self._check(self._lib.dnaln_gpu_seed_tuning(self._h, C.byref(t)))
        return {f: getattr(t, f) for f, _ in N.SeedTuning._fields_}

    def sw_tuning(self) -> list[dict]:
        """The SW kernel forms chosen so far (dnaln_gpu_sw_tuning)."""
        n = C.c_int32()
        self._check(self._lib.dnaln_gpu_sw_tuning(self._h, None, 0, C.byref(n)))
        arr = (N.SwTuning * max(n.value, 1))()
        self._check(self._lib.dnaln_gpu_sw_tuning(self._h, arr, n.value, C.byref(n)))
        return [{f: getattr(arr[i], f) for f, _ in N.SwTuning._fields_} for i in range(n.value)]

    def set_sub_batch(self, reads: int) -> None:
        """Reads per pipelined sub-batch of map_batch (0 = the whole batch at once)."""
        self._check(self._lib.dnaln_gpu_set_sub_batch(self._h, int(reads)))

    # -- index --------------------------------------------------------------------------
    def index_build(self, g: Genome, k: int = 15, w: int = 10) -> int:
        iid = C.c_int32()
        self._check(self._lib.dnaln_gpu_index_build(self._h, ptr(g.codes), len(g.codes), ptr(g.contig_off),
                                                    ptr(g.contig_len), g.n_contigs, k, w, C.byref(iid)))
        return iid.value

    def index_stats(self, iid: int) -> dict:
        out = np.zeros(6, dtype=np.uint64)
        self._check(self._lib.dnaln_gpu_index_stats(self._h, iid, ptr(out)))
        return dict(zip(["n_keys", "n_positions", "max_count", "memory_bytes", "n_buckets", "device_bytes"],
                        map(int, out)))

    def index_export(self, iid: int):
        st = self.index_stats(iid)
        nb, npos = st["n_buckets"], st["n_positions"]
        keys = np.zeros(nb, np.uint64)
        offs = np.zeros(nb, np.uint32)
        cnts = np.zeros(nb, np.uint32)
        pos = np.zeros(max(npos, 1), np.uint32)
        self._check(self._lib.dnaln_gpu_index_export(self._h, iid, ptr(keys), ptr(offs), ptr(cnts), ptr(pos)))
        return keys, offs, cnts, pos[:npos]

    def index_free(self, iid: int) -> None:
        self._check(self._lib.dnaln_gpu_index_free(self._h, iid))

    def index_save(self, iid: int, path) -> None:
        """Writes index `iid` with its genome as an image file (dnaln_gpu_index_save)."""
        self._check(self._lib.dnaln_gpu_index_save(self._h, iid, os.fsencode(path)))

    def index_load(self, path) -> int:
        """A new resident index from an image file written by index_save (checked, no rebuild)."""
        iid = C.c_int32()
        self._check(self._lib.dnaln_gpu_index_load(self._h, os.fsencode(path), C.byref(iid)))
        return iid.value

    def index_upload(self, g: Genome, keys, offsets, counts, positions, k: int = 15, w: int = 10) -> int:
        """A new resident index from a bucket table built on the host in the reference's layout
        (MinimizerIndex, src/index.hpp:49-56): keys (~0 = empty) / offsets / counts of a power-of-two
        number of buckets into positions (pos << 1 | strand)."""
        keys = np.ascontiguousarray(keys, np.uint64)
        offsets = np.ascontiguousarray(offsets, np.uint32)
        counts = np.ascontiguousarray(counts, np.uint32)
        positions = np.ascontiguousarray(positions, np.uint32)
        if not (len(keys) == len(offsets) == len(counts)):
            raise ValueError("keys, offsets and counts must have one entry per bucket")
        iid = C.c_int32()
        self._check(self._lib.dnaln_gpu_index_upload(
            self._h, ptr(g.codes), len(g.codes), ptr(g.contig_off), ptr(g.contig_len), g.n_contigs, k, w, ptr(keys),
            ptr(offsets), ptr(counts), len(keys), ptr(positions) if len(positions) else None, len(positions),
            C.byref(iid)))
        return iid.value

    def index_attach(self, src: "Context", iid: int) -> int:
        """Shares index `iid` of context `src` (same device) with this context, no copy."""
        out = C.c_int32()
        self._check(self._lib.dnaln_gpu_index_attach(self._h, src.handle, iid, C.byref(out)))
        return out.value

    # -- stages -------------------------------------------------------------------------
    def sketch(self, seqs: list[np.ndarray], k: int, w: int, pos_offset: list[int] | None = None):
        """Minimizers of each code sequence: list of (hash u64, pos u32, strand u32) arrays."""
        buf, off, lens = _concat(seqs)
        n = len(seqs)
        ext = max(int(buf.size), 1)
        h = np.zeros(ext, np.uint64)
        p = np.zeros(ext, np.uint32)
        s = np.zeros(ext, np.uint32)
        cnt = np.zeros(max(n, 1), np.int32)
        po = None if pos_offset is None else np.ascontiguousarray(pos_offset, dtype=np.uint32)
        self._check(self._lib.dnaln_gpu_sketch(self._h, ptr(buf), ptr(off), ptr(lens), ptr(po), n, k, w, ptr(h),
                                               ptr(p), ptr(s), ptr(cnt)))
        return [(h[o:o + c].copy(), p[o:o + c].copy(), s[o:o + c].copy()) for o, c in zip(off, cnt[:n])]

    def lookup(self, iid: int, hashes: np.ndarray):
        hashes = np.ascontiguousarray(hashes, dtype=np.uint64)
        off = np.zeros(max(len(hashes), 1), np.uint32)
        cnt = np.zeros(max(len(hashes), 1), np.uint32)
        self._check(self._lib.dnaln_gpu_lookup(self._h, iid, ptr(hashes), len(hashes), ptr(off), ptr(cnt)))
        return off[:len(hashes)], cnt[:len(hashes)]

    def chain(self, sets: list[tuple[np.ndarray, np.ndarray, np.ndarray]], k: int, p: ChainParams | None = None):
        """Chainer::run per anchor set (rpos, qpos, strand). Returns, per set, the sorted
        anchors and a dict of chain columns (score, strand, n_anchors, dmin, dmax, rpos)."""
        p = p or ChainParams(5000, 16, 50, 20, 2)
        sizes = np.array([len(s[0]) for s in sets], dtype=np.int64)
        so = np.zeros(len(sets) + 1, np.int64)
        so[1:] = np.cumsum(sizes)
        tot = max(int(so[-1]), 1)
        rp = np.zeros(tot, np.uint32)
        qp = np.zeros(tot, np.int32)
        sd = np.zeros(tot, np.uint32)
        for i, (r, q, s) in enumerate(sets):
            rp[so[i]:so[i + 1]], qp[so[i]:so[i + 1]], sd[so[i]:so[i + 1]] = r, q, s
        outs = dict(score=np.zeros(tot, np.int32), strand=np.zeros(tot, np.uint32), n_anchors=np.zeros(tot, np.int32),
                    dmin=np.zeros(tot, np.int64), dmax=np.zeros(tot, np.int64), rpos=np.zeros(tot, np.uint32))
        cnt = np.zeros(max(len(sets), 1), np.int32)
        self._check(self._lib.dnaln_gpu_chain(self._h, ptr(rp), ptr(qp), ptr(sd), ptr(so), len(sets), k, C.byref(p),
                                              ptr(outs["score"]), ptr(outs["strand"]), ptr(outs["n_anchors"]),
                                              ptr(outs["dmin"]), ptr(outs["dmax"]), ptr(outs["rpos"]), ptr(cnt)))
        res = []
        for i in range(len(sets)):
            a, b = so[i], so[i + 1]
            m = int(cnt[i])
            res.append(((rp[a:b].copy(), qp[a:b].copy(), sd[a:b].copy()),
                        {kk: v[a:a + m].copy() for kk, v in outs.items()}))
        return res

    def align(self, queries: list[np.ndarray], targets: list[np.ndarray], traceback: bool,
              sp: ScoreParams | None = None) -> AlignOut:
        """Aligner::align over (query, target) code pairs."""
        sp = sp or ScoreParams(2, 4, 4, 2, 1, 16)
        qb, qo, ql = _concat(queries)
        tb, to, tl = _concat(targets)
        n = len(queries)
        res = np.zeros(max(n, 1), dtype=ALIGN_RESULT_DTYPE)
        cap = int(np.sum(2 * ql.astype(np.int64) + 1)) if traceback else 0
        cig = np.zeros(max(cap, 1), np.uint32)
        used = C.c_int64()
        self._check(self._lib.dnaln_gpu_align(self._h, ptr(qb), ptr(qo), ptr(ql), ptr(tb), ptr(to), ptr(tl), n,
                                              int(bool(traceback)), C.byref(sp), ptr(res), ptr(cig), cap,
                                              C.byref(used)))
        return AlignOut(res[:n], cig[:used.value])

    def map_batch(self, iid: int, reads: ReadBatch, p: MapParams | None = None) -> MapResult:
        """Mapper::map over one batch; host buffers in, records + CIGARs out."""
        p = p or default_map_params()
        n = len(reads)
        lens = reads.seq_len
        rec = np.zeros(max(n, 1), dtype=MAP_RECORD_DTYPE)
        cap = int(np.sum(2 * lens.astype(np.int64) + 3)) if n else 0
        cig = np.zeros(max(cap, 1), np.uint32)
        used = C.c_int64()
        off = np.ascontiguousarray(reads.seq_off[:-1])
        nh = reads.name_hash()
        self._check(self._lib.dnaln_gpu_map_batch(self._h, iid, ptr(reads.seq), ptr(off), ptr(lens), ptr(nh), n,
                                                  C.byref(p), ptr(rec), ptr(cig), cap, C.byref(used)))
        return MapResult(rec[:n], cig[:used.value])

    def map_submit(self, iid: int, reads: ReadBatch, p: MapParams | None = None) -> "MapTicket":
        """Queues Mapper::map over one batch and returns at once (dnaln_gpu_map_submit);
        map_wait(ticket) returns its MapResult. Batches run in submission order, the copies of
        one overlapping the kernels of the others."""
        p = p or default_map_params()
        n = len(reads)
        lens = np.ascontiguousarray(reads.seq_len)
        cap = int(np.sum(2 * lens.astype(np.int64) + 3)) if n else 0
        t = MapTicket(n=n, params=p, keep=[reads.seq, np.ascontiguousarray(reads.seq_off[:-1]), lens,
                                           reads.name_hash()],
                      records=np.zeros(max(n, 1), dtype=MAP_RECORD_DTYPE), cigar=np.zeros(max(cap, 1), np.uint32))
        tid = C.c_int64()
        seq, off, ln, nh = t.keep
        self._check(self._lib.dnaln_gpu_map_submit(self._h, iid, ptr(seq), ptr(off), ptr(ln), ptr(nh), n,
                                                   C.byref(t.params), ptr(t.records), ptr(t.cigar), cap,
                                                   C.byref(t.used), C.byref(tid)))
        t.ticket = tid.value
        return t

    def map_wait(self, t: "MapTicket") -> MapResult:
        self._check(self._lib.dnaln_gpu_map_wait(self._h, t.ticket))
        return MapResult(t.records[:t.n], t.cigar[:t.used.value])


@dataclass
class MapTicket:
    """A queued batch: keeps its host buffers alive until map_wait."""
    n: int
    params: MapParams
    keep: list
    records: np.ndarray
    cigar: np.ndarray
    used: C.c_int64 = field(default_factory=C.c_int64)
    ticket: int = 0


def parse_reads(text: bytes, threads: int = 0) -> ReadBatch:
    """FASTA/FASTQ text -> ReadBatch (SeqReader::next, src/seqio.cpp:59-80), on `threads`
    host threads (0 = all) for four-line FASTQ; raises DnalnError on malformed FASTQ."""
    buf = np.frombuffer(text, np.uint8) if len(text) else np.zeros(1, np.uint8)
    h = C.c_void_p()
    err = C.create_string_buffer(256)
    rc = lib().dnaln_parse_reads(ptr(buf), len(text), threads, C.byref(h), C.addressof(err), 256)
    if rc != N.OK:
        raise DnalnError(rc, err.value.decode(errors="replace"))
    try:
        n = C.c_int64()
        v = [C.c_void_p() for _ in range(8)]
        lib().dnaln_reads_view(h, C.byref(n), *[C.byref(x) for x in v])
        m = n.value

        def arr(p, dt, cnt):
            if cnt == 0 or not p.value:
                return np.zeros(cnt, dt)
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(np.ctypeslib.as_ctypes_type(dt))), (cnt,)).copy()
        so = arr(v[1], np.int64, m + 1)
        no = arr(v[4], np.int64, m + 1)
        seq = arr(v[0], np.uint8, int(so[-1]) if m else 0)
        names = arr(v[3], np.uint8, int(no[-1]) if m else 0)
        qual = None
        qo = None
        if v[5].value:
            qo = arr(v[6], np.int64, m + 1)
            qual = arr(v[5], np.uint8, int(qo[-1]) if m else 0)
            if np.array_equal(qo, so):
                qo = None
        rb = ReadBatch(seq if len(seq) else np.zeros(1, np.uint8), so, names if len(names) else np.zeros(1, np.uint8),
                       no, qual, qo)
        rb._hash = arr(v[7], np.uint32, m)
        return rb
    finally:
        lib().dnaln_reads_free(h)


def evaluate(res: MapResult, truth_contig, truth_start, truth_rev, tol: int = 10) -> dict:
    """Evaluator::add over a batch (src/evaluate.cpp:57-84): placed-correctly counts and the
    per-MAPQ mapped / wrong tallies."""
    tc = np.ascontiguousarray(truth_contig, np.int32)
    ts = np.ascontiguousarray(truth_start, np.int64)
    tr = np.ascontiguousarray(truth_rev, np.uint8)
    out = N.EvalCounts()
    rec = np.ascontiguousarray(res.records)
    cig = np.ascontiguousarray(res.cigar, np.uint32) if len(res.cigar) else np.zeros(1, np.uint32)
    rc = lib().dnaln_eval_records(ptr(rec), ptr(cig), ptr(tc), ptr(ts), ptr(tr), len(rec), tol, C.byref(out))
    if rc != N.OK:
        raise DnalnError(rc, "evaluation failed")
    mq = np.array(out.mapped_at_mapq, np.uint64)
    wq = np.array(out.wrong_at_mapq, np.uint64)
    return {"records": out.records, "mapped": out.mapped, "correct": out.correct,
            "placed_correctly": out.correct / max(out.records, 1),
            "mapq60_mapped": int(mq[60]), "mapq60_wrong": int(wq[60]), "mapped_at_mapq": mq, "wrong_at_mapq": wq}


def sam_format(reads: ReadBatch, res: MapResult, genome: Genome, threads: int = 1) -> bytes:
    """SAM body lines of a mapped batch (Mapper::append_sam, src/mapper.cpp:231-270), on
    `threads` host threads (0 = all)."""
    n = len(reads)
    if n == 0:
        return b""
    cn, co = genome.name_buffers()
    qual = reads.qual
    used = C.c_int64()
    # every array handed to C is bound to a local so that it outlives the call
    off = np.ascontiguousarray(reads.seq_off[:-1])
    lens = reads.seq_len
    recs = np.ascontiguousarray(res.records)
    cig = np.ascontiguousarray(res.cigar, dtype=np.uint32) if len(res.cigar) else np.zeros(1, np.uint32)
    args = [ptr(reads.seq), ptr(off), ptr(lens), ptr(reads.names), ptr(reads.name_off),
            ptr(qual) if qual is not None else None,
            (ptr(reads.qual_off) if reads.qual_off is not None else ptr(reads.seq_off)) if qual is not None else None,
            ptr(recs), ptr(cig), n, ptr(cn), ptr(co)]
    if threads != 1:
        est = int(2 * np.sum(lens.astype(np.int64)) + 512 * n + 4096)
        out = np.zeros(est, np.uint8)
        rc = lib().dnaln_sam_format_mt(*args, threads, ptr(out), est, C.byref(used))
        if rc == N.ERR_CAPACITY:
            out = np.zeros(used.value + 1, np.uint8)
            rc = lib().dnaln_sam_format_mt(*args, threads, ptr(out), used.value + 1, C.byref(used))
        if rc != N.OK:
            raise DnalnError(rc, "SAM formatting failed")
        return out[:used.value].tobytes()
    lib().dnaln_sam_format(*args, None, 0, C.byref(used))
    out = np.zeros(used.value + 1, np.uint8)
    rc = lib().dnaln_sam_format(*args, ptr(out), used.value + 1, C.byref(used))
    if rc != N.OK:
        raise DnalnError(rc, "SAM formatting failed")
    return out[:used.value].tobytes()
