"""TEST INFRASTRUCTURE ONLY — the oracle of the mapping path.

Two CPU implementations with one Python API, used by tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline leg to compare the CUDA path against, never by the product:

* :class:`Port` — ``_oracle.so``, our plain-C restatement of the reference's algorithm
  (dnaln_oracle.c, each function citing the dnaln lines it follows);
* :class:`Reference` — ``_ref/libdnaln_ref.so``, the reference itself compiled from its
  own sources by oracle/Makefile, driven through ref_shim.cpp.

Parity of Port with Reference is pinned by tests/test_oracle.py and by the fixtures in
tests/golden/ (made by tests/golden/make_golden.py from the Reference).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_SO = HERE / "_oracle.so"
REF_SO = HERE / "_ref" / "libdnaln_ref.so"
REF_BIN = HERE / "_ref" / "dnaln"

P = C.c_void_p
i32, i64, u32, u64 = C.c_int32, C.c_int64, C.c_uint32, C.c_uint64


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


class _ScoreP(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("match", "mismatch", "gap_open", "gap_ext", "ambig", "bw")]


class _ChainP(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("max_gap", "band", "lookback", "min_score", "min_anchors")]


class _MapP(C.Structure):
    _fields_ = [("k", C.c_int32), ("w", C.c_int32), ("max_occ", C.c_int32), ("max_cand", C.c_int32),
                ("min_aln_score", C.c_int32), ("pri_ratio", C.c_double), ("sc", _ScoreP), ("ch", _ChainP)]


def _concat(seqs):
    lens = np.array([len(s) for s in seqs], dtype=np.int32)
    off = np.zeros(len(seqs), dtype=np.int64)
    if len(seqs) > 1:
        off[1:] = np.cumsum(lens[:-1])
    buf = np.concatenate([np.asarray(s, np.uint8) for s in seqs]) if len(seqs) and lens.sum() else np.zeros(1, np.uint8)
    return np.ascontiguousarray(buf), off, lens


def score_tuple(sp) -> tuple:
    """(match, mismatch, gap_open, gap_ext, ambig, bw) from a tuple or a ScoreParams-like object."""
    if isinstance(sp, tuple):
        return sp
    return (sp.match, sp.mismatch, sp.gap_open, sp.gap_ext, sp.ambig, sp.bw)


def map_tuple(p) -> dict:
    """Plain dict of mapping parameters from a dnaln_b200 MapParams-like object."""
    return dict(k=p.k, w=p.w, max_occ=p.max_occ, max_cand=p.max_cand, min_aln_score=p.min_aln_score,
                pri_ratio=p.pri_ratio, sc=score_tuple(p.sc),
                ch=(p.ch.max_gap, p.ch.band, p.ch.lookback, p.ch.min_score, p.ch.min_anchors))


class Port:
    """The plain-C restatement (oracle/dnaln_oracle.c)."""

    def __init__(self):
        if not PORT_SO.exists():
            raise RuntimeError(f"{PORT_SO} missing: run `make -C oracle oracle`")
        L = C.CDLL(str(PORT_SO))
        L.or_hash64.restype = u64
        L.or_hash64.argtypes = [u64, u64]
        L.or_fnv1a.restype = u32
        L.or_fnv1a.argtypes = [P, i64]
        L.or_sketch.restype = i64
        L.or_sketch.argtypes = [P, u32, C.c_int, C.c_int, u32, P, P, P, i64]
        L.or_index_build.restype = P
        L.or_index_build.argtypes = [P, u64, P, P, i32, C.c_int, C.c_int]
        L.or_index_free.argtypes = [P]
        L.or_index_stats.argtypes = [P, P]
        L.or_index_export.argtypes = [P, P, P, P, P]
        L.or_index_lookup.restype = u32
        L.or_index_lookup.argtypes = [P, u64, C.POINTER(u32)]
        L.or_chain.restype = i64
        L.or_chain.argtypes = [P, P, P, i64, C.c_int, C.POINTER(_ChainP), P, P, P, P, P, P, i64]
        L.or_align.restype = i32
        L.or_align.argtypes = [P, i32, P, i32, C.c_int, C.POINTER(_ScoreP), P, P, i32]
        L.or_map.restype = i64
        L.or_map.argtypes = [P, P, P, P, i32, P, P, P, P, P, i64, C.POINTER(_MapP), P, P, P, i64]
        L.or_chain_cost_mismatches.restype = i64
        L.or_chain_cost_mismatches.argtypes = [C.c_int, C.c_int, C.c_int]
        self.L = L

    kind = "port"

    def hash64(self, key: int, mask: int) -> int:
        return int(self.L.or_hash64(key, mask))

    def sketch(self, seq: np.ndarray, k: int, w: int, offset: int = 0):
        seq = np.ascontiguousarray(seq, np.uint8)
        cap = len(seq) + 1
        h, p, s = np.zeros(cap, np.uint64), np.zeros(cap, np.uint32), np.zeros(cap, np.uint32)
        n = self.L.or_sketch(_p(seq), len(seq), k, w, offset, _p(h), _p(p), _p(s), cap)
        assert n >= 0
        return h[:n], p[:n], s[:n]

    def index(self, genome, k: int = 15, w: int = 10) -> "_PortIndex":
        return _PortIndex(self, genome, k, w)

    def chain(self, rpos, qpos, strand, k: int, cp=(5000, 16, 50, 20, 2)):
        rpos = np.ascontiguousarray(rpos, np.uint32).copy()
        qpos = np.ascontiguousarray(qpos, np.int32).copy()
        strand = np.ascontiguousarray(strand, np.uint32).copy()
        n = len(rpos)
        cap = max(n, 1)
        o = dict(score=np.zeros(cap, np.int32), strand=np.zeros(cap, np.uint32), n_anchors=np.zeros(cap, np.int32),
                 dmin=np.zeros(cap, np.int64), dmax=np.zeros(cap, np.int64), rpos=np.zeros(cap, np.uint32))
        p = _ChainP(*cp)
        m = self.L.or_chain(_p(rpos), _p(qpos), _p(strand), n, k, C.byref(p), _p(o["score"]), _p(o["strand"]),
                            _p(o["n_anchors"]), _p(o["dmin"]), _p(o["dmax"]), _p(o["rpos"]), cap)
        return (rpos, qpos, strand), {kk: v[:m] for kk, v in o.items()}

    def align(self, queries, targets, traceback: bool, sp=(2, 4, 4, 2, 1, 16)):
        """List of (score, qb, qe, tb, te, nm, cigar ops array)."""
        spp = _ScoreP(*score_tuple(sp))
        out = []
        for q, t in zip(queries, targets):
            q = np.ascontiguousarray(q, np.uint8)
            t = np.ascontiguousarray(t, np.uint8)
            res = np.zeros(6, np.int32)
            cig = np.zeros(2 * len(q) + 2, np.uint32)
            n = self.L.or_align(_p(q) if len(q) else _p(np.zeros(1, np.uint8)), len(q),
                                _p(t) if len(t) else _p(np.zeros(1, np.uint8)), len(t), int(traceback),
                                C.byref(spp), _p(res), _p(cig), len(cig))
            assert n >= 0
            out.append((*map(int, res), cig[:n].copy()))
        return out

    def map(self, idx: "_PortIndex", reads, params) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(records n x 7 [contig, pos, rev, mapq, score, nm, n_cand], cigar ops, cigar offsets n+1)."""
        mp = map_tuple(params)
        p = _MapP(mp["k"], mp["w"], mp["max_occ"], mp["max_cand"], mp["min_aln_score"], mp["pri_ratio"],
                  _ScoreP(*mp["sc"]), _ChainP(*mp["ch"]))
        n = len(reads)
        rec = np.zeros((max(n, 1), 7), np.int64)
        cap = int(np.sum(2 * reads.seq_len.astype(np.int64) + 3)) + 1
        cig = np.zeros(cap, np.uint32)
        co = np.zeros(n + 1, np.int64)
        g = idx.genome
        off = np.ascontiguousarray(reads.seq_off[:-1])
        lens = reads.seq_len  # keep the arrays alive across the call
        tot = self.L.or_map(idx.h, _p(g.codes), _p(g.contig_off), _p(g.contig_len), g.n_contigs, _p(reads.seq),
                            _p(off), _p(lens), _p(reads.names), _p(reads.name_off), n, C.byref(p), _p(rec), _p(cig),
                            _p(co), cap)
        assert tot >= 0
        return rec[:n], cig[:tot], co

    def chain_cost_mismatches(self, k_max: int = 28, dd_max: int = 2000) -> int:
        return int(self.L.or_chain_cost_mismatches(4, k_max, dd_max))


class _PortIndex:
    def __init__(self, port: Port, genome, k: int, w: int):
        self.port, self.genome, self.k, self.w = port, genome, k, w
        self.h = port.L.or_index_build(_p(genome.codes), len(genome.codes), _p(genome.contig_off),
                                       _p(genome.contig_len), genome.n_contigs, k, w)

    def __del__(self):
        try:
            self.port.L.or_index_free(self.h)
        except Exception:
            pass

    def stats(self) -> dict:
        out = np.zeros(5, np.uint64)
        self.port.L.or_index_stats(self.h, _p(out))
        return dict(zip(["n_keys", "n_positions", "max_count", "memory_bytes", "n_buckets"], map(int, out)))

    def export(self):
        st = self.stats()
        keys = np.zeros(st["n_buckets"], np.uint64)
        offs = np.zeros(st["n_buckets"], np.uint32)
        cnts = np.zeros(st["n_buckets"], np.uint32)
        pos = np.zeros(max(st["n_positions"], 1), np.uint32)
        self.port.L.or_index_export(self.h, _p(keys), _p(offs), _p(cnts), _p(pos))
        return keys, offs, cnts, pos[:st["n_positions"]]

    def lookup(self, h: int):
        off = u32()
        n = self.port.L.or_index_lookup(self.h, h, C.byref(off))
        return int(off.value), int(n)


class Reference:
    """The reference compiled from its own sources (oracle/_ref/libdnaln_ref.so)."""

    kind = "reference"

    def __init__(self):
        if not REF_SO.exists():
            raise RuntimeError(f"{REF_SO} missing: run `make -C oracle ref` where the reference sources are present")
        L = C.CDLL(str(REF_SO))
        L.ref_sketch.restype = i64
        L.ref_sketch.argtypes = [P, u32, C.c_int, C.c_int, u32, P, P, P, i64]
        L.ref_genome_new.restype = P
        L.ref_genome_new.argtypes = [P, u64, P, P, i32, P, P, C.c_int, C.c_int]
        L.ref_genome_free.argtypes = [P]
        L.ref_index_stats.argtypes = [P, P]
        L.ref_index_lookup.restype = u32
        L.ref_index_lookup.argtypes = [P, u64, P, u32]
        L.ref_chain.restype = i64
        L.ref_chain.argtypes = [P, P, P, i64, C.c_int, P, P, P, P, P, P, P, i64]
        L.ref_align.restype = i64
        L.ref_align.argtypes = [P, P, P, P, P, P, i64, C.c_int, P, C.c_int, P, P, P, i64]
        L.ref_map.restype = i64
        L.ref_map.argtypes = [P, P, P, P, P, P, P, i64, P, C.c_double, C.c_int, i64, P, P, P, i64, P, i64,
                              C.POINTER(i64)]
        L.ref_fnv1a.restype = u32
        L.ref_fnv1a.argtypes = [P, i64]
        L.ref_eval.restype = None
        L.ref_eval.argtypes = [P, P, P, P, P, P, i64, C.c_int, P]
        L.ref_read_records.restype = C.c_int
        L.ref_read_records.argtypes = [C.c_char_p, P, P, P, P, P, P, P]
        self.L = L

    def evaluate(self, rec, cig, co, truth_contig, truth_start, truth_rev, tol: int = 10) -> np.ndarray:
        """Evaluator::add over records (n x 7 as map returns them): [records, mapped, correct,
        mapped_at(0..60), wrong_at(0..60)] (cumulative over MAPQ >= q)."""
        out = np.zeros(3 + 2 * 61, np.uint64)
        rec = np.ascontiguousarray(rec, np.int64)
        cig = np.ascontiguousarray(cig, np.uint32) if len(cig) else np.zeros(1, np.uint32)
        tc = np.ascontiguousarray(truth_contig, np.int32)
        ts = np.ascontiguousarray(truth_start, np.int64)
        tr = np.ascontiguousarray(truth_rev, np.uint8)
        self.L.ref_eval(_p(rec), _p(cig), _p(np.ascontiguousarray(co, np.int64)), _p(tc), _p(ts), _p(tr), len(rec),
                        tol, _p(out))
        return out

    def read_records(self, path: str):
        """read_all_records of a FASTA/FASTQ file: (seq, seq_off, names, name_off, qual, qual_off)."""
        sz = np.zeros(4, np.int64)
        self.L.ref_read_records(path.encode(), _p(sz), None, None, None, None, None, None)
        n, sb, nb, qb = map(int, sz)
        seq, names, qual = np.zeros(max(sb, 1), np.uint8), np.zeros(max(nb, 1), np.uint8), np.zeros(max(qb, 1), np.uint8)
        so, no, qo = np.zeros(n + 1, np.int64), np.zeros(n + 1, np.int64), np.zeros(n + 1, np.int64)
        self.L.ref_read_records(path.encode(), _p(sz), _p(seq), _p(so), _p(names), _p(no), _p(qual), _p(qo))
        return seq[:sb], so, names[:nb], no, qual[:qb], qo

    def sketch(self, seq: np.ndarray, k: int, w: int, offset: int = 0):
        seq = np.ascontiguousarray(seq, np.uint8)
        cap = len(seq) + 1
        h, p, s = np.zeros(cap, np.uint64), np.zeros(cap, np.uint32), np.zeros(cap, np.uint32)
        n = self.L.ref_sketch(_p(seq), len(seq), k, w, offset, _p(h), _p(p), _p(s), cap)
        assert n >= 0
        return h[:n], p[:n], s[:n]

    def genome(self, g, k: int = 15, w: int = 10) -> "_RefGenome":
        return _RefGenome(self, g, k, w)

    def chain(self, rpos, qpos, strand, k: int, cp=(5000, 16, 50, 20, 2)):
        rpos = np.ascontiguousarray(rpos, np.uint32).copy()
        qpos = np.ascontiguousarray(qpos, np.int32).copy()
        strand = np.ascontiguousarray(strand, np.uint32).copy()
        n = len(rpos)
        cap = max(n, 1)
        o = dict(score=np.zeros(cap, np.int32), strand=np.zeros(cap, np.uint32), n_anchors=np.zeros(cap, np.int32),
                 dmin=np.zeros(cap, np.int64), dmax=np.zeros(cap, np.int64), rpos=np.zeros(cap, np.uint32))
        cpa = np.array(cp, np.int32)
        m = self.L.ref_chain(_p(rpos), _p(qpos), _p(strand), n, k, _p(cpa), _p(o["score"]), _p(o["strand"]),
                             _p(o["n_anchors"]), _p(o["dmin"]), _p(o["dmax"]), _p(o["rpos"]), cap)
        return (rpos, qpos, strand), {kk: v[:m] for kk, v in o.items()}

    def align(self, queries, targets, traceback: bool, sp=(2, 4, 4, 2, 1, 16), simd: bool = False):
        qb, qo, ql = _concat(queries)
        tb, to, tl = _concat(targets)
        n = len(queries)
        res = np.zeros((max(n, 1), 6), np.int32)
        cap = int(np.sum(2 * ql.astype(np.int64) + 1)) + 1
        cig = np.zeros(cap, np.uint32)
        co = np.zeros(n + 1, np.int64)
        spa = np.array(score_tuple(sp), np.int32)
        tot = self.L.ref_align(_p(qb), _p(qo), _p(ql), _p(tb), _p(to), _p(tl), n, int(traceback), _p(spa), int(simd),
                               _p(res), _p(cig), _p(co), cap)
        assert tot >= 0
        return [(*map(int, res[i]), cig[co[i]:co[i + 1]].copy()) for i in range(n)]

    def map(self, rg: "_RefGenome", reads, params, nthreads: int = 1, simd: bool = True, batch: int = 8192,
            want_sam: bool = False):
        """(records n x 7, cigar ops, cigar offsets n+1[, SAM body bytes])."""
        mp = map_tuple(params)
        arr = np.array([mp["k"], mp["w"], mp["max_occ"], mp["max_cand"], mp["min_aln_score"], int(simd), *mp["sc"],
                        *mp["ch"]], np.int32)
        n = len(reads)
        rec = np.zeros((max(n, 1), 7), np.int64)
        cap = int(np.sum(2 * reads.seq_len.astype(np.int64) + 3)) + 1
        cig = np.zeros(cap, np.uint32)
        co = np.zeros(n + 1, np.int64)
        sam_len = i64()
        sam = None
        sam_cap = 0
        if want_sam:
            sam_cap = int(len(reads.seq) * 2 + n * 200 + 1024)
            sam = np.zeros(sam_cap, np.uint8)
        off = np.ascontiguousarray(reads.seq_off[:-1])
        lens = reads.seq_len  # keep the arrays alive across the call
        tot = self.L.ref_map(rg.h, _p(reads.seq), _p(off), _p(lens), _p(reads.qual), _p(reads.names),
                             _p(reads.name_off), n, _p(arr), mp["pri_ratio"], nthreads, batch, _p(rec), _p(cig), _p(co),
                             cap, _p(sam), sam_cap, C.byref(sam_len))
        assert tot >= 0
        if want_sam:
            assert sam_len.value <= sam_cap
            return rec[:n], cig[:tot], co, sam[:sam_len.value].tobytes()
        return rec[:n], cig[:tot], co

    def time_map(self, rg: "_RefGenome", reads, params, nthreads: int, simd: bool = True, batch: int = 8192) -> float:
        """Wall seconds of Mapper::map over the reads with nthreads Mapper instances."""
        import time
        mp = map_tuple(params)
        arr = np.array([mp["k"], mp["w"], mp["max_occ"], mp["max_cand"], mp["min_aln_score"], int(simd), *mp["sc"],
                        *mp["ch"]], np.int32)
        n = len(reads)
        rec = np.zeros((max(n, 1), 7), np.int64)
        off = np.ascontiguousarray(reads.seq_off[:-1])
        lens = reads.seq_len
        t0 = time.perf_counter()
        tot = self.L.ref_map(rg.h, _p(reads.seq), _p(off), _p(lens), None, _p(reads.names), _p(reads.name_off), n,
                             _p(arr), mp["pri_ratio"], nthreads, batch, _p(rec), None, None, 0, None, 0, None)
        dt = time.perf_counter() - t0
        assert tot >= 0
        return dt


class _RefGenome:
    def __init__(self, ref: Reference, g, k: int, w: int):
        self.ref, self.g = ref, g
        names = [n.encode() for n in g.names]
        no = np.zeros(len(names) + 1, np.int64)
        no[1:] = np.cumsum([len(x) for x in names])
        nb = np.frombuffer(b"".join(names) or b"\0", np.uint8).copy()
        self.h = ref.L.ref_genome_new(_p(g.codes), len(g.codes), _p(g.contig_off), _p(g.contig_len), g.n_contigs,
                                      _p(nb), _p(no), k, w)

    def __del__(self):
        try:
            self.ref.L.ref_genome_free(self.h)
        except Exception:
            pass

    def stats(self) -> dict:
        out = np.zeros(4, np.uint64)
        self.ref.L.ref_index_stats(self.h, _p(out))
        return dict(zip(["n_keys", "n_positions", "max_count", "memory_bytes"], map(int, out)))

    def lookup(self, h: int) -> np.ndarray:
        buf = np.zeros(4096, np.uint32)
        n = self.ref.L.ref_index_lookup(self.h, h, _p(buf), len(buf))
        if n > len(buf):
            buf = np.zeros(n, np.uint32)
            n = self.ref.L.ref_index_lookup(self.h, h, _p(buf), len(buf))
        return buf[:n]


def available() -> dict:
    return {"port": PORT_SO.exists(), "reference": REF_SO.exists()}
