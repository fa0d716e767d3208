"""Host-side parts of the path, no GPU needed: the C ABI library loads and exports every
function its headers declare; SAM formatting equals the reference's append_sam byte for
byte; FNV-1a tie-break hashes; the seeded workload generator; error codes without a GPU."""
import re
from pathlib import Path

import numpy as np
import pytest

import dnaln_b200 as D
from dnaln_b200 import _native as N
from dnaln_b200 import synth

ROOT = Path(__file__).resolve().parent.parent


def declared_functions(header: str):
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / header).read_text(), flags=re.S)
    return set(re.findall(r"\b(dnaln_\w+)\s*\(", text))


def test_library_exports_every_declared_function():
    assert sorted(h.name for h in (ROOT / "include").glob("*.h")) == ["dnaln_b200.h", "dnaln_synth.h"]
    for header, lib, sigs in [("dnaln_b200.h", N.lib(), N.SIGNATURES),
                              ("dnaln_synth.h", N.synth_lib(), N.SYNTH_SIGNATURES)]:
        names = declared_functions(header)
        assert len(names) >= 3
        for n in sorted(names):
            assert hasattr(lib, n), f"{n} declared in include/{header} but not exported"
        assert set(sigs) <= names
    assert len(declared_functions("dnaln_b200.h")) >= 20


def test_generator_library_is_separate_from_the_mapping_path():
    # a program that only generates workloads never loads the mapping library
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", str(N.SYNTH_LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.split() and ln.split()[-1].startswith("dnaln_")}
    assert exported == declared_functions("dnaln_synth.h")


def test_context_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(D.DnalnError) as e:
        D.Context(0)
    assert e.value.code == N.ERR_NO_DEVICE


def records_from_oracle(rec, cig, co):
    n = len(rec)
    out = np.zeros(n, dtype=D.MAP_RECORD_DTYPE)
    out["contig"], out["pos"], out["rev"], out["mapq"] = rec[:, 0], rec[:, 1], rec[:, 2], rec[:, 3]
    out["score"], out["nm"], out["n_cand"] = rec[:, 4], rec[:, 5], rec[:, 6]
    out["cigar_off"], out["cigar_len"] = co[:-1], np.diff(co)
    return D.MapResult(out, cig)


@pytest.mark.parametrize("wl,seed", [("small-1Mbp-10k-150bp", 7), ("repeat-2Mbp-20k-150bp", 3)])
def test_sam_format_matches_reference_append_sam(ref, wl, seed):
    g, reads, _ = synth.workload(wl, seed=seed, n_reads=3000, with_qual=True)
    p = D.default_map_params()
    rec, cig, co, sam = ref.map(ref.genome(g), reads, p, want_sam=True)
    assert D.sam_format(reads, records_from_oracle(rec, cig, co), g) == sam


def test_sam_format_edge_cases(ref):
    # unmapped reads, empty reads, lowercase/IUPAC bases in reverse-complemented SEQ
    g = synth.make_genome(synth.GenomeSpec(contig_len=50_000), 3)
    acgt = np.frombuffer(b"ACGTN", np.uint8)
    exact = acgt[g.codes[1000:1150]].tobytes()
    rc = exact[::-1].translate(bytes.maketrans(b"ACGT", b"TGCA"))
    seqs = [b"", b"ACGTNRYacgtn", exact, rc.lower(), rc[:70] + b"RYKM" + rc[74:], b"N" * 150]
    reads = D.ReadBatch.from_lists(seqs, [f"q{i}".encode() for i in range(len(seqs))],
                                   [bytes([33 + (i * 7 + j) % 40 for j in range(len(s))]) for i, s in enumerate(seqs)])
    p = D.default_map_params()
    rec, cig, co, sam = ref.map(ref.genome(g), reads, p, want_sam=True)
    assert D.sam_format(reads, records_from_oracle(rec, cig, co), g) == sam
    assert (rec[:, 0] >= 0).sum() >= 3


def test_fnv1a_matches_reference(ref):
    for s in [b"", b"a", b"sim_1", b"read/1 extra", bytes(range(256))]:
        assert D.fnv1a(s) == ref.L.ref_fnv1a(s, len(s))
    reads = D.ReadBatch.from_lists([b"A"] * 3, [b"x", b"sim_12345", b""])
    assert list(reads.name_hash()) == [D.fnv1a(b"x"), D.fnv1a(b"sim_12345"), D.fnv1a(b"")]


def test_generator_is_seeded_and_has_the_workload_statistics():
    g1 = synth.make_genome(synth.GENOME_1M, 5)
    g2 = synth.make_genome(synth.GENOME_1M, 5)
    g3 = synth.make_genome(synth.GENOME_1M, 6)
    assert np.array_equal(g1.codes, g2.codes) and not np.array_equal(g1.codes, g3.codes)
    frac = np.bincount(g1.codes, minlength=5) / len(g1.codes)
    assert abs(frac[1] - 0.254) < 0.003 and abs(frac[2] - 0.254) < 0.003 and frac[4] == 0
    r1, t1 = synth.make_reads(g1, synth.ReadsSpec(n_reads=2000), 9)
    r2, _ = synth.make_reads(g1, synth.ReadsSpec(n_reads=2000), 9)
    assert np.array_equal(r1.seq, r2.seq) and np.array_equal(r1.names, r2.names)
    assert set(r1.seq_len) == {150} and r1.name(0) == b"sim_1" and r1.name(1999) == b"sim_2000"
    assert 0.4 < t1.rev.mean() < 0.6
    # reads come from their truth locus: few differences against the forward genome
    acgt = np.frombuffer(b"ACGT", np.uint8)
    diffs = []
    for i in range(200):
        s = np.frombuffer(r1.read(i), np.uint8)
        if t1.rev[i]:
            s = np.frombuffer(r1.read(i)[::-1].translate(bytes.maketrans(b"ACGT", b"TGCA")), np.uint8)
        ref_seg = acgt[g1.codes[t1.start[i]:t1.start[i] + 150]]
        diffs.append((s[:40] != ref_seg[:40]).sum())
    assert np.mean(diffs) < 2


def test_repeat_and_mixed_generators():
    g = synth.make_genome(synth.GENOME_REPEAT_2M, 1)
    nfrac = (g.codes == 4).mean()
    assert 0.004 < nfrac < 0.006
    frac_gc = np.isin(g.codes, [1, 2]).sum() / (g.codes < 4).sum()
    assert abs(frac_gc - 0.42) < 0.01
    r, _ = synth.make_reads(g, synth.ReadsSpec(n_reads=3000, len_min=50, len_max=1000, len_dist=1), 2)
    L = r.seq_len
    assert L.min() >= 50 and L.max() <= 1000 and 150 < np.median(L) < 300
    assert not np.any(np.frombuffer(r.seq.tobytes(), np.uint8) == ord("N"))


def test_default_params_are_the_references():
    p = D.default_map_params()
    assert (p.k, p.w, p.max_occ, p.max_cand, p.min_aln_score) == (15, 10, 500, 10, 40)
    assert (p.sc.match, p.sc.mismatch, p.sc.gap_open, p.sc.gap_ext, p.sc.ambig, p.sc.bw) == (2, 4, 4, 2, 1, 16)
    assert (p.ch.max_gap, p.ch.band, p.ch.lookback, p.ch.min_score, p.ch.min_anchors) == (5000, 16, 50, 20, 2)
    assert p.pri_ratio == 0.5


def test_eval_records_matches_reference_evaluator(ref):
    # Evaluator::add (src/evaluate.cpp:57-84) on the reference mapper's own records of a
    # workload with repeats (multi-candidate reads, MAPQ < 60, some misplaced)
    g, reads, truth = synth.workload("repeat-2Mbp-20k-150bp", seed=9)
    p = D.default_map_params()
    rec, cig, co = ref.map(ref.genome(g), reads, p, nthreads=4)
    res = records_from_oracle(rec, cig, co)
    for tol in (10, 0, 1000):
        ours = D.evaluate(res, truth.contig, truth.start, truth.rev, tol)
        exp = ref.evaluate(rec, cig, co, truth.contig, truth.start, truth.rev, tol)
        assert (ours["records"], ours["mapped"], ours["correct"]) == tuple(int(x) for x in exp[:3])
        cum_m = np.cumsum(ours["mapped_at_mapq"][::-1])[::-1]
        cum_w = np.cumsum(ours["wrong_at_mapq"][::-1])[::-1]
        assert np.array_equal(cum_m, exp[3:64]) and np.array_equal(cum_w, exp[64:125])
    assert 0.9 < D.evaluate(res, truth.contig, truth.start, truth.rev)["placed_correctly"] <= 1.0
