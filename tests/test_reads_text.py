"""Host text paths of the mapping boundary: FASTA/FASTQ parsing (SeqReader::next,
src/seqio.cpp:59-80) on several threads against the reference's own reader, and SAM
formatting on several threads against the one-thread formatter (Mapper::append_sam)."""
import numpy as np
import pytest

import dnaln_b200 as D
from dnaln_b200 import synth


def ours(text: bytes, threads: int):
    rb = D.parse_reads(text, threads)
    n = len(rb)
    names = [rb.name(i) for i in range(n)]
    seqs = [rb.read(i) for i in range(n)]
    if rb.qual is None:
        quals = [b""] * n
    else:
        qo = rb.seq_off if rb.qual_off is None else rb.qual_off
        quals = [rb.qual[qo[i]:qo[i + 1]].tobytes() for i in range(n)]
    return names, seqs, quals, rb.name_hash()


def theirs(ref, text: bytes, tmp_path):
    path = tmp_path / "reads.txt"
    path.write_bytes(text)
    seq, so, names, no, qual, qo = ref.read_records(str(path))
    n = len(so) - 1
    return ([names[no[i]:no[i + 1]].tobytes() for i in range(n)], [seq[so[i]:so[i + 1]].tobytes() for i in range(n)],
            [qual[qo[i]:qo[i + 1]].tobytes() for i in range(n)])


CASES = {
    "crlf_and_junk": b"junk line\r\n@r1 desc\tmore\r\nACGTN\r\n+r1\r\nIIIII\r\n\r\nnot a record\n@r2\nacgu\n+\n@@@@\n",
    "fasta_multiline": b">c1 x\nACGT\nTTGA\n\n>c2\nNNNN\n>empty\n>c3\nA\n",
    "mixed": b"@q1\nACGT\n+\nIIII\n>f1\nGGGG\nCC\n@q2\nTT\n+\n#\n#\n",
    "empty_seq_fastq": b"@e\n\n+\n\n@f\nAC\n+\nII\n",
    "at_in_quality": b"@a\nAC\n+\n@I\n@b\nGT\n+\n@@\n",
    "no_final_newline": b"@a\nACGT\n+\nIIII",
    "header_only_at": b"@\nAC\n+\nII\n",
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("threads", [1, 4])
def test_edge_cases_match_reference_reader(ref, tmp_path, case, threads):
    text = CASES[case]
    n, s, q, h = ours(text, threads)
    rn, rs, rq = theirs(ref, text, tmp_path)
    assert (n, s, q) == (rn, rs, rq)
    assert list(h) == [D.fnv1a(x) for x in n]


def test_large_fastq_in_threads_matches_reference_reader(ref, tmp_path):
    g = synth.make_genome(synth.GenomeSpec(contig_len=300_000), 3)
    reads, _ = synth.make_reads(g, synth.ReadsSpec(n_reads=30_000, len_min=50, len_max=400, len_dist=2), 4,
                                with_qual=True)
    path = tmp_path / "r.fq"
    synth.write_fastq(reads, str(path))
    text = path.read_bytes()
    rn, rs, rq = theirs(ref, text, tmp_path)
    for threads in (1, 3, 16):
        n, s, q, h = ours(text, threads)
        assert n == rn and s == rs and q == rq, threads
        assert np.array_equal(h, reads.name_hash())
    # a junk line between records and a trailing blank line are skipped by both
    cut = text.index(b"\n@" + reads.name(15_000) + b"\n") + 1
    text2 = text[:cut] + b"stray line\n" + text[cut:] + b"\n\n"
    assert ours(text2, 8)[:3] == theirs(ref, text2, tmp_path)


def test_malformed_fastq_is_an_error_with_the_reference_message():
    with pytest.raises(D.DnalnError) as e:
        D.parse_reads(b"@r1\nACGT\n@r2\n", 1)
    assert "malformed FASTQ record 'r1'" in str(e.value)
    with pytest.raises(D.DnalnError) as e:
        D.parse_reads(b"@r1\nACGT\n+\nIII", 4)
    assert "quality length mismatch" in str(e.value)


def test_sam_format_threads_identical():
    g = synth.make_genome(synth.GenomeSpec(n_contigs=3, contig_len=100_000), 5)
    reads, truth = synth.make_reads(g, synth.ReadsSpec(n_reads=20_000, len_min=30, len_max=300, len_dist=2), 6,
                                    with_qual=True)
    n = len(reads)
    rng = np.random.default_rng(0)
    rec = np.zeros(n, D.MAP_RECORD_DTYPE)
    rec["contig"] = np.where(rng.random(n) < 0.1, -1, truth.contig)
    rec["pos"] = truth.start
    rec["rev"] = truth.rev
    rec["mapq"] = rng.integers(0, 61, n)
    rec["score"] = rng.integers(0, 600, n)
    rec["nm"] = rng.integers(0, 9, n)
    lens = reads.seq_len
    cig = np.zeros(3 * n, np.uint32)
    for i in range(n):  # S M I M (a synthetic but valid-looking CIGAR per read)
        cig[3 * i:3 * i + 3] = [(2 << 4) | 4, (max(lens[i] - 3, 0) << 4) | 0, (1 << 4) | 1]
    rec["cigar_off"] = 3 * np.arange(n)
    rec["cigar_len"] = np.where(rec["contig"] >= 0, 3, 0)
    res = D.MapResult(rec, cig)
    one = D.sam_format(reads, res, g, threads=1)
    for t in (2, 7, 0):
        assert D.sam_format(reads, res, g, threads=t) == one
