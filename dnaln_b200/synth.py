"""Seeded synthetic workloads (genomes + reads) for the mapping path.

The five workloads the path is measured on, with their sizes; each is generated from a
seed by the native generator (include/dnaln_synth.h), so the same seed gives the same
bytes everywhere. No public dataset is involved: these are the workloads' own synthetic
definitions (i.i.d. genomes of a given base composition, optional repeat units and N
runs; reads with the 1% substitution / 0.1% indel error model).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import Genome, ReadBatch
from ._native import SynthGenomeSpec, SynthReadsSpec, ptr, synth_lib

# error model shared by every workload: 1% substitution, 0.1% indel (half ins, half del),
# indel length geometric(p = 0.7) capped at 5
ERR = dict(sub=0.01, indel=0.001, indel_geom_p=0.7, indel_cap=5)


@dataclass(frozen=True)
class GenomeSpec:
    n_contigs: int = 1
    contig_len: int = 1_000_000
    gc: float = 0.508  # P(G) = P(C) = 0.254
    n_repeat_units: int = 0
    repeat_unit_len: int = 0
    repeat_frac: float = 0.0
    repeat_div: float = 0.0
    n_frac: float = 0.0
    n_run_min: int = 0
    n_run_max: int = 0


@dataclass(frozen=True)
class ReadsSpec:
    n_reads: int = 10_000
    len_min: int = 150
    len_max: int = 150
    len_dist: int = 0  # 0 fixed, 1 log-uniform, 2 uniform
    big_del_frac: float = 0.0
    big_del_min: int = 0
    big_del_max: int = 0
    name_base: int = 1


GENOME_1M = GenomeSpec(contig_len=1_000_000)
GENOME_4M6 = GenomeSpec(contig_len=4_600_000)
GENOME_120M = GenomeSpec(n_contigs=8, contig_len=15_000_000, gc=0.42, n_repeat_units=200, repeat_unit_len=2000,
                         repeat_frac=0.06, repeat_div=0.02, n_frac=0.005, n_run_min=10, n_run_max=100)
# the 120 Mbp genome's composition, repeat density and N runs at 2 Mbp (parity tests)
GENOME_REPEAT_2M = GenomeSpec(n_contigs=4, contig_len=500_000, gc=0.42, n_repeat_units=20, repeat_unit_len=2000,
                              repeat_frac=0.06, repeat_div=0.02, n_frac=0.005, n_run_min=10, n_run_max=100)

# name -> (genome spec, reads spec, description)
WORKLOADS = {
    "small-1Mbp-10k-150bp": (GENOME_1M, ReadsSpec(n_reads=10_000), "10,000 x 150 bp on a 1 Mbp genome"),
    "ecoli-4.6Mbp-1M-150bp": (GENOME_4M6, ReadsSpec(n_reads=1_000_000),
                              "1,000,000 x 150 bp on a 4.6 Mbp genome, batches of 262,144"),
    "mixed-4.6Mbp-1M-50to1000bp": (GENOME_4M6, ReadsSpec(n_reads=1_000_000, len_min=50, len_max=1000, len_dist=1,
                                                          big_del_frac=0.02, big_del_min=8, big_del_max=15),
                                   "1,000,000 reads log-uniform 50-1000 bp, 2% with an 8-15 bp deletion"),
    "repeat-120Mbp-10M-150bp": (GENOME_120M, ReadsSpec(n_reads=10_000_000),
                                "10,000,000 x 150 bp on 8 x 15 Mbp contigs with repeats and N runs"),
    "repeat-2Mbp-20k-150bp": (GENOME_REPEAT_2M, ReadsSpec(n_reads=20_000),
                              "20,000 x 150 bp on 4 x 500 kbp contigs with repeats and N runs"),
    "mixed-1Mbp-5k-50to1000bp": (GENOME_1M, ReadsSpec(n_reads=5_000, len_min=50, len_max=1000, len_dist=1,
                                                       big_del_frac=0.02, big_del_min=8, big_del_max=15),
                                 "5,000 reads log-uniform 50-1000 bp on a 1 Mbp genome"),
}


def make_genome(spec: GenomeSpec, seed: int) -> Genome:
    s = SynthGenomeSpec(spec.n_contigs, spec.contig_len, spec.gc, spec.n_repeat_units, spec.repeat_unit_len,
                        spec.repeat_frac, spec.repeat_div, spec.n_frac, spec.n_run_min, spec.n_run_max)
    total = spec.n_contigs * spec.contig_len
    codes = np.zeros(total, np.uint8)
    rc = synth_lib().dnaln_synth_genome(seed, C.byref(s), ptr(codes))
    if rc:
        raise RuntimeError(f"genome generation failed ({rc})")
    off = np.arange(spec.n_contigs, dtype=np.uint64) * np.uint64(spec.contig_len)
    ln = np.full(spec.n_contigs, spec.contig_len, np.uint32)
    names = ["synth" if spec.n_contigs == 1 else f"synth{i + 1}" for i in range(spec.n_contigs)]
    return Genome(codes, off, ln, names)


@dataclass
class Truth:
    contig: np.ndarray
    start: np.ndarray
    rev: np.ndarray


def make_reads(g: Genome, spec: ReadsSpec, seed: int, with_qual: bool = False) -> tuple[ReadBatch, Truth]:
    s = SynthReadsSpec(spec.n_reads, spec.len_min, spec.len_max, spec.len_dist, ERR["sub"], ERR["indel"],
                       ERR["indel_geom_p"], ERR["indel_cap"], spec.big_del_frac, spec.big_del_min, spec.big_del_max,
                       spec.name_base)
    L = synth_lib()
    nbytes = int(L.dnaln_synth_reads_bytes(seed, C.byref(s)))
    n = spec.n_reads
    seq = np.zeros(max(nbytes, 1), np.uint8)
    so = np.zeros(n + 1, np.int64)
    name_cap = n * (5 + len(str(spec.name_base + n))) + 16
    names = np.zeros(name_cap, np.uint8)
    no = np.zeros(n + 1, np.int64)
    tc = np.zeros(max(n, 1), np.int32)
    ts = np.zeros(max(n, 1), np.int64)
    tr = np.zeros(max(n, 1), np.uint8)
    rc = L.dnaln_synth_reads(seed, ptr(g.codes), ptr(g.contig_off), ptr(g.contig_len), g.n_contigs, C.byref(s),
                             ptr(seq), nbytes, ptr(so), ptr(names), name_cap, ptr(no), ptr(tc), ptr(ts), ptr(tr))
    if rc:
        raise RuntimeError(f"read generation failed ({rc})")
    qual = np.full(nbytes, ord("I"), np.uint8) if with_qual else None
    return ReadBatch(seq[:nbytes], so, names[:no[-1]], no, qual), Truth(tc[:n], ts[:n], tr[:n])


def workload(name: str, seed: int = 1, n_reads: int | None = None, with_qual: bool = False):
    """(genome, reads, truth) of a named workload; n_reads overrides the read count."""
    gspec, rspec, _ = WORKLOADS[name]
    if n_reads is not None:
        rspec = ReadsSpec(**{**rspec.__dict__, "n_reads": n_reads})
    g = make_genome(gspec, seed)
    reads, truth = make_reads(g, rspec, seed + 1000, with_qual)
    return g, reads, truth


def write_fasta(g: Genome, path: str) -> None:
    acgt = np.frombuffer(b"ACGTN", np.uint8)
    with open(path, "wb") as f:
        for name, o, ln in zip(g.names, g.contig_off, g.contig_len):
            f.write(b">" + name.encode() + b"\n")
            s = acgt[g.codes[int(o):int(o) + int(ln)]]
            for i in range(0, len(s), 80):
                f.write(s[i:i + 80].tobytes() + b"\n")


def write_fastq(reads: ReadBatch, path: str) -> None:
    with open(path, "wb") as f:
        for i in range(len(reads)):
            s = reads.read(i)
            f.write(b"@" + reads.name(i) + b"\n" + s + b"\n+\n" + b"I" * len(s) + b"\n")
