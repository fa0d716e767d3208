"""The drop-in classes of dnaln_b200/binding/ inside the reference's own programs, built by
oracle/Makefile's `binding` target from the reference's unmodified sources:

* dnaln_tests_gpu — the reference's tests/test_main.cpp with GpuAligner in SimdAligner's
  place, so simd_kernel_bit_identical_to_scalar, perfect_match_alignment and
  end_to_end_mapping_accuracy check the GPU aligner against the reference's ScalarAligner;
* dnaln_gpu_aligner — `dnaln map` whose Mapper constructs a GpuAligner at
  src/mapper.cpp:10;
* dnaln_gpu_mapper — `dnaln map` whose cmd_map maps every batch through GpuMapper (the
  whole path on the device), SAM still written by the reference's append_sam.

The SAM bodies of both GPU programs must be byte-identical to the stock `dnaln map`'s on
the 1 Mbp / 10,000 x 150 bp workload."""
import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
REF = ROOT / "oracle" / "_ref"
PROGRAMS = ["dnaln_gpu_aligner", "dnaln_gpu_mapper", "dnaln_tests_gpu"]


def need(name: str) -> Path:
    p = REF / name
    if not p.exists():
        pytest.skip(f"{p} not built (make -C oracle binding, where the reference sources are present)")
    return p


@pytest.mark.parametrize("name", ["dnaln_gpu_aligner", "dnaln_gpu_mapper"])
def test_binding_programs_load_the_library(name):
    # no GPU needed: --version runs before any device call, but the dynamic loader has
    # already resolved libdnaln_b200.so by then
    r = subprocess.run([str(need(name)), "--version"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("dnaln ")


@pytest.mark.gpu
def test_reference_unit_tests_with_the_gpu_aligner():
    prog = need("dnaln_tests_gpu")
    r = subprocess.run([str(prog)], capture_output=True, text=True, timeout=900, cwd=str(REF))
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-4000:]
    assert "CUDA sm_100a" in out  # the header line names GpuAligner::isa(), not the CPU's SIMD
    assert "FAILED" not in out, out[-4000:]


def sam_body(path: Path) -> bytes:
    return b"".join(line for line in path.read_bytes().splitlines(keepends=True) if not line.startswith(b"@PG"))


@pytest.mark.gpu
def test_gpu_programs_write_the_reference_sam(tmp_path):
    from dnaln_b200 import synth
    stock = need("dnaln")
    g, reads, _ = synth.workload("small-1Mbp-10k-150bp", seed=7)
    fa, fq = tmp_path / "ref.fa", tmp_path / "reads.fq"
    synth.write_fasta(g, str(fa))
    synth.write_fastq(reads, str(fq))
    outs = {}
    for name in ["dnaln", "dnaln_gpu_aligner", "dnaln_gpu_mapper"]:
        prog = stock if name == "dnaln" else need(name)
        out = tmp_path / f"{name}.sam"
        r = subprocess.run([str(prog), "map", "-o", str(out), str(fa), str(fq)], capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        outs[name] = sam_body(out)
        if name != "dnaln":
            assert "B200" in r.stderr  # its log line names the GPU kernel
    assert outs["dnaln"].count(b"\n") > 10_000
    assert outs["dnaln_gpu_aligner"] == outs["dnaln"]
    assert outs["dnaln_gpu_mapper"] == outs["dnaln"]
