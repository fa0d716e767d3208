"""Build of the in-tree native library ``dnaln_b200/libdnaln_b200.so``.

CUDA sources are compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
host C++ sources with g++. Objects go to ``dnaln_b200/_build/``; the shared library is
linked with the static CUDA runtime, so loading it needs no GPU (CUDA calls then fail
with DNALN_ERR_NO_DEVICE). Rebuilds only when a source or header is newer than the
library. Run ``python -m dnaln_b200.build`` or call :func:`build`.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
BUILD = PKG / "_build"
LIB = PKG / "libdnaln_b200.so"

CUDA_SOURCES = ["csrc/sw.cu", "csrc/seed.cu", "csrc/seed_thread.cu", "csrc/map.cu", "csrc/capi.cu", "csrc/noalloc.cu",
                "csrc/serve.cu", "csrc/index_build.cu",
                "csrc/seed_long.cu", "csrc/peak.cu", "csrc/encode_bulk.cu"]
HOST_SOURCES = ["host/sam.cpp", "host/reads.cpp", "host/eval.cpp"]
# the seeded workload generator, a library of its own (no CUDA): programs that only need
# workloads, such as the reference's CPU baseline, load it without the mapping path
SYNTH_SOURCES = ["host/synth.cpp"]
SYNTH_LIB = PKG / "libdnaln_synth.so"
HEADERS = ["csrc/common.cuh", "csrc/sw.cuh", "csrc/seed.cuh", "csrc/map.cuh", "csrc/index_build.cuh"]
PUBLIC_HEADERS = ["dnaln_b200.h", "dnaln_synth.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found (CUDA toolkit required to build dnaln_b200)")


def _includes() -> list[str]:
    return [f"-I{ROOT / 'include'}", f"-I{PKG / 'csrc'}", f"-I{PKG / 'host'}"]


def _newest_input() -> float:
    files = [PKG / s for s in CUDA_SOURCES + HOST_SOURCES + SYNTH_SOURCES + HEADERS] + \
        [ROOT / "include" / h for h in PUBLIC_HEADERS]
    files.append(Path(__file__))
    return max(f.stat().st_mtime for f in files)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def _compile_cuda(src: str, nvcc: str, extra: list[str]) -> Path:
    obj = BUILD / (Path(src).stem + ".cu.o")
    cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC",
           *_includes(), *extra, "-c", str(PKG / src), "-o", str(obj)]
    _run(cmd)
    return obj


def _compile_host(src: str) -> Path:
    obj = BUILD / (Path(src).stem + ".o")
    cxx = os.environ.get("CXX", "g++")
    _run([cxx, "-O3", "-std=c++17", "-fPIC", "-Wall", "-Wextra", *_includes(), "-c", str(PKG / src), "-o", str(obj)])
    return obj


def build(force: bool = False, verbose: bool = False, extra_nvcc: list[str] | None = None) -> Path:
    """Compiles the CUDA and host sources and links ``libdnaln_b200.so`` (and the generator,
    ``libdnaln_synth.so``); returns the mapping library's path."""
    newest = _newest_input()
    if not force and LIB.exists() and SYNTH_LIB.exists() and min(LIB.stat().st_mtime,
                                                                 SYNTH_LIB.stat().st_mtime) >= newest:
        return LIB
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    extra = list(extra_nvcc or [])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        futs = [ex.submit(_compile_cuda, s, nvcc, extra) for s in CUDA_SOURCES]
        futs += [ex.submit(_compile_host, s) for s in HOST_SOURCES]
        sfuts = [ex.submit(_compile_host, s) for s in SYNTH_SOURCES]
        objs = [f.result() for f in futs]
        sobjs = [f.result() for f in sfuts]
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lpthread"])
    os.replace(tmp, LIB)
    tmp = SYNTH_LIB.with_suffix(".so.tmp")
    _run([os.environ.get("CXX", "g++"), "-shared", "-o", str(tmp), *map(str, sobjs)])
    os.replace(tmp, SYNTH_LIB)
    if verbose:
        print(f"built {LIB}", file=sys.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
