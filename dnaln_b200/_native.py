"""ctypes declarations of the C ABI in include/dnaln_b200.h (libdnaln_b200.so, the mapping
path) and include/dnaln_synth.h (libdnaln_synth.so, the seeded workload generator).

Both libraries are loaded from the package directory only (the in-tree build); a missing
library is an ImportError-like failure, never a silent fallback. The generator is a
library of its own so that programs which only need workloads (the reference's CPU
baseline) never load the mapping path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libdnaln_b200.so"
SYNTH_LIB_PATH = Path(__file__).resolve().parent / "libdnaln_synth.so"

OK, ERR_INVALID_ARG, ERR_CUDA, ERR_OOM, ERR_CAPACITY, ERR_NO_DEVICE, ERR_DEVICE, ERR_NOT_FOUND, ERR_IO, \
    ERR_CANCELLED = range(10)
ERR_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "CUDA", 3: "OOM", 4: "CAPACITY", 5: "NO_DEVICE", 6: "DEVICE",
             7: "NOT_FOUND", 8: "IO", 9: "CANCELLED"}


class ScoreParams(C.Structure):
    """ScoreParams of src/align.hpp:34-40."""
    _fields_ = [("match", C.c_int32), ("mismatch", C.c_int32), ("gap_open", C.c_int32), ("gap_ext", C.c_int32),
                ("ambig", C.c_int32), ("bw", C.c_int32)]


class ChainParams(C.Structure):
    """ChainParams of src/chain.hpp:30-36."""
    _fields_ = [("max_gap", C.c_int32), ("band", C.c_int32), ("lookback", C.c_int32), ("min_score", C.c_int32),
                ("min_anchors", C.c_int32)]


class MapParams(C.Structure):
    """MapParams of src/mapper.hpp:25-35."""
    _fields_ = [("k", C.c_int32), ("w", C.c_int32), ("max_occ", C.c_uint32), ("max_cand", C.c_int32),
                ("pri_ratio", C.c_double), ("min_aln_score", C.c_int32), ("sc", ScoreParams), ("ch", ChainParams)]


class AlignResult(C.Structure):
    _fields_ = [("score", C.c_int32), ("qb", C.c_int32), ("qe", C.c_int32), ("tb", C.c_int32), ("te", C.c_int32),
                ("nm", C.c_int32), ("cigar_off", C.c_int64), ("cigar_len", C.c_int32), ("pad_", C.c_int32)]


class MapRecord(C.Structure):
    _fields_ = [("pos", C.c_int64), ("cigar_off", C.c_int64), ("contig", C.c_int32), ("score", C.c_int32),
                ("nm", C.c_int32), ("n_cand", C.c_int32), ("cigar_len", C.c_int32), ("rev", C.c_uint8),
                ("mapq", C.c_uint8), ("pad_", C.c_uint8 * 2)]


class Stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("reads", "mapped", "anchors", "candidates", "cells", "sw_tasks_score",
                                          "sw_tasks_tb", "minimizers")] + \
               [(n, C.c_double) for n in ("ms_seed", "ms_chain", "ms_sw_score", "ms_sw_tb", "ms_post", "ms_h2d",
                                          "ms_d2h", "ms_total")] + \
               [(n, C.c_uint64) for n in ("launches", "warp_reads", "warp_minimizers", "warp_anchors",
                                          "warp_bases", "long_reads", "graph_launches", "batch_retries")]


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("launches", C.c_int64), ("ms", C.c_double)]


class SwTuning(C.Structure):
    _fields_ = [("W", C.c_int32), ("traceback", C.c_int32), ("len_bucket", C.c_int32), ("form", C.c_int32),
                ("ms_inter", C.c_double), ("ms_intra", C.c_double), ("tasks", C.c_int64), ("ms_narrow", C.c_double),
                ("lanes_per_pair", C.c_int32), ("pad_", C.c_int32)]


class SeedTuning(C.Structure):
    _fields_ = [("tuned", C.c_int32), ("reads_per_block", C.c_int32), ("ms_64", C.c_double), ("ms_128", C.c_double),
                ("reads", C.c_int64)]


class ServeParams(C.Structure):
    _fields_ = [("lanes", C.c_int32), ("coalesce", C.c_int32), ("max_batch_reads", C.c_int64),
                ("hbm_budget_bytes", C.c_int64)]


class ServeStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("requests", "reads", "bases", "batches")] + \
               [(n, C.c_double) for n in ("p50_ms", "p99_ms", "max_ms", "mean_ms", "mean_batch_reads")] + \
               [("max_queue_depth", C.c_int64), ("budget_bytes", C.c_int64), ("lane_budget_bytes", C.c_int64),
                ("lanes", C.c_int32), ("pad_", C.c_int32)] + \
               [(n, C.c_double) for n in ("ms_form", "ms_gather", "ms_device", "ms_scatter", "ms_complete")]


class EvalCounts(C.Structure):
    _fields_ = [("records", C.c_uint64), ("mapped", C.c_uint64), ("correct", C.c_uint64),
                ("mapped_at_mapq", C.c_uint64 * 61), ("wrong_at_mapq", C.c_uint64 * 61)]


class SynthGenomeSpec(C.Structure):
    _fields_ = [("n_contigs", C.c_int32), ("contig_len", C.c_uint32), ("gc", C.c_double),
                ("n_repeat_units", C.c_int32), ("repeat_unit_len", C.c_int32), ("repeat_frac", C.c_double),
                ("repeat_div", C.c_double), ("n_frac", C.c_double), ("n_run_min", C.c_int32),
                ("n_run_max", C.c_int32)]


class SynthReadsSpec(C.Structure):
    _fields_ = [("n_reads", C.c_int64), ("len_min", C.c_int32), ("len_max", C.c_int32), ("len_dist", C.c_int32),
                ("sub", C.c_double), ("indel", C.c_double), ("indel_geom_p", C.c_double), ("indel_cap", C.c_int32),
                ("big_del_frac", C.c_double), ("big_del_min", C.c_int32), ("big_del_max", C.c_int32),
                ("name_base", C.c_int64)]


MAP_RECORD_DTYPE = np.dtype({"names": ["pos", "cigar_off", "contig", "score", "nm", "n_cand", "cigar_len", "rev",
                                       "mapq"],
                             "formats": ["<i8", "<i8", "<i4", "<i4", "<i4", "<i4", "<i4", "u1", "u1"],
                             "offsets": [0, 8, 16, 20, 24, 28, 32, 36, 37], "itemsize": 40})
ALIGN_RESULT_DTYPE = np.dtype({"names": ["score", "qb", "qe", "tb", "te", "nm", "cigar_off", "cigar_len"],
                               "formats": ["<i4"] * 6 + ["<i8", "<i4"],
                               "offsets": [0, 4, 8, 12, 16, 20, 24, 32], "itemsize": 40})
assert C.sizeof(MapRecord) == 40 and C.sizeof(AlignResult) == 40

P = C.c_void_p
i32, i64, u32, u64, dbl = C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    "dnaln_gpu_version": (C.c_char_p, []),
    "dnaln_gpu_ctx_create": (C.c_int, [C.c_int, C.POINTER(P)]),
    "dnaln_gpu_ctx_destroy": (C.c_int, [P]),
    "dnaln_gpu_last_error": (C.c_char_p, [P]),
    "dnaln_gpu_set_stream": (C.c_int, [P, P]),
    "dnaln_gpu_get_stats": (C.c_int, [P, C.POINTER(Stats)]),
    "dnaln_gpu_reset_stats": (C.c_int, [P]),
    "dnaln_gpu_set_kernel_trace": (C.c_int, [P, i32, C.c_char_p]),
    "dnaln_gpu_kernel_times": (C.c_int, [P, C.POINTER(KernelTime), i32, C.POINTER(i32)]),
    "dnaln_gpu_set_sub_batch": (C.c_int, [P, i64]),
    "dnaln_gpu_set_option": (C.c_int, [P, C.c_char_p, i64]),
    "dnaln_gpu_sw_tuning": (C.c_int, [P, C.POINTER(SwTuning), i32, C.POINTER(i32)]),
    "dnaln_gpu_seed_tuning": (C.c_int, [P, C.POINTER(SeedTuning)]),
    "dnaln_gpu_map_submit": (C.c_int, [P, i32, P, P, P, P, i64, C.POINTER(MapParams), P, P, i64, C.POINTER(i64),
                             C.POINTER(i64)]),
    "dnaln_gpu_map_wait": (C.c_int, [P, i64]),
    "dnaln_gpu_host_alloc": (C.c_int, [P, C.c_size_t, C.POINTER(P)]),
    "dnaln_gpu_host_free": (C.c_int, [P, P]),
    "dnaln_gpu_index_build": (C.c_int, [P, P, u64, P, P, i32, i32, i32, C.POINTER(i32)]),
    "dnaln_gpu_index_stats": (C.c_int, [P, i32, P]),
    "dnaln_gpu_index_export": (C.c_int, [P, i32, P, P, P, P]),
    "dnaln_gpu_index_free": (C.c_int, [P, i32]),
    "dnaln_gpu_index_attach": (C.c_int, [P, P, i32, C.POINTER(i32)]),
    "dnaln_gpu_index_save": (C.c_int, [P, i32, C.c_char_p]),
    "dnaln_gpu_index_load": (C.c_int, [P, C.c_char_p, C.POINTER(i32)]),
    "dnaln_gpu_index_upload": (C.c_int, [P, P, u64, P, P, i32, i32, i32, P, P, P, u64, P, u64, C.POINTER(i32)]),
    "dnaln_gpu_ctx_device": (C.c_int, [P, C.POINTER(i32)]),
    "dnaln_serve_create": (C.c_int, [P, C.POINTER(ServeParams), C.POINTER(P)]),
    "dnaln_serve_submit": (C.c_int, [P, i32, P, P, P, P, i64, C.POINTER(MapParams), P, P, i64, C.POINTER(i64),
                                     C.POINTER(i64)]),
    "dnaln_serve_wait": (C.c_int, [P, i64, C.POINTER(dbl)]),
    "dnaln_serve_cancel": (C.c_int, [P, i64]),
    "dnaln_serve_get_stats": (C.c_int, [P, C.POINTER(ServeStats)]),
    "dnaln_serve_reset_stats": (C.c_int, [P]),
    "dnaln_serve_last_error": (C.c_char_p, [P]),
    "dnaln_serve_destroy": (C.c_int, [P]),
    "dnaln_gpu_sketch": (C.c_int, [P, P, P, P, P, i64, i32, i32, P, P, P, P]),
    "dnaln_gpu_lookup": (C.c_int, [P, i32, P, i64, P, P]),
    "dnaln_gpu_chain": (C.c_int, [P, P, P, P, P, i64, i32, C.POINTER(ChainParams), P, P, P, P, P, P, P]),
    "dnaln_gpu_align": (C.c_int, [P, P, P, P, P, P, P, i64, i32, C.POINTER(ScoreParams), P, P, i64,
                                  C.POINTER(i64)]),
    "dnaln_gpu_int_peak": (C.c_int, [i32, i32, P, C.POINTER(dbl), C.POINTER(dbl)]),
    "dnaln_gpu_align_noalloc": (C.c_int, [P, P, P, P, P, P, i64, i32, i32, C.POINTER(ScoreParams), P, P, i64, P]),
    "dnaln_gpu_map_batch": (C.c_int, [P, i32, P, P, P, P, i64, C.POINTER(MapParams), P, P, i64, C.POINTER(i64)]),
    "dnaln_gpu_map_batch_device": (C.c_int, [P, i32, P, P, P, P, i64, C.POINTER(MapParams), P, P, i64,
                                             C.POINTER(i64)]),
    "dnaln_fnv1a": (u32, [C.c_char_p, i64]),
    "dnaln_fnv1a_batch": (None, [P, P, i64, P]),
    "dnaln_sam_format": (C.c_int, [P, P, P, P, P, P, P, P, P, i64, P, P, P, i64, C.POINTER(i64)]),
    "dnaln_sam_format_mt": (C.c_int, [P, P, P, P, P, P, P, P, P, i64, P, P, i32, P, i64, C.POINTER(i64)]),
    "dnaln_parse_reads": (C.c_int, [P, i64, i32, C.POINTER(P), P, i64]),
    "dnaln_reads_view": (C.c_int, [P, C.POINTER(i64)] + [C.POINTER(P)] * 8),
    "dnaln_reads_free": (None, [P]),
    "dnaln_eval_records": (C.c_int, [P, P, P, P, P, i64, i32, C.POINTER(EvalCounts)]),
}

# include/dnaln_synth.h, in libdnaln_synth.so
SYNTH_SIGNATURES = {
    "dnaln_synth_genome": (C.c_int, [u64, C.POINTER(SynthGenomeSpec), P]),
    "dnaln_synth_reads_bytes": (i64, [u64, C.POINTER(SynthReadsSpec)]),
    "dnaln_synth_reads": (C.c_int, [u64, P, P, P, i32, C.POINTER(SynthReadsSpec), P, i64, P, P, i64, P, P, P, P]),
}

_lib: C.CDLL | None = None
_synth: C.CDLL | None = None


def _load(path: Path, sigs: dict) -> C.CDLL:
    if not path.exists():
        raise RuntimeError(f"{path} is missing: run `python -m dnaln_b200.build` (needs nvcc)")
    L = C.CDLL(str(path))
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


def lib() -> C.CDLL:
    """The loaded mapping library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        _lib = _load(LIB_PATH, SIGNATURES)
    return _lib


def synth_lib() -> C.CDLL:
    """The loaded workload-generator library (raises if it has not been built)."""
    global _synth
    if _synth is None:
        _synth = _load(SYNTH_LIB_PATH, SYNTH_SIGNATURES)
    return _synth


def ptr(a: np.ndarray | None) -> int | None:
    """Address of a C-contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the C ABI must be contiguous"
    return a.ctypes.data
