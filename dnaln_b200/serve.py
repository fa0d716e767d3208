"""Request server over resident indexes (dnaln_serve_* of include/dnaln_b200.h).

Continuous batching: requests (read sets of any size, each against one index of the home
context) are submitted from any thread and mapped by worker lanes that coalesce waiting
requests for the same index and parameters into batches, several batches in flight on
the device at once. Each request's records and CIGARs equal ``Context.map_batch`` of
the request alone. No reference counterpart: dnaln maps one FASTQ per process
(src/main.cpp:33-61).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import MAP_RECORD_DTYPE, Context, DnalnError, MapParams, MapResult, ReadBatch, default_map_params
from . import _native as N
from ._native import lib, ptr


@dataclass
class Request:
    """A submitted request: keeps its host buffers alive until Server.wait."""
    n: int
    params: MapParams
    keep: list
    records: np.ndarray
    cigar: np.ndarray
    used: C.c_int64 = field(default_factory=C.c_int64)
    id: int = 0
    latency_ms: float | None = None


class Server:
    """dnaln_serve_create over a home Context whose indexes it serves.

    lanes: concurrent batches; coalesce: requests share batches (False = one request per
    batch); max_batch_reads: reads per batch; hbm_budget_bytes: device memory for the
    batches in flight (0 = free memory at creation minus 2 GiB)."""

    def __init__(self, home: Context, lanes: int = 3, coalesce: bool = True, max_batch_reads: int = 262_144,
                 hbm_budget_bytes: int = 0):
        self._lib = lib()
        self.home = home
        sp = N.ServeParams(lanes, 1 if coalesce else 0, max_batch_reads, hbm_budget_bytes)
        h = C.c_void_p()
        rc = self._lib.dnaln_serve_create(home.handle, C.byref(sp), C.byref(h))
        if rc != N.OK:
            raise DnalnError(rc, "cannot create the server")
        self._h = h

    def _check(self, rc: int) -> None:
        if rc != N.OK:
            raise DnalnError(rc, self._lib.dnaln_serve_last_error(self._h).decode())

    def submit(self, iid: int, reads: ReadBatch, p: MapParams | None = None) -> Request:
        p = p or default_map_params()
        n = len(reads)
        lens = np.ascontiguousarray(reads.seq_len)
        cap = int(np.sum(2 * lens.astype(np.int64) + 3)) if n else 0
        r = Request(n=n, params=p, keep=[reads.seq, np.ascontiguousarray(reads.seq_off[:-1]), lens,
                                         reads.name_hash()],
                    records=np.zeros(max(n, 1), dtype=MAP_RECORD_DTYPE), cigar=np.zeros(max(cap, 1), np.uint32))
        rid = C.c_int64()
        seq, off, ln, nh = r.keep
        self._check(self._lib.dnaln_serve_submit(self._h, iid, ptr(seq), ptr(off), ptr(ln), ptr(nh), n,
                                                 C.byref(r.params), ptr(r.records), ptr(r.cigar), cap,
                                                 C.byref(r.used), C.byref(rid)))
        r.id = rid.value
        return r

    def cancel(self, r: Request) -> None:
        """dnaln_serve_cancel: the request's wait then raises DnalnError(ERR_CANCELLED),
        unless it had already completed."""
        self._check(self._lib.dnaln_serve_cancel(self._h, r.id))

    def wait(self, r: Request) -> MapResult:
        lat = C.c_double()
        self._check(self._lib.dnaln_serve_wait(self._h, r.id, C.byref(lat)))
        r.latency_ms = lat.value
        return MapResult(r.records[:r.n], r.cigar[:r.used.value])

    def stats(self) -> dict:
        s = N.ServeStats()
        self._check(self._lib.dnaln_serve_get_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in N.ServeStats._fields_ if f != "pad_"}

    def reset_stats(self) -> None:
        self._check(self._lib.dnaln_serve_reset_stats(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.dnaln_serve_destroy(self._h)
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
