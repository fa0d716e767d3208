#!/usr/bin/env python
"""Throughput of the B200 read-mapping path (reads/s) on the 4.6 Mbp / 1,000,000 x 150 bp
workload, in batches of 262,144 reads per launch of the pipeline.

One step maps the whole 1,000,000-read workload (4 batches). Two measurements:
* value — inputs already resident in HBM, dnaln_gpu_map_batch_device, timed with CUDA
  events on the launching stream;
* e2e   — the reference-facing C call dnaln_gpu_map_batch on pinned HOST buffers, with the
  host->device copy of the reads and the device->host copy of records and CIGARs inside
  the timed region.

`--impl reference` times the reference's own CPU mapper (Mapper::map, compiled from its
sources into oracle/_ref) on the host cores with all threads, same workload and metric.

Multi-GPU (`torchrun --nproc-per-node N bench.py --gpus N`): each rank maps its own
1,000,000 reads against a replica of the index (weak scaling); no collective on the data
path, timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "ecoli-4.6Mbp-1M-150bp"
BATCH = 262_144
METRIC = "reads/s"
PROFILE_STEPS = 2  # untimed steps whose every kernel launch is timed (the per-kernel breakdown)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--n-reads", type=int, default=None, help="override the workload's read count (testing)")
    ap.add_argument("--e2e-steps", type=int, default=None,
                    help="timed steps of the e2e leg (default: the larger of --steps and 30; the "
                         "pipeline's fill and drain are inside the window and amortised over them)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-e2e", action="store_true",
                    help="also time the step through the request server (each batch one request)")
    ap.add_argument("--workload", default=WORKLOAD,
                    help="synthetic workload (dnaln_b200.synth.WORKLOADS); the default is the headline one")
    ap.add_argument("--bw", type=int, default=16, help="SW band half-width (16, or 64 for the mixed-length workload)")
    ap.add_argument("--sw-form", type=int, default=0, choices=[0, 1, 2, 3],
                    help="SW kernel form: 0 tuned per context, 1 inter-sequence, 2 intra-sequence, 3 intra-sequence "
                         "narrow (pin it under a profiler, whose serialised replays distort the tuner's timing)")
    ap.add_argument("--cigar-per-read", type=int, default=0,
                    help="CIGAR capacity per read of the output buffers (0 = the 2*len+3 bound)")
    ap.add_argument("--serve-requests", type=int, default=1500, help="requests per rate point (--workload serve)")
    ap.add_argument("--serve-lanes", type=int, default=4, help="lanes of the batching server (4 measured best of 3, 4, 6)")
    ap.add_argument("--serve-loads", type=float, nargs="*", default=[0.5, 0.8],
                    help="offered loads as fractions of the measured capacity (--workload serve)")
    ap.add_argument("--lanes", type=int, default=2, choices=[1, 2, 3, 4],
                    help="mapping lanes: contexts sharing the resident index, each with its own stream and host "
                         "thread; the step's batches alternate between them so one batch's kernels overlap "
                         "another's (1 = one context, batches in sequence)")
    ap.add_argument("--dir-cap-bytes", type=int, default=0,
                    help="traceback direction-code scratch per launch (0 = the library's default; smaller splits "
                         "launches, e.g. to keep a profiled case small)")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the mixed-length (batched vs plain, bw 16 / 64) and serving legs of the default run")
    ap.add_argument("--leg-requests", type=int, default=600, help="requests per load point of the serving leg")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler(threading.Thread):
    """Samples SM clock and clock-event reasons of one GPU through NVML (read-only)."""
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x2: "applications_clocks_setting"}

    def __init__(self, device: int, period: float = 0.02):
        super().__init__(daemon=True)
        self.period, self.samples, self.reasons, self.stop_ev = period, [], set(), threading.Event()
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def run(self):
        if not self.nv:
            return
        get_r = getattr(self.nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            self.nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop_ev.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = get_r(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(self.period)

    def result(self):
        self.stop_ev.set()
        self.join(timeout=2)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def workload_config(n_reads: int, world: int, name: str = WORKLOAD, bw: int = 16, genome_bp: int = 4_600_000,
                    mean_len: float = 150.0) -> dict:
    if name == WORKLOAD:
        desc = (f"{WORKLOAD}: 4.6 Mbp i.i.d. genome (P(G)=P(C)=0.254), {n_reads:,} x 150 bp reads "
                f"(1% substitution, 0.1% indel), k=15 w=10 bw={bw} A2 B4 O4 E2, batches of 262,144")
    else:
        from dnaln_b200 import synth
        desc = f"{name}: {synth.WORKLOADS[name][2]}, {n_reads:,} reads, k=15 w=10 bw={bw} A2 B4 O4 E2"
    return {"workload": desc, "reads_per_step": n_reads, "batch": BATCH, "genome_bp": genome_bp,
            "mean_read_len": round(mean_len, 1),
            "l2": f"no flush: each step streams {n_reads * mean_len / 1e6:.0f} MB of reads plus the per-batch "
                  "scratch (both well above the 126 MB L2)",
            "parallelism": f"dp{world} read shards, index replica per GPU"}


def measured_peaks() -> tuple[float, str]:
    try:
        j = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


TASK_BYTES = 48 + 32  # SW task descriptor in, result out


def kernel_bytes(kernel: str, st: dict, mean_len: float, bw: int = 16) -> float | None:
    """Algorithmic HBM bytes of all launches of one kernel, from the batch counters in st
    (reads, minimizers, anchors, candidates, SW tasks; the warp_* counters cover the reads
    listed for the warp-per-read kernels). None for kernels not modelled."""
    n = st["reads"]
    mins = st["minimizers"] if st.get("minimizers") else 0.18 * mean_len * n
    W = 2 * bw + 1
    cand_per_read = st["candidates"] / max(n, 1)
    dir_row = (W + 3) // 4 * 2  # direction-code bytes per query row: ceil(W/4) 16-bit words per alignment
    if kernel == "k_seed_chain_t":  # ASCII in, 16-B bucket per minimizer, 4-B occurrence per anchor,
        # 21-B candidate out, 28 B of per-read offsets / lengths / counts
        return n * mean_len + mins * 16 + (st["anchors"] - st["warp_anchors"]) * 4 + \
            st["candidates"] * 21 + n * 28
    if kernel == "k_encode_reads":  # ASCII in, codes of both strands out, offsets / lengths
        return n * mean_len * (1 + 2) + n * 20
    if kernel == "k_seed":        # ASCII in, codes of both strands out, 20-B minimizer slot out + 16-B bucket
        return n * mean_len * (1 + 2) + mins * (20 + 16) + n * 24
    if kernel == "k_seed<list>":  # listed reads: ASCII in (codes already written), slots out + buckets
        return st["warp_bases"] + st["warp_minimizers"] * (20 + 16) + st["warp_reads"] * 24
    if kernel in ("k_chain_map", "k_chain_map<list>"):  # minimizer slots in, 4-B occurrence per anchor,
        # 21-B candidate out, 28 B of per-read offsets / counts
        r = st["warp_reads"]
        return st["warp_minimizers"] * 20 + st["warp_anchors"] * 4 + r * cand_per_read * 21 + r * 28
    if kernel in ("k_sw_u2<tb>", "k_sw_wide<tb>"):  # query + window in, direction codes out, task/result
        t = st["sw_tasks_tb"]
        return t * (mean_len + (mean_len + 2 * bw) + mean_len * dir_row + TASK_BYTES)
    if kernel in ("k_sw_u2<score>", "k_sw_wide<score>"):
        t = st["sw_tasks_score"]
        return t * (mean_len + (mean_len + 2 * bw) + TASK_BYTES)
    if kernel == "k_sw_walk":     # one direction word per step (~len steps), query/window bytes on the path, CIGAR
        t = st["sw_tasks_tb"]
        return t * (mean_len * (4 + 2) + 16 + TASK_BYTES)
    return None


def index_image_round_trip(ctx, iid) -> dict:
    """Index admission from a file: dnaln_gpu_index_save, then dnaln_gpu_index_load of the
    image (read, checksum and structural checks, upload) against the device build above."""
    import tempfile
    try:
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "index.img")
            t0 = time.perf_counter()
            ctx.index_save(iid, path)
            t1 = time.perf_counter()
            size = os.path.getsize(path)
            iid2 = ctx.index_load(path)
            t2 = time.perf_counter()
            ctx.index_free(iid2)
        return {"bytes": size, "save_s": t1 - t0, "load_s": t2 - t1, "load_gbs": size / (t2 - t1) / 1e9,
                "where": "dnaln_gpu_index_save / dnaln_gpu_index_load"}
    except (OSError, D.DnalnError) as e:
        return {"error": str(e)}


def cpu_baseline(g, reads, params) -> dict:
    """The reference's CPU mapper on this host (all hardware threads), on one batch."""
    import oracle
    sample = reads.slice(0, min(len(reads), BATCH))
    threads = len(os.sched_getaffinity(0))
    if oracle.REF_SO.exists():
        ref = oracle.Reference()
        rg = ref.genome(g)
        ref.time_map(rg, sample.slice(0, min(len(sample), 20_000)), params, threads)  # warm-up
        reps, dt = 0, 0.0
        while dt < 5.0 and reps < 20:   # >= ~5 s wall (x threads of CPU work)
            dt += ref.time_map(rg, sample, params, threads)
            reps += 1
        one = sample.slice(0, min(len(sample), 50_000))
        dt1 = ref.time_map(rg, one, params, 1)
        return {"value": reps * len(sample) / dt, "unit": METRIC, "cores": threads, "kind": "reference",
                "sample": f"{reps} x {len(sample):,} reads of the workload (one batch), Mapper::map with "
                          f"{threads} threads (one Mapper per thread over read shards)",
                "single_thread_value": len(one) / dt1, "cpu": _cpu_model()}
    port = oracle.Port()
    pi = port.index(g)
    one = sample.slice(0, min(len(sample), 20_000))
    t0 = time.perf_counter()
    port.map(pi, one, params)
    dt = time.perf_counter() - t0
    return {"value": len(one) / dt, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"{len(one):,} reads of the workload, scalar C port, 1 thread", "cpu": _cpu_model()}


def _cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args) -> None:
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    import dnaln_b200 as D
    from dnaln_b200 import synth
    if args.workload == SERVE:
        run_reference_serve(args)
        return
    g, reads, _ = synth.workload(args.workload, seed=args.seed, n_reads=args.n_reads)
    p = D.default_map_params(bw=args.bw)
    threads = len(os.sched_getaffinity(0))
    if oracle.REF_SO.exists():
        ref, kind = oracle.Reference(), "reference"
        rg = ref.genome(g)
        run = lambda s: ref.time_map(rg, s, p, threads)  # noqa: E731
        cores = threads
        sample = reads
    else:  # the C port, single-threaded, on a bounded sample
        port, kind = oracle.Port(), "port"
        pi = port.index(g)
        sample = reads.slice(0, min(len(reads), 50_000))

        def run(s):
            t0 = time.perf_counter()
            port.map(pi, s, p)
            return time.perf_counter() - t0
        cores = 1
    for _ in range(args.warmup):
        run(sample)
    dt = sum(run(sample) for _ in range(args.steps))
    value = args.steps * len(sample) / dt
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator)",
            "config": workload_config(len(sample), 1, args.workload, args.bw, len(g.codes),
                                      float(np.mean(sample.seq_len))), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": kind,
                             "sample": f"{len(sample):,} reads per step, Mapper::map, {cores} threads",
                             "cpu": _cpu_model()},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference_serve(args) -> None:
    """The reference's CPU mapper on the serving workload's requests, back to back, all
    host threads: requests are mapped in arrival order, each split over the threads."""
    import oracle
    import dnaln_b200 as D
    pools = ServePools(args.seed)
    p = D.default_map_params(bw=args.bw)
    threads = len(os.sched_getaffinity(0))
    if not oracle.REF_SO.exists():
        print(json.dumps({"impl": "reference", "unavailable": "the reference build (oracle/_ref) is missing"}))
        return
    ref = oracle.Reference()
    rgs = [ref.genome(g) for g in pools.genomes]
    reqs = pools.stream(args.serve_requests, args.seed + 100)
    sample, tot = [], 0
    for r in reqs:  # a bounded sample of the stream: ~20 s of CPU work
        sample.append(r)
        tot += r[2]
        if tot >= 400_000:
            break
    dt = 0.0
    for gi, a, m in sample:
        dt += ref.time_map(rgs[gi], pools.pools[gi].slice(a, a + m), p, threads)
    value = tot / dt
    line = {"metric": "reads/s (served)", "value": value, "unit": "reads/s", "n_gpus": 1, "steps": 1, "warmup": 0,
            "ms_per_step": 1e3 * dt, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic (seeded generator)",
            "config": {"workload": "serve (reference CPU mapper, requests back to back)", "requests": len(sample),
                       "reads": tot}, "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "reads/s", "cores": threads, "kind": "reference",
                             "sample": f"first {len(sample)} requests of the stream ({tot:,} reads), Mapper::map, "
                                       f"{threads} threads", "cpu": _cpu_model()},
            "e2e": {"value": value, "unit": "reads/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def text_pipeline(ctx, iid, reads, g, p, steps: int) -> dict:
    """The workload from FASTQ text in memory to SAM text in memory, through the C ABI with
    no copies in between: dnaln_parse_reads on all host threads, the host-buffer mapping
    call on the parsed arrays in batches of 262,144 (submit / wait, so one batch's copies
    overlap the next one's kernels), dnaln_sam_format_mt on all host threads into one
    reused buffer, each batch as soon as it is mapped while the later ones map. Wall clock
    per step."""
    import tempfile

    import dnaln_b200 as D
    from dnaln_b200 import _native as N
    from dnaln_b200 import synth
    L = N.lib()
    with tempfile.NamedTemporaryFile(suffix=".fq") as f:
        synth.write_fastq(reads, f.name)
        text = np.fromfile(f.name, np.uint8)
    threads = len(os.sched_getaffinity(0))
    n_all = len(reads)
    spans = [(a, min(n_all, a + BATCH)) for a in range(0, n_all, BATCH)]
    lens_all = reads.seq_len.astype(np.int64)
    caps = [int(np.sum(2 * lens_all[a:b] + 3)) for a, b in spans]
    recs = [np.zeros(b - a, D.MAP_RECORD_DTYPE) for a, b in spans]
    cigs = [np.zeros(c, np.uint32) for c in caps]
    used = [C.c_int64() for _ in spans]
    cn, co = g.name_buffers()
    sam = np.zeros(int(np.sum(2 * lens_all)) + 200 * n_all + (1 << 20), np.uint8)
    err = C.create_string_buffer(256)
    t_parse = t_map = t_sam = 0.0
    sam_bytes = 0
    for step in range(steps + 1):  # the first step warms the page cache and the buffers
        t0 = time.perf_counter()
        h = C.c_void_p()
        rc = L.dnaln_parse_reads(text.ctypes.data, len(text), threads, C.byref(h), C.addressof(err), 256)
        if rc:
            raise RuntimeError(err.value.decode())
        n = C.c_int64()
        v = [C.c_void_p() for _ in range(8)]
        L.dnaln_reads_view(h, C.byref(n), *[C.byref(x) for x in v])
        seq, so, sl, nm, no, ql, qo, nh = [x.value for x in v]
        t1 = time.perf_counter()
        tickets = []
        for k, (a, b) in enumerate(spans):
            t = C.c_int64()
            rc = L.dnaln_gpu_map_submit(ctx.handle, iid, seq, so + 8 * a, sl + 4 * a, nh + 4 * a, b - a, C.byref(p),
                                        recs[k].ctypes.data, cigs[k].ctypes.data, caps[k], C.byref(used[k]),
                                        C.byref(t))
            if rc:
                raise RuntimeError(L.dnaln_gpu_last_error(ctx.handle).decode())
            tickets.append(t.value)
        # batch k is formatted as soon as it is mapped, while the later batches map
        out_at = 0
        wait_s = 0.0
        for k, (a, b) in enumerate(spans):
            tw = time.perf_counter()
            if L.dnaln_gpu_map_wait(ctx.handle, tickets[k]):
                raise RuntimeError(L.dnaln_gpu_last_error(ctx.handle).decode())
            wait_s += time.perf_counter() - tw
            u = C.c_int64()
            rc = L.dnaln_sam_format_mt(seq, so + 8 * a, sl + 4 * a, nm, no + 8 * a, ql, qo + 8 * a, recs[k].ctypes.data,
                                       cigs[k].ctypes.data, b - a, cn.ctypes.data, co.ctypes.data, threads,
                                       sam.ctypes.data + out_at, len(sam) - out_at, C.byref(u))
            if rc:
                raise RuntimeError(f"SAM formatting failed ({rc})")
            out_at += u.value
        t3 = time.perf_counter()
        L.dnaln_reads_free(h)
        if step:
            t_parse += t1 - t0
            t_map += wait_s
            t_sam += (t3 - t1) - wait_s
            sam_bytes = out_at
    total = t_parse + t_map + t_sam
    return {"value": steps * n_all / total, "unit": METRIC, "host_threads": threads,
            "ms_per_step": {"parse": 1e3 * t_parse / steps, "map_wait": 1e3 * t_map / steps,
                            "sam_and_submit": 1e3 * t_sam / steps},
            "text_bytes_in": int(len(text)), "sam_bytes_out": int(sam_bytes),
            "what": "FASTQ text in memory -> dnaln_parse_reads -> dnaln_gpu_map_submit on the parsed (pageable) "
                    "arrays -> per batch dnaln_gpu_map_wait then dnaln_sam_format_mt while the later batches map "
                    "-> SAM text in memory; wall clock per step (map_wait = time the host waited for the GPU)"}


MIXED = "mixed-4.6Mbp-1M-50to1000bp"


def device_parts(reads, cigar_per_read: int = 0) -> list[dict]:
    """The workload's batches of 262,144 reads as device tensors (reads, offsets, lengths,
    name hashes) with their output buffers."""
    import torch
    n_reads = len(reads)
    out = []
    for a in range(0, n_reads, BATCH):
        part = reads.slice(a, min(n_reads, a + BATCH))
        n = len(part)
        lens = part.seq_len
        cap = int(np.sum(2 * lens.astype(np.int64) + 3)) if not cigar_per_read else n * cigar_per_read
        out.append(dict(
            n=n, cap=cap,
            seq=torch.from_numpy(part.seq).cuda(),
            off=torch.from_numpy(np.ascontiguousarray(part.seq_off[:-1])).cuda(),
            len=torch.from_numpy(lens).cuda(),
            hash=torch.from_numpy(part.name_hash().view(np.int32)).cuda(),
            out=torch.empty(n * 40, dtype=torch.uint8, device="cuda"),
            cig=torch.empty(cap, dtype=torch.int32, device="cuda")))
    return out


def map_device_step(ctx, iid, dev: list[dict], p) -> None:
    """One step: every batch through dnaln_gpu_map_batch_device (inputs resident in HBM)."""
    from dnaln_b200 import _native as N
    L = N.lib()
    used = C.c_int64()
    for d in dev:
        rc = L.dnaln_gpu_map_batch_device(ctx.handle, iid, d["seq"].data_ptr(), d["off"].data_ptr(),
                                          d["len"].data_ptr(), d["hash"].data_ptr(), d["n"], C.byref(p),
                                          d["out"].data_ptr(), d["cig"].data_ptr(), d["cap"], C.byref(used))
        if rc:
            raise RuntimeError(L.dnaln_gpu_last_error(ctx.handle).decode())


def timed_steps(ctx, iid, dev, p, stream, steps: int, warmup: int) -> float:
    """Milliseconds per step over `steps` steps after `warmup` untimed ones (CUDA events on
    the launching stream, synchronized on both sides)."""
    import torch
    for _ in range(warmup):
        map_device_step(ctx, iid, dev, p)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        map_device_step(ctx, iid, dev, p)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def mixed_leg(ctx, stream, seed: int, steps: int, warmup: int) -> dict:
    """The mixed-length workload (1,000,000 reads, log-uniform 50-1000 bp, 2% with an 8-15 bp
    deletion, on the 4.6 Mbp genome), inputs resident in HBM, batches of 262,144, at band
    width 16 and 64: the batched form (short reads one thread each, long reads one thread
    each longest first, the rest one warp each; SW tasks longest first) against the plain
    per-batch form (every read one warp, SW tasks in read order)."""
    import dnaln_b200 as D
    from dnaln_b200 import synth
    g, reads, _ = synth.workload(MIXED, seed=seed)
    iid = ctx.index_build(g)
    dev = device_parts(reads)
    out = {"workload": f"{MIXED}: {synth.WORKLOADS[MIXED][2]}, k=15 w=10 A2 B4 O4 E2, batches of 262,144",
           "reads_per_step": len(reads), "mean_read_len": round(float(np.mean(reads.seq_len)), 1),
           "steps": steps, "warmup": warmup,
           "what": "reads/s, inputs resident in HBM, CUDA events; plain = every read one warp, SW tasks in read order"}
    try:
        for bw in (16, 64):
            p = D.default_map_params(bw=bw)
            ms_b = timed_steps(ctx, iid, dev, p, stream, steps, warmup)
            ctx.set_option("warp_seed_only", 1)
            ctx.set_option("length_order", 0)
            try:
                ms_p = timed_steps(ctx, iid, dev, p, stream, steps, warmup)
            finally:
                ctx.set_option("warp_seed_only", 0)
                ctx.set_option("length_order", 1)
            vb, vp = len(reads) / (ms_b / 1e3), len(reads) / (ms_p / 1e3)
            out[f"bw{bw}"] = {"batched": vb, "plain": vp, "batched_vs_plain": vb / vp,
                              "ms_per_step": {"batched": ms_b, "plain": ms_p}}
    finally:
        ctx.index_free(iid)
    return out


def serve_leg(ctx, seed: int, n_req: int, loads: list[float], lanes: int, bw: int) -> dict:
    """The serving workload (both indexes resident, Poisson arrivals, requests of log-uniform
    1-50,000 reads of U[100, 300] bp to either genome): capacity and p50 / p99 latency of the
    continuously batching server and of the plain one (one lane, one request per batch)."""
    import dnaln_b200 as D
    pools = ServePools(seed)
    iids = [ctx.index_build(g) for g in pools.genomes]
    try:
        points, reqs = serve_points(ctx, pools, iids, D.default_map_params(bw=bw), n_req, loads, lanes, seed)
    finally:
        for i in iids:
            ctx.index_free(i)
    lat = {}
    for name, pts in points.items():
        for v in pts:
            lat[f"{name}@{v['load']}"] = {"p50_ms": round(v["p50_ms"], 3), "p99_ms": round(v["p99_ms"], 3),
                                          "reads_per_s": v["reads_per_s"]}
    cap_b, cap_p = points["batched"][0]["reads_per_s"], points["plain"][0]["reads_per_s"]
    return {"requests_per_point": n_req, "mean_reads_per_request": float(np.mean([r[2] for r in reqs])),
            "lanes": lanes, "capacity_reads_per_s": {"batched": cap_b, "plain": cap_p},
            "batched_vs_plain_capacity": cap_b / cap_p, "latency": lat,
            "what": "load = fraction of that server's own capacity (saturation = all requests at once); "
                    "batched_at_plain_rates = the batching server at the plain server's offered rates; "
                    "latency from submit to completion, measured in the library"}


def int_roofline(local: int, stream, kernel: str, cells_per_launch: float, avg_launch_ms: float,
                 inst_per_cell: float | None) -> dict:
    """Integer roofline of an SW kernel: cells/s against the measured issue rate of the
    recurrence's instruction mix (dnaln_gpu_int_peak, run here) divided by the cost model's
    2.5 thread instructions per cell (at least 5 integer instructions per cell, two cells
    per 16x2 instruction)."""
    from dnaln_b200 import _native as N
    L = N.lib()
    rates = {}
    for mode, name in ((0, "add_dpxmax3_mix"), (1, "add"), (2, "dpxmax3")):
        r, ms = C.c_double(), C.c_double()
        rc = L.dnaln_gpu_int_peak(local, mode, C.c_void_p(stream.cuda_stream), C.byref(r), C.byref(ms))
        if rc:
            return {"error": f"dnaln_gpu_int_peak failed ({rc})"}
        rates[name] = r.value
    model = 2.5
    peak_cells = rates["add_dpxmax3_mix"] / model
    achieved = cells_per_launch / (avg_launch_ms / 1e3)
    out = {"kernel": kernel, "bound": "int", "achieved_cells_per_s": achieved, "peak_cells_per_s": peak_cells,
           "frac_int": achieved / peak_cells, "peak_thread_inst_per_s": rates,
           "model_thread_inst_per_cell": model, "cells_per_launch": cells_per_launch,
           "what": "peak = measured issue rate of 32-bit add + 16x2 DPX max3 (one to one, every SM, this run) / "
                   "2.5 thread instructions per cell (5 integer ops per cell, 2 cells per 16x2 op)"}
    if inst_per_cell:
        out["thread_inst_per_cell"] = inst_per_cell
        out["issue_frac"] = achieved * inst_per_cell / rates["add_dpxmax3_mix"]
    return out


def run_ours(args) -> None:
    import torch
    import dnaln_b200 as D
    from dnaln_b200 import _native as N
    from dnaln_b200 import synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    g, reads, truth = synth.workload(args.workload, seed=args.seed + 7919 * rank, n_reads=args.n_reads)
    n_reads = len(reads)
    p = D.default_map_params(bw=args.bw)
    ctx = D.Context(local)
    t_ix = time.perf_counter()
    iid = ctx.index_build(g)
    index_build_s = time.perf_counter() - t_ix
    L = N.lib()
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    # mapping lanes: further contexts share the one resident index (dnaln_gpu_index_attach),
    # each with its own stream and buffers; batch k of a step goes to lane k % lanes
    n_lanes = max(1, args.lanes)
    lanes = [(ctx, iid, stream)]
    for _ in range(1, n_lanes):
        c2 = D.Context(local)
        s2 = torch.cuda.Stream()
        c2.set_stream(s2.cuda_stream)
        lanes.append((c2, c2.index_attach(ctx, iid), s2))
    for c, _, _ in lanes:
        c.set_option("sw_form", args.sw_form)
        if args.dir_cap_bytes:
            c.set_option("dir_cap_bytes", args.dir_cap_bytes)

    spans = [(a, min(n_reads, a + BATCH)) for a in range(0, n_reads, BATCH)]
    parts = [reads.slice(a, b) for a, b in spans]

    # ---- device-resident inputs (value) --------------------------------------------
    dev = device_parts(reads, args.cigar_per_read)
    lane_parts = [dev[k::n_lanes] for k in range(n_lanes)]
    import concurrent.futures as cf
    pool = cf.ThreadPoolExecutor(max_workers=n_lanes) if n_lanes > 1 else None

    def step_device():
        if pool is None:
            map_device_step(ctx, iid, dev, p)
            return
        futs = [pool.submit(map_device_step, c, ix, lane_parts[k], p) for k, (c, ix, _) in enumerate(lanes)]
        for f in futs:
            f.result()

    def all_lanes(fn):
        for c, _, _ in lanes:
            fn(c)

    def merged_kernel_times():
        out = {}
        for c, _, _ in lanes:
            for k, (n, t) in c.kernel_times().items():
                a = out.get(k, (0, 0.0))
                out[k] = (a[0] + n, a[1] + t)
        return out

    def merged_stats():
        out = {}
        for c, _, _ in lanes:
            for k, v in c.stats().items():
                out[k] = out.get(k, 0) + v
        return out

    def barrier():
        if dist is not None:
            dist.barrier(device_ids=[local])
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # each lane's first batches alone: its tuners (SW kernel form, reads per block) time the
    # kernels without another lane's work on the GPU
    for c, ix, _ in lanes:
        map_device_step(c, ix, dev[:2], p)
        torch.cuda.synchronize()
    for _ in range(max(args.warmup, 3)):
        step_device()
    # kernel breakdown: every launch of PROFILE_STEPS untimed steps bracketed by event pairs
    # (one lane, batches in sequence, so each launch's span is its own)
    barrier()
    ctx.reset_stats()
    ctx.set_kernel_trace(True)
    for _ in range(PROFILE_STEPS):
        map_device_step(ctx, iid, dev, p)
    barrier()
    breakdown = ctx.kernel_times()
    ctx.set_kernel_trace(False)
    dom = max(breakdown, key=lambda k: breakdown[k][1])
    # timed region: only the dominant kernel's launches carry event pairs (one per batch).
    # The start event is on the first lane's stream and every other lane's stream waits for
    # it; the end event follows every lane's work (max over the lanes)
    all_lanes(lambda c: c.reset_stats())
    all_lanes(lambda c: c.set_kernel_trace(True, only=dom))
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _, _, sk in lanes[1:]:
        sk.wait_event(e0)
    for _ in range(args.steps):
        step_device()
    for _, _, sk in lanes[1:]:
        stream.wait_stream(sk)
    e1.record(stream)
    barrier()
    clk = clocks.result()
    ms = max_over_ranks(e0.elapsed_time(e1))
    st = merged_stats()
    ktimes = merged_kernel_times()
    # traceback SW tasks of the lanes whose dominant kernel is the traced one (a lane whose
    # tuner chose another SW form ran its tasks there)
    dom_tb_tasks = sum(c.stats()["sw_tasks_tb"] for c, _, _ in lanes if dom in c.kernel_times())
    all_lanes(lambda c: c.set_kernel_trace(False))
    value = world * n_reads * args.steps / (ms / 1e3)

    # ---- the plain per-batch form of the same step: every read through the warp-per-read
    # seeding and chaining kernels (no length buckets), SW tasks in read order ----------
    # (one lane, batches in sequence: the per-batch GPU path)
    ctx.set_option("warp_seed_only", 1)
    ctx.set_option("length_order", 0)
    map_device_step(ctx, iid, dev, p)
    barrier()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(args.steps):
        map_device_step(ctx, iid, dev, p)
    g1.record(stream)
    barrier()
    ms_plain = max_over_ranks(g0.elapsed_time(g1))
    ctx.set_option("warp_seed_only", 0)
    ctx.set_option("length_order", 1)
    plain_value = world * n_reads * args.steps / (ms_plain / 1e3)

    # ---- end to end through the host-buffer C call (e2e) ----------------------------
    host = []
    for part in parts:
        n = len(part)
        lens = part.seq_len
        cap = int(np.sum(2 * lens.astype(np.int64) + 3)) if not args.cigar_per_read else n * args.cigar_per_read
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        host.append(dict(n=n, cap=cap, seq=pin(part.seq), off=pin(part.seq_off[:-1]), len=pin(lens),
                         hash=pin(part.name_hash().view(np.int32)),
                         h2d=int(part.seq.nbytes) + 16 * n,
                         # two sets of result buffers: a step's batches are submitted while the
                         # previous step's are still in flight (each lane's queue stays full)
                         slots=[dict(out=torch.empty(n * 40, dtype=torch.uint8).pin_memory(),
                                     cig=torch.empty(cap, dtype=torch.int32).pin_memory(),
                                     used=C.c_int64(), ticket=None) for _ in range(2)]))
    # batch i goes to lane i % lanes (its worker and streams are its context's own); a batch
    # is resubmitted once its result set of two steps before has been waited for, so the
    # copies of one batch overlap the kernels of the others and no lane waits for the host
    for i, h in enumerate(host):
        h["lane"] = lanes[i % n_lanes]
    e2e_used = {}
    e2e_step = [0]

    def wait_slot(i, h, sl):
        if sl["ticket"] is not None:
            c = h["lane"][0]
            rc = L.dnaln_gpu_map_wait(c.handle, sl["ticket"])
            sl["ticket"] = None
            if rc:
                raise RuntimeError(L.dnaln_gpu_last_error(c.handle).decode())
            e2e_used[i] = sl["used"].value

    def step_e2e():
        k = e2e_step[0] & 1
        for i, h in enumerate(host):
            sl = h["slots"][k]
            wait_slot(i, h, sl)
            t = C.c_int64()
            c, ix, _ = h["lane"]
            rc = L.dnaln_gpu_map_submit(c.handle, ix, h["seq"].data_ptr(), h["off"].data_ptr(),
                                        h["len"].data_ptr(), h["hash"].data_ptr(), h["n"], C.byref(p),
                                        sl["out"].data_ptr(), sl["cig"].data_ptr(), h["cap"], C.byref(sl["used"]),
                                        C.byref(t))
            if rc:
                raise RuntimeError(L.dnaln_gpu_last_error(c.handle).decode())
            sl["ticket"] = t.value
        e2e_step[0] += 1

    def drain_e2e():
        for k in (e2e_step[0] & 1, 1 - (e2e_step[0] & 1)):  # the older step first
            for i, h in enumerate(host):
                wait_slot(i, h, h["slots"][k])

    # Batches stream through the host-buffer call two steps deep; the window opens with
    # the pipeline empty and closes once it has drained, so its fill and drain (the first
    # batch's copy in, the last batch's copy out, ~3 ms) are inside it. Over 10 steps they
    # cost 5% of the step time, over 30 about 1-2%.
    e2e_steps = args.e2e_steps or max(args.steps, 30)
    for _ in range(2):
        step_e2e()
    drain_e2e()
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    f0.record(stream)
    for _ in range(e2e_steps):
        step_e2e()
    drain_e2e()
    f1.record(stream)
    barrier()
    wall_e2e = time.perf_counter() - w0
    ms_e2e = max_over_ranks(f0.elapsed_time(f1))
    e2e_value = world * n_reads * e2e_steps / (ms_e2e / 1e3)
    # ---- the same step through the request server (dnaln_serve_*): each batch a request,
    # three lanes whose batches overlap on the device ------------------------------------
    e2e_serve = None
    if world == 1 and args.serve_e2e:
        from dnaln_b200.serve import Server
        with Server(ctx, lanes=3, max_batch_reads=BATCH) as srv:
            for _ in range(2):
                [srv.wait(r) for r in [srv.submit(iid, part, p) for part in parts]]
            barrier()
            s0 = time.perf_counter()
            for _ in range(e2e_steps):
                [srv.wait(r) for r in [srv.submit(iid, part, p) for part in parts]]
            barrier()
            ws = time.perf_counter() - s0
        e2e_serve = {"value": n_reads * e2e_steps / ws, "unit": METRIC, "ms_per_step": 1e3 * ws / e2e_steps,
                     "what": "dnaln_serve_submit / wait, each batch of the step one request, 3 lanes; wall clock"}

    # accuracy gate on the end-to-end results (Evaluator::add against the simulator's truth)
    acc = {"records": 0, "correct": 0, "mapq60_mapped": 0, "mapq60_wrong": 0}
    last = (e2e_step[0] - 1) & 1  # the result set the last timed step wrote
    for (a, b), h in zip(spans, host):
        sl = h["slots"][last]
        recs = sl["out"].numpy().view(D.MAP_RECORD_DTYPE)[:b - a]
        ev = D.evaluate(D.MapResult(recs, sl["cig"].numpy().view(np.uint32)), truth.contig[a:b], truth.start[a:b],
                        truth.rev[a:b])
        for k in acc:
            acc[k] += int(ev[k])
    h2d = sum(h["h2d"] for h in host)
    d2h = sum(40 * h["n"] for h in host) + 4 * sum(e2e_used.values())

    # ---- end to end from FASTQ text to SAM text (host parse and format included) -------
    e2e_text = None
    if args.workload == WORKLOAD and rank == 0 and world == 1:
        e2e_text = text_pipeline(ctx, iid, reads, g, p, max(2, min(args.steps, 5)))

    # ---- roofline of the dominant kernel ----------------------------------------------
    stage_ms = {"seed": st["ms_seed"], "chain": st["ms_chain"], "sw_score": st["ms_sw_score"], "sw_tb": st["ms_sw_tb"],
                "post": st["ms_post"]}
    mean_len = float(np.mean(reads.seq_len))
    launches, dom_ms = ktimes[dom]
    avg_launch_ms = dom_ms / launches
    algo = kernel_bytes(dom, dict(st, sw_tasks_tb=dom_tb_tasks), mean_len, args.bw)
    peak, peak_kind = measured_peaks()
    achieved = (algo / launches) / (avg_launch_ms / 1e3) / 1e9 if algo is not None else None
    traffic = None  # DRAM bytes per launch of this kernel from the committed ncu summary
    issue_active = None  # its fraction of issue slots used, same capture
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        try:
            prof = json.loads(tf.read_text())
            traffic = prof.get(args.workload, {}).get(dom.split("<")[0])
            issue_active = prof.get("issue_active", {}).get(args.workload, {}).get(dom.split("<")[0])
        except (OSError, ValueError, AttributeError):
            traffic = issue_active = None
    cells = st["cells"]
    sw_ms = st["ms_sw_score"] + st["ms_sw_tb"]
    ranked = sorted(breakdown.items(), key=lambda kv: -kv[1][1])
    kernels_total = sum(t for _, (_, t) in ranked) / PROFILE_STEPS
    kernels = {k: {"launches_per_step": n / PROFILE_STEPS, "ms_per_step": t / PROFILE_STEPS,
                   "share": t / PROFILE_STEPS / kernels_total} for k, (n, t) in ranked[:8]}
    rest = ranked[8:]
    if rest:
        kernels["(other kernels)"] = {"kernels": len(rest), "ms_per_step": sum(t for _, (_, t) in rest) / PROFILE_STEPS,
                                      "share": sum(t for _, (_, t) in rest) / PROFILE_STEPS / kernels_total}
    inst_per_cell = None  # thread instructions per cell of the dominant SW kernel, same ncu capture
    if tf.exists():
        try:
            inst_per_cell = json.loads(tf.read_text()).get("thread_inst_per_cell", {}).get(args.workload, {}).get(
                dom.split("<")[0])
        except (OSError, ValueError, AttributeError):
            inst_per_cell = None
    roof_int = None
    if dom.startswith("k_sw_u2<tb>") or dom.startswith("k_sw_wide<tb>"):
        W = 2 * args.bw + 1
        cells_per_launch = dom_tb_tasks * mean_len * W / launches
        roof_int = int_roofline(local, stream, dom, cells_per_launch, avg_launch_ms, inst_per_cell)
        one = breakdown[dom][1] / breakdown[dom][0]
        if "peak_cells_per_s" in roof_int:
            roof_int["achieved_cells_per_s_one_lane"] = cells_per_launch / (one / 1e3)
            roof_int["frac_int_one_lane"] = roof_int["achieved_cells_per_s_one_lane"] / roof_int["peak_cells_per_s"]

    out = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
           "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator, no dataset)",
           "config": dict(workload_config(n_reads, world, args.workload, args.bw, len(g.codes), mean_len),
                          lanes=n_lanes),
           "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                   "ms_per_step": ms_e2e / e2e_steps, "steps": e2e_steps, "wall_s": wall_e2e,
                   "note": "pinned host buffers in and out through dnaln_gpu_map_submit/wait, two steps in "
                           "flight; the copies overlap the neighbouring batches' kernels, pipeline fill and "
                           "drain are inside the window"},
           "gpu_launches": int(st["launches"]),
           "e2e_server": e2e_serve,
           "plain": {"value": plain_value, "ms_per_step": ms_plain / args.steps,
                     "what": "same step, every read through the warp-per-read kernels, SW tasks in read order"},
           "batched_vs_plain": value / plain_value,
           "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak if achieved is not None else None, "traffic": traffic,
                        "peak_kind": peak_kind,
                        "algorithmic_bytes_per_launch": algo / launches if algo is not None else None,
                        "avg_launch_ms": avg_launch_ms, "launches_timed": launches,
                        "issue_active": issue_active,
                        "issue_note": "fraction of the kernel's issue slots used, from the committed ncu capture "
                                      "(profiles/): HBM is not what bounds these integer kernels",
                        "avg_launch_ms_one_lane": breakdown[dom][1] / breakdown[dom][0],
                        "lanes_note": "avg_launch_ms is each launch's event span in the timed region, where the "
                                      "lanes' batches overlap on the GPU; avg_launch_ms_one_lane is the same kernel "
                                      "in the untimed one-lane traced steps"},
           "kernels": kernels, "kernels_note": f"untimed breakdown over {PROFILE_STEPS} one-lane steps, every launch "
                                               "traced; stages_ms_per_step and sw_gcups sum the lanes' event spans, "
                                               "which overlap",
           "stages_ms_per_step": {k: v / args.steps for k, v in stage_ms.items()},
           "sw_gcups": cells / (sw_ms / 1e3) / 1e9 if sw_ms > 0 else None,
           "sw_cells_per_step": cells / args.steps,
           "mapped_frac": st["mapped"] / max(st["reads"], 1),
           "accuracy": {"placed_correctly": acc["correct"] / max(acc["records"], 1), **acc,
                        "how": "dnaln_eval_records (Evaluator::add, tol 10) on the e2e records vs the generator's truth"},
           "clocks": clk,
           "index": dict(build_s=index_build_s, where="dnaln_gpu_index_build",
                         **{k: v for k, v in ctx.index_stats(iid).items() if k in ("n_keys", "device_bytes")}),
           "candidates_per_read": st["candidates"] / max(st["reads"], 1)}
    if e2e_text:
        out["e2e_text"] = e2e_text
    if rank == 0:
        out["index"]["image"] = index_image_round_trip(ctx, iid)
    if roof_int:
        out["roofline_int"] = roof_int
    # the other two measured workloads, compact (they close the line, so a truncated log
    # still shows them): mixed lengths batched vs plain, and the request server
    if rank == 0 and world == 1 and args.workload == WORKLOAD and not args.no_legs:
        ctx.index_free(iid)
        del dev, host
        torch.cuda.empty_cache()
        leg_steps, leg_warm = max(2, min(args.steps, 5)), 2
        out["mixed"] = mixed_leg(ctx, stream, args.seed, leg_steps, leg_warm)
        out["serve"] = serve_leg(ctx, args.seed, args.leg_requests, args.serve_loads, args.serve_lanes, args.bw)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(g, reads, p)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if pool is not None:
        pool.shutdown()
    for c, _, _ in lanes[1:]:
        c.close()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


# ---- serving: a Poisson request stream over two resident indexes ------------------------
SERVE = "serve"
SERVE_POOL = 400_000       # reads generated per genome; a request is a contiguous slice of a pool
SERVE_MAX_REQ = 50_000     # request sizes log-uniform in [1, 50,000] reads
SERVE_CIGAR_PER_READ = 16  # CIGAR capacity per read of a request's output (DNALN_ERR_CAPACITY if short)


class ServePools:
    """The two genomes of the serving workload (4.6 Mbp and 120 Mbp), a pool of reads of
    length uniform in [100, 300] on each, and a seeded request stream over them."""

    def __init__(self, seed: int, pool: int = SERVE_POOL):
        from dnaln_b200 import synth
        self.genomes = [synth.make_genome(synth.GENOME_4M6, seed), synth.make_genome(synth.GENOME_120M, seed + 1)]
        spec = synth.ReadsSpec(n_reads=pool, len_min=100, len_max=300, len_dist=2)
        self.pools = [synth.make_reads(g, spec, seed + 10 + i)[0] for i, g in enumerate(self.genomes)]
        self._arrays = None

    @property
    def arrays(self):
        """Per pool: reads, offsets, lengths and name hashes as the C ABI takes them (the
        hashes come from the mapping library, so the reference arm never asks for them)."""
        if self._arrays is None:
            self._arrays = [(rb.seq, np.ascontiguousarray(rb.seq_off[:-1]), np.ascontiguousarray(rb.seq_len),
                             rb.name_hash()) for rb in self.pools]
        return self._arrays

    def stream(self, n_req: int, seed: int):
        """(genome, first read, size) per request: genome 50/50, size log-uniform."""
        rng = np.random.default_rng(seed)
        g = rng.integers(0, 2, n_req)
        size = np.minimum(SERVE_MAX_REQ, np.floor(np.exp(rng.uniform(0, np.log(SERVE_MAX_REQ + 1), n_req)))).astype(
            np.int64)
        size = np.maximum(size, 1)
        start = np.array([rng.integers(0, len(self.pools[gi]) - sz + 1) for gi, sz in zip(g, size)], np.int64)
        return list(zip(g.tolist(), start.tolist(), size.tolist()))


def replay(srv, pools: ServePools, iids, reqs, rate: float | None, p) -> dict:
    """Submits reqs at Poisson arrival times of `rate` requests/s (None: all at once) from
    one producer thread, waits for all; latencies are the server's (submit to completion)."""
    from dnaln_b200 import _native as N
    L = N.lib()
    n_tot = sum(r[2] for r in reqs)
    rec = np.zeros(n_tot, dtype=__import__("dnaln_b200").MAP_RECORD_DTYPE)
    cig = np.zeros(n_tot * SERVE_CIGAR_PER_READ, np.uint32)
    used = [C.c_int64() for _ in reqs]
    ids = [C.c_int64() for _ in reqs]
    rng = np.random.default_rng(12345)
    arrivals = np.zeros(len(reqs)) if rate is None else np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
    base = np.concatenate([[0], np.cumsum([r[2] for r in reqs])])
    errors = []

    def produce():
        t0 = time.perf_counter()
        for i, (gi, a, m) in enumerate(reqs):
            while True:
                dt = arrivals[i] - (time.perf_counter() - t0)
                if dt <= 0:
                    break
                if dt > 0.002:
                    time.sleep(dt - 0.001)
            seq, off, ln, nh = pools.arrays[gi]
            rc = L.dnaln_serve_submit(srv._h, iids[gi], seq.ctypes.data, off.ctypes.data + 8 * a,
                                      ln.ctypes.data + 4 * a, nh.ctypes.data + 4 * a, m, C.byref(p),
                                      rec.ctypes.data + 40 * int(base[i]),
                                      cig.ctypes.data + 4 * SERVE_CIGAR_PER_READ * int(base[i]),
                                      SERVE_CIGAR_PER_READ * m, C.byref(used[i]), C.byref(ids[i]))
            if rc:
                errors.append(L.dnaln_serve_last_error(srv._h).decode())
                ids[i].value = 0

    srv.reset_stats()
    w0 = time.perf_counter()
    th = threading.Thread(target=produce)
    th.start()
    lat = []
    for i in range(len(reqs)):
        while ids[i].value == 0 and th.is_alive():
            time.sleep(0.0002)
        if ids[i].value == 0:
            continue
        x = C.c_double()
        rc = L.dnaln_serve_wait(srv._h, ids[i].value, C.byref(x))
        if rc:
            errors.append(L.dnaln_serve_last_error(srv._h).decode())
        lat.append(x.value)
    th.join()
    wall = time.perf_counter() - w0
    if errors:
        raise RuntimeError(f"serving failed: {errors[0]}")
    st = srv.stats()
    lat = np.array(lat)
    return {"offered_req_per_s": rate, "requests": len(reqs), "reads": n_tot, "wall_s": wall,
            "reads_per_s": n_tot / wall, "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()), "batches": st["batches"],
            "mean_batch_reads": st["mean_batch_reads"], "max_queue_depth": st["max_queue_depth"],
            "lane_ms": {k[3:]: st[k] for k in ("ms_form", "ms_gather", "ms_device", "ms_scatter", "ms_complete")}}


def serve_points(ctx, pools: ServePools, iids, p, n_req: int, loads: list[float], lanes: int, seed: int):
    """Replays the seeded request stream through the continuously batching server (`lanes`
    lanes, requests coalesced) and the plain one (one lane, one request per batch): first all
    at once (capacity), then at Poisson arrivals of each fraction in `loads` of that server's
    capacity; then the batching server at the plain server's rates. Returns (points by
    server, the requests)."""
    from dnaln_b200.serve import Server
    warm = pools.stream(64, seed + 99)
    reqs = pools.stream(n_req, seed + 100)
    modes = {"batched": dict(lanes=lanes, coalesce=True),
             "plain": dict(lanes=1, coalesce=False, max_batch_reads=BATCH)}
    points = {}
    for name, kw in modes.items():
        with Server(ctx, **kw) as srv:
            replay(srv, pools, iids, warm, None, p)        # warm-up: the lanes' staging and scratch
            replay(srv, pools, iids, reqs, None, p)        # grow to the stream's batch sizes
            sat = replay(srv, pools, iids, reqs, None, p)  # all requests at once: capacity
            cap_req = sat["requests"] / sat["wall_s"]
            pts = [dict(sat, load="saturation")]
            for frac in loads:
                r = replay(srv, pools, iids, reqs, frac * cap_req, p)
                r["load"] = frac
                pts.append(r)
            points[name] = pts
    # offered loads of the plain server, replayed on the batched one: same absolute rates
    with Server(ctx, **modes["batched"]) as srv:
        replay(srv, pools, iids, reqs, None, p)
        plain_cap = points["plain"][0]["requests"] / points["plain"][0]["wall_s"]
        points["batched_at_plain_rates"] = [dict(replay(srv, pools, iids, reqs, f * plain_cap, p),
                                                 load=f"{f} x plain capacity") for f in loads]
    return points, reqs


def run_serve(args) -> None:
    """The serving workload: both indexes resident, Poisson arrivals at a swept rate,
    requests of log-uniform 1..50,000 reads (length uniform in [100, 300]) to either genome.
    The continuously batching server (`--serve-lanes` lanes, default 4, requests coalesced) is measured against
    serving the same stream with the plain per-batch kernels (one lane, one request per batch)."""
    import torch
    import dnaln_b200 as D
    from dnaln_b200.serve import Server
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    pools = ServePools(args.seed)
    ctx = D.Context(local)
    t_ix = time.perf_counter()
    iids = [ctx.index_build(g) for g in pools.genomes]
    build_s = time.perf_counter() - t_ix
    p = D.default_map_params(bw=args.bw)
    n_req = args.serve_requests
    clocks = ClockSampler(local)
    clocks.start()
    points, reqs = serve_points(ctx, pools, iids, p, n_req, args.serve_loads, args.serve_lanes, args.seed)
    clk = clocks.result()
    mean_reads = float(np.mean([r[2] for r in reqs]))
    head = points["batched"][0]
    out = {"metric": "reads/s (served)", "value": head["reads_per_s"], "unit": "reads/s", "n_gpus": 1,
           "steps": len(args.serve_loads) + 1, "warmup": 1, "ms_per_step": 1e3 * head["wall_s"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
           "data": "synthetic (seeded generator, no dataset)",
           "config": {"workload": "serve: 4.6 Mbp + 120 Mbp indexes resident, Poisson arrivals, requests of "
                                  "log-uniform 1-50,000 reads of length U[100, 300] to either genome 50/50, "
                                  f"k=15 w=10 bw={args.bw}",
                      "requests_per_point": n_req, "mean_reads_per_request": mean_reads,
                      "l2": "no flush: each point streams its requests' reads (GBs) through the lanes",
                      "parallelism": "1 GPU, request server lanes"},
           "e2e": {"value": head["reads_per_s"], "unit": "reads/s",
                   "h2d_bytes_per_step": int(head["reads"] * (200 + 16)), "d2h_bytes_per_step": int(head["reads"] * 40),
                   "note": "host buffers in, records and CIGARs out: the served path is end to end"},
           "latency": {k: [{kk: v[kk] for kk in ("load", "offered_req_per_s", "reads_per_s", "p50_ms", "p99_ms",
                                                 "mean_ms", "max_ms", "batches", "mean_batch_reads",
                                                 "max_queue_depth", "lane_ms")} for v in pts]
                       for k, pts in points.items()},
           "batched_vs_plain_capacity": head["reads_per_s"] / points["plain"][0]["reads_per_s"],
           "index_build_s": build_s, "clocks": clk}
    print(json.dumps(out), flush=True)
    ctx.close()


def main():
    args = parse()
    if args.workload == SERVE and args.impl != "reference":
        run_serve(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
