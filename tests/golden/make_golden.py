"""Regenerates the golden fixtures of tests/golden/ from the reference compiled from its own
sources (oracle/_ref, built by `make -C oracle ref` where the dnaln sources are present).

    python tests/golden/make_golden.py

Inputs are seeded (numpy RNG for stage cases, the workload generator for whole batches);
expected outputs are the reference's: sketch (src/minimizer.cpp), Chainer::run
(src/chain.cpp), ScalarAligner both modes (src/align.cpp), and Mapper::map records +
append_sam text (src/mapper.cpp). Whole-batch inputs are stored as generator seeds plus a
SHA-256 of the generated bytes, so a change of the generator is detected, not absorbed.
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE.parent))

import dnaln_b200 as D  # noqa: E402
import oracle  # noqa: E402
from dnaln_b200 import synth  # noqa: E402
from helpers import SCHEMES, known_answer_anchors, random_anchor_set, random_codes, random_tasks  # noqa: E402

MAP_CASES = [("small-1Mbp-10k-150bp", 7, 2000, 16), ("repeat-2Mbp-20k-150bp", 3, 3000, 16),
             ("repeat-2Mbp-20k-150bp", 3, 1500, 64), ("mixed-1Mbp-5k-50to1000bp", 4, 600, 64)]


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def flat(seqs):
    lens = np.array([len(s) for s in seqs], np.int64)
    off = np.zeros(len(seqs) + 1, np.int64)
    off[1:] = np.cumsum(lens)
    return (np.concatenate(seqs) if off[-1] else np.zeros(0, np.uint8)).astype(np.uint8), off


def main():
    ref = oracle.Reference()
    rng = np.random.default_rng(20260)

    # sketch: the reference's brute-force case shapes (k 5..24, w 1..20, N in a third)
    seqs, ks, ws, mh, mp, ms, mo = [], [], [], [], [], [], [0]
    for trial in range(80):
        k, w = 5 + int(rng.integers(20)), 1 + int(rng.integers(20))
        s = random_codes(rng, 50 + int(rng.integers(400)), 0.01 if trial % 3 == 0 else 0.0)
        h, p, st = ref.sketch(s, k, w, 1000)
        seqs.append(s)
        ks.append(k)
        ws.append(w)
        mh.append(h)
        mp.append(p)
        ms.append(st)
        mo.append(mo[-1] + len(h))
    sb, so = flat(seqs)
    np.savez_compressed(HERE / "sketch.npz", seq=sb, seq_off=so, k=np.array(ks), w=np.array(ws),
                        hash=np.concatenate(mh), pos=np.concatenate(mp), strand=np.concatenate(ms),
                        min_off=np.array(mo, np.int64))

    # banded SW, both modes, the four scoring schemes
    out = {}
    for si, sc in enumerate(SCHEMES):
        qs, ts = random_tasks(rng, 150, sc[5], max_len=200)
        qb, qo = flat(qs)
        tb, to = flat(ts)
        so_ = ref.align(qs, ts, False, sc)
        tr = ref.align(qs, ts, True, sc)
        cig, co = flat([x[6].view(np.uint8) for x in tr])
        out.update({f"q{si}": qb, f"qo{si}": qo, f"t{si}": tb, f"to{si}": to,
                    f"score_only{si}": np.array([x[0] for x in so_], np.int32),
                    f"res{si}": np.array([x[:6] for x in tr], np.int32), f"cig{si}": cig.view(np.uint32),
                    f"co{si}": co // 4})
    np.savez_compressed(HERE / "align.npz", schemes=np.array(SCHEMES, np.int32), **out)

    # chaining: random sets + the reference's known-answer set, three parameter sets
    sets = [random_anchor_set(rng, int(rng.integers(0, 50)), int(rng.integers(0, 30))) for _ in range(120)]
    sets.append(known_answer_anchors())
    params = [(5000, 16, 50, 20, 2), (200, 5, 10, 0, 1), (100000, 64, 80, 30, 3)]
    rows = {"r": [], "q": [], "s": [], "off": [0]}
    for r_, q_, s_ in sets:
        rows["r"].append(r_)
        rows["q"].append(q_)
        rows["s"].append(s_)
        rows["off"].append(rows["off"][-1] + len(r_))
    res = {}
    for pi, cp in enumerate(params):
        cols = {k: [] for k in ("score", "strand", "n_anchors", "dmin", "dmax", "rpos")}
        coff = [0]
        for r_, q_, s_ in sets:
            _, ch = ref.chain(r_, q_, s_, 15, cp)
            for k in cols:
                cols[k].append(ch[k])
            coff.append(coff[-1] + len(ch["score"]))
        for k, v in cols.items():
            res[f"{k}{pi}"] = np.concatenate(v)
        res[f"coff{pi}"] = np.array(coff, np.int64)
    np.savez_compressed(HERE / "chain.npz", rpos=np.concatenate(rows["r"]), qpos=np.concatenate(rows["q"]),
                        strand=np.concatenate(rows["s"]), set_off=np.array(rows["off"], np.int64),
                        params=np.array(params, np.int32), **res)

    # whole batches: records, CIGARs and the SAM body of the reference mapper
    mres = {}
    for ci, (wl, seed, n, bw) in enumerate(MAP_CASES):
        g, reads, _ = synth.workload(wl, seed=seed, n_reads=n, with_qual=True)
        p = D.default_map_params(bw=bw)
        rec, cig, co, sam = ref.map(ref.genome(g), reads, p, want_sam=True)
        mres.update({f"rec{ci}": rec, f"cig{ci}": cig, f"co{ci}": co,
                     f"genome_sha{ci}": np.frombuffer(sha(g.codes).encode(), np.uint8),
                     f"reads_sha{ci}": np.frombuffer(sha(reads.seq, reads.seq_off, reads.names).encode(), np.uint8),
                     f"sam_sha{ci}": np.frombuffer(hashlib.sha256(sam).hexdigest().encode(), np.uint8)})
    np.savez_compressed(HERE / "map.npz", cases=np.array([f"{a}|{b}|{c}|{d}" for a, b, c, d in MAP_CASES]), **mres)
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
