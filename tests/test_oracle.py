"""Pins the oracle (oracle/dnaln_oracle.c) to the reference: against the committed golden
fixtures made from the reference compiled from its own sources (tests/golden/), and live
against that compiled reference where it is present. CPU only."""
import hashlib
from pathlib import Path

import numpy as np
import pytest

import dnaln_b200 as D
from dnaln_b200 import synth
from helpers import SCHEMES, known_answer_anchors, random_anchor_set, random_codes, random_tasks

GOLD = Path(__file__).resolve().parent / "golden"


def test_sketch_golden(port):
    z = np.load(GOLD / "sketch.npz")
    for i in range(len(z["k"])):
        s = z["seq"][z["seq_off"][i]:z["seq_off"][i + 1]]
        h, p, st = port.sketch(s, int(z["k"][i]), int(z["w"][i]), 1000)
        a, b = z["min_off"][i], z["min_off"][i + 1]
        assert np.array_equal(h, z["hash"][a:b]) and np.array_equal(p, z["pos"][a:b])
        assert np.array_equal(st, z["strand"][a:b])


def test_align_golden_four_schemes_both_modes(port):
    z = np.load(GOLD / "align.npz")
    for si, sc in enumerate(map(tuple, z["schemes"])):
        qo, to = z[f"qo{si}"], z[f"to{si}"]
        qs = [z[f"q{si}"][qo[i]:qo[i + 1]] for i in range(len(qo) - 1)]
        ts = [z[f"t{si}"][to[i]:to[i + 1]] for i in range(len(to) - 1)]
        so = port.align(qs, ts, False, sc)
        tb = port.align(qs, ts, True, sc)
        assert [x[0] for x in so] == list(z[f"score_only{si}"])
        co = z[f"co{si}"]
        for i, x in enumerate(tb):
            assert tuple(x[:6]) == tuple(z[f"res{si}"][i])
            assert np.array_equal(x[6], z[f"cig{si}"][co[i]:co[i + 1]])


def test_chain_golden(port):
    z = np.load(GOLD / "chain.npz")
    so = z["set_off"]
    for pi, cp in enumerate(map(tuple, z["params"])):
        coff = z[f"coff{pi}"]
        for i in range(len(so) - 1):
            _, ch = port.chain(z["rpos"][so[i]:so[i + 1]], z["qpos"][so[i]:so[i + 1]], z["strand"][so[i]:so[i + 1]],
                               15, cp)
            for k in ch:
                assert np.array_equal(ch[k], z[f"{k}{pi}"][coff[i]:coff[i + 1]]), (pi, i, k)


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def test_map_golden(port):
    z = np.load(GOLD / "map.npz")
    for ci, case in enumerate(z["cases"]):
        wl, seed, n, bw = str(case).split("|")
        g, reads, _ = synth.workload(wl, seed=int(seed), n_reads=int(n), with_qual=True)
        # the generator still produces the fixture's inputs
        assert _sha(g.codes) == z[f"genome_sha{ci}"].tobytes().decode()
        assert _sha(reads.seq, reads.seq_off, reads.names) == z[f"reads_sha{ci}"].tobytes().decode()
        rec, cig, co = port.map(port.index(g), reads, D.default_map_params(bw=int(bw)))
        assert np.array_equal(rec, z[f"rec{ci}"]) and np.array_equal(cig, z[f"cig{ci}"])
        assert np.array_equal(co, z[f"co{ci}"])
        # our SAM formatter on these records reproduces the reference's SAM body
        out = np.zeros(len(rec), dtype=D.MAP_RECORD_DTYPE)
        for j, f in enumerate(("contig", "pos", "rev", "mapq", "score", "nm", "n_cand")):
            out[f] = rec[:, j]
        out["cigar_off"], out["cigar_len"] = co[:-1], np.diff(co)
        sam = D.sam_format(reads, D.MapResult(out, cig), g)
        assert hashlib.sha256(sam).hexdigest() == z[f"sam_sha{ci}"].tobytes().decode()


def test_known_answers(port):
    # the reference's fixed chaining case and its perfect-match alignment
    _, ch = port.chain(*known_answer_anchors(), 15)
    assert ch["n_anchors"][0] == 10 and ch["dmin"][0] == 1000 and ch["dmax"][0] == 1003
    rng = np.random.default_rng(17)
    q = random_codes(rng, 150)
    t = np.concatenate([random_codes(rng, 16), q, random_codes(rng, 16)])
    (score, qb, qe, tb, te, nm, cig), = port.align([q], [t], True)
    assert (score, qb, qe, tb, nm) == (300, 0, 150, 16, 0) and D.cigar_to_string(cig) == "150M"


def test_chain_cost_contraction_does_not_change_the_table(port):
    # gcc -march=native contracts the cost expression into an FMA; truncation is unchanged
    assert port.chain_cost_mismatches(28, 2000) == 0


def test_port_matches_reference_live_stages(port, ref):
    rng = np.random.default_rng(99)
    for trial in range(150):
        k, w = 4 + int(rng.integers(25)), 1 + int(rng.integers(40))
        s = random_codes(rng, int(rng.integers(0, 600)), [0, 0.005, 0.05][trial % 3])
        for a, b in zip(port.sketch(s, k, w, 7), ref.sketch(s, k, w, 7)):
            assert np.array_equal(a, b), (trial, k, w)
    for sc in SCHEMES:
        qs, ts = random_tasks(rng, 120, sc[5])
        for tb in (False, True):
            for a, b in zip(port.align(qs, ts, tb, sc), ref.align(qs, ts, tb, sc)):
                assert tuple(a[:6]) == tuple(b[:6]) and np.array_equal(a[6], b[6])
    for _ in range(200):
        s = random_anchor_set(rng, int(rng.integers(0, 80)), int(rng.integers(0, 60)))
        (sa, ca), (sb, cb) = port.chain(*s, 15), ref.chain(*s, 15)
        assert all(np.array_equal(x, y) for x, y in zip(sa, sb))
        assert all(np.array_equal(ca[k], cb[k]) for k in ca)


@pytest.mark.parametrize("wl,seed,n,bw", [("small-1Mbp-10k-150bp", 11, 3000, 16), ("repeat-2Mbp-20k-150bp", 12, 4000, 16),
                                          ("mixed-1Mbp-5k-50to1000bp", 13, 800, 64)])
def test_port_matches_reference_live_map(port, ref, wl, seed, n, bw):
    g, reads, _ = synth.workload(wl, seed=seed, n_reads=n)
    p = D.default_map_params(bw=bw)
    a = port.map(port.index(g), reads, p)
    b = ref.map(ref.genome(g), reads, p)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_index_port_matches_reference(port, ref):
    g = synth.make_genome(synth.GENOME_REPEAT_2M, 8)
    pi, rg = port.index(g), ref.genome(g)
    ps, rs = pi.stats(), rg.stats()
    for k in rs:
        assert ps[k] == rs[k]
    keys, offs, cnts, pos = pi.export()
    rng = np.random.default_rng(0)
    present = keys[keys != np.uint64(2**64 - 1)]
    for h in list(present[rng.permutation(len(present))[:3000]]) + [1 << 40, 12345]:
        off, n = pi.lookup(int(h))
        assert np.array_equal(pos[off:off + n], rg.lookup(int(h)))
