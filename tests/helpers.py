"""Seeded generators of test inputs (numpy RNG; shapes follow the reference's tests:
random sequences with N, related/unrelated SW pairs with short targets, anchor sets)."""
from __future__ import annotations

import numpy as np

# The four scoring schemes the reference tests every kernel with (match, mismatch,
# gap_open, gap_ext, ambig, bw): default, BWA-like, short-read-like, zero gap-open.
SCHEMES = [(2, 4, 4, 2, 1, 16), (1, 4, 6, 1, 1, 8), (2, 8, 12, 2, 1, 5), (3, 2, 0, 3, 1, 21)]


def random_codes(rng: np.random.Generator, n: int, n_rate: float = 0.0) -> np.ndarray:
    c = rng.integers(0, 4, size=n).astype(np.uint8)
    if n_rate > 0:
        c[rng.random(n) < n_rate] = 4
    return c


def mutate(rng: np.random.Generator, s: np.ndarray, sub: float, indel: float) -> np.ndarray:
    out = []
    for x in s:
        if rng.random() < indel:
            if rng.integers(2):
                continue  # deletion
            out.append(int(rng.integers(4)))  # insertion
        out.append(int(rng.integers(4)) if rng.random() < sub else int(x))
    return np.array(out, np.uint8)


def random_tasks(rng: np.random.Generator, n: int, bw: int, max_len: int = 300):
    """Banded-SW problems: 80% target = flank + mutated query + flank shifted within the
    band, 20% unrelated; a quarter with 2% N; 10% with truncated (N-padded) targets."""
    qs, ts = [], []
    for _ in range(n):
        ql = 1 + int(rng.integers(max_len))
        nrate = 0.02 if rng.integers(4) == 0 else 0.0
        q = random_codes(rng, ql, nrate)
        tl = ql + 2 * bw
        if rng.integers(5) == 0:
            t = random_codes(rng, tl, nrate)
        else:
            shift = int(rng.integers(2 * bw + 1))
            m = mutate(rng, q, 0.03 * rng.random(), 0.02 * rng.random())
            t = np.concatenate([random_codes(rng, shift), m, random_codes(rng, max(0, tl - shift - len(m)))])
        if rng.integers(10) == 0:
            t = t[:int(rng.integers(len(t) + 1))]
        qs.append(q)
        ts.append(t.astype(np.uint8))
    return qs, ts


def random_anchor_set(rng: np.random.Generator, n_true: int, n_noise: int):
    """Colinear anchors on one or two diagonals (with small indels) plus scattered noise."""
    r, q, s = [], [], []
    strand = int(rng.integers(2))
    base = int(rng.integers(1000, 1_000_000))
    qp, rp = int(rng.integers(0, 20)), base
    for _ in range(n_true):
        step = int(rng.integers(3, 20))
        qp += step
        rp += step + int(rng.integers(-3, 4)) * (rng.random() < 0.2)
        r.append(rp)
        q.append(qp)
        s.append(strand)
    for _ in range(n_noise):
        r.append(int(rng.integers(0, 2_000_000)))
        q.append(int(rng.integers(0, 300)))
        s.append(int(rng.integers(2)))
    # duplicates of (strand, rpos, qpos) cannot occur in the mapping path: drop them
    seen, rr, qq, ss = set(), [], [], []
    for a, b, c in zip(r, q, s):
        if (c, a, b) not in seen:
            seen.add((c, a, b))
            rr.append(a)
            qq.append(b)
            ss.append(c)
    perm = rng.permutation(len(rr))
    return (np.array(rr, np.uint32)[perm], np.array(qq, np.int32)[perm], np.array(ss, np.uint32)[perm])


def known_answer_anchors():
    """The reference's fixed chaining case: 10 anchors on one diagonal with a 3 bp
    deletion after the fifth, plus two noise anchors; expected best chain has 10 anchors,
    dmin 1000, dmax 1003."""
    r = [1000 + i * 12 + (3 if i >= 5 else 0) for i in range(10)] + [50000, 90000]
    q = [i * 12 for i in range(10)] + [30, 60]
    s = [0] * 10 + [0, 1]
    return np.array(r, np.uint32), np.array(q, np.int32), np.array(s, np.uint32)
