/* dnaln_oracle.c — TEST INFRASTRUCTURE ONLY. A plain-C restatement of dnaln's read-mapping
 * path (sketch -> index probe -> chain -> banded SW + traceback -> MAPQ), written for
 * clarity, not speed: it is the oracle the CUDA path is compared against and the scalar
 * CPU baseline. It is never linked into the product. Its agreement with the reference is
 * pinned by tests/test_oracle.py (against the reference built from its own sources in
 * oracle/_ref) and by the committed fixtures in tests/golden/.
 *
 * Each function names the dnaln source lines (src/...) whose behaviour it restates. */
#include "dnaln_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_INVALID (~0ULL) /* palindromic k-mer / empty bucket key */

/* --------------------------------------------------------------------------- utilities */

/* Thomas Wang's 64-bit invertible integer mix, every step masked to 2k bits
 * (src/minimizer.hpp:21-31). The index keys are defined by these exact steps. */
uint64_t or_hash64(uint64_t key, uint64_t mask) {
  key = (~key + (key << 21)) & mask;
  key = key ^ key >> 24;
  key = ((key + (key << 3)) + (key << 8)) & mask;
  key = key ^ key >> 14;
  key = ((key + (key << 2)) + (key << 4)) & mask;
  key = key ^ key >> 28;
  key = (key + (key << 31)) & mask;
  return key;
}

/* ASCII -> 0..4: A/a 0, C/c 1, G/g 2, T/t/U/u 3, anything else 4 (src/common.hpp:23-38). */
static uint8_t nt4(unsigned char c) {
  switch (c) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': case 'U': case 'u': return 3;
    default: return 4;
  }
}

void or_encode(const char* s, int64_t n, uint8_t* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = nt4((unsigned char)s[i]);
}

/* Reverse complement of codes; N stays N (src/common.hpp:34,40-42). */
void or_revcomp(const uint8_t* in, int64_t n, uint8_t* out) {
  for (int64_t i = 0; i < n; ++i) {
    const uint8_t c = in[n - 1 - i];
    out[i] = c < 4 ? (uint8_t)(3 - c) : 4;
  }
}

/* FNV-1a over the read name, the tie-break hash (src/common.hpp:136-140). */
uint32_t or_fnv1a(const char* s, int64_t n) {
  uint32_t h = 2166136261u;
  for (int64_t i = 0; i < n; ++i) h = (h ^ (unsigned char)s[i]) * 16777619u;
  return h;
}

static int ilog2_u64(uint64_t x) { return 63 - __builtin_clzll(x); }

/* ----------------------------------------------------------------------------- sketch */

/* Minimizers of seq[0, len) (src/minimizer.cpp:5-68), restated from the definition the
 * reference's streamed van Herk scheme computes: inside each N-free run, each window of
 * w consecutive k-mers selects its leftmost smallest canonical hash; palindromic k-mers
 * (forward == reverse complement) never win; a selection is emitted unless its position
 * equals the last emitted one (`last` survives N runs). */
int64_t or_sketch(const uint8_t* seq, uint32_t len, int k, int w, uint32_t offset, uint64_t* hash, uint32_t* pos,
                  uint32_t* strand, int64_t cap) {
  const uint64_t mask = (k >= 32) ? ~0ULL : ((1ULL << (2 * k)) - 1);
  uint64_t* kh = (uint64_t*)malloc(sizeof(uint64_t) * (len + 1));
  uint32_t* kp = (uint32_t*)malloc(sizeof(uint32_t) * (len + 1));
  uint32_t* ks = (uint32_t*)malloc(sizeof(uint32_t) * (len + 1));
  int64_t n_out = 0, last = -1;
  int run = 0;
  int64_t nk = 0; /* k-mers in the current N-free run */
  for (uint32_t i = 0; i < len; ++i) {
    if (seq[i] > 3) {
      run = 0;
      nk = 0;
      continue;
    }
    if (++run < k) continue;
    const uint32_t s = i - (uint32_t)k + 1;
    uint64_t fwd = 0, rev = 0;
    for (int m = 0; m < k; ++m) {
      fwd |= (uint64_t)seq[s + m] << (2 * (k - 1 - m));
      rev |= (uint64_t)(3 - seq[s + m]) << (2 * m);
    }
    const uint32_t st = rev < fwd;
    kh[nk] = fwd != rev ? or_hash64(st ? rev : fwd, mask) : OR_INVALID;
    kp[nk] = s;
    ks[nk] = st;
    ++nk;
    if (nk >= w) {
      int64_t b = nk - w;
      for (int64_t j = nk - w + 1; j < nk; ++j)
        if (kh[j] < kh[b]) b = j;
      if (kh[b] != OR_INVALID) {
        if ((int64_t)kp[b] != last) {
          if (n_out < cap) {
            hash[n_out] = kh[b];
            pos[n_out] = kp[b] + offset;
            strand[n_out] = ks[b];
          }
          ++n_out;
        }
        last = kp[b];
      }
    }
  }
  free(kh);
  free(kp);
  free(ks);
  return n_out <= cap ? n_out : -n_out;
}

/* ------------------------------------------------------------------------------ index */

struct or_index {
  uint64_t* key;
  uint32_t *off, *cnt, *pos;
  uint64_t mask, n_buckets, n_keys, n_pos;
  uint32_t max_count;
  int k, w;
};

typedef struct {
  uint64_t hash;
  uint32_t pos, strand;
} or_min;

static int cmp_min(const void* a, const void* b) {
  const or_min* x = (const or_min*)a;
  const or_min* y = (const or_min*)b;
  if (x->hash != y->hash) return x->hash < y->hash ? -1 : 1;
  return x->pos < y->pos ? -1 : (x->pos > y->pos);
}

/* Index build (src/index.cpp:10-45): sketch every contig at its global offset, sort by
 * (hash, pos), one bucket per distinct hash in an open-addressing table of the smallest
 * power of two >= max(16, 2 * n_keys) with linear probing from hash & mask; the
 * occurrence list of a key is the contiguous run of (pos << 1 | strand). */
or_index* or_index_build(const uint8_t* codes, uint64_t n_bases, const uint64_t* contig_off,
                         const uint32_t* contig_len, int32_t n_contigs, int k, int w) {
  (void)n_bases;
  int64_t cap = 1024;
  for (int32_t c = 0; c < n_contigs; ++c) cap += contig_len[c];
  or_min* mins = (or_min*)malloc(sizeof(or_min) * (size_t)cap);
  uint64_t* h = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)cap);
  uint32_t* p = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)cap);
  uint32_t* s = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)cap);
  int64_t n = 0;
  for (int32_t c = 0; c < n_contigs; ++c) {
    const int64_t m = or_sketch(codes + contig_off[c], contig_len[c], k, w, (uint32_t)contig_off[c], h, p, s, cap);
    for (int64_t i = 0; i < m; ++i) mins[n + i] = (or_min){h[i], p[i], s[i]};
    n += m;
  }
  free(h);
  free(p);
  free(s);
  qsort(mins, (size_t)n, sizeof(or_min), cmp_min);

  or_index* ix = (or_index*)calloc(1, sizeof(or_index));
  ix->k = k;
  ix->w = w;
  for (int64_t i = 0; i < n; ++i)
    if (i == 0 || mins[i].hash != mins[i - 1].hash) ++ix->n_keys;
  uint64_t nb = 16;
  while (nb < ix->n_keys * 2) nb <<= 1;
  ix->n_buckets = nb;
  ix->mask = nb - 1;
  ix->key = (uint64_t*)malloc(sizeof(uint64_t) * nb);
  ix->off = (uint32_t*)calloc(nb, sizeof(uint32_t));
  ix->cnt = (uint32_t*)calloc(nb, sizeof(uint32_t));
  for (uint64_t i = 0; i < nb; ++i) ix->key[i] = OR_INVALID;
  ix->n_pos = (uint64_t)n;
  ix->pos = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n + 1));
  for (int64_t i = 0; i < n;) {
    int64_t j = i;
    for (; j < n && mins[j].hash == mins[i].hash; ++j) ix->pos[j] = mins[j].pos << 1 | mins[j].strand;
    uint64_t b = mins[i].hash & ix->mask;
    while (ix->key[b] != OR_INVALID) b = (b + 1) & ix->mask;
    ix->key[b] = mins[i].hash;
    ix->off[b] = (uint32_t)i;
    ix->cnt[b] = (uint32_t)(j - i);
    if ((uint32_t)(j - i) > ix->max_count) ix->max_count = (uint32_t)(j - i);
    i = j;
  }
  free(mins);
  return ix;
}

void or_index_free(or_index* ix) {
  if (!ix) return;
  free(ix->key);
  free(ix->off);
  free(ix->cnt);
  free(ix->pos);
  free(ix);
}

void or_index_stats(const or_index* ix, uint64_t* out5) {
  out5[0] = ix->n_keys;
  out5[1] = ix->n_pos;
  out5[2] = ix->max_count;
  out5[3] = ix->n_buckets * 16 + ix->n_pos * 4; /* src/index.hpp:46 */
  out5[4] = ix->n_buckets;
}

void or_index_export(const or_index* ix, uint64_t* keys, uint32_t* offs, uint32_t* cnts, uint32_t* positions) {
  memcpy(keys, ix->key, sizeof(uint64_t) * ix->n_buckets);
  memcpy(offs, ix->off, sizeof(uint32_t) * ix->n_buckets);
  memcpy(cnts, ix->cnt, sizeof(uint32_t) * ix->n_buckets);
  memcpy(positions, ix->pos, sizeof(uint32_t) * ix->n_pos);
}

/* Linear probe from hash & mask until the key or an empty bucket (src/index.hpp:24-38). */
uint32_t or_index_lookup(const or_index* ix, uint64_t h, uint32_t* off) {
  uint64_t i = h & ix->mask;
  for (;;) {
    if (ix->key[i] == h) {
      *off = ix->off[i];
      return ix->cnt[i];
    }
    if (ix->key[i] == OR_INVALID) {
      *off = 0;
      return 0;
    }
    i = (i + 1) & ix->mask;
  }
}

/* ------------------------------------------------------------------------------ chain */

typedef struct {
  uint32_t rpos;
  int32_t qpos;
  uint32_t strand;
} or_anchor;

static int cmp_anchor(const void* a, const void* b) {
  const or_anchor* x = (const or_anchor*)a;
  const or_anchor* y = (const or_anchor*)b;
  if (x->strand != y->strand) return x->strand < y->strand ? -1 : 1;
  if (x->rpos != y->rpos) return x->rpos < y->rpos ? -1 : 1;
  return x->qpos < y->qpos ? -1 : (x->qpos > y->qpos);
}

typedef struct {
  int32_t key1, key2; /* sort keys */
  int32_t idx;
} or_kv;

static int cmp_kv(const void* a, const void* b) {
  const or_kv* x = (const or_kv*)a;
  const or_kv* y = (const or_kv*)b;
  if (x->key1 != y->key1) return x->key1 > y->key1 ? -1 : 1; /* key1 descending */
  return x->key2 < y->key2 ? -1 : (x->key2 > y->key2);      /* then key2 ascending */
}

/* Gap cost of the chaining DP, int(0.01*k*dd + 0.5*floor(log2 dd)) (src/chain.cpp:36). */
static int chain_cost(int k, int64_t dd) {
  return dd ? (int)(0.01 * k * (double)dd + 0.5 * ilog2_u64((uint64_t)dd)) : 0;
}

/* Number of (k, dd) with k in [k_lo, k_hi], dd in [1, dd_max] where the chain gap cost
 * truncates differently with the product 0.01*k*dd fused into the add (the FMA that
 * gcc -march=native emits for src/chain.cpp:36) than without: the product path computes
 * the cost table on the host and relies on this being 0 over its parameter range. */
int64_t or_chain_cost_mismatches(int k_lo, int k_hi, int dd_max) {
  int64_t bad = 0;
  for (int k = k_lo; k <= k_hi; ++k)
    for (int dd = 1; dd <= dd_max; ++dd) {
      volatile double a = 0.01 * k;
      volatile double prod = a * (double)dd;
      const double half = 0.5 * ilog2_u64((uint64_t)dd);
      const int plain = (int)(prod + half);
      const int fused1 = (int)fma(a, (double)dd, half);
      const int fused2 = (int)fma(0.5, (double)ilog2_u64((uint64_t)dd), prod);
      bad += (plain != fused1) + (plain != fused2);
    }
  return bad;
}

typedef struct {
  int32_t score;
  uint32_t strand;
  int32_t n;
  int64_t dmin, dmax;
  uint32_t rpos;
} or_chain_t;

/* Chaining (src/chain.cpp:12-69): sort by (strand, rpos, qpos); f(i) = max(k, f(j) +
 * min(dq, dr, k) - cost(|dr - dq|)) over up to `lookback` predecessors scanned nearest
 * first, stopping at a strand change or dr > max_gap, skipping non-increasing pairs and
 * |dr - dq| > band, strict '>' so the nearest j wins ties. Then chains are extracted
 * from end points in (f desc, index asc) order, each walking prev until an anchor that
 * is already used, and finally ordered by score, stably. */
static int64_t chain_core(or_anchor* a, int64_t n, int k, const or_chain_params* p, or_chain_t* out) {
  if (n == 0) return 0;
  qsort(a, (size_t)n, sizeof(or_anchor), cmp_anchor);
  int32_t* f = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  int32_t* prev = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    int best = k, best_j = -1;
    const int64_t lo = i - p->lookback > 0 ? i - p->lookback : 0;
    for (int64_t j = i - 1; j >= lo; --j) {
      if (a[j].strand != a[i].strand) break;
      const int64_t dr = (int64_t)a[i].rpos - (int64_t)a[j].rpos;
      if (dr > p->max_gap) break;
      const int64_t dq = (int64_t)a[i].qpos - (int64_t)a[j].qpos;
      if (dr <= 0 || dq <= 0) continue;
      const int64_t dd = dr > dq ? dr - dq : dq - dr;
      if (dd > p->band) continue;
      int64_t g = dq < dr ? dq : dr;
      if (g > k) g = k;
      const int sc = f[j] + (int)g - chain_cost(k, dd);
      if (sc > best) {
        best = sc;
        best_j = (int)j;
      }
    }
    f[i] = best;
    prev[i] = best_j;
  }
  or_kv* ord = (or_kv*)malloc(sizeof(or_kv) * (size_t)n);
  for (int64_t i = 0; i < n; ++i) ord[i] = (or_kv){f[i], (int32_t)i, (int32_t)i};
  qsort(ord, (size_t)n, sizeof(or_kv), cmp_kv);
  uint8_t* used = (uint8_t*)calloc((size_t)n, 1);
  or_chain_t* tmp = (or_chain_t*)malloc(sizeof(or_chain_t) * (size_t)n);
  int64_t m = 0;
  for (int64_t e = 0; e < n; ++e) {
    const int end = ord[e].idx;
    if (used[end]) continue;
    int i = end, cnt = 0;
    int64_t dmin = INT64_MAX, dmax = INT64_MIN;
    while (i >= 0 && !used[i]) {
      used[i] = 1;
      ++cnt;
      const int64_t d = (int64_t)a[i].rpos - a[i].qpos;
      if (d < dmin) dmin = d;
      if (d > dmax) dmax = d;
      i = prev[i];
    }
    const int score = f[end] - (i >= 0 ? f[i] : 0);
    if (score < p->min_score || cnt < p->min_anchors) continue;
    tmp[m++] = (or_chain_t){score, a[end].strand, cnt, dmin, dmax, a[end].rpos};
  }
  /* stable order by score descending: sort (score desc, production index asc) */
  or_kv* so = (or_kv*)malloc(sizeof(or_kv) * (size_t)(m + 1));
  for (int64_t i = 0; i < m; ++i) so[i] = (or_kv){tmp[i].score, (int32_t)i, (int32_t)i};
  qsort(so, (size_t)m, sizeof(or_kv), cmp_kv);
  for (int64_t i = 0; i < m; ++i) out[i] = tmp[so[i].idx];
  free(so);
  free(tmp);
  free(used);
  free(ord);
  free(f);
  free(prev);
  return m;
}

int64_t or_chain(uint32_t* rpos, int32_t* qpos, uint32_t* strand, int64_t n, int k, const or_chain_params* p,
                 int32_t* o_score, uint32_t* o_strand, int32_t* o_n, int64_t* o_dmin, int64_t* o_dmax,
                 uint32_t* o_rpos, int64_t cap) {
  or_anchor* a = (or_anchor*)malloc(sizeof(or_anchor) * (size_t)(n + 1));
  for (int64_t i = 0; i < n; ++i) a[i] = (or_anchor){rpos[i], qpos[i], strand[i]};
  or_chain_t* ch = (or_chain_t*)malloc(sizeof(or_chain_t) * (size_t)(n + 1));
  const int64_t m = chain_core(a, n, k, p, ch);
  for (int64_t i = 0; i < n; ++i) {
    rpos[i] = a[i].rpos;
    qpos[i] = a[i].qpos;
    strand[i] = a[i].strand;
  }
  if (m <= cap) {
    for (int64_t i = 0; i < m; ++i) {
      o_score[i] = ch[i].score;
      o_strand[i] = ch[i].strand;
      o_n[i] = ch[i].n;
      o_dmin[i] = ch[i].dmin;
      o_dmax[i] = ch[i].dmax;
      o_rpos[i] = ch[i].rpos;
    }
  }
  free(a);
  free(ch);
  return m <= cap ? m : -m;
}

/* ------------------------------------------------------------------------ banded SW */

static int sub_score(const or_score_params* sp, uint8_t a, uint8_t b) {
  return (a > 3 || b > 3) ? -sp->ambig : (a == b ? sp->match : -sp->mismatch); /* src/align.hpp:39 */
}

enum { OR_DIR_DIAG = 0x80, OR_DIR_E = 0x40, OR_DIR_EXT_E = 0x20, OR_DIR_EXT_F = 0x10 };

static void cig_push(uint32_t* c, int32_t* n, uint32_t op, int len) {
  if (*n > 0 && (c[*n - 1] & 0xf) == op) c[*n - 1] += (uint32_t)len << 4;
  else c[(*n)++] = (uint32_t)len << 4 | op;
}

/* Banded local affine-gap SW in diagonal coordinates (src/align.cpp:31-84): row i, band
 * column d in [0, W), W = 2bw+1, target column i+d; the target is N-padded to qlen+W-1;
 * H and E of row -1 and of the fixed out-of-band cell d = W are 0; every row starts with
 * F = 0 and H(left) = 0. With traceback, a direction byte per cell (src/align.cpp:67-68)
 * and the first strict maximum in row-major order; then the walk of src/align.cpp:87-143. */
int32_t or_align(const uint8_t* q, int32_t qlen, const uint8_t* t, int32_t tlen, int traceback,
                 const or_score_params* sp, int32_t* res, uint32_t* cigar, int32_t cig_cap) {
  const int W = 2 * sp->bw + 1, tmax = qlen + W - 1;
  const int oe = sp->gap_open + sp->gap_ext, ge = sp->gap_ext;
  uint8_t* tt = (uint8_t*)malloc((size_t)(tmax > 0 ? tmax : 1));
  const int tl = tlen < tmax ? tlen : tmax;
  for (int j = 0; j < tmax; ++j) tt[j] = j < tl ? t[j] : 4;
  int32_t* H = (int32_t*)calloc((size_t)W + 1, sizeof(int32_t));
  int32_t* E = (int32_t*)calloc((size_t)W + 1, sizeof(int32_t));
  uint8_t* D = traceback ? (uint8_t*)malloc((size_t)qlen * W + 1) : NULL;
  int best = 0, bi = -1, bd = -1;
  for (int i = 0; i < qlen; ++i) {
    int f = 0, hleft = 0, hdiag = H[0];
    for (int d = 0; d < W; ++d) {
      const int hup = H[d + 1], eup = E[d + 1];
      const int hd = hdiag + sub_score(sp, q[i], tt[i + d]);
      const int eo = hup - oe, ee = eup - ge;
      const int e = eo > ee ? eo : ee;
      const int fo = hleft - oe, fe = f - ge;
      f = fo > fe ? fo : fe;
      int h = hd > e ? hd : e;
      h = h > 0 ? h : 0;
      h = h > f ? h : f;
      H[d] = h;
      E[d] = e;
      if (traceback) {
        D[(size_t)i * W + d] = (uint8_t)((h == hd ? OR_DIR_DIAG : 0) | (h == e ? OR_DIR_E : 0) |
                                         (ee > eo ? OR_DIR_EXT_E : 0) | (fe > fo ? 0x1F : 0));
        if (h > best) {
          best = h;
          bi = i;
          bd = d;
        }
      } else if (h > best) {
        best = h;
      }
      hleft = h;
      hdiag = hup;
    }
  }
  for (int x = 0; x < 6; ++x) res[x] = 0;
  res[0] = best;
  int32_t nops = 0;
  if (traceback && best > 0) {
    uint32_t* c = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(2 * qlen + 2));
    int i = bi, d = bd, v = best, nm = 0;
    for (;;) {
      int run = 0;
      uint8_t x = 0;
      while (i >= 0 && v > 0 && ((x = D[(size_t)i * W + d]) & OR_DIR_DIAG)) {
        const uint8_t a = q[i], b = tt[i + d];
        v -= sub_score(sp, a, b);
        nm += a != b || a > 3;
        ++run;
        --i;
      }
      if (run) cig_push(c, &nops, 0 /* M */, run);
      if (i < 0 || v <= 0) break;
      run = 0;
      if (x & OR_DIR_E) {
        int ext;
        do {
          ext = (D[(size_t)i * W + d] & OR_DIR_EXT_E) != 0;
          v += ext ? ge : oe;
          ++run;
          --i;
          ++d;
        } while (ext);
        cig_push(c, &nops, 1 /* I */, run);
      } else {
        int ext;
        do {
          ext = (D[(size_t)i * W + d] & OR_DIR_EXT_F) != 0;
          v += ext ? ge : oe;
          ++run;
          --d;
        } while (ext);
        cig_push(c, &nops, 2 /* D */, run);
      }
      nm += run;
    }
    res[1] = i + 1;
    res[2] = bi + 1;
    res[3] = i + 1 + d;
    res[4] = bi + bd + 1;
    res[5] = nm;
    if (nops > cig_cap) {
      nops = -1;
    } else {
      for (int32_t x = 0; x < nops; ++x) cigar[x] = c[nops - 1 - x];
    }
    free(c);
  }
  free(tt);
  free(H);
  free(E);
  free(D);
  return nops;
}

/* ---------------------------------------------------------------------------- mapper */

static int contig_of(const uint64_t* off, int32_t n, uint64_t gpos) { /* src/reference.cpp:25-32 */
  int64_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) / 2;
    if (off[mid] <= gpos) lo = mid;
    else hi = mid;
  }
  return (int)lo;
}

typedef struct {
  uint32_t rev;
  int32_t contig;
  int64_t diag, wstart;
  int32_t sw;
} or_cand;

/* One batch through the mapping pipeline (src/mapper.cpp:14-63 seed_and_chain and
 * src/mapper.cpp:75-223 map). Reads are independent, so this processes them one by one. */
int64_t or_map(const or_index* ix, const uint8_t* genome, const uint64_t* contig_off, const uint32_t* contig_len,
               int32_t n_contigs, const char* seq, const int64_t* seq_off, const int32_t* seq_len,
               const char* names, const int64_t* name_off, int64_t n, const or_map_params* p, int64_t* rec,
               uint32_t* cigar, int64_t* cig_off, int64_t cig_cap) {
  const int k = p->k, bw = p->sc.bw, W = 2 * bw + 1;
  or_chain_params chp = p->ch;
  if (chp.band > bw) chp.band = bw; /* src/mapper.cpp:9 */
  int64_t o = 0;
  int overflow = 0;
  int32_t maxlen = 0;
  for (int64_t r = 0; r < n; ++r)
    if (seq_len[r] > maxlen) maxlen = seq_len[r];
  uint8_t* codes = (uint8_t*)malloc((size_t)2 * maxlen + 1);
  uint64_t* mh = (uint64_t*)malloc(sizeof(uint64_t) * ((size_t)maxlen + 1));
  uint32_t* mp = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)maxlen + 1));
  uint32_t* ms = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)maxlen + 1));
  uint8_t* tw = (uint8_t*)malloc((size_t)maxlen + 2 * bw + 1);
  uint32_t* cg = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)2 * maxlen + 4));
  or_cand* cands = (or_cand*)malloc(sizeof(or_cand) * ((size_t)p->max_cand + 1));
  int64_t acap = 1024;
  or_anchor* an = (or_anchor*)malloc(sizeof(or_anchor) * (size_t)acap);
  or_chain_t* ch = (or_chain_t*)malloc(sizeof(or_chain_t) * (size_t)acap);

  for (int64_t r = 0; r < n; ++r) {
    const int len = seq_len[r];
    uint8_t* fwd = codes;
    uint8_t* rc = codes + len;
    or_encode(seq + seq_off[r], len, fwd);
    or_revcomp(fwd, len, rc);
    /* seed: minimizers -> lookups -> anchors (src/mapper.cpp:16-40) */
    const int64_t nm = or_sketch(fwd, (uint32_t)len, k, p->w, 0, mh, mp, ms, maxlen + 1);
    int64_t na = 0;
    for (int64_t i = 0; i < nm; ++i) {
      uint32_t off = 0;
      const uint32_t cnt = or_index_lookup(ix, mh[i], &off);
      if (cnt == 0 || cnt > (uint32_t)p->max_occ) continue;
      if (na + cnt > acap) {
        while (na + cnt > acap) acap *= 2;
        an = (or_anchor*)realloc(an, sizeof(or_anchor) * (size_t)acap);
        ch = (or_chain_t*)realloc(ch, sizeof(or_chain_t) * (size_t)acap);
      }
      for (uint32_t j = 0; j < cnt; ++j) {
        const uint32_t v = ix->pos[off + j];
        const uint32_t rev = (v & 1) ^ ms[i];
        const int32_t qpos = rev ? len - (int32_t)mp[i] - k : (int32_t)mp[i];
        an[na++] = (or_anchor){v >> 1, qpos, rev};
      }
    }
    const int64_t nc = chain_core(an, na, k, &chp, ch);
    /* candidates (src/mapper.cpp:40-62) */
    int nd = 0;
    if (nc > 0) {
      const double min_score = ch[0].score * p->pri_ratio;
      for (int64_t c = 0; c < nc; ++c) {
        if (ch[c].score < min_score || nd >= p->max_cand) break;
        const int64_t diag = ch[c].dmin + (ch[c].dmax - ch[c].dmin) / 2;
        int dup = 0;
        for (int i = 0; i < nd && !dup; ++i) {
          const int64_t dd = cands[i].diag - diag;
          dup = cands[i].rev == ch[c].strand && (dd < 0 ? -dd : dd) <= bw;
        }
        if (dup) continue;
        cands[nd].rev = ch[c].strand;
        cands[nd].contig = contig_of(contig_off, n_contigs, ch[c].rpos);
        cands[nd].diag = diag;
        cands[nd].wstart = diag - bw;
        cands[nd].sw = 0;
        ++nd;
      }
    }
    int64_t* x = rec + 7 * r;
    x[0] = -1;
    x[1] = x[2] = x[3] = x[4] = x[5] = 0;
    x[6] = nd;
    cig_off[r] = o;
    if (nd == 0) continue;
    /* target windows with N outside the candidate's contig (src/mapper.cpp:100-121) */
    const int wl = len + 2 * bw;
    int32_t resv[6];
    int chosen = 0, s2 = 0;
    if (nd >= 2) { /* rank by score-only SW (src/mapper.cpp:125-140), choose (:142-174) */
      for (int c = 0; c < nd; ++c) {
        const int64_t b = (int64_t)contig_off[cands[c].contig], e = b + contig_len[cands[c].contig];
        for (int j = 0; j < wl; ++j) {
          const int64_t gp = cands[c].wstart + j;
          tw[j] = (gp >= b && gp < e) ? genome[gp] : 4;
        }
        or_align(cands[c].rev ? rc : fwd, len, tw, wl, 0, &p->sc, resv, NULL, 0);
        cands[c].sw = resv[0];
      }
      int s1 = -1, ties = 0;
      for (int c = 0; c < nd; ++c) {
        if (cands[c].sw > s1) {
          s1 = cands[c].sw;
          ties = 1;
        } else if (cands[c].sw == s1) {
          ++ties;
        }
      }
      if (ties > 1) s2 = s1;
      else
        for (int c = 0; c < nd; ++c)
          if (cands[c].sw != s1 && cands[c].sw > s2) s2 = cands[c].sw;
      uint32_t pick = or_fnv1a(names + name_off[r], name_off[r + 1] - name_off[r]) % (uint32_t)ties;
      for (int c = 0; c < nd; ++c)
        if (cands[c].sw == s1 && pick-- == 0) {
          chosen = c;
          break;
        }
    }
    const or_cand* cd = &cands[chosen];
    {
      const int64_t b = (int64_t)contig_off[cd->contig], e = b + contig_len[cd->contig];
      for (int j = 0; j < wl; ++j) {
        const int64_t gp = cd->wstart + j;
        tw[j] = (gp >= b && gp < e) ? genome[gp] : 4;
      }
    }
    const int32_t nops = or_align(cd->rev ? rc : fwd, len, tw, wl, 1, &p->sc, resv, cg, 2 * maxlen + 4);
    /* record + MAPQ (src/mapper.cpp:189-222) */
    if (resv[0] < p->min_aln_score) continue;
    x[0] = cd->contig;
    x[1] = cd->wstart + resv[3] - (int64_t)contig_off[cd->contig];
    x[2] = cd->rev;
    x[4] = resv[0];
    x[5] = resv[5];
    if (nd <= 1) {
      x[3] = 60;
    } else {
      const double qv = s2 >= resv[0] ? 0.0 : 6.02 * (resv[0] - s2) / p->sc.match + 0.499;
      x[3] = (int64_t)(uint8_t)(qv < 60.0 ? qv : 60.0);
    }
    const int64_t need = (resv[1] > 0) + nops + (len > resv[2]);
    if (o + need > cig_cap) {
      overflow = 1;
      o += need;
      continue;
    }
    if (resv[1] > 0) cigar[o++] = (uint32_t)resv[1] << 4 | 4 /* S */;
    for (int32_t i = 0; i < nops; ++i) cigar[o++] = cg[i];
    if (len > resv[2]) cigar[o++] = (uint32_t)(len - resv[2]) << 4 | 4;
  }
  cig_off[n] = o;
  (void)W;
  free(codes);
  free(mh);
  free(mp);
  free(ms);
  free(tw);
  free(cg);
  free(cands);
  free(an);
  free(ch);
  return overflow ? -o : o;
}
