// ref_shim.cpp — TEST INFRASTRUCTURE ONLY. A C-ABI over the reference implementation's
// own C++ classes, so that Python tests and the CPU baseline can call the unmodified
// reference code path. oracle/Makefile compiles this file together with the reference's
// sources (src/*.cpp of dnaln) into oracle/_ref/libdnaln_ref.so; nothing in the product
// links it.
//
// Every entry point forwards to the reference function named beside it:
//   ref_sketch        -> dnaln::sketch                      (src/minimizer.hpp:34)
//   ref_index_*       -> dnaln::MinimizerIndex              (src/index.hpp:19-60)
//   ref_chain         -> dnaln::Chainer::run                (src/chain.hpp:41)
//   ref_align         -> dnaln::ScalarAligner / SimdAligner (src/align.hpp:70-104)
//   ref_map           -> dnaln::Mapper::map + append_sam    (src/mapper.hpp:51-58)
//   ref_read_records  -> dnaln::read_all_records            (src/seqio.hpp:47)
//   ref_eval          -> dnaln::Evaluator::add              (src/evaluate.hpp:29-31)
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "align.hpp"
#include "chain.hpp"
#include "common.hpp"
#include "evaluate.hpp"
#include "index.hpp"
#include "mapper.hpp"
#include "minimizer.hpp"
#include "reference.hpp"
#include "seqio.hpp"

using namespace dnaln;

namespace {

struct RefGenome {
  Reference ref;
  MinimizerIndex idx;
};

ScoreParams score_params(const int32_t* sp) {
  ScoreParams s;
  s.match = sp[0];
  s.mismatch = sp[1];
  s.gap_open = sp[2];
  s.gap_ext = sp[3];
  s.ambig = sp[4];
  s.bw = sp[5];
  return s;
}

}  // namespace

extern "C" {

int ref_version(void) { return 1; }

// Minimizers of one sequence. Returns the count, or -(count) if `cap` was too small.
int64_t ref_sketch(const uint8_t* seq, uint32_t len, int k, int w, uint32_t offset, uint64_t* hash,
                   uint32_t* pos, uint32_t* strand, int64_t cap) {
  std::vector<Minimizer> out;
  sketch(seq, len, k, w, offset, out);
  const int64_t n = static_cast<int64_t>(out.size());
  if (n > cap) return -n;
  for (int64_t i = 0; i < n; ++i) {
    hash[i] = out[i].hash;
    pos[i] = out[i].pos;
    strand[i] = out[i].strand;
  }
  return n;
}

// Genome = concatenated base codes plus a contig table; builds the reference index.
// Contig names are concatenated in `cnames` with offsets cname_off[0..n_contigs]; when
// cnames is null the contigs are named chr1, chr2, ...
void* ref_genome_new(const uint8_t* codes, uint64_t n_bases, const uint64_t* contig_off,
                     const uint32_t* contig_len, int32_t n_contigs, const char* cnames, const int64_t* cname_off,
                     int k, int w) {
  auto* g = new RefGenome;
  g->ref.seq.assign(codes, codes + n_bases);
  for (int32_t c = 0; c < n_contigs; ++c) {
    Contig ct;
    ct.name = cnames ? std::string(cnames + cname_off[c], static_cast<size_t>(cname_off[c + 1] - cname_off[c]))
                     : "chr" + std::to_string(c + 1);
    ct.offset = contig_off[c];
    ct.len = contig_len[c];
    g->ref.contigs.push_back(ct);
  }
  g->idx.build(g->ref, k, w);
  return g;
}

void ref_genome_free(void* g) { delete static_cast<RefGenome*>(g); }

// n_keys, n_positions, max_count, memory_bytes
void ref_index_stats(void* gp, uint64_t* out4) {
  const auto* g = static_cast<RefGenome*>(gp);
  out4[0] = g->idx.n_keys();
  out4[1] = g->idx.n_positions();
  out4[2] = g->idx.max_count();
  out4[3] = g->idx.memory_bytes();
}

// Occurrence list of hash h; returns the count (copies at most cap entries).
uint32_t ref_index_lookup(void* gp, uint64_t h, uint32_t* out, uint32_t cap) {
  const auto* g = static_cast<RefGenome*>(gp);
  uint32_t n = 0;
  const uint32_t* p = g->idx.lookup(h, n);
  for (uint32_t i = 0; i < n && i < cap; ++i) out[i] = p[i];
  return n;
}

// Chains of one anchor set. Anchors are sorted in place (as the reference does).
// chain_p = {max_gap, band, lookback, min_score, min_anchors}. Output columns per chain:
// score, strand, n_anchors, rpos (i32/u32) and dmin, dmax (i64). Returns #chains or -n.
int64_t ref_chain(uint32_t* rpos, int32_t* qpos, uint32_t* strand, int64_t n, int k, const int32_t* chain_p,
                  int32_t* o_score, uint32_t* o_strand, int32_t* o_n, int64_t* o_dmin, int64_t* o_dmax,
                  uint32_t* o_rpos, int64_t cap) {
  std::vector<Anchor> a(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) a[i] = {rpos[i], qpos[i], strand[i]};
  ChainParams p;
  p.max_gap = chain_p[0];
  p.band = chain_p[1];
  p.lookback = chain_p[2];
  p.min_score = chain_p[3];
  p.min_anchors = chain_p[4];
  Chainer ch;
  std::vector<Chain> out;
  ch.run(a, k, p, out);
  for (int64_t i = 0; i < n; ++i) {
    rpos[i] = a[i].rpos;
    qpos[i] = a[i].qpos;
    strand[i] = a[i].strand;
  }
  const int64_t m = static_cast<int64_t>(out.size());
  if (m > cap) return -m;
  for (int64_t i = 0; i < m; ++i) {
    o_score[i] = out[i].score;
    o_strand[i] = out[i].strand;
    o_n[i] = out[i].n_anchors;
    o_dmin[i] = out[i].dmin;
    o_dmax[i] = out[i].dmax;
    o_rpos[i] = out[i].rpos;
  }
  return m;
}

// Banded SW over n tasks. score_p = {match, mismatch, gap_open, gap_ext, ambig, bw}.
// res columns (n x 6): score, qb, qe, tb, te, nm. CIGAR ops of task i go to
// cigar[cig_off[i] .. cig_off[i+1]); returns total ops, or -(needed) if cig_cap is short.
int64_t ref_align(const uint8_t* qbuf, const int64_t* qoff, const int32_t* qlen, const uint8_t* tbuf,
                  const int64_t* toff, const int32_t* tlen, int64_t n, int traceback, const int32_t* score_p,
                  int simd, int32_t* res, uint32_t* cigar, int64_t* cig_off, int64_t cig_cap) {
  const ScoreParams sp = score_params(score_p);
  std::vector<AlignTask> tasks(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) tasks[i] = {qbuf + qoff[i], qlen[i], tbuf + toff[i], tlen[i]};
  std::vector<AlignResult> out(static_cast<size_t>(n));
  std::unique_ptr<Aligner> al;
  if (simd) al = std::make_unique<SimdAligner>(sp);
  else al = std::make_unique<ScalarAligner>(sp);
  al->align(tasks.data(), static_cast<size_t>(n), traceback != 0, out.data());
  int64_t total = 0;
  for (int64_t i = 0; i < n; ++i) total += static_cast<int64_t>(out[i].cigar.size());
  if (total > cig_cap) return -total;
  int64_t o = 0;
  for (int64_t i = 0; i < n; ++i) {
    const AlignResult& r = out[i];
    int32_t* x = res + 6 * i;
    x[0] = r.score;
    x[1] = r.qb;
    x[2] = r.qe;
    x[3] = r.tb;
    x[4] = r.te;
    x[5] = r.nm;
    cig_off[i] = o;
    for (uint32_t c : r.cigar) cigar[o++] = c;
  }
  cig_off[n] = o;
  return total;
}

// Maps n reads (ASCII, concatenated; qualities at the same offsets or null for none;
// names concatenated with name_off) with the reference Mapper, `nthreads` independent
// Mapper instances over contiguous read shards, `batch` reads per Mapper::map call (the
// CLI uses 8192).
// map_p = {k, w, max_occ, max_cand, min_aln_score, simd, match, mismatch, gap_open,
//          gap_ext, ambig, bw, ch_max_gap, ch_band, ch_lookback, ch_min_score, ch_min_anchors}
// pri_ratio passed separately. rec columns (n x 7): contig, pos, rev, mapq, score, nm, n_cand.
// If sam != null, the SAM body (append_sam) is written there (cap sam_cap bytes) and its
// length returned through *sam_len. Returns total CIGAR ops, or -(needed).
int64_t ref_map(void* gp, const char* seq, const int64_t* seq_off, const int32_t* seq_len, const char* qual,
                const char* names, const int64_t* name_off, int64_t n, const int32_t* map_p, double pri_ratio,
                int nthreads, int64_t batch, int64_t* rec, uint32_t* cigar, int64_t* cig_off, int64_t cig_cap,
                char* sam, int64_t sam_cap, int64_t* sam_len) {
  const auto* g = static_cast<RefGenome*>(gp);
  MapParams mp;
  mp.k = map_p[0];
  mp.w = map_p[1];
  mp.max_occ = static_cast<uint32_t>(map_p[2]);
  mp.max_cand = map_p[3];
  mp.min_aln_score = map_p[4];
  mp.simd = map_p[5] != 0;
  mp.sc.match = map_p[6];
  mp.sc.mismatch = map_p[7];
  mp.sc.gap_open = map_p[8];
  mp.sc.gap_ext = map_p[9];
  mp.sc.ambig = map_p[10];
  mp.sc.bw = map_p[11];
  mp.ch.max_gap = map_p[12];
  mp.ch.band = map_p[13];
  mp.ch.lookback = map_p[14];
  mp.ch.min_score = map_p[15];
  mp.ch.min_anchors = map_p[16];
  mp.pri_ratio = pri_ratio;

  std::vector<SeqRecord> reads(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    reads[i].name.assign(names + name_off[i], static_cast<size_t>(name_off[i + 1] - name_off[i]));
    reads[i].seq.assign(seq + seq_off[i], static_cast<size_t>(seq_len[i]));
    if (qual) reads[i].qual.assign(qual + seq_off[i], static_cast<size_t>(seq_len[i]));  // else FASTA-like: '*'
  }
  std::vector<MapRecord> recs(static_cast<size_t>(n));
  const int T = std::max(1, nthreads);
  if (batch <= 0) batch = 8192;
  auto work = [&](int64_t b, int64_t e) {
    Mapper m(g->ref, g->idx, mp);
    std::vector<MapRecord> part;
    for (int64_t s = b; s < e; s += batch) {
      const int64_t c = std::min<int64_t>(batch, e - s);
      m.map(reads.data() + s, static_cast<size_t>(c), part);
      for (int64_t i = 0; i < c; ++i) recs[static_cast<size_t>(s + i)] = std::move(part[static_cast<size_t>(i)]);
    }
  };
  if (T == 1) {
    work(0, n);
  } else {
    std::vector<std::thread> th;
    const int64_t per = (n + T - 1) / T;
    for (int t = 0; t < T; ++t) {
      const int64_t b = std::min<int64_t>(n, t * per), e = std::min<int64_t>(n, b + per);
      if (b < e) th.emplace_back(work, b, e);
    }
    for (auto& x : th) x.join();
  }
  int64_t total = 0;
  for (const MapRecord& r : recs) total += static_cast<int64_t>(r.cigar.size());
  if (cigar && total > cig_cap) return -total;
  int64_t o = 0;
  for (int64_t i = 0; i < n; ++i) {
    const MapRecord& r = recs[static_cast<size_t>(i)];
    int64_t* x = rec + 7 * i;
    x[0] = r.contig;
    x[1] = r.pos;
    x[2] = r.rev;
    x[3] = r.mapq;
    x[4] = r.score;
    x[5] = r.nm;
    x[6] = r.n_cand;
    if (cigar) {
      cig_off[i] = o;
      for (uint32_t c : r.cigar) cigar[o++] = c;
    }
  }
  if (cigar) cig_off[n] = o;
  if (sam) {
    Mapper m(g->ref, g->idx, mp);
    std::string body;
    for (int64_t i = 0; i < n; ++i) m.append_sam(reads[static_cast<size_t>(i)], recs[static_cast<size_t>(i)], body);
    *sam_len = static_cast<int64_t>(body.size());
    if (static_cast<int64_t>(body.size()) <= sam_cap) std::memcpy(sam, body.data(), body.size());
  }
  return total;
}

// read_all_records of a FASTA/FASTQ file (src/seqio.cpp:89-96). sizes4 = {records, sequence
// bytes, name bytes, quality bytes}; with non-null buffers the records are also written
// out, concatenated, with n + 1 offsets each. Well-formed input only: the reference exits
// on malformed records.
int ref_read_records(const char* path, int64_t* sizes4, char* seq, int64_t* seq_off, char* names, int64_t* name_off,
                     char* qual, int64_t* qual_off) {
  const std::vector<SeqRecord> v = read_all_records(path);
  int64_t sb = 0, nb = 0, qb = 0;
  for (size_t i = 0; i < v.size(); ++i) {
    if (seq) {
      seq_off[i] = sb;
      name_off[i] = nb;
      qual_off[i] = qb;
      std::memcpy(seq + sb, v[i].seq.data(), v[i].seq.size());
      std::memcpy(names + nb, v[i].name.data(), v[i].name.size());
      std::memcpy(qual + qb, v[i].qual.data(), v[i].qual.size());
    }
    sb += static_cast<int64_t>(v[i].seq.size());
    nb += static_cast<int64_t>(v[i].name.size());
    qb += static_cast<int64_t>(v[i].qual.size());
  }
  if (seq) {
    seq_off[v.size()] = sb;
    name_off[v.size()] = nb;
    qual_off[v.size()] = qb;
  }
  sizes4[0] = static_cast<int64_t>(v.size());
  sizes4[1] = sb;
  sizes4[2] = nb;
  sizes4[3] = qb;
  return 0;
}

// Evaluator::add over n records (read i named "r<i>", contig names "c<index>"): rec
// columns as ref_map writes them (contig, pos, rev, mapq, ...), CIGAR of record i at
// cigar[cig_off[i], cig_off[i+1]). out = {records, mapped, correct, mapped_at(q) for q =
// 0..60, wrong_at(q) for q = 0..60} (cumulative over MAPQ >= q, as the reference reports).
void ref_eval(const int64_t* rec, const uint32_t* cigar, const int64_t* cig_off, const int32_t* t_contig,
              const int64_t* t_start, const uint8_t* t_rev, int64_t n, int tol, uint64_t* out) {
  TruthMap truth;
  for (int64_t i = 0; i < n; ++i) {
    TruthRec t;
    t.contig = "c" + std::to_string(t_contig[i]);
    t.start = t_start[i];
    t.end = t_start[i];
    t.rev = t_rev[i] != 0;
    truth.emplace("r" + std::to_string(i), std::move(t));
  }
  Evaluator ev(truth, tol);
  std::vector<uint32_t> cg;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t* x = rec + 7 * i;
    cg.assign(cigar + cig_off[i], cigar + cig_off[i + 1]);
    ev.add("r" + std::to_string(i), x[0] >= 0, x[0] >= 0 ? "c" + std::to_string(x[0]) : "*", x[1], x[2] != 0,
           static_cast<int>(x[3]), cg);
  }
  out[0] = ev.records();
  out[1] = ev.mapped();
  out[2] = ev.correct();
  for (int q = 0; q <= 60; ++q) {
    out[3 + q] = ev.mapped_at(q);
    out[64 + q] = ev.wrong_at(q);
  }
}

// fnv1a of the reference (src/common.hpp:136-140), for tie-break checks.
uint32_t ref_fnv1a(const char* s, int64_t n) { return fnv1a(std::string(s, static_cast<size_t>(n))); }

}  // extern "C"
