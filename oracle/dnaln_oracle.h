/* dnaln_oracle.h — TEST INFRASTRUCTURE ONLY: a plain-C restatement of dnaln's read-mapping
 * path, used by tests/ to check the CUDA path and by bench.py's cpu_baseline leg. The
 * product never links it. Parity of this restatement with the reference is pinned by
 * tests/test_oracle.py against the reference compiled from its own sources (oracle/_ref)
 * and against the committed fixtures in tests/golden/.
 *
 * Citations are to files of the dnaln project (src/...). */
#ifndef DNALN_ORACLE_H
#define DNALN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t match, mismatch, gap_open, gap_ext, ambig, bw; /* src/align.hpp:34-40 */
} or_score_params;

typedef struct {
  int32_t max_gap, band, lookback, min_score, min_anchors; /* src/chain.hpp:30-36 */
} or_chain_params;

typedef struct {
  int32_t k, w, max_occ, max_cand, min_aln_score; /* src/mapper.hpp:25-35 */
  double pri_ratio;
  or_score_params sc;
  or_chain_params ch;
} or_map_params;

typedef struct or_index or_index;

uint64_t or_hash64(uint64_t key, uint64_t mask);
void or_encode(const char* s, int64_t n, uint8_t* out);
void or_revcomp(const uint8_t* in, int64_t n, uint8_t* out);
uint32_t or_fnv1a(const char* s, int64_t n);

int64_t or_sketch(const uint8_t* seq, uint32_t len, int k, int w, uint32_t offset, uint64_t* hash, uint32_t* pos,
                  uint32_t* strand, int64_t cap);

or_index* or_index_build(const uint8_t* codes, uint64_t n_bases, const uint64_t* contig_off,
                         const uint32_t* contig_len, int32_t n_contigs, int k, int w);
void or_index_free(or_index* ix);
/* n_keys, n_positions, max_count, memory_bytes, n_buckets */
void or_index_stats(const or_index* ix, uint64_t* out5);
/* Copies the table (keys, offsets, counts; n_buckets each) and the position array. */
void or_index_export(const or_index* ix, uint64_t* keys, uint32_t* offs, uint32_t* cnts, uint32_t* positions);
/* Returns the occurrence count of h; *off receives the start in the position array. */
uint32_t or_index_lookup(const or_index* ix, uint64_t h, uint32_t* off);

int64_t or_chain_cost_mismatches(int k_lo, int k_hi, int dd_max);

int64_t or_chain(uint32_t* rpos, int32_t* qpos, uint32_t* strand, int64_t n, int k, const or_chain_params* p,
                 int32_t* o_score, uint32_t* o_strand, int32_t* o_n, int64_t* o_dmin, int64_t* o_dmax,
                 uint32_t* o_rpos, int64_t cap);

/* One banded SW task. res = {score, qb, qe, tb, te, nm}; returns #CIGAR ops written to
 * cigar (capacity 2*qlen+1 always suffices), or -1 if cig_cap is too small. */
int32_t or_align(const uint8_t* q, int32_t qlen, const uint8_t* t, int32_t tlen, int traceback,
                 const or_score_params* sp, int32_t* res, uint32_t* cigar, int32_t cig_cap);

/* Maps n ASCII reads. rec columns (n x 7): contig, pos, rev, mapq, score, nm, n_cand.
 * CIGAR ops (with soft clips) of read i go to cigar[cig_off[i] .. cig_off[i+1]).
 * Returns the total number of ops, or -(needed) when cig_cap is too small. */
int64_t or_map(const or_index* ix, const uint8_t* genome, const uint64_t* contig_off, const uint32_t* contig_len,
               int32_t n_contigs, const char* seq, const int64_t* seq_off, const int32_t* seq_len,
               const char* names, const int64_t* name_off, int64_t n, const or_map_params* p, int64_t* rec,
               uint32_t* cigar, int64_t* cig_off, int64_t cig_cap);

#ifdef __cplusplus
}
#endif
#endif
