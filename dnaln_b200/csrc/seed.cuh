// seed.cuh — launch interface of the seeding and chaining kernels (seed.cu).
#pragma once

#include "common.cuh"

namespace dnb {

// Resident minimizer index: the reference's table of 16-byte buckets {key, offset,
// count} with linear probing from key & mask (src/index.hpp:3-9,49-56), the position
// array (pos << 1 | strand), the genome (1 code per byte) and its contig table.
struct DevIndex {
  const ulonglong2* table;  // .x = key, .y = offset | (uint64)count << 32
  const uint32_t* positions;
  const uint8_t* genome;
  const uint64_t* contig_off;
  const uint32_t* contig_len;
  const uint2* n_runs;  // maximal runs of non-ACGT codes, [x, y), sorted
  uint64_t mask;
  int32_t n_contigs, k, w, n_n_runs;
};

// True when genome[a, b) holds a non-ACGT code (binary search over the N runs).
__device__ __forceinline__ bool genome_has_n(const DevIndex& ix, int64_t a, int64_t b) {
  int lo = 0, hi = ix.n_n_runs;  // first run with end > a
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (static_cast<int64_t>(ix.n_runs[mid].y) <= a) lo = mid + 1;
    else hi = mid;
  }
  return lo < ix.n_n_runs && static_cast<int64_t>(ix.n_runs[lo].x) < b;
}

// hash64 for 2k <= 32: every step is either reduced mod 2^32 and then masked to 2k bits,
// or a right shift of a value below 2^2k, so 32-bit arithmetic gives the same bits.
__device__ __forceinline__ uint32_t hash32(uint32_t key, uint32_t mask) {
  key = (~key + (key << 21)) & mask;
  key = key ^ key >> 24;
  key = ((key + (key << 3)) + (key << 8)) & mask;
  key = key ^ key >> 14;
  key = ((key + (key << 2)) + (key << 4)) & mask;
  key = key ^ key >> 28;
  key = (key + (key << 31)) & mask;
  return key;
}

// Probes the table for key h (src/index.hpp:24-38): off/cnt of its position list, cnt = 0
// when absent. The table is at most half full, so an empty bucket always ends the walk;
// the loop bound only guards a corrupted table.
__device__ __forceinline__ void probe(const DevIndex& ix, uint64_t h, uint32_t& off, uint32_t& cnt,
                                      uint32_t* err) {
  uint64_t i = h & ix.mask;
  off = 0;
  cnt = 0;
  for (uint64_t it = 0; it <= ix.mask; ++it) {  // load <= 0.5: an empty bucket always ends the walk
    const ulonglong2 b = __ldg(ix.table + i);
    if (b.x == h) {
      off = static_cast<uint32_t>(b.y);
      cnt = static_cast<uint32_t>(b.y >> 32);
      return;
    }
    if (b.x == kInvalidHash) return;
    i = (i + 1) & ix.mask;
  }
  atomicOr(err, kErrProbeLoop);
}

// Contig holding genome position gpos (src/reference.cpp:25-32).
__device__ __forceinline__ int contig_of(const DevIndex& ix, uint64_t gpos) {
  int64_t lo = 0, hi = ix.n_contigs;
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) / 2;
    if (ix.contig_off[mid] <= gpos) lo = mid;
    else hi = mid;
  }
  return static_cast<int>(lo);
}

struct SeedParams {
  int32_t k, w;
  uint32_t max_occ;
};

struct ChainParamsDev {
  int32_t max_gap, band, lookback, min_score, min_anchors, k;
  const int32_t* cost;  // cost[dd] for dd in [0, band]: int(0.01*k*dd + 0.5*ilog2(dd)), host-computed
};

struct CandParams {
  int32_t max_cand, bw;
  double pri_ratio;
};

// Minimizers of one read: slot j of read r is at index seq_off[r] + j.
struct MinBuf {
  uint64_t* hash;
  uint32_t* pos;     // position | strand << 31
  uint32_t* hit_off; // offset into the position array (valid when hit_cnt > 0)
  uint32_t* hit_cnt; // occurrences kept (0 when absent or above max_occ)
};

struct AnchorScratch {  // per anchor of reads too large for the shared-memory path
  uint64_t* keys;
  int32_t* f;
  int32_t* prev;
  uint64_t* ord;
  uint8_t* used;
  int32_t* ch_score;
  uint32_t* ch_sn;   // strand | n_anchors << 1
  int64_t* ch_dmin;
  int64_t* ch_dmax;
  uint32_t* ch_rpos;
};

struct CandBuf {
  int32_t* n_cand;
  uint8_t* rev;
  int32_t* contig;
  int64_t* diag;
  int64_t* wstart;
};

// Pass 1 of a read batch: encode the ASCII read seq[seq_off[r] - seq_base, + seq_len[r])
// to codes (forward at 2*pofs[r], reverse complement right after it; pofs = exclusive
// prefix of the lengths), sketch, probe (minimizer slots at pofs[r]); writes n_min[r] and
// n_anchor[r]. seq_base lets a sub-batch staged on the device keep the caller's offsets.
void launch_seed(cudaStream_t st, const char* seq, const int64_t* seq_off, int64_t seq_base, const int32_t* seq_len,
                 const int64_t* pofs, int64_t n, uint8_t* codes, const DevIndex& ix, const SeedParams& sp, MinBuf mb,
                 int32_t* n_min, int64_t* n_anchor, uint32_t* err);

// Pass 1 for the reads list[0, *list_n) only (n_max >= *list_n), codes already written.
void launch_seed_list(cudaStream_t st, const char* seq, const int64_t* seq_off, int64_t seq_base,
                      const int32_t* seq_len, const int64_t* pofs, int64_t n_max, const int32_t* list,
                      const int* list_n, uint8_t* codes, const DevIndex& ix, const SeedParams& sp, MinBuf mb,
                      int32_t* n_min, int64_t* n_anchor, uint32_t* err);

// Pass 2: anchors, chaining, candidates of the reads [0, n), or with a list of the reads
// list[0, *list_n) (n = the list's size). n_anchor[r] = the read's anchor count (pass 1);
// reads of more than 32 anchors take their scratch (as, pool_cap entries per array) from
// the pool by an atomic add on *pool_top; past the capacity a read sets kErrChainPool.
// With `claim` (an int zeroed by the caller) the grid is the resident warps only and each
// warp takes its next read by an atomic add on *claim (work stealing); without, the warps
// stride over the reads.
void launch_chain_map(cudaStream_t st, const int64_t* pofs, const int32_t* seq_len, int64_t n, const int32_t* list,
                      const int* list_n, const int32_t* n_min, const int64_t* n_anchor, MinBuf mb,
                      const DevIndex& ix, const ChainParamsDev& cp, const CandParams& cand, AnchorScratch as,
                      unsigned long long* pool_top, int64_t pool_cap, CandBuf cb, int* claim, uint32_t* err);

// Codes of both strands of reads [0, n) (seed_thread.cu): forward at codes[2*pofs[r]],
// reverse complement right after it (src/mapper.cpp:88-99), from the ASCII reads.
void launch_encode_reads(cudaStream_t st, const char* seq, const int64_t* seq_off, int64_t seq_base,
                         const int32_t* seq_len, const int64_t* pofs, int64_t n, uint8_t* codes);
// The same codes through shared memory by bulk (TMA) copies, tiles of back-to-back reads
// (encode_bulk.cu); a tile that is not back to back is encoded read by read. err gets
// kErrAsyncCopy if a bulk load's bounded wait runs out.
void launch_encode_reads_bulk(cudaStream_t st, const char* seq, const int64_t* seq_off, int64_t seq_base,
                              const int32_t* seq_len, const int64_t* pofs, int64_t n, uint8_t* codes, uint32_t* err);

// One thread per read (seed_thread.cu): passes 1 and 2 of the reads the per-thread budgets
// admit, from their forward codes (codes + 2 * pofs[r], written by launch_encode_reads on
// the same stream before), writing
// candidates of the admitted reads, n_min, n_anc_t (their anchor counts, for statistics)
// and n_anchor = 0 (no scratch); the others are appended to big_list (count in *big_n,
// zeroed by the caller) for launch_seed_list / launch_chain_map. reads_per_block: 64 or
// 128 (threads per block; same results). Returns false, launching nothing, when the
// parameters are outside the path's range.
bool seed_thread_supported(const SeedParams& sp, const ChainParamsDev& cp);
int seed_thread_max_len();  // the longest read the short thread kernel stages
bool launch_seed_chain_thread(cudaStream_t st, const uint8_t* codes, const int64_t* pofs,
                              const int32_t* seq_len, int64_t n, const DevIndex& ix, const SeedParams& sp,
                              const ChainParamsDev& cp,
                              const CandParams& cand, CandBuf cb, int32_t* n_min, int64_t* n_anchor,
                              int32_t* n_anc_t, int32_t* big_list, int* big_n, uint32_t* err,
                              int reads_per_block = 128);

// Long reads, one thread each (seed_long.cu): the reads of list[0, *list_n) longer than
// min_len (typically those the short kernel listed) with their state in `scratch`
// (seed_long_scratch_words(threads) words); the others, and reads past its bounds, go to
// next_list (count *next_n) for the warp kernels.
// threads = seed_long_threads(upper bound of the list length).
bool seed_long_supported(const SeedParams& sp, const ChainParamsDev& cp);
int64_t seed_long_threads(int64_t n_max);
size_t seed_long_scratch_words(int64_t threads);
bool launch_seed_chain_long(cudaStream_t st, const int32_t* seq_len, const int64_t* pofs, const uint8_t* codes,
                            const int32_t* list, const int* list_n, int64_t threads, const DevIndex& ix,
                            const SeedParams& sp, const ChainParamsDev& cp, const CandParams& cand, CandBuf cb,
                            int32_t* n_min, int64_t* n_anchor, int32_t* n_anc_t, uint32_t* scratch,
                            int32_t* next_list, int* next_n, int min_len, uint32_t* err);
// Sort keys (longest first; slots at or past *list_n last) and values (read ids) of a list
// whose length is only known on the device; n_max = the list buffer's size, max_len at
// least the longest read. Returns the number of low key bits the sort must cover.
int launch_long_order(cudaStream_t st, const int32_t* list, const int* list_n, int n_max, const int32_t* seq_len,
                      int64_t max_len, uint32_t* keys, int32_t* vals);

// Stage entry points: sketch of code sequences, lookups, chaining of given anchor sets.
void launch_sketch_codes(cudaStream_t st, const uint8_t* codes, const int64_t* seq_off, const int32_t* seq_len,
                         const uint32_t* pos_offset, int64_t n, int32_t k, int32_t w, uint64_t* out_hash,
                         uint32_t* out_pos, uint32_t* out_strand, int32_t* out_count);
void launch_lookup(cudaStream_t st, const DevIndex& ix, const uint64_t* hashes, int64_t n, uint32_t* out_off,
                   uint32_t* out_cnt, uint32_t* err);
// Anchors of set s are [set_off[s], set_off[s+1]) of keys (see anchor_key); sorted in
// place. Chains of set s go to the ch_* arrays of `as` at set_off[s] + j, count to out_count.
void launch_chain_sets(cudaStream_t st, const int64_t* set_off, int64_t n_sets, const ChainParamsDev& cp,
                       AnchorScratch as, int32_t* out_count, uint32_t* err);

// Sort key of an anchor: strand, then rpos, then qpos (src/chain.cpp:16-20); qpos is
// biased by 2^30 so that it sorts as a signed value.
__host__ __device__ __forceinline__ uint64_t anchor_key(uint32_t strand, uint32_t rpos, int32_t qpos) {
  return (static_cast<uint64_t>(strand & 1u) << 62) | (static_cast<uint64_t>(rpos & 0x7FFFFFFFu) << 31) |
         static_cast<uint64_t>(static_cast<uint32_t>(qpos + (1 << 30)) & 0x7FFFFFFFu);
}
__host__ __device__ __forceinline__ uint32_t key_strand(uint64_t k) { return static_cast<uint32_t>(k >> 62); }
__host__ __device__ __forceinline__ uint32_t key_rpos(uint64_t k) {
  return static_cast<uint32_t>((k >> 31) & 0x7FFFFFFFu);
}
__host__ __device__ __forceinline__ int32_t key_qpos(uint64_t k) {
  return static_cast<int32_t>(k & 0x7FFFFFFFu) - (1 << 30);
}

}  // namespace dnb
