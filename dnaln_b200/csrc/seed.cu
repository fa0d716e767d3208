// seed.cu — minimizer sketching, index probing, anchor generation, colinear chaining and
// candidate selection, one warp per read (sm_100a).
//
// Sketch (src/minimizer.cpp:5-68). The reference streams a van Herk/Gil-Werman window
// minimum; here the 32 lanes of a warp take 32 consecutive k-mer starts at a time. Each
// lane builds its k-mer's forward and reverse-complement 2-bit words, its canonical hash
// (palindromes get the never-selected hash ~0) and parks it in a per-warp ring in shared
// memory; a ballot gives every lane the last k-mer start hit by an N, so "the window of w
// k-mers ending here lies in one N-free run" is a compare. A full window's minimum is its
// leftmost smallest hash (strict '<' scan over the ring). The reference emits the window
// minimum unless its position equals the last emitted one; because window minima move
// monotonically, that is the local rule "emit unless the previous window is full, has a
// valid minimum and picked the same position", evaluated with one shuffle. Emitted
// minimizers are compacted in order with a ballot.
//
// Probe (src/index.hpp:24-38, src/mapper.cpp:24-30): one lane per minimizer walks the
// open-addressing table with 16-byte vector loads; hits with count 0 or above max_occ
// are dropped.
//
// Chaining (src/chain.cpp:12-69). Anchors (src/mapper.cpp:32-40) are packed into one
// 64-bit key (strand, rpos, qpos) so the reference's sort is a warp bitonic sort of
// integers. The DP scans predecessors nearest-first with a `break` on strand change or
// dr > max_gap; because anchors are sorted by (strand, rpos), the scanned predecessors
// form one contiguous range, so the lanes test up to 32 predecessors each round
// independently and a warp max over (score << 32 | j) picks the best with ties to the
// nearest j, as the reference's strict '>' does. The FP64 gap cost comes from a
// host-computed table (exactly the reference's expression). Chains are extracted from end
// points in (f desc, index asc) order — another bitonic sort of packed keys — walked by
// one lane, and ordered by score with ties in extraction order (the reference's
// stable_sort). Candidate loci follow src/mapper.cpp:40-62.
#include <algorithm>

#include "common.cuh"
#include "seed.cuh"

namespace dnb {

namespace {

constexpr int kSeedWarps = 8;
constexpr int kRing = 512;  // >= 32 + max w (255)
constexpr int kChainWarps = 4;
constexpr int kSmCap = 256;  // anchors per read held in shared memory

struct SketchSmem {
  uint64_t hash[kRing];
  uint8_t strand[kRing];
};

// Sketches one sequence with the whole warp. code_at(i) returns the base code (0..4) at
// i; emit(rank, hash, pos, strand) is called by the emitting lanes, ranks in order.
// Returns the number of minimizers (same in all lanes).
template <class CodeAt, class Emit>
__device__ int warp_sketch(CodeAt code_at, int len, int k, int w, SketchSmem& sm, Emit emit) {
  const int lane = threadIdx.x & 31;
  const uint64_t mask = (1ULL << (2 * k)) - 1;
  const int nk = len - k + 1;  // k-mer starts
  int count = 0, carry_bad = -1, p_arg = -1;
  for (int base = 0; base < nk; base += 32) {
    const int s = base + lane;
    bool kv = false;
    uint64_t h = kInvalidHash;
    uint32_t st = 0;
    if (s < nk) {
      uint64_t fwd = 0, rev = 0;
      bool hasn = false;
      for (int m = 0; m < k; ++m) {
        const uint32_t c = code_at(s + m);
        hasn |= c > 3;
        fwd = (fwd << 2) | (c & 3u);
        rev |= static_cast<uint64_t>(3u - (c & 3u)) << (2 * m);
      }
      kv = !hasn;
      if (kv) {
        st = rev < fwd;
        h = fwd != rev ? hash64(st ? rev : fwd, mask) : kInvalidHash;
      }
    }
    __syncwarp();
    sm.hash[s & (kRing - 1)] = h;
    sm.strand[s & (kRing - 1)] = static_cast<uint8_t>(st);
    const unsigned bad = __ballot_sync(0xffffffffu, s < nk && !kv);
    const unsigned upto = bad & (0xffffffffu >> (31 - lane));
    const int lastbad = upto ? base + 31 - __clz(upto) : carry_bad;
    carry_bad = bad ? base + 31 - __clz(bad) : carry_bad;
    __syncwarp();
    int arg = -1;
    uint64_t mh = kInvalidHash;
    if (s < nk && s >= w - 1 && lastbad < s - w + 1) {  // full window of w k-mers
      int b = s - w + 1;
      uint64_t bh = sm.hash[b & (kRing - 1)];
      for (int j = b + 1; j <= s; ++j) {
        const uint64_t x = sm.hash[j & (kRing - 1)];
        if (x < bh) {
          bh = x;
          b = j;
        }
      }
      mh = bh;
      arg = bh != kInvalidHash ? b : -1;
    }
    const int up = __shfl_up_sync(0xffffffffu, arg, 1);
    const int prev_arg = lane == 0 ? p_arg : up;
    const bool em = arg >= 0 && arg != prev_arg;
    const unsigned ball = __ballot_sync(0xffffffffu, em);
    if (em) emit(count + __popc(ball & ((1u << lane) - 1u)), mh, arg, sm.strand[arg & (kRing - 1)]);
    count += __popc(ball);
    p_arg = __shfl_sync(0xffffffffu, arg, 31);
  }
  return count;
}

// 16-bit x -> its bits at the even positions of a 32-bit word.
__device__ __forceinline__ uint32_t spread16(uint32_t x) {
  x = (x | (x << 8)) & 0x00FF00FFu;
  x = (x | (x << 4)) & 0x0F0F0F0Fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}

// Value of `cur` held d lanes to the left (0 <= d <= 31); lanes left of d read `prv`, the
// previous chunk's value.
__device__ __forceinline__ uint64_t from_left(uint64_t cur, uint64_t prv, int d) {
  const int lane = threadIdx.x & 31;
  const int src = (lane - d) & 31;
  const uint64_t a = __shfl_sync(0xffffffffu, cur, src);
  const uint64_t b = __shfl_sync(0xffffffffu, prv, src);
  return lane >= d ? a : b;
}

__device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return b < a ? b : a; }

// warp_sketch for k <= 15 and w <= 32 (the defaults are 15 and 10), same output. Per
// chunk of 32 k-mer starts each lane loads one base code; three ballots give the 64
// positions the chunk's k-mers cover as bit planes (low bit, high bit, N), from which a
// lane assembles its k-mer directly: spreading the k low/high bits into alternate bit
// positions gives the reverse-complement word, and a bit reversal the forward word. The
// hash runs in 32 bits. Each lane packs (hash, position, strand) into one 64-bit key, so
// the leftmost minimum of a window is the minimum key; windows of w keys are minima of
// power-of-two windows (doubling with shuffles), previous-chunk values kept in registers.
template <class CodeAt, class Emit>
__device__ int warp_sketch_fast(CodeAt code_at, int len, int k, int w, Emit emit) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const uint32_t kmask = (1u << k) - 1u, mask2k = (1u << (2 * k)) - 1u;
  const int nk = len - k + 1;
  uint64_t P[6], prvP[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) prvP[j] = ~0ULL;
  int count = 0, carry_bad = -1, p_arg = -1;
  uint32_t c_lo = lane < len ? code_at(lane) : 4u;
  uint32_t c_hi = 32 + lane < len ? code_at(32 + lane) : 4u;
  for (int base = 0; base < nk; base += 32) {
    if (base > 0) {
      c_lo = c_hi;
      c_hi = base + 32 + lane < len ? code_at(base + 32 + lane) : 4u;
    }
    const uint64_t plo = static_cast<uint64_t>(__ballot_sync(FULL, c_lo & 1u)) |
                         static_cast<uint64_t>(__ballot_sync(FULL, c_hi & 1u)) << 32;
    const uint64_t phi = static_cast<uint64_t>(__ballot_sync(FULL, (c_lo >> 1) & 1u)) |
                         static_cast<uint64_t>(__ballot_sync(FULL, (c_hi >> 1) & 1u)) << 32;
    const uint64_t pn = static_cast<uint64_t>(__ballot_sync(FULL, c_lo > 3u)) |
                        static_cast<uint64_t>(__ballot_sync(FULL, c_hi > 3u)) << 32;
    const int s = base + lane;
    const bool kv = s < nk && ((static_cast<uint32_t>(pn >> lane) & kmask) == 0u);
    uint64_t key = ~0ULL;
    if (kv) {
      const uint32_t L = static_cast<uint32_t>(plo >> lane) & kmask, H = static_cast<uint32_t>(phi >> lane) & kmask;
      const uint32_t sl = spread16(L), sh = spread16(H);
      const uint32_t rev = (sl | sh << 1) ^ mask2k;       // base m at bits 2m, complemented
      const uint32_t fwd = __brev(sh | sl << 1) >> (32 - 2 * k);  // base m at bits 2(k-1-m)
      const uint32_t st = rev < fwd;
      const uint32_t h = fwd != rev ? hash32(st ? rev : fwd, mask2k) : 0xFFFFFFFFu;
      key = static_cast<uint64_t>(h) << 32 | static_cast<uint32_t>(s) << 1 | st;
    }
    const unsigned bad = __ballot_sync(FULL, s < nk && !kv);
    const unsigned upto = bad & (0xffffffffu >> (31 - lane));
    const int lastbad = upto ? base + 31 - __clz(upto) : carry_bad;
    carry_bad = bad ? base + 31 - __clz(bad) : carry_bad;
    // minima of windows of 2^j keys ending at s
    P[0] = key;
#pragma unroll
    for (int j = 0; j < 5; ++j)
      if ((2 << j) <= w) P[j + 1] = umin64(P[j], from_left(P[j], prvP[j], 1 << j));
    uint64_t m = ~0ULL;
    int off = 0;
#pragma unroll
    for (int j = 5; j >= 0; --j)
      if (w & (1 << j)) {
        m = umin64(m, from_left(P[j], prvP[j], off));
        off += 1 << j;
      }
#pragma unroll
    for (int j = 0; j < 6; ++j)
      if ((1 << j) <= w) prvP[j] = P[j];
    int arg = -1;
    if (s < nk && s >= w - 1 && lastbad < s - w + 1 && static_cast<uint32_t>(m >> 32) != 0xFFFFFFFFu)
      arg = static_cast<int>(static_cast<uint32_t>(m) >> 1);
    const int up = __shfl_up_sync(FULL, arg, 1);
    const int prev_arg = lane == 0 ? p_arg : up;
    const bool em = arg >= 0 && arg != prev_arg;
    const unsigned ball = __ballot_sync(FULL, em);
    if (em) emit(count + __popc(ball & ((1u << lane) - 1u)), m >> 32, arg, static_cast<uint32_t>(m) & 1u);
    count += __popc(ball);
    p_arg = __shfl_sync(FULL, arg, 31);
  }
  return count;
}

// Ascending sort of a[0, n) by the warp: bitonic network in its all-ascending form (the
// first comparator of each merge pairs mirrored indices), so indices >= n act as +inf
// padding and their comparators are skipped.
__device__ void warp_sort_u64(uint64_t* a, int n) {
  if (n <= 1) return;
  const int lane = threadIdx.x & 31;
  int lgN = 0;
  while ((1 << lgN) < n) ++lgN;
  const int halfN = 1 << (lgN - 1);
  for (int lgs = 1; lgs <= lgN; ++lgs) {
    const int lgh = lgs - 1, size = 1 << lgs;
    for (int idx = lane; idx < halfN; idx += 32) {
      const int blk = idx >> lgh, off = idx & ((1 << lgh) - 1);
      const int i = blk * size + off, j = blk * size + size - 1 - off;
      if (j < n) {
        const uint64_t x = a[i], y = a[j];
        if (y < x) {
          a[i] = y;
          a[j] = x;
        }
      }
    }
    __syncwarp();
    for (int lgt = lgh - 1; lgt >= 0; --lgt) {
      const int stride = 1 << lgt;
      for (int idx = lane; idx < halfN; idx += 32) {
        const int blk = idx >> lgt, off = idx & (stride - 1);
        const int i = blk * 2 * stride + off, j = i + stride;
        if (j < n) {
          const uint64_t x = a[i], y = a[j];
          if (y < x) {
            a[i] = y;
            a[j] = x;
          }
        }
      }
      __syncwarp();
    }
  }
}

__device__ __forceinline__ uint32_t desc32(int32_t x) { return 0x7FFFFFFFu - static_cast<uint32_t>(x); }

struct ChainArrays {
  uint64_t* keys;
  int32_t* f;
  int32_t* prev;
  uint64_t* ord;
  uint8_t* used;
};

// The chaining DP for any lookback, in rounds of 32 predecessors (src/chain.cpp:22-45).
// Per round one redux over score * 32 + (31 - lane): the largest score, ties to the
// smallest lane = the nearest j; earlier (nearer) rounds win ties across rounds through
// the strict '>' below — the reference's scan order.
__device__ void chain_dp_rounds(const ChainArrays& a, int n, const ChainParamsDev& cp) {
  const int lane = threadIdx.x & 31;
  for (int i = 0; i < n; ++i) {
    const uint64_t ki = a.keys[i];
    const uint32_t si = key_strand(ki);
    const int64_t ri = key_rpos(ki), qi = key_qpos(ki);
    int best_sc = 0, best_j = -1;
    for (int r0 = 0; r0 < cp.lookback; r0 += 32) {
      const int t = r0 + lane, j = i - 1 - t;
      bool stop = true;
      int key = INT_MIN;
      if (t < cp.lookback && j >= 0) {
        const uint64_t kj = a.keys[j];
        const int64_t dr = ri - key_rpos(kj);
        if (key_strand(kj) == si && dr <= cp.max_gap) {
          stop = false;
          const int64_t dq = qi - key_qpos(kj);
          if (dr > 0 && dq > 0) {
            const int64_t dd = dr > dq ? dr - dq : dq - dr;
            if (dd <= cp.band) {
              int64_t g = dq < dr ? dq : dr;
              if (g > cp.k) g = cp.k;
              const int sc = a.f[j] + static_cast<int>(g) - cp.cost[dd];
              key = sc * 32 + (31 - lane);
            }
          }
        }
      }
      const int m = __reduce_max_sync(0xffffffffu, key);
      if (m != INT_MIN && (best_j < 0 || (m >> 5) > best_sc)) {
        best_sc = m >> 5;
        best_j = i - 1 - (r0 + 31 - (m & 31));
      }
      if (__all_sync(0xffffffffu, stop)) break;  // every later predecessor is out of range too
    }
    if (lane == 0) {
      if (best_j >= 0 && best_sc > cp.k) {
        a.f[i] = best_sc;
        a.prev[i] = best_j;
      } else {
        a.f[i] = cp.k;
        a.prev[i] = -1;
      }
    }
    __syncwarp();
  }
}

// Chain extraction (src/chain.cpp:49-68) as the reference runs it: ends in order of f
// descending, index ascending; each walks prev links until an anchor an earlier chain
// took. Chains go to as.ch_*[c0 + j]; returns m with the final order in ord[0, m).
__device__ int extract_serial(const ChainArrays& a, int n, const ChainParamsDev& cp, const AnchorScratch& as,
                              int64_t c0) {
  const int lane = threadIdx.x & 31;
  // extraction order: f descending, index ascending (src/chain.cpp:49-50)
  for (int i = lane; i < n; i += 32) {
    a.ord[i] = static_cast<uint64_t>(desc32(a.f[i])) << 32 | static_cast<uint32_t>(i);
    a.used[i] = 0;
  }
  __syncwarp();
  warp_sort_u64(a.ord, n);
  int m = 0;
  if (lane == 0) {  // walk (src/chain.cpp:52-67)
    for (int e = 0; e < n; ++e) {
      const int end = static_cast<int>(a.ord[e] & 0xffffffffu);
      if (a.used[end]) continue;
      int i = end, cnt = 0;
      int64_t dmin = LLONG_MAX, dmax = LLONG_MIN;
      while (i >= 0 && !a.used[i]) {
        a.used[i] = 1;
        ++cnt;
        const uint64_t ki = a.keys[i];
        const int64_t d = static_cast<int64_t>(key_rpos(ki)) - key_qpos(ki);
        dmin = d < dmin ? d : dmin;
        dmax = d > dmax ? d : dmax;
        i = a.prev[i];
      }
      const int score = a.f[end] - (i >= 0 ? a.f[i] : 0);
      if (score < cp.min_score || cnt < cp.min_anchors) continue;
      const uint64_t ke = a.keys[end];
      as.ch_score[c0 + m] = score;
      as.ch_sn[c0 + m] = key_strand(ke) | static_cast<uint32_t>(cnt) << 1;
      as.ch_dmin[c0 + m] = dmin;
      as.ch_dmax[c0 + m] = dmax;
      as.ch_rpos[c0 + m] = key_rpos(ke);
      ++m;
    }
  }
  m = __shfl_sync(0xffffffffu, m, 0);
  __syncwarp();
  // final order: score descending, extraction order ascending (stable_sort, src/chain.cpp:68)
  for (int j = lane; j < m; j += 32)
    a.ord[j] = static_cast<uint64_t>(desc32(as.ch_score[c0 + j])) << 32 | static_cast<uint32_t>(j);
  __syncwarp();
  warp_sort_u64(a.ord, m);
  return m;
}

// The same chains for n <= 32 * E <= 256 anchors, found without the serial walk. Rank the
// anchors by the extraction order (f descending, index ascending). The walk of end e
// takes exactly the anchors x whose lowest-ranked descendant in the prev forest (the
// anchors whose prev path passes through x, x included) is e: ranks of ends taken
// earlier are lower, and a walk stops at the first anchor an earlier walk took, from
// where on its path every anchor is taken by earlier walks too. An end whose own
// lowest-ranked descendant is not itself lies on an earlier walk and is skipped. So:
//  1. claim[x] = min over descendants of (desc f, index), by pointer jumping: each round
//     every anchor pushes its claim to its ancestor 2^t links up (a shared-memory atomic
//     min) and then doubles its link, until no link is left (log2 n + 1 rounds);
//  2. the chain of end e is {x : claim[x] = e}; its last member's prev is the anchor
//     where the walk stopped (score = f[e] - f[stop]), and count, min and max diagonal
//     are shared-memory atomics into slots at index e.
// Chain records go to as.ch_*[c0 + e] (slot = end index) and ord[0, m) holds the final
// order (score descending, extraction order ascending; low 32 bits = slot). The rank key
// (desc f, index) is packed into 32 bits as (0x7FFFFF - f) << 8 | index, which needs
// 0 <= f <= 0x7FFFFF; a read outside that (never for k <= 32) uses extract_serial.
template <int E>
__device__ int extract_par(const ChainArrays& a, int n, const ChainParamsDev& cp, const AnchorScratch& as,
                           int64_t c0) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  bool f_ok = true;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int y = e * 32 + lane;
    if (y < n) f_ok = f_ok && a.f[y] >= 0 && a.f[y] <= 0x7FFFFF;
  }
  if (!__all_sync(FULL, f_ok)) return extract_serial(a, n, cp, as, c0);
  uint64_t* claim = a.ord;  // claim keys: desc32(f) << 32 | index, min over descendants
  uint8_t* link = a.used;   // pointer-jumping links + 1 (0 = none); every link < n <= 256
  int anc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int y = e * 32 + lane;
    anc[e] = -1;
    if (y < n) {
      anc[e] = a.prev[y];
      link[y] = static_cast<uint8_t>(anc[e] + 1);
      claim[y] = static_cast<uint64_t>(desc32(a.f[y])) << 32 | static_cast<uint32_t>(y);
    }
  }
  __syncwarp();
  for (;;) {
    bool more = false;
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (anc[e] >= 0) atomicMin(reinterpret_cast<unsigned long long*>(claim + anc[e]),
                                 static_cast<unsigned long long>(claim[e * 32 + lane]));
    __syncwarp();
#pragma unroll
    for (int e = 0; e < E; ++e) {
      if (anc[e] >= 0) anc[e] = static_cast<int>(link[anc[e]]) - 1;
      more = more || anc[e] >= 0;
    }
    if (!__any_sync(FULL, more)) break;
    __syncwarp();
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int y = e * 32 + lane;
      if (y < n) link[y] = static_cast<uint8_t>(anc[e] + 1);
    }
    __syncwarp();
  }
  __syncwarp();
  // per anchor: its chain's end, or (ends) 0x80000000 | f; the stop and score of a chain
  // from its last member
  uint32_t pk[E];
  int sc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int y = e * 32 + lane;
    pk[e] = 0;
    sc[e] = INT_MIN;
    if (y < n) {
      const int c = static_cast<int>(claim[y] & 0xFFu);
      const int p = a.prev[y];
      pk[e] = c == y ? 0x80000000u | static_cast<uint32_t>(a.f[y]) : static_cast<uint32_t>(c);
      if (p < 0 || static_cast<int>(claim[p] & 0xFFu) != c) sc[e] = a.f[c] - (p >= 0 ? a.f[p] : 0);
    }
  }
  __syncwarp();
  // slots at the end's index: claim -> min | max biased diagonal, prev -> count, f -> score
  uint32_t* dlo = reinterpret_cast<uint32_t*>(claim);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int y = e * 32 + lane;
    if (y < n && (pk[e] >> 31)) {
      claim[y] = 0xFFFFFFFFull;
      a.prev[y] = 0;
    }
    if (sc[e] != INT_MIN) a.f[(pk[e] >> 31) ? y : static_cast<int>(pk[e])] = sc[e];
  }
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int y = e * 32 + lane;
    if (y < n) {
      const int c = (pk[e] >> 31) ? y : static_cast<int>(pk[e]);
      const uint64_t ky = a.keys[y];
      // rpos < 2^31 and |qpos| < 2^30: rpos - qpos + 2^30 fits 32 bits unsigned
      const uint32_t d = key_rpos(ky) - static_cast<uint32_t>(key_qpos(ky)) + (1u << 30);
      atomicMin(dlo + 2 * c, d);
      atomicMax(dlo + 2 * c + 1, d);
      atomicAdd(a.prev + c, 1);
    }
  }
  __syncwarp();
  // chain records of the ends that pass the filters
  bool keep[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int y = e * 32 + lane;
    keep[e] = false;
    if (y < n && (pk[e] >> 31)) {
      const int score = a.f[y], cnt = a.prev[y];
      keep[e] = !(score < cp.min_score || cnt < cp.min_anchors);
      if (keep[e]) {
        const uint64_t ke = a.keys[y];
        as.ch_score[c0 + y] = score;
        as.ch_sn[c0 + y] = key_strand(ke) | static_cast<uint32_t>(cnt) << 1;
        as.ch_dmin[c0 + y] = static_cast<int64_t>(dlo[2 * y]) - (1ll << 30);
        as.ch_dmax[c0 + y] = static_cast<int64_t>(dlo[2 * y + 1]) - (1ll << 30);
        as.ch_rpos[c0 + y] = key_rpos(ke);
      }
    }
  }
  __syncwarp();
  // final order: score descending, extraction order ascending (stable_sort, src/chain.cpp:68)
  int m = 0;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const unsigned b = __ballot_sync(FULL, keep[e]);
    if (keep[e]) {
      const int y = e * 32 + lane;
      const uint32_t rank = (0x7FFFFFu - (pk[e] & 0x7FFFFFu)) << 8 | static_cast<uint32_t>(y);
      a.ord[m + __popc(b & ((1u << lane) - 1u))] = static_cast<uint64_t>(desc32(a.f[y])) << 32 | rank;
    }
    m += __popc(b);
  }
  __syncwarp();
  warp_sort_u64(a.ord, m);
  for (int j = lane; j < m; j += 32) a.ord[j] = (a.ord[j] & 0xFFFFFFFF00000000ull) | (a.ord[j] & 0xFFu);
  __syncwarp();
  return m;
}

// Sorts the n anchor keys, runs the DP, extracts chains into as.ch_*[c0 + j] (j a slot
// below n) and leaves their final order in ord[0, m) (low 32 bits = j). Returns m in
// every lane.
__device__ int chain_core(ChainArrays a, int n, const ChainParamsDev& cp, const AnchorScratch& as, int64_t c0) {
  const int lane = threadIdx.x & 31;
  warp_sort_u64(a.keys, n);
  // DP (src/chain.cpp:22-45). For row i, lane t holds in registers the key and f of
  // anchor i-1-t (the 32 nearest predecessors); after the row the window moves up one
  // lane and row i enters at lane 0, so f never makes a round trip through memory on the
  // DP's serial path. Predecessors at distance 33..lookback are read from a.keys / a.f
  // only when the one at distance 32 has not stopped the scan: anchors are sorted by
  // (strand, rpos), so a strand change or dr > max_gap at j holds for every farther j
  // too (and each lane can test its own j). One redux per row takes the max of
  // score * 64 + (63 - distance): the largest score, ties to the nearest predecessor
  // (the reference scans j downward with a strict '>').
  const unsigned FULL = 0xffffffffu;
  if (cp.lookback > 64) {
    chain_dp_rounds(a, n, cp);
  } else {
  int rw = 0, qw = 0, fw = 0;
  uint32_t sw = 0;
  const bool two = cp.lookback > 32;
  uint64_t ki = n > 0 ? a.keys[0] : 0;
  for (int i = 0; i < n; ++i) {
    const uint64_t knext = i + 1 < n ? a.keys[i + 1] : 0;
    const uint32_t si = key_strand(ki);
    const int ri = static_cast<int>(key_rpos(ki)), qi = key_qpos(ki);
    // rpos < 2^31 and |qpos| < 2^30, so dr and dq fit 32 bits; dd is formed in unsigned
    // arithmetic and used only when dr and dq passed the range tests
    const auto score_of = [&](int rj, int qj, uint32_t sj, int fj, int t) -> int {
      const int dr = ri - rj, dq = qi - qj;
      const int dd = static_cast<int>(dr > dq ? static_cast<uint32_t>(dr) - static_cast<uint32_t>(dq)
                                              : static_cast<uint32_t>(dq) - static_cast<uint32_t>(dr));
      if (t >= cp.lookback || t >= i || sj != si || dr > cp.max_gap || dr <= 0 || dq <= 0 || dd > cp.band)
        return INT_MIN;
      const int g = min(min(dq, dr), cp.k);
      return (fj + g - cp.cost[dd]) * 64 + (63 - t);
    };
    int c = score_of(rw, qw, sw, fw, lane);
    if (two && i > 32) {
      const bool live = sw == si && ri - rw <= cp.max_gap;  // lane 31: the predecessor i-32
      if (__shfl_sync(FULL, live, 31)) {
        __syncwarp();  // f of rows <= i-33, written by lane 0, is visible to every lane
        const int j = i - 33 - lane;
        if (j >= 0) {
          const uint64_t kj = a.keys[j];
          c = max(c, score_of(static_cast<int>(key_rpos(kj)), key_qpos(kj), key_strand(kj), a.f[j], 32 + lane));
        }
      }
    }
    const int m = __reduce_max_sync(FULL, c);
    int fi = cp.k, pi = -1;
    if (m != INT_MIN && (m >> 6) > cp.k) {
      fi = m >> 6;
      pi = i - 1 - (63 - (m & 63));
    }
    if (lane == 0) {
      a.f[i] = fi;
      a.prev[i] = pi;
    }
    // move the window up one lane; row i enters at lane 0
    rw = __shfl_up_sync(FULL, rw, 1);
    qw = __shfl_up_sync(FULL, qw, 1);
    fw = __shfl_up_sync(FULL, fw, 1);
    sw = __shfl_up_sync(FULL, sw, 1);
    if (lane == 0) {
      rw = ri;
      qw = qi;
      fw = fi;
      sw = si;
    }
    ki = knext;
  }
  }
  __syncwarp();
  if (n <= 32) return extract_par<1>(a, n, cp, as, c0);
  if (n <= 64) return extract_par<2>(a, n, cp, as, c0);
  if (n <= 128) return extract_par<4>(a, n, cp, as, c0);
  if (n <= 256) return extract_par<8>(a, n, cp, as, c0);
  return extract_serial(a, n, cp, as, c0);
}

// Ascending bitonic sort of one 64-bit key per lane across the warp (lane order).
__device__ __forceinline__ uint64_t warp_bitonic_u64(uint64_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const uint64_t o = __shfl_xor_sync(0xffffffffu, v, j);
      const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
      v = keep_min ? (o < v ? o : v) : (o > v ? o : v);
    }
  }
  return v;
}

// Chaining and candidate selection of a read with n <= 32 anchors, entirely in registers:
// lane j holds anchor j (after the sort), its f and prev; every sequential step of the
// reference (DP rows, the walk, the candidate loop) runs as a warp-uniform loop whose
// operands come from shuffles, and the DP's predecessor max is one redux per row.
// Same results as chain_core + the candidate loop of k_chain_map.
__device__ void chain_map_small(uint64_t key, int n, const ChainParamsDev& cp, const CandParams& cand,
                                const DevIndex& ix, const CandBuf& cb, int64_t r) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  key = warp_bitonic_u64(key);  // lanes >= n hold ~0 and sort last
  const uint32_t st = key_strand(key);
  const int32_t rp = static_cast<int32_t>(key_rpos(key)), qp = key_qpos(key);
  // DP (src/chain.cpp:22-45); row i's best predecessor: max over lanes j < i of
  // score * 32 + j, i.e. ties to the nearest j
  int f = cp.k, prev = -1;
  for (int i = 1; i < n; ++i) {
    const uint32_t si = __shfl_sync(FULL, st, i);
    const int32_t ri = __shfl_sync(FULL, rp, i), qi = __shfl_sync(FULL, qp, i);
    int kv = INT_MIN;
    if (lane < i && lane >= i - cp.lookback && st == si) {
      const int64_t dr = static_cast<int64_t>(ri) - rp;
      const int64_t dq = static_cast<int64_t>(qi) - qp;
      if (dr <= cp.max_gap && dr > 0 && dq > 0) {
        const int64_t dd = dr > dq ? dr - dq : dq - dr;
        if (dd <= cp.band) {
          int64_t g = dq < dr ? dq : dr;
          if (g > cp.k) g = cp.k;
          kv = (f + static_cast<int>(g) - cp.cost[dd]) * 32 + lane;
        }
      }
    }
    const int m = __reduce_max_sync(FULL, kv);
    if (lane == i && m != INT_MIN && (m >> 5) > cp.k) {
      f = m >> 5;
      prev = m & 31;
    }
  }
  // extraction order: f descending, index ascending (src/chain.cpp:49-50)
  const uint64_t ok = lane < n ? (static_cast<uint64_t>(desc32(f)) << 32 | static_cast<uint32_t>(lane)) : ~0ULL;
  const int end_of = static_cast<int>(warp_bitonic_u64(ok) & 0xffffffffu);
  const int64_t dg = static_cast<int64_t>(rp) - qp;
  // walk (src/chain.cpp:52-67); chain m is kept in the registers of lane m
  uint32_t used = 0;
  int m = 0, c_score = 0;
  uint32_t c_strand = 0, c_rpos = 0;
  int64_t c_dmin = 0, c_dmax = 0;
  for (int e = 0; e < n; ++e) {
    const int end = __shfl_sync(FULL, end_of, e);
    if ((used >> end) & 1u) continue;
    int i = end, cnt = 0;
    int64_t dmin = LLONG_MAX, dmax = LLONG_MIN;
    while (i >= 0 && !((used >> i) & 1u)) {
      used |= 1u << i;
      ++cnt;
      const int64_t d = __shfl_sync(FULL, dg, i);
      dmin = d < dmin ? d : dmin;
      dmax = d > dmax ? d : dmax;
      i = __shfl_sync(FULL, prev, i);
    }
    const int f_end = __shfl_sync(FULL, f, end);
    const int f_stop = __shfl_sync(FULL, f, i >= 0 ? i : 0);
    const uint32_t s_end = __shfl_sync(FULL, st, end);
    const int32_t r_end = __shfl_sync(FULL, rp, end);
    const int score = f_end - (i >= 0 ? f_stop : 0);
    if (score < cp.min_score || cnt < cp.min_anchors) continue;
    if (lane == m) {
      c_score = score;
      c_strand = s_end;
      c_rpos = static_cast<uint32_t>(r_end);
      c_dmin = dmin;
      c_dmax = dmax;
    }
    ++m;
  }
  // chains by score descending, ties in extraction order (stable_sort, src/chain.cpp:68)
  const uint64_t sk = lane < m ? (static_cast<uint64_t>(desc32(c_score)) << 32 | static_cast<uint32_t>(lane)) : ~0ULL;
  const int chain_at = static_cast<int>(warp_bitonic_u64(sk) & 0xffffffffu);
  // candidate loci (src/mapper.cpp:40-62); accepted candidate x is kept by lane x
  int nd = 0;
  int64_t my_diag = 0;
  uint32_t my_rev = 0;
  const int64_t cbase = r * cand.max_cand;
  if (m > 0) {
    const double min_score =
        static_cast<double>(__shfl_sync(FULL, c_score, __shfl_sync(FULL, chain_at, 0))) * cand.pri_ratio;
    for (int c = 0; c < m; ++c) {
      const int ci = __shfl_sync(FULL, chain_at, c);
      const int sc = __shfl_sync(FULL, c_score, ci);
      if (static_cast<double>(sc) < min_score || nd >= cand.max_cand) break;
      const int64_t dmin = __shfl_sync(FULL, c_dmin, ci), dmax = __shfl_sync(FULL, c_dmax, ci);
      const int64_t diag = dmin + (dmax - dmin) / 2;
      const uint32_t strand = __shfl_sync(FULL, c_strand, ci);
      const uint32_t rpos = __shfl_sync(FULL, c_rpos, ci);
      const int64_t dd = my_diag - diag;
      if (__any_sync(FULL, lane < nd && my_rev == strand && (dd < 0 ? -dd : dd) <= cand.bw)) continue;
      if (lane == nd) {
        my_diag = diag;
        my_rev = strand;
      }
      if (lane == 0) {
        cb.rev[cbase + nd] = static_cast<uint8_t>(strand);
        cb.contig[cbase + nd] = contig_of(ix, rpos);
        cb.diag[cbase + nd] = diag;
        cb.wstart[cbase + nd] = diag - cand.bw;
      }
      ++nd;
    }
  }
  if (lane == 0) cb.n_cand[r] = nd;
}

struct ChainSmem {
  uint64_t keys[kSmCap];
  uint64_t ord[kSmCap];
  int32_t f[kSmCap];
  int32_t prev[kSmCap];
  uint8_t used[kSmCap];
};

// Pass 1 of read r by one warp (codes of both strands unless `encode` is false, because
// another kernel already wrote them).
__device__ void seed_read(int64_t r, bool encode, const char* __restrict__ seq, const int64_t* __restrict__ seq_off,
                          int64_t seq_base, const int32_t* __restrict__ seq_len, const int64_t* __restrict__ pofs,
                          uint8_t* __restrict__ codes, const DevIndex& ix, const SeedParams& sp, const MinBuf& mb,
                          int32_t* __restrict__ n_min, int64_t* __restrict__ n_anchor, uint32_t* __restrict__ err,
                          SketchSmem& smw) {
  const int lane = threadIdx.x & 31;
  const int64_t so = pofs[r];  // packed offset of this read's codes and minimizer slots
  const int len = seq_len[r];
  const uint8_t* s = reinterpret_cast<const uint8_t*>(seq) + (seq_off[r] - seq_base);
  uint8_t* fw = codes + 2 * so;
  uint8_t* rc = fw + len;
  if (encode) {
    for (int i = lane; i < len; i += 32) {  // src/mapper.cpp:88-99
      const uint8_t c = nt4(s[i]);
      fw[i] = c;
      rc[len - 1 - i] = c < 4 ? static_cast<uint8_t>(3 - c) : 4;
    }
  }
  const auto code_at = [&](int i) { return nt4(s[i]); };
  const auto emit = [&](int rank, uint64_t h, int pos, uint32_t st) {
    mb.hash[so + rank] = h;
    mb.pos[so + rank] = static_cast<uint32_t>(pos) | st << 31;
  };
  const int cnt = (sp.k <= 15 && sp.w <= 32) ? warp_sketch_fast(code_at, len, sp.k, sp.w, emit)
                                             : warp_sketch(code_at, len, sp.k, sp.w, smw, emit);
  __syncwarp();
  long long anchors = 0;
  for (int j = lane; j < cnt; j += 32) {
    uint32_t off, c;
    probe(ix, mb.hash[so + j], off, c, err);
    if (c > sp.max_occ) c = 0;
    mb.hit_off[so + j] = off;
    mb.hit_cnt[so + j] = c;
    anchors += c;
  }
  anchors = warp_sum(anchors);
  if (lane == 0) {
    n_min[r] = cnt;
    n_anchor[r] = anchors;
  }
}

// One warp per read: reads [0, n), or with a list the reads list[0, *list_n) (grid-stride).
__global__ void __launch_bounds__(kSeedWarps * 32)
    k_seed(const char* __restrict__ seq, const int64_t* __restrict__ seq_off, int64_t seq_base,
           const int32_t* __restrict__ seq_len, const int64_t* __restrict__ pofs, int64_t n,
           const int32_t* __restrict__ list, const int* __restrict__ list_n, uint8_t* __restrict__ codes,
           DevIndex ix, SeedParams sp, MinBuf mb, int32_t* __restrict__ n_min, int64_t* __restrict__ n_anchor,
           uint32_t* __restrict__ err) {
  __shared__ SketchSmem sm[kSeedWarps];
  const int wib = threadIdx.x >> 5;
  const int64_t gw = static_cast<int64_t>(blockIdx.x) * kSeedWarps + wib;
  if (!list) {
    if (gw < n) seed_read(gw, true, seq, seq_off, seq_base, seq_len, pofs, codes, ix, sp, mb, n_min, n_anchor, err, sm[wib]);
    return;
  }
  const int m = *list_n;
  for (int64_t x = gw; x < m; x += static_cast<int64_t>(gridDim.x) * kSeedWarps)
    seed_read(list[x], false, seq, seq_off, seq_base, seq_len, pofs, codes, ix, sp, mb, n_min, n_anchor, err, sm[wib]);
}

// Pass 2 of read r by one warp.
// Scratch of a read with more than 32 anchors (chain records, and the anchors themselves
// past kSmCap) is taken from a pool by one atomic add; a read the pool cannot hold sets
// kErrChainPool, and the host maps the batch again with a pool of the size asked for.
__device__ void chain_read(int64_t r, const int64_t* __restrict__ pofs, const int32_t* __restrict__ seq_len,
                           const int32_t* __restrict__ n_min, const int64_t* __restrict__ n_anchor, const MinBuf& mb,
                           const DevIndex& ix, const ChainParamsDev& cp, const CandParams& cand,
                           const AnchorScratch& as, unsigned long long* __restrict__ pool_top, int64_t pool_cap,
                           const CandBuf& cb, uint32_t* __restrict__ err, ChainSmem& smw) {
  const int lane = threadIdx.x & 31;
  const int64_t na64 = n_anchor[r];
  if (na64 > 0x3FFFFFFF) {
    if (lane == 0) {
      atomicOr(err, kErrChainScratch);
      cb.n_cand[r] = 0;
    }
    return;
  }
  const int na = static_cast<int>(na64);
  int64_t a0 = 0;
  if (na > 32) {
    unsigned long long b = 0;
    if (lane == 0) b = atomicAdd(pool_top, static_cast<unsigned long long>(na));
    a0 = static_cast<int64_t>(__shfl_sync(0xffffffffu, b, 0));
    if (a0 + na > pool_cap) {
      if (lane == 0) {
        atomicOr(err, kErrChainPool);
        cb.n_cand[r] = 0;
      }
      return;
    }
  }
  const bool small = na <= kSmCap;
  ChainArrays a;
  a.keys = small ? smw.keys : as.keys + a0;
  a.ord = small ? smw.ord : as.ord + a0;
  a.f = small ? smw.f : as.f + a0;
  a.prev = small ? smw.prev : as.prev + a0;
  a.used = small ? smw.used : as.used + a0;
  const int64_t so = pofs[r];
  const int len = seq_len[r], nm = n_min[r], k = cp.k;
  // anchors in minimizer order x occurrence order (src/mapper.cpp:32-40)
  int w_off = 0;
  for (int base = 0; base < nm; base += 32) {
    const int j = base + lane;
    const int c = j < nm ? static_cast<int>(mb.hit_cnt[so + j]) : 0;
    int total;
    const int ex = warp_exclusive_scan(c, &total);
    if (c) {
      const uint32_t off = mb.hit_off[so + j], mp = mb.pos[so + j];
      const int32_t pos = static_cast<int32_t>(mp & 0x7FFFFFFFu);
      const uint32_t mst = mp >> 31;
      for (int t = 0; t < c; ++t) {
        const uint32_t v = __ldg(ix.positions + off + t);
        const uint32_t rev = (v & 1u) ^ mst;
        const int32_t qpos = rev ? len - pos - k : pos;
        a.keys[w_off + ex + t] = anchor_key(rev, v >> 1, qpos);
      }
    }
    w_off += total;
  }
  __syncwarp();
  if (na <= 32) {  // the common case: everything in registers
    chain_map_small(lane < na ? a.keys[lane] : ~0ULL, na, cp, cand, ix, cb, r);
    return;
  }
  const int m = chain_core(a, na, cp, as, a0);
  // candidate loci (src/mapper.cpp:40-62)
  const int64_t cbase = r * cand.max_cand;
  if (cand.max_cand <= 32) {
    // the chains are read 32 at a time, one per lane (one memory round trip for all of
    // them), then taken in order by a warp-uniform loop over shuffles; accepted
    // candidate x is kept by lane x and written out at the end
    const unsigned FULL = 0xffffffffu;
    int nd = 0;
    int64_t my_diag = 0;
    uint32_t my_rev = 0, my_rpos = 0;
    double min_score = 0;
    bool done = m == 0;
    for (int base = 0; base < m && !done; base += 32) {
      const int c = base + lane;
      int sc = 0;
      int64_t dg = 0;
      uint32_t st = 0, rp = 0;
      if (c < m) {
        const int64_t ci = a0 + static_cast<int64_t>(a.ord[c] & 0xffffffffu);
        sc = as.ch_score[ci];
        const int64_t dmin = as.ch_dmin[ci], dmax = as.ch_dmax[ci];
        dg = dmin + (dmax - dmin) / 2;
        st = as.ch_sn[ci] & 1u;
        rp = as.ch_rpos[ci];
      }
      if (base == 0) min_score = static_cast<double>(__shfl_sync(FULL, sc, 0)) * cand.pri_ratio;
      const int cnt = min(32, m - base);
      for (int t = 0; t < cnt; ++t) {
        const int sc_t = __shfl_sync(FULL, sc, t);
        if (static_cast<double>(sc_t) < min_score || nd >= cand.max_cand) {
          done = true;
          break;
        }
        const int64_t diag = __shfl_sync(FULL, dg, t);
        const uint32_t strand = __shfl_sync(FULL, st, t);
        const int64_t dd = my_diag - diag;
        if (__any_sync(FULL, lane < nd && my_rev == strand && (dd < 0 ? -dd : dd) <= cand.bw)) continue;
        const uint32_t rpos = __shfl_sync(FULL, rp, t);
        if (lane == nd) {
          my_diag = diag;
          my_rev = strand;
          my_rpos = rpos;
        }
        ++nd;
      }
    }
    if (lane < nd) {
      cb.rev[cbase + lane] = static_cast<uint8_t>(my_rev);
      cb.contig[cbase + lane] = contig_of(ix, my_rpos);
      cb.diag[cbase + lane] = my_diag;
      cb.wstart[cbase + lane] = my_diag - cand.bw;
    }
    if (lane == 0) cb.n_cand[r] = nd;
    return;
  }
  if (lane == 0) {
    int nd = 0;
    if (m > 0) {
      const double min_score = static_cast<double>(as.ch_score[a0 + (a.ord[0] & 0xffffffffu)]) * cand.pri_ratio;
      for (int c = 0; c < m; ++c) {
        const int64_t ci = a0 + (a.ord[c] & 0xffffffffu);
        if (static_cast<double>(as.ch_score[ci]) < min_score || nd >= cand.max_cand) break;
        const int64_t dmin = as.ch_dmin[ci], dmax = as.ch_dmax[ci];
        const int64_t diag = dmin + (dmax - dmin) / 2;
        const uint8_t strand = static_cast<uint8_t>(as.ch_sn[ci] & 1u);
        bool dup = false;
        for (int x = 0; x < nd && !dup; ++x) {
          const int64_t dd = cb.diag[cbase + x] - diag;
          dup = cb.rev[cbase + x] == strand && (dd < 0 ? -dd : dd) <= cand.bw;
        }
        if (dup) continue;
        cb.rev[cbase + nd] = strand;
        cb.contig[cbase + nd] = contig_of(ix, as.ch_rpos[ci]);
        cb.diag[cbase + nd] = diag;
        cb.wstart[cbase + nd] = diag - cand.bw;
        ++nd;
      }
    }
    cb.n_cand[r] = nd;
  }
}

// One warp per read: reads [0, n), or with a list the reads list[0, list_n) (grid-stride).
__global__ void __launch_bounds__(kChainWarps * 32, 8)
    k_chain_map(const int64_t* __restrict__ pofs, const int32_t* __restrict__ seq_len, int64_t n,
                const int32_t* __restrict__ list, const int* __restrict__ list_n, const int32_t* __restrict__ n_min,
                const int64_t* __restrict__ n_anchor, MinBuf mb, DevIndex ix, ChainParamsDev cp, CandParams cand,
                AnchorScratch as, unsigned long long* __restrict__ pool_top, int64_t pool_cap, CandBuf cb,
                int* __restrict__ claim, uint32_t* __restrict__ err) {
  __shared__ ChainSmem sm[kChainWarps];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t gw = static_cast<int64_t>(blockIdx.x) * kChainWarps + wib;
  const int64_t m = list ? static_cast<int64_t>(*list_n) : n;
  if (claim) {  // work stealing: the warp takes the next read when it is done with its last
    for (;;) {
      int x = 0;
      if (lane == 0) x = atomicAdd(claim, 1);
      x = __shfl_sync(0xffffffffu, x, 0);
      if (x >= m) break;
      chain_read(list ? list[x] : x, pofs, seq_len, n_min, n_anchor, mb, ix, cp, cand, as, pool_top, pool_cap, cb,
                 err, sm[wib]);
    }
    return;
  }
  for (int64_t x = gw; x < m; x += static_cast<int64_t>(gridDim.x) * kChainWarps)
    chain_read(list ? list[x] : x, pofs, seq_len, n_min, n_anchor, mb, ix, cp, cand, as, pool_top, pool_cap, cb, err,
               sm[wib]);
}

__global__ void __launch_bounds__(kSeedWarps * 32)
    k_sketch_codes(const uint8_t* __restrict__ codes, const int64_t* __restrict__ seq_off,
                   const int32_t* __restrict__ seq_len, const uint32_t* __restrict__ pos_offset, int64_t n, int k,
                   int w, uint64_t* __restrict__ out_hash, uint32_t* __restrict__ out_pos,
                   uint32_t* __restrict__ out_strand, int32_t* __restrict__ out_count) {
  __shared__ SketchSmem sm[kSeedWarps];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t r = static_cast<int64_t>(blockIdx.x) * kSeedWarps + wib;
  if (r >= n) return;
  const int64_t so = seq_off[r];
  const uint8_t* s = codes + so;
  const uint32_t po = pos_offset ? pos_offset[r] : 0u;
  const auto code_at = [&](int i) { return static_cast<uint32_t>(s[i]); };
  const auto emit = [&](int rank, uint64_t h, int pos, uint32_t st) {
    out_hash[so + rank] = h;
    out_pos[so + rank] = static_cast<uint32_t>(pos) + po;
    out_strand[so + rank] = st;
  };
  const int cnt = (k <= 15 && w <= 32) ? warp_sketch_fast(code_at, seq_len[r], k, w, emit)
                                       : warp_sketch(code_at, seq_len[r], k, w, sm[wib], emit);
  if (lane == 0) out_count[r] = cnt;
}

__global__ void k_lookup(DevIndex ix, const uint64_t* __restrict__ hashes, int64_t n, uint32_t* __restrict__ out_off,
                         uint32_t* __restrict__ out_cnt, uint32_t* __restrict__ err) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t off, c;
  probe(ix, hashes[i], off, c, err);
  out_off[i] = off;
  out_cnt[i] = c;
}

__global__ void __launch_bounds__(kChainWarps * 32)
    k_chain_sets(const int64_t* __restrict__ set_off, int64_t n_sets, ChainParamsDev cp, AnchorScratch as,
                 int32_t* __restrict__ out_count, uint32_t* __restrict__ err) {
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t s = static_cast<int64_t>(blockIdx.x) * kChainWarps + wib;
  if (s >= n_sets) return;
  const int64_t a0 = set_off[s];
  const int64_t na64 = set_off[s + 1] - a0;
  if (na64 > 0x3FFFFFFF) {
    if (lane == 0) {
      atomicOr(err, kErrChainScratch);
      out_count[s] = 0;
    }
    return;
  }
  ChainArrays a{as.keys + a0, as.f + a0, as.prev + a0, as.ord + a0, as.used + a0};
  const int m = chain_core(a, static_cast<int>(na64), cp, as, a0);
  if (lane == 0) out_count[s] = m;
}

}  // namespace

void launch_seed(cudaStream_t st, const char* seq, const int64_t* seq_off, int64_t seq_base, const int32_t* seq_len,
                 const int64_t* pofs, int64_t n, uint8_t* codes, const DevIndex& ix, const SeedParams& sp, MinBuf mb,
                 int32_t* n_min, int64_t* n_anchor, uint32_t* err) {
  if (n <= 0) return;
  const int64_t blocks = (n + kSeedWarps - 1) / kSeedWarps;
  k_seed<<<static_cast<unsigned>(blocks), kSeedWarps * 32, 0, st>>>(seq, seq_off, seq_base, seq_len, pofs, n, nullptr,
                                                                   nullptr, codes, ix, sp, mb, n_min, n_anchor, err);
}

void launch_seed_list(cudaStream_t st, const char* seq, const int64_t* seq_off, int64_t seq_base,
                      const int32_t* seq_len, const int64_t* pofs, int64_t n_max, const int32_t* list,
                      const int* list_n, uint8_t* codes, const DevIndex& ix, const SeedParams& sp, MinBuf mb,
                      int32_t* n_min, int64_t* n_anchor, uint32_t* err) {
  if (n_max <= 0) return;
  // grid-stride over a list whose length is only known on the device: a few resident waves
  const int64_t blocks = std::min<int64_t>((n_max + kSeedWarps - 1) / kSeedWarps, int64_t{8} * device_sm_count());
  k_seed<<<static_cast<unsigned>(blocks), kSeedWarps * 32, 0, st>>>(seq, seq_off, seq_base, seq_len, pofs, n_max,
                                                                   list, list_n, codes, ix, sp, mb, n_min, n_anchor,
                                                                   err);
}

void launch_chain_map(cudaStream_t st, const int64_t* pofs, const int32_t* seq_len, int64_t n, const int32_t* list,
                      const int* list_n, const int32_t* n_min, const int64_t* n_anchor, MinBuf mb,
                      const DevIndex& ix, const ChainParamsDev& cp, const CandParams& cand, AnchorScratch as,
                      unsigned long long* pool_top, int64_t pool_cap, CandBuf cb, int* claim, uint32_t* err) {
  if (n <= 0) return;
  // a count that may be known on the device only: with work stealing the resident blocks,
  // otherwise a grid-stride over a few resident waves
  int64_t cap = int64_t{16} * device_sm_count();
  if (claim) {
    static std::atomic<int> resident[kMaxDevices];
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < kMaxDevices) {
      v = resident[dev].load(std::memory_order_relaxed);
      if (v <= 0 && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_chain_map, kChainWarps * 32, 0) == cudaSuccess &&
          v > 0)
        resident[dev].store(v, std::memory_order_relaxed);
    }
    cudaGetLastError();
    cap = int64_t{v > 0 ? v : 8} * device_sm_count();
  }
  const int64_t blocks = std::min<int64_t>((n + kChainWarps - 1) / kChainWarps, cap);
  k_chain_map<<<static_cast<unsigned>(blocks), kChainWarps * 32, 0, st>>>(
      pofs, seq_len, n, list, list_n, n_min, n_anchor, mb, ix, cp, cand, as, pool_top, pool_cap, cb, claim, err);
}

void launch_sketch_codes(cudaStream_t st, const uint8_t* codes, const int64_t* seq_off, const int32_t* seq_len,
                         const uint32_t* pos_offset, int64_t n, int32_t k, int32_t w, uint64_t* out_hash,
                         uint32_t* out_pos, uint32_t* out_strand, int32_t* out_count) {
  if (n <= 0) return;
  const int64_t blocks = (n + kSeedWarps - 1) / kSeedWarps;
  k_sketch_codes<<<static_cast<unsigned>(blocks), kSeedWarps * 32, 0, st>>>(codes, seq_off, seq_len, pos_offset, n, k,
                                                                           w, out_hash, out_pos, out_strand,
                                                                           out_count);
}

void launch_lookup(cudaStream_t st, const DevIndex& ix, const uint64_t* hashes, int64_t n, uint32_t* out_off,
                   uint32_t* out_cnt, uint32_t* err) {
  if (n <= 0) return;
  const int64_t blocks = (n + 255) / 256;
  k_lookup<<<static_cast<unsigned>(blocks), 256, 0, st>>>(ix, hashes, n, out_off, out_cnt, err);
}

void launch_chain_sets(cudaStream_t st, const int64_t* set_off, int64_t n_sets, const ChainParamsDev& cp,
                       AnchorScratch as, int32_t* out_count, uint32_t* err) {
  if (n_sets <= 0) return;
  const int64_t blocks = (n_sets + kChainWarps - 1) / kChainWarps;
  k_chain_sets<<<static_cast<unsigned>(blocks), kChainWarps * 32, 0, st>>>(set_off, n_sets, cp, as, out_count, err);
}

}  // namespace dnb
