// seed_thread.cu — one thread per read: sketch, probe, anchors, chaining DP, chain
// extraction and candidate loci of a short read, in one pass with the read's whole state
// in shared memory (sm_100a).
//
// The warp-per-read kernels of seed.cu spend most of their instructions on warp
// collectives (ballots, shuffles, reductions) over reads whose work is a few dozen
// sequential steps. Here each thread owns a read and runs the reference's sequential
// algorithms directly; the 32 reads of a warp advance in lockstep (same k-mer index, same
// DP row), so the shared-memory layouts [slot][thread] are bank-conflict free.
//
//  * Staging: the codes of both strands in HBM (src/mapper.cpp:88-99), which this kernel,
//    SW and the warp kernels read, are written by k_encode_reads, launched before this
//    one. The warp copies the forward codes of its 32 reads into shared memory, each
//    read's aligned words into its thread's column, with one batch of cp.async for all
//    of them and one wait (one memory latency per warp, not one per group of reads).
//  * Sketch (src/minimizer.cpp:5-68): rolling 2-bit forward / reverse-complement words,
//    canonical strand, 32-bit hash (hash32); the window minimum of w keys (hash, position,
//    strand) by van Herk / Gil-Werman blocks of w: a running prefix minimum of the current
//    block and the suffix minima of the previous one, so each window costs one compare.
//    Emission follows the same local rule as the warp sketch (emit unless the previous
//    window was full and valid and picked the same position).
//  * Probe (src/index.hpp:24-38) in groups of four independent bucket loads; anchors
//    (src/mapper.cpp:32-40) in minimizer x occurrence order.
//  * Chaining (src/chain.cpp:12-69): the anchors are sorted as 64-bit keys (insertion sort
//    after reversing a descending run, which is how reverse-strand anchors arrive), the DP
//    scans j = i-1 down with the reference's break / skip rules and strict '>'. Extraction
//    repeatedly walks from the unused anchor of largest f (ties: smallest index): every
//    walk of the reference's (f desc, index asc) loop starts at exactly that anchor, since
//    all anchors before it in that order are used. Chains are taken in (score desc,
//    extraction order) order, which is the reference's stable_sort.
//  * Candidates (src/mapper.cpp:40-62).
//
// A read leaves this path — listed for the warp kernels, which recompute it from scratch —
// when it is longer than kTMaxLen, has more than kTMaxMin minimizers, kTMaxAnc anchors or
// kTMaxChains chains, or when the parameters are outside this path's range (see
// seed_thread_supported).
#include <algorithm>

#include "common.cuh"
#include "seed.cuh"

namespace dnb {

namespace {

constexpr int kTMaxLen = 256;             // longest read staged
constexpr int kTWords = kTMaxLen / 4;     // staged code words per read
constexpr int kTMaxMin = 32;              // minimizers per read
constexpr int kTMaxAnc = 32;              // anchors per read (one bit each in a 32-bit mask)
constexpr int kTMaxChains = 8;            // chains per read passing the score / anchor filters
constexpr int kTW = 10;                   // window length of the compiled sketch
constexpr int kProbe = 8;                 // minimizers probed with independent loads at once

// Dynamic shared memory of a block of TT threads (= reads): two regions of 32-bit words,
// each thread owning one column of each (word w of thread T at w * pitch + T), so that
// after the cooperative staging no thread ever touches another thread's words. Region A
// (pitch TT + 1, which spreads the banks): the staged code words, later the anchor keys
// (two words each). Region B (pitch TT): the minimizers {hash, pos | strand << 31} (two
// words each), later f << 8 | (prev + 1) of each anchor (words 0..31) and the chain table
// (words 32..63). The block size is the tuner's reads-per-block choice (64 or 128); the
// shared memory per read, and so the reads resident per SM, barely depend on it.
constexpr int kWordsA = kTWords + 2;  // a read of kTMaxLen bytes at any offset within its first word
constexpr int kWordsB = 64;
static_assert(2 * kTMaxAnc <= kWordsA, "anchor keys must fit a staging column");
static_assert((3 + kTMaxLen + 3) / 4 <= kWordsA, "a staged read must fit its column");
static_assert(2 * kTMaxMin <= kWordsB && kTMaxAnc + 4 * kTMaxChains <= kWordsB, "region B column too small");
constexpr int kTMaxBand = 256;  // chaining band the shared gap-cost table holds
template <int TT>
struct TLayout {
  static constexpr int kPitch = TT + 1;
  static constexpr int kRegionA = kWordsA * kPitch * 4;
  static constexpr int kRegionB = kWordsB * TT * 4;
  static constexpr int kSmem = kRegionA + kRegionB + (kTMaxBand + 1) * 4;
};

// 4-byte asynchronous copy global -> shared (both 4-byte aligned).
__device__ __forceinline__ void cp_async4(uint32_t* dst_smem, const void* src) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst_smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}

// Codes of both strands of every read (src/mapper.cpp:88-99): forward at codes[2*pofs[r]],
// reverse complement right after it. One warp per read (grid-stride), bytes in lane order
// so loads and stores are coalesced.
__global__ void __launch_bounds__(256)
    k_encode_reads(const char* __restrict__ seq, const int64_t* __restrict__ seq_off, int64_t seq_base,
                   const int32_t* __restrict__ seq_len, const int64_t* __restrict__ pofs, int64_t n,
                   uint8_t* __restrict__ codes) {
  // both codes of every byte value from a table in shared memory (forward code in the low
  // byte, its complement in the high byte): one lookup per base instead of the arithmetic
  __shared__ uint16_t s_code[256];
  for (int b = threadIdx.x; b < 256; b += blockDim.x) {
    const uint32_t c = nt4(static_cast<uint32_t>(b));
    s_code[b] = static_cast<uint16_t>(c | (c < 4 ? 3 - c : 4u) << 8);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t nw = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t r = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
    const int len = seq_len[r];
    const uint8_t* s = reinterpret_cast<const uint8_t*>(seq) + (seq_off[r] - seq_base);
    uint8_t* fw = codes + 2 * pofs[r];
    uint8_t* rc = fw + len;
#pragma unroll 4
    for (int i = lane; i < len; i += 32) {
      const uint32_t cc = s_code[s[i]];
      fw[i] = static_cast<uint8_t>(cc);
      rc[len - 1 - i] = static_cast<uint8_t>(cc >> 8);
    }
  }
}

template <int W, int TT>
__global__ void __launch_bounds__(TT)
    k_seed_chain_t(const uint8_t* __restrict__ codes, const int64_t* __restrict__ pofs,
                   const int32_t* __restrict__ seq_len, int64_t n, DevIndex ix, SeedParams sp, ChainParamsDev cp,
                   CandParams cand,
                   CandBuf cb, int32_t* __restrict__ n_min, int64_t* __restrict__ n_anchor,
                   int32_t* __restrict__ n_anc_t, int32_t* __restrict__ big_list, int* __restrict__ big_n,
                   uint32_t* __restrict__ err) {
  using L = TLayout<TT>;
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* const stg = reinterpret_cast<uint32_t*>(smem);  // region A (all columns, for the staging)
  int32_t* const lut = reinterpret_cast<int32_t*>(smem + L::kRegionA + L::kRegionB);  // chaining gap costs
  const int T = threadIdx.x, lane = T & 31;
  for (int d = T; d <= cp.band; d += TT) lut[d] = cp.cost[d];
  __syncthreads();
  uint32_t* const ca = stg + T;                                                   // this thread's A column
  uint32_t* const cbw = reinterpret_cast<uint32_t*>(smem + L::kRegionA) + T;         // this thread's B column
  // anchor a: word 2a = strand << 31 | rpos, word 2a+1 = qpos (>= 0 here); as one 64-bit
  // key (word 2a high) it orders like (strand, rpos, qpos), the reference's anchor order
  const auto a_hi = [&](int a) -> uint32_t& { return ca[2 * a * L::kPitch]; };
  const auto a_lo = [&](int a) -> uint32_t& { return ca[(2 * a + 1) * L::kPitch]; };
  const auto key_ld = [&](int a) { return static_cast<uint64_t>(a_hi(a)) << 32 | a_lo(a); };
  const auto key_st = [&](int a, uint64_t v) {
    a_hi(a) = static_cast<uint32_t>(v >> 32);
    a_lo(a) = static_cast<uint32_t>(v);
  };
  // DP word of anchor i: (prev + 1) | f << 8 | max(f[0..i]) << 20 (f <= k * 32 < 4096)
  const auto fp_at = [&](int i) -> uint32_t& { return cbw[i * TT]; };
  const auto f_of = [](uint32_t w) { return static_cast<int>((w >> 8) & 0xFFFu); };
  const auto ch_at = [&](int field, int c) -> int32_t& {
    return reinterpret_cast<int32_t&>(cbw[(kTMaxAnc + field * kTMaxChains + c) * TT]);
  };

  const int64_t r0 = static_cast<int64_t>(blockIdx.x) * TT + (T & ~31);  // first read of this warp
  const int64_t r = r0 + lane;
  int len = 0;
  uint64_t a_word = 0;  // this read's first code byte rounded down to a 4-byte boundary
  int offb = 0, nwords = 0;
  if (r < n) {
    len = seq_len[r];
    const uint64_t a = reinterpret_cast<uint64_t>(codes) + 2 * static_cast<uint64_t>(pofs[r]);  // forward codes
    offb = static_cast<int>(a & 3u);
    a_word = a - static_cast<uint64_t>(offb);
    if (len > 0 && len <= kTMaxLen) nwords = (offb + len + 3) >> 2;
  }

  // ---- staging: word w of read j's codes (from its aligned start) into word w of column j.
  // Every copied word holds at least one byte of its read, so it lies in the pages the
  // read is in. All copies of the warp are in flight before the one wait.
  for (int j = 0; j < 32; ++j) {
    const uint64_t aj = __shfl_sync(0xffffffffu, a_word, j);
    const int nwj = __shfl_sync(0xffffffffu, nwords, j);
    const int tj = (T & ~31) + j;
    for (int w = lane; w < nwj; w += 32)
      cp_async4(stg + w * L::kPitch + tj, reinterpret_cast<const void*>(aj + 4u * static_cast<uint64_t>(w)));
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncwarp();
  if (r >= n) return;

  const int k = sp.k;
  bool big = len > kTMaxLen;
  int nmin = 0;
  // ---- sketch (src/minimizer.cpp:5-68)
  if (!big && len >= k) {
    const uint32_t mask2k = (1u << (2 * k)) - 1u;
    const int nk = len - k + 1;
    uint32_t fwd = 0, rev = 0, wcur = ca[0], wsh = 8u * static_cast<uint32_t>(offb);
    const uint32_t* wnext = ca + L::kPitch;
    int run = 0;
    // consumes the next code; a staged word is loaded as soon as the one before is used up,
    // a whole position's work ahead of its first byte (the column holds one word past the
    // read's last, so the load after the read's last word stays inside it)
    auto roll = [&](int) {
      const uint32_t c = (wcur >> wsh) & 0xFFu;  // 0..3, 4 for N
      wsh += 8u;
      if (wsh == 32u) {
        wsh = 0u;
        wcur = *wnext;
        wnext += L::kPitch;
      }
      run = c < 4 ? run + 1 : 0;
      fwd = ((fwd << 2) | (c & 3u)) & mask2k;
      rev = (rev >> 2) | ((3u - (c & 3u)) << (2 * k - 2));
    };
    for (int i = 0; i < k - 1; ++i) roll(i);
    // Window minimum over (hash, position) pairs: hashes are below 2^(2k) <= 2^30 and an
    // invalid position has hash ~0, so one 32-bit compare of the hashes orders two entries
    // when ties go to the left operand (the earlier position), as the reference's leftmost
    // rule asks: position words are pos << 1 | strand.
    uint32_t cur_h[W], cur_p[W], suf_h[W], suf_p[W];
#pragma unroll
    for (int u = 0; u < W; ++u) {
      suf_h[u] = 0xFFFFFFFFu;
      suf_p[u] = 0;
    }
    uint32_t pre_h = 0xFFFFFFFFu, pre_p = 0;
    int lastbad = -1, prev_arg = -1;
    for (int s0 = 0; s0 < nk; s0 += W) {
#pragma unroll
      for (int u = 0; u < W; ++u) {
        const int s = s0 + u;
        cur_h[u] = 0xFFFFFFFFu;
        cur_p[u] = 0;
        if (s < nk) {
          roll(s + k - 1);
          uint32_t h = 0xFFFFFFFFu, pw = 0;
          if (run >= k) {
            const uint32_t st = rev < fwd;
            h = fwd != rev ? hash32(st ? rev : fwd, mask2k) : 0xFFFFFFFFu;
            pw = static_cast<uint32_t>(s) << 1 | st;
          } else {
            lastbad = s;
          }
          cur_h[u] = h;
          cur_p[u] = pw;
          if (u == 0 || h < pre_h) {  // prefix of this block: ties keep the earlier
            pre_h = h;
            pre_p = pw;
          }
          // window [s - W + 1, s]: suffix of the previous block from u + 1 (to the left, so
          // it wins ties), prefix of this one
          uint32_t m_h = pre_h, m_p = pre_p;
          if (u + 1 < W && !(pre_h < suf_h[u + 1 < W ? u + 1 : 0])) {
            m_h = suf_h[u + 1 < W ? u + 1 : 0];
            m_p = suf_p[u + 1 < W ? u + 1 : 0];
          }
          int arg = -1;
          if (s >= W - 1 && lastbad < s - W + 1 && m_h != 0xFFFFFFFFu) arg = static_cast<int>(m_p >> 1);
          // emission as predicated stores and an add, not a branch per position
          const bool emit = arg >= 0 && arg != prev_arg;
          uint32_t* const slot = cbw + 2 * min(nmin, kTMaxMin - 1) * TT;
          if (emit && nmin < kTMaxMin) {
            slot[0] = m_h;
            slot[TT] = static_cast<uint32_t>(arg) | (m_p & 1u) << 31;
          }
          nmin += emit ? 1 : 0;
          prev_arg = arg;
        }
      }
      // suffix minima of this block for the next one (ties keep the earlier)
      suf_h[W - 1] = cur_h[W - 1];
      suf_p[W - 1] = cur_p[W - 1];
#pragma unroll
      for (int u = W - 2; u >= 0; --u) {
        const bool left = cur_h[u] <= suf_h[u + 1];
        suf_h[u] = left ? cur_h[u] : suf_h[u + 1];
        suf_p[u] = left ? cur_p[u] : suf_p[u + 1];
      }
    }
    if (nmin > kTMaxMin) big = true;
  }

  // ---- probe and anchors (src/mapper.cpp:16-40); region A becomes the anchor keys
  int na = 0;
  if (!big) {
    for (int j0 = 0; j0 < nmin && !big; j0 += kProbe) {
      // kProbe keys walk the table (src/index.hpp:24-38) in lockstep rounds: each round
      // loads the next bucket of every key still unresolved, as independent loads, so
      // colliding keys cost the longest chain of the group, not the sum of the chains.
      uint2 m[kProbe];
      ulonglong2 bk[kProbe];
      uint64_t slot[kProbe];
      uint32_t pending = 0;
#pragma unroll
      for (int q = 0; q < kProbe; ++q) {
        m[q] = make_uint2(0, 0);
        bk[q] = make_ulonglong2(kInvalidHash, 0);
        slot[q] = 0;
        if (j0 + q < nmin) {
          m[q] = make_uint2(cbw[2 * (j0 + q) * TT], cbw[(2 * (j0 + q) + 1) * TT]);
          slot[q] = static_cast<uint64_t>(m[q].x) & ix.mask;
          bk[q] = __ldg(ix.table + slot[q]);
          pending |= 1u << q;
        }
      }
      uint32_t off[kProbe], cnt[kProbe], v0[kProbe];
#pragma unroll
      for (int q = 0; q < kProbe; ++q) off[q] = cnt[q] = 0;
      for (uint64_t round = 0; pending; ++round) {
        if (round > ix.mask) {  // the table is at most half full: an empty bucket ends every walk
          atomicOr(err, kErrProbeLoop);
          break;
        }
        uint32_t next = 0;
#pragma unroll
        for (int q = 0; q < kProbe; ++q) {
          if ((pending >> q) & 1u) {
            if (bk[q].x == static_cast<uint64_t>(m[q].x)) {
              off[q] = static_cast<uint32_t>(bk[q].y);
              cnt[q] = static_cast<uint32_t>(bk[q].y >> 32);
            } else if (bk[q].x != kInvalidHash) {
              slot[q] = (slot[q] + 1) & ix.mask;
              next |= 1u << q;
            }
          }
        }
#pragma unroll
        for (int q = 0; q < kProbe; ++q)
          if ((next >> q) & 1u) bk[q] = __ldg(ix.table + slot[q]);
        pending = next;
      }
#pragma unroll
      for (int q = 0; q < kProbe; ++q) {
        if (cnt[q] > sp.max_occ) cnt[q] = 0;
        v0[q] = cnt[q] ? __ldg(ix.positions + off[q]) : 0u;
      }
#pragma unroll
      for (int q = 0; q < kProbe; ++q) {
        if (j0 + q >= nmin || big) break;
        if (na + static_cast<int>(cnt[q]) > kTMaxAnc) {
          big = true;
          break;
        }
        const int32_t pos = static_cast<int32_t>(m[q].y & 0x7FFFFFFFu);
        const uint32_t mst = m[q].y >> 31;
        const auto anchor = [&](uint32_t v) {
          const uint32_t rv = (v & 1u) ^ mst;
          const int32_t qpos = rv ? len - pos - k : pos;
          a_hi(na) = rv << 31 | v >> 1;
          a_lo(na) = static_cast<uint32_t>(qpos);
        };
        // the first occurrence (most keys have one) with predicated stores, the rest in a loop
        if (cnt[q] > 0) anchor(v0[q]);
        na += cnt[q] > 0 ? 1 : 0;
        for (uint32_t t = 1; t < cnt[q]; ++t) {
          anchor(__ldg(ix.positions + off[q] + t));
          ++na;
        }
      }
    }
  }

  int nd = 0;
  if (!big && na > 0) {
    // ---- sort the anchor keys ascending (src/chain.cpp:16-20; keys are unique)
    if (key_ld(0) > key_ld(na - 1)) {
      for (int a = 0, b2 = na - 1; a < b2; ++a, --b2) {
        const uint64_t x = key_ld(a);
        key_st(a, key_ld(b2));
        key_st(b2, x);
      }
    }
    for (int i = 1; i < na; ++i) {
      const uint64_t x = key_ld(i);
      int j = i - 1;
      while (j >= 0) {
        const uint64_t y = key_ld(j);
        if (y <= x) break;
        key_st(j + 1, y);
        --j;
      }
      key_st(j + 1, x);
    }
    // ---- DP (src/chain.cpp:22-45); region B becomes the DP words
    // A predecessor j' <= j scores at most max(f[0..j]) + k (gain <= k, cost >= 0), so once
    // that is <= best no remaining candidate can win the strict '>': the scan stops there
    // with the reference's result. On colinear chains this ends it after a step or two.
    const uint32_t max_gap = static_cast<uint32_t>(cp.max_gap);
    int pm = 0;
    for (int i = 0; i < na; ++i) {
      const uint32_t hi_i = a_hi(i);
      const int32_t qi = static_cast<int32_t>(a_lo(i));
      int best = k, bj = -1;
      const int lo = i - cp.lookback > 0 ? i - cp.lookback : 0;
      for (int j = i - 1; j >= lo; --j) {
        const uint32_t wj = fp_at(j);
        if (static_cast<int>(wj >> 20) + k <= best) break;
        const uint32_t hi_j = a_hi(j);
        if ((hi_i ^ hi_j) >> 31) break;  // strand change
        const uint32_t dr = hi_i - hi_j;  // same strand, sorted: rpos_i - rpos_j >= 0
        if (dr > max_gap) break;
        const int32_t dq = qi - static_cast<int32_t>(a_lo(j));
        // the rest as selects (the pairs a warp's reads skip differ): a skipped pair still
        // reads the gap table, at an index clamped to the band
        const int32_t dri = static_cast<int32_t>(dr);  // <= max_gap < 2^29
        const int32_t dd = dri > dq ? dri - dq : dq - dri;
        const bool ok = dr != 0 && dq > 0 && dd <= cp.band;
        int g = dq < dri ? dq : dri;
        if (g > k) g = k;
        const int sc = f_of(wj) + g - lut[dd < cp.band ? dd : cp.band];
        const bool up = ok && sc > best;
        best = up ? sc : best;
        bj = up ? j : bj;
      }
      pm = best > pm ? best : pm;
      fp_at(i) = static_cast<uint32_t>(bj + 1) | static_cast<uint32_t>(best) << 8 | static_cast<uint32_t>(pm) << 20;
    }
    // ---- chains (src/chain.cpp:47-68)
    uint32_t used = 0;
    int nch = 0;
    for (;;) {
      int end = -1, bf = INT_MIN;
      for (int i = 0; i < na; ++i) {
        const int f = f_of(fp_at(i));
        if (!((used >> i) & 1u) && f > bf) {
          bf = f;
          end = i;
        }
      }
      if (end < 0) break;
      int i = end, cnt = 0;
      int32_t dmin = INT_MAX, dmax = INT_MIN;
      while (i >= 0 && !((used >> i) & 1u)) {
        used |= 1u << i;
        ++cnt;
        const int32_t d = static_cast<int32_t>(a_hi(i) & 0x7FFFFFFFu) - static_cast<int32_t>(a_lo(i));
        dmin = d < dmin ? d : dmin;
        dmax = d > dmax ? d : dmax;
        i = static_cast<int>(fp_at(i) & 0xFFu) - 1;
      }
      const int score = bf - (i >= 0 ? f_of(fp_at(i)) : 0);
      if (score < cp.min_score || cnt < cp.min_anchors) continue;
      if (nch == kTMaxChains) {
        big = true;
        break;
      }
      const uint32_t he = a_hi(end);
      ch_at(0, nch) = score;
      ch_at(1, nch) = static_cast<int32_t>(he >> 31);
      ch_at(2, nch) = static_cast<int32_t>(dmin + (static_cast<int64_t>(dmax) - dmin) / 2);  // no int32 overflow
      ch_at(3, nch) = static_cast<int32_t>(he & 0x7FFFFFFFu);
      ++nch;
    }
    // ---- candidate loci (src/mapper.cpp:40-62), chains by (score desc, extraction order)
    if (!big && nch > 0) {
      const int64_t cbase = r * cand.max_cand;
      int last_s = INT_MAX, last_i = -1;
      double min_score = 0.0;
      for (int c = 0; c < nch; ++c) {
        int bi = -1, bs = INT_MIN;
        for (int x = 0; x < nch; ++x) {
          const int s = ch_at(0, x);
          if ((s < last_s || (s == last_s && x > last_i)) && s > bs) {
            bs = s;
            bi = x;
          }
        }
        last_s = bs;
        last_i = bi;
        if (c == 0) min_score = static_cast<double>(bs) * cand.pri_ratio;
        if (static_cast<double>(bs) < min_score || nd >= cand.max_cand) break;
        const uint8_t strand = static_cast<uint8_t>(ch_at(1, bi));
        const int64_t diag = ch_at(2, bi);
        bool dup = false;
        for (int x = 0; x < nd && !dup; ++x) {
          const int64_t dd = cb.diag[cbase + x] - diag;
          dup = cb.rev[cbase + x] == strand && (dd < 0 ? -dd : dd) <= cand.bw;
        }
        if (dup) continue;
        cb.rev[cbase + nd] = strand;
        cb.contig[cbase + nd] = contig_of(ix, static_cast<uint32_t>(ch_at(3, bi)));
        cb.diag[cbase + nd] = diag;
        cb.wstart[cbase + nd] = diag - cand.bw;
        ++nd;
      }
    }
  }
  n_anchor[r] = 0;  // no anchor scratch: this read either finished here or is listed below
  if (big) {
    n_min[r] = 0;
    n_anc_t[r] = 0;
    big_list[atomicAdd(big_n, 1)] = static_cast<int32_t>(r);
    return;
  }
  n_min[r] = nmin;
  n_anc_t[r] = na;
  cb.n_cand[r] = nd;
}

template <int TT>
bool launch_thread_tt(cudaStream_t st, const uint8_t* codes, const int64_t* pofs,
                      const int32_t* seq_len, int64_t n, const DevIndex& ix, const SeedParams& sp,
                      const ChainParamsDev& cp, const CandParams& cand, CandBuf cb, int32_t* n_min, int64_t* n_anchor,
                      int32_t* n_anc_t, int32_t* big_list, int* big_n, uint32_t* err) {
  static std::atomic<bool> attr_set[kMaxDevices];
  if (!set_smem_limit_once(k_seed_chain_t<kTW, TT>, TLayout<TT>::kSmem, attr_set)) return false;
  const int64_t blocks = (n + TT - 1) / TT;
  k_seed_chain_t<kTW, TT><<<static_cast<unsigned>(blocks), TT, TLayout<TT>::kSmem, st>>>(
      codes, pofs, seq_len, n, ix, sp, cp, cand, cb, n_min, n_anchor, n_anc_t, big_list, big_n, err);
  return true;
}

}  // namespace

int seed_thread_max_len() { return kTMaxLen; }

bool seed_thread_supported(const SeedParams& sp, const ChainParamsDev& cp) {
  return sp.w == kTW && sp.k >= 4 && sp.k <= 15 && cp.max_gap >= 0 && cp.max_gap < (1 << 29) && cp.band >= 0 &&
         cp.band <= kTMaxBand && cp.lookback >= 0;
}

void launch_encode_reads(cudaStream_t st, const char* seq, const int64_t* seq_off, int64_t seq_base,
                         const int32_t* seq_len, const int64_t* pofs, int64_t n, uint8_t* codes) {
  if (n <= 0) return;
  const int64_t blocks = std::min<int64_t>((n + 7) / 8, int64_t{16} * device_sm_count());  // 8 warps a block, grid-stride
  k_encode_reads<<<static_cast<unsigned>(blocks), 256, 0, st>>>(seq, seq_off, seq_base, seq_len, pofs, n, codes);
}

bool launch_seed_chain_thread(cudaStream_t st, const uint8_t* codes, const int64_t* pofs,
                              const int32_t* seq_len, int64_t n, const DevIndex& ix, const SeedParams& sp,
                              const ChainParamsDev& cp,
                              const CandParams& cand, CandBuf cb, int32_t* n_min, int64_t* n_anchor,
                              int32_t* n_anc_t, int32_t* big_list, int* big_n, uint32_t* err, int reads_per_block) {
  if (!seed_thread_supported(sp, cp)) return false;
  if (n <= 0) return true;
  if (reads_per_block == 64)
    return launch_thread_tt<64>(st, codes, pofs, seq_len, n, ix, sp, cp, cand, cb, n_min, n_anchor, n_anc_t,
                                big_list, big_n, err);
  if (reads_per_block == 128)
    return launch_thread_tt<128>(st, codes, pofs, seq_len, n, ix, sp, cp, cand, cb, n_min, n_anchor,
                                 n_anc_t, big_list, big_n, err);
  return false;
}

}  // namespace dnb
