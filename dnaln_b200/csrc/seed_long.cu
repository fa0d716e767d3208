// seed_long.cu — one thread per long read: sketch, probe, anchors, chaining DP, chain
// extraction and candidate loci of the reads the short thread-per-read kernel
// (seed_thread.cu) listed, with each read's state in global memory.
//
// The short kernel keeps a read's whole state in 512 bytes of shared memory, which bounds
// it to 256 bp, 32 minimizers and 32 anchors. Reads past that (long reads, or reads whose
// minimizers hit a repeat a few times) used to go one warp per read, where every DP row
// evaluates 64 candidate predecessors and every sort is a bitonic network — about 20,000
// warp instructions for a read of 80 anchors. Here one thread runs the reference's
// sequential algorithms with the short kernel's shortcuts (prefix-max cutoff of the
// predecessor scan, insertion sort after putting the dominant direction first), the
// listed reads sorted by length so that the 32 reads of a warp advance in near lockstep.
// Per-thread state lives in global memory in column layout (word e of thread t at
// e * stride + t), so a warp's lockstep access to word e is one 128-byte line.
//
// Only reads longer than min_len (the short kernel's length bound) are taken: a short read
// is listed because a repeat gave it many anchors, and those sets, out of order and dense,
// are what the warp kernels' parallel sort and DP are good at.
//
// Bounds: 256 minimizers, 256 anchors, 32 kept chains, and budgets on the insertion sort
// (moves) and on the chain extraction (scan steps) that only repeat-rich anchor sets
// reach. A read past any of them is appended to the next list, for the warp-per-read
// kernels (seed.cu), which recompute it from scratch — same results on every path.
#include "common.cuh"
#include "seed.cuh"

namespace dnb {

namespace {

constexpr int kLT = 128;          // threads per block
constexpr int kLBlocksPerSm = 8;  // blocks per SM the grid is sized for: 6 resident (80 registers), then the rest
constexpr int kLMaxMin = 256;
constexpr int kLMaxAnc = 256;
constexpr int kLMaxChains = 32;
constexpr int kLMaxBand = 256;    // chaining band of the shared gap-cost table
// column words per thread: A = anchor keys (hi, lo); B = minimizer slots (hash, pos |
// strand << 31), later the DP words (f | maxf << 16, prev + 1) and the chain table;
// U = used bits of the anchors
constexpr int kLWordsA = 2 * kLMaxAnc;
constexpr int kLWordsB = 2 * kLMaxAnc + 4 * kLMaxChains + kLMaxAnc;  // DP words, chains, extraction order
constexpr int kLWordsU = kLMaxAnc / 32;
static_assert(2 * kLMaxMin <= kLWordsB, "minimizer slots must fit region B");
constexpr int kLWords = kLWordsA + kLWordsB + kLWordsU;

// Sort keys of the listed reads, longest first; slots at or past the device count last.
// Keys are top - length with top = 2^bits - 1 (every length of the batch at most top), the
// empty slots 2^bits: a sort over bits + 1 key bits.
__global__ void k_long_keys(const int32_t* __restrict__ list, const int* __restrict__ list_n, int n_max,
                            const int32_t* __restrict__ seq_len, uint32_t top, uint32_t* __restrict__ keys,
                            int32_t* __restrict__ vals) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_max) return;
  const int m = *list_n;
  if (x < m) {
    const int32_t r = list[x];
    const uint32_t len = static_cast<uint32_t>(seq_len[r]);
    keys[x] = len < top ? top - len : 0u;  // a length past top (not expected) still sorts first
    vals[x] = r;
  } else {
    keys[x] = top + 1u;
    vals[x] = -1;
  }
}

template <int W>
__global__ void __launch_bounds__(kLT, 6)
    k_seed_chain_tl(const int32_t* __restrict__ seq_len, const int64_t* __restrict__ pofs,
                    const uint8_t* __restrict__ codes, const int32_t* __restrict__ list, const int* __restrict__ list_n,
                    DevIndex ix, SeedParams sp, ChainParamsDev cp, CandParams cand, CandBuf cb,
                    int32_t* __restrict__ n_min, int64_t* __restrict__ n_anchor, int32_t* __restrict__ n_anc_t,
                    uint32_t* __restrict__ scratch, int32_t* __restrict__ next_list, int* __restrict__ next_n,
                    int min_len, uint32_t* __restrict__ err) {
  __shared__ int32_t lut[kLMaxBand + 1];
  for (int d = threadIdx.x; d <= cp.band; d += kLT) lut[d] = cp.cost[d];
  __syncthreads();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * kLT;
  const int64_t tid = static_cast<int64_t>(blockIdx.x) * kLT + threadIdx.x;
  uint32_t* const colA = scratch + tid;
  uint32_t* const colB = scratch + kLWordsA * stride + tid;
  uint32_t* const colU = scratch + (kLWordsA + kLWordsB) * stride + tid;
  const auto A = [&](int e) -> uint32_t& { return colA[e * stride]; };
  const auto B = [&](int e) -> uint32_t& { return colB[e * stride]; };
  const auto key_ld = [&](int a) { return static_cast<uint64_t>(A(2 * a)) << 32 | A(2 * a + 1); };
  const auto key_st = [&](int a, uint64_t v) {
    A(2 * a) = static_cast<uint32_t>(v >> 32);
    A(2 * a + 1) = static_cast<uint32_t>(v);
  };
  // DP words of anchor i: B(2i) = f | max(f[0..i]) << 16, B(2i+1) = prev + 1 (f <= 15 * 256)
  const auto ch_at = [&](int field, int c) -> int32_t& {
    return reinterpret_cast<int32_t&>(B(2 * kLMaxAnc + field * kLMaxChains + c));
  };
  const int m_list = *list_n;
  const int k = sp.k;
  // The grid is more blocks than are resident: the first wave takes the longest reads of
  // the (longest-first) list, and the later blocks start as the first's finish. A thread
  // with more than one read takes them in serpentine order: round j takes positions
  // [j*stride, (j+1)*stride), forward on even rounds and reversed on odd ones, so the
  // thread with the longest read of one round gets the shortest of the next. Nothing in
  // the loop synchronises the lanes of a warp, so a lane runs its reads back to back:
  // taking work by warp-wide atomic claims instead (a shuffle per claim) made the lanes
  // reconverge every round and measured 2.35x slower (4.65 against 1.98 ms per batch).
  for (int64_t round = 0;; ++round) {
    const int64_t x = (round & 1) ? (round + 1) * stride - 1 - tid : round * stride + tid;
    if (x >= m_list) break;  // every later round's position is further still
    const int64_t r = list[x];
    const int len = seq_len[r];
    if (len <= min_len) {  // listed for its anchors, not its length: the warp kernels are faster there
      next_list[atomicAdd(next_n, 1)] = static_cast<int32_t>(r);
      continue;
    }
    const uint8_t* fw = codes + 2 * pofs[r];
    bool big = false;
    int nmin = 0;
    // ---- sketch (src/minimizer.cpp:5-68): as the short kernel, codes read from HBM
    if (len >= k) {
      const uint32_t mask2k = (1u << (2 * k)) - 1u;
      const int nk = len - k + 1;
      uint32_t fwd = 0, rev = 0;
      int run = 0;
      // codes in order, four per aligned 32-bit load (the words before the read's first and
      // after its last code lie in the codes buffer: the reverse strand follows each read)
      const uint32_t* wp = reinterpret_cast<const uint32_t*>(reinterpret_cast<uintptr_t>(fw) & ~uintptr_t(3));
      uint32_t wsh = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(fw) & 3u) * 8u;
      uint32_t wcur = __ldg(wp);
      auto roll = [&](int) {  // consumes the next code
        const uint32_t c = (wcur >> wsh) & 0xFFu;
        wsh += 8u;
        if (wsh == 32u) {
          wsh = 0u;
          wcur = __ldg(++wp);
        }
        run = c < 4 ? run + 1 : 0;
        fwd = ((fwd << 2) | (c & 3u)) & mask2k;
        rev = (rev >> 2) | ((3u - (c & 3u)) << (2 * k - 2));
      };
      for (int i = 0; i < k - 1; ++i) roll(i);
      // window minimum over (hash, pos << 1 | strand) pairs by 32-bit hash compares, ties to
      // the left operand, the earlier position (hashes < 2^(2k), invalid ones ~0)
      uint32_t cur_h[W], cur_p[W], suf_h[W], suf_p[W];
#pragma unroll
      for (int u = 0; u < W; ++u) {
        suf_h[u] = 0xFFFFFFFFu;
        suf_p[u] = 0;
      }
      uint32_t pre_h = 0xFFFFFFFFu, pre_p = 0;
      int lastbad = -1, prev_arg = -1;
      for (int s0 = 0; s0 < nk && !big; s0 += W) {
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
            if (u == 0 || h < pre_h) {
              pre_h = h;
              pre_p = pw;
            }
            uint32_t m_h = pre_h, m_p = pre_p;
            if (u + 1 < W && !(pre_h < suf_h[u + 1 < W ? u + 1 : 0])) {
              m_h = suf_h[u + 1 < W ? u + 1 : 0];
              m_p = suf_p[u + 1 < W ? u + 1 : 0];
            }
            int arg = -1;
            if (s >= W - 1 && lastbad < s - W + 1 && m_h != 0xFFFFFFFFu) arg = static_cast<int>(m_p >> 1);
            const bool emit = arg >= 0 && arg != prev_arg;  // predicated, not a branch
            if (emit && nmin < kLMaxMin) {
              B(2 * nmin) = m_h;
              B(2 * nmin + 1) = static_cast<uint32_t>(arg) | (m_p & 1u) << 31;
            }
            nmin += emit ? 1 : 0;
            prev_arg = arg;
          }
        }
        suf_h[W - 1] = cur_h[W - 1];
        suf_p[W - 1] = cur_p[W - 1];
#pragma unroll
        for (int u = W - 2; u >= 0; --u) {
          const bool left = cur_h[u] <= suf_h[u + 1];
          suf_h[u] = left ? cur_h[u] : suf_h[u + 1];
          suf_p[u] = left ? cur_p[u] : suf_p[u + 1];
        }
        if (nmin > kLMaxMin) big = true;
      }
    }
    // ---- probe and anchors (src/mapper.cpp:16-40)
    int na = 0;
    constexpr int kP = 4;  // keys probed at once: four keep the kernel at 6 blocks per SM
    for (int j0 = 0; j0 < nmin && !big; j0 += kP) {
      uint32_t mh[kP], mp[kP];
      ulonglong2 bk[kP];
      uint64_t slot[kP];
      uint32_t pending = 0;
#pragma unroll
      for (int q = 0; q < kP; ++q) {
        mh[q] = mp[q] = 0;
        bk[q] = make_ulonglong2(kInvalidHash, 0);
        slot[q] = 0;
        if (j0 + q < nmin) {
          mh[q] = B(2 * (j0 + q));
          mp[q] = B(2 * (j0 + q) + 1);
          slot[q] = static_cast<uint64_t>(mh[q]) & ix.mask;
          bk[q] = __ldg(ix.table + slot[q]);
          pending |= 1u << q;
        }
      }
      uint32_t off[kP], cnt[kP];
#pragma unroll
      for (int q = 0; q < kP; ++q) off[q] = cnt[q] = 0;
      for (uint64_t round = 0; pending; ++round) {
        if (round > ix.mask) {
          atomicOr(err, kErrProbeLoop);
          break;
        }
        uint32_t next = 0;
#pragma unroll
        for (int q = 0; q < kP; ++q) {
          if ((pending >> q) & 1u) {
            if (bk[q].x == static_cast<uint64_t>(mh[q])) {
              off[q] = static_cast<uint32_t>(bk[q].y);
              cnt[q] = static_cast<uint32_t>(bk[q].y >> 32);
            } else if (bk[q].x != kInvalidHash) {
              slot[q] = (slot[q] + 1) & ix.mask;
              next |= 1u << q;
            }
          }
        }
#pragma unroll
        for (int q = 0; q < kP; ++q)
          if ((next >> q) & 1u) bk[q] = __ldg(ix.table + slot[q]);
        pending = next;
      }
      // first occurrences of the group's keys as independent loads; each key's first anchor
      // through predicated stores, the further ones in a loop
      uint32_t v0[kP];
#pragma unroll
      for (int q = 0; q < kP; ++q) {
        if (cnt[q] > sp.max_occ) cnt[q] = 0;
        v0[q] = j0 + q < nmin && cnt[q] ? __ldg(ix.positions + off[q]) : 0u;
      }
      for (int q = 0; q < kP && !big; ++q) {
        if (j0 + q >= nmin) break;
        const uint32_t c = cnt[q];
        if (na + static_cast<int>(c) > kLMaxAnc) {
          big = true;
          break;
        }
        const int32_t pos = static_cast<int32_t>(mp[q] & 0x7FFFFFFFu);
        const uint32_t mst = mp[q] >> 31;
        const auto anchor = [&](uint32_t v) {
          const uint32_t rv = (v & 1u) ^ mst;
          const int32_t qpos = rv ? len - pos - k : pos;
          A(2 * na) = rv << 31 | v >> 1;
          A(2 * na + 1) = static_cast<uint32_t>(qpos);
        };
        if (c > 0) anchor(v0[q]);
        na += c > 0 ? 1 : 0;
        for (uint32_t t = 1; t < c; ++t) {
          anchor(__ldg(ix.positions + off[q] + t));
          ++na;
        }
      }
    }
    int nd = 0;
    if (!big && na > 0) {
      // ---- sort the anchor keys ascending (src/chain.cpp:16-20; keys are unique): the
      // dominant direction first (a reverse-strand read's anchors arrive descending), then
      // insertion sort within a budget of moves that colinear sets never reach
      int desc = 0;
      uint64_t kprev = key_ld(0);
      for (int a = 1; a < na; ++a) {
        const uint64_t kc = key_ld(a);
        desc += kc < kprev;
        kprev = kc;
      }
      if (2 * desc > na - 1) {
        for (int a = 0, b2 = na - 1; a < b2; ++a, --b2) {
          const uint64_t t0 = key_ld(a);
          key_st(a, key_ld(b2));
          key_st(b2, t0);
        }
      }
      // The key at position i-1 is kept in a register and key i+1 is loaded while key i is
      // placed: an anchor already in order costs no wait.
      int budget = 8 * na + 64;
      uint64_t last = key_ld(0), v_next = na > 1 ? key_ld(1) : 0;
      for (int i = 1; i < na && !big; ++i) {
        const uint64_t v = v_next;
        if (i + 1 < na) v_next = key_ld(i + 1);
        if (last <= v) {  // in place
          last = v;
          continue;
        }
        key_st(i, last);  // the key at i-1 moves up; it is the key at i from here on
        int j = i - 2;
        if (--budget >= 0) {
          while (j >= 0) {
            const uint64_t y = key_ld(j);
            if (y <= v) break;
            key_st(j + 1, y);
            --j;
            if (--budget < 0) break;
          }
        }
        key_st(j + 1, v);
        if (budget < 0) big = true;
      }
    }
    if (!big && na > 0) {
      // ---- DP (src/chain.cpp:22-45) with the prefix-max cutoff: a predecessor j' <= j
      // scores at most max(f[0..j]) + k, so the scan stops once that cannot beat best
      // Anchors i-1 and i-2 (key words and DP word) stay in registers and anchor i+1's
      // key is loaded while row i runs: with the cutoff the scan rarely reaches farther,
      // so a row waits on no load of its own.
      const uint32_t max_gap = static_cast<uint32_t>(cp.max_gap);
      int pm = 0;
      uint32_t h1 = 0, q1 = 0, w1 = 0, h2 = 0, q2 = 0, w2 = 0;
      uint32_t h_next = A(0), q_next = A(1);
      for (int i = 0; i < na; ++i) {
        const uint32_t hi_i = h_next;
        const int32_t qi = static_cast<int32_t>(q_next);
        if (i + 1 < na) {
          h_next = A(2 * (i + 1));
          q_next = A(2 * (i + 1) + 1);
        }
        int best = k, bj = -1;
        const int lo = i - cp.lookback > 0 ? i - cp.lookback : 0;
        for (int j = i - 1; j >= lo; --j) {
          const bool r1 = j == i - 1, r2 = j == i - 2;
          const uint32_t wj = r1 ? w1 : (r2 ? w2 : B(2 * j));
          if (static_cast<int>(wj >> 16) + k <= best) break;
          const uint32_t hi_j = r1 ? h1 : (r2 ? h2 : A(2 * j));
          if ((hi_i ^ hi_j) >> 31) break;  // strand change
          const uint32_t dr = hi_i - hi_j;
          if (dr > max_gap) break;
          const int32_t dq = qi - static_cast<int32_t>(r1 ? q1 : (r2 ? q2 : A(2 * j + 1)));
          // the rest as selects (a skipped pair reads the gap table at an index clamped to
          // the band)
          const int32_t dri = static_cast<int32_t>(dr);
          const int32_t dd = dri > dq ? dri - dq : dq - dri;
          const bool ok = dr != 0 && dq > 0 && dd <= cp.band;
          int g = dq < dri ? dq : dri;
          if (g > k) g = k;
          const int sc = static_cast<int>(wj & 0xFFFFu) + g - lut[dd < cp.band ? dd : cp.band];
          const bool up = ok && sc > best;
          best = up ? sc : best;
          bj = up ? j : bj;
        }
        pm = best > pm ? best : pm;
        const uint32_t wi = static_cast<uint32_t>(best) | static_cast<uint32_t>(pm) << 16;
        B(2 * i) = wi;
        B(2 * i + 1) = static_cast<uint32_t>(bj + 1);
        h2 = h1;
        q2 = q1;
        w2 = w1;
        h1 = hi_i;
        q1 = static_cast<uint32_t>(qi);
        w1 = wi;
      }
      // ---- chains (src/chain.cpp:47-68): walks from each anchor in (f desc, index asc)
      // order, skipping used ones. The order is sorted by insertion after reversing
      // (f rises along a chain, so index order is close to the reverse of f desc), within
      // a budget of moves
      const auto ord = [&](int e) -> uint32_t& { return B(2 * kLMaxAnc + 4 * kLMaxChains + e); };
      for (int i = 0; i < na; ++i)
        ord(na - 1 - i) = (0xFFFu - (B(2 * i) & 0xFFFu)) << 16 | static_cast<uint32_t>(i);
      int budget2 = 8 * na + 64;  // the same register-cached insertion as the key sort
      uint32_t olast = ord(0), o_next = na > 1 ? ord(1) : 0u;
      for (int i = 1; i < na && !big; ++i) {
        const uint32_t v = o_next;
        if (i + 1 < na) o_next = ord(i + 1);
        if (olast <= v) {
          olast = v;
          continue;
        }
        ord(i) = olast;
        int j = i - 2;
        if (--budget2 >= 0) {
          while (j >= 0) {
            const uint32_t y = ord(j);
            if (y <= v) break;
            ord(j + 1) = y;
            --j;
            if (--budget2 < 0) break;
          }
        }
        ord(j + 1) = v;
        if (budget2 < 0) big = true;
      }
      for (int u = 0; u < (na + 31) / 32; ++u) colU[u * stride] = 0;
      int nch = 0;
      for (int e = 0; e < na && !big; ++e) {
        const int end = static_cast<int>(ord(e) & 0xFFFFu);
        if ((colU[(end >> 5) * stride] >> (end & 31)) & 1u) continue;
        const int bf = static_cast<int>(B(2 * end) & 0xFFFFu);
        int i = end, cnt = 0;
        int32_t dmin = INT_MAX, dmax = INT_MIN;
        while (i >= 0 && !((colU[(i >> 5) * stride] >> (i & 31)) & 1u)) {
          colU[(i >> 5) * stride] |= 1u << (i & 31);
          ++cnt;
          const int32_t d = static_cast<int32_t>(A(2 * i) & 0x7FFFFFFFu) - static_cast<int32_t>(A(2 * i + 1));
          dmin = d < dmin ? d : dmin;
          dmax = d > dmax ? d : dmax;
          i = static_cast<int>(B(2 * i + 1)) - 1;
        }
        const int score = bf - (i >= 0 ? static_cast<int>(B(2 * i) & 0xFFFFu) : 0);
        if (score < cp.min_score || cnt < cp.min_anchors) continue;
        if (nch == kLMaxChains) {
          big = true;
          break;
        }
        const uint32_t he = A(2 * end);
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
          for (int y = 0; y < nch; ++y) {
            const int s = ch_at(0, y);
            if ((s < last_s || (s == last_s && y > last_i)) && s > bs) {
              bs = s;
              bi = y;
            }
          }
          last_s = bs;
          last_i = bi;
          if (c == 0) min_score = static_cast<double>(bs) * cand.pri_ratio;
          if (static_cast<double>(bs) < min_score || nd >= cand.max_cand) break;
          const uint8_t strand = static_cast<uint8_t>(ch_at(1, bi));
          const int64_t diag = ch_at(2, bi);
          bool dup = false;
          for (int y = 0; y < nd && !dup; ++y) {
            const int64_t dd = cb.diag[cbase + y] - diag;
            dup = cb.rev[cbase + y] == strand && (dd < 0 ? -dd : dd) <= cand.bw;
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
    n_anchor[r] = 0;
    if (big) {
      n_min[r] = 0;
      n_anc_t[r] = 0;
      next_list[atomicAdd(next_n, 1)] = static_cast<int32_t>(r);
      continue;
    }
    n_min[r] = nmin;
    n_anc_t[r] = na;
    cb.n_cand[r] = nd;
  }
}

}  // namespace

bool seed_long_supported(const SeedParams& sp, const ChainParamsDev& cp) {
  return sp.w == 10 && sp.k >= 4 && sp.k <= 15 && cp.max_gap >= 0 && cp.max_gap < (1 << 29) && cp.band >= 0 &&
         cp.band <= kLMaxBand && cp.lookback >= 0;
}

int64_t seed_long_threads(int64_t n_max) {
  const int64_t cap = static_cast<int64_t>(device_sm_count()) * kLBlocksPerSm * kLT;
  const int64_t want = (n_max + kLT - 1) / kLT * kLT;
  return want < cap ? want : cap;
}

size_t seed_long_scratch_words(int64_t threads) { return static_cast<size_t>(threads) * kLWords; }

int launch_long_order(cudaStream_t st, const int32_t* list, const int* list_n, int n_max, const int32_t* seq_len,
                      int64_t max_len, uint32_t* keys, int32_t* vals) {
  int bits = 16;  // 16 bits cover reads up to 65,535 bp: two radix passes instead of four
  while (bits < 31 && max_len > (int64_t{1} << bits) - 1) ++bits;
  if (n_max > 0)
    k_long_keys<<<(n_max + 255) / 256, 256, 0, st>>>(list, list_n, n_max, seq_len, (1u << bits) - 1u, keys, vals);
  return bits + 1;
}

bool launch_seed_chain_long(cudaStream_t st, const int32_t* seq_len, const int64_t* pofs, const uint8_t* codes,
                            const int32_t* list, const int* list_n, int64_t threads, const DevIndex& ix,
                            const SeedParams& sp, const ChainParamsDev& cp, const CandParams& cand, CandBuf cb,
                            int32_t* n_min, int64_t* n_anchor, int32_t* n_anc_t, uint32_t* scratch,
                            int32_t* next_list, int* next_n, int min_len, uint32_t* err) {
  if (!seed_long_supported(sp, cp)) return false;
  if (threads <= 0) return true;
  const unsigned blocks = static_cast<unsigned>(threads / kLT);
  k_seed_chain_tl<10><<<blocks, kLT, 0, st>>>(seq_len, pofs, codes, list, list_n, ix, sp, cp, cand, cb, n_min,
                                              n_anchor, n_anc_t, scratch, next_list, next_n, min_len, err);
  return true;
}

}  // namespace dnb
