// sw.cu — banded affine-gap Smith–Waterman (score-only and with traceback) for sm_100a.
//
// The recurrence is the reference's diagonal-coordinate band (src/align.hpp:3-15,
// src/align.cpp:31-84): row i, band column d in [0, W), target column i+d,
//   hd = H(i-1,d) + s(q_i, t_{i+d})
//   E(i,d) = max(H(i-1,d+1) - (O+E), E(i-1,d+1) - E)
//   F(i,d) = max(H(i,d-1) - (O+E),   F(i,d-1) - E)
//   H(i,d) = max(hd, E(i,d), F(i,d), 0)
// with H = E = 0 for row -1 and for the fixed out-of-band cell d = W, F = H(left) = 0 at
// each row start, and the target N-padded to qlen + W - 1.
//
// Kernels (inter-sequence: a thread owns whole alignments, no intra-row shuffles):
//  * k_sw_u2<W>: two alignments per thread, one in each 16-bit half of 32-bit
//    registers, the band row (H, E of W+1 cells, W target selectors) in registers.
//    Values are kept biased by +16384, so every half stays positive and every add or
//    subtract of the recurrence is one 32-bit integer add on both halves (no borrow can
//    cross halves); E and F are DPX add-maxima (viaddmax), the other maxima unsigned 16x2
//    max (vmaxu2 / DPX vimax3_u16x2). The substitution scores of both alignments are one
//    prmt.b32 from an 8-byte per-row profile {s(qA, A..T) + 64, s(qB, A..T) + 64}.
//    Direction bits come from non-negative differences (hd vs max(hd, E), ...)
//    saturated to 0/1 with vminu2 and combined with integer multiply-adds.
//    With traceback it stores the direction codes and only the best cell; the walk is a
//    separate kernel (k_sw_walk, one thread per alignment, few registers, full occupancy)
//    so the DP kernel's register footprint does not carry the walk.
//  * A task whose target window may contain an N (the 4-entry profile cannot score it),
//    or whose scores or lengths do not fit the biased 16-bit range, is appended by
//    k_sw_u2 to a device-side list; k_sw_fb runs the same cell update in int32 for the
//    listed tasks (sw_one_reg), same outputs and codes. Genome windows that the task
//    builder marked N-free (kTaskNoN) skip the per-task N scan.
//  * k_sw_any: any band width and any scores (int32, band rows in per-warp scratch).
//
// Direction code of a cell (4 bits):
//   bit 3: hd < E            bit 2: max(hd, E) < F
//   bit 1: E extends E(i-1,d+1) (ee > eo)    bit 0: F extends F(i,d-1) (fe > fo)
// On every cell the walk reads, H is the positive value being traced; there "H from the
// diagonal" (h == hd, src/align.cpp:67) is bits 3,2 = 0,0, "H from E" with no diagonal
// (h == e) is 1,0, and otherwise H came from F — so the walk (src/align.cpp:87-143)
// takes the reference's steps. The best cell is the first strict maximum in row-major
// order (per-row maximum with its first column, then strict across rows).
#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "sw.cuh"

namespace dnb {

namespace {

constexpr int kSwThreads = 128;
constexpr uint32_t kNotDiagE = 8u, kFromF = 4u, kExtE = 2u, kExtF = 1u;
constexpr uint32_t kBias = 16384u, kBias2 = 0x40004000u, kOne2 = 0x00010001u;
constexpr int kScoreBias = 64;  // profile bytes are score + 64, in [0, 127]
constexpr int kAhead = 8;       // cells of a diagonal run the walk fetches at once

// prmt.b32 in its default mode (the sign-replicate bit of each selector nibble is
// honoured; the __byte_perm intrinsic uses only the low 3 bits of each nibble).
__device__ __forceinline__ uint32_t prmt(uint32_t lo, uint32_t hi, uint32_t sel) {
  uint32_t r;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(lo), "r"(hi), "r"(sel));
  return r;
}

// Selector of the sign-extended profile byte c (0..7) as one 32-bit value.
__device__ __forceinline__ uint32_t sel1(uint32_t c) {
  const uint32_t s = c | 8u;
  return c | (s << 4) | (s << 8) | (s << 12);
}

// Selector of two zero-extended 16-bit values: byte a (0..3) of the low profile word into
// the low half, byte b of the high word into the high half (the profile bytes are
// below 128, so the sign-replicating nibbles give zero high bytes).
__device__ __forceinline__ uint32_t sel2(uint32_t a, uint32_t b) {
  const uint32_t x = 4u + b;
  return a | ((a | 8u) << 4) | (x << 8) | ((x | 8u) << 12);
}

__device__ __forceinline__ uint32_t tcode(const uint8_t* __restrict__ tbase, const SwTask& tk, int64_t j) {
  const int64_t x = tk.t_start + j;
  if (x < tk.t_lo || x >= tk.t_hi) return 4;
  const uint32_t c = __ldg(tbase + x);
  return c > 3 ? 4u : c;
}

// Profile word of query code qc for the int32 path: byte t = match if t == qc else
// -mismatch; an N query row scores -ambig everywhere.
__device__ __forceinline__ uint32_t prof_lo(const SwParams& p, uint32_t qc) {
  if (qc > 3) return p.prof_n;
  const uint32_t mm = (static_cast<uint32_t>(static_cast<uint8_t>(-p.mismatch))) * 0x01010101u;
  const uint32_t sh = 8u * qc;
  return (mm & ~(0xFFu << sh)) | (static_cast<uint32_t>(static_cast<uint8_t>(p.match)) << sh);
}

// The same profile biased by +64 (every byte in [0, 127]) for the 16-bit path.
__device__ __forceinline__ uint32_t prof_biased(const SwParams& p, uint32_t qc) {
  if (qc > 3) return static_cast<uint32_t>(kScoreBias - p.ambig) * 0x01010101u;
  const uint32_t mm = static_cast<uint32_t>(kScoreBias - p.mismatch) * 0x01010101u;
  const uint32_t sh = 8u * qc;
  return (mm & ~(0xFFu << sh)) | (static_cast<uint32_t>(kScoreBias + p.match) << sh);
}

__device__ __forceinline__ uint32_t pack2(uint32_t v) { return (v & 0xFFFFu) * 0x10001u; }

__device__ __forceinline__ uint32_t dir_code32(bool hd_ge_e, bool m1_ge_f, bool e_not_ext, bool f_not_ext) {
  return (hd_ge_e ? 0u : kNotDiagE) | (m1_ge_f ? 0u : kFromF) | (e_not_ext ? 0u : kExtE) | (f_not_ext ? 0u : kExtF);
}

// Global store with an L2 evict-first policy: streaming data (the direction codes, read
// once by the walk) should not push the resident index out of L2.
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ void st_evict_first(uint32_t* p, uint32_t v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.b32 [%0], %1, %2;" ::"l"(p), "r"(v), "l"(pol) : "memory");
}

struct CigarWriter {
  uint32_t* out;
  int cap, n;
  uint32_t op;
  int len;
  __device__ void push(uint32_t o, int l) {
    if (o == op) {
      len += l;
      return;
    }
    flush();
    op = o;
    len = l;
  }
  __device__ void flush() {
    if (len) {
      if (n < cap) out[n] = static_cast<uint32_t>(len) << 4 | op;
      ++n;
    }
    len = 0;
  }
};

// Direction codes of the pair layout: word (i, g), g < WQ = ceil(W/4), holds cells 4g..4g+3
// of both alignments of a thread (A in the low 16 bits, B in the high 16), cell 4g+c at
// bits 4*(3-c) of its half; the 32 pairs of a warp are interleaved word by word.
struct PairCodes {
  const uint32_t* D;  // this pair's first word
  int WQ, half;
  __device__ uint32_t word(int i, int d) const { return D[(static_cast<size_t>(i) * WQ + (d >> 2)) * 32]; }
  __device__ int shift(int d) const { return 16 * half + 4 * (3 - (d & 3)); }
  __device__ uint32_t operator()(int i, int d) const { return (word(i, d) >> shift(d)) & 0xFu; }
};

// Direction codes of the generic kernel: word (i, w), w < WW = ceil(W/8), holds cells
// 8w..8w+7, cell 8w+c at bits 4c; 32 alignments of a warp interleaved word by word.
struct NibbleCodes {
  const uint32_t* D;
  int WW;
  __device__ uint32_t word(int i, int d) const { return D[(static_cast<size_t>(i) * WW + (d >> 3)) * 32]; }
  __device__ int shift(int d) const { return 4 * (d & 7); }
  __device__ uint32_t operator()(int i, int d) const { return (word(i, d) >> shift(d)) & 0xFu; }
};

// High bit of each byte of x set where that byte is zero, every other bit clear.
__device__ __forceinline__ uint64_t zero_bytes(uint64_t x) {
  constexpr uint64_t kLow7 = 0x7F7F7F7F7F7F7F7Full;
  return ~(((x & kLow7) + kLow7) | x | kLow7);
}

// The bytes p[0..7] as one little-endian word, from the aligned 8-byte word holding p[0]
// and, unless p is aligned, the next one. Each of the two holds at least one of the eight
// bytes asked for, so neither lies outside the pages those bytes are in.
__device__ __forceinline__ uint64_t load8u(const uint8_t* p) {
  static_assert(kAhead == 8, "one 8-byte word per block of the diagonal run");
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uint64_t* w = reinterpret_cast<const uint64_t*>(a & ~static_cast<uintptr_t>(7));
  const unsigned sh = static_cast<unsigned>(a & 7) * 8u;
  const uint64_t lo = __ldg(w);
  if (sh == 0) return lo;
  return (lo >> sh) | (__ldg(w + 1) << (64u - sh));
}

// Walks the direction codes back from (bi, bd) (src/align.cpp:87-143). CIGAR ops are
// written in walk order (last op first), adjacent equal ops merged as the reference's
// push() does. Guards flag, and never read, a cell outside the band.
template <class Codes>
__device__ void traceback(const Codes& code, int W, int bi, int bd, int best, const uint8_t* __restrict__ q,
                          const uint8_t* __restrict__ tbase, const SwTask& tk, const SwParams& p, SwResult& r,
                          uint32_t* __restrict__ cig, int cap, uint32_t* __restrict__ err) {
  CigarWriter cw{cig, cap, 0, 0xFu, 0};
  int i = bi, d = bd, v = best, nm = 0;
  const int smax = max(p.match, max(-p.mismatch, -p.ambig));  // the most one step can lower v
  if (d < 0 || d >= W) {
    atomicOr(err, kErrTracebackBounds);
    i = -1;
    v = 0;
  }
  for (;;) {
    int run = 0;
    uint32_t x = 0;
    if (i >= 0 && v > 0 && (d < 0 || d >= W)) {
      atomicOr(err, kErrTracebackBounds);
      break;
    }
    // Diagonal run. The next kAhead cells (i-k, d) are fetched together (codes, query and
    // target bases: independent loads, one memory latency per kAhead steps) and then
    // consumed in order exactly as the one-cell-at-a-time walk would.
    bool stop = false;
    while (!stop && i >= 0 && v > 0) {
      uint32_t cx[kAhead];
      int qa[kAhead], ta[kAhead];
      const int64_t x0 = tk.t_start + (i - (kAhead - 1)) + d;  // target of row i - 7
      if (i >= kAhead - 1 && x0 >= tk.t_lo && x0 + kAhead <= tk.t_hi) {
        // the block's 8 query and 8 target bytes are contiguous: two 8-byte words each
        // instead of 16 byte loads (the walk is bound by its L1 requests)
        const uint64_t qw = load8u(q + i - (kAhead - 1)), tw = load8u(tbase + x0);
        uint32_t wk[kAhead], any = 0;
#pragma unroll
        for (int k = 0; k < kAhead; ++k) {
          wk[k] = code.word(i - k, d);
          any |= wk[k];
        }
        const int sh = code.shift(d);
        // A block that is diagonal throughout, with v > 0 before each of its steps (each
        // step lowers v by at most smax), is taken whole: its score and mismatches from the
        // two byte words (bytes equal and both below 4: match; either above 3: ambiguous;
        // else mismatch), exactly the sums of the steps below.
        if (((any >> sh) & (kNotDiagE | kFromF)) == 0 && v > (kAhead - 1) * smax) {
          const uint64_t amb = (qw | tw) & 0xFCFCFCFCFCFCFCFCull;
          const uint64_t ok_amb = zero_bytes(amb);
          const int n_match = __popcll(zero_bytes(qw ^ tw) & ok_amb);
          const int n_amb = kAhead - __popcll(ok_amb);
          v -= n_match * p.match - (kAhead - n_match - n_amb) * p.mismatch - n_amb * p.ambig;
          nm += kAhead - n_match;
          run += kAhead;
          i -= kAhead;
          continue;
        }
#pragma unroll
        for (int k = 0; k < kAhead; ++k) {
          cx[k] = (wk[k] >> sh) & 0xFu;
          qa[k] = static_cast<int>((qw >> (8 * (kAhead - 1 - k))) & 0xFFu);
          const int t8 = static_cast<int>((tw >> (8 * (kAhead - 1 - k))) & 0xFFu);
          ta[k] = t8 > 3 ? 4 : t8;
        }
      } else {
#pragma unroll
        for (int k = 0; k < kAhead; ++k) {
          cx[k] = 0;
          qa[k] = ta[k] = 0;
          if (i - k >= 0) {
            cx[k] = code(i - k, d);
            qa[k] = q[i - k];
            ta[k] = static_cast<int>(tcode(tbase, tk, static_cast<int64_t>(i - k) + d));
          }
        }
      }
#pragma unroll
      for (int k = 0; k < kAhead; ++k) {
        if (i < 0 || v <= 0) {
          stop = true;
          break;
        }
        x = cx[k];
        if (x & (kNotDiagE | kFromF)) {  // not from the diagonal
          stop = true;
          break;
        }
        v -= sub_score(p, qa[k], ta[k]);
        nm += (qa[k] != ta[k] || qa[k] > 3) ? 1 : 0;
        ++run;
        --i;
      }
    }
    if (run) cw.push(0u /* M */, run);
    if (i < 0 || v <= 0) break;
    run = 0;
    bool ext;
    if (!(x & kFromF)) {  // from E, an insertion: E(i,d) <- (i-1, d+1)
      do {
        if (i < 0 || d >= W) {
          atomicOr(err, kErrTracebackBounds);
          goto done;
        }
        ext = (code(i, d) & kExtE) != 0;
        v += ext ? p.ge : p.oe;
        ++run;
        --i;
        ++d;
      } while (ext);
      cw.push(1u /* I */, run);
    } else {  // from F, a deletion: F(i,d) <- (i, d-1)
      do {
        if (d < 0 || d >= W) {
          atomicOr(err, kErrTracebackBounds);
          goto done;
        }
        ext = (code(i, d) & kExtF) != 0;
        v += ext ? p.ge : p.oe;
        ++run;
        --d;
      } while (ext);
      cw.push(2u /* D */, run);
    }
    nm += run;
  }
done:
  cw.flush();
  if (cw.n > cap) atomicOr(err, kErrCigarOverflow);
  r.qb = i + 1;
  r.tb = i + 1 + d;
  r.qe = bi + 1;
  r.te = bi + bd + 1;
  r.nm = nm;
  r.n_ops = cw.n < cap ? cw.n : cap;
}


// Best-row checkpoints of the two halves of a pair share two row buffers: a row that
// improves both halves is stored once (the packed row serves both), and a half that
// improves alone writes the buffer the other half is not using. Returns the buffer to
// write; buf_a / buf_b say where each half's best row is.
__device__ __forceinline__ int row_buffer(bool up_a, bool up_b, int buf_a, int buf_b) {
  if (up_a && up_b) return buf_a;
  if (up_a) return buf_a == buf_b ? 1 - buf_b : buf_a;
  return buf_a == buf_b ? 1 - buf_a : buf_b;
}

// The DP kernels leave, for the walk, the best cell in the result: qb = its row, qe = its
// column (the walk kernel then writes the final coordinates).
__device__ __forceinline__ SwResult stash(int score, int bi, int bd) { return SwResult{score, bi, bd, 0, 0, 0, 0, 0}; }

// Direction-code base of local task lt (pairs 2p, 2p+1 share words; 32 pairs per warp).
__device__ __forceinline__ uint32_t* pair_base(uint32_t* dir, int lt, int rows_max, int WQ) {
  const int pair = lt >> 1;
  return dir + static_cast<size_t>(pair >> 5) * rows_max * WQ * 32 + (pair & 31);
}

// One alignment, int32 scores, band row of compile-time width W in registers; direction
// codes into its half of the pair layout (DP = the pair's first word).
template <int W, bool TB>
__device__ SwResult sw_one_reg(const SwTask& tk, const uint8_t* __restrict__ qbase, const uint8_t* __restrict__ tbase,
                               const SwParams& p, uint32_t* __restrict__ DP, int half) {
  constexpr int WQ = (W + 3) / 4;
  const uint8_t* __restrict__ q = qbase + tk.q_off;
  const int ql = tk.qlen;
  int H[W + 1], E[W + 1];
  uint32_t T[W];
#pragma unroll
  for (int d = 0; d <= W; ++d) {
    H[d] = 0;
    E[d] = 0;
  }
#pragma unroll
  for (int d = 0; d < W; ++d) T[d] = sel1(tcode(tbase, tk, d));
  int best = 0, bi = -1, bd = -1;
  for (int i = 0; i < ql; ++i) {
    const uint32_t qc = min(static_cast<uint32_t>(q[i]), 4u);
    const uint32_t plo = prof_lo(p, qc), phi = p.prof_n;
    const uint32_t t_next = sel1(tcode(tbase, tk, static_cast<int64_t>(i) + W));
    int f = 0, hleft = 0, hdiag = H[0], rmax = 0, rd = -1;
    uint32_t dw = 0;
#pragma unroll
    for (int d = 0; d < W; ++d) {
      const int hup = H[d + 1], eup = E[d + 1];
      const int hd = hdiag + static_cast<int>(prmt(plo, phi, T[d]));
      const int eo = hup - p.oe, ee = eup - p.ge, fo = hleft - p.oe, fe = f - p.ge;
      const int e = max(eo, ee);
      f = max(fo, fe);
      const int m1 = max(hd, e);
      const int h = max(max(m1, f), 0);
      H[d] = h;
      E[d] = e;
      if constexpr (TB) {
        dw = dw * 16u + dir_code32(hd >= e, m1 >= f, eo >= ee, fo >= fe);
        if ((d & 3) == 3 || d == W - 1) {
          if ((d & 3) != 3) dw <<= 4 * (3 - (d & 3));
          reinterpret_cast<uint16_t*>(DP + (static_cast<size_t>(i) * WQ + (d >> 2)) * 32)[half] =
              static_cast<uint16_t>(dw);
          dw = 0;
        }
        if (d == 0 || h > rmax) {  // first strict maximum of the row (every H >= 0)
          rmax = h;
          rd = d;
        }
      } else {
        best = max(best, h);
      }
      hleft = h;
      hdiag = hup;
    }
    if (TB && rmax > best) {
      best = rmax;
      bi = i;
      bd = rd;
    }
#pragma unroll
    for (int d = 0; d + 1 < W; ++d) T[d] = T[d + 1];
    T[W - 1] = t_next;
  }
  return TB ? stash(best, bi, bd) : stash(best, 0, 0);
}

// True if the target window [0, qlen + W - 1) of the task reads any N, including the
// padding outside the candidate's contig or past a short target.
__device__ bool window_has_n(const SwTask& tk, int W, const uint8_t* __restrict__ tbase) {
  if (tk.flags & kTaskNoN) return false;
  const int64_t tmax = static_cast<int64_t>(tk.qlen) + W - 1;
  if (tk.t_lo > tk.t_start || tk.t_hi < tk.t_start + tmax) return true;
  const uint8_t* t = tbase + tk.t_start;
  bool any = false;
  for (int64_t j = 0; j < tmax; ++j) any |= __ldg(t + j) > 3;
  return any;
}

// Two alignments per thread in biased 16-bit halves (A low, B high). Pairs it cannot take
// (an N in a target window, or scores/lengths outside the 16-bit range) are listed in fb
// (fb[0] = count, then local task indices) for k_sw_fb. With traceback at W <= 33 the
// launch bound asks for three resident blocks (<= 170 registers, no spills): 12 warps per
// SM instead of 8. Per cell:
//  * E and F by the DPX add-max (max(a + b, c) in one instruction, signed 16x2: the biased
//    values lie in [0, 32767], where signed and unsigned order agree), so the open-gap
//    candidates hup - (O+E) and hleft - (O+E) are never materialised; the extension bits
//    come from e - hup + (O+E) and f - hleft + (O+E), one 3-input add each (both halves
//    non-negative, so no borrow crosses them);
//  * the substitution scores of both alignments are one prmt.b32 on the row's profile
//    words, taken from a 5-entry table in shared memory one row ahead;
//  * target codes are read without range or N checks: the pair reaches the DP only when
//    both windows [0, qlen + W - 1) are N-free and inside their contigs, and reads past a
//    window are clamped to its last base (a row past a query's end is an N row for it,
//    whose scores do not depend on the target), so a code is always 0..3 and the prmt
//    selector of two codes is two multiply-adds.
// Against the former form (vmax of materialised open/extend candidates, profile words
// rebuilt per row, range-checked target reads) this took the traceback kernel from 3.06 to
// 2.56 ms per 1,000,000 x 150 bp reads.
template <int W, bool TB>
__global__ void __launch_bounds__(kSwThreads, (TB && W <= 33) ? 3 : 1)
    k_sw_u2(const SwTask* __restrict__ tasks, int base, int n, const int* __restrict__ n_dev,
             const uint8_t* __restrict__ qbase, const uint8_t* __restrict__ tbase, SwParams p,
             SwResult* __restrict__ res, uint32_t* __restrict__ dir, int rows_max, int* __restrict__ fb) {
  static_assert(W >= 3, "a window of at least two columns past an empty query");
  constexpr int WQ = (W + 3) / 4;
  __shared__ uint32_t s_prof[8];
  if (threadIdx.x < 5) s_prof[threadIdx.x] = prof_biased(p, threadIdx.x);
  __syncthreads();
  const int lt = blockIdx.x * blockDim.x + threadIdx.x;  // pair index within this launch
  const int nn = n_dev ? min(n, *n_dev) : n;
  const int ia = base + 2 * lt, ib = ia + 1;
  if (ia >= nn) return;
  const bool has_b = ib < nn;
  uint32_t* DP = TB ? pair_base(dir, 2 * lt, rows_max, WQ) : nullptr;
  const SwTask ta = tasks[ia];
  SwTask tb = ta;
  if (has_b) tb = tasks[ib];
  else tb.qlen = 0;
  const int qmax = max(ta.qlen, tb.qlen);
  const bool fits = qmax * p.match + 2 * (p.oe + p.ge + p.mismatch + p.ambig) < 16000 &&
                    p.match + kScoreBias <= 127 && p.mismatch <= kScoreBias && p.ambig <= kScoreBias;
  if (!fits || window_has_n(ta, W, tbase) || (has_b && window_has_n(tb, W, tbase))) {
    const int k = atomicAdd(fb, has_b ? 2 : 1);
    fb[1 + k] = 2 * lt;
    if (has_b) fb[2 + k] = 2 * lt + 1;
    return;
  }
  const uint8_t* __restrict__ qa = qbase + ta.q_off;
  const uint8_t* __restrict__ qb = qbase + tb.q_off;
  const int qla = ta.qlen, qlb = tb.qlen;
  // both windows are N-free over [0, qlen + W - 1): column j of each reads its window at
  // min(j, qlen + W - 2), a code in 0..3
  const uint8_t* __restrict__ wa = tbase + ta.t_start;
  const uint8_t* __restrict__ wb = tbase + tb.t_start;
  const int ja = qla + W - 2, jb = qlb + W - 2;
  auto tc2 = [&](int j) {
    const uint32_t a = __ldg(wa + min(j, ja)), b = __ldg(wb + min(j, jb));
    return a * 17u + b * 4352u + 50304u;  // sel2(a, b)
  };
  auto qcode = [&](const uint8_t* __restrict__ q, int ql, int i) {
    return i < ql ? min(static_cast<uint32_t>(q[i]), 4u) : 4u;
  };
  uint32_t H[W + 1], E[W + 1], T[W];
#pragma unroll
  for (int d = 0; d <= W; ++d) {
    H[d] = kBias2;
    E[d] = kBias2;
  }
#pragma unroll
  for (int d = 0; d < W; ++d) T[d] = tc2(d);
  const uint32_t OE = pack2(p.oe), GE = pack2(p.ge), SB = pack2(kScoreBias);
  const uint32_t NOE = pack2(static_cast<uint32_t>(-p.oe));  // -(O+E) in each signed half
  uint32_t best2 = kBias2;
  uint32_t best_a = kBias, best_b = kBias;
  int bi_a = -1, bi_b = -1;
  extern __shared__ uint32_t sw_rows[];
  uint32_t* const row_a = sw_rows + threadIdx.x;
  uint32_t* const row_b = sw_rows + W * kSwThreads + threadIdx.x;
  int buf_a = 0, buf_b = 1;
  uint32_t plo = s_prof[qcode(qa, qla, 0)], phi = s_prof[qcode(qb, qlb, 0)];
  uint32_t ca = qcode(qa, qla, 1), cb = qcode(qb, qlb, 1);  // codes of the next row
  uint32_t* rowp = DP;
  const uint64_t pol = l2_evict_first_policy();
  for (int i = 0; i < qmax; ++i) {
    // the next row's codes and profile words and the target column entering the band are
    // loaded up front, so their latency hides behind this row
    const uint32_t t_next = tc2(i + W);
    const uint32_t plo_next = s_prof[ca], phi_next = s_prof[cb];
    const uint32_t ca_next = qcode(qa, qla, i + 2), cb_next = qcode(qb, qlb, i + 2);
    uint32_t f = kBias2, hleft = kBias2, hdiag = H[0], rmax = 0, dw = 0;
#pragma unroll
    for (int d = 0; d < W; ++d) {
      const uint32_t hup = H[d + 1], eup = E[d + 1];
      const uint32_t hd = hdiag + prmt(plo, phi, T[d]) - SB;
      const uint32_t e = __viaddmax_s16x2(hup, NOE, eup - GE);
      const uint32_t fn = __viaddmax_s16x2(hleft, NOE, f - GE);
      const uint32_t m1 = __vmaxu2(hd, e);
      const uint32_t h = __vimax3_u16x2(m1, fn, kBias2);
      if constexpr (TB) {
        // each term is >= 0 per half; saturated to 0/1 it is one code bit
        const uint32_t b3 = __vminu2(m1 - hd, kOne2), b2 = __vminu2(h - m1, kOne2);
        const uint32_t b1 = __vminu2(e - hup + OE, kOne2), b0 = __vminu2(fn - hleft + OE, kOne2);
        dw = dw * 16u + ((b3 * 2u + b2) * 4u + (b1 * 2u + b0));
        if ((d & 3) == 3 || d == W - 1) {
          if ((d & 3) != 3) dw <<= 4 * (3 - (d & 3));
          st_evict_first(rowp + (d >> 2) * 32, dw, pol);
          dw = 0;
        }
        rmax = d == 0 ? h : __vmaxu2(rmax, h);
      } else {
        best2 = __vmaxu2(best2, h);
      }
      H[d] = h;
      E[d] = e;
      f = fn;
      hleft = h;
      hdiag = hup;
    }
    if constexpr (TB) {  // a strictly better row (rows in order: the first strict maximum)
      const bool up_a = (rmax & 0xFFFFu) > best_a, up_b = (rmax >> 16) > best_b;
      if (up_a || up_b) {
        const int dst = row_buffer(up_a, up_b, buf_a, buf_b);
        uint32_t* const row = dst ? row_b : row_a;
#pragma unroll
        for (int d = 0; d < W; ++d) row[d * kSwThreads] = H[d];
        if (up_a) {
          best_a = rmax & 0xFFFFu;
          bi_a = i;
          buf_a = dst;
        }
        if (up_b) {
          best_b = rmax >> 16;
          bi_b = i;
          buf_b = dst;
        }
      }
      rowp += WQ * 32;
    }
#pragma unroll
    for (int d = 0; d + 1 < W; ++d) T[d] = T[d + 1];
    T[W - 1] = t_next;
    plo = plo_next;
    phi = phi_next;
    ca = ca_next;
    cb = cb_next;
  }
  int bd_a = 0, bd_b = 0;
  if constexpr (!TB) {
    best_a = best2 & 0xFFFFu;
    best_b = best2 >> 16;
  } else {  // first column of the best row holding the best value, per half
    bd_a = bi_a >= 0 ? W : -1;
    bd_b = bi_b >= 0 ? W : -1;
    const uint32_t* const ra = buf_a ? row_b : row_a;
    const uint32_t* const rb = buf_b ? row_b : row_a;
#pragma unroll 1
    for (int d = W - 1; d >= 0; --d) {
      if (bi_a >= 0 && (ra[d * kSwThreads] & 0xFFFFu) == best_a) bd_a = d;
      if (bi_b >= 0 && (rb[d * kSwThreads] >> 16) == best_b) bd_b = d;
    }
  }
  res[ta.slot] = stash(static_cast<int>(best_a) - static_cast<int>(kBias), TB ? bi_a : 0, bd_a);
  if (has_b) res[tb.slot] = stash(static_cast<int>(best_b) - static_cast<int>(kBias), TB ? bi_b : 0, bd_b);
}

// Wide bands, W = CH * LANES + 1: LANES consecutive lanes of a warp share one pair of
// alignments (A and B in the 16-bit halves, as in k_sw_u2), lane c holding band cells
// [CH c, CH c + CH) of the row in registers (the last lane also cell W - 1); CH = 32, or 16
// for twice the lanes per pair (fewer registers, more pairs in flight, a longer skew). Lane c works on
// row t - c at step t, so its left neighbour finished the same row one step earlier: the
// row's running F and H(left) arrive by one shuffle at the start of the step. The one value
// a lane needs from its right neighbour — H and E of the previous row at the neighbour's
// first cell (the E input of the lane's last cell) — is exactly what the neighbour
// computes first in the same step, so a second shuffle after each lane's first cell
// delivers it; every lane is busy on every step. Each lane tracks the first strict
// maximum of its own cells (best-row checkpoint in shared memory, as k_sw_u2), and the
// lanes of a pair combine (value, then earliest row, then smallest column) at the end:
// the first strict maximum of the whole band in row-major order. Pairs k_sw_u2 would
// hand to the int32 kernel are listed in fb the same way.
template <int LANES, int CH, bool TB>
__global__ void __launch_bounds__(kSwThreads, TB ? (CH == 16 ? 4 : 3) : 1)
    k_sw_wide(const SwTask* __restrict__ tasks, int base, int n, const int* __restrict__ n_dev,
              const uint8_t* __restrict__ qbase, const uint8_t* __restrict__ tbase, SwParams p,
              SwResult* __restrict__ res, uint32_t* __restrict__ dir, int rows_max, int* __restrict__ fb) {
  static_assert(CH % 4 == 0 && CH >= 8, "a lane's cells fill whole direction words");
  constexpr int W = CH * LANES + 1, WQ = (W + 3) / 4;
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ uint32_t s_prof[8];  // profile words of the five query codes
  if (threadIdx.x < 5) s_prof[threadIdx.x] = prof_biased(p, threadIdx.x);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int c = lane % LANES;  // chunk of this lane
  const int lt = (blockIdx.x * blockDim.x + threadIdx.x) / LANES;  // pair index within this launch
  const int nn = n_dev ? min(n, *n_dev) : n;
  const int warp_first = (blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / LANES;
  if (base + 2 * warp_first >= nn) return;  // the whole warp is past the tasks (warp-uniform)
  const int ia = base + 2 * lt, ib = ia + 1;
  const bool live = ia < nn, has_b = ib < nn;
  SwTask ta{}, tb{};
  if (live) ta = tasks[ia];
  if (has_b) tb = tasks[ib];
  else tb = ta, tb.qlen = 0;
  const int qmax = live ? max(ta.qlen, tb.qlen) : 0;
  const bool fits = qmax * p.match + 2 * (p.oe + p.ge + p.mismatch + p.ambig) < 16000 &&
                    p.match + kScoreBias <= 127 && p.mismatch <= kScoreBias && p.ambig <= kScoreBias;
  bool skip = !live;
  if (live && (!fits || window_has_n(ta, W, tbase) || (has_b && window_has_n(tb, W, tbase)))) {
    skip = true;
    if (c == 0) {
      const int k = atomicAdd(fb, has_b ? 2 : 1);
      fb[1 + k] = 2 * lt;
      if (has_b) fb[2 + k] = 2 * lt + 1;
    }
  }
  const int steps = __reduce_max_sync(FULL, skip ? 0 : qmax + LANES - 1);
  uint32_t* DP = TB ? pair_base(dir, 2 * lt, rows_max, WQ) : nullptr;
  const uint8_t* __restrict__ qa = qbase + ta.q_off;
  const uint8_t* __restrict__ qb = qbase + tb.q_off;
  const int qla = ta.qlen, qlb = tb.qlen;
  // called for pairs that run here only: both windows [0, qlen + W - 1) N-free and inside
  // their contigs, so column j reads its window at min(j, qlen + W - 2), a code in 0..3
  // (past a window's end it feeds N rows only), and the prmt selector of two codes is two
  // multiply-adds (as k_sw_u2)
  const uint8_t* __restrict__ wa = tbase + ta.t_start;
  const uint8_t* __restrict__ wb = tbase + tb.t_start;
  const int ja = ta.qlen + W - 2, jb = tb.qlen + W - 2;
  auto tc2 = [&](int j) {
    const uint32_t a = __ldg(wa + min(j, ja)), b = __ldg(wb + min(j, jb));
    return a * 17u + b * 4352u + 50304u;  // sel2(a, b)
  };
  auto qcode = [&](const uint8_t* __restrict__ q, int ql, int i) {
    return i >= 0 && i < ql ? min(static_cast<uint32_t>(q[i]), 4u) : 4u;
  };
  const int d0 = CH * c;  // band column of local cell 0
  uint32_t H[CH + 2], E[CH + 2], T[CH + 1];
#pragma unroll
  for (int k = 0; k < CH + 2; ++k) {
    H[k] = kBias2;
    E[k] = kBias2;
  }
#pragma unroll
  for (int k = 0; k <= CH; ++k) T[k] = skip ? 0u : tc2(d0 + k);  // row 0
  const uint32_t OE = pack2(p.oe), GE = pack2(p.ge), SB = pack2(kScoreBias);
  uint32_t best2 = kBias2, best_a = kBias, best_b = kBias;
  int bi_a = -1, bi_b = -1;
  extern __shared__ uint32_t sw_rows[];
  uint32_t* const row_a = sw_rows + threadIdx.x;
  uint32_t* const row_b = sw_rows + (CH + 1) * kSwThreads + threadIdx.x;
  int buf_a = 0, buf_b = 1;  // which of the two row buffers holds each half's best row
  uint32_t hout = kBias2, fout = kBias2;  // this lane's last cell of its previous row
  // the row's profile words, and the codes of the next step's row: loaded a step ahead so
  // their latency hides behind the step (row -c of a lane that has not reached row 0 is N)
  uint32_t plo = s_prof[qcode(qa, qla, -c)], phi = s_prof[qcode(qb, qlb, -c)];
  uint32_t cna = qcode(qa, qla, 1 - c), cnb = qcode(qb, qlb, 1 - c);
  const auto step = [&](const int t, auto steady) {
    constexpr bool kSteady = decltype(steady)::value;
    const int i = t - c;
    const bool act = !skip && i >= 0 && i < qmax;
    // H, E and the target window advance once the lane has reached row 0 (rows past the
    // pair's end are N rows: they change no result and no code is stored for them); from
    // step LANES - 1 on every lane has, so the steady steps carry no per-cell guard
    const bool he_ok = kSteady || i >= 0;
    // row i's F and H(left) at column d0 - 1, from the left lane (its step t - 1)
    uint32_t hleft = __shfl_up_sync(FULL, hout, 1), f = __shfl_up_sync(FULL, fout, 1);
    if (c == 0) hleft = f = kBias2;
    const uint32_t plo_next = s_prof[cna], phi_next = s_prof[cnb];
    const uint32_t cna_next = qcode(qa, qla, i + 2), cnb_next = qcode(qb, qlb, i + 2);
    // past the pair's end the window shifts in a valid selector (code A for both): the
    // profile of an N row scores every target alike
    const uint32_t t_next = act ? tc2(i + 1 + d0 + CH) : sel2(0u, 0u);
    uint32_t hdiag = H[0], rmax = 0, dw = 0;
    // local cell 0, then hand (H, E) of it to the left lane: the E input of its last cell
    uint32_t h0, e0;
    {
      const uint32_t hup = H[1], eup = E[1];
      const uint32_t hd = hdiag + prmt(plo, phi, T[0]) - SB;
      const uint32_t eo = hup - OE, ee = eup - GE, fo = hleft - OE, fe = f - GE;
      e0 = __vmaxu2(eo, ee);
      f = __vmaxu2(fo, fe);
      const uint32_t m1 = __vmaxu2(hd, e0);
      h0 = __vimax3_u16x2(m1, f, kBias2);
      if constexpr (TB)
        dw = ((__vminu2(m1 - hd, kOne2) * 2u + __vminu2(h0 - m1, kOne2)) * 2u + __vminu2(e0 - eo, kOne2)) * 2u +
             __vminu2(f - fo, kOne2);
      rmax = h0;
      hleft = h0;
      hdiag = hup;
    }
    // a lane that has not reached row 0 passes row -1's values (zero)
    uint32_t nh = __shfl_down_sync(FULL, i >= 0 ? h0 : kBias2, 1);
    uint32_t ne = __shfl_down_sync(FULL, i >= 0 ? e0 : kBias2, 1);
    if (c == LANES - 1) {
      nh = H[CH];
      ne = E[CH];
    }
    if (he_ok) {
      H[0] = h0;
      E[0] = e0;
    }
#pragma unroll
    for (int k = 1; k <= CH; ++k) {
      if (k == CH && c != LANES - 1) break;  // the extra cell W - 1 belongs to the last lane
      const uint32_t hup = k == CH - 1 ? nh : (k == CH ? kBias2 : H[k + 1]);
      const uint32_t eup = k == CH - 1 ? ne : (k == CH ? kBias2 : E[k + 1]);
      const uint32_t hd = hdiag + prmt(plo, phi, T[k]) - SB;
      const uint32_t eo = hup - OE, ee = eup - GE, fo = hleft - OE, fe = f - GE;
      const uint32_t e = __vmaxu2(eo, ee);
      f = __vmaxu2(fo, fe);
      const uint32_t m1 = __vmaxu2(hd, e);
      const uint32_t h = __vimax3_u16x2(m1, f, kBias2);
      if (he_ok) {
        H[k] = h;
        E[k] = e;
      }
      if constexpr (TB) {
        const uint32_t code = ((__vminu2(m1 - hd, kOne2) * 2u + __vminu2(h - m1, kOne2)) * 2u +
                               __vminu2(e - eo, kOne2)) * 2u + __vminu2(f - fo, kOne2);
        dw = dw * 16u + code;
        if ((k & 3) == 3) {
          if (act) DP[(static_cast<size_t>(i) * WQ + ((d0 + k) >> 2)) * 32] = dw;
          dw = 0;
        } else if (k == CH) {  // cell W - 1 opens the last, partial word
          dw <<= 12;
          if (act) DP[(static_cast<size_t>(i) * WQ + ((d0 + k) >> 2)) * 32] = dw;
        }
        rmax = __vmaxu2(rmax, h);
      } else {
        best2 = __vmaxu2(best2, h);
      }
      hleft = h;
      hdiag = hup;
    }
    if constexpr (!TB) best2 = __vmaxu2(best2, h0);
    hout = hleft;
    fout = f;
    if (act) {
      if constexpr (TB) {  // a strictly better row of this lane's cells
        const bool up_a = (rmax & 0xFFFFu) > best_a, up_b = (rmax >> 16) > best_b;
        if (up_a || up_b) {
          const int dst = row_buffer(up_a, up_b, buf_a, buf_b);
          uint32_t* const row = dst ? row_b : row_a;
#pragma unroll
          for (int k = 0; k <= CH; ++k) row[k * kSwThreads] = H[k];
          if (up_a) {
            best_a = rmax & 0xFFFFu;
            bi_a = i;
            buf_a = dst;
          }
          if (up_b) {
            best_b = rmax >> 16;
            bi_b = i;
            buf_b = dst;
          }
        }
      }
    }
    if (he_ok) {
#pragma unroll
      for (int k = 0; k < CH; ++k) T[k] = T[k + 1];
      T[CH] = t_next;
    }
    plo = plo_next;
    phi = phi_next;
    cna = cna_next;
    cnb = cnb_next;
  };
  const int ramp = steps < LANES - 1 ? steps : LANES - 1;
  for (int t = 0; t < ramp; ++t) step(t, std::false_type{});
  for (int t = ramp; t < steps; ++t) step(t, std::true_type{});
  // combine the lanes of the pair: larger value, then earlier row, then smaller column
  uint64_t key_a, key_b;
  const int ncell = c == LANES - 1 ? CH + 1 : CH;
  if constexpr (TB) {
    int bd_a = 0xFFF, bd_b = 0xFFF;
    const uint32_t* const ra = buf_a ? row_b : row_a;
    const uint32_t* const rb = buf_b ? row_b : row_a;
#pragma unroll 1
    for (int k = ncell - 1; k >= 0; --k) {
      if (bi_a >= 0 && (ra[k * kSwThreads] & 0xFFFFu) == best_a) bd_a = d0 + k;
      if (bi_b >= 0 && (rb[k * kSwThreads] >> 16) == best_b) bd_b = d0 + k;
    }
    key_a = static_cast<uint64_t>(best_a) << 40 | static_cast<uint64_t>(0xFFFFFu - static_cast<uint32_t>(bi_a + 1)) << 12 |
            (0xFFFu - static_cast<uint32_t>(bd_a));
    key_b = static_cast<uint64_t>(best_b) << 40 | static_cast<uint64_t>(0xFFFFFu - static_cast<uint32_t>(bi_b + 1)) << 12 |
            (0xFFFu - static_cast<uint32_t>(bd_b));
  } else {
    key_a = static_cast<uint64_t>(best2 & 0xFFFFu) << 40;
    key_b = static_cast<uint64_t>(best2 >> 16) << 40;
  }
#pragma unroll
  for (int o = 1; o < LANES; o <<= 1) {
    const uint64_t xa = __shfl_xor_sync(FULL, key_a, o), xb = __shfl_xor_sync(FULL, key_b, o);
    key_a = xa > key_a ? xa : key_a;
    key_b = xb > key_b ? xb : key_b;
  }
  if (c != 0 || skip) return;
  const auto unpack = [](uint64_t key) {
    const int best = static_cast<int>(key >> 40) - static_cast<int>(kBias);
    const int bi = static_cast<int>(0xFFFFFu - static_cast<uint32_t>((key >> 12) & 0xFFFFFu)) - 1;
    const int bd = static_cast<int>(0xFFFu - static_cast<uint32_t>(key & 0xFFFu));
    return TB ? stash(best, bi, bd) : stash(best, 0, 0);
  };
  res[ta.slot] = unpack(key_a);
  if (has_b) res[tb.slot] = unpack(key_b);
}

// The pairs k_sw_u2 listed, one alignment per thread, int32.
template <int W, bool TB>
__global__ void __launch_bounds__(kSwThreads) k_sw_fb(const SwTask* __restrict__ tasks, int base,
                                                      const uint8_t* __restrict__ qbase,
                                                      const uint8_t* __restrict__ tbase, SwParams p,
                                                      SwResult* __restrict__ res, uint32_t* __restrict__ dir,
                                                      int rows_max, const int* __restrict__ fb) {
  constexpr int WQ = (W + 3) / 4;
  const int nfb = fb[0];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nfb; j += gridDim.x * blockDim.x) {
    const int lt = fb[1 + j];
    const SwTask tk = tasks[base + lt];
    res[tk.slot] = sw_one_reg<W, TB>(tk, qbase, tbase, p, TB ? pair_base(dir, lt, rows_max, WQ) : nullptr, lt & 1);
  }
}

// The tasks k_sw_u2 / k_sw_wide listed (an N in the target window, or outside the biased
// 16-bit range) for bands of W = CH * LANES + 1 columns, one alignment per LANES lanes in
// int32: lane c holds band columns [CH c, CH c + CH) (the last lane also column W - 1) and
// computes row t - c at step t — k_sw_wide's skewed wavefront, exchanging the left lane's
// last (H, F) and the right lane's first (H, E) by shuffles. Scores come from the 5-entry
// profile (N scored as the reference scores it), direction codes go to the task's half of
// the pair words, the best cell is the first strict maximum in row-major order: the same
// results and codes as sw_one_reg, which runs one alignment per thread and, at W = 129,
// spills its band to local memory. The list is short (windows that cross a contig end or
// an N run), so the kernel's time is one task's serial latency: narrow chunks (8 or 16
// cells per lane) spread a task over more lanes and shorten it.
template <int LANES, int CH, bool TB>
__global__ void __launch_bounds__(kSwThreads)
    k_sw_fb_lanes(const SwTask* __restrict__ tasks, int base, const uint8_t* __restrict__ qbase,
                  const uint8_t* __restrict__ tbase, SwParams p, SwResult* __restrict__ res,
                  uint32_t* __restrict__ dir, int rows_max, const int* __restrict__ fb) {
  static_assert(CH % 4 == 0 && CH >= 8, "a lane's cells fill whole direction words");
  constexpr int W = CH * LANES + 1, WQ = (W + 3) / 4;
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int c = lane % LANES;
  const int nfb = fb[0];
  const int stride = static_cast<int>(gridDim.x * blockDim.x / LANES);
  // a warp takes 32 / LANES consecutive entries of the fallback list per round (jw, the
  // first, is warp-uniform, so every lane takes the same rounds)
  for (int jw = static_cast<int>((blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / LANES); jw < nfb; jw += stride) {
  const int j = jw + lane / LANES;  // entry of the fallback list
  const bool live = j < nfb;
  const int lt = live ? fb[1 + j] : 0;
  SwTask tk{};
  if (live) tk = tasks[base + lt];
  const int ql = live ? tk.qlen : 0;
  const int steps = __reduce_max_sync(FULL, live ? ql + LANES - 1 : 0);
  const uint8_t* __restrict__ q = qbase + tk.q_off;
  uint32_t* DP = TB ? pair_base(dir, lt, rows_max, WQ) : nullptr;
  const int half = lt & 1;
  const int d0 = CH * c;
  int H[CH + 2], E[CH + 2];
  uint32_t T[CH + 1];
#pragma unroll
  for (int k = 0; k < CH + 2; ++k) {
    H[k] = 0;
    E[k] = 0;
  }
#pragma unroll
  for (int k = 0; k <= CH; ++k) T[k] = live ? sel1(tcode(tbase, tk, d0 + k)) : sel1(4u);
  int best = 0, bi = -1, bd = -1;
  int hout = 0, fout = 0;  // this lane's last cell of its previous row
  for (int t = 0; t < steps; ++t) {
    const int i = t - c;
    const bool act = live && i >= 0 && i < ql;
    int hleft = __shfl_up_sync(FULL, hout, 1), f = __shfl_up_sync(FULL, fout, 1);
    if (c == 0) hleft = f = 0;
    const uint32_t qc = act ? min(static_cast<uint32_t>(q[i]), 4u) : 4u;
    const uint32_t plo = prof_lo(p, qc), phi = p.prof_n;
    const uint32_t t_next = act ? sel1(tcode(tbase, tk, static_cast<int64_t>(i) + 1 + d0 + CH)) : sel1(4u);
    int hdiag = H[0], rmax = 0, rk = 0;
    uint32_t dw = 0;
    int h0, e0;
    {
      const int hup = H[1], eup = E[1];
      const int hd = hdiag + static_cast<int>(prmt(plo, phi, T[0]));
      const int eo = hup - p.oe, ee = eup - p.ge, fo = hleft - p.oe, fe = f - p.ge;
      e0 = max(eo, ee);
      f = max(fo, fe);
      const int m1 = max(hd, e0);
      h0 = max(max(m1, f), 0);
      if constexpr (TB) dw = dir_code32(hd >= e0, m1 >= f, eo >= ee, fo >= fe);
      rmax = h0;
      hleft = h0;
      hdiag = hup;
    }
    // a lane that has not reached row 0 passes row -1's values (zero)
    int nh = __shfl_down_sync(FULL, i >= 0 ? h0 : 0, 1);
    int ne = __shfl_down_sync(FULL, i >= 0 ? e0 : 0, 1);
    if (c == LANES - 1) {
      nh = H[CH];
      ne = E[CH];
    }
    if (act) {
      H[0] = h0;
      E[0] = e0;
    }
#pragma unroll
    for (int k = 1; k <= CH; ++k) {
      if (k == CH && c != LANES - 1) break;  // the extra cell W - 1 belongs to the last lane
      const int hup = k == CH - 1 ? nh : (k == CH ? 0 : H[k + 1]);
      const int eup = k == CH - 1 ? ne : (k == CH ? 0 : E[k + 1]);
      const int hd = hdiag + static_cast<int>(prmt(plo, phi, T[k]));
      const int eo = hup - p.oe, ee = eup - p.ge, fo = hleft - p.oe, fe = f - p.ge;
      const int e = max(eo, ee);
      f = max(fo, fe);
      const int m1 = max(hd, e);
      const int h = max(max(m1, f), 0);
      if (act) {
        H[k] = h;
        E[k] = e;
      }
      if constexpr (TB) {
        dw = dw * 16u + dir_code32(hd >= e, m1 >= f, eo >= ee, fo >= fe);
        if ((k & 3) == 3) {
          if (act) reinterpret_cast<uint16_t*>(DP + (static_cast<size_t>(i) * WQ + ((d0 + k) >> 2)) * 32)[half] =
              static_cast<uint16_t>(dw);
          dw = 0;
        } else if (k == CH) {  // cell W - 1 opens the last, partial word
          dw <<= 12;
          if (act) reinterpret_cast<uint16_t*>(DP + (static_cast<size_t>(i) * WQ + ((d0 + k) >> 2)) * 32)[half] =
              static_cast<uint16_t>(dw);
        }
        if (h > rmax) {  // first strict maximum of the lane's part of the row
          rmax = h;
          rk = k;
        }
      } else {
        rmax = max(rmax, h);
      }
      hleft = h;
      hdiag = hup;
    }
    hout = hleft;
    fout = f;
    if (act) {
      if (rmax > best) {
        best = rmax;
        bi = i;
        bd = d0 + rk;
      }
#pragma unroll
      for (int k = 0; k < CH; ++k) T[k] = T[k + 1];
      T[CH] = t_next;
    }
  }
  // the lanes of the alignment: larger value, then earlier row, then smaller column
  uint64_t key = static_cast<uint64_t>(best) << 40 |
                 static_cast<uint64_t>(0xFFFFFu - static_cast<uint32_t>(bi + 1)) << 12 |
                 (0xFFFu - static_cast<uint32_t>(bd < 0 ? 0xFFF : bd));
#pragma unroll
  for (int o = 1; o < LANES; o <<= 1) {
    const uint64_t x = __shfl_xor_sync(FULL, key, o);
    key = x > key ? x : key;
  }
  if (c == 0 && live) {
    const int kb = static_cast<int>(key >> 40);
    const int kbi = static_cast<int>(0xFFFFFu - static_cast<uint32_t>((key >> 12) & 0xFFFFFu)) - 1;
    const int kbd = static_cast<int>(0xFFFu - static_cast<uint32_t>(key & 0xFFFu));
    res[tk.slot] = TB ? stash(kb, kbi, kbd) : stash(kb, 0, 0);
  }
  }
}

// Traceback of every task of the launch from the stashed best cell (one task per thread;
// the DP kernels are done with the scratch). The walk waits on memory, so the launch bound
// asks for seven resident blocks (72 registers, no spills) rather than the six that 80
// registers allow: 0.52 -> 0.48 ms per 1,000,000 150-bp walks (eight blocks, 64 registers
// with spills: 0.51 ms).
template <int W>
__global__ void __launch_bounds__(kSwThreads, 7) k_sw_walk(const SwTask* __restrict__ tasks, int base, int count, int n,
                                                        const int* __restrict__ n_dev,
                                                        const uint8_t* __restrict__ qbase,
                                                        const uint8_t* __restrict__ tbase, SwParams p,
                                                        SwResult* __restrict__ res, const uint32_t* __restrict__ dir,
                                                        int rows_max, uint32_t* __restrict__ cig,
                                                        const int64_t* __restrict__ cig_off,
                                                        uint32_t* __restrict__ err) {
  constexpr int WQ = (W + 3) / 4;
  const int lt = blockIdx.x * blockDim.x + threadIdx.x;
  const int nn = n_dev ? min(n, *n_dev) : n;
  if (lt >= count || base + lt >= nn) return;
  const SwTask tk = tasks[base + lt];
  const SwResult s = res[tk.slot];
  SwResult r{s.score, 0, 0, 0, 0, 0, 0, 0};
  if (s.score > 0) {
    const PairCodes codes{pair_base(const_cast<uint32_t*>(dir), lt, rows_max, WQ), WQ, lt & 1};
    traceback(codes, W, s.qb, s.qe, s.score, qbase + tk.q_off, tbase, tk, p, r, cig + cig_off[tk.slot],
              2 * tk.qlen + 1, err);
  }
  res[tk.slot] = r;
}

// Any band width and any scores: one alignment per thread, int32, band rows H, E in
// per-warp scratch, lane-interleaved ([d][lane]); walks its own traceback.
template <bool TB>
__global__ void __launch_bounds__(kSwThreads) k_sw_any(const SwTask* __restrict__ tasks, int base, int n,
                                                       const int* __restrict__ n_dev,
                                                       const uint8_t* __restrict__ qbase,
                                                       const uint8_t* __restrict__ tbase, SwParams p,
                                                       SwResult* __restrict__ res, uint32_t* __restrict__ dir,
                                                       int rows_max, uint32_t* __restrict__ cig,
                                                       const int64_t* __restrict__ cig_off, int* __restrict__ band,
                                                       uint32_t* __restrict__ err) {
  const int W = p.W, WW = (W + 7) / 8;
  const int lt = blockIdx.x * blockDim.x + threadIdx.x;  // index within this launch
  const int gt = base + lt;
  if (gt >= (n_dev ? min(n, *n_dev) : n)) return;
  const int lane = threadIdx.x & 31;
  const SwTask tk = tasks[gt];
  const uint8_t* __restrict__ q = qbase + tk.q_off;
  const int ql = tk.qlen;
  uint32_t* D = TB ? dir + (static_cast<size_t>(lt >> 5) * rows_max * WW) * 32 + lane : nullptr;
  int* Hs = band + static_cast<size_t>(lt >> 5) * 2 * (W + 1) * 32 + lane;
  int* Es = Hs + static_cast<size_t>(W + 1) * 32;
  for (int d = 0; d <= W; ++d) {
    Hs[d * 32] = 0;
    Es[d * 32] = 0;
  }
  int best = 0, bi = -1, bd = -1;
  for (int i = 0; i < ql; ++i) {
    const int qc = min(static_cast<int>(q[i]), 4);
    int f = 0, hleft = 0, hdiag = Hs[0], rmax = 0, rd = -1;
    uint32_t dw = 0;
    for (int d = 0; d < W; ++d) {
      const int hup = Hs[(d + 1) * 32], eup = Es[(d + 1) * 32];
      const int tc = static_cast<int>(tcode(tbase, tk, static_cast<int64_t>(i) + d));
      const int hd = hdiag + sub_score(p, qc, tc);
      const int eo = hup - p.oe, ee = eup - p.ge, fo = hleft - p.oe, fe = f - p.ge;
      const int e = max(eo, ee);
      f = max(fo, fe);
      const int m1 = max(hd, e);
      const int h = max(max(m1, f), 0);
      Hs[d * 32] = h;
      Es[d * 32] = e;
      if (TB) {
        dw |= dir_code32(hd >= e, m1 >= f, eo >= ee, fo >= fe) << (4 * (d & 7));
        if ((d & 7) == 7 || d == W - 1) {
          D[(static_cast<size_t>(i) * WW + (d >> 3)) * 32] = dw;
          dw = 0;
        }
        if (d == 0 || h > rmax) {
          rmax = h;
          rd = d;
        }
      } else {
        best = max(best, h);
      }
      hleft = h;
      hdiag = hup;
    }
    if (TB && rmax > best) {
      best = rmax;
      bi = i;
      bd = rd;
    }
  }
  SwResult r{best, 0, 0, 0, 0, 0, 0, 0};
  if (TB && best > 0)
    traceback(NibbleCodes{D, WW}, W, bi, bd, best, q, tbase, tk, p, r, cig + cig_off[tk.slot], 2 * ql + 1, err);
  res[tk.slot] = r;
}

template <int W>
void launch_u2(cudaStream_t st, bool tb, const SwTask* tasks, int base, int count, int n, const int* n_dev,
               const uint8_t* qbase, const uint8_t* tbase, const SwParams& p, SwResult* res, uint32_t* dir,
               int rows_max, uint32_t* cig, const int64_t* cig_off, int* fb, uint32_t* err, const KernelTrace* kt) {
  const int pairs = (count + 1) / 2;
  const int blocks_pairs = (pairs + kSwThreads - 1) / kSwThreads;
  const int blocks_tasks = (count + kSwThreads - 1) / kSwThreads;
  // W = 33 and 65: the fallback list runs four lanes per alignment (k_sw_fb_lanes), the
  // other widths the one-thread kernel, whose band fits in registers
  constexpr bool kLanesFb = W == 33 || W == 65;
  constexpr int kFbCh = (W - 1) / 4;
  // the fallback kernels stride over a list whose length only the device knows (usually
  // short or empty): a few resident waves, not one block per possible entry
  const int fb_cap = 8 * device_sm_count();
  const int blocks_fb =
      std::min(fb_cap, static_cast<int>((static_cast<int64_t>(count) * 4 + kSwThreads - 1) / kSwThreads));
  const int blocks_fb1 = std::min(fb_cap, blocks_tasks);
  const KernelTrace none;
  const KernelTrace& t = kt ? *kt : none;
  cudaMemsetAsync(fb, 0, sizeof(int), st);
  if (tb) {
    constexpr int kRowBytes = 2 * W * kSwThreads * 4;  // the two saved best rows of each thread
    if (kRowBytes > 48 * 1024) {
      static std::atomic<bool> attr_set[kMaxDevices];
      set_smem_limit_once(k_sw_u2<W, true>, kRowBytes, attr_set);
    }
    t.begin(st, "k_sw_u2<tb>");
    k_sw_u2<W, true><<<blocks_pairs, kSwThreads, kRowBytes, st>>>(tasks, base, n, n_dev, qbase, tbase, p, res, dir,
                                                                  rows_max, fb);
    t.end(st);
    t.begin(st, "k_sw_fb<tb>");
    if constexpr (kLanesFb)
      k_sw_fb_lanes<4, kFbCh, true><<<blocks_fb, kSwThreads, 0, st>>>(tasks, base, qbase, tbase, p, res, dir,
                                                                      rows_max, fb);
    else
      k_sw_fb<W, true><<<blocks_fb1, kSwThreads, 0, st>>>(tasks, base, qbase, tbase, p, res, dir, rows_max, fb);
    t.end(st);
    t.begin(st, "k_sw_walk");
    k_sw_walk<W><<<blocks_tasks, kSwThreads, 0, st>>>(tasks, base, count, n, n_dev, qbase, tbase, p, res, dir,
                                                      rows_max, cig, cig_off, err);
    t.end(st);
  } else {
    t.begin(st, "k_sw_u2<score>");
    k_sw_u2<W, false><<<blocks_pairs, kSwThreads, 0, st>>>(tasks, base, n, n_dev, qbase, tbase, p, res, dir, rows_max,
                                                           fb);
    t.end(st);
    t.begin(st, "k_sw_fb<score>");
    if constexpr (kLanesFb)
      k_sw_fb_lanes<4, kFbCh, false><<<blocks_fb, kSwThreads, 0, st>>>(tasks, base, qbase, tbase, p, res, dir,
                                                                       rows_max, fb);
    else
      k_sw_fb<W, false><<<blocks_fb1, kSwThreads, 0, st>>>(tasks, base, qbase, tbase, p, res, dir, rows_max, fb);
    t.end(st);
  }
}

template <int LANES, int CH = 32>
void launch_wide(cudaStream_t st, bool tb, const SwTask* tasks, int base, int count, int n, const int* n_dev,
                 const uint8_t* qbase, const uint8_t* tbase, const SwParams& p, SwResult* res, uint32_t* dir,
                 int rows_max, uint32_t* cig, const int64_t* cig_off, int* fb, uint32_t* err, const KernelTrace* kt) {
  constexpr int W = CH * LANES + 1;
  constexpr int FBCH = W == 33 ? 8 : 16;  // cells per lane of the int32 fallback kernel
  constexpr int FBL = (W - 1) / FBCH;     // its lanes per alignment
  const int pairs = (count + 1) / 2;
  const int blocks_pairs = static_cast<int>((static_cast<int64_t>(pairs) * LANES + kSwThreads - 1) / kSwThreads);
  const int blocks_tasks = (count + kSwThreads - 1) / kSwThreads;
  // the fallback list holds at most `count` tasks (its length is known on the device only;
  // the kernel strides over it, so a few resident waves suffice)
  const int blocks_fb = std::min(8 * device_sm_count(),
                                 static_cast<int>((static_cast<int64_t>(count) * FBL + kSwThreads - 1) / kSwThreads));
  const KernelTrace none;
  const KernelTrace& t = kt ? *kt : none;
  cudaMemsetAsync(fb, 0, sizeof(int), st);
  if (tb) {
    constexpr int kRowBytes = 2 * (CH + 1) * kSwThreads * 4;  // the two saved best rows of each lane
    t.begin(st, "k_sw_wide<tb>");
    k_sw_wide<LANES, CH, true><<<blocks_pairs, kSwThreads, kRowBytes, st>>>(tasks, base, n, n_dev, qbase, tbase, p,
                                                                            res, dir, rows_max, fb);
    t.end(st);
    t.begin(st, "k_sw_fb<tb>");
    k_sw_fb_lanes<FBL, FBCH, true><<<blocks_fb, kSwThreads, 0, st>>>(tasks, base, qbase, tbase, p, res, dir, rows_max,
                                                                     fb);
    t.end(st);
    t.begin(st, "k_sw_walk");
    k_sw_walk<W><<<blocks_tasks, kSwThreads, 0, st>>>(tasks, base, count, n, n_dev, qbase, tbase, p, res, dir,
                                                      rows_max, cig, cig_off, err);
    t.end(st);
  } else {
    t.begin(st, "k_sw_wide<score>");
    k_sw_wide<LANES, CH, false><<<blocks_pairs, kSwThreads, 0, st>>>(tasks, base, n, n_dev, qbase, tbase, p, res, dir,
                                                                     rows_max, fb);
    t.end(st);
    t.begin(st, "k_sw_fb<score>");
    k_sw_fb_lanes<FBL, FBCH, false><<<blocks_fb, kSwThreads, 0, st>>>(tasks, base, qbase, tbase, p, res, dir,
                                                                      rows_max, fb);
    t.end(st);
  }
}

}  // namespace

bool sw_bytes_ok(const dnaln_score_params& s) {
  return s.match <= 127 && s.mismatch <= 128 && s.ambig <= 128 && s.match >= -128;
}

bool sw_band_in_registers(int W) { return W == 11 || W == 17 || W == 33 || W == 43 || W == 65 || W == 129; }

bool sw_uses_generic(int W, bool bytes_ok) { return !(bytes_ok && sw_band_in_registers(W)); }

SwParams make_sw_params(const dnaln_score_params& s) {
  SwParams p;
  p.match = s.match;
  p.mismatch = s.mismatch;
  p.oe = s.gap_open + s.gap_ext;
  p.ge = s.gap_ext;
  p.ambig = s.ambig;
  p.bw = s.bw;
  p.W = 2 * s.bw + 1;
  p.prof_n = static_cast<uint32_t>(static_cast<uint8_t>(-s.ambig)) * 0x01010101u;
  return p;
}

size_t sw_dir_bytes_per_task(int W, int rows_max) {
  const size_t pair = static_cast<size_t>((W + 3) / 4) * 2, nib = static_cast<size_t>((W + 7) / 8) * 4;
  return static_cast<size_t>(rows_max > 0 ? rows_max : 1) * (pair > nib ? pair : nib);
}

size_t sw_band_bytes_per_task(int W, bool bytes_ok) {
  return sw_uses_generic(W, bytes_ok) ? static_cast<size_t>(2) * (W + 1) * sizeof(int) : 0;
}

int sw_launches(int W, bool bytes_ok, bool tb) { return sw_uses_generic(W, bytes_ok) ? 1 : (tb ? 3 : 2); }

bool sw_has_form(int W, bool bytes_ok, SwForm form) {
  if (sw_uses_generic(W, bytes_ok)) return form == kSwInter;
  switch (form) {
    case kSwInter: return W != 129;
    case kSwIntra: return W == 33 || W == 65 || W == 129;
    case kSwIntraNarrow: return W == 33 || W == 65 || W == 129;
    default: return false;
  }
}

int sw_lanes_per_pair(int W, SwForm form) {
  if (form == kSwIntra) return (W - 1) / 32;
  if (form == kSwIntraNarrow) return (W - 1) / 16;
  return 1;
}

bool launch_sw(cudaStream_t st, bool tb, bool bytes_ok, const SwTask* tasks, int base, int count, int n,
               const int* n_dev, const uint8_t* qbase, const uint8_t* tbase, const SwParams& p, SwResult* res,
               uint32_t* dir, int rows_max, uint32_t* cig, const int64_t* cig_off, int* band, int* fb,
               uint32_t* err, const KernelTrace* kt, SwForm form) {
  if (count <= 0) return true;
  const bool generic = sw_uses_generic(p.W, bytes_ok);
  if ((tb && !dir) || (generic && !band) || (!generic && !fb) || (base % kSwTaskGroup) != 0) return false;
  // the kernels bound their tasks by n (and the device count): a launch covers tasks
  // [base, base + count) only, so that no thread of a grid rounded up past `count` takes a
  // task of the next chunk, whose scratch this launch does not hold
  if (n > base + count) n = base + count;
  if (!generic && form != kSwInter && sw_has_form(p.W, bytes_ok, form)) {
#define DNB_SW_WIDE(L, CHV) \
  launch_wide<L, CHV>(st, tb, tasks, base, count, n, n_dev, qbase, tbase, p, res, dir, rows_max, cig, cig_off, fb, err, kt)
    const bool narrow = form == kSwIntraNarrow;
    if (p.W == 33) {
      if (narrow) DNB_SW_WIDE(2, 16);
      else DNB_SW_WIDE(1, 32);
    } else if (p.W == 65) {
      if (narrow) DNB_SW_WIDE(4, 16);
      else DNB_SW_WIDE(2, 32);
    } else {
      if (narrow) DNB_SW_WIDE(8, 16);
      else DNB_SW_WIDE(4, 32);
    }
#undef DNB_SW_WIDE
    return true;
  }
  if (!generic) {
#define DNB_SW_U2(WV)                                                                                       \
  case WV:                                                                                                  \
    launch_u2<WV>(st, tb, tasks, base, count, n, n_dev, qbase, tbase, p, res, dir, rows_max, cig, cig_off, \
                  fb, err, kt);                                                                             \
    return true;
    switch (p.W) {
      DNB_SW_U2(11)
      DNB_SW_U2(17)
      DNB_SW_U2(33)
      DNB_SW_U2(43)
      DNB_SW_U2(65)
      case 129:  // no inter-sequence form at this width
        launch_wide<4, 32>(st, tb, tasks, base, count, n, n_dev, qbase, tbase, p, res, dir, rows_max, cig, cig_off, fb,
                           err, kt);
        return true;
      default: break;
    }
#undef DNB_SW_U2
  }
  const int blocks = (count + kSwThreads - 1) / kSwThreads;
  if (kt) kt->begin(st, tb ? "k_sw_any<tb>" : "k_sw_any<score>");
  if (tb)
    k_sw_any<true><<<blocks, kSwThreads, 0, st>>>(tasks, base, n, n_dev, qbase, tbase, p, res, dir, rows_max, cig,
                                                 cig_off, band, err);
  else
    k_sw_any<false><<<blocks, kSwThreads, 0, st>>>(tasks, base, n, n_dev, qbase, tbase, p, res, dir, rows_max, cig,
                                                  cig_off, band, err);
  if (kt) kt->end(st);
  return true;
}

}  // namespace dnb
