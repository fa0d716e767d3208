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
// Kernels (inter-sequence: every thread owns whole alignments, no intra-row shuffles):
//  * k_sw_x2<W>: two alignments per thread, one in each 16-bit half of 32-bit registers,
//    the band row (H, E of W+1 cells, W target selectors) in registers. Each cell is a
//    handful of Blackwell DPX instructions: __viaddmax_s16x2 for the adds,
//    __vibmax_s16x2 for the maxima — which also yields, per half, the predicate a >= b
//    the traceback needs, so direction bits come with the max — and
//    __vimax_s16x2_relu for H. The substitution score of both alignments is one
//    prmt.b32 from an 8-byte per-row profile {s(qA,A..T), s(qB,A..T)}. 16-bit scores are
//    exact while match * qlen stays far from 32767 (checked per pair).
//  * A pair whose target window contains an N (or is too long for 16 bits) runs the
//    int32 form of the same cell update, one alignment after the other (sw_one_reg).
//  * k_sw_any: any band width and any scores (int32, band rows in per-warp scratch).
//
// Traceback: a 4-bit direction code per cell, packed 8 cells per word and stored
// lane-interleaved (word (i, d/8) of 32 alignments is one 128-byte line). The code is
//   bit 3: p1 = hd >= E     bit 2: p2 = max(hd, E) >= F
//   bit 1: E(i,d) extends E(i-1,d+1) (ee > eo)     bit 0: F extends (fe > fo)
// On every cell the walk reads, H is the positive value being traced, and there
// "H from the diagonal" (h == hd in src/align.cpp:67) is p1 && p2 and "H from E"
// (h == e) with no diagonal is !p1 && p2, so the walk (src/align.cpp:87-143) takes the
// reference's steps. The best cell is the first strict maximum in row-major order.
#include "common.cuh"
#include "sw.cuh"

namespace dnb {

namespace {

constexpr int kSwThreads = 128;
constexpr uint32_t kP1 = 8u, kP2 = 4u, kExtE = 2u, kExtF = 1u;

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

// Selector of two sign-extended 16-bit scores: alignment A's byte a (0..3) into the low
// half, alignment B's byte 4 + b into the high half.
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

// Profile word of query code qc: byte t = match if t == qc else -mismatch; an N query
// row scores -ambig everywhere.
__device__ __forceinline__ uint32_t prof_lo(const SwParams& p, uint32_t qc) {
  if (qc > 3) return p.prof_n;
  const uint32_t mm = (static_cast<uint32_t>(static_cast<uint8_t>(-p.mismatch))) * 0x01010101u;
  const uint32_t sh = 8u * qc;
  return (mm & ~(0xFFu << sh)) | (static_cast<uint32_t>(static_cast<uint8_t>(p.match)) << sh);
}

__device__ __forceinline__ uint32_t pack2(int v) { return (static_cast<uint32_t>(v) & 0xFFFFu) * 0x10001u; }
__device__ __forceinline__ int lo16(uint32_t x) { return static_cast<int>(static_cast<int16_t>(x & 0xFFFFu)); }
__device__ __forceinline__ int hi16(uint32_t x) { return static_cast<int>(static_cast<int16_t>(x >> 16)); }

__device__ __forceinline__ uint32_t dir_code(bool p1, bool p2, bool e_not_ext, bool f_not_ext) {
  return (p1 ? kP1 : 0u) | (p2 ? kP2 : 0u) | (e_not_ext ? 0u : kExtE) | (f_not_ext ? 0u : kExtF);
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

// Walks the direction codes back from (bi, bd) (src/align.cpp:87-143). `D` points at
// this alignment's first word; word (i, w) is D[(i * WW + w) * stride]. CIGAR ops are
// written in walk order (last op first), adjacent equal ops merged as the reference's
// push() does.
__device__ void traceback(const uint32_t* __restrict__ D, int stride, int WW, int W, int bi, int bd, int best,
                          const uint8_t* __restrict__ q, const uint8_t* __restrict__ tbase, const SwTask& tk,
                          const SwParams& p, SwResult& r, uint32_t* __restrict__ cig, int cap,
                          uint32_t* __restrict__ err) {
  auto code = [&](int i, int d) -> uint32_t {
    return (D[(static_cast<size_t>(i) * WW + (d >> 3)) * stride] >> (4 * (d & 7))) & 0xFu;
  };
  CigarWriter cw{cig, cap, 0, 0xFu, 0};
  int i = bi, d = bd, v = best, nm = 0;
  for (;;) {
    int run = 0;
    uint32_t x = 0;
    while (i >= 0 && v > 0) {
      x = code(i, d);
      if ((x & (kP1 | kP2)) != (kP1 | kP2)) break;  // not from the diagonal
      const int a = q[i];
      const int b = static_cast<int>(tcode(tbase, tk, static_cast<int64_t>(i) + d));
      v -= sub_score(p, a, b);
      nm += (a != b || a > 3) ? 1 : 0;
      ++run;
      --i;
    }
    if (run) cw.push(0u /* M */, run);
    if (i < 0 || v <= 0) break;
    run = 0;
    bool ext;
    if (x & kP2) {  // from E, an insertion: E(i,d) <- (i-1, d+1)
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

// One alignment, int32 scores, band row of compile-time width W in registers. D is this
// alignment's direction-word base (words `stride` apart).
template <int W, bool TB>
__device__ SwResult sw_one_reg(const SwTask& tk, const uint8_t* __restrict__ qbase, const uint8_t* __restrict__ tbase,
                               const SwParams& p, uint32_t* __restrict__ D, int stride, uint32_t* __restrict__ cig,
                               const int64_t* __restrict__ cig_off, uint32_t* __restrict__ err) {
  constexpr int WW = (W + 7) / 8;
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
    int f = 0, hleft = 0, hdiag = H[0], rmax = 0, rd = -1;
    uint32_t dw = 0;
#pragma unroll
    for (int d = 0; d < W; ++d) {
      const int hup = H[d + 1], eup = E[d + 1];
      const int hd = hdiag + static_cast<int>(prmt(plo, phi, T[d]));
      bool pe, pf, p1, p2;
      const int e = __vibmax_s32(hup - p.oe, eup - p.ge, &pe);
      f = __vibmax_s32(hleft - p.oe, f - p.ge, &pf);
      const int m1 = __vibmax_s32(hd, e, &p1);
      const int h = __vimax_s32_relu(__vibmax_s32(m1, f, &p2), 0);
      H[d] = h;
      E[d] = e;
      if constexpr (TB) {
        dw |= dir_code(p1, p2, pe, pf) << (4 * (d & 7));
        if ((d & 7) == 7 || d == W - 1) {
          D[(static_cast<size_t>(i) * WW + (d >> 3)) * stride] = dw;
          dw = 0;
        }
        if (d == 0) {  // the row's first cell starts its running maximum (every H >= 0)
          rmax = h;
          rd = 0;
        } else {
          bool pr;
          rmax = __vibmax_s32(rmax, h, &pr);
          if (!pr) rd = d;  // strictly above the row's running max: first occurrence wins
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
    T[W - 1] = sel1(tcode(tbase, tk, static_cast<int64_t>(i) + W));
  }
  SwResult r{best, 0, 0, 0, 0, 0, 0, 0};
  if (TB && best > 0) traceback(D, stride, WW, W, bi, bd, best, q, tbase, tk, p, r, cig + cig_off[tk.slot], 2 * ql + 1, err);
  return r;
}

// True if the target window [0, qlen + W - 1) of the task reads any N, including the
// padding outside the candidate's contig or past a short target.
__device__ bool window_has_n(const SwTask& tk, int W, const uint8_t* __restrict__ tbase) {
  const int64_t tmax = static_cast<int64_t>(tk.qlen) + W - 1;
  if (tk.t_lo > tk.t_start || tk.t_hi < tk.t_start + tmax) return true;
  const uint8_t* t = tbase + tk.t_start;
  for (int64_t j = 0; j < tmax; ++j)
    if (__ldg(t + j) > 3) return true;
  return false;
}

// Two alignments per thread in 16-bit halves (A low, B high).
template <int W, bool TB>
__global__ void __launch_bounds__(kSwThreads) k_sw_x2(const SwTask* __restrict__ tasks, int base, int n,
                                                      const int* __restrict__ n_dev, const uint8_t* __restrict__ qbase,
                                                      const uint8_t* __restrict__ tbase, SwParams p,
                                                      SwResult* __restrict__ res, uint32_t* __restrict__ dir,
                                                      int rows_max, uint32_t* __restrict__ cig,
                                                      const int64_t* __restrict__ cig_off,
                                                      uint32_t* __restrict__ err) {
  constexpr int WW = (W + 7) / 8;
  const int lt = blockIdx.x * blockDim.x + threadIdx.x;  // pair index within this launch
  const int nn = n_dev ? min(n, *n_dev) : n;
  const int ia = base + 2 * lt, ib = ia + 1;
  if (ia >= nn) return;
  const bool has_b = ib < nn;
  const int lane = threadIdx.x & 31;
  // direction words: 64 alignments per warp, word (i, w) = [32 A lanes][32 B lanes]
  uint32_t* DA = TB ? dir + static_cast<size_t>(lt >> 5) * rows_max * WW * 64 + lane : nullptr;
  uint32_t* DB = TB ? DA + 32 : nullptr;
  const SwTask ta = tasks[ia];
  SwTask tb = ta;
  if (has_b) tb = tasks[ib];
  else tb.qlen = 0;
  const int qmax = max(ta.qlen, tb.qlen);
  const bool fits16 = qmax * p.match + 2 * (p.oe + p.ge + p.mismatch + p.ambig) < 30000;
  if (!fits16 || window_has_n(ta, W, tbase) || (has_b && window_has_n(tb, W, tbase))) {
    res[ta.slot] = sw_one_reg<W, TB>(ta, qbase, tbase, p, DA, 64, cig, cig_off, err);
    if (has_b) res[tb.slot] = sw_one_reg<W, TB>(tb, qbase, tbase, p, DB, 64, cig, cig_off, err);
    return;
  }
  const uint8_t* __restrict__ qa = qbase + ta.q_off;
  const uint8_t* __restrict__ qb = qbase + tb.q_off;
  const int qla = ta.qlen, qlb = tb.qlen;
  // a target code of A or B past its own window only feeds rows that cannot matter to it
  auto tc2 = [&](int64_t j) {
    const uint32_t a = tcode(tbase, ta, j), b = has_b ? tcode(tbase, tb, j) : 0u;
    return sel2(a > 3 ? 0u : a, b > 3 ? 0u : b);
  };
  uint32_t H[W + 1], E[W + 1], T[W];
#pragma unroll
  for (int d = 0; d <= W; ++d) {
    H[d] = 0;
    E[d] = 0;
  }
#pragma unroll
  for (int d = 0; d < W; ++d) T[d] = tc2(d);
  const uint32_t NOE = pack2(-p.oe), NGE = pack2(-p.ge), NEG = 0x80008000u;
  uint32_t best2 = 0;
  int best_a = 0, bi_a = -1, bd_a = -1, best_b = 0, bi_b = -1, bd_b = -1;
  for (int i = 0; i < qmax; ++i) {
    // rows past a query's end are N rows for it: they cannot raise its best (src of the
    // values only decreases) and its walk never reaches them
    const uint32_t ca = i < qla ? min(static_cast<uint32_t>(qa[i]), 4u) : 4u;
    const uint32_t cb = i < qlb ? min(static_cast<uint32_t>(qb[i]), 4u) : 4u;
    const uint32_t plo = prof_lo(p, ca), phi = prof_lo(p, cb);
    uint32_t f = 0, hleft = 0, hdiag = H[0], rmax = 0, dwa = 0, dwb = 0;
    int rda = -1, rdb = -1;
#pragma unroll
    for (int d = 0; d < W; ++d) {
      const uint32_t hup = H[d + 1], eup = E[d + 1];
      const uint32_t hd = __viaddmax_s16x2(hdiag, prmt(plo, phi, T[d]), NEG);
      bool peh, pel, pfh, pfl, p1h, p1l, p2h, p2l;
      const uint32_t e = __vibmax_s16x2(__viaddmax_s16x2(hup, NOE, NEG), __viaddmax_s16x2(eup, NGE, NEG), &peh, &pel);
      f = __vibmax_s16x2(__viaddmax_s16x2(hleft, NOE, NEG), __viaddmax_s16x2(f, NGE, NEG), &pfh, &pfl);
      const uint32_t m1 = __vibmax_s16x2(hd, e, &p1h, &p1l);
      const uint32_t h = __vimax_s16x2_relu(__vibmax_s16x2(m1, f, &p2h, &p2l), 0u);
      H[d] = h;
      E[d] = e;
      if constexpr (TB) {
        dwa |= dir_code(p1l, p2l, pel, pfl) << (4 * (d & 7));
        dwb |= dir_code(p1h, p2h, peh, pfh) << (4 * (d & 7));
        if ((d & 7) == 7 || d == W - 1) {
          const size_t o = (static_cast<size_t>(i) * WW + (d >> 3)) * 64;
          DA[o] = dwa;
          DB[o] = dwb;
          dwa = dwb = 0;
        }
        // row maximum, first strict occurrence; the row starts at cell 0 (every H >= 0,
        // so cell 0 is the first maximum of the cells seen so far)
        if (d == 0) {
          rmax = h;
          rda = rdb = 0;
        } else {
          bool rh, rl;
          rmax = __vibmax_s16x2(rmax, h, &rh, &rl);
          if (!rl) rda = d;
          if (!rh) rdb = d;
        }
      } else {
        best2 = __vimax_s16x2_relu(best2, h);
      }
      hleft = h;
      hdiag = hup;
    }
    if constexpr (TB) {
      if (lo16(rmax) > best_a) {
        best_a = lo16(rmax);
        bi_a = i;
        bd_a = rda;
      }
      if (hi16(rmax) > best_b) {
        best_b = hi16(rmax);
        bi_b = i;
        bd_b = rdb;
      }
    }
#pragma unroll
    for (int d = 0; d + 1 < W; ++d) T[d] = T[d + 1];
    T[W - 1] = tc2(static_cast<int64_t>(i) + W);
  }
  if constexpr (!TB) {
    best_a = lo16(best2);
    best_b = hi16(best2);
  }
  SwResult ra{best_a, 0, 0, 0, 0, 0, 0, 0};
  if (TB && best_a > 0)
    traceback(DA, 64, WW, W, bi_a, bd_a, best_a, qa, tbase, ta, p, ra, cig + cig_off[ta.slot], 2 * qla + 1, err);
  res[ta.slot] = ra;
  if (has_b) {
    SwResult rb{best_b, 0, 0, 0, 0, 0, 0, 0};
    if (TB && best_b > 0)
      traceback(DB, 64, WW, W, bi_b, bd_b, best_b, qb, tbase, tb, p, rb, cig + cig_off[tb.slot], 2 * qlb + 1, err);
    res[tb.slot] = rb;
  }
}

// Any band width and any scores: one alignment per thread, int32, band rows H, E in
// per-warp scratch, lane-interleaved ([d][lane]).
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
      bool pe, pf, p1, p2;
      const int e = __vibmax_s32(hup - p.oe, eup - p.ge, &pe);
      f = __vibmax_s32(hleft - p.oe, f - p.ge, &pf);
      const int m1 = __vibmax_s32(hd, e, &p1);
      const int h = __vimax_s32_relu(__vibmax_s32(m1, f, &p2), 0);
      Hs[d * 32] = h;
      Es[d * 32] = e;
      if (TB) {
        dw |= dir_code(p1, p2, pe, pf) << (4 * (d & 7));
        if ((d & 7) == 7 || d == W - 1) {
          D[(static_cast<size_t>(i) * WW + (d >> 3)) * 32] = dw;
          dw = 0;
        }
        bool pr;
        rmax = __vibmax_s32(rmax, h, &pr);
        if (!pr) rd = d;
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
    traceback(D, 32, WW, W, bi, bd, best, q, tbase, tk, p, r, cig + cig_off[tk.slot], 2 * ql + 1, err);
  res[tk.slot] = r;
}

template <int W>
void launch_x2(cudaStream_t st, bool tb, const SwTask* tasks, int base, int count, int n, const int* n_dev,
               const uint8_t* qbase, const uint8_t* tbase, const SwParams& p, SwResult* res, uint32_t* dir,
               int rows_max, uint32_t* cig, const int64_t* cig_off, uint32_t* err) {
  const int pairs = (count + 1) / 2;
  const int blocks = (pairs + kSwThreads - 1) / kSwThreads;
  if (tb)
    k_sw_x2<W, true><<<blocks, kSwThreads, 0, st>>>(tasks, base, n, n_dev, qbase, tbase, p, res, dir, rows_max, cig,
                                                    cig_off, err);
  else
    k_sw_x2<W, false><<<blocks, kSwThreads, 0, st>>>(tasks, base, n, n_dev, qbase, tbase, p, res, dir, rows_max, cig,
                                                     cig_off, err);
}

}  // namespace

bool sw_bytes_ok(const dnaln_score_params& s) {
  return s.match <= 127 && s.mismatch <= 128 && s.ambig <= 128 && s.match >= -128;
}

bool sw_band_in_registers(int W) { return W == 11 || W == 17 || W == 33 || W == 43 || W == 65; }

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
  return static_cast<size_t>(rows_max > 0 ? rows_max : 1) * ((W + 7) / 8) * sizeof(uint32_t);
}

size_t sw_band_bytes_per_task(int W, bool bytes_ok) {
  return sw_uses_generic(W, bytes_ok) ? static_cast<size_t>(2) * (W + 1) * sizeof(int) : 0;
}

bool launch_sw(cudaStream_t st, bool tb, bool bytes_ok, const SwTask* tasks, int base, int count, int n,
               const int* n_dev, const uint8_t* qbase, const uint8_t* tbase, const SwParams& p, SwResult* res,
               uint32_t* dir, int rows_max, uint32_t* cig, const int64_t* cig_off, int* band, uint32_t* err) {
  if (count <= 0) return true;
  if ((tb && !dir) || (sw_uses_generic(p.W, bytes_ok) && !band) || (base % kSwTaskGroup) != 0) return false;
  if (bytes_ok) {
#define DNB_SW_X2(WV)                                                                                       \
  case WV:                                                                                                  \
    launch_x2<WV>(st, tb, tasks, base, count, n, n_dev, qbase, tbase, p, res, dir, rows_max, cig, cig_off, \
                  err);                                                                                     \
    return true;
    switch (p.W) {
      DNB_SW_X2(11)
      DNB_SW_X2(17)
      DNB_SW_X2(33)
      DNB_SW_X2(43)
      DNB_SW_X2(65)
      default: break;
    }
#undef DNB_SW_X2
  }
  const int blocks = (count + kSwThreads - 1) / kSwThreads;
  if (tb)
    k_sw_any<true><<<blocks, kSwThreads, 0, st>>>(tasks, base, n, n_dev, qbase, tbase, p, res, dir, rows_max, cig,
                                                 cig_off, band, err);
  else
    k_sw_any<false><<<blocks, kSwThreads, 0, st>>>(tasks, base, n, n_dev, qbase, tbase, p, res, dir, rows_max, cig,
                                                  cig_off, band, err);
  return true;
}

}  // namespace dnb
