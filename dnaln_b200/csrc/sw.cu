// sw.cu — banded affine-gap Smith–Waterman (score-only and with traceback) for sm_100a.
//
// Inter-sequence layout: one alignment per thread, the whole band row (H, E of the W+1
// band cells and the W target codes under the band) held in registers for the band
// widths listed in sw_band_in_registers(), so a cell update is pure register ALU work. The recurrence is the
// reference's diagonal-coordinate band (src/align.hpp:3-15, src/align.cpp:31-84):
//   hd = H(i-1,d) + s(q_i, t_{i+d});  E(i,d) = max(H(i-1,d+1) - (O+E), E(i-1,d+1) - E)
//   F(i,d) = max(H(i,d-1) - (O+E), F(i,d-1) - E);  H(i,d) = max(hd, E, 0, F)
// with H = E = 0 for row -1 and for the fixed out-of-band cell d = W, and F = H(left) = 0
// at the start of every row. Scores are int32, so every band width and read length is
// exact (the reference's int16 SIMD kernel falls back to int32 above 30000/match bp).
//
// The substitution score is one byte-permute (PTX prmt.b32) per cell: each row builds an
// 8-byte profile {s(q_i, A), s(q_i, C), s(q_i, G), s(q_i, T), s(q_i, N) x4} and the
// register holding target column i+d is a PRMT selector that returns the sign-extended
// profile byte of that base.
//
// Traceback: 4 direction bits per cell — H from the diagonal (h == hd), H from E
// (h == e), E extends (ee > eo), F extends (fe > fo), the bits of src/align.cpp:67-68 —
// packed 8 cells per 32-bit word and stored lane-interleaved (word (i, d/8) of the 32
// lanes of a warp is one 128-byte line), then walked by the same thread exactly as
// src/align.cpp:87-143. The best cell is the first strict maximum in row-major order.
#include <cstdio>

#include "common.cuh"
#include "sw.cuh"

namespace dnb {

namespace {

constexpr int kSwThreads = 128;

// PRMT selector returning the sign-extended byte c (0..7) of the {hi:lo} profile: result
// byte 0 copies byte c, bytes 1-3 replicate its sign (selector nibble msb set).
__device__ __forceinline__ uint32_t prof_sel(uint32_t c) {
  const uint32_t s = c | 8u;
  return c | (s << 4) | (s << 8) | (s << 12);
}

// prmt.b32 in its default mode, which honours the sign-replicate bit of each selector
// nibble (the __byte_perm intrinsic uses only the low 3 bits of each nibble).
__device__ __forceinline__ int prmt_score(uint32_t lo, uint32_t hi, uint32_t sel) {
  uint32_t r;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(lo), "r"(hi), "r"(sel));
  return static_cast<int>(r);
}

__device__ __forceinline__ uint32_t tcode(const uint8_t* __restrict__ tbase, const SwTask& tk, int64_t j) {
  const int64_t x = tk.t_start + j;
  if (x < tk.t_lo || x >= tk.t_hi) return 4;
  const uint32_t c = __ldg(tbase + x);
  return c > 3 ? 4u : c;
}

// Low profile word of query code qc: byte t = match if t == qc else -mismatch; an N
// query row scores -ambig everywhere.
__device__ __forceinline__ uint32_t prof_lo(const SwParams& p, uint32_t qc) {
  if (qc > 3) return p.prof_n;
  const uint32_t mm = (static_cast<uint32_t>(static_cast<uint8_t>(-p.mismatch))) * 0x01010101u;
  const uint32_t sh = 8u * qc;
  return (mm & ~(0xFFu << sh)) | (static_cast<uint32_t>(static_cast<uint8_t>(p.match)) << sh);
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

// Walks the direction nibbles back from (bi, bd) (src/align.cpp:87-143). `D` points at
// this lane's first word; word (i, w) is D[(i * WW + w) * 32]. CIGAR ops are written in
// walk order (last op first); merging of adjacent equal ops as the reference's push().
__device__ void traceback(const uint32_t* __restrict__ D, int WW, int W, int bi, int bd, int best,
                          const uint8_t* __restrict__ q, const uint8_t* __restrict__ tbase, const SwTask& tk,
                          const SwParams& p, SwResult& r, uint32_t* __restrict__ cig, int cap,
                          uint32_t* __restrict__ err) {
  auto nib = [&](int i, int d) -> uint32_t {
    return (D[(static_cast<size_t>(i) * WW + (d >> 3)) * 32] >> (4 * (d & 7))) & 0xFu;
  };
  CigarWriter cw{cig, cap, 0, 0xFu, 0};
  int i = bi, d = bd, v = best, nm = 0;
  for (;;) {
    int run = 0;
    uint32_t x = 0;
    while (i >= 0 && v > 0) {
      x = nib(i, d);
      if (!(x & 8u)) break;
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
    if (x & 4u) {  // insertion: E(i,d) <- (i-1, d+1)
      do {
        if (i < 0 || d >= W) {
          atomicOr(err, kErrTracebackBounds);
          goto done;
        }
        ext = (nib(i, d) & 2u) != 0;
        v += ext ? p.ge : p.oe;
        ++run;
        --i;
        ++d;
      } while (ext);
      cw.push(1u /* I */, run);
    } else {  // deletion: F(i,d) <- (i, d-1)
      do {
        if (d < 0 || d >= W) {
          atomicOr(err, kErrTracebackBounds);
          goto done;
        }
        ext = (nib(i, d) & 1u) != 0;
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

// Register-resident band of compile-time width W.
template <int W, bool TB>
__global__ void __launch_bounds__(kSwThreads) k_sw_reg(const SwTask* __restrict__ tasks, int base, int n,
                                                       const int* __restrict__ n_dev,
                                                       const uint8_t* __restrict__ qbase,
                                                       const uint8_t* __restrict__ tbase, SwParams p,
                                                       SwResult* __restrict__ res, uint32_t* __restrict__ dir,
                                                       int rows_max, uint32_t* __restrict__ cig,
                                                       const int64_t* __restrict__ cig_off,
                                                       uint32_t* __restrict__ err) {
  constexpr int WW = (W + 7) / 8;
  const int lt = blockIdx.x * blockDim.x + threadIdx.x;  // index within this launch
  const int gt = base + lt;
  if (gt >= (n_dev ? min(n, *n_dev) : n)) return;
  const int lane = threadIdx.x & 31;
  const SwTask tk = tasks[gt];
  const uint8_t* __restrict__ q = qbase + tk.q_off;
  const int ql = tk.qlen;
  uint32_t* D = TB ? dir + (static_cast<size_t>(lt >> 5) * rows_max * WW) * 32 + lane : nullptr;

  int H[W + 1], E[W + 1];
  uint32_t T[W];
#pragma unroll
  for (int d = 0; d <= W; ++d) {
    H[d] = 0;
    E[d] = 0;
  }
#pragma unroll
  for (int d = 0; d < W; ++d) T[d] = prof_sel(tcode(tbase, tk, d));

  int best = 0, bi = -1, bd = -1;
  for (int i = 0; i < ql; ++i) {
    const uint32_t qc = min(static_cast<uint32_t>(q[i]), 4u);
    const uint32_t plo = prof_lo(p, qc), phi = p.prof_n;
    int f = 0, hleft = 0, hdiag = H[0];
    uint32_t dw = 0;
#pragma unroll
    for (int d = 0; d < W; ++d) {
      const int hup = H[d + 1], eup = E[d + 1];
      const int hd = hdiag + prmt_score(plo, phi, T[d]);
      const int eo = hup - p.oe, ee = eup - p.ge;
      const int e = max(eo, ee);
      const int fo = hleft - p.oe, fe = f - p.ge;
      f = max(fo, fe);
      const int h = max(max(max(hd, e), 0), f);
      H[d] = h;
      E[d] = e;
      if constexpr (TB) {
        const uint32_t nb = (h == hd ? 8u : 0u) | (h == e ? 4u : 0u) | (ee > eo ? 2u : 0u) | (fe > fo ? 1u : 0u);
        dw |= nb << (4 * (d & 7));
        if ((d & 7) == 7 || d == W - 1) {
          D[(static_cast<size_t>(i) * WW + (d >> 3)) * 32] = dw;
          dw = 0;
        }
        if (h > best) {
          best = h;
          bi = i;
          bd = d;
        }
      } else {
        best = max(best, h);
      }
      hleft = h;
      hdiag = hup;
    }
#pragma unroll
    for (int d = 0; d + 1 < W; ++d) T[d] = T[d + 1];
    T[W - 1] = prof_sel(tcode(tbase, tk, static_cast<int64_t>(i) + W));
  }
  SwResult r{best, 0, 0, 0, 0, 0, 0, 0};
  if (TB && best > 0)
    traceback(D, WW, W, bi, bd, best, q, tbase, tk, p, r, cig + cig_off[tk.slot], 2 * ql + 1, err);
  res[tk.slot] = r;
}

// Any band width: H, E and the target codes under the band live in per-warp global
// scratch, lane-interleaved ([d][lane]), which stays in L1/L2 for the alignment.
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
    int f = 0, hleft = 0, hdiag = Hs[0];
    uint32_t dw = 0;
    for (int d = 0; d < W; ++d) {
      const int hup = Hs[(d + 1) * 32], eup = Es[(d + 1) * 32];
      const int tc = static_cast<int>(tcode(tbase, tk, static_cast<int64_t>(i) + d));
      const int hd = hdiag + sub_score(p, qc, tc);
      const int eo = hup - p.oe, ee = eup - p.ge;
      const int e = max(eo, ee);
      const int fo = hleft - p.oe, fe = f - p.ge;
      f = max(fo, fe);
      const int h = max(max(max(hd, e), 0), f);
      Hs[d * 32] = h;
      Es[d * 32] = e;
      if (TB) {
        const uint32_t nb = (h == hd ? 8u : 0u) | (h == e ? 4u : 0u) | (ee > eo ? 2u : 0u) | (fe > fo ? 1u : 0u);
        dw |= nb << (4 * (d & 7));
        if ((d & 7) == 7 || d == W - 1) {
          D[(static_cast<size_t>(i) * WW + (d >> 3)) * 32] = dw;
          dw = 0;
        }
        if (h > best) {
          best = h;
          bi = i;
          bd = d;
        }
      } else {
        best = max(best, h);
      }
      hleft = h;
      hdiag = hup;
    }
  }
  SwResult r{best, 0, 0, 0, 0, 0, 0, 0};
  if (TB && best > 0)
    traceback(D, WW, W, bi, bd, best, q, tbase, tk, p, r, cig + cig_off[tk.slot], 2 * ql + 1, err);
  res[tk.slot] = r;
}

template <int W>
void launch_reg(cudaStream_t st, bool tb, const SwTask* tasks, int base, int count, int n, const int* n_dev,
                const uint8_t* qbase, const uint8_t* tbase, const SwParams& p, SwResult* res, uint32_t* dir,
                int rows_max, uint32_t* cig, const int64_t* cig_off, uint32_t* err) {
  const int blocks = (count + kSwThreads - 1) / kSwThreads;
  if (tb)
    k_sw_reg<W, true><<<blocks, kSwThreads, 0, st>>>(tasks, base, n, n_dev, qbase, tbase, p, res, dir, rows_max, cig,
                                                     cig_off, err);
  else
    k_sw_reg<W, false><<<blocks, kSwThreads, 0, st>>>(tasks, base, n, n_dev, qbase, tbase, p, res, dir, rows_max,
                                                      cig, cig_off, err);
}

}  // namespace

bool sw_bytes_ok(const dnaln_score_params& s) {
  return s.match <= 127 && s.mismatch <= 128 && s.ambig <= 128 && s.match >= -128;
}

bool sw_band_in_registers(int W) { return W == 11 || W == 17 || W == 33 || W == 43 || W == 65; }

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

size_t sw_dir_bytes_per_warp(int W, int rows_max) {
  return static_cast<size_t>(rows_max) * ((W + 7) / 8) * 32 * sizeof(uint32_t);
}

bool sw_uses_generic(int W, bool bytes_ok) { return !(bytes_ok && sw_band_in_registers(W)); }

size_t sw_band_bytes_per_warp(int W, bool bytes_ok) {
  return sw_uses_generic(W, bytes_ok) ? static_cast<size_t>(2) * (W + 1) * 32 * sizeof(int) : 0;
}

bool launch_sw(cudaStream_t st, bool tb, bool bytes_ok, const SwTask* tasks, int base, int count, int n,
               const int* n_dev, const uint8_t* qbase, const uint8_t* tbase, const SwParams& p, SwResult* res,
               uint32_t* dir, int rows_max, uint32_t* cig, const int64_t* cig_off, int* band, uint32_t* err) {
  if (count <= 0) return true;
  if ((tb && !dir) || (sw_uses_generic(p.W, bytes_ok) && !band)) return false;  // scratch missing: never launch
  if (bytes_ok) {
#define DNB_SW_REG(WV)                                                                                      \
  case WV:                                                                                                  \
    launch_reg<WV>(st, tb, tasks, base, count, n, n_dev, qbase, tbase, p, res, dir, rows_max, cig, cig_off, \
                   err);                                                                                    \
    return true;
    switch (p.W) {
      DNB_SW_REG(11)
      DNB_SW_REG(17)
      DNB_SW_REG(33)
      DNB_SW_REG(43)
      DNB_SW_REG(65)
      default: break;
    }
#undef DNB_SW_REG
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
