// synth.cpp — seeded synthetic genomes and reads (see include/dnaln_synth.h).
//
// Read model (the mapping workloads' error model): start uniform over positions where the
// read fits in its contig, strand 50/50 (reverse-complemented when minus). Walking the
// reference from the start, each emitted base is substituted with probability `sub` to one
// of the other three bases uniformly; after a non-indel base, with probability `indel` an
// indel is placed instead, insertion or deletion with equal odds, its length geometric(p)
// capped at indel_cap. Reads that would cross an N or a contig end are redrawn. A
// `big_del_frac` share of reads carries one extra deletion of big_del_min..big_del_max bp
// at a uniform interior read offset.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "dnaln_synth.h"

namespace {

// xoshiro256** (Blackman & Vigna) seeded by splitmix64, the generator family the
// reference's tools use (src/common.hpp:80-107).
class Xoshiro {
 public:
  explicit Xoshiro(uint64_t seed) {
    for (int i = 0; i < 4; ++i) {
      seed += 0x9e3779b97f4a7c15ULL;
      uint64_t z = seed;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      s_[i] = z ^ (z >> 31);
    }
  }
  uint64_t next() {
    const uint64_t out = rotl(s_[1] * 5, 7) * 9;
    const uint64_t t = s_[1] << 17;
    s_[2] ^= s_[0];
    s_[3] ^= s_[1];
    s_[1] ^= s_[2];
    s_[0] ^= s_[3];
    s_[2] ^= t;
    s_[3] = rotl(s_[3], 45);
    return out;
  }
  double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }
  uint64_t below(uint64_t n) { return next() % n; }

 private:
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t s_[4];
};

constexpr char kAcgt[] = "ACGT";

uint8_t draw_base(Xoshiro& r, double gc) {
  const double u = r.uniform();
  if (u < gc / 2) return 2;  // G
  if (u < gc) return 1;      // C
  if (u < gc + (1 - gc) / 2) return 0;  // A
  return 3;  // T
}

int32_t draw_len(Xoshiro& r, const dnaln_synth_reads_spec& s) {
  if (s.len_dist == 1) {
    const double a = std::log(static_cast<double>(s.len_min)), b = std::log(static_cast<double>(s.len_max));
    int32_t L = static_cast<int32_t>(std::lround(std::exp(a + (b - a) * r.uniform())));
    return L < s.len_min ? s.len_min : (L > s.len_max ? s.len_max : L);
  }
  if (s.len_dist == 2) return s.len_min + static_cast<int32_t>(r.below(static_cast<uint64_t>(s.len_max - s.len_min + 1)));
  return s.len_min;
}

uint64_t len_seed(uint64_t seed) { return seed * 0x2545F4914F6CDD1DULL + 0x5851F42D4C957F2DULL; }

}  // namespace

extern "C" {

int dnaln_synth_genome(uint64_t seed, const dnaln_synth_genome_spec* sp, uint8_t* out) {
  if (!sp || !out || sp->n_contigs < 1) return 1;
  const dnaln_synth_genome_spec& s = *sp;
  Xoshiro r(seed);
  const uint64_t L = s.contig_len, total = L * static_cast<uint64_t>(s.n_contigs);
  for (uint64_t i = 0; i < total; ++i) out[i] = draw_base(r, s.gc);
  // Repeat units, each copied (with per-copy substitutions, random strand) over random
  // positions inside one contig until repeat_frac of the genome is covered.
  if (s.n_repeat_units > 0 && s.repeat_unit_len > 0 && s.repeat_frac > 0 &&
      static_cast<uint64_t>(s.repeat_unit_len) < L) {
    const int U = s.n_repeat_units, UL = s.repeat_unit_len;
    std::vector<uint8_t> units(static_cast<size_t>(U) * UL);
    for (auto& b : units) b = draw_base(r, s.gc);
    const uint64_t copies = static_cast<uint64_t>(std::llround(s.repeat_frac * static_cast<double>(total) / UL));
    std::vector<uint8_t> cp(static_cast<size_t>(UL));
    for (uint64_t c = 0; c < copies; ++c) {
      const uint8_t* u = units.data() + static_cast<size_t>(c % U) * UL;
      for (int i = 0; i < UL; ++i) {
        uint8_t b = u[i];
        if (r.uniform() < s.repeat_div) b = static_cast<uint8_t>((b + 1 + r.below(3)) & 3);
        cp[static_cast<size_t>(i)] = b;
      }
      if (r.next() & 1) {  // reverse complement
        int i = 0, j = UL - 1;
        for (; i < j; ++i, --j) {
          const uint8_t x = cp[static_cast<size_t>(i)], y = cp[static_cast<size_t>(j)];
          cp[static_cast<size_t>(i)] = static_cast<uint8_t>(3 - y);
          cp[static_cast<size_t>(j)] = static_cast<uint8_t>(3 - x);
        }
        if (i == j) cp[static_cast<size_t>(i)] = static_cast<uint8_t>(3 - cp[static_cast<size_t>(i)]);
      }
      const uint64_t ci = r.below(static_cast<uint64_t>(s.n_contigs));
      const uint64_t at = ci * L + r.below(L - static_cast<uint64_t>(UL));
      std::memcpy(out + at, cp.data(), static_cast<size_t>(UL));
    }
  }
  // N runs until n_frac of the genome is covered (runs may overlap).
  if (s.n_frac > 0 && s.n_run_max >= s.n_run_min && s.n_run_min > 0) {
    const uint64_t want = static_cast<uint64_t>(s.n_frac * static_cast<double>(total));
    uint64_t placed = 0;
    while (placed < want) {
      const uint64_t len = static_cast<uint64_t>(s.n_run_min) + r.below(static_cast<uint64_t>(s.n_run_max - s.n_run_min + 1));
      if (len >= L) break;
      const uint64_t ci = r.below(static_cast<uint64_t>(s.n_contigs));
      const uint64_t at = ci * L + r.below(L - len);
      std::memset(out + at, 4, static_cast<size_t>(len));
      placed += len;
    }
  }
  return 0;
}

int64_t dnaln_synth_reads_bytes(uint64_t seed, const dnaln_synth_reads_spec* sp) {
  Xoshiro lr(len_seed(seed));
  int64_t b = 0;
  for (int64_t i = 0; i < sp->n_reads; ++i) b += draw_len(lr, *sp);
  return b;
}

int dnaln_synth_reads(uint64_t seed, const uint8_t* genome, const uint64_t* contig_off, const uint32_t* contig_len,
                      int32_t n_contigs, const dnaln_synth_reads_spec* sp, char* out_seq, int64_t seq_cap,
                      int64_t* out_seq_off, char* out_names, int64_t names_cap, int64_t* out_name_off,
                      int32_t* truth_contig, int64_t* truth_start, uint8_t* truth_rev) {
  if (!sp || n_contigs < 1) return 1;
  const dnaln_synth_reads_spec& s = *sp;
  Xoshiro r(seed), lr(len_seed(seed));
  std::vector<uint8_t> rd;
  int64_t so = 0, no = 0;
  for (int64_t i = 0; i < s.n_reads; ++i) {
    const int32_t L = draw_len(lr, s);
    const bool big = s.big_del_frac > 0 && r.uniform() < s.big_del_frac;
    const int32_t big_len = big ? s.big_del_min + static_cast<int32_t>(r.below(static_cast<uint64_t>(s.big_del_max - s.big_del_min + 1))) : 0;
    const int32_t big_at = big ? 1 + static_cast<int32_t>(r.below(static_cast<uint64_t>(L > 2 ? L - 2 : 1))) : -1;
    // room for the read plus its worst-case deletions
    const uint64_t span = static_cast<uint64_t>(L) * 2 + static_cast<uint64_t>(big_len) + 16;
    int32_t ci = 0;
    int64_t start = 0;
    for (int attempt = 0;; ++attempt) {
      if (attempt > 100000) return 2;  // genome mostly N or contigs too short
      ci = static_cast<int32_t>(r.below(static_cast<uint64_t>(n_contigs)));
      if (contig_len[ci] <= span) continue;
      start = static_cast<int64_t>(r.below(contig_len[ci] - span));
      const int64_t gbeg = static_cast<int64_t>(contig_off[ci]) + start;
      const int64_t gend = static_cast<int64_t>(contig_off[ci]) + contig_len[ci];
      rd.clear();
      int64_t rp = gbeg;
      bool ok = true, after_indel = false;
      while (static_cast<int32_t>(rd.size()) < L) {
        if (rp >= gend) {
          ok = false;
          break;
        }
        if (big && static_cast<int32_t>(rd.size()) == big_at && big_len > 0 && !after_indel) {
          rp += big_len;
          after_indel = true;
          continue;
        }
        if (!rd.empty() && !after_indel && r.uniform() < s.indel) {
          int32_t len = 1;
          while (len < s.indel_cap && r.uniform() >= s.indel_geom_p) ++len;
          if (r.uniform() < 0.5) {
            if (static_cast<int32_t>(rd.size()) + len >= L) continue;
            for (int32_t x = 0; x < len; ++x) rd.push_back(static_cast<uint8_t>(r.below(4)));
          } else {
            rp += len;
          }
          after_indel = true;
          continue;
        }
        after_indel = false;
        if (rp >= gend) {
          ok = false;
          break;
        }
        uint8_t b = genome[rp];
        if (b > 3) {
          ok = false;
          break;
        }
        if (r.uniform() < s.sub) b = static_cast<uint8_t>((b + 1 + r.below(3)) & 3);
        rd.push_back(b);
        ++rp;
      }
      if (ok) break;
    }
    const bool rev = r.next() & 1;
    if (so + L > seq_cap) return 3;
    out_seq_off[i] = so;
    for (int32_t x = 0; x < L; ++x)
      out_seq[so + x] = rev ? kAcgt[3 - rd[static_cast<size_t>(L - 1 - x)]] : kAcgt[rd[static_cast<size_t>(x)]];
    so += L;
    const std::string nm = "sim_" + std::to_string(s.name_base + i);
    if (no + static_cast<int64_t>(nm.size()) > names_cap) return 4;
    out_name_off[i] = no;
    std::memcpy(out_names + no, nm.data(), nm.size());
    no += static_cast<int64_t>(nm.size());
    if (truth_contig) truth_contig[i] = ci;
    if (truth_start) truth_start[i] = start;
    if (truth_rev) truth_rev[i] = rev;
  }
  out_seq_off[s.n_reads] = so;
  out_name_off[s.n_reads] = no;
  return 0;
}

}  // extern "C"
