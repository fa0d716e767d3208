// sam.cpp — SAM text for mapped batches, Mapper::append_sam (src/mapper.cpp:231-270).
//
// Fields: QNAME, FLAG 0/16/4, RNAME, 1-based POS, MAPQ, CIGAR (soft clips included),
// "*\t0\t0", SEQ and QUAL (reverse complement / reversed for reverse-strand hits), NM:i,
// AS:i. Unmapped reads print "4\t*\t0\t0\t*\t*\t0\t0" and SEQ/QUAL as given.
#include <algorithm>
#include <charconv>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "dnaln_b200.h"

namespace {

// Complement of an ASCII base as the reference writes it: A/C/G/T and lowercase a/c/g/t
// complemented, 'n' kept, everything else 'N' (src/common.cpp:5-14).
char comp_char(char c) {
  switch (c) {
    case 'A': return 'T';
    case 'C': return 'G';
    case 'G': return 'C';
    case 'T': return 'A';
    case 'a': return 't';
    case 'c': return 'g';
    case 'g': return 'c';
    case 't': return 'a';
    case 'n': return 'n';
    default: return 'N';
  }
}

struct Out {
  char* p;
  int64_t cap, n;
  void put(const char* s, int64_t len) {
    if (len > 0 && n + len <= cap) std::memcpy(p + n, s, static_cast<size_t>(len));
    n += len;
  }
  void put(const char* s) { put(s, static_cast<int64_t>(std::strlen(s))); }
  void put(char c) {
    if (n < cap) p[n] = c;
    ++n;
  }
  void num(long long v) {
    char b[24];
    const auto r = std::to_chars(b, b + sizeof b, v);
    put(b, r.ptr - b);
  }
};

constexpr char kCigOps[] = "MIDNSHP=X";

// Appends the SAM lines of records [a, b) to o.
void format_range(const char* seq, const int64_t* seq_off, const int32_t* seq_len, const char* names,
                  const int64_t* name_off, const char* qual, const int64_t* qual_off, const dnaln_map_record* rec,
                  const uint32_t* cigar, int64_t a, int64_t b, const char* cnames, const int64_t* cname_off, Out& o);

}  // namespace

extern "C" int dnaln_sam_format(const char* seq, const int64_t* seq_off, const int32_t* seq_len, const char* names,
                                const int64_t* name_off, const char* qual, const int64_t* qual_off,
                                const dnaln_map_record* rec, const uint32_t* cigar, int64_t n, const char* cnames,
                                const int64_t* cname_off, char* out, int64_t cap, int64_t* used) {
  if (n < 0 || !used || (n > 0 && (!seq || !seq_off || !seq_len || !names || !name_off || !rec)))
    return DNALN_ERR_INVALID_ARG;
  Out o{out, out ? cap : 0, 0};
  format_range(seq, seq_off, seq_len, names, name_off, qual, qual_off, rec, cigar, 0, n, cnames, cname_off, o);
  *used = o.n;
  return o.n <= cap ? DNALN_OK : DNALN_ERR_CAPACITY;
}

namespace {

void format_range(const char* seq, const int64_t* seq_off, const int32_t* seq_len, const char* names,
                  const int64_t* name_off, const char* qual, const int64_t* qual_off, const dnaln_map_record* rec,
                  const uint32_t* cigar, int64_t a, int64_t b, const char* cnames, const int64_t* cname_off, Out& o) {
  for (int64_t r = a; r < b; ++r) {
    const char* s = seq + seq_off[r];
    const int64_t len = seq_len[r];
    const char* q = qual ? qual + qual_off[r] : nullptr;
    const int64_t qlen = qual ? qual_off[r + 1] - qual_off[r] : 0;
    o.put(names + name_off[r], name_off[r + 1] - name_off[r]);
    const dnaln_map_record& m = rec[r];
    if (m.contig < 0) {
      o.put("\t4\t*\t0\t0\t*\t*\t0\t0\t");
      if (len) o.put(s, len);
      else o.put('*');
      o.put('\t');
      if (qlen) o.put(q, qlen);
      else o.put('*');
      o.put('\n');
      continue;
    }
    o.put('\t');
    o.num(m.rev ? 16 : 0);
    o.put('\t');
    o.put(cnames + cname_off[m.contig], cname_off[m.contig + 1] - cname_off[m.contig]);
    o.put('\t');
    o.num(m.pos + 1);
    o.put('\t');
    o.num(m.mapq);
    o.put('\t');
    for (int32_t i = 0; i < m.cigar_len; ++i) {
      const uint32_t c = cigar[m.cigar_off + i];
      o.num(c >> 4);
      o.put(kCigOps[c & 0xf]);
    }
    o.put("\t*\t0\t0\t");
    if (m.rev) {
      for (int64_t i = len - 1; i >= 0; --i) o.put(comp_char(s[i]));
      o.put('\t');
      if (!qlen) o.put('*');
      else
        for (int64_t i = qlen - 1; i >= 0; --i) o.put(q[i]);
    } else {
      o.put(s, len);
      o.put('\t');
      if (qlen) o.put(q, qlen);
      else o.put('*');
    }
    o.put("\tNM:i:");
    o.num(m.nm);
    o.put("\tAS:i:");
    o.num(m.score);
    o.put('\n');
  }
}

}  // namespace

// The same text as dnaln_sam_format, formatted by several host threads over contiguous
// ranges of records: a counting pass gives each range's exact size, then every thread
// writes its range straight into `out` at its offset.
extern "C" int dnaln_sam_format_mt(const char* seq, const int64_t* seq_off, const int32_t* seq_len,
                                   const char* names, const int64_t* name_off, const char* qual,
                                   const int64_t* qual_off, const dnaln_map_record* rec, const uint32_t* cigar,
                                   int64_t n, const char* cnames, const int64_t* cname_off, int32_t threads, char* out,
                                   int64_t cap, int64_t* used) {
  if (n < 0 || !used || (n > 0 && (!seq || !seq_off || !seq_len || !names || !name_off || !rec)))
    return DNALN_ERR_INVALID_ARG;
  int t = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
  if (t < 1) t = 1;
  if (static_cast<int64_t>(t) * 4096 > n) t = static_cast<int>(std::max<int64_t>(1, n / 4096));
  if (t == 1)
    return dnaln_sam_format(seq, seq_off, seq_len, names, name_off, qual, qual_off, rec, cigar, n, cnames, cname_off,
                            out, cap, used);
  // pass 1: the exact bytes of each thread's range (formatting into nothing counts them);
  // pass 2: each thread formats its range straight into `out` at its offset
  std::vector<int64_t> at(static_cast<size_t>(t) + 1, 0);
  const auto range = [&](int i, int64_t& a, int64_t& b) {
    a = n * i / t;
    b = n * (i + 1) / t;
  };
  const auto parallel = [&](auto&& f) {
    std::vector<std::thread> th;
    for (int i = 1; i < t; ++i) th.emplace_back(f, i);
    f(0);
    for (auto& x : th) x.join();
  };
  parallel([&](int i) {
    int64_t a, b;
    range(i, a, b);
    Out o{nullptr, 0, 0};
    format_range(seq, seq_off, seq_len, names, name_off, qual, qual_off, rec, cigar, a, b, cnames, cname_off, o);
    at[static_cast<size_t>(i) + 1] = o.n;
  });
  for (int i = 0; i < t; ++i) at[static_cast<size_t>(i) + 1] += at[static_cast<size_t>(i)];
  *used = at.back();
  if (!out || at.back() > cap) return DNALN_ERR_CAPACITY;
  parallel([&](int i) {
    int64_t a, b;
    range(i, a, b);
    Out o{out + at[static_cast<size_t>(i)], at[static_cast<size_t>(i) + 1] - at[static_cast<size_t>(i)], 0};
    format_range(seq, seq_off, seq_len, names, name_off, qual, qual_off, rec, cigar, a, b, cnames, cname_off, o);
  });
  return DNALN_OK;
}
