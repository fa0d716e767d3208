// reads.cpp — FASTA/FASTQ text to the batch layout of dnaln_gpu_map_batch, on several host
// threads: SeqReader::next (src/seqio.cpp:59-80) over an in-memory buffer.
//
// The reference's reader, restated for a buffer: lines end at '\n' with one trailing '\r'
// dropped; lines before a record that do not start with '>' or '@' are skipped; the name is
// the header after its first byte up to the first space or tab; sequence lines are
// appended until a line starting with '>', '+' or '@'; a FASTQ record then needs a '+' line
// and takes quality lines until they are at least as long as the sequence, and their
// lengths must match. That sequential parser is the definition, and the one-thread path.
//
// With several threads, text made of plain four-line FASTQ records is split into chunks:
// each chunk starts at the first line that begins with '@' and whose second next line
// begins with '+' (in such a file only headers do: a quality line that begins with '@' is
// followed, two lines down, by a sequence line), and every thread checks that its records
// have exactly that shape (header, one sequence line not starting with '>', '+' or '@', a
// '+' line, one quality line as long as the sequence; lines between records that start
// neither '>' nor '@' are skipped, as the reference skips them) and ends exactly where the
// next chunk starts. Any record that does not fit makes the whole buffer go through the
// sequential parser, so the result never differs from it.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "dnaln_b200.h"

#include <memory>

struct dnaln_reads {  // arrays left uninitialised at allocation: every byte is written once
  int64_t n = 0;
  std::unique_ptr<char[]> seq, names, qual;
  std::unique_ptr<int64_t[]> seq_off, name_off, qual_off;
  std::unique_ptr<int32_t[]> seq_len;
  std::unique_ptr<uint32_t[]> name_hash;
  bool has_qual = false;
  void alloc(int64_t records, int64_t seq_bytes, int64_t name_bytes, int64_t qual_bytes) {
    n = records;
    seq.reset(new char[static_cast<size_t>(seq_bytes) + 1]);
    names.reset(new char[static_cast<size_t>(name_bytes) + 1]);
    qual.reset(new char[static_cast<size_t>(qual_bytes) + 1]);
    seq_off.reset(new int64_t[static_cast<size_t>(records) + 1]);
    name_off.reset(new int64_t[static_cast<size_t>(records) + 1]);
    qual_off.reset(new int64_t[static_cast<size_t>(records) + 1]);
    seq_len.reset(new int32_t[static_cast<size_t>(records) + 1]);
    name_hash.reset(new uint32_t[static_cast<size_t>(records) + 1]);
  }
};

namespace {

struct Line {  // [a, b) of the text, '\r' and '\n' excluded; next = start of the following line
  int64_t a, b, next;
};

inline Line line_at(const char* t, int64_t len, int64_t p) {
  const void* nl = std::memchr(t + p, '\n', static_cast<size_t>(len - p));
  const int64_t e = nl ? static_cast<const char*>(nl) - t : len;
  int64_t b = e;
  if (b > p && t[b - 1] == '\r') --b;
  return Line{p, b, nl ? e + 1 : len};
}

uint32_t fnv1a_bytes(const char* s, int64_t n) {  // src/common.hpp:136-140
  uint32_t h = 2166136261u;
  for (int64_t i = 0; i < n; ++i) h = (h ^ static_cast<unsigned char>(s[i])) * 16777619u;
  return h;
}

struct Part {  // records of one thread
  std::vector<char> seq, names, qual;
  std::vector<int32_t> seq_len, name_len, qual_len;
  std::vector<uint32_t> hash;
  bool ok = true;
};

void add_record(Part& P, const char* t, int64_t na, int64_t nb, const std::string& seq, const std::string& qual) {
  P.names.insert(P.names.end(), t + na, t + nb);
  P.name_len.push_back(static_cast<int32_t>(nb - na));
  P.hash.push_back(fnv1a_bytes(t + na, nb - na));
  P.seq.insert(P.seq.end(), seq.begin(), seq.end());
  P.seq_len.push_back(static_cast<int32_t>(seq.size()));
  P.qual.insert(P.qual.end(), qual.begin(), qual.end());
  P.qual_len.push_back(static_cast<int32_t>(qual.size()));
}

// The reference's reader over t[0, len). Returns false (message in err) where it dies.
bool parse_sequential(const char* t, int64_t len, Part& P, bool& any_fastq, std::string& err) {
  int64_t p = 0;
  std::string seq, qual;
  const auto peek = [&]() -> int { return p < len ? static_cast<unsigned char>(t[p]) : -1; };
  for (;;) {
    int c;
    while ((c = peek()) != -1 && c != '>' && c != '@') p = line_at(t, len, p).next;  // junk lines
    if (c == -1) return true;
    const Line h = line_at(t, len, p);
    p = h.next;
    const bool fastq = t[h.a] == '@';
    int64_t ne = h.a + 1;
    while (ne < h.b && t[ne] != ' ' && t[ne] != '\t') ++ne;
    seq.clear();
    qual.clear();
    while ((c = peek()) != -1 && c != '>' && c != '+' && c != '@') {
      const Line l = line_at(t, len, p);
      seq.append(t + l.a, static_cast<size_t>(l.b - l.a));
      p = l.next;
    }
    if (fastq) {
      any_fastq = true;
      if (c != '+') {
        err = "malformed FASTQ record '" + std::string(t + h.a + 1, static_cast<size_t>(ne - h.a - 1)) + "'";
        return false;
      }
      p = line_at(t, len, p).next;  // the '+' separator
      while (qual.size() < seq.size() && p < len) {
        const Line l = line_at(t, len, p);
        qual.append(t + l.a, static_cast<size_t>(l.b - l.a));
        p = l.next;
      }
      if (qual.size() != seq.size()) {
        err = "FASTQ record '" + std::string(t + h.a + 1, static_cast<size_t>(ne - h.a - 1)) +
              "': quality length mismatch";
        return false;
      }
    }
    add_record(P, t, h.a + 1, ne, seq, qual);
  }
}

// First line start in [from, len) that begins a four-line record ('@' line whose second
// next line starts with '+'); len if none.
int64_t record_start_from(const char* t, int64_t len, int64_t from) {
  int64_t p = from;
  if (p > 0 && t[p - 1] != '\n') p = line_at(t, len, p).next;
  while (p < len) {
    if (t[p] == '@') {
      const int64_t l2 = line_at(t, len, p).next;
      const int64_t l3 = l2 < len ? line_at(t, len, l2).next : len;
      if (l3 < len && t[l3] == '+') return p;
    }
    p = line_at(t, len, p).next;
  }
  return len;
}

// Walks the four-line FASTQ records from p (a record start) up to end, calling
// visit(name_a, name_b, seq_a, seq_b, qual_a) for each; false if a record does not fit the
// shape or the walk does not end exactly at end.
template <class Visit>
bool walk_four_line(const char* t, int64_t len, int64_t p, int64_t end, Visit&& visit) {
  while (p < end) {
    if (t[p] != '@') {  // the reference skips lines that start neither '>' nor '@' between records
      if (t[p] == '>') return false;
      p = line_at(t, len, p).next;
      continue;
    }
    const Line h = line_at(t, len, p);
    if (h.next >= len) return false;
    const Line s = line_at(t, len, h.next);
    if (s.b == s.a || t[s.a] == '>' || t[s.a] == '+' || t[s.a] == '@' || s.next >= len) return false;
    const Line pl = line_at(t, len, s.next);
    if (t[pl.a] != '+' || pl.next >= len) return false;
    const Line q = line_at(t, len, pl.next);
    if (q.b - q.a != s.b - s.a) return false;
    int64_t ne = h.a + 1;
    while (ne < h.b && t[ne] != ' ' && t[ne] != '\t') ++ne;
    visit(h.a + 1, ne, s.a, s.b, q.a);
    p = q.next;
  }
  return p == end;
}

void assemble(const Part& P, dnaln_reads& R) {
  const int64_t n = static_cast<int64_t>(P.seq_len.size());
  R.alloc(n, static_cast<int64_t>(P.seq.size()), static_cast<int64_t>(P.names.size()),
          static_cast<int64_t>(P.qual.size()));
  if (!P.seq.empty()) std::memcpy(R.seq.get(), P.seq.data(), P.seq.size());
  if (!P.names.empty()) std::memcpy(R.names.get(), P.names.data(), P.names.size());
  if (!P.qual.empty()) std::memcpy(R.qual.get(), P.qual.data(), P.qual.size());
  int64_t so = 0, no = 0, qo = 0;
  for (int64_t j = 0; j < n; ++j) {
    R.seq_off[j] = so;
    R.name_off[j] = no;
    R.qual_off[j] = qo;
    R.seq_len[j] = P.seq_len[static_cast<size_t>(j)];
    R.name_hash[j] = P.hash[static_cast<size_t>(j)];
    so += P.seq_len[static_cast<size_t>(j)];
    no += P.name_len[static_cast<size_t>(j)];
    qo += P.qual_len[static_cast<size_t>(j)];
  }
  R.seq_off[n] = so;
  R.name_off[n] = no;
  R.qual_off[n] = qo;
}

// Four-line FASTQ on t threads: chunk starts, a counting walk per chunk, offsets, then a
// writing walk per chunk straight into R. False (R untouched) if any chunk does not fit.
bool parse_parallel(const char* text, int64_t len, int t, dnaln_reads& R) {
  std::vector<int64_t> start(static_cast<size_t>(t) + 1, len);
  start[0] = 0;
  for (int i = 1; i < t; ++i) start[static_cast<size_t>(i)] = record_start_from(text, len, len * i / t);
  for (int i = t - 1; i >= 1; --i)  // keep the chunk starts ordered
    start[static_cast<size_t>(i)] = std::min(start[static_cast<size_t>(i)], start[static_cast<size_t>(i) + 1]);
  const auto parallel = [&](auto&& f) {
    std::vector<std::thread> th;
    for (int i = 1; i < t; ++i) th.emplace_back(f, i);
    f(0);
    for (auto& x : th) x.join();
  };
  struct Count {
    int64_t n = 0, sb = 0, nb = 0;
    bool ok = false;
  };
  std::vector<Count> cnt(static_cast<size_t>(t) + 1);
  parallel([&](int i) {
    Count& c = cnt[static_cast<size_t>(i)];
    c.ok = walk_four_line(text, len, start[static_cast<size_t>(i)], start[static_cast<size_t>(i) + 1],
                          [&](int64_t na, int64_t nb, int64_t sa, int64_t sb, int64_t) {
                            c.n += 1;
                            c.sb += sb - sa;
                            c.nb += nb - na;
                          });
  });
  Count tot;
  for (int i = 0; i < t; ++i) {
    if (!cnt[static_cast<size_t>(i)].ok) return false;
    const Count c = cnt[static_cast<size_t>(i)];
    cnt[static_cast<size_t>(i)] = tot;  // becomes the chunk's first record / byte offsets
    tot.n += c.n;
    tot.sb += c.sb;
    tot.nb += c.nb;
  }
  R.alloc(tot.n, tot.sb, tot.nb, tot.sb);
  parallel([&](int i) {
    int64_t r = cnt[static_cast<size_t>(i)].n, so = cnt[static_cast<size_t>(i)].sb, no = cnt[static_cast<size_t>(i)].nb;
    walk_four_line(text, len, start[static_cast<size_t>(i)], start[static_cast<size_t>(i) + 1],
                   [&](int64_t na, int64_t nb, int64_t sa, int64_t sb, int64_t qa) {
                     const int64_t m = sb - sa;
                     std::memcpy(R.seq.get() + so, text + sa, static_cast<size_t>(m));
                     std::memcpy(R.qual.get() + so, text + qa, static_cast<size_t>(m));
                     std::memcpy(R.names.get() + no, text + na, static_cast<size_t>(nb - na));
                     R.seq_off[r] = so;
                     R.qual_off[r] = so;
                     R.name_off[r] = no;
                     R.seq_len[r] = static_cast<int32_t>(m);
                     R.name_hash[r] = fnv1a_bytes(text + na, nb - na);
                     so += m;
                     no += nb - na;
                     ++r;
                   });
  });
  R.seq_off[tot.n] = tot.sb;
  R.qual_off[tot.n] = tot.sb;
  R.name_off[tot.n] = tot.nb;
  R.has_qual = true;
  return true;
}

}  // namespace

extern "C" {

int dnaln_parse_reads(const char* text, int64_t len, int32_t threads, dnaln_reads** out, char* err, int64_t err_cap) {
  if (!out || len < 0 || (len > 0 && !text)) return DNALN_ERR_INVALID_ARG;
  *out = nullptr;
  auto R = new dnaln_reads;
  int t = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
  if (t < 1) t = 1;
  if (static_cast<int64_t>(t) * (1 << 20) > len) t = static_cast<int>(std::max<int64_t>(1, len >> 20));
  bool done = len > 0 && text[0] == '@' && parse_parallel(text, len, t, *R);
  if (!done) {
    std::vector<Part> parts(1);
    bool any_fastq = false;
    std::string why;
    if (!parse_sequential(text, len, parts[0], any_fastq, why)) {
      if (err && err_cap > 0) {
        const size_t m = std::min<size_t>(why.size(), static_cast<size_t>(err_cap - 1));
        std::memcpy(err, why.data(), m);
        err[m] = '\0';
      }
      delete R;
      return DNALN_ERR_INVALID_ARG;
    }
    assemble(parts[0], *R);
    R->has_qual = any_fastq;
  }
  *out = R;
  return DNALN_OK;
}

int dnaln_reads_view(const dnaln_reads* r, int64_t* n, const char** seq, const int64_t** seq_off,
                     const int32_t** seq_len, const char** names, const int64_t** name_off, const char** qual,
                     const int64_t** qual_off, const uint32_t** name_hash) {
  if (!r || !n) return DNALN_ERR_INVALID_ARG;
  *n = r->n;
  if (seq) *seq = r->seq.get();
  if (seq_off) *seq_off = r->seq_off.get();
  if (seq_len) *seq_len = r->seq_len.get();
  if (names) *names = r->names.get();
  if (name_off) *name_off = r->name_off.get();
  if (qual) *qual = r->has_qual ? r->qual.get() : nullptr;
  if (qual_off) *qual_off = r->has_qual ? r->qual_off.get() : nullptr;
  if (name_hash) *name_hash = r->name_hash.get();
  return DNALN_OK;
}

void dnaln_reads_free(dnaln_reads* r) { delete r; }

}  // extern "C"
