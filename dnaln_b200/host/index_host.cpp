// index_host.cpp — host construction of the minimizer index that the GPU keeps resident.
//
// MinimizerIndex::build (src/index.cpp:10-45): minimizers of every contig at their global
// offsets, sorted by (hash, pos); one bucket per distinct hash in an open-addressing
// table of the smallest power of two >= max(16, 2 * n_keys), inserted in ascending hash
// order with linear probing from hash & mask, so the table is bucket-for-bucket the
// reference's; each key's occurrences are the contiguous run of (pos << 1 | strand) in
// the position array. The sketch here is a plain sliding-window minimum (the reference
// streams a van Herk scheme): same windows, same leftmost-minimum rule, same emission.
#include "index_host.hpp"

#include <algorithm>
#include <cstring>

namespace dnb {

namespace {

constexpr uint64_t kEmpty = ~0ULL;

inline uint64_t hash64_host(uint64_t key, uint64_t mask) {  // src/minimizer.hpp:21-31
  key = (~key + (key << 21)) & mask;
  key = key ^ key >> 24;
  key = ((key + (key << 3)) + (key << 8)) & mask;
  key = key ^ key >> 14;
  key = ((key + (key << 2)) + (key << 4)) & mask;
  key = key ^ key >> 28;
  key = (key + (key << 31)) & mask;
  return key;
}

struct Min {
  uint64_t hash;
  uint32_t val;  // pos << 1 | strand
};

// Minimizers of seq[0, len): windows of w k-mers inside N-free runs, leftmost minimum,
// palindromes never selected, consecutive duplicates dropped (src/minimizer.cpp:5-68).
void sketch_contig(const uint8_t* seq, uint32_t len, int k, int w, uint32_t offset, std::vector<Min>& out) {
  const uint64_t mask = (1ULL << (2 * k)) - 1;
  const int shift = 2 * (k - 1);
  std::vector<uint64_t> h(static_cast<size_t>(w));
  std::vector<uint32_t> ps(static_cast<size_t>(w)), stv(static_cast<size_t>(w));
  uint64_t fwd = 0, rev = 0;
  int run = 0;
  int64_t nk = 0, last = -1, cur = -1;  // k-mers in run; last emitted pos; ring index of window min
  for (uint32_t i = 0; i < len; ++i) {
    const uint8_t c = seq[i];
    if (c > 3) {
      run = 0;
      nk = 0;
      cur = -1;
      continue;
    }
    fwd = ((fwd << 2) | c) & mask;
    rev = (rev >> 2) | (static_cast<uint64_t>(3 - c) << shift);
    if (++run < k) continue;
    const uint32_t st = rev < fwd;
    const uint64_t hv = fwd != rev ? hash64_host(st ? rev : fwd, mask) : kEmpty;
    const size_t slot = static_cast<size_t>(nk % w);
    h[slot] = hv;
    ps[slot] = i - static_cast<uint32_t>(k) + 1;
    stv[slot] = st;
    ++nk;
    // keep `cur` = leftmost minimum of the last min(nk, w) k-mers
    if (cur < 0 || nk - 1 - cur >= w) {
      cur = nk - 1 - std::min<int64_t>(nk, w) + 1;
      for (int64_t j = cur + 1; j < nk; ++j)
        if (h[static_cast<size_t>(j % w)] < h[static_cast<size_t>(cur % w)]) cur = j;
    } else if (hv < h[static_cast<size_t>(cur % w)]) {
      cur = nk - 1;
    }
    if (nk >= w) {
      const size_t cs = static_cast<size_t>(cur % w);
      if (h[cs] != kEmpty) {
        if (static_cast<int64_t>(ps[cs]) != last) out.push_back({h[cs], (ps[cs] + offset) << 1 | stv[cs]});
        last = ps[cs];
      }
    }
  }
}

}  // namespace

bool build_index_host(const uint8_t* genome, const uint64_t* contig_off, const uint32_t* contig_len,
                      int32_t n_contigs, int k, int w, HostIndex& ix) {
  std::vector<Min> mins;
  uint64_t total = 0;
  for (int32_t c = 0; c < n_contigs; ++c) total += contig_len[c];
  mins.reserve(static_cast<size_t>(total * 2 / (w + 1) + 1024));
  for (int32_t c = 0; c < n_contigs; ++c)
    sketch_contig(genome + contig_off[c], contig_len[c], k, w, static_cast<uint32_t>(contig_off[c]), mins);
  std::sort(mins.begin(), mins.end(), [](const Min& a, const Min& b) {
    return a.hash != b.hash ? a.hash < b.hash : (a.val >> 1) < (b.val >> 1);
  });
  ix.k = k;
  ix.w = w;
  ix.n_keys = 0;
  for (size_t i = 0; i < mins.size(); ++i)
    if (i == 0 || mins[i].hash != mins[i - 1].hash) ++ix.n_keys;
  uint64_t cap = 16;
  while (cap < ix.n_keys * 2) cap <<= 1;
  ix.mask = cap - 1;
  ix.keys.assign(cap, kEmpty);
  ix.offs.assign(cap, 0);
  ix.cnts.assign(cap, 0);
  ix.pos.resize(mins.size());
  ix.max_count = 0;
  for (size_t i = 0; i < mins.size();) {
    size_t j = i;
    for (; j < mins.size() && mins[j].hash == mins[i].hash; ++j) ix.pos[j] = mins[j].val;
    uint64_t s = mins[i].hash & ix.mask;
    while (ix.keys[s] != kEmpty) s = (s + 1) & ix.mask;
    ix.keys[s] = mins[i].hash;
    ix.offs[s] = static_cast<uint32_t>(i);
    ix.cnts[s] = static_cast<uint32_t>(j - i);
    ix.max_count = std::max(ix.max_count, static_cast<uint32_t>(j - i));
    i = j;
  }
  return true;
}

}  // namespace dnb
