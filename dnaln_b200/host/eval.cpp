// eval.cpp — the accuracy gate of the mapping path as a batch call: Evaluator::add
// (src/evaluate.cpp:57-84) over a batch of records against the simulator's truth.
//
// A record counts when it is mapped with a CIGAR; it is placed correctly when its contig
// and strand are the truth's and its unclipped start (POS minus a leading S/H clip) is
// within `tol` of the true start; mapped and wrong records are also tallied per MAPQ
// (clamped to [0, 60]), as the reference's report prints them.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "dnaln_b200.h"

extern "C" int dnaln_eval_records(const dnaln_map_record* rec, const uint32_t* cigar, const int32_t* truth_contig,
                                  const int64_t* truth_start, const uint8_t* truth_rev, int64_t n, int32_t tol,
                                  dnaln_eval_counts* out) {
  if (!out || n < 0 || (n > 0 && (!rec || !truth_contig || !truth_start || !truth_rev))) return DNALN_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof *out);
  for (int64_t r = 0; r < n; ++r) {
    ++out->records;
    const dnaln_map_record& m = rec[r];
    if (m.contig < 0 || m.cigar_len <= 0) continue;
    ++out->mapped;
    int64_t clip = 0;
    const uint32_t c0 = cigar[m.cigar_off];
    if ((c0 & 0xFu) == 4u || (c0 & 0xFu) == 5u) clip = c0 >> 4;  // S or H
    const bool ok = m.contig == truth_contig[r] && (m.rev != 0) == (truth_rev[r] != 0) &&
                    std::llabs(m.pos - clip - truth_start[r]) <= tol;
    const int q = std::clamp(static_cast<int>(m.mapq), 0, 60);
    ++out->mapped_at_mapq[q];
    if (ok) ++out->correct;
    else ++out->wrong_at_mapq[q];
  }
  return DNALN_OK;
}
