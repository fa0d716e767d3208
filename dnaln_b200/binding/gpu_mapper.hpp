// gpu_mapper.hpp — GpuMapper, dnaln's Mapper (src/mapper.hpp:51-58) with map() on the B200.
//
// The same constructor and methods as Mapper, so a caller written against Mapper (the
// reference's cmd_map, src/main.cpp:46-61) compiles against this class unchanged:
//   * map(reads, n, out): the whole path of Mapper::map (src/mapper.cpp:75-223) — sketch,
//     index probe, chaining, candidate ranking, SW with traceback, MAPQ — as one
//     dnaln_gpu_map_batch call per batch, records identical to Mapper::map's;
//   * append_sam / write_sam_header: the host's, delegated to a reference Mapper held
//     inside (SAM formatting stays on the host);
//   * stats(): MapStats from the library's counters (t_seed = seeding + chaining time,
//     t_align = both SW passes, cells = the reference's MapStats::cells definition);
//   * kernel_name(): the device path.
// The minimizer index is built on the device from the Reference with the index's own k
// and w; the device build gives the reference's table bucket for bucket, so the caller's
// MinimizerIndex is used only for its parameters. Errors end the process through die().
//
// Include path: dnaln's src/ and this library's include/.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "gpu_aligner.hpp"
#include "mapper.hpp"

namespace dnaln {

class GpuMapper {
 public:
  GpuMapper(const Reference& ref, const MinimizerIndex& idx, const MapParams& p)
      : host_(ref, idx, p), ctx_(GpuAligner::shared_context()) {
    std::vector<uint64_t> off;
    std::vector<uint32_t> len;
    for (const Contig& c : ref.contigs) {
      off.push_back(c.offset);
      len.push_back(c.len);
    }
    if (dnaln_gpu_index_build(ctx_, ref.seq.data(), ref.seq.size(), off.data(), len.data(),
                              static_cast<int32_t>(off.size()), idx.k(), idx.w(), &index_) != DNALN_OK)
      die("GPU index build failed: %s", dnaln_gpu_last_error(ctx_));
    mp_.k = p.k;
    mp_.w = p.w;
    mp_.max_occ = p.max_occ;
    mp_.max_cand = p.max_cand;
    mp_.pri_ratio = p.pri_ratio;
    mp_.min_aln_score = p.min_aln_score;
    mp_.sc = dnaln_score_params{p.sc.match, p.sc.mismatch, p.sc.gap_open, p.sc.gap_ext, p.sc.ambig, p.sc.bw};
    mp_.ch = dnaln_chain_params{p.ch.max_gap, p.ch.band, p.ch.lookback, p.ch.min_score, p.ch.min_anchors};
    dnaln_gpu_reset_stats(ctx_);
  }
  ~GpuMapper() { dnaln_gpu_index_free(ctx_, index_); }
  GpuMapper(const GpuMapper&) = delete;
  GpuMapper& operator=(const GpuMapper&) = delete;

  void map(const SeqRecord* reads, size_t n, std::vector<MapRecord>& out) {
    out.resize(n);
    if (n == 0) return;
    seq_.clear();
    so_.resize(n);
    sl_.resize(n);
    hash_.resize(n);
    int64_t cap = 0;
    for (size_t r = 0; r < n; ++r) {
      so_[r] = static_cast<int64_t>(seq_.size());
      sl_[r] = static_cast<int32_t>(reads[r].seq.size());
      seq_ += reads[r].seq;
      hash_[r] = fnv1a(reads[r].name);  // the tie-break between equal best candidates
      cap += 2 * static_cast<int64_t>(sl_[r]) + 3;
    }
    if (seq_.empty()) seq_.push_back('N');
    rec_.resize(n);
    cig_.resize(static_cast<size_t>(cap));
    int64_t used = 0;
    if (dnaln_gpu_map_batch(ctx_, index_, seq_.data(), so_.data(), sl_.data(), hash_.data(), static_cast<int64_t>(n),
                            &mp_, rec_.data(), cig_.data(), cap, &used) != DNALN_OK)
      die("GPU mapping failed: %s", dnaln_gpu_last_error(ctx_));
    for (size_t r = 0; r < n; ++r) {
      const dnaln_map_record& g = rec_[r];
      MapRecord& m = out[r];
      m.contig = g.contig;
      m.pos = g.pos;
      m.rev = g.rev;
      m.mapq = g.mapq;
      m.score = g.score;
      m.nm = g.nm;
      m.n_cand = g.n_cand;
      m.cigar.assign(cig_.begin() + g.cigar_off, cig_.begin() + g.cigar_off + g.cigar_len);
    }
    dnaln_stats s;
    dnaln_gpu_get_stats(ctx_, &s);
    stats_.reads = s.reads;
    stats_.mapped = s.mapped;
    stats_.anchors = s.anchors;
    stats_.candidates = s.candidates;
    stats_.cells = s.cells;
    stats_.t_seed = (s.ms_seed + s.ms_chain) * 1e-3;
    stats_.t_align = (s.ms_sw_score + s.ms_sw_tb) * 1e-3;
  }

  void append_sam(const SeqRecord& r, const MapRecord& m, std::string& out) const { host_.append_sam(r, m, out); }
  void write_sam_header(FILE* fp, const std::string& cmdline) const { host_.write_sam_header(fp, cmdline); }
  const MapStats& stats() const { return stats_; }
  std::string kernel_name() const { return "B200 sm_100a whole path (seed, chain, SW, MAPQ on the device)"; }

 private:
  Mapper host_;
  dnaln_ctx* ctx_;
  int32_t index_ = -1;
  dnaln_map_params mp_{};
  MapStats stats_;
  std::string seq_;
  std::vector<int64_t> so_;
  std::vector<int32_t> sl_;
  std::vector<uint32_t> hash_;
  std::vector<dnaln_map_record> rec_;
  std::vector<uint32_t> cig_;
};

}  // namespace dnaln
