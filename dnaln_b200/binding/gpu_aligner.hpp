// gpu_aligner.hpp — GpuAligner, dnaln's Aligner interface (src/align.hpp:62-68) on the B200.
//
// A drop-in for SimdAligner / ScalarAligner: the same virtual align(tasks, n, traceback,
// out) and name(), plus the static lanes() / isa() that SimdAligner offers
// (src/align.hpp:92-93), so that code written against SimdAligner compiles against this
// class unchanged. A batch of tasks becomes one dnaln_gpu_align call: the borrowed query
// and target pointers of the tasks are gathered into two flat host buffers, and the
// results (score, ranges, NM and the CIGAR ops) come back into the caller's AlignResults.
// Results are bit-identical to ScalarAligner's and SimdAligner's.
//
// Errors end the process through dnaln's die() (src/common.hpp:123), as the reference does
// for every unusable input. All GpuAligners of a process share one library context per
// device (created on first use, never destroyed: the process exit releases it); a context
// serves one call at a time, like the reference's aligners, which are not thread-safe.
//
// Include path: dnaln's src/ (align.hpp, common.hpp) and this library's include/.
#pragma once

#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "align.hpp"
#include "common.hpp"
#include "dnaln_b200.h"

namespace dnaln {

class GpuAligner final : public Aligner {
 public:
  explicit GpuAligner(const ScoreParams& sp)
      : ctx_(shared_context()), sp_{sp.match, sp.mismatch, sp.gap_open, sp.gap_ext, sp.ambig, sp.bw} {}

  // Alignments one warp of the inter-sequence kernel carries (two per thread); a batch of
  // this many tasks fills one warp. Only informative, like SimdAligner::lanes().
  static int lanes() { return 64; }
  static const char* isa() { return "CUDA sm_100a"; }
  std::string name() const override { return "B200 sm_100a, 16x2 lanes per thread"; }

  void align(const AlignTask* tasks, size_t n, bool traceback, AlignResult* out) override {
    if (n == 0) return;
    q_.clear();
    t_.clear();
    q_off_.resize(n);
    q_len_.resize(n);
    t_off_.resize(n);
    t_len_.resize(n);
    int64_t cap = 0;
    for (size_t i = 0; i < n; ++i) {
      const AlignTask& tk = tasks[i];
      q_off_[i] = static_cast<int64_t>(q_.size());
      q_len_[i] = tk.qlen;
      if (tk.qlen > 0) q_.insert(q_.end(), tk.q, tk.q + tk.qlen);
      t_off_[i] = static_cast<int64_t>(t_.size());
      t_len_[i] = tk.tlen;
      if (tk.tlen > 0) t_.insert(t_.end(), tk.t, tk.t + tk.tlen);
      cap += 2 * static_cast<int64_t>(tk.qlen > 0 ? tk.qlen : 0) + 1;
    }
    if (q_.empty()) q_.push_back(4);  // the call wants non-null buffers
    if (t_.empty()) t_.push_back(4);
    res_.resize(n);
    cig_.resize(traceback ? static_cast<size_t>(cap) : 1);
    int64_t used = 0;
    const int rc = dnaln_gpu_align(ctx_, q_.data(), q_off_.data(), q_len_.data(), t_.data(), t_off_.data(),
                                   t_len_.data(), static_cast<int64_t>(n), traceback ? 1 : 0, &sp_, res_.data(),
                                   cig_.data(), traceback ? cap : 0, &used);
    if (rc != DNALN_OK) die("GPU alignment failed: %s", dnaln_gpu_last_error(ctx_));
    for (size_t i = 0; i < n; ++i) {
      const dnaln_align_result& r = res_[i];
      AlignResult& o = out[i];
      o.score = r.score;
      o.qb = r.qb;
      o.qe = r.qe;
      o.tb = r.tb;
      o.te = r.te;
      o.nm = r.nm;
      if (traceback) o.cigar.assign(cig_.begin() + r.cigar_off, cig_.begin() + r.cigar_off + r.cigar_len);
      else o.cigar.clear();
    }
  }

  // The process-wide context of the device DNALN_DEVICE names (default 0).
  static dnaln_ctx* shared_context() {
    static std::once_flag once;
    static dnaln_ctx* ctx = nullptr;
    std::call_once(once, [] {
      const char* d = std::getenv("DNALN_DEVICE");
      const int dev = d ? std::atoi(d) : 0;
      if (dnaln_gpu_ctx_create(dev, &ctx) != DNALN_OK || !ctx)
        die("no usable CUDA device for the B200 aligner (device %d)", dev);
    });
    return ctx;
  }

 private:
  dnaln_ctx* ctx_;
  dnaln_score_params sp_;
  std::vector<uint8_t> q_, t_;
  std::vector<int64_t> q_off_, t_off_;
  std::vector<int32_t> q_len_, t_len_;
  std::vector<dnaln_align_result> res_;
  std::vector<uint32_t> cig_;
};

}  // namespace dnaln
