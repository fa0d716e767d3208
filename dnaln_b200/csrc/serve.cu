// serve.cu — the request server of include/dnaln_b200.h (dnaln_serve_*): continuous
// batching of mapping requests over indexes kept resident in HBM.
//
// No reference counterpart: the reference maps one FASTQ per process against one index,
// batch after batch in one thread (src/main.cpp:33-61). Here producers submit requests
// (read sets of 1 to any number of reads, each against one index) at any time, and worker
// lanes turn the waiting requests into batches:
//
//   * a lane is a context of its own (stream, grow-only scratch) that shares the home
//     context's indexes (dnaln_gpu_index_attach), so the lanes' batches overlap on the
//     device and one lane's host work (gather, read-backs, scatter) hides behind another
//     lane's kernels;
//   * a lane that frees up takes the oldest request with reads not yet in a batch and
//     fills its batch, in arrival order, with the reads of every waiting request for the
//     same index and parameters (coalesce = 1) or of that request alone (coalesce = 0),
//     splitting large requests across batches;
//   * a batch takes reads while its estimated device footprint fits the lane's share of
//     the HBM budget (free device memory at creation, or the caller's figure);
//   * a request completes when the last of its parts has been mapped: its records keep
//     their places, its CIGARs are laid out in read order, as dnaln_gpu_map_batch does
//     for the request alone.
//
// Mapping is per read (src/mapper.cpp:88-222: every stage reads only the read's own
// codes, candidates and the index), so the batch a read lands in cannot change its
// record: a request's result is the same alone and in any mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "dnaln_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

// Device bytes one read of `len` bases adds to a batch, an upper estimate of the
// buffers the mapping pipeline grows for it: per base, the codes of both strands (2),
// minimizer slots (20), traceback CIGAR slots (8), the ASCII read (1), the CIGAR output
// bound (8) and anchor scratch of the warp path (53 per anchor, budgeted at one anchor
// per four bases); per read, offsets, counts and records (~200), and per candidate the
// score-only task, its result, its length-sorted copy and the candidate columns (~175).
constexpr int64_t kBytesPerBase = 2 + 20 + 8 + 1 + 8 + 14;
constexpr int64_t kBytesPerRead = 256;
constexpr int64_t kBytesPerCand = 176;

int64_t read_bytes(int64_t len, int max_cand) { return kBytesPerRead + kBytesPerCand * max_cand + kBytesPerBase * len; }

struct Request {
  int64_t id = 0;
  int32_t index_id = 0;
  const char* seq = nullptr;
  const int64_t* seq_off = nullptr;
  const int32_t* seq_len = nullptr;
  const uint32_t* name_hash = nullptr;
  int64_t n = 0;
  dnaln_map_params p{};
  dnaln_map_record* out = nullptr;
  uint32_t* cigar = nullptr;
  int64_t cigar_cap = 0;
  int64_t* cigar_used = nullptr;
  int64_t next = 0;                              // first read not yet given to a batch
  int parts = 0, parts_done = 0;                 // parts handed out / finished
  std::vector<std::vector<uint32_t>> part_cig;   // CIGAR ops of each part, read order
  std::vector<std::pair<int64_t, int64_t>> part_span;
  int status = DNALN_OK;
  bool done = false, cancelled = false;
  Clock::time_point t_submit;
  double latency_ms = 0.0;
};

struct Part {  // reads [a, b) of request r, the part_no-th part of it
  Request* r = nullptr;
  int64_t a = 0, b = 0, lo = 0, hi = 0;
  int part_no = 0;
};

// Grow-only page-locked / device buffer.
struct HostBuf {
  void* p = nullptr;
  size_t cap = 0;
  bool grow(size_t bytes) {
    if (bytes <= cap) return true;
    const size_t old = cap;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    const size_t want = std::max(bytes + bytes / 4, 2 * old) + 4096;  // geometric: few regrowths
    if (cudaHostAlloc(&p, want, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    cap = want;
    return true;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  bool grow(size_t bytes) {
    if (bytes <= cap) return true;
    const size_t old = cap;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t want = std::max(bytes + bytes / 4, 2 * old) + 4096;
    if (cudaMalloc(&p, want) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    cap = want;
    return true;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

struct Lane {
  dnaln_ctx* ctx = nullptr;
  cudaStream_t st = nullptr;
  std::map<int32_t, int32_t> ids;  // home index id -> this lane's id
  HostBuf h_seq, h_off, h_len, h_hash, h_rec, h_cig;
  DevBuf d_seq, d_off, d_len, d_hash, d_rec, d_cig;
  std::thread th;
};

}  // namespace

struct dnaln_server {
  dnaln_ctx* home = nullptr;
  int device = 0;
  dnaln_serve_params sp{};
  int64_t budget = 0, lane_budget = 0;
  std::vector<std::unique_ptr<Lane>> lanes;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> waiting;                          // requests with reads not yet in a batch
  std::map<int64_t, std::unique_ptr<Request>> requests;  // every request not yet waited for
  int64_t next_id = 1;
  bool stop = false;
  // statistics since creation or reset
  std::vector<double> lat;
  uint64_t n_req = 0, n_reads = 0, n_bases = 0, n_batches = 0, batch_reads = 0;
  int64_t max_depth = 0;
  double ms_form = 0, ms_gather = 0, ms_device = 0, ms_scatter = 0, ms_complete = 0;
  std::string err;
};

namespace {

int sfail(dnaln_server* s, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (s) {
    std::lock_guard<std::mutex> g(s->mu);
    s->err = buf;
  }
  return code;
}

bool same_key(const Request& a, const Request& b) {
  return a.index_id == b.index_id && std::memcmp(&a.p, &b.p, sizeof a.p) == 0;
}

// Takes the next batch off the waiting requests (caller holds s->mu). Empty when nothing waits.
std::vector<Part> form_batch(dnaln_server* s) {
  std::vector<Part> parts;
  if (s->waiting.empty()) return parts;
  const Request* first = s->waiting.front();
  const int64_t limit_bytes = s->lane_budget;
  int64_t reads = 0, bytes = 0;
  for (auto it = s->waiting.begin(); it != s->waiting.end();) {
    Request* r = *it;
    if (!same_key(*r, *first) || (!s->sp.coalesce && r != first)) {
      ++it;
      continue;
    }
    Part pt;
    pt.r = r;
    pt.a = pt.b = r->next;
    pt.lo = r->n > r->next ? r->seq_off[r->next] : 0;
    pt.hi = pt.lo;
    bool full = false;
    while (pt.b < r->n) {
      const int64_t i = pt.b;
      const int64_t rb = read_bytes(r->seq_len[i], r->p.max_cand);
      if (reads > 0 && (reads >= s->sp.max_batch_reads || bytes + rb > limit_bytes)) {
        full = true;
        break;
      }
      reads += 1;
      bytes += rb;
      pt.lo = std::min(pt.lo, r->seq_off[i]);
      pt.hi = std::max(pt.hi, r->seq_off[i] + r->seq_len[i]);
      ++pt.b;
    }
    if (pt.b > pt.a) {
      pt.part_no = r->parts++;
      r->part_span.emplace_back(pt.a, pt.b);
      r->part_cig.emplace_back();
      r->next = pt.b;
      parts.push_back(pt);
    }
    if (r->next >= r->n)
      it = s->waiting.erase(it);
    else
      ++it;
    if (full) break;
  }
  return parts;
}

// Lays out a finished request's CIGARs in read order and publishes it (caller holds s->mu).
void complete(dnaln_server* s, Request* r) {
  int64_t base = 0;
  for (int k = 0; k < r->parts && r->status == DNALN_OK; ++k) {
    const std::vector<uint32_t>& ops = r->part_cig[k];
    const int64_t m = static_cast<int64_t>(ops.size());
    if (base + m > r->cigar_cap || (m > 0 && !r->cigar)) {
      r->status = DNALN_ERR_CAPACITY;
      s->err = "CIGAR buffer of a request is too small";
      break;
    }
    if (m) std::memcpy(r->cigar + base, ops.data(), m * sizeof(uint32_t));
    for (int64_t i = r->part_span[k].first; i < r->part_span[k].second; ++i) r->out[i].cigar_off += base;
    base += m;
  }
  *r->cigar_used = r->status == DNALN_OK ? base : 0;
  r->part_cig.clear();
  r->part_cig.shrink_to_fit();
  r->latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - r->t_submit).count();
  r->done = true;
  if (r->status == DNALN_OK) {
    s->lat.push_back(r->latency_ms);
    s->n_req += 1;
    s->n_reads += static_cast<uint64_t>(r->n);
  }
}

// Maps one batch on lane L; returns its status.
int run_batch(dnaln_server* s, Lane& L, const std::vector<Part>& parts, double ms[3]) {
  const Clock::time_point t0 = Clock::now();
  int64_t n = 0, bytes = 0, cig_bound = 0;
  for (const Part& pt : parts) {
    n += pt.b - pt.a;
    bytes += pt.hi - pt.lo;
    for (int64_t i = pt.a; i < pt.b; ++i) cig_bound += 2 * static_cast<int64_t>(pt.r->seq_len[i]) + 3;
  }
  const Request& r0 = *parts.front().r;
  // this lane's id of the batch's index
  auto idit = L.ids.find(r0.index_id);
  if (idit == L.ids.end()) {
    int32_t lid = 0;
    if (int e = dnaln_gpu_index_attach(L.ctx, s->home, r0.index_id, &lid))
      return sfail(s, e, "index %d: %s", r0.index_id, dnaln_gpu_last_error(L.ctx));
    idit = L.ids.emplace(r0.index_id, lid).first;
  }
  if (!L.h_seq.grow(bytes + 1) || !L.h_off.grow(n * 8) || !L.h_len.grow(n * 4) || !L.h_hash.grow(n * 4) ||
      !L.h_rec.grow(n * sizeof(dnaln_map_record)))
    return sfail(s, DNALN_ERR_OOM, "out of page-locked host memory for a batch of %lld reads",
                 static_cast<long long>(n));
  if (!L.d_seq.grow(bytes + 1) || !L.d_off.grow(n * 8) || !L.d_len.grow(n * 4) || !L.d_hash.grow(n * 4) ||
      !L.d_rec.grow(n * sizeof(dnaln_map_record)) || !L.d_cig.grow(cig_bound * 4))
    return sfail(s, DNALN_ERR_OOM, "out of device memory for a batch of %lld reads", static_cast<long long>(n));
  // gather the parts' reads into one staged batch
  char* hs = static_cast<char*>(L.h_seq.p);
  int64_t* ho = static_cast<int64_t*>(L.h_off.p);
  int32_t* hl = static_cast<int32_t*>(L.h_len.p);
  uint32_t* hh = static_cast<uint32_t*>(L.h_hash.p);
  int64_t cur = 0, j = 0;
  for (const Part& pt : parts) {
    const Request& r = *pt.r;
    if (pt.hi > pt.lo) std::memcpy(hs + cur, r.seq + pt.lo, pt.hi - pt.lo);
    for (int64_t i = pt.a; i < pt.b; ++i, ++j) ho[j] = r.seq_off[i] - pt.lo + cur;
    std::memcpy(hl + (j - (pt.b - pt.a)), r.seq_len + pt.a, (pt.b - pt.a) * sizeof(int32_t));
    std::memcpy(hh + (j - (pt.b - pt.a)), r.name_hash + pt.a, (pt.b - pt.a) * sizeof(uint32_t));
    cur += pt.hi - pt.lo;
  }
  const Clock::time_point t1 = Clock::now();
  auto ck = [&](cudaError_t x) {
    if (x == cudaSuccess) return DNALN_OK;
    cudaGetLastError();
    return sfail(s, DNALN_ERR_CUDA, "%s", cudaGetErrorString(x));
  };
  if (int e = ck(cudaMemcpyAsync(L.d_seq.p, hs, bytes ? bytes : 1, cudaMemcpyHostToDevice, L.st))) return e;
  if (int e = ck(cudaMemcpyAsync(L.d_off.p, ho, n * 8, cudaMemcpyHostToDevice, L.st))) return e;
  if (int e = ck(cudaMemcpyAsync(L.d_len.p, hl, n * 4, cudaMemcpyHostToDevice, L.st))) return e;
  if (int e = ck(cudaMemcpyAsync(L.d_hash.p, hh, n * 4, cudaMemcpyHostToDevice, L.st))) return e;
  int64_t used = 0;
  if (int e = dnaln_gpu_map_batch_device(L.ctx, idit->second, static_cast<const char*>(L.d_seq.p),
                                         static_cast<const int64_t*>(L.d_off.p), static_cast<const int32_t*>(L.d_len.p),
                                         static_cast<const uint32_t*>(L.d_hash.p), n, &r0.p,
                                         static_cast<dnaln_map_record*>(L.d_rec.p), static_cast<uint32_t*>(L.d_cig.p),
                                         cig_bound, &used))
    return sfail(s, e, "%s", dnaln_gpu_last_error(L.ctx));
  if (int e = ck(cudaMemcpyAsync(L.h_rec.p, L.d_rec.p, n * sizeof(dnaln_map_record), cudaMemcpyDeviceToHost, L.st)))
    return e;
  // the staging of the CIGARs read back holds what the batch wrote (a few ops per read),
  // not the 2 * len + 3 bound the device buffer must allow
  if (!L.h_cig.grow(static_cast<size_t>(used > 0 ? used : 1) * 4))
    return sfail(s, DNALN_ERR_OOM, "out of page-locked host memory for %lld CIGAR ops", static_cast<long long>(used));
  if (used > 0)
    if (int e = ck(cudaMemcpyAsync(L.h_cig.p, L.d_cig.p, used * 4, cudaMemcpyDeviceToHost, L.st))) return e;
  if (int e = ck(cudaStreamSynchronize(L.st))) return e;
  const Clock::time_point t2 = Clock::now();
  // scatter: records to their requests (CIGAR offsets made part-relative), CIGARs per part
  const dnaln_map_record* rec = static_cast<const dnaln_map_record*>(L.h_rec.p);
  const uint32_t* cig = static_cast<const uint32_t*>(L.h_cig.p);
  j = 0;
  for (const Part& pt : parts) {
    const int64_t m = pt.b - pt.a;
    const int64_t c0 = rec[j].cigar_off;
    const int64_t c1 = rec[j + m - 1].cigar_off + rec[j + m - 1].cigar_len;
    dnaln_map_record* dst = pt.r->out + pt.a;
    std::memcpy(dst, rec + j, m * sizeof(dnaln_map_record));
    for (int64_t i = 0; i < m; ++i) dst[i].cigar_off -= c0;
    pt.r->part_cig[pt.part_no].assign(cig + c0, cig + c1);
    j += m;
  }
  ms[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
  ms[1] = std::chrono::duration<double, std::milli>(t2 - t1).count();
  ms[2] = std::chrono::duration<double, std::milli>(Clock::now() - t2).count();
  return DNALN_OK;
}

void lane_main(dnaln_server* s, Lane* L) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    s->cv_work.wait(lk, [&] { return s->stop || !s->waiting.empty(); });
    if (s->waiting.empty()) break;  // stopping and nothing left
    const Clock::time_point f0 = Clock::now();
    std::vector<Part> parts = form_batch(s);
    s->ms_form += std::chrono::duration<double, std::milli>(Clock::now() - f0).count();
    if (parts.empty()) continue;
    lk.unlock();
    double ms[3] = {0, 0, 0};
    const int st = run_batch(s, *L, parts, ms);
    lk.lock();
    s->ms_gather += ms[0];
    s->ms_device += ms[1];
    s->ms_scatter += ms[2];
    const Clock::time_point c0 = Clock::now();
    int64_t n = 0, bases = 0;
    for (const Part& pt : parts) {
      Request* r = pt.r;
      n += pt.b - pt.a;
      for (int64_t i = pt.a; i < pt.b; ++i) bases += r->seq_len[i];
      if (st != DNALN_OK && r->status == DNALN_OK) r->status = st;
      r->parts_done += 1;
      if (!r->done && r->next >= r->n && r->parts_done == r->parts) complete(s, r);
    }
    s->ms_complete += std::chrono::duration<double, std::milli>(Clock::now() - c0).count();
    s->n_batches += 1;
    s->batch_reads += static_cast<uint64_t>(n);
    s->n_bases += static_cast<uint64_t>(bases);
    s->cv_done.notify_all();
    if (!s->waiting.empty()) s->cv_work.notify_one();
  }
}

void release_lane(Lane& L) {
  if (L.ctx) dnaln_gpu_ctx_destroy(L.ctx);  // also drops its references to the indexes
  L.ctx = nullptr;
  for (HostBuf* b : {&L.h_seq, &L.h_off, &L.h_len, &L.h_hash, &L.h_rec, &L.h_cig}) b->release();
  for (DevBuf* b : {&L.d_seq, &L.d_off, &L.d_len, &L.d_hash, &L.d_rec, &L.d_cig}) b->release();
  if (L.st) cudaStreamDestroy(L.st);
  L.st = nullptr;
}

}  // namespace

extern "C" {

int dnaln_serve_create(dnaln_ctx* home, const dnaln_serve_params* sp, dnaln_server** out) {
  if (!home || !out) return DNALN_ERR_INVALID_ARG;
  *out = nullptr;
  dnaln_serve_params p = sp ? *sp : dnaln_serve_params{};
  if (p.lanes <= 0) p.lanes = 3;
  if (p.lanes > 16) return DNALN_ERR_INVALID_ARG;
  if (p.max_batch_reads <= 0) p.max_batch_reads = 262144;
  if (p.coalesce != 0) p.coalesce = 1;
  if (p.hbm_budget_bytes < 0) return DNALN_ERR_INVALID_ARG;
  int32_t device = 0;
  if (dnaln_gpu_ctx_device(home, &device) != DNALN_OK) return DNALN_ERR_INVALID_ARG;
  auto s = std::make_unique<dnaln_server>();
  s->home = home;
  s->sp = p;
  s->device = device;
  size_t free_b = 0, total_b = 0;
  if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    cudaGetLastError();
    return DNALN_ERR_CUDA;
  }
  const int64_t reserve = int64_t(2) << 30;
  int64_t avail = static_cast<int64_t>(free_b) > reserve + (int64_t(256) << 20)
                      ? static_cast<int64_t>(free_b) - reserve
                      : static_cast<int64_t>(256) << 20;
  s->budget = p.hbm_budget_bytes > 0 ? std::min<int64_t>(p.hbm_budget_bytes, static_cast<int64_t>(free_b)) : avail;
  s->lane_budget = s->budget / p.lanes;
  // each lane keeps a quarter of its share for traceback direction codes (at most 1 GiB)
  const int64_t dir_cap = std::min<int64_t>(int64_t(1) << 30, std::max<int64_t>(s->lane_budget / 4, 8 << 20));
  s->lane_budget -= dir_cap;
  if (s->lane_budget < (int64_t(1) << 20)) return DNALN_ERR_OOM;
  for (int i = 0; i < p.lanes; ++i) {
    auto L = std::make_unique<Lane>();
    int e = dnaln_gpu_ctx_create(device, &L->ctx);
    if (e == DNALN_OK && cudaStreamCreateWithFlags(&L->st, cudaStreamNonBlocking) != cudaSuccess) e = DNALN_ERR_CUDA;
    if (e == DNALN_OK) e = dnaln_gpu_set_stream(L->ctx, L->st);
    if (e == DNALN_OK) e = dnaln_gpu_set_option(L->ctx, "dir_cap_bytes", dir_cap);
    // a server's batches are made of whatever requests are waiting, so a batch shape
    // seldom repeats: lanes launch kernel by kernel instead of paying a graph capture on
    // the latency path of every shape seen twice
    if (e == DNALN_OK) e = dnaln_gpu_set_option(L->ctx, "graphs", 0);
    if (e != DNALN_OK) {
      release_lane(*L);
      for (auto& l : s->lanes) release_lane(*l);
      return e;
    }
    s->lanes.push_back(std::move(L));
  }
  for (auto& L : s->lanes) L->th = std::thread(lane_main, s.get(), L.get());
  *out = s.release();
  return DNALN_OK;
}

int dnaln_serve_submit(dnaln_server* s, int32_t index_id, const char* seq, const int64_t* seq_off,
                       const int32_t* seq_len, const uint32_t* name_hash, int64_t n, const dnaln_map_params* p,
                       dnaln_map_record* out, uint32_t* cigar, int64_t cigar_cap, int64_t* cigar_used,
                       int64_t* request) {
  if (!s) return DNALN_ERR_INVALID_ARG;
  if (!request || !cigar_used || !p || n < 0 || (n > 0 && (!seq || !seq_off || !seq_len || !name_hash || !out)))
    return sfail(s, DNALN_ERR_INVALID_ARG, "null argument");
  *request = 0;
  *cigar_used = 0;
  if (p->max_cand < 1 || p->max_cand > 1024) return sfail(s, DNALN_ERR_INVALID_ARG, "max_cand must be in [1, 1024]");
  {
    uint64_t st[6];
    if (dnaln_gpu_index_stats(s->home, index_id, st) != DNALN_OK)
      return sfail(s, DNALN_ERR_NOT_FOUND, "unknown index id %d", index_id);
  }
  for (int64_t i = 0; i < n; ++i) {
    if (seq_len[i] < 0 || seq_off[i] < 0) return sfail(s, DNALN_ERR_INVALID_ARG, "negative offset or length");
    if (read_bytes(seq_len[i], p->max_cand) > s->lane_budget)
      return sfail(s, DNALN_ERR_OOM, "read %lld (%d bases) does not fit a lane's share of the HBM budget",
                   static_cast<long long>(i), seq_len[i]);
  }
  auto r = std::make_unique<Request>();
  r->index_id = index_id;
  r->seq = seq;
  r->seq_off = seq_off;
  r->seq_len = seq_len;
  r->name_hash = name_hash;
  r->n = n;
  r->p = *p;
  r->out = out;
  r->cigar = cigar;
  r->cigar_cap = cigar_cap;
  r->cigar_used = cigar_used;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop) return DNALN_ERR_INVALID_ARG;
    r->id = s->next_id++;
    *request = r->id;
    Request* raw = r.get();
    s->requests[raw->id] = std::move(r);
    if (n == 0) {
      complete(s, raw);
    } else {
      s->waiting.push_back(raw);
      s->max_depth = std::max<int64_t>(s->max_depth, static_cast<int64_t>(s->waiting.size()));
    }
  }
  if (n == 0)
    s->cv_done.notify_all();
  else
    s->cv_work.notify_one();
  return DNALN_OK;
}

int dnaln_serve_cancel(dnaln_server* s, int64_t request) {
  if (!s) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->requests.find(request);
  if (it == s->requests.end()) {
    s->err = "unknown request (or already waited for)";
    return DNALN_ERR_INVALID_ARG;
  }
  Request* r = it->second.get();
  if (r->done) return DNALN_OK;  // finished before the cancel: its result stands
  // no further part of it goes into a batch; parts already in a batch finish first (their
  // lanes write into the caller's buffers), then the request completes as cancelled
  r->cancelled = true;
  r->status = DNALN_ERR_CANCELLED;
  r->next = r->n;
  s->waiting.erase(std::remove(s->waiting.begin(), s->waiting.end(), r), s->waiting.end());
  if (r->parts_done == r->parts) {
    complete(s, r);
    s->cv_done.notify_all();
  }
  return DNALN_OK;
}

int dnaln_serve_wait(dnaln_server* s, int64_t request, double* latency_ms) {
  if (!s) return DNALN_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->requests.find(request);
  if (it == s->requests.end()) {
    s->err = "unknown request (or already waited for)";
    return DNALN_ERR_INVALID_ARG;
  }
  Request* r = it->second.get();
  s->cv_done.wait(lk, [&] { return r->done; });
  const int st = r->status;
  if (latency_ms) *latency_ms = r->latency_ms;
  s->requests.erase(it);
  return st;
}

int dnaln_serve_get_stats(dnaln_server* s, dnaln_serve_stats* out) {
  if (!s || !out) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(s->mu);
  *out = dnaln_serve_stats{};
  out->requests = s->n_req;
  out->reads = s->n_reads;
  out->bases = s->n_bases;
  out->batches = s->n_batches;
  out->mean_batch_reads = s->n_batches ? static_cast<double>(s->batch_reads) / s->n_batches : 0.0;
  out->max_queue_depth = s->max_depth;
  out->budget_bytes = s->budget;
  out->lane_budget_bytes = s->lane_budget;
  out->lanes = static_cast<int32_t>(s->lanes.size());
  out->ms_form = s->ms_form;
  out->ms_gather = s->ms_gather;
  out->ms_device = s->ms_device;
  out->ms_scatter = s->ms_scatter;
  out->ms_complete = s->ms_complete;
  if (!s->lat.empty()) {
    std::vector<double> v = s->lat;
    std::sort(v.begin(), v.end());
    auto rank = [&](double q) {  // nearest rank
      size_t k = static_cast<size_t>(q * v.size() + 0.999999);
      return v[std::min(v.size() - 1, k ? k - 1 : 0)];
    };
    out->p50_ms = rank(0.50);
    out->p99_ms = rank(0.99);
    out->max_ms = v.back();
    double sum = 0;
    for (double x : v) sum += x;
    out->mean_ms = sum / v.size();
  }
  return DNALN_OK;
}

int dnaln_serve_reset_stats(dnaln_server* s) {
  if (!s) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(s->mu);
  s->lat.clear();
  s->n_req = s->n_reads = s->n_bases = s->n_batches = s->batch_reads = 0;
  s->max_depth = static_cast<int64_t>(s->waiting.size());
  s->ms_form = s->ms_gather = s->ms_device = s->ms_scatter = s->ms_complete = 0;
  return DNALN_OK;
}

const char* dnaln_serve_last_error(const dnaln_server* s) { return s ? s->err.c_str() : "null server"; }

int dnaln_serve_destroy(dnaln_server* s) {
  if (!s) return DNALN_OK;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& L : s->lanes)
    if (L->th.joinable()) L->th.join();
  cudaSetDevice(s->device);
  for (auto& L : s->lanes) release_lane(*L);
  delete s;
  return DNALN_OK;
}

}  // extern "C"
