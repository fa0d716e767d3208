// capi.cu — the C ABI (include/dnaln_b200.h): contexts, HBM-resident genome indexes, and
// the orchestration of each batch through the kernels of seed_thread.cu, seed_long.cu,
// seed.cu, sw.cu and map.cu.
//
// One batch (Mapper::map, src/mapper.cpp:75-223) is enqueued on the context's stream as:
//   k_len64 + scan: packed read offsets, total bases, longest read (read back first only
//     when the caller did not give the batch's size, so the rest can run as a graph)
//   k_encode_reads: codes of both strands of every read
//   k_seed_chain_t: short reads one thread each (sketch, probe, anchors, chaining DP,
//     chains, candidate loci); reads it cannot take are listed
//   k_seed_chain_tl: listed long reads one thread each, longest first; what exceeds its
//     bounds is listed again
//   k_seed<list> + k_chain_map<list>: the reads still listed, one warp each
//   score-only SW over every candidate of reads with >= 2 candidates, then k_choose
//     (best / ties / second best, fnv1a tie-break, the traceback task of each read)
//   SW with traceback over each read's chosen candidate (chunked by scratch size), walk
//   k_records (MAPQ, positions, soft clips), CIGAR offsets (scan), k_cigar_gather
//   one read-back of the batch's totals, task counts, error flags and counters
// Task and list counts produced on the device are consumed on the device, so the host
// waits once per batch. The host-buffer entry points queue parts of a batch to a worker
// thread that overlaps their copies in and out with the compute (two device slots, two
// copy streams).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
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

#include "common.cuh"
#include "dnaln_b200.h"
#include "index_build.cuh"
#include "map.cuh"
#include "seed.cuh"
#include "sw.cuh"

using namespace dnb;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

// Device memory of one resident index. Contexts that share the index (index_attach) hold
// it through a shared pointer; the last holder to release it frees the memory.
struct IndexMem {
  DevBuf table, positions, genome, coff, clen, nruns;
  IndexMem() = default;
  IndexMem(const IndexMem&) = delete;
  IndexMem& operator=(const IndexMem&) = delete;
  ~IndexMem() {
    for (DevBuf* b : {&table, &positions, &genome, &coff, &clen, &nruns})
      if (b->p) cudaFree(b->p);
  }
  size_t bytes() const { return table.cap + positions.cap + genome.cap + coff.cap + clen.cap + nruns.cap; }
};

struct IndexRes {
  std::shared_ptr<IndexMem> mem;
  int device = 0;
  uint64_t n_keys = 0, n_pos = 0, n_buckets = 0, n_bases = 0;
  uint32_t max_count = 0;
  int32_t n_contigs = 0, k = 0, w = 0;
  DevIndex dev{};
};

enum Ev { kEvSeed0, kEvSeed1, kEvChain0, kEvChain1, kEvSc0, kEvSc1, kEvTb0, kEvTb1, kEvPost0, kEvPost1, kNumEv };

constexpr int kMaxTrace = 256;  // traced launches per batch

struct KernelTime {
  int64_t launches = 0;
  double ms = 0.0;
};

// One queued part of a host-buffer batch (dnaln_gpu_map_submit): reads [a, b) of the
// caller's arrays, with the facts the host knows about them.
struct MapPart {
  int64_t ticket = 0;
  bool last = false;  // last part of its ticket
  int32_t index_id = 0;
  const char* seq = nullptr;
  const int64_t* seq_off = nullptr;
  const int32_t* seq_len = nullptr;
  const uint32_t* name_hash = nullptr;
  int64_t a = 0, b = 0;
  int64_t lo = 0, hi = 0, bases = 0, max_len = 0, cig_bound = 0;
  dnaln_map_params p{};
  dnaln_map_record* out = nullptr;
  uint32_t* cigar = nullptr;
  int64_t cigar_cap = 0;
  int64_t* cigar_used = nullptr;
};

// Per-batch facts the caller may already know (host-buffer path), sparing a device read-back.
struct BatchHints {
  int64_t seq_base = 0;    // subtracted from every read offset (sub-batch staged on the device)
  int64_t bases = -1;      // total bases of the batch, -1 = read back from the device
  int64_t max_len = -1;    // longest read, -1 = read back from the device
  int64_t cigar_base = 0;  // added to every record's cigar_off
  bool retry = false;      // the batch is being mapped again with a grown chaining pool
  bool caller_cigar = false;  // the CIGARs go to the caller's buffer (not the internal one)
};

// Host facts of an enqueued batch that its completion needs.
struct MapRun {
  int64_t B = 0, max_len = 0, cigar_cap = 0;
  uint32_t* d_cigar = nullptr;
  bool thread_path = false, long_used = false;
  uint64_t launches = 0;  // kernels the enqueue issued (counted again at each graph replay)
};

struct CachedGraph {  // an instantiated batch graph and the buffer epoch it was captured at
  cudaGraphExec_t exec;
  uint64_t epoch;
  MapRun run;
};

}  // namespace

struct dnaln_ctx {
  int device = 0;
  cudaStream_t own = nullptr, st = nullptr;
  std::string err;
  std::map<int32_t, IndexRes> idx;
  int32_t next_id = 1;
  std::map<std::string, DevBuf> bufs;
  uint32_t* d_err = nullptr;   // kernel error flags
  int* d_count = nullptr;      // [0] score tasks, [1] traceback tasks, [2] reads listed for the warp path
  int64_t* h_info = nullptr;   // pinned read-back slots
  cudaEvent_t ev[kNumEv] = {};
  dnaln_stats stats{};
  size_t dir_cap_bytes = size_t(1) << 30;  // direction-bit scratch per traceback launch
  // pipelined host-buffer path: copy streams, per-slot events, sub-batch size (reads)
  cudaStream_t cp_in = nullptr, cp_out = nullptr;
  cudaEvent_t in_ready[2] = {}, out_free[2] = {}, h2d_ev[4] = {}, d2h_ev[4] = {};
  int64_t sub_batch = 0;
  // submit / wait: queue of parts, a worker thread, finished tickets with their status
  mutable std::mutex mu;  // held by the worker while it drives the device, and by every other entry point
  std::mutex err_mu;      // the last error message (set by the worker and by callers)
  std::mutex qmu;   // queue, tickets, results
  std::condition_variable qcv;
  std::deque<MapPart> queue;
  std::map<int64_t, int> results;     // finished tickets -> status
  std::map<int64_t, int> first_err;   // status of a ticket's first failed part
  std::map<int64_t, int64_t> ticket_ops;  // CIGAR ops written so far per ticket
  int64_t next_ticket = 1;
  std::thread worker;
  bool stop = false;
  bool warp_seed_only = false;  // option: every read through the warp-per-read seeding kernels
  bool length_order = true;     // option: SW tasks of mixed-length batches run longest first
  bool long_thread = true;      // option: listed long reads one thread each before the warp kernels
  // option "work_stealing": the warp chaining kernel takes reads by atomic claims on
  // resident blocks (default) instead of striding over a fixed grid
  bool stealing = true;
  // option "encode_bulk": the codes of both strands through shared memory by bulk (TMA)
  // copies, or read by read from global memory (default: measured faster)
  bool encode_bulk = false;
  // reads per block of the thread-per-read seeding kernel: option "seed_block" (0 = tuned
  // on the first batch of at least kSeedTuneReads reads, else 64 or 128) and the tuning
  int seed_block = 0;
  dnaln_seed_tuning seed_tune{};
  // SW kernel form per (band width, traceback, read-length bucket): option "sw_form" 0 =
  // tuned on the first batch that needs it, 1 = inter-sequence, 2 = intra-sequence
  int sw_mode = 0;
  std::map<int, dnaln_sw_tuning> sw_tune;
  cudaEvent_t tune_ev[kSwForms + 1] = {};
  int* h_tune = nullptr;  // pinned read-back of a device task count
  int64_t pool_cap = 0;   // entries of the warp-path chaining pool (grown from the batches' use)
  int64_t pool_min = int64_t(1) << 16;  // the pool's floor (option "chain_pool" lowers it)
  // fault injection on the host (option "fail_alloc_after"): the device allocation after
  // this many more succeed fails as if the device were out of memory; -1 = off
  int64_t fail_alloc_after = -1;
  // CUDA graphs of batches (run_map): cache by launch key, keys seen once, and the buffer
  // epoch, bumped whenever a buffer a graph may reference is reallocated or rewritten
  bool graphs = true, capturing = false;
  std::map<std::string, CachedGraph> graph_cache;
  std::map<std::string, uint64_t> graph_seen;
  uint64_t epoch = 0, graph_launches = 0;
  // kernel trace: event pairs of the current batch, totals per kernel name
  bool trace_on = false, trace_open = false;
  std::string trace_only;  // non-empty: trace only the kernel of this name
  int trace_n = 0;
  std::vector<cudaEvent_t> trace_ev;
  const char* trace_name[kMaxTrace] = {};
  std::map<std::string, KernelTime> ktimes;
  // chaining gap-cost table on the device, for (lut_k, lut_band); re-uploaded on change
  int lut_k = -1, lut_band = -1;
  int32_t* h_lut = nullptr;  // page-locked staging of the table
  size_t h_lut_cap = 0;
};

namespace {

constexpr int64_t kSeedTuneReads = 32768;  // smallest batch the reads-per-block tuner times
constexpr int64_t kSwTuneMinTasks = 4096;  // smallest SW sample whose timing picks a form

int fail(dnaln_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) {
    std::lock_guard<std::mutex> g(c->err_mu);
    c->err = buf;
  }
  return code;
}

#define CK(call)                                                                                 \
  do {                                                                                           \
    const cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) return fail(c, DNALN_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

// Grow-only device buffer; returns nullptr (and sets the context error) on failure.
template <class T>
T* dbuf(dnaln_ctx* c, const char* name, size_t count) {
  DevBuf& b = c->bufs[name];
  const size_t need = (count ? count : 1) * sizeof(T);
  if (b.cap < need) {
    if (c->capturing) {  // a graph cannot hold an allocation: the caller runs the batch eagerly
      fail(c, DNALN_ERR_CUDA, "capture stopped: buffer %s must grow", name);
      return nullptr;
    }
    ++c->epoch;  // graphs captured before may reference the old buffer
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    if (c->fail_alloc_after >= 0 && c->fail_alloc_after-- == 0) {
      fail(c, DNALN_ERR_OOM, "out of device memory allocating %zu bytes for %s (injected)", need, name);
      return nullptr;
    }
    size_t cap = need + need / 4;
    if (cudaMalloc(&b.p, cap) != cudaSuccess) {
      cudaGetLastError();
      cap = need;
      if (cudaMalloc(&b.p, cap) != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        fail(c, DNALN_ERR_OOM, "out of device memory allocating %zu bytes for %s", need, name);
        return nullptr;
      }
    }
    b.cap = cap;
  }
  return static_cast<T*>(b.p);
}

#define DBUF(ptr, T, name, count)                         \
  T* ptr = dbuf<T>(c, name, (count));                     \
  if (!ptr) return DNALN_ERR_OOM;

int set_device(dnaln_ctx* c) {
  CK(cudaSetDevice(c->device));
  return DNALN_OK;
}

int exclusive_scan(dnaln_ctx* c, const int64_t* in, int64_t* out, int64_t n);

double ev_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();
    return 0.0;
  }
  return ms;
}

double ev_ms(dnaln_ctx* c, int a, int b) { return ev_ms(c->ev[a], c->ev[b]); }

void trace_mark(void* self, cudaStream_t st, const char* kernel) {
  auto* c = static_cast<dnaln_ctx*>(self);
  if (kernel) {
    c->trace_open = c->trace_n < kMaxTrace && (c->trace_only.empty() || c->trace_only == kernel) &&
                    cudaEventRecord(c->trace_ev[2 * c->trace_n], st) == cudaSuccess;
    if (c->trace_open) c->trace_name[c->trace_n] = kernel;
  } else if (c->trace_open) {
    if (cudaEventRecord(c->trace_ev[2 * c->trace_n + 1], st) == cudaSuccess) ++c->trace_n;
    c->trace_open = false;
  }
}

// The context's tracer (a no-op when tracing is off).
KernelTrace tracer(dnaln_ctx* c) {
  KernelTrace t;
  if (c->trace_on) {
    t.mark = trace_mark;
    t.self = c;
  }
  return t;
}

// Adds the traced launches of the batch to the totals; call once the stream is idle.
void trace_collect(dnaln_ctx* c) {
  for (int i = 0; i < c->trace_n; ++i) {
    KernelTime& k = c->ktimes[c->trace_name[i]];
    ++k.launches;
    k.ms += ev_ms(c->trace_ev[2 * i], c->trace_ev[2 * i + 1]);
  }
  c->trace_n = 0;
  c->trace_open = false;
}

int exclusive_scan(dnaln_ctx* c, const int64_t* in, int64_t* out, int64_t n) {
  size_t tmp = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, n, c->st));
  DBUF(t, uint8_t, "cub_tmp", tmp);
  const KernelTrace kt = tracer(c);
  kt.begin(c->st, "cub_scan");
  const cudaError_t e = cub::DeviceScan::ExclusiveSum(t, tmp, in, out, n, c->st);
  kt.end(c->st);
  CK(e);
  return DNALN_OK;
}

bool score_params_ok(const dnaln_score_params& s, std::string& why) {
  // src/cli.hpp:93-95 (bw in [1, 1000]; A >= 1, B >= 0, O >= 0, E >= 1)
  if (s.bw < 1 || s.bw > 1000) return why = "--bw must be in [1, 1000]", false;
  if (s.match < 1 || s.mismatch < 0 || s.gap_open < 0 || s.gap_ext < 1)
    return why = "scores must satisfy A >= 1, B >= 0, O >= 0, E >= 1", false;
  if (s.ambig < 0) return why = "ambiguous-base penalty must be >= 0", false;
  return true;
}

// Gap cost of the chaining DP for dd in [0, band] (src/chain.cpp:36).
std::vector<int32_t> chain_cost_lut(int k, int band) {
  std::vector<int32_t> lut(static_cast<size_t>(band) + 1, 0);
  for (int dd = 1; dd <= band; ++dd) {
    const int lg = 63 - __builtin_clzll(static_cast<unsigned long long>(dd));
    lut[static_cast<size_t>(dd)] = static_cast<int>(0.01 * k * static_cast<double>(dd) + 0.5 * lg);
  }
  return lut;
}

// The gap-cost table on the device for (k, band), uploaded (stream-ordered, from
// page-locked staging) only when the pair changes: a pageable upload per batch would
// block the host behind copies in flight on other streams.
int chain_lut_dev(dnaln_ctx* c, int k, int band, const int32_t** out) {
  const size_t n = static_cast<size_t>(band) + 1;
  DBUF(d, int32_t, "chain_lut", n);
  if (c->lut_k != k || c->lut_band != band) {
    if (c->capturing) return fail(c, DNALN_ERR_CUDA, "capture stopped: the gap-cost table must be uploaded");
    ++c->epoch;  // graphs captured before read the previous table
    const std::vector<int32_t> lut = chain_cost_lut(k, band);
    CK(cudaStreamSynchronize(c->st));  // the staging buffer may still feed an earlier upload
    if (c->h_lut_cap < n) {
      if (c->h_lut) cudaFreeHost(c->h_lut);
      c->h_lut = nullptr;
      c->h_lut_cap = 0;
      CK(cudaHostAlloc(&c->h_lut, n * sizeof(int32_t), cudaHostAllocDefault));
      c->h_lut_cap = n;
    }
    std::memcpy(c->h_lut, lut.data(), n * sizeof(int32_t));
    CK(cudaMemcpyAsync(d, c->h_lut, n * sizeof(int32_t), cudaMemcpyHostToDevice, c->st));
    c->lut_k = k;
    c->lut_band = band;
  }
  *out = d;
  return DNALN_OK;
}

__global__ void k_len64(const int32_t* __restrict__ len, int64_t n, int64_t* __restrict__ out,
                        unsigned long long* __restrict__ max_len) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  int32_t l = 0;
  if (i < n) {
    l = len[i] < 0 ? 0 : len[i];
    out[i] = l;
  } else if (i == n) {
    out[n] = 0;
  }
  l = __reduce_max_sync(0xffffffffu, l);  // one atomic per warp instead of one per read
  if ((threadIdx.x & 31) == 0 && l > 0) atomicMax(max_len, static_cast<unsigned long long>(l));
}

__global__ void k_list_sum64(const int64_t* __restrict__ vals, const int32_t* __restrict__ list,
                             const int* __restrict__ list_n, unsigned long long* __restrict__ out) {
  const int m = *list_n;
  long long acc = 0;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < m; x += gridDim.x * blockDim.x) acc += vals[list[x]];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, static_cast<unsigned long long>(acc));
}

// *out += sum of vals[list[x]] for x < *list_n (minimizers of the reads listed for the
// warp path): a warp sum, then one atomic per warp.
__global__ void k_list_sum(const int32_t* __restrict__ vals, const int32_t* __restrict__ list,
                           const int* __restrict__ list_n, unsigned long long* __restrict__ out) {
  const int m = *list_n;
  long long acc = 0;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < m; x += gridDim.x * blockDim.x) acc += vals[list[x]];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, static_cast<unsigned long long>(acc));
}

__global__ void k_cig_slots(const int64_t* __restrict__ pofs, int64_t n, int64_t* __restrict__ out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = 2 * pofs[i] + i;
}

inline unsigned nblk(int64_t n, int t = 256) { return static_cast<unsigned>((n + t - 1) / t); }

int check_device_errors(dnaln_ctx* c, uint32_t bits) {
  if (bits == 0) return DNALN_OK;
  return fail(c, DNALN_ERR_DEVICE, "kernel error flags 0x%x (traceback bounds %d, cigar overflow %d, chain scratch %d, "
                                   "probe loop %d, bulk copy wait %d)",
              bits, !!(bits & kErrTracebackBounds), !!(bits & kErrCigarOverflow), !!(bits & kErrChainScratch),
              !!(bits & kErrProbeLoop), !!(bits & kErrAsyncCopy));
}

// SW tasks of a batch whose reads differ in length, longest first (a thread's two
// alignments and a warp's 64 then have similar lengths, so no lane idles through a long
// partner's rows). *sorted = tasks when there is nothing to gain.
int sort_tasks_by_length(dnaln_ctx* c, const SwTask* tasks, int n_max, const int* n_dev, const char* tag,
                         const SwTask** sorted) {
  *sorted = tasks;
  if (n_max < 2) return DNALN_OK;
  const std::string t = tag;
  DBUF(keys_in, uint32_t, (t + "_kin").c_str(), n_max);
  DBUF(keys_out, uint32_t, (t + "_kout").c_str(), n_max);
  DBUF(idx_in, int32_t, (t + "_iin").c_str(), n_max);
  DBUF(idx_out, int32_t, (t + "_iout").c_str(), n_max);
  DBUF(out, SwTask, (t + "_sorted").c_str(), n_max);
  const KernelTrace kt = tracer(c);
  kt.begin(c->st, "k_task_keys");
  launch_task_keys(c->st, tasks, n_max, n_dev, keys_in, idx_in);
  kt.end(c->st);
  size_t tmp = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys_in, keys_out, idx_in, idx_out, n_max, 0, 17, c->st));
  DBUF(tb, uint8_t, "cub_tmp_sort", tmp);
  kt.begin(c->st, "cub_sort");
  const cudaError_t e = cub::DeviceRadixSort::SortPairs(tb, tmp, keys_in, keys_out, idx_in, idx_out, n_max, 0, 17,
                                                        c->st);
  kt.end(c->st);
  CK(e);
  kt.begin(c->st, "k_task_gather");
  launch_task_gather(c->st, tasks, n_max, n_dev, idx_out, out);
  kt.end(c->st);
  c->stats.launches += 2;
  *sorted = out;
  return DNALN_OK;
}

// Launches traceback SW over tasks [0, n_max) (count read on the device from n_dev),
// chunked so the direction-bit scratch stays within dir_cap_bytes.
int launch_sw_chunked(dnaln_ctx* c, bool tb, bool bytes_ok, const SwTask* tasks, int n_max, const int* n_dev,
                      const uint8_t* qbase, const uint8_t* tbase, const SwParams& sp, SwResult* res, int rows_max,
                      uint32_t* cig, const int64_t* cig_off) {
  if (n_max <= 0) return DNALN_OK;
  const int64_t G = kSwTaskGroup;
  const size_t dir_t = tb ? sw_dir_bytes_per_task(sp.W, rows_max) : 0;
  const size_t band_t = sw_band_bytes_per_task(sp.W, bytes_ok);
  const size_t per_group = G * (dir_t + band_t);
  int64_t chunk = ((n_max + G - 1) / G) * G;
  if (per_group > 0) {
    const int64_t groups = static_cast<int64_t>(c->dir_cap_bytes / per_group);
    chunk = std::min<int64_t>(chunk, (groups < 1 ? 1 : groups) * G);
  }
  uint32_t* dir = nullptr;
  int* band = nullptr;
  if (dir_t) {
    dir = dbuf<uint32_t>(c, "sw_dir", static_cast<size_t>(chunk) * dir_t / sizeof(uint32_t));
    if (!dir) return DNALN_ERR_OOM;
  }
  if (band_t) {
    band = dbuf<int>(c, "sw_band", static_cast<size_t>(chunk) * band_t / sizeof(int));
    if (!band) return DNALN_ERR_OOM;
  }
  int* fb = dbuf<int>(c, "sw_fb", static_cast<size_t>(chunk) + 1);
  if (!fb) return DNALN_ERR_OOM;
  const KernelTrace kt = tracer(c);
  // the kernel form: fixed by the option, or tuned once per (W, traceback, length bucket)
  // by timing every form the band width has on the first chunk (they give identical
  // results, so each later run only rewrites the same outputs)
  std::vector<SwForm> forms;
  for (int f = 0; f < kSwForms; ++f)
    if (sw_has_form(sp.W, bytes_ok, static_cast<SwForm>(f))) forms.push_back(static_cast<SwForm>(f));
  SwForm form = forms.empty() ? kSwInter : forms.front();
  bool tune = false;
  const int bucket = rows_max <= 256 ? 0 : (rows_max <= 1024 ? 1 : 2);
  const int key = sp.W | (tb ? 1 : 0) << 10 | bucket << 11;
  if (forms.size() > 1) {
    const SwForm pinned = c->sw_mode == 1 ? kSwInter : (c->sw_mode == 2 ? kSwIntra : (c->sw_mode == 3 ? kSwIntraNarrow
                                                                                                      : kSwInter));
    if (c->sw_mode != 0 && std::find(forms.begin(), forms.end(), pinned) != forms.end()) {
      form = pinned;
    } else {
      auto it = c->sw_tune.find(key);
      if (it != c->sw_tune.end()) form = static_cast<SwForm>(it->second.form);
      else if (c->capturing) return fail(c, DNALN_ERR_CUDA, "capture stopped: a kernel form is still to be tuned");
      else tune = true;
    }
  }
  for (int64_t b = 0; b < n_max; b += chunk) {
    const int cnt = static_cast<int>(n_max - b < chunk ? n_max - b : chunk);
    const auto run = [&](SwForm f) {
      const bool ok = launch_sw(c->st, tb, bytes_ok, tasks, static_cast<int>(b), cnt, n_max, n_dev, qbase, tbase, sp,
                                res, dir, rows_max, cig, cig_off, band, fb, c->d_err, &kt, f);
      c->stats.launches += static_cast<uint64_t>(sw_launches(sp.W, bytes_ok, tb));
      return ok;
    };
    if (b == 0 && tune) {
      // every form once untimed first: a kernel's first launch in a process also loads it
      for (SwForm f : forms)
        if (!run(f)) return fail(c, DNALN_ERR_DEVICE, "SW launch without its scratch (W=%d)", sp.W);
      double ms[kSwForms] = {0, 0, 0};
      CK(cudaEventRecord(c->tune_ev[0], c->st));
      for (size_t x = 0; x < forms.size(); ++x) {
        if (!run(forms[x])) return fail(c, DNALN_ERR_DEVICE, "SW launch without its scratch (W=%d)", sp.W);
        CK(cudaEventRecord(c->tune_ev[1 + x], c->st));
      }
      int64_t live = cnt;
      if (n_dev) {
        CK(cudaMemcpyAsync(c->h_tune, n_dev, sizeof(int), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        live = std::min<int64_t>(cnt, *c->h_tune);
      } else {
        CK(cudaEventSynchronize(c->tune_ev[forms.size()]));
      }
      dnaln_sw_tuning t{};
      t.W = sp.W;
      t.traceback = tb ? 1 : 0;
      t.len_bucket = bucket;
      double best = 1e30;
      for (size_t x = 0; x < forms.size(); ++x) {
        ms[forms[x]] = ev_ms(c->tune_ev[x], c->tune_ev[1 + x]);
        if (ms[forms[x]] < best) {
          best = ms[forms[x]];
          form = forms[x];
        }
      }
      // a sample of a few tasks times launch overheads, not the forms: keep the width's
      // first form (inter-sequence where it has one)
      if (live < kSwTuneMinTasks) form = forms.front();
      t.ms_inter = sw_has_form(sp.W, bytes_ok, kSwInter) ? ms[kSwInter] : -1.0;
      t.ms_intra = sw_has_form(sp.W, bytes_ok, kSwIntra) ? ms[kSwIntra] : -1.0;
      t.ms_narrow = sw_has_form(sp.W, bytes_ok, kSwIntraNarrow) ? ms[kSwIntraNarrow] : -1.0;
      t.form = form;
      t.lanes_per_pair = sw_lanes_per_pair(sp.W, form);
      t.tasks = live;
      c->sw_tune[key] = t;
      continue;
    }
    if (!run(form)) return fail(c, DNALN_ERR_DEVICE, "SW launch without its scratch (W=%d)", sp.W);
  }
  CK(cudaGetLastError());
  return DNALN_OK;
}

// Checks that need no index.
int validate_map_params_basic(dnaln_ctx* c, const dnaln_map_params* p) {
  if (!p) return fail(c, DNALN_ERR_INVALID_ARG, "null map params");
  std::string why;
  if (!score_params_ok(p->sc, why)) return fail(c, DNALN_ERR_INVALID_ARG, "%s", why.c_str());
  if (p->max_cand < 1 || p->max_cand > 1024) return fail(c, DNALN_ERR_INVALID_ARG, "max_cand must be in [1, 1024]");
  if (p->ch.lookback < 0 || p->ch.band < 0 || p->ch.band > (1 << 20))
    return fail(c, DNALN_ERR_INVALID_ARG, "chain lookback must be >= 0 and band in [0, 2^20]");
  return DNALN_OK;
}

int validate_map_params(dnaln_ctx* c, const dnaln_map_params* p, const IndexRes& ix) {
  if (int e = validate_map_params_basic(c, p)) return e;
  if (p->k != ix.k || p->w != ix.w)
    return fail(c, DNALN_ERR_INVALID_ARG, "map k/w (%d/%d) differ from the index's (%d/%d)", p->k, p->w, ix.k, ix.w);
  return DNALN_OK;
}

// Enqueues the whole batch on the context's stream, ending with the copies of its totals
// and counters into h_info. With the batch's total bases and longest read given (hints)
// and no kernel-form tuning pending it waits for nothing, so it can be captured as a CUDA
// graph; while capturing (c->capturing) anything that would allocate, upload or wait
// fails it instead.
int map_enqueue(dnaln_ctx* c, IndexRes& ix, const char* d_seq, const int64_t* d_seq_off, const int32_t* d_seq_len,
                const uint32_t* d_hash, int64_t n, const dnaln_map_params& p, dnaln_map_record* d_out,
                uint32_t* d_cigar, int64_t cigar_cap, const BatchHints& hint, MapRun& run) {
  cudaStream_t st = c->st;
  const KernelTrace kt = tracer(c);
  c->trace_n = 0;
  c->trace_open = false;
  const uint64_t launches0 = c->stats.launches;  // the enqueue's own launches go to run.launches
  const int bw = p.sc.bw, W = 2 * bw + 1, MC = p.max_cand;
  const int chain_band = p.ch.band < bw ? p.ch.band : bw;  // src/mapper.cpp:9

  // packed offsets, total bases, longest read
  DBUF(len64, int64_t, "len64", n + 1);
  DBUF(pofs, int64_t, "pofs", n + 1);
  // info: [0] longest read, [1..3] cells, mapped, candidates (map.cuh), [4] minimizers,
  // [5] anchors of the thread path
  // [6] minimizers, [7] bases and [9] anchors of the reads left for the warp path, [8] the
  // chaining pool's fill
  DBUF(info, unsigned long long, "info", 10);
  CK(cudaMemsetAsync(info, 0, 10 * sizeof(unsigned long long), st));
  CK(cudaMemsetAsync(c->d_err, 0, sizeof(uint32_t), st));
  CK(cudaMemsetAsync(c->d_count, 0, 4 * sizeof(int), st));
  // work-stealing claim counters: [1] warp chaining kernel ([0] spare)
  DBUF(claims, int, "claims", 2);
  CK(cudaMemsetAsync(claims, 0, 2 * sizeof(int), st));
  unsigned long long* ctr = info + 1;  // cells, mapped, candidates (map.cuh)
  kt.begin(st, "k_len64");
  k_len64<<<nblk(n + 1), 256, 0, st>>>(d_seq_len, n, len64, info);
  kt.end(st);
  if (int e = exclusive_scan(c, len64, pofs, n + 1)) return e;
  int64_t B = hint.bases, max_len = hint.max_len;
  if (B < 0 || max_len < 0) {
    if (c->capturing) return fail(c, DNALN_ERR_CUDA, "capture needs the batch's size");
    CK(cudaMemcpyAsync(c->h_info, pofs + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(c->h_info + 1, info, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    B = c->h_info[0];
    max_len = c->h_info[1];
  }
  if (max_len > (1 << 28)) return fail(c, DNALN_ERR_INVALID_ARG, "read longer than 2^28 bases");

  // pass 1: encode, sketch, probe
  DBUF(codes, uint8_t, "codes", 2 * B);
  MinBuf mb;
  mb.hash = dbuf<uint64_t>(c, "m_hash", B);
  mb.pos = dbuf<uint32_t>(c, "m_pos", B);
  mb.hit_off = dbuf<uint32_t>(c, "m_off", B);
  mb.hit_cnt = dbuf<uint32_t>(c, "m_cnt", B);
  if (!mb.hash || !mb.pos || !mb.hit_off || !mb.hit_cnt) return DNALN_ERR_OOM;
  DBUF(n_min, int32_t, "n_min", n);
  DBUF(n_anchor, int64_t, "n_anchor", n + 1);
  SeedParams sp{p.k, p.w, p.max_occ};
  CandBuf cb;
  cb.n_cand = dbuf<int32_t>(c, "cand_n", n);
  cb.rev = dbuf<uint8_t>(c, "cand_rev", n * MC);
  cb.contig = dbuf<int32_t>(c, "cand_contig", n * MC);
  cb.diag = dbuf<int64_t>(c, "cand_diag", n * MC);
  cb.wstart = dbuf<int64_t>(c, "cand_wstart", n * MC);
  if (!cb.n_cand || !cb.rev || !cb.contig || !cb.diag || !cb.wstart) return DNALN_ERR_OOM;
  const int32_t* d_lut = nullptr;
  if (int e = chain_lut_dev(c, p.k, chain_band, &d_lut)) return e;
  ChainParamsDev cp{p.ch.max_gap, chain_band, p.ch.lookback, p.ch.min_score, p.ch.min_anchors, p.k, d_lut};
  CandParams cand{MC, bw, p.pri_ratio};
  // short reads run passes 1 and 2 one thread per read; the rest (listed) one warp per read
  const bool thread_path = !c->warp_seed_only && seed_thread_supported(sp, cp);
  DBUF(big_list, int32_t, "big_list", n);
  DBUF(n_anc_t, int32_t, "n_anc_t", n);
  int* big_n = c->d_count + 2;
  // reads of mixed lengths: SW tasks (and the long reads of the seeding) longest first
  const bool by_length =
      c->length_order && static_cast<double>(max_len) > 1.25 * static_cast<double>(B) / static_cast<double>(n);
  // the reads left for the warp kernels: those the thread kernels listed
  int32_t* warp_list = big_list;
  int* warp_n = big_n;
  CK(cudaEventRecord(c->ev[kEvSeed0], st));
  if (thread_path) {
    kt.begin(st, "k_encode_reads");
    if (c->encode_bulk)
      launch_encode_reads_bulk(st, d_seq, d_seq_off, hint.seq_base, d_seq_len, pofs, n, codes, c->d_err);
    else
      launch_encode_reads(st, d_seq, d_seq_off, hint.seq_base, d_seq_len, pofs, n, codes);
    kt.end(st);
    c->stats.launches += 1;
    const auto seed_t = [&](int rpb) {
      return launch_seed_chain_thread(st, codes, pofs, d_seq_len, n, ix.dev, sp, cp, cand, cb,
                                      n_min, n_anchor, n_anc_t, big_list, big_n, c->d_err, rpb);
    };
    int rpb = c->seed_block ? c->seed_block : (c->seed_tune.tuned ? c->seed_tune.reads_per_block : 0);
    if (rpb == 0 && (n < kSeedTuneReads || c->capturing)) rpb = 128;  // too small to time, or no host waits now
    if (rpb == 0) {
      // the reads-per-block tuner: each block size once untimed (a kernel's first launch
      // also loads it), then each timed; every run rewrites the same outputs (the list of
      // reads handed on is cleared before each), so the last run's stand
      const int sizes[2] = {64, 128};
      for (int x = 0; x < 2; ++x) {
        CK(cudaMemsetAsync(big_n, 0, sizeof(int), st));
        if (!seed_t(sizes[x])) return fail(c, DNALN_ERR_CUDA, "thread-per-read seeding kernel could not be configured");
      }
      for (int x = 0; x < 2; ++x) {
        CK(cudaMemsetAsync(big_n, 0, sizeof(int), st));
        CK(cudaEventRecord(c->tune_ev[x], st));
        if (!seed_t(sizes[x])) return fail(c, DNALN_ERR_CUDA, "thread-per-read seeding kernel could not be configured");
        CK(cudaEventRecord(c->tune_ev[x + 2], st));
      }
      CK(cudaEventSynchronize(c->tune_ev[3]));
      dnaln_seed_tuning& t = c->seed_tune;
      t.ms_64 = ev_ms(c->tune_ev[0], c->tune_ev[2]);
      t.ms_128 = ev_ms(c->tune_ev[1], c->tune_ev[3]);
      t.reads_per_block = t.ms_64 < t.ms_128 ? 64 : 128;
      t.reads = n;
      t.tuned = 1;
      c->stats.launches += 3;
    } else {
      kt.begin(st, "k_seed_chain_t");
      const bool ok = seed_t(rpb);
      kt.end(st);
      if (!ok) return fail(c, DNALN_ERR_CUDA, "thread-per-read seeding kernel could not be configured");
    }
    if (c->long_thread && seed_long_supported(sp, cp) && max_len > seed_thread_max_len()) {
      // long reads one thread each, in length order; what exceeds its bounds goes on
      const int64_t lt = seed_long_threads(n);
      DBUF(lscr, uint32_t, "long_scratch", seed_long_scratch_words(lt));
      DBUF(big2, int32_t, "big2_list", n);
      const int32_t* order = big_list;
      if (by_length && n > 1) {
        DBUF(lk_in, uint32_t, "long_kin", n);
        DBUF(lk_out, uint32_t, "long_kout", n);
        DBUF(lv_in, int32_t, "long_vin", n);
        DBUF(lv_out, int32_t, "long_vout", n);
        kt.begin(st, "k_long_keys");
        const int key_bits = launch_long_order(st, big_list, big_n, static_cast<int>(n), d_seq_len, max_len, lk_in, lv_in);
        kt.end(st);
        size_t tmp = 0;
        CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, lk_in, lk_out, lv_in, lv_out, static_cast<int>(n), 0, key_bits,
                                           st));
        DBUF(tb, uint8_t, "cub_tmp_lsort", tmp);
        kt.begin(st, "cub_sort");
        CK(cub::DeviceRadixSort::SortPairs(tb, tmp, lk_in, lk_out, lv_in, lv_out, static_cast<int>(n), 0, key_bits, st));
        kt.end(st);
        order = lv_out;
        c->stats.launches += 1;
      }
      kt.begin(st, "k_seed_chain_tl");
      if (!launch_seed_chain_long(st, d_seq_len, pofs, codes, order, big_n, lt, ix.dev, sp, cp, cand, cb, n_min,
                                  n_anchor, n_anc_t, lscr, big2, c->d_count + 3, seed_thread_max_len(), c->d_err))
        return fail(c, DNALN_ERR_CUDA, "long-read seeding kernel could not be configured");
      kt.end(st);
      warp_list = big2;
      warp_n = c->d_count + 3;
      c->stats.launches += 1;
    }
    kt.begin(st, "k_seed<list>");
    launch_seed_list(st, d_seq, d_seq_off, hint.seq_base, d_seq_len, pofs, n, warp_list, warp_n, codes, ix.dev, sp,
                     mb, n_min, n_anchor, c->d_err);
    kt.end(st);
  } else {
    kt.begin(st, "k_seed");
    launch_seed(st, d_seq, d_seq_off, hint.seq_base, d_seq_len, pofs, n, codes, ix.dev, sp, mb, n_min, n_anchor,
                c->d_err);
    kt.end(st);
  }
  CK(cudaEventRecord(c->ev[kEvSeed1], st));
  CK(cudaGetLastError());
  {  // minimizer and anchor totals (MapStats-style counters), read back with the results
    size_t tmp = 0;
    int64_t* total = reinterpret_cast<int64_t*>(info + 4);
    CK(cub::DeviceReduce::Sum(nullptr, tmp, n_min, total, n, st));
    DBUF(t, uint8_t, "cub_tmp_red", tmp);
    CK(cub::DeviceReduce::Sum(t, tmp, n_min, total, n, st));
    if (thread_path) {
      CK(cub::DeviceReduce::Sum(t, tmp, n_anc_t, total + 1, n, st));
      kt.begin(st, "k_list_sum");
      const unsigned lb = nblk(std::min<int64_t>(n, int64_t{256} * device_sm_count()));
      k_list_sum<<<lb, 256, 0, st>>>(n_min, warp_list, warp_n, info + 6);
      k_list_sum<<<lb, 256, 0, st>>>(d_seq_len, warp_list, warp_n, info + 7);
      k_list_sum64<<<lb, 256, 0, st>>>(n_anchor, warp_list, warp_n, info + 9);
      kt.end(st);
    } else {
      size_t tmp2 = 0;
      CK(cub::DeviceReduce::Sum(nullptr, tmp2, n_anchor, reinterpret_cast<int64_t*>(info + 9), n, st));
      DBUF(t2, uint8_t, "cub_tmp_red2", tmp2);
      CK(cub::DeviceReduce::Sum(t2, tmp2, n_anchor, reinterpret_cast<int64_t*>(info + 9), n, st));
    }
  }

  // pass 2 of the warp path: anchors, chains, candidates; the scratch of reads with many
  // anchors comes from a pool (sized from the previous batches; a batch that outgrows it
  // is mapped again with the size it asked for)
  const int64_t pool_cap = std::max<int64_t>(c->pool_cap, c->pool_min);
  AnchorScratch as;
  as.keys = dbuf<uint64_t>(c, "a_keys", pool_cap);
  as.f = dbuf<int32_t>(c, "a_f", pool_cap);
  as.prev = dbuf<int32_t>(c, "a_prev", pool_cap);
  as.ord = dbuf<uint64_t>(c, "a_ord", pool_cap);
  as.used = dbuf<uint8_t>(c, "a_used", pool_cap);
  as.ch_score = dbuf<int32_t>(c, "c_score", pool_cap);
  as.ch_sn = dbuf<uint32_t>(c, "c_sn", pool_cap);
  as.ch_dmin = dbuf<int64_t>(c, "c_dmin", pool_cap);
  as.ch_dmax = dbuf<int64_t>(c, "c_dmax", pool_cap);
  as.ch_rpos = dbuf<uint32_t>(c, "c_rpos", pool_cap);
  if (!as.keys || !as.f || !as.prev || !as.ord || !as.used || !as.ch_score || !as.ch_sn || !as.ch_dmin ||
      !as.ch_dmax || !as.ch_rpos)
    return DNALN_ERR_OOM;
  unsigned long long* pool_top = info + 8;
  CK(cudaEventRecord(c->ev[kEvChain0], st));
  kt.begin(st, thread_path ? "k_chain_map<list>" : "k_chain_map");
  launch_chain_map(st, pofs, d_seq_len, n, thread_path ? warp_list : nullptr, thread_path ? warp_n : nullptr, n_min,
                   n_anchor, mb, ix.dev, cp, cand, as, pool_top, pool_cap, cb, c->stealing ? claims + 1 : nullptr,
                   c->d_err);
  kt.end(st);
  CK(cudaEventRecord(c->ev[kEvChain1], st));
  CK(cudaGetLastError());
  // score-only ranking of multi-candidate reads
  const dnaln_score_params& sc = p.sc;
  const SwParams swp = make_sw_params(sc);
  const bool bytes_ok = sw_bytes_ok(sc);
  MapConsts mc{MC, bw, W, p.min_aln_score, sc.match};
  DBUF(sc_tasks, SwTask, "sc_tasks", n * MC);
  DBUF(res_sc, SwResult, "res_sc", n * MC);
  CK(cudaEventRecord(c->ev[kEvSc0], st));
  kt.begin(st, "k_score_tasks");
  launch_score_tasks(st, n, pofs, d_seq_len, cb, ix.dev, mc, sc_tasks, c->d_count, ctr);
  kt.end(st);
  // reads of very different lengths: SW tasks longest first (lengths known on the host)
  const SwTask* sc_run = sc_tasks;
  if (by_length)
    if (int e = sort_tasks_by_length(c, sc_tasks, static_cast<int>(n * MC), c->d_count, "sc", &sc_run)) return e;
  if (int e = launch_sw_chunked(c, false, bytes_ok, sc_run, static_cast<int>(n * MC), c->d_count, codes,
                                ix.dev.genome, swp, res_sc, static_cast<int>(max_len), nullptr, nullptr))
    return e;
  CK(cudaEventRecord(c->ev[kEvSc1], st));

  // choose, then traceback on the chosen candidate
  DBUF(chosen, int32_t, "chosen", n);
  DBUF(s2, int32_t, "s2", n);
  DBUF(tb_tasks, SwTask, "tb_tasks", n);
  DBUF(res_tb, SwResult, "res_tb", n);
  DBUF(cig_tb, uint32_t, "cig_tb", 2 * B + n);
  DBUF(cig_slot, int64_t, "cig_slot", n);
  CK(cudaEventRecord(c->ev[kEvTb0], st));
  kt.begin(st, "k_choose");
  launch_choose(st, n, pofs, d_seq_len, cb, res_sc, d_hash, ix.dev, mc, chosen, s2, tb_tasks, c->d_count + 1, ctr);
  kt.end(st);
  kt.begin(st, "k_cig_slots");
  k_cig_slots<<<nblk(n), 256, 0, st>>>(pofs, n, cig_slot);
  kt.end(st);
  const SwTask* tb_run = tb_tasks;
  if (by_length)
    if (int e = sort_tasks_by_length(c, tb_tasks, static_cast<int>(n), c->d_count + 1, "tb", &tb_run)) return e;
  if (int e = launch_sw_chunked(c, true, bytes_ok, tb_run, static_cast<int>(n), c->d_count + 1, codes,
                                ix.dev.genome, swp, res_tb, static_cast<int>(max_len), cig_tb, cig_slot))
    return e;
  CK(cudaEventRecord(c->ev[kEvTb1], st));

  // records, CIGAR offsets and compaction
  DBUF(cig_cnt, int64_t, "cig_cnt", n + 1);
  DBUF(cig_off, int64_t, "cig_off", n + 1);
  CK(cudaEventRecord(c->ev[kEvPost0], st));
  kt.begin(st, "k_records");
  launch_records(st, n, d_seq_len, cb, chosen, s2, res_tb, ix.dev, mc, d_out, cig_cnt, ctr);
  kt.end(st);
  if (int e = exclusive_scan(c, cig_cnt, cig_off, n + 1)) return e;
  // final CIGARs: into the caller's buffer, or an internal one of the bound 2 * len + 3 per
  // read; the kernel checks the capacity itself, so nothing waits for the total here
  if (!d_cigar) {
    cigar_cap = 2 * B + 3 * n;
    d_cigar = dbuf<uint32_t>(c, "cig_out", cigar_cap);
    if (!d_cigar) return DNALN_ERR_OOM;
  }
  kt.begin(st, "k_cigar_gather");
  launch_cigar_gather(st, n, pofs, d_seq_len, res_tb, cig_tb, cig_off, hint.cigar_base, d_out, d_cigar, cigar_cap,
                      c->d_err);
  kt.end(st);
  CK(cudaEventRecord(c->ev[kEvPost1], st));
  CK(cudaGetLastError());
  // the batch's one read-back: totals, task counts, error flags, counters
  int64_t* h = c->h_info;
  CK(cudaMemcpyAsync(h, cig_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(h + 1, c->d_count, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(h + 3, c->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(h + 4, ctr, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(h + 7, info + 4, 6 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  run.B = B;
  run.max_len = max_len;
  run.cigar_cap = cigar_cap;
  run.d_cigar = d_cigar;
  run.thread_path = thread_path;
  run.long_used = warp_list != big_list;
  run.launches = c->stats.launches - launches0;
  c->stats.launches = launches0;
  return DNALN_OK;
}

int run_map(dnaln_ctx* c, IndexRes& ix, const char* d_seq, const int64_t* d_seq_off, const int32_t* d_seq_len,
            const uint32_t* d_hash, int64_t n, const dnaln_map_params& p, dnaln_map_record* d_out, uint32_t* d_cigar,
            int64_t cigar_cap, int64_t* cigar_used, uint32_t** cigar_dev, const BatchHints& hint);

// Waits for an enqueued batch and turns its read-back into the call's result and the
// context's counters; a batch that outgrew the chaining pool is mapped again.
int map_finish(dnaln_ctx* c, IndexRes& ix, const char* d_seq, const int64_t* d_seq_off, const int32_t* d_seq_len,
               const uint32_t* d_hash, int64_t n, const dnaln_map_params& p, dnaln_map_record* d_out,
               int64_t* cigar_used, uint32_t** cigar_dev, const BatchHints& hint, const MapRun& run) {
  cudaStream_t st = c->st;
  const int64_t B = run.B, max_len = run.max_len, cigar_cap = run.cigar_cap;
  const bool thread_path = run.thread_path;
  int64_t* h = c->h_info;
  CK(cudaStreamSynchronize(st));
  const int64_t total_ops = h[0];
  int counts[4];
  std::memcpy(counts, h + 1, sizeof counts);
  uint32_t errbits;
  std::memcpy(&errbits, h + 3, sizeof errbits);
  const uint64_t n_cells = static_cast<uint64_t>(h[4]), n_mapped = static_cast<uint64_t>(h[5]),
                 n_cands = static_cast<uint64_t>(h[6]);
  const int64_t n_minimizers = h[7], n_anchors_thread = h[8], n_minimizers_warp_l = h[9], n_bases_warp_l = h[10];
  const int64_t pool_used = h[11], n_anchors_warp = h[12];
  if (errbits & kErrChainPool) {
    // the chaining pool was too small for this batch: grow it to what the batch asked for
    // and map the batch again (outputs are rewritten in full; counters are not yet added)
    c->pool_cap = std::max<int64_t>(c->pool_cap, pool_used + pool_used / 4 + 1024);
    if (hint.retry) return fail(c, DNALN_ERR_DEVICE, "chaining pool still too small after growing it");
    c->stats.batch_retries += 1;
    BatchHints again = hint;
    again.retry = true;
    again.bases = B;
    again.max_len = max_len;
    trace_collect(c);
    return run_map(c, ix, d_seq, d_seq_off, d_seq_len, d_hash, n, p, d_out, hint.caller_cigar ? run.d_cigar : nullptr,
                   hint.caller_cigar ? cigar_cap : 0, cigar_used, cigar_dev, again);
  }
  if (cigar_dev) *cigar_dev = run.d_cigar;
  if (pool_used > c->pool_cap / 2) c->pool_cap = std::max<int64_t>(c->pool_cap, pool_used + pool_used / 2);
  *cigar_used = total_ops;
  if (errbits & kErrOutputCapacity)
    return fail(c, DNALN_ERR_CAPACITY, "CIGAR buffer holds %lld ops, batch needs %lld",
                static_cast<long long>(cigar_cap), static_cast<long long>(total_ops));
  if (int e = check_device_errors(c, errbits)) return e;
  trace_collect(c);

  const int n_listed = counts[2];                                        // reads the short thread kernel listed
  const int n_warp = thread_path ? counts[run.long_used ? 3 : 2] : static_cast<int>(n);  // warp kernels
  dnaln_stats& s = c->stats;
  s.reads += static_cast<uint64_t>(n);
  s.anchors += static_cast<uint64_t>(n_anchors_thread + n_anchors_warp);
  s.minimizers += static_cast<uint64_t>(n_minimizers);
  s.warp_reads += static_cast<uint64_t>(n_warp);
  s.warp_minimizers += static_cast<uint64_t>(thread_path ? n_minimizers_warp_l : n_minimizers);
  s.warp_anchors += static_cast<uint64_t>(n_anchors_warp);
  s.warp_bases += static_cast<uint64_t>(thread_path ? n_bases_warp_l : B);
  s.long_reads += static_cast<uint64_t>(thread_path && run.long_used ? n_listed - n_warp : 0);
  s.sw_tasks_score += static_cast<uint64_t>(counts[0]);
  s.sw_tasks_tb += static_cast<uint64_t>(counts[1]);
  s.cells += n_cells;
  s.mapped += n_mapped;
  s.candidates += n_cands;
  // k_len64, k_score_tasks, k_choose, k_cig_slots, k_records, k_cigar_gather, pass 1 / 2,
  // plus the SW and sorting kernels the enqueue counted
  s.launches += 7 + (thread_path ? 5 : 1) + run.launches;
  s.ms_seed += ev_ms(c, kEvSeed0, kEvSeed1);
  s.ms_chain += ev_ms(c, kEvChain0, kEvChain1);
  s.ms_sw_score += ev_ms(c, kEvSc0, kEvSc1);
  s.ms_sw_tb += ev_ms(c, kEvTb0, kEvTb1);
  s.ms_post += ev_ms(c, kEvPost0, kEvPost1);
  s.ms_total += ev_ms(c, kEvSeed0, kEvPost1);
  s.graph_launches = c->graph_launches;
  return DNALN_OK;
}

// Everything that decides the launches of a batch and their arguments, as bytes: a cached
// graph is replayed only for an identical key captured at the current buffer epoch.
std::string graph_key(const dnaln_ctx* c, const IndexRes& ix, const char* d_seq, const int64_t* d_seq_off,
                      const int32_t* d_seq_len, const uint32_t* d_hash, int64_t n, const dnaln_map_params& p,
                      const dnaln_map_record* d_out, const uint32_t* d_cigar, int64_t cigar_cap,
                      const BatchHints& hint) {
  std::string k;
  const auto put = [&](const void* v, size_t bytes) { k.append(static_cast<const char*>(v), bytes); };
  put(&ix.dev, sizeof ix.dev);  // every pointer and dimension of the index the kernels take
  const void* ptrs[] = {d_seq, d_seq_off, d_seq_len, d_hash, d_out, d_cigar, c->st};
  put(ptrs, sizeof ptrs);
  const int64_t nums[] = {n, hint.seq_base, hint.bases, hint.max_len, hint.cigar_base, cigar_cap, c->pool_cap,
                          static_cast<int64_t>(c->dir_cap_bytes), c->sw_mode, c->warp_seed_only, c->long_thread,
                          c->length_order, c->stealing, c->encode_bulk, c->seed_block,
                          c->seed_tune.tuned ? c->seed_tune.reads_per_block : 0};
  put(nums, sizeof nums);
  put(&p, sizeof p);
  return k;
}

// The device pipeline. Inputs and d_out in device memory; CIGARs go to d_cigar
// (capacity cigar_cap) or, when d_cigar is null, to an internal buffer returned via
// *cigar_dev. *cigar_used = total ops.
//
// A batch whose size is known on the host (hints) is a candidate for a CUDA graph: the
// first time its key is seen it runs eagerly (growing buffers, tuning kernel forms); the
// second time, with nothing reallocated since, its launches are captured into a graph;
// from then on the graph is launched, one launch for the batch's ~30 kernels, copies and
// event records.
int run_map(dnaln_ctx* c, IndexRes& ix, const char* d_seq, const int64_t* d_seq_off, const int32_t* d_seq_len,
            const uint32_t* d_hash, int64_t n, const dnaln_map_params& p, dnaln_map_record* d_out, uint32_t* d_cigar,
            int64_t cigar_cap, int64_t* cigar_used, uint32_t** cigar_dev, const BatchHints& hint0) {
  *cigar_used = 0;
  if (n == 0) return DNALN_OK;
  BatchHints hint = hint0;
  hint.caller_cigar = d_cigar != nullptr;
  if ((hint.bases < 0 || hint.max_len < 0) && c->graphs && !c->trace_on) {
    // the batch's size first (two small kernels and one read-back), so that the rest of it
    // can run as a graph
    cudaStream_t st = c->st;
    DBUF(len64, int64_t, "len64", n + 1);
    DBUF(pofs, int64_t, "pofs", n + 1);
    DBUF(info, unsigned long long, "info", 10);
    CK(cudaMemsetAsync(info, 0, sizeof(unsigned long long), st));
    k_len64<<<nblk(n + 1), 256, 0, st>>>(d_seq_len, n, len64, info);
    if (int e = exclusive_scan(c, len64, pofs, n + 1)) return e;
    CK(cudaMemcpyAsync(c->h_info, pofs + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(c->h_info + 1, info, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    hint.bases = c->h_info[0];
    hint.max_len = c->h_info[1];
    c->stats.launches += 1;
  }
  const bool graphable = c->graphs && hint.bases >= 0 && hint.max_len >= 0 && !c->trace_on && !hint.retry;
  std::string key;
  if (graphable) {
    key = graph_key(c, ix, d_seq, d_seq_off, d_seq_len, d_hash, n, p, d_out, d_cigar, cigar_cap, hint);
    auto it = c->graph_cache.find(key);
    if (it != c->graph_cache.end() && it->second.epoch == c->epoch) {
      CK(cudaGraphLaunch(it->second.exec, c->st));
      ++c->graph_launches;
      return map_finish(c, ix, d_seq, d_seq_off, d_seq_len, d_hash, n, p, d_out, cigar_used, cigar_dev, hint,
                        it->second.run);
    }
    if (it != c->graph_cache.end()) {  // captured before a reallocation: stale
      cudaGraphExecDestroy(it->second.exec);
      c->graph_cache.erase(it);
    }
    auto seen = c->graph_seen.find(key);
    if (seen != c->graph_seen.end() && seen->second == c->epoch) {
      // second sighting with the same buffers: capture, instantiate, launch
      if (c->graph_cache.size() >= 64) {
        for (auto& kv : c->graph_cache) cudaGraphExecDestroy(kv.second.exec);
        c->graph_cache.clear();
      }
      MapRun run;
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
      c->capturing = true;
      const int e = map_enqueue(c, ix, d_seq, d_seq_off, d_seq_len, d_hash, n, p, d_out, d_cigar, cigar_cap, hint,
                                run);
      c->capturing = false;
      const cudaError_t ce = cudaStreamEndCapture(c->st, &g);
      cudaGraphExec_t x = nullptr;
      if (e == DNALN_OK && ce == cudaSuccess && g && cudaGraphInstantiate(&x, g, 0) == cudaSuccess) {
        cudaGraphDestroy(g);
        c->graph_cache[key] = CachedGraph{x, c->epoch, run};
        CK(cudaGraphLaunch(x, c->st));
        ++c->graph_launches;
        return map_finish(c, ix, d_seq, d_seq_off, d_seq_len, d_hash, n, p, d_out, cigar_used, cigar_dev, hint, run);
      }
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      c->graph_seen.erase(key);  // not capturable now: run eagerly below
    }
  }
  MapRun run;
  if (int e = map_enqueue(c, ix, d_seq, d_seq_off, d_seq_len, d_hash, n, p, d_out, d_cigar, cigar_cap, hint, run))
    return e;
  if (graphable) {
    if (c->graph_seen.size() > 4096) c->graph_seen.clear();
    c->graph_seen[key] = c->epoch;
  }
  return map_finish(c, ix, d_seq, d_seq_off, d_seq_len, d_hash, n, p, d_out, cigar_used, cigar_dev, hint, run);
}

IndexRes* find_index(dnaln_ctx* c, int32_t id) {
  auto it = c->idx.find(id);
  if (it == c->idx.end()) {
    fail(c, DNALN_ERR_NOT_FOUND, "unknown index id %d", id);
    return nullptr;
  }
  return &it->second;
}

int dalloc(dnaln_ctx* c, DevBuf& b, size_t bytes) {
  if (c->fail_alloc_after >= 0 && c->fail_alloc_after-- == 0) {
    b.p = nullptr;
    return fail(c, DNALN_ERR_OOM, "out of device memory allocating %zu bytes for the index (injected)", bytes);
  }
  if (cudaMalloc(&b.p, bytes ? bytes : 1) != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    return fail(c, DNALN_ERR_OOM, "out of device memory allocating %zu bytes for the index", bytes);
  }
  b.cap = bytes;
  return DNALN_OK;
}

// Drops this holder's reference; the memory goes with the last one.
void free_index(IndexRes& r) { r.mem.reset(); }

// Points r.dev at r.mem's buffers, fills its scalars from r and registers r under a new id.
void register_index(dnaln_ctx* c, IndexRes& r, uint64_t mask, int32_t n_n_runs, int32_t* index_id) {
  IndexMem& m = *r.mem;
  r.dev.table = static_cast<const ulonglong2*>(m.table.p);
  r.dev.positions = static_cast<const uint32_t*>(m.positions.p);
  r.dev.genome = static_cast<const uint8_t*>(m.genome.p);
  r.dev.contig_off = static_cast<const uint64_t*>(m.coff.p);
  r.dev.contig_len = static_cast<const uint32_t*>(m.clen.p);
  r.dev.n_runs = static_cast<const uint2*>(m.nruns.p);
  r.dev.n_n_runs = n_n_runs;
  r.dev.mask = mask;
  r.dev.n_contigs = r.n_contigs;
  r.dev.k = r.k;
  r.dev.w = r.w;
  const int32_t id = c->next_id++;
  c->idx[id] = r;
  *index_id = id;
}

// Checks a contig table against the genome length: in bounds and in order.
int check_contigs(dnaln_ctx* c, const uint64_t* contig_off, const uint32_t* contig_len, int32_t n_contigs,
                  uint64_t n_bases, int code) {
  for (int32_t i = 0; i < n_contigs; ++i)
    if (contig_off[i] + contig_len[i] > n_bases || (i > 0 && contig_off[i] < contig_off[i - 1]))
      return fail(c, code, "contig %d is outside the genome or out of order", i);
  return DNALN_OK;
}

// Structural checks of a bucket table / position array, chunk by chunk: every non-empty
// bucket's positions lie inside the array, every position inside the genome. Counts the
// non-empty buckets and the largest count.
struct TableCheck {
  uint64_t n_pos = 0, n_bases = 0, n_keys = 0;
  uint32_t max_count = 0;
  bool ok = true;
  void buckets(const ulonglong2* t, size_t n) {
    for (size_t i = 0; i < n; ++i) {
      if (t[i].x == kInvalidHash) continue;
      const uint64_t off = static_cast<uint32_t>(t[i].y), cnt = t[i].y >> 32;
      ok = ok && off + cnt <= n_pos;
      ++n_keys;
      if (cnt > max_count) max_count = static_cast<uint32_t>(cnt);
    }
  }
  void positions(const uint32_t* v, size_t n) {
    for (size_t i = 0; i < n; ++i) ok = ok && (v[i] >> 1) < n_bases;
  }
};


// ---- the worker behind dnaln_gpu_map_submit ----------------------------------------------
// Parts are taken from the queue in order. While part j computes on the context's stream
// (run_map), part j+1's reads are already on their way into the other device slot (copy
// stream cp_in) and part j-1's records and CIGARs are on their way back (cp_out), so the
// host<->device traffic of full-size batches hides behind the kernels of their neighbours.

struct SlotBufs {
  char* seq = nullptr;
  int64_t* off = nullptr;
  int32_t* len = nullptr;
  uint32_t* hash = nullptr;
  dnaln_map_record* out = nullptr;
  uint32_t* cig = nullptr;
};

const char* const kSlotNames[2][6] = {{"in_seq0", "in_off0", "in_len0", "in_hash0", "out_rec0", "out_cig0"},
                                      {"in_seq1", "in_off1", "in_len1", "in_hash1", "out_rec1", "out_cig1"}};

bool pop_part(dnaln_ctx* c, MapPart& pt) {
  std::lock_guard<std::mutex> g(c->qmu);
  if (c->queue.empty()) return false;
  pt = c->queue.front();
  c->queue.pop_front();
  return true;
}

// Copies a part's reads into slot k (stream cp_in) and records in_ready[k].
int stage_in(dnaln_ctx* c, int k, const MapPart& pt, SlotBufs& sb) {
  const int64_t m = pt.b - pt.a;
  sb.seq = dbuf<char>(c, kSlotNames[k][0], pt.hi - pt.lo);
  sb.off = dbuf<int64_t>(c, kSlotNames[k][1], m);
  sb.len = dbuf<int32_t>(c, kSlotNames[k][2], m);
  sb.hash = dbuf<uint32_t>(c, kSlotNames[k][3], m);
  if (!sb.seq || !sb.off || !sb.len || !sb.hash) return DNALN_ERR_OOM;
  CK(cudaEventRecord(c->h2d_ev[2 * k], c->cp_in));
  if (pt.hi > pt.lo) CK(cudaMemcpyAsync(sb.seq, pt.seq + pt.lo, pt.hi - pt.lo, cudaMemcpyHostToDevice, c->cp_in));
  CK(cudaMemcpyAsync(sb.off, pt.seq_off + pt.a, m * sizeof(int64_t), cudaMemcpyHostToDevice, c->cp_in));
  CK(cudaMemcpyAsync(sb.len, pt.seq_len + pt.a, m * sizeof(int32_t), cudaMemcpyHostToDevice, c->cp_in));
  CK(cudaMemcpyAsync(sb.hash, pt.name_hash + pt.a, m * sizeof(uint32_t), cudaMemcpyHostToDevice, c->cp_in));
  CK(cudaEventRecord(c->h2d_ev[2 * k + 1], c->cp_in));
  CK(cudaEventRecord(c->in_ready[k], c->cp_in));
  return DNALN_OK;
}

struct PendingPart {  // a part whose results are being copied out of slot k
  bool active = false;
  MapPart pt;
  int status = DNALN_OK;
};

// Records a finished part; the last part of a ticket publishes the ticket's status.
void finish_part(dnaln_ctx* c, int k, PendingPart& pp) {
  if (!pp.active) return;
  pp.active = false;
  if (pp.status == DNALN_OK) c->stats.ms_d2h += ev_ms(c->d2h_ev[2 * k], c->d2h_ev[2 * k + 1]);
  {
    std::lock_guard<std::mutex> g(c->qmu);
    const int64_t t = pp.pt.ticket;
    if (pp.status != DNALN_OK && !c->first_err.count(t)) c->first_err[t] = pp.status;
    if (pp.pt.last) {
      auto fe = c->first_err.find(t);
      const int st = fe == c->first_err.end() ? DNALN_OK : fe->second;
      if (fe != c->first_err.end()) c->first_err.erase(fe);
      *pp.pt.cigar_used = c->ticket_ops[t];
      c->ticket_ops.erase(t);
      c->results[t] = st;
    }
  }
  if (pp.pt.last) c->qcv.notify_all();
}

// Runs part pt (inputs in slot k) and starts copying its results out. Returns the part's status.
int compute_part(dnaln_ctx* c, int k, const MapPart& pt, const SlotBufs& sb, int64_t base, int64_t* used) {
  *used = 0;
  IndexRes* r = find_index(c, pt.index_id);
  if (!r) return DNALN_ERR_NOT_FOUND;
  if (int e = validate_map_params(c, &pt.p, *r)) return e;
  const int64_t m = pt.b - pt.a;
  dnaln_map_record* d_out = dbuf<dnaln_map_record>(c, kSlotNames[k][4], m);
  uint32_t* d_cig = dbuf<uint32_t>(c, kSlotNames[k][5], pt.cig_bound);
  if (!d_out || !d_cig) return DNALN_ERR_OOM;
  CK(cudaStreamWaitEvent(c->st, c->in_ready[k], 0));
  CK(cudaStreamWaitEvent(c->st, c->out_free[k], 0));  // the results of part j-2 have left the slot
  BatchHints hint;
  hint.seq_base = pt.lo;
  hint.bases = pt.bases;
  hint.max_len = pt.max_len;
  hint.cigar_base = base;
  if (int e = run_map(c, *r, sb.seq, sb.off, sb.len, sb.hash, m, pt.p, d_out, d_cig, pt.cig_bound, used, nullptr,
                      hint))
    return e;
  c->stats.ms_h2d += ev_ms(c->h2d_ev[2 * k], c->h2d_ev[2 * k + 1]);  // complete: run_map waited for it
  if (base + *used > pt.cigar_cap || (*used > 0 && !pt.cigar))
    return fail(c, DNALN_ERR_CAPACITY, "CIGAR buffer holds %lld ops, batch needs at least %lld",
                static_cast<long long>(pt.cigar_cap), static_cast<long long>(base + *used));
  CK(cudaEventRecord(c->d2h_ev[2 * k], c->cp_out));
  CK(cudaMemcpyAsync(pt.out + pt.a, d_out, m * sizeof(dnaln_map_record), cudaMemcpyDeviceToHost, c->cp_out));
  if (*used > 0)
    CK(cudaMemcpyAsync(pt.cigar + base, d_cig, *used * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->cp_out));
  CK(cudaEventRecord(c->d2h_ev[2 * k + 1], c->cp_out));
  CK(cudaEventRecord(c->out_free[k], c->cp_out));
  return DNALN_OK;
}

// Drives queued parts through the two slots until the queue is empty.
void drive_parts(dnaln_ctx* c) {
  PendingPart pend[2];
  SlotBufs sb[2];
  MapPart pt;
  if (!pop_part(c, pt)) return;
  int k = 0;
  int staged = stage_in(c, k, pt, sb[k]);
  for (;;) {
    MapPart nx;
    const bool have_next = pop_part(c, nx);
    int next_staged = DNALN_OK;
    if (have_next) next_staged = stage_in(c, 1 - k, nx, sb[1 - k]);  // slot 1-k's inputs are free
    int64_t base = 0;
    bool failed = false;
    {
      std::lock_guard<std::mutex> g(c->qmu);
      base = c->ticket_ops[pt.ticket];
      failed = c->first_err.count(pt.ticket) != 0;
    }
    int64_t used = 0;
    int st = staged;
    if (st == DNALN_OK && failed) st = DNALN_ERR_INVALID_ARG;  // an earlier part of the ticket failed
    if (st == DNALN_OK) st = compute_part(c, k, pt, sb[k], base, &used);
    // the stream is idle (run_map synchronised it after waiting for out_free[k]): the part
    // that used slot k before is fully copied out
    finish_part(c, k, pend[k]);
    if (st == DNALN_OK) {
      std::lock_guard<std::mutex> g(c->qmu);
      c->ticket_ops[pt.ticket] = base + used;
    }
    pend[k].pt = pt;
    pend[k].status = st;
    pend[k].active = true;
    if (st != DNALN_OK) {
      cudaStreamSynchronize(c->cp_out);
      finish_part(c, 1 - k, pend[1 - k]);
      finish_part(c, k, pend[k]);
    } else if (pend[1 - k].active && cudaEventQuery(c->out_free[1 - k]) == cudaSuccess) {
      finish_part(c, 1 - k, pend[1 - k]);
    }
    cudaGetLastError();
    if (!have_next) break;
    pt = nx;
    staged = next_staged;
    k = 1 - k;
  }
  cudaStreamSynchronize(c->cp_out);
  finish_part(c, 1 - k, pend[1 - k]);  // older first
  finish_part(c, k, pend[k]);
}

void map_worker(dnaln_ctx* c) {
  cudaSetDevice(c->device);
  std::unique_lock<std::mutex> ql(c->qmu);
  for (;;) {
    c->qcv.wait(ql, [&] { return c->stop || !c->queue.empty(); });
    if (c->queue.empty()) break;  // stopping, nothing left
    ql.unlock();
    {
      std::lock_guard<std::mutex> g(c->mu);
      drive_parts(c);
    }
    ql.lock();
  }
}
}  // namespace

extern "C" {

const char* dnaln_gpu_version(void) { return "dnaln-b200 0.1.0 (sm_100a)"; }

uint32_t dnaln_fnv1a(const char* s, int64_t n) {  // src/common.hpp:136-140
  uint32_t h = 2166136261u;
  for (int64_t i = 0; i < n; ++i) h = (h ^ static_cast<unsigned char>(s[i])) * 16777619u;
  return h;
}

void dnaln_fnv1a_batch(const char* names, const int64_t* name_off, int64_t n, uint32_t* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = dnaln_fnv1a(names + name_off[i], name_off[i + 1] - name_off[i]);
}

int dnaln_gpu_ctx_create(int device, dnaln_ctx** out) {
  if (!out) return DNALN_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return DNALN_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return DNALN_ERR_NO_DEVICE;
  auto* c = new dnaln_ctx;
  c->device = device;
  int e = DNALN_OK;
  auto bad = [&](cudaError_t x) {
    if (x != cudaSuccess && e == DNALN_OK) e = fail(c, DNALN_ERR_CUDA, "%s", cudaGetErrorString(x));
  };
  bad(cudaSetDevice(device));
  {  // direction-code scratch: 1/32 of the device's memory, in [1, 8] GiB, so that a
     // traceback launch over long reads and wide bands still holds enough tasks to fill
     // the SMs (1 GiB held ~16,000 1,000-row tasks at W = 129: ~1.7 blocks per SM)
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess)
      c->dir_cap_bytes = std::min<size_t>(size_t(8) << 30, std::max<size_t>(size_t(1) << 30, prop.totalGlobalMem / 32));
    else
      cudaGetLastError();
  }
  bad(cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking));
  c->st = c->own;
  for (auto& x : c->ev) bad(cudaEventCreate(&x));
  bad(cudaStreamCreateWithFlags(&c->cp_in, cudaStreamNonBlocking));
  bad(cudaStreamCreateWithFlags(&c->cp_out, cudaStreamNonBlocking));
  for (auto& x : c->in_ready) bad(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
  for (auto& x : c->out_free) bad(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
  for (auto& x : c->h2d_ev) bad(cudaEventCreate(&x));
  for (auto& x : c->d2h_ev) bad(cudaEventCreate(&x));
  bad(cudaMalloc(&c->d_err, sizeof(uint32_t)));
  bad(cudaMalloc(&c->d_count, 4 * sizeof(int)));
  bad(cudaHostAlloc(&c->h_info, 16 * sizeof(int64_t), cudaHostAllocDefault));
  bad(cudaHostAlloc(&c->h_tune, sizeof(int), cudaHostAllocDefault));
  for (auto& x : c->tune_ev) bad(cudaEventCreate(&x));
  if (e != DNALN_OK) {
    dnaln_gpu_ctx_destroy(c);
    return e;
  }
  *out = c;
  return DNALN_OK;
}

int dnaln_gpu_ctx_destroy(dnaln_ctx* c) {
  if (!c) return DNALN_OK;
  {  // the worker finishes what is queued, then exits
    std::lock_guard<std::mutex> g(c->qmu);
    c->stop = true;
  }
  c->qcv.notify_all();
  if (c->worker.joinable()) c->worker.join();
  cudaSetDevice(c->device);
  if (c->st) cudaStreamSynchronize(c->st);
  for (auto& kv : c->graph_cache) cudaGraphExecDestroy(kv.second.exec);
  c->graph_cache.clear();
  for (auto& kv : c->idx) free_index(kv.second);
  for (auto& kv : c->bufs)
    if (kv.second.p) cudaFree(kv.second.p);
  if (c->cp_in) cudaStreamSynchronize(c->cp_in);
  if (c->cp_out) cudaStreamSynchronize(c->cp_out);
  for (auto& x : c->ev)
    if (x) cudaEventDestroy(x);
  for (cudaEvent_t* set : {c->in_ready, c->out_free})
    for (int i = 0; i < 2; ++i)
      if (set[i]) cudaEventDestroy(set[i]);
  for (cudaEvent_t* set : {c->h2d_ev, c->d2h_ev})
    for (int i = 0; i < 4; ++i)
      if (set[i]) cudaEventDestroy(set[i]);
  for (auto& x : c->trace_ev)
    if (x) cudaEventDestroy(x);
  if (c->cp_in) cudaStreamDestroy(c->cp_in);
  if (c->cp_out) cudaStreamDestroy(c->cp_out);
  if (c->d_err) cudaFree(c->d_err);
  if (c->d_count) cudaFree(c->d_count);
  if (c->h_info) cudaFreeHost(c->h_info);
  if (c->h_tune) cudaFreeHost(c->h_tune);
  for (auto& x : c->tune_ev)
    if (x) cudaEventDestroy(x);
  if (c->h_lut) cudaFreeHost(c->h_lut);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
  return DNALN_OK;
}

const char* dnaln_gpu_last_error(const dnaln_ctx* c) { return c ? c->err.c_str() : "null context"; }

int dnaln_gpu_ctx_device(const dnaln_ctx* c, int32_t* device) {
  if (!c || !device) return DNALN_ERR_INVALID_ARG;
  *device = c->device;
  return DNALN_OK;
}

int dnaln_gpu_set_stream(dnaln_ctx* c, void* stream) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c) return DNALN_ERR_INVALID_ARG;
  c->st = stream ? static_cast<cudaStream_t>(stream) : c->own;
  return DNALN_OK;
}

int dnaln_gpu_get_stats(const dnaln_ctx* c, dnaln_stats* out) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c || !out) return DNALN_ERR_INVALID_ARG;
  *out = c->stats;
  return DNALN_OK;
}

int dnaln_gpu_reset_stats(dnaln_ctx* c) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c) return DNALN_ERR_INVALID_ARG;
  c->stats = dnaln_stats{};
  c->ktimes.clear();
  return DNALN_OK;
}

int dnaln_gpu_set_kernel_trace(dnaln_ctx* c, int32_t on, const char* only) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c) return DNALN_ERR_INVALID_ARG;
  c->trace_only = only ? only : "";
  if (on && c->trace_ev.empty()) {
    if (int e = set_device(c)) return e;
    c->trace_ev.assign(2 * kMaxTrace, nullptr);
    for (auto& x : c->trace_ev) CK(cudaEventCreate(&x));
  }
  c->trace_on = on != 0;
  c->trace_n = 0;
  c->trace_open = false;
  return DNALN_OK;
}

int dnaln_gpu_kernel_times(const dnaln_ctx* c, dnaln_kernel_time* out, int32_t cap, int32_t* n_out) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c || !n_out || cap < 0 || (cap > 0 && !out)) return DNALN_ERR_INVALID_ARG;
  int32_t i = 0;
  for (const auto& kv : c->ktimes) {
    if (i < cap) {
      dnaln_kernel_time& o = out[i];
      std::memset(&o, 0, sizeof o);
      std::snprintf(o.name, sizeof o.name, "%s", kv.first.c_str());
      o.launches = kv.second.launches;
      o.ms = kv.second.ms;
    }
    ++i;
  }
  *n_out = i;
  return DNALN_OK;
}

int dnaln_gpu_set_sub_batch(dnaln_ctx* c, int64_t reads) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c || reads < 0) return DNALN_ERR_INVALID_ARG;
  c->sub_batch = reads;
  return DNALN_OK;
}

int dnaln_gpu_set_option(dnaln_ctx* c, const char* name, int64_t value) {
  if (!c || !name) return DNALN_ERR_INVALID_ARG;
  const std::string k = name;
  if (k == "sub_batch") return dnaln_gpu_set_sub_batch(c, value);
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (k == "warp_seed_only") {
    c->warp_seed_only = value != 0;
    return DNALN_OK;
  }
  if (k == "graphs") {
    c->graphs = value != 0;
    return DNALN_OK;
  }
  if (k == "sw_form") {
    if (value < 0 || value > 3) return fail(c, DNALN_ERR_INVALID_ARG, "sw_form must be 0 (tuned), 1, 2 or 3");
    c->sw_mode = static_cast<int>(value);
    return DNALN_OK;
  }
  if (k == "long_thread") {
    c->long_thread = value != 0;
    return DNALN_OK;
  }
  if (k == "length_order") {
    c->length_order = value != 0;
    return DNALN_OK;
  }
  if (k == "seed_block") {
    if (value != 0 && value != 64 && value != 128)
      return fail(c, DNALN_ERR_INVALID_ARG, "seed_block must be 0 (tuned), 64 or 128");
    c->seed_block = static_cast<int>(value);
    return DNALN_OK;
  }
  if (k == "encode_bulk") {
    c->encode_bulk = value != 0;
    return DNALN_OK;
  }
  if (k == "work_stealing") {
    c->stealing = value != 0;
    return DNALN_OK;
  }
  if (k == "chain_pool") {  // entries of the chaining pool from now on (a floor and a start)
    if (value < 64) return fail(c, DNALN_ERR_INVALID_ARG, "chain_pool must be >= 64");
    c->pool_min = value;
    c->pool_cap = value;
    return DNALN_OK;
  }
  if (k == "fail_alloc_after") {
    c->fail_alloc_after = value < 0 ? -1 : value;
    return DNALN_OK;
  }
  if (k == "dir_cap_bytes") {
    if (value < (int64_t(1) << 20)) return fail(c, DNALN_ERR_INVALID_ARG, "dir_cap_bytes must be >= 1 MiB");
    c->dir_cap_bytes = static_cast<size_t>(value);
    return DNALN_OK;
  }
  return fail(c, DNALN_ERR_INVALID_ARG, "unknown option '%s'", name);
}

int dnaln_gpu_sw_tuning(const dnaln_ctx* cc, dnaln_sw_tuning* out, int32_t cap, int32_t* n_out) {
  if (!cc || !n_out) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(cc->mu);
  int32_t i = 0;
  for (const auto& kv : cc->sw_tune) {
    if (out && i < cap) out[i] = kv.second;
    ++i;
  }
  *n_out = i;
  return DNALN_OK;
}

int dnaln_gpu_seed_tuning(const dnaln_ctx* cc, dnaln_seed_tuning* out) {
  if (!cc || !out) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(cc->mu);
  *out = cc->seed_tune;
  return DNALN_OK;
}

int dnaln_gpu_host_alloc(dnaln_ctx* c, size_t bytes, void** out) {
  if (!c || !out) return DNALN_ERR_INVALID_ARG;
  if (int e = set_device(c)) return e;
  CK(cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault));
  return DNALN_OK;
}

int dnaln_gpu_host_free(dnaln_ctx* c, void* p) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  if (p) CK(cudaFreeHost(p));
  return DNALN_OK;
}

int dnaln_gpu_index_build(dnaln_ctx* c, const uint8_t* genome, uint64_t n_bases, const uint64_t* contig_off,
                          const uint32_t* contig_len, int32_t n_contigs, int32_t k, int32_t w, int32_t* index_id) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c || !genome || !contig_off || !contig_len || !index_id || n_contigs < 1)
    return fail(c, DNALN_ERR_INVALID_ARG, "null argument or no contigs");
  if (k < 4 || k > 28) return fail(c, DNALN_ERR_INVALID_ARG, "k must be in [4, 28] (got %d)", k);
  if (w < 1 || w > 255) return fail(c, DNALN_ERR_INVALID_ARG, "w must be in [1, 255] (got %d)", w);
  if (n_bases >= (1ULL << 31)) return fail(c, DNALN_ERR_INVALID_ARG, "reference is too large (limit: 2^31 bp)");
  for (int32_t i = 0; i < n_contigs; ++i)
    if (contig_off[i] + contig_len[i] > n_bases || (i > 0 && contig_off[i] < contig_off[i - 1]))
      return fail(c, DNALN_ERR_INVALID_ARG, "contig %d is outside the genome or out of order", i);
  if (int e = set_device(c)) return e;
  // the genome and contig table go up first; the index is then built where it will live
  IndexRes r;
  r.mem = std::make_shared<IndexMem>();
  r.device = c->device;
  IndexMem& m = *r.mem;
  int e = DNALN_OK;
  if ((e = dalloc(c, m.genome, n_bases)) || (e = dalloc(c, m.coff, n_contigs * sizeof(uint64_t))) ||
      (e = dalloc(c, m.clen, n_contigs * sizeof(uint32_t))))
    return e;
  cudaError_t x = cudaSuccess;
  auto up = [&](DevBuf& b, const void* src, size_t bytes) {  // ordered before the build on c->st
    if (x == cudaSuccess && bytes) x = cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, c->st);
  };
  up(m.genome, genome, n_bases);
  up(m.coff, contig_off, n_contigs * sizeof(uint64_t));
  up(m.clen, contig_len, n_contigs * sizeof(uint32_t));
  if (x != cudaSuccess) return fail(c, DNALN_ERR_CUDA, "index upload: %s", cudaGetErrorString(x));
  DeviceIndexBuild b;
  char why[256] = {};
  e = build_index_on_device(c->st, static_cast<const uint8_t*>(m.genome.p), n_bases, contig_off, contig_len, n_contigs,
                            k, w, &b, why, sizeof why);
  // the built arrays belong to the index from here on (freed with it on every path)
  m.table = DevBuf{b.table, b.n_buckets * sizeof(ulonglong2)};
  m.positions = DevBuf{b.positions, b.n_pos * sizeof(uint32_t)};
  m.nruns = DevBuf{b.n_runs, static_cast<size_t>(b.n_n_runs) * sizeof(uint2)};
  if (e != DNALN_OK) {
    cudaStreamSynchronize(c->st);
    return fail(c, e, "%s", why);
  }
  r.n_keys = b.n_keys;
  r.n_pos = b.n_pos;
  r.n_buckets = b.n_buckets;
  r.n_bases = n_bases;
  r.max_count = b.max_count;
  r.n_contigs = n_contigs;
  r.k = k;
  r.w = w;
  register_index(c, r, b.mask, b.n_n_runs, index_id);
  return DNALN_OK;
}

int dnaln_gpu_index_stats(const dnaln_ctx* cc, int32_t id, uint64_t out6[6]) {
  if (!cc) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(cc->mu);
  auto* c = const_cast<dnaln_ctx*>(cc);
  if (!c || !out6) return DNALN_ERR_INVALID_ARG;
  IndexRes* r = find_index(c, id);
  if (!r) return DNALN_ERR_NOT_FOUND;
  out6[0] = r->n_keys;
  out6[1] = r->n_pos;
  out6[2] = r->max_count;
  out6[3] = r->n_buckets * 16 + r->n_pos * 4;  // src/index.hpp:46
  out6[4] = r->n_buckets;
  out6[5] = r->mem->bytes();
  return DNALN_OK;
}

int dnaln_gpu_index_export(dnaln_ctx* c, int32_t id, uint64_t* keys, uint32_t* offsets, uint32_t* counts,
                           uint32_t* positions) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c) return DNALN_ERR_INVALID_ARG;
  if (int e = set_device(c)) return e;
  IndexRes* r = find_index(c, id);
  if (!r) return DNALN_ERR_NOT_FOUND;
  std::vector<ulonglong2> t(r->n_buckets);
  CK(cudaMemcpy(t.data(), r->mem->table.p, t.size() * sizeof(ulonglong2), cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < t.size(); ++i) {
    if (keys) keys[i] = t[i].x;
    if (offsets) offsets[i] = static_cast<uint32_t>(t[i].y);
    if (counts) counts[i] = static_cast<uint32_t>(t[i].y >> 32);
  }
  if (positions && r->n_pos)
    CK(cudaMemcpy(positions, r->mem->positions.p, r->n_pos * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  return DNALN_OK;
}

int dnaln_gpu_index_free(dnaln_ctx* c, int32_t id) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c) return DNALN_ERR_INVALID_ARG;
  if (int e = set_device(c)) return e;
  IndexRes* r = find_index(c, id);
  if (!r) return DNALN_ERR_NOT_FOUND;
  cudaStreamSynchronize(c->st);
  free_index(*r);
  c->idx.erase(id);
  return DNALN_OK;
}

// ---- index image files ---------------------------------------------------------------
namespace {

constexpr char kImageMagic[8] = {'D', 'N', 'B', 'I', 'D', 'X', '0', '1'};
constexpr uint32_t kImageVersion = 1;
constexpr size_t kImageChunk = 64ull << 20;  // staging chunk (a multiple of 32 bytes)

struct ImageHeader {
  char magic[8];
  uint32_t version, header_bytes;
  int32_t k, w, n_contigs, n_n_runs;
  uint32_t max_count, reserved;
  uint64_t n_bases, n_keys, n_pos, n_buckets, mask;
  uint64_t checksum;  // ImageHash of every section, in file order
};

// 64-bit checksum of a byte stream given in chunks whose sizes are multiples of 32 except
// the last of each section: four independent multiply-rotate lanes over 8-byte words.
struct ImageHash {
  uint64_t h[4] = {0x243F6A8885A308D3ull, 0x13198A2E03707344ull, 0xA4093822299F31D0ull, 0x082EFA98EC4E6C89ull};
  static uint64_t mix(uint64_t h, uint64_t w) {
    h ^= w * 0x9E3779B97F4A7C15ull;
    return ((h << 27) | (h >> 37)) * 0xBF58476D1CE4E5B9ull;
  }
  void add(const void* data, size_t len) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    size_t i = 0;
    for (; i + 32 <= len; i += 32) {
      uint64_t w[4];
      std::memcpy(w, p + i, 32);
      for (int l = 0; l < 4; ++l) h[l] = mix(h[l], w[l]);
    }
    for (; i + 8 <= len; i += 8) {
      uint64_t w;
      std::memcpy(&w, p + i, 8);
      h[0] = mix(h[0], w);
    }
    if (i < len) {
      uint64_t w = 0;
      std::memcpy(&w, p + i, len - i);
      h[1] = mix(h[1], w ^ static_cast<uint64_t>(len - i) << 56);
    }
  }
  uint64_t done() const { return mix(mix(h[0], h[1]), mix(h[2], h[3])); }
};

struct FileCloser {
  FILE* f = nullptr;
  ~FileCloser() {
    if (f) std::fclose(f);
  }
};

struct PinnedChunks {  // two page-locked staging chunks
  void* p[2] = {nullptr, nullptr};
  ~PinnedChunks() {
    for (void* x : p)
      if (x) cudaFreeHost(x);
  }
};

}  // namespace

int dnaln_gpu_index_save(dnaln_ctx* c, int32_t id, const char* path) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!path) return fail(c, DNALN_ERR_INVALID_ARG, "null path");
  if (int e = set_device(c)) return e;
  IndexRes* r = find_index(c, id);
  if (!r) return DNALN_ERR_NOT_FOUND;
  const IndexMem& m = *r->mem;
  ImageHeader h{};
  std::memcpy(h.magic, kImageMagic, sizeof h.magic);
  h.version = kImageVersion;
  h.header_bytes = sizeof(ImageHeader);
  h.k = r->k;
  h.w = r->w;
  h.n_contigs = r->n_contigs;
  h.n_n_runs = r->dev.n_n_runs;
  h.max_count = r->max_count;
  h.n_bases = r->n_bases;
  h.n_keys = r->n_keys;
  h.n_pos = r->n_pos;
  h.n_buckets = r->n_buckets;
  h.mask = r->dev.mask;
  const struct {
    const void* d;
    size_t bytes;
  } sec[] = {{m.coff.p, static_cast<size_t>(h.n_contigs) * sizeof(uint64_t)},
             {m.clen.p, static_cast<size_t>(h.n_contigs) * sizeof(uint32_t)},
             {m.genome.p, h.n_bases},
             {m.table.p, h.n_buckets * sizeof(ulonglong2)},
             {m.positions.p, h.n_pos * sizeof(uint32_t)},
             {m.nruns.p, static_cast<size_t>(h.n_n_runs) * sizeof(uint2)}};
  CK(cudaStreamSynchronize(c->st));  // nothing queued may still write the index
  PinnedChunks pc;
  CK(cudaMallocHost(&pc.p[0], kImageChunk));
  const std::string tmp = std::string(path) + ".tmp";
  FileCloser fc;
  fc.f = std::fopen(tmp.c_str(), "wb");
  if (!fc.f) return fail(c, DNALN_ERR_IO, "cannot open %s for writing", tmp.c_str());
  bool ok = std::fwrite(&h, sizeof h, 1, fc.f) == 1;  // the checksum is filled in at the end
  ImageHash hs;
  for (const auto& x : sec) {
    for (size_t at = 0; ok && at < x.bytes; at += kImageChunk) {
      const size_t n = std::min(kImageChunk, x.bytes - at);
      CK(cudaMemcpy(pc.p[0], static_cast<const char*>(x.d) + at, n, cudaMemcpyDeviceToHost));
      hs.add(pc.p[0], n);
      ok = std::fwrite(pc.p[0], 1, n, fc.f) == n;
    }
  }
  h.checksum = hs.done();
  ok = ok && std::fseek(fc.f, 0, SEEK_SET) == 0 && std::fwrite(&h, sizeof h, 1, fc.f) == 1;
  ok = ok && std::fflush(fc.f) == 0;
  const bool closed = std::fclose(fc.f) == 0;
  fc.f = nullptr;
  if (!ok || !closed || std::rename(tmp.c_str(), path) != 0) {
    std::remove(tmp.c_str());
    return fail(c, DNALN_ERR_IO, "writing the index image %s failed", path);
  }
  return DNALN_OK;
}

int dnaln_gpu_index_load(dnaln_ctx* c, const char* path, int32_t* index_id) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!path || !index_id) return fail(c, DNALN_ERR_INVALID_ARG, "null argument");
  if (int e = set_device(c)) return e;
  FileCloser fc;
  fc.f = std::fopen(path, "rb");
  if (!fc.f) return fail(c, DNALN_ERR_IO, "cannot open %s", path);
  ImageHeader h{};
  if (std::fread(&h, sizeof h, 1, fc.f) != 1 || std::memcmp(h.magic, kImageMagic, sizeof h.magic) != 0 ||
      h.version != kImageVersion || h.header_bytes != sizeof(ImageHeader))
    return fail(c, DNALN_ERR_IO, "%s is not an index image of this version", path);
  const bool pow2 = h.n_buckets >= 1 && (h.n_buckets & (h.n_buckets - 1)) == 0;
  if (h.k < 4 || h.k > 28 || h.w < 1 || h.w > 255 || h.n_contigs < 1 || h.n_bases >= (1ULL << 31) || !pow2 ||
      h.mask != h.n_buckets - 1 || h.n_keys >= h.n_buckets || h.n_pos >= (1ULL << 32) || h.n_n_runs < 0 ||
      static_cast<uint64_t>(h.n_n_runs) > h.n_bases || h.n_buckets > (1ULL << 34))
    return fail(c, DNALN_ERR_IO, "%s: header out of range", path);
  IndexRes r;
  r.mem = std::make_shared<IndexMem>();
  r.device = c->device;
  IndexMem& m = *r.mem;
  int e = DNALN_OK;
  if ((e = dalloc(c, m.coff, h.n_contigs * sizeof(uint64_t))) || (e = dalloc(c, m.clen, h.n_contigs * sizeof(uint32_t))) ||
      (e = dalloc(c, m.genome, h.n_bases)) || (e = dalloc(c, m.table, h.n_buckets * sizeof(ulonglong2))) ||
      (e = dalloc(c, m.positions, h.n_pos * sizeof(uint32_t))) ||
      (e = dalloc(c, m.nruns, static_cast<size_t>(h.n_n_runs) * sizeof(uint2))))
    return e;
  std::vector<uint64_t> coff(static_cast<size_t>(h.n_contigs));
  std::vector<uint32_t> clen(static_cast<size_t>(h.n_contigs));
  const struct {
    void* d;
    size_t bytes;
    int kind;  // 0 contig offsets, 1 contig lengths, 2 genome, 3 buckets, 4 positions, 5 N runs
  } sec[] = {{m.coff.p, coff.size() * sizeof(uint64_t), 0},
             {m.clen.p, clen.size() * sizeof(uint32_t), 1},
             {m.genome.p, h.n_bases, 2},
             {m.table.p, h.n_buckets * sizeof(ulonglong2), 3},
             {m.positions.p, h.n_pos * sizeof(uint32_t), 4},
             {m.nruns.p, static_cast<size_t>(h.n_n_runs) * sizeof(uint2), 5}};
  PinnedChunks pc;
  CK(cudaMallocHost(&pc.p[0], kImageChunk));
  CK(cudaMallocHost(&pc.p[1], kImageChunk));
  cudaEvent_t done[2] = {nullptr, nullptr};
  CK(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
  if (cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming) != cudaSuccess) {
    cudaEventDestroy(done[0]);
    return fail(c, DNALN_ERR_CUDA, "event creation failed");
  }
  ImageHash hs;
  TableCheck tc;
  tc.n_pos = h.n_pos;
  tc.n_bases = h.n_bases;
  bool ok = true;
  uint32_t prev_end = 0;
  int slot = 0;
  cudaError_t x = cudaSuccess;
  // chunk j is read into staging slot j % 2 while chunk j-1's copy to the device runs
  for (const auto& s : sec) {
    for (size_t at = 0; ok && x == cudaSuccess && at < s.bytes; at += kImageChunk) {
      const size_t n = std::min(kImageChunk, s.bytes - at);
      x = cudaEventSynchronize(done[slot]);  // the copy that last used this slot is done
      if (x != cudaSuccess) break;
      void* buf = pc.p[slot];
      if (std::fread(buf, 1, n, fc.f) != n) {
        ok = false;
        break;
      }
      hs.add(buf, n);
      switch (s.kind) {
        case 0: std::memcpy(coff.data(), buf, n); break;
        case 1: std::memcpy(clen.data(), buf, n); break;
        case 3: tc.buckets(static_cast<const ulonglong2*>(buf), n / sizeof(ulonglong2)); break;
        case 4: tc.positions(static_cast<const uint32_t*>(buf), n / sizeof(uint32_t)); break;
        case 5: {
          const uint2* v = static_cast<const uint2*>(buf);
          for (size_t i = 0; i < n / sizeof(uint2); ++i) {
            ok = ok && v[i].x < v[i].y && v[i].y <= h.n_bases && v[i].x >= prev_end;
            prev_end = v[i].y;
          }
          break;
        }
        default: break;
      }
      x = cudaMemcpyAsync(static_cast<char*>(s.d) + at, buf, n, cudaMemcpyHostToDevice, c->st);
      if (x == cudaSuccess) x = cudaEventRecord(done[slot], c->st);
      slot ^= 1;
    }
  }
  if (x == cudaSuccess) x = cudaStreamSynchronize(c->st);
  cudaEventDestroy(done[0]);
  cudaEventDestroy(done[1]);
  if (x != cudaSuccess) return fail(c, DNALN_ERR_CUDA, "index image upload: %s", cudaGetErrorString(x));
  const bool at_end = ok && std::fgetc(fc.f) == EOF;
  if (!at_end || hs.done() != h.checksum)
    return fail(c, DNALN_ERR_IO, "%s: truncated, longer than its header says, or its checksum does not match", path);
  if (!tc.ok || tc.n_keys != h.n_keys || tc.max_count != h.max_count)
    return fail(c, DNALN_ERR_IO, "%s: the bucket table or positions are inconsistent with the header", path);
  if (check_contigs(c, coff.data(), clen.data(), h.n_contigs, h.n_bases, DNALN_ERR_IO)) return DNALN_ERR_IO;
  r.n_keys = h.n_keys;
  r.n_pos = h.n_pos;
  r.n_buckets = h.n_buckets;
  r.n_bases = h.n_bases;
  r.max_count = h.max_count;
  r.n_contigs = h.n_contigs;
  r.k = h.k;
  r.w = h.w;
  register_index(c, r, h.mask, h.n_n_runs, index_id);
  return DNALN_OK;
}

int dnaln_gpu_index_upload(dnaln_ctx* c, const uint8_t* genome, uint64_t n_bases, const uint64_t* contig_off,
                           const uint32_t* contig_len, int32_t n_contigs, int32_t k, int32_t w, const uint64_t* keys,
                           const uint32_t* offsets, const uint32_t* counts, uint64_t n_buckets,
                           const uint32_t* positions, uint64_t n_pos, int32_t* index_id) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!genome || !contig_off || !contig_len || !keys || !offsets || !counts || (n_pos && !positions) || !index_id ||
      n_contigs < 1)
    return fail(c, DNALN_ERR_INVALID_ARG, "null argument or no contigs");
  if (k < 4 || k > 28) return fail(c, DNALN_ERR_INVALID_ARG, "k must be in [4, 28] (got %d)", k);
  if (w < 1 || w > 255) return fail(c, DNALN_ERR_INVALID_ARG, "w must be in [1, 255] (got %d)", w);
  if (n_bases >= (1ULL << 31)) return fail(c, DNALN_ERR_INVALID_ARG, "reference is too large (limit: 2^31 bp)");
  if (n_buckets < 1 || (n_buckets & (n_buckets - 1)) != 0 || n_buckets > (1ULL << 34))
    return fail(c, DNALN_ERR_INVALID_ARG, "n_buckets must be a power of two (got %llu)",
                static_cast<unsigned long long>(n_buckets));
  if (n_pos >= (1ULL << 32)) return fail(c, DNALN_ERR_INVALID_ARG, "too many positions");
  if (int e = check_contigs(c, contig_off, contig_len, n_contigs, n_bases, DNALN_ERR_INVALID_ARG)) return e;
  if (int e = set_device(c)) return e;
  // the table in the device layout, checked as it is packed
  std::vector<ulonglong2> t(static_cast<size_t>(n_buckets));
  for (size_t i = 0; i < t.size(); ++i)
    t[i] = make_ulonglong2(keys[i], keys[i] == kInvalidHash
                                        ? 0ull
                                        : (static_cast<uint64_t>(offsets[i]) | static_cast<uint64_t>(counts[i]) << 32));
  TableCheck tc;
  tc.n_pos = n_pos;
  tc.n_bases = n_bases;
  tc.buckets(t.data(), t.size());
  tc.positions(positions, static_cast<size_t>(n_pos));
  if (!tc.ok) return fail(c, DNALN_ERR_INVALID_ARG, "a bucket or position lies outside the positions or the genome");
  if (tc.n_keys >= n_buckets) return fail(c, DNALN_ERR_INVALID_ARG, "the table has no empty bucket");
  IndexRes r;
  r.mem = std::make_shared<IndexMem>();
  r.device = c->device;
  IndexMem& m = *r.mem;
  int e = DNALN_OK;
  if ((e = dalloc(c, m.genome, n_bases)) || (e = dalloc(c, m.coff, n_contigs * sizeof(uint64_t))) ||
      (e = dalloc(c, m.clen, n_contigs * sizeof(uint32_t))) || (e = dalloc(c, m.table, t.size() * sizeof(ulonglong2))) ||
      (e = dalloc(c, m.positions, n_pos * sizeof(uint32_t))))
    return e;
  CK(cudaMemcpy(m.genome.p, genome, n_bases, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(m.coff.p, contig_off, n_contigs * sizeof(uint64_t), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(m.clen.p, contig_len, n_contigs * sizeof(uint32_t), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(m.table.p, t.data(), t.size() * sizeof(ulonglong2), cudaMemcpyHostToDevice));
  if (n_pos) CK(cudaMemcpy(m.positions.p, positions, n_pos * sizeof(uint32_t), cudaMemcpyHostToDevice));
  uint2* runs = nullptr;
  int32_t n_runs = 0;
  char why[256] = {};
  e = find_n_runs_on_device(c->st, static_cast<const uint8_t*>(m.genome.p), n_bases, &runs, &n_runs, why, sizeof why);
  m.nruns = DevBuf{runs, static_cast<size_t>(n_runs) * sizeof(uint2)};
  if (e != DNALN_OK) return fail(c, e, "%s", why);
  r.n_keys = tc.n_keys;
  r.n_pos = n_pos;
  r.n_buckets = n_buckets;
  r.n_bases = n_bases;
  r.max_count = tc.max_count;
  r.n_contigs = n_contigs;
  r.k = k;
  r.w = w;
  register_index(c, r, n_buckets - 1, n_runs, index_id);
  return DNALN_OK;
}

int dnaln_gpu_index_attach(dnaln_ctx* dst, dnaln_ctx* src, int32_t src_id, int32_t* dst_id) {
  if (!dst || !src || !dst_id) return dst ? fail(dst, DNALN_ERR_INVALID_ARG, "null argument") : DNALN_ERR_INVALID_ARG;
  if (dst == src) return fail(dst, DNALN_ERR_INVALID_ARG, "a context cannot attach its own index");
  // both locks, in address order, so that two attaches in opposite directions cannot deadlock
  std::unique_lock<std::mutex> l1(dst < src ? dst->mu : src->mu, std::defer_lock);
  std::unique_lock<std::mutex> l2(dst < src ? src->mu : dst->mu, std::defer_lock);
  std::lock(l1, l2);
  if (src->device != dst->device)
    return fail(dst, DNALN_ERR_INVALID_ARG, "index %d lives on device %d, this context on device %d", src_id,
                src->device, dst->device);
  auto it = src->idx.find(src_id);
  if (it == src->idx.end()) return fail(dst, DNALN_ERR_NOT_FOUND, "unknown index id %d", src_id);
  const int32_t id = dst->next_id++;
  dst->idx[id] = it->second;  // shares the device memory (shared pointer), copies the descriptors
  *dst_id = id;
  return DNALN_OK;
}

int dnaln_gpu_sketch(dnaln_ctx* c, const uint8_t* codes, const int64_t* seq_off, const int32_t* seq_len,
                     const uint32_t* pos_offset, int64_t n, int32_t k, int32_t w, uint64_t* out_hash,
                     uint32_t* out_pos, uint32_t* out_strand, int32_t* out_count) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c || n < 0 || (n > 0 && (!codes || !seq_off || !seq_len || !out_hash || !out_pos || !out_strand || !out_count)))
    return fail(c, DNALN_ERR_INVALID_ARG, "null argument");
  if (k < 1 || k > 31) return fail(c, DNALN_ERR_INVALID_ARG, "k must be in [1, 31] (got %d)", k);
  if (w < 1 || w > 255) return fail(c, DNALN_ERR_INVALID_ARG, "w must be in [1, 255] (got %d)", w);
  if (n == 0) return DNALN_OK;
  if (int e = set_device(c)) return e;
  int64_t ext = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (seq_len[i] < 0 || seq_off[i] < 0) return fail(c, DNALN_ERR_INVALID_ARG, "negative offset or length");
    ext = std::max<int64_t>(ext, seq_off[i] + seq_len[i]);
  }
  cudaStream_t st = c->st;
  DBUF(d_codes, uint8_t, "sk_codes", ext);
  DBUF(d_off, int64_t, "sk_off", n);
  DBUF(d_len, int32_t, "sk_len", n);
  DBUF(d_po, uint32_t, "sk_po", n);
  DBUF(d_h, uint64_t, "sk_h", ext);
  DBUF(d_p, uint32_t, "sk_p", ext);
  DBUF(d_s, uint32_t, "sk_s", ext);
  DBUF(d_cnt, int32_t, "sk_cnt", n);
  CK(cudaMemcpyAsync(d_codes, codes, ext, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_off, seq_off, n * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_len, seq_len, n * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  if (pos_offset) CK(cudaMemcpyAsync(d_po, pos_offset, n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  launch_sketch_codes(st, d_codes, d_off, d_len, pos_offset ? d_po : nullptr, n, k, w, d_h, d_p, d_s, d_cnt);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out_hash, d_h, ext * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(out_pos, d_p, ext * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(out_strand, d_s, ext * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(out_count, d_cnt, n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return DNALN_OK;
}

int dnaln_gpu_lookup(dnaln_ctx* c, int32_t id, const uint64_t* hashes, int64_t n, uint32_t* out_offset,
                     uint32_t* out_count) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c || n < 0 || (n > 0 && (!hashes || !out_offset || !out_count)))
    return fail(c, DNALN_ERR_INVALID_ARG, "null argument");
  if (int e = set_device(c)) return e;
  IndexRes* r = find_index(c, id);
  if (!r) return DNALN_ERR_NOT_FOUND;
  if (n == 0) return DNALN_OK;
  cudaStream_t st = c->st;
  DBUF(d_h, uint64_t, "lk_h", n);
  DBUF(d_o, uint32_t, "lk_o", n);
  DBUF(d_c, uint32_t, "lk_c", n);
  CK(cudaMemsetAsync(c->d_err, 0, sizeof(uint32_t), st));
  CK(cudaMemcpyAsync(d_h, hashes, n * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  launch_lookup(st, r->dev, d_h, n, d_o, d_c, c->d_err);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out_offset, d_o, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(out_count, d_c, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  uint32_t bits = 0;
  CK(cudaMemcpyAsync(&bits, c->d_err, sizeof bits, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return check_device_errors(c, bits);
}

int dnaln_gpu_chain(dnaln_ctx* c, uint32_t* rpos, int32_t* qpos, uint32_t* strand, const int64_t* set_off,
                    int64_t n_sets, int32_t k, const dnaln_chain_params* p, int32_t* out_score, uint32_t* out_strand,
                    int32_t* out_n, int64_t* out_dmin, int64_t* out_dmax, uint32_t* out_rpos, int32_t* out_count) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c || !p || !set_off || n_sets < 0 || !out_count) return fail(c, DNALN_ERR_INVALID_ARG, "null argument");
  if (p->lookback < 0 || p->band < 0 || p->band > (1 << 20))
    return fail(c, DNALN_ERR_INVALID_ARG, "chain lookback must be >= 0 and band in [0, 2^20]");
  if (n_sets == 0) return DNALN_OK;
  if (int e = set_device(c)) return e;
  const int64_t total = set_off[n_sets] - set_off[0];
  if (set_off[0] != 0 || total < 0) return fail(c, DNALN_ERR_INVALID_ARG, "set_off must start at 0 and increase");
  std::vector<uint64_t> keys(static_cast<size_t>(total));
  for (int64_t i = 0; i < total; ++i) {
    if (strand[i] > 1 || rpos[i] >= (1u << 31) || qpos[i] < -(1 << 30) || qpos[i] >= (1 << 30))
      return fail(c, DNALN_ERR_INVALID_ARG, "anchor %lld out of range (strand 0/1, rpos < 2^31, |qpos| < 2^30)",
                  static_cast<long long>(i));
    keys[static_cast<size_t>(i)] = anchor_key(strand[i], rpos[i], qpos[i]);
  }
  cudaStream_t st = c->st;
  AnchorScratch as;
  as.keys = dbuf<uint64_t>(c, "a_keys", total);
  as.f = dbuf<int32_t>(c, "a_f", total);
  as.prev = dbuf<int32_t>(c, "a_prev", total);
  as.ord = dbuf<uint64_t>(c, "a_ord", total);
  as.used = dbuf<uint8_t>(c, "a_used", total);
  as.ch_score = dbuf<int32_t>(c, "c_score", total);
  as.ch_sn = dbuf<uint32_t>(c, "c_sn", total);
  as.ch_dmin = dbuf<int64_t>(c, "c_dmin", total);
  as.ch_dmax = dbuf<int64_t>(c, "c_dmax", total);
  as.ch_rpos = dbuf<uint32_t>(c, "c_rpos", total);
  if (!as.keys || !as.f || !as.prev || !as.ord || !as.used || !as.ch_score || !as.ch_sn || !as.ch_dmin ||
      !as.ch_dmax || !as.ch_rpos)
    return DNALN_ERR_OOM;
  DBUF(d_set, int64_t, "ch_set", n_sets + 1);
  DBUF(d_cnt, int32_t, "ch_cnt", n_sets);
  const int32_t* d_lut = nullptr;
  if (int e = chain_lut_dev(c, k, p->band, &d_lut)) return e;
  CK(cudaMemsetAsync(c->d_err, 0, sizeof(uint32_t), st));
  CK(cudaMemcpyAsync(as.keys, keys.data(), total * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_set, set_off, (n_sets + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  ChainParamsDev cp{p->max_gap, p->band, p->lookback, p->min_score, p->min_anchors, k, d_lut};
  launch_chain_sets(st, d_set, n_sets, cp, as, d_cnt, c->d_err);
  CK(cudaGetLastError());
  std::vector<uint64_t> ord(static_cast<size_t>(total));
  std::vector<int32_t> score(static_cast<size_t>(total));
  std::vector<uint32_t> sn(static_cast<size_t>(total)), crp(static_cast<size_t>(total));
  std::vector<int64_t> dmin(static_cast<size_t>(total)), dmax(static_cast<size_t>(total));
  CK(cudaMemcpyAsync(keys.data(), as.keys, total * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(ord.data(), as.ord, total * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(score.data(), as.ch_score, total * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(sn.data(), as.ch_sn, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(crp.data(), as.ch_rpos, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(dmin.data(), as.ch_dmin, total * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(dmax.data(), as.ch_dmax, total * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(out_count, d_cnt, n_sets * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  uint32_t bits = 0;
  CK(cudaMemcpyAsync(&bits, c->d_err, sizeof bits, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (int e = check_device_errors(c, bits)) return e;
  for (int64_t i = 0; i < total; ++i) {
    rpos[i] = key_rpos(keys[static_cast<size_t>(i)]);
    qpos[i] = key_qpos(keys[static_cast<size_t>(i)]);
    strand[i] = key_strand(keys[static_cast<size_t>(i)]);
  }
  for (int64_t s = 0; s < n_sets; ++s) {
    const int64_t a0 = set_off[s];
    for (int32_t j = 0; j < out_count[s]; ++j) {
      const size_t src = static_cast<size_t>(a0 + static_cast<int64_t>(ord[static_cast<size_t>(a0 + j)] & 0xffffffffu));
      const size_t dst = static_cast<size_t>(a0 + j);
      out_score[dst] = score[src];
      out_strand[dst] = sn[src] & 1u;
      out_n[dst] = static_cast<int32_t>(sn[src] >> 1);
      out_dmin[dst] = dmin[src];
      out_dmax[dst] = dmax[src];
      out_rpos[dst] = crp[src];
    }
  }
  return DNALN_OK;
}

int dnaln_gpu_align(dnaln_ctx* c, const uint8_t* q, const int64_t* q_off, const int32_t* q_len, const uint8_t* t,
                    const int64_t* t_off, const int32_t* t_len, int64_t n, int32_t traceback,
                    const dnaln_score_params* sp, dnaln_align_result* out, uint32_t* cigar, int64_t cigar_cap,
                    int64_t* cigar_used) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c || !sp || n < 0 || (n > 0 && (!q || !q_off || !q_len || !t || !t_off || !t_len || !out)))
    return fail(c, DNALN_ERR_INVALID_ARG, "null argument");
  if (sp->bw < 0 || sp->bw > 1000 || sp->gap_ext < 0 || sp->gap_open < 0 || sp->mismatch < 0 || sp->ambig < 0)
    return fail(c, DNALN_ERR_INVALID_ARG, "invalid score parameters");
  if (cigar_used) *cigar_used = 0;
  if (n == 0) return DNALN_OK;
  if (n > (int64_t(1) << 31) - 64) return fail(c, DNALN_ERR_INVALID_ARG, "too many tasks in one call");
  if (int e = set_device(c)) return e;
  const int W = 2 * sp->bw + 1;
  int64_t qext = 0, text = 0, cig_total = 0;
  int rows_max = 0;
  std::vector<SwTask> tasks(static_cast<size_t>(n));
  std::vector<int64_t> slot_off(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) {
    if (q_len[i] < 0 || t_len[i] < 0 || q_off[i] < 0 || t_off[i] < 0)
      return fail(c, DNALN_ERR_INVALID_ARG, "negative offset or length in task %lld", static_cast<long long>(i));
    qext = std::max<int64_t>(qext, q_off[i] + q_len[i]);
    const int64_t tmax = static_cast<int64_t>(q_len[i]) + W - 1;
    const int64_t tl = t_len[i] < tmax ? t_len[i] : tmax;
    text = std::max<int64_t>(text, t_off[i] + tl);
    SwTask& tk = tasks[static_cast<size_t>(i)];
    tk.q_off = q_off[i];
    tk.qlen = q_len[i];
    tk.t_start = t_off[i];
    tk.t_lo = t_off[i];
    tk.t_hi = t_off[i] + tl;
    tk.slot = static_cast<int32_t>(i);
    slot_off[static_cast<size_t>(i)] = cig_total;
    cig_total += 2 * static_cast<int64_t>(q_len[i]) + 1;
    rows_max = std::max(rows_max, q_len[i]);
  }
  cudaStream_t st = c->st;
  const bool tb = traceback != 0;
  DBUF(d_q, uint8_t, "al_q", qext);
  DBUF(d_t, uint8_t, "al_t", text);
  DBUF(d_tasks, SwTask, "al_tasks", n);
  DBUF(d_res, SwResult, "al_res", n);
  CK(cudaMemsetAsync(c->d_err, 0, sizeof(uint32_t), st));
  if (qext) CK(cudaMemcpyAsync(d_q, q, qext, cudaMemcpyHostToDevice, st));
  if (text) CK(cudaMemcpyAsync(d_t, t, text, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_tasks, tasks.data(), n * sizeof(SwTask), cudaMemcpyHostToDevice, st));
  const SwParams swp = make_sw_params(*sp);
  uint32_t* d_cig = nullptr;
  int64_t* d_slot = nullptr;
  if (tb) {
    d_cig = dbuf<uint32_t>(c, "al_cig", cig_total);
    d_slot = dbuf<int64_t>(c, "al_slot", n);
    if (!d_cig || !d_slot) return DNALN_ERR_OOM;
    CK(cudaMemcpyAsync(d_slot, slot_off.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  }
  c->trace_n = 0;
  c->trace_open = false;
  CK(cudaEventRecord(c->ev[tb ? kEvTb0 : kEvSc0], st));
  if (int e = launch_sw_chunked(c, tb, sw_bytes_ok(*sp), d_tasks, static_cast<int>(n), nullptr, d_q, d_t, swp, d_res,
                                rows_max, d_cig, d_slot))
    return e;
  CK(cudaEventRecord(c->ev[tb ? kEvTb1 : kEvSc1], st));
  int64_t total = 0;
  if (!tb) {
    std::vector<SwResult> res(static_cast<size_t>(n));
    CK(cudaMemcpyAsync(res.data(), d_res, n * sizeof(SwResult), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int64_t i = 0; i < n; ++i) {
      dnaln_align_result& o = out[i];
      std::memset(&o, 0, sizeof o);
      o.score = res[static_cast<size_t>(i)].score;
    }
  } else {
    DBUF(d_cnt, int64_t, "al_cnt", n + 1);
    DBUF(d_doff, int64_t, "al_doff", n + 1);
    DBUF(d_out, dnaln_align_result, "al_out", n);
    launch_align_counts(st, n, d_res, d_cnt);
    if (int e = exclusive_scan(c, d_cnt, d_doff, n + 1)) return e;
    CK(cudaMemcpyAsync(c->h_info, d_doff + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    total = c->h_info[0];
    DBUF(d_final, uint32_t, "al_final", total);
    launch_align_gather(st, n, d_res, d_cig, d_slot, d_doff, d_out, d_final);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, d_out, n * sizeof(dnaln_align_result), cudaMemcpyDeviceToHost, st));
    if (cigar && total <= cigar_cap && total > 0)
      CK(cudaMemcpyAsync(cigar, d_final, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }
  trace_collect(c);
  uint32_t bits = 0;
  CK(cudaMemcpy(&bits, c->d_err, sizeof bits, cudaMemcpyDeviceToHost));
  if (int e = check_device_errors(c, bits)) return e;
  if (cigar_used) *cigar_used = total;
  c->stats.cells += 0;
  for (int64_t i = 0; i < n; ++i) c->stats.cells += static_cast<uint64_t>(q_len[i]) * W;
  if (tb) {
    c->stats.sw_tasks_tb += static_cast<uint64_t>(n);
    c->stats.ms_sw_tb += ev_ms(c, kEvTb0, kEvTb1);
  } else {
    c->stats.sw_tasks_score += static_cast<uint64_t>(n);
    c->stats.ms_sw_score += ev_ms(c, kEvSc0, kEvSc1);
  }
  if (tb && total > cigar_cap)
    return fail(c, DNALN_ERR_CAPACITY, "CIGAR buffer holds %lld ops, tasks need %lld",
                static_cast<long long>(cigar_cap), static_cast<long long>(total));
  return DNALN_OK;
}

int dnaln_gpu_map_batch_device(dnaln_ctx* c, int32_t id, const char* d_seq, const int64_t* d_seq_off,
                               const int32_t* d_seq_len, const uint32_t* d_name_hash, int64_t n,
                               const dnaln_map_params* p, dnaln_map_record* d_out, uint32_t* d_cigar,
                               int64_t cigar_cap, int64_t* cigar_used) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> ctx_lock(c->mu);
  if (!c || n < 0 || !cigar_used || (n > 0 && (!d_seq || !d_seq_off || !d_seq_len || !d_name_hash || !d_out)))
    return fail(c, DNALN_ERR_INVALID_ARG, "null argument");
  if (int e = set_device(c)) return e;
  IndexRes* r = find_index(c, id);
  if (!r) return DNALN_ERR_NOT_FOUND;
  if (int e = validate_map_params(c, p, *r)) return e;
  if (!d_cigar) return fail(c, DNALN_ERR_INVALID_ARG, "null CIGAR buffer");
  const int e = run_map(c, *r, d_seq, d_seq_off, d_seq_len, d_name_hash, n, *p, d_out, d_cigar, cigar_cap,
                        cigar_used, nullptr, BatchHints{});
  if (e == DNALN_OK) c->stats.cells += 0;
  return e;
}

int dnaln_gpu_map_submit(dnaln_ctx* c, int32_t id, const char* seq, const int64_t* seq_off, const int32_t* seq_len,
                         const uint32_t* name_hash, int64_t n, const dnaln_map_params* p, dnaln_map_record* out,
                         uint32_t* cigar, int64_t cigar_cap, int64_t* cigar_used, int64_t* ticket) {
  if (!c || n < 0 || !cigar_used || !ticket || !p || (n > 0 && (!seq || !seq_off || !seq_len || !name_hash || !out)))
    return fail(c, DNALN_ERR_INVALID_ARG, "null argument");
  *ticket = 0;
  *cigar_used = 0;
  // the index-dependent checks run in the worker (the index table belongs to it while it
  // drives the device); their failures come back from dnaln_gpu_map_wait
  if (int e = validate_map_params_basic(c, p)) return e;
  // parts of at most sub_batch reads, with their host-side facts (lengths are known here)
  const int64_t S = c->sub_batch > 0 ? c->sub_batch : (n > 0 ? n : 1);
  std::vector<MapPart> parts;
  for (int64_t a = 0; a < n; a += S) {
    MapPart pt;
    pt.index_id = id;
    pt.seq = seq;
    pt.seq_off = seq_off;
    pt.seq_len = seq_len;
    pt.name_hash = name_hash;
    pt.a = a;
    pt.b = std::min(n, a + S);
    pt.lo = seq_off[a];
    pt.p = *p;
    pt.out = out;
    pt.cigar = cigar;
    pt.cigar_cap = cigar_cap;
    pt.cigar_used = cigar_used;
    for (int64_t i = pt.a; i < pt.b; ++i) {
      if (seq_len[i] < 0 || seq_off[i] < 0) return fail(c, DNALN_ERR_INVALID_ARG, "negative offset or length");
      pt.lo = std::min(pt.lo, seq_off[i]);
      pt.hi = std::max(pt.hi, seq_off[i] + seq_len[i]);
      pt.bases += seq_len[i];
      pt.max_len = std::max<int64_t>(pt.max_len, seq_len[i]);
      pt.cig_bound += 2 * static_cast<int64_t>(seq_len[i]) + 3;  // walk ops (<= 2*len+1) + 2 clips
    }
    if (pt.hi < pt.lo) pt.hi = pt.lo;
    parts.push_back(pt);
  }
  {
    std::lock_guard<std::mutex> g(c->qmu);
    const int64_t t = c->next_ticket++;
    *ticket = t;
    if (parts.empty()) {
      c->results[t] = DNALN_OK;
      return DNALN_OK;
    }
    parts.back().last = true;
    for (MapPart& pt : parts) {
      pt.ticket = t;
      c->queue.push_back(pt);
    }
    c->ticket_ops[t] = 0;
    if (!c->worker.joinable()) c->worker = std::thread(map_worker, c);
  }
  c->qcv.notify_all();
  return DNALN_OK;
}

int dnaln_gpu_map_wait(dnaln_ctx* c, int64_t ticket) {
  if (!c) return DNALN_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> ql(c->qmu);
  if (ticket <= 0 || ticket >= c->next_ticket) return fail(c, DNALN_ERR_INVALID_ARG, "unknown ticket %lld",
                                                           static_cast<long long>(ticket));
  c->qcv.wait(ql, [&] { return c->results.count(ticket) != 0 || c->stop; });
  auto it = c->results.find(ticket);
  if (it == c->results.end()) return fail(c, DNALN_ERR_INVALID_ARG, "ticket %lld was already waited for",
                                          static_cast<long long>(ticket));
  const int e = it->second;
  c->results.erase(it);
  return e;
}

int dnaln_gpu_map_batch(dnaln_ctx* c, int32_t id, const char* seq, const int64_t* seq_off, const int32_t* seq_len,
                        const uint32_t* name_hash, int64_t n, const dnaln_map_params* p, dnaln_map_record* out,
                        uint32_t* cigar, int64_t cigar_cap, int64_t* cigar_used) {
  int64_t ticket = 0;
  if (int e = dnaln_gpu_map_submit(c, id, seq, seq_off, seq_len, name_hash, n, p, out, cigar, cigar_cap, cigar_used,
                                   &ticket))
    return e;
  return dnaln_gpu_map_wait(c, ticket);
}

}  // extern "C"
