// noalloc.cu — banded SW with traceback for callers that cannot allocate device memory.
//
// Some callers of this library must not call cudaMalloc: code that runs under a host
// framework owning every device allocation (a fixed memory pool, a strict budget, an
// allocator that must not fragment), or inside a serving loop that is not allowed to
// allocate per request. dnaln_gpu_align allocates its scratch through the context;
// dnaln_gpu_align_noalloc instead takes caller-owned device inputs and outputs and draws
// every piece of scratch (task descriptors, per-task results, the direction-bit matrices
// of the traceback, the band rows of wide-band kernels, the error flag) from one
// file-scope device array of fixed size, kNoAllocScratchBytes, which every GPU that
// loads this library holds until the process exits. Work larger than the array is split
// into consecutive launches on the caller's stream; a task whose single warp of scratch
// would not fit (very long queries with wide bands) is rejected up front.
//
// The array is shared by every call: calls whose work overlaps on the GPU (different
// streams, or different host threads on one device) race on it, so callers serialize
// them. Each call clears the error flag before its first launch; nothing else in the
// array needs clearing (every scratch cell is written before it is read).
//
// Set-up: host code cannot use the array's name as a device address (in host code it
// names a host-side stand-in), so each call takes the address with cudaGetSymbolAddress
// for the device current at the call, unless the caller's stream is being captured, when
// the address the last uncaptured call on that device took is used instead. The first
// call on each device should therefore come before any stream capture. The caller's stream
// must belong to the device that is current at the call.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "dnaln_b200.h"
#include "sw.cuh"

namespace dnb {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;  // 64 MiB
constexpr size_t kHeader = 256;                            // error flag lives at offset 0

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Task descriptors for tasks [base, base + count) of the caller's arrays. A task the
// caller described wrongly (a query longer than max_qlen, a negative length or offset) is
// flagged with kErrBadTask and aligned as empty, so that no scratch is overrun and no
// byte before the caller's buffers is read.
__global__ void k_na_tasks(int64_t base, int count, const int64_t* __restrict__ q_off,
                           const int32_t* __restrict__ q_len, const int64_t* __restrict__ t_off,
                           const int32_t* __restrict__ t_len, int max_qlen, int W, int64_t cigar_stride,
                           SwTask* __restrict__ tasks, int64_t* __restrict__ cig_off, uint32_t* __restrict__ err) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  const int64_t i = base + j;
  int ql = q_len[i];
  int tl = t_len[i];
  int64_t qo = q_off[i], to = t_off[i];
  if (ql < 0 || ql > max_qlen || tl < 0 || qo < 0 || to < 0) {
    atomicOr(err, kErrBadTask);
    ql = 0;
    tl = 0;
    qo = 0;
    to = 0;
  }
  const int64_t tmax = static_cast<int64_t>(ql) + W - 1;
  SwTask t;
  t.q_off = qo;
  t.qlen = ql;
  t.t_start = to;
  t.t_lo = to;
  t.t_hi = to + (tl < tmax ? tl : tmax);
  t.slot = j;
  t.flags = 0;
  t.pad_ = 0;
  tasks[j] = t;
  cig_off[j] = i * cigar_stride;
}

// Results of the chunk into the caller's array; CIGAR ops reversed in place from walk
// order to the reference's order (src/align.cpp:139).
__global__ void k_na_finish(int64_t base, int count, const SwResult* __restrict__ res, int64_t cigar_stride,
                            bool traceback, dnaln_align_result* __restrict__ out, uint32_t* __restrict__ cigar) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  const int64_t i = base + j;
  const SwResult a = res[j];
  dnaln_align_result o;
  o.score = a.score;
  o.qb = a.qb;
  o.qe = a.qe;
  o.tb = a.tb;
  o.te = a.te;
  o.nm = a.nm;
  o.cigar_off = i * cigar_stride;
  o.cigar_len = traceback ? a.n_ops : 0;
  o.pad_ = 0;
  out[i] = o;
  if (traceback && a.n_ops > 1) {
    uint32_t* c = cigar + i * cigar_stride;
    for (int x = 0, y = a.n_ops - 1; x < y; ++x, --y) {
      const uint32_t t = c[x];
      c[x] = c[y];
      c[y] = t;
    }
  }
}

// The device address of g_noalloc_scratch for the current device. Looked up again on
// every call made outside a stream capture (so a context created after cudaDeviceReset
// gets its own array's address); inside a capture the address of the last uncaptured
// call on this device is used.
int scratch_address(cudaStream_t st, unsigned char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return DNALN_ERR_NO_DEVICE;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const bool capturing = cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
  cudaGetLastError();
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!capturing) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return DNALN_ERR_CUDA;
    }
    g_addr[dev] = p;
  }
  if (!g_addr[dev]) return DNALN_ERR_CUDA;  // first call on this device made inside a capture
  *out = static_cast<unsigned char*>(g_addr[dev]);
  return DNALN_OK;
}

}  // namespace
}  // namespace dnb

extern "C" int dnaln_gpu_align_noalloc(const uint8_t* d_q, const int64_t* d_q_off, const int32_t* d_q_len,
                                       const uint8_t* d_t, const int64_t* d_t_off, const int32_t* d_t_len, int64_t n,
                                       int32_t max_qlen, int32_t traceback, const dnaln_score_params* sp,
                                       dnaln_align_result* d_out, uint32_t* d_cigar, int64_t cigar_stride,
                                       void* stream) {
  using namespace dnb;
  if (!sp || n < 0 || max_qlen < 0) return DNALN_ERR_INVALID_ARG;
  if (sp->bw < 0 || sp->bw > 1000 || sp->gap_ext < 0 || sp->gap_open < 0 || sp->mismatch < 0 || sp->ambig < 0)
    return DNALN_ERR_INVALID_ARG;
  const bool tb = traceback != 0;
  if (tb && cigar_stride < 2 * static_cast<int64_t>(max_qlen) + 1) return DNALN_ERR_INVALID_ARG;
  if (n == 0) return DNALN_OK;
  if (!d_q || !d_q_off || !d_q_len || !d_t || !d_t_off || !d_t_len || !d_out || (tb && !d_cigar))
    return DNALN_ERR_INVALID_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* base_ptr = nullptr;
  if (int e = scratch_address(st, &base_ptr)) return e;

  const SwParams p = make_sw_params(*sp);
  const bool bytes_ok = sw_bytes_ok(*sp);
  const int rows = max_qlen > 0 ? max_qlen : 1;
  const size_t dir_t = tb ? sw_dir_bytes_per_task(p.W, rows) : 0;
  const size_t band_t = sw_band_bytes_per_task(p.W, bytes_ok);
  // scratch per group of kSwTaskGroup tasks: descriptors, CIGAR offsets, results,
  // direction codes, band rows, int32-path task list (one more int for its count)
  const int64_t G = kSwTaskGroup;
  const size_t per_group = G * (sizeof(SwTask) + sizeof(int64_t) + sizeof(SwResult) + dir_t + band_t + sizeof(int));
  const size_t avail = kNoAllocScratchBytes - kHeader - 6 * 256;
  const int64_t groups = static_cast<int64_t>(avail / per_group);
  if (groups < 1) return DNALN_ERR_INVALID_ARG;  // one group of this query length / band does not fit 64 MiB
  const int64_t chunk = std::min<int64_t>(groups * G, ((n + G - 1) / G) * G);
  const size_t dir_w = dir_t, band_w = band_t;

  uint32_t* err = reinterpret_cast<uint32_t*>(base_ptr);
  unsigned char* cur = base_ptr + kHeader;
  SwTask* tasks = reinterpret_cast<SwTask*>(cur);
  cur += align256(chunk * sizeof(SwTask));
  int64_t* cig_off = reinterpret_cast<int64_t*>(cur);
  cur += align256(chunk * sizeof(int64_t));
  SwResult* res = reinterpret_cast<SwResult*>(cur);
  cur += align256(chunk * sizeof(SwResult));
  uint32_t* dir = dir_w ? reinterpret_cast<uint32_t*>(cur) : nullptr;
  cur += align256(chunk * dir_w);
  int* band = band_w ? reinterpret_cast<int*>(cur) : nullptr;
  cur += align256(chunk * band_w);
  int* fb = reinterpret_cast<int*>(cur);

  if (cudaMemsetAsync(err, 0, sizeof(uint32_t), st) != cudaSuccess) return DNALN_ERR_CUDA;
  for (int64_t b = 0; b < n; b += chunk) {
    const int cnt = static_cast<int>(std::min<int64_t>(chunk, n - b));
    const int blocks = (cnt + 127) / 128;
    k_na_tasks<<<blocks, 128, 0, st>>>(b, cnt, d_q_off, d_q_len, d_t_off, d_t_len, max_qlen, p.W,
                                       tb ? cigar_stride : 0, tasks, cig_off, err);
    if (!launch_sw(st, tb, bytes_ok, tasks, 0, cnt, cnt, nullptr, d_q, d_t, p, res, dir, rows,
                   tb ? d_cigar : nullptr, cig_off, band, fb, err, nullptr))
      return DNALN_ERR_DEVICE;
    k_na_finish<<<blocks, 128, 0, st>>>(b, cnt, res, tb ? cigar_stride : 0, tb, d_out, d_cigar);
    if (cudaGetLastError() != cudaSuccess) return DNALN_ERR_CUDA;
  }
  uint32_t bits = 0;
  if (cudaMemcpyAsync(&bits, err, sizeof bits, cudaMemcpyDeviceToHost, st) != cudaSuccess) return DNALN_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return DNALN_ERR_CUDA;
  if (bits & ~kErrBadTask) return DNALN_ERR_DEVICE;  // a kernel's own consistency check
  return bits ? DNALN_ERR_INVALID_ARG : DNALN_OK;       // only tasks the caller described wrongly
}
