// common.cuh — shared device-side definitions of the B200 mapping path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "dnaln_b200.h"

namespace dnb {

constexpr int kMaxDevices = 64;

// Streaming multiprocessors of the current device (148 on a B200), looked up once per
// device; grids that stride over their work are sized by it.
inline int device_sm_count() {
  static std::atomic<int> sms[kMaxDevices];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return 148;
  }
  int v = sms[dev].load(std::memory_order_relaxed);
  if (v > 0) return v;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
    cudaGetLastError();
    v = 148;
  }
  sms[dev].store(v, std::memory_order_relaxed);
  return v;
}

// Raises a kernel's dynamic shared-memory limit once per device; host threads that map
// batches at the same time may race to do it, which is harmless (the attribute is the same).
template <class Kernel>
bool set_smem_limit_once(Kernel* kernel, int bytes, std::atomic<bool>* done) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return false;
  }
  if (done[dev].load(std::memory_order_acquire)) return true;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  done[dev].store(true, std::memory_order_release);
  return true;
}

constexpr uint64_t kInvalidHash = ~0ULL;  // palindromic k-mer / empty bucket (src/minimizer.cpp:7, src/index.hpp:53)
constexpr int kWarp = 32;

// Device error flags (bitwise OR into ErrorFlags::bits); any set bit fails the call with
// DNALN_ERR_DEVICE. None of them can occur for well-formed input: they guard index
// arithmetic so that a broken invariant is reported instead of reading out of bounds.
enum : uint32_t {
  kErrTracebackBounds = 1u << 0,
  kErrCigarOverflow = 1u << 1,
  kErrChainScratch = 1u << 2,
  kErrProbeLoop = 1u << 3,
  // not failures of the input: the chaining scratch pool of a batch was too small (the
  // host grows it and maps the batch again), and the caller's CIGAR buffer was too small
  kErrChainPool = 1u << 4,
  kErrOutputCapacity = 1u << 5,
  // a task the caller described wrongly, found on the device (dnaln_gpu_align_noalloc: a
  // query longer than the stated maximum, a negative length or offset); the call fails
  // with DNALN_ERR_INVALID_ARG and the other tasks' results stand
  kErrBadTask = 1u << 6,
  // a bulk (TMA) copy into shared memory did not complete within its wait's bound
  kErrAsyncCopy = 1u << 7,
};

// Thomas Wang's 64-bit mix restricted to `mask` bits, step for step as the index keys are
// defined (src/minimizer.hpp:21-31).
__host__ __device__ __forceinline__ uint64_t hash64(uint64_t key, uint64_t mask) {
  key = (~key + (key << 21)) & mask;
  key = key ^ key >> 24;
  key = ((key + (key << 3)) + (key << 8)) & mask;
  key = key ^ key >> 14;
  key = ((key + (key << 2)) + (key << 4)) & mask;
  key = key ^ key >> 28;
  key = (key + (key << 31)) & mask;
  return key;
}

// ASCII -> base code, A/a 0, C/c 1, G/g 2, T/t/U/u 3, else 4 (src/common.hpp:23-31),
// branch-free: (c & 0xDF) - 'A' indexes a bit set of {A, C, G, T, U}; for those letters
// ((c >> 1) ^ (c >> 2)) & 3 is 0, 1, 2, 3, 3. Checked against the table for all 256 bytes.
__host__ __device__ __forceinline__ uint32_t nt4(uint32_t c) {
  const uint32_t u = (c & 0xDFu) - 0x41u;
  const bool ok = u < 21u && ((0x180045u >> u) & 1u);
  return ok ? (((c >> 1) ^ (c >> 2)) & 3u) : 4u;
}

// One band-SW task, in either addressing mode:
//   query  = qbase[q_off .. q_off + qlen)
//   target column j = tbase[t_start + j] when t_lo <= t_start + j < t_hi, else N.
// GpuAligner tasks use a flat target buffer (t_lo = t_start, t_hi = t_start + tlen);
// mapping tasks index the resident genome with the candidate contig's bounds, which
// is the N-padded window of src/mapper.cpp:100-121 without a copy.
struct SwTask {
  int64_t q_off;
  int64_t t_start, t_lo, t_hi;
  int32_t qlen;
  int32_t slot;   // result / CIGAR slot
  int32_t flags;  // kTaskNoN: the producer checked that the window [0, qlen + W - 1) has no N
  int32_t pad_;
};
constexpr int32_t kTaskNoN = 1;

struct SwResult {
  int32_t score, qb, qe, tb, te, nm;
  int32_t n_ops;  // CIGAR ops written (traceback order, i.e. reversed)
  int32_t pad_;
};

struct SwParams {
  int32_t match, mismatch, oe, ge, ambig, bw, W;
  uint32_t prof_n;  // 4 bytes of -ambig (table entries 4..7 of the byte-permute profile)
};

// Optional per-kernel timing hook of the orchestrator: begin() before a launch and end()
// after it record an event pair on the launching stream under the kernel's name. A null
// hook (or one with no callback) costs nothing.
struct KernelTrace {
  void (*mark)(void* self, cudaStream_t st, const char* kernel) = nullptr;  // kernel == nullptr: end
  void* self = nullptr;
  void begin(cudaStream_t st, const char* kernel) const {
    if (mark) mark(self, st, kernel);
  }
  void end(cudaStream_t st) const {
    if (mark) mark(self, st, nullptr);
  }
};

__host__ __device__ __forceinline__ int sub_score(const SwParams& p, int a, int b) {
  return (a > 3 || b > 3) ? -p.ambig : (a == b ? p.match : -p.mismatch);  // src/align.hpp:39
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ long long warp_max_ll(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const long long x = __shfl_xor_sync(0xffffffffu, v, o);
    v = x > v ? x : v;
  }
  return v;
}

// Exclusive prefix sum across the warp; *total receives the warp-wide sum.
__device__ __forceinline__ int warp_exclusive_scan(int v, int* total) {
  const int lane = threadIdx.x & 31;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  *total = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}

}  // namespace dnb
