// peak.cu — measured issue rate of the integer instructions the banded SW recurrence is made
// of: the denominator of the SW kernels' integer roofline (no reference counterpart).
//
// The 16x2 SW kernels (sw.cu) spend their cells on two kinds of instruction: 32-bit integer
// adds, each serving both biased 16-bit halves, and 16x2 maxima (vmaxu2 and the DPX three-
// way maximum vimax3_u16x2). k_int_peak runs long chains of exactly these on every SM: each
// thread keeps eight independent chains, and per step a chain does one add and one DPX
// maximum that depend on each other (so no step can be folded away or hoisted), for
// `iters` steps. Mode 0 issues the two one to one (the recurrence's mix), mode 1 adds
// only, mode 2 DPX maxima only. The result is thread instructions of the mode per second,
// timed with CUDA events on the given stream, the best of `reps` launches.
#include <cuda_runtime.h>

#include "common.cuh"
#include "dnaln_b200.h"

namespace dnb {
namespace {

constexpr int kPeakThreads = 256;
constexpr int kChains = 8;
constexpr int kUnroll = 4;

template <int MODE>
__global__ void __launch_bounds__(kPeakThreads) k_int_peak(int iters, uint32_t seed, uint32_t* __restrict__ sink) {
  uint32_t a[kChains], b[kChains];
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
  for (int u = 0; u < kChains; ++u) {
    a[u] = seed ^ (t * 0x9E3779B9u + static_cast<uint32_t>(u));
    b[u] = (seed + static_cast<uint32_t>(u)) * 0x85EBCA6Bu ^ t;
  }
  const uint32_t c = seed | 0x00010001u;
  for (int it = 0; it < iters; it += kUnroll) {
#pragma unroll
    for (int r = 0; r < kUnroll; ++r) {
#pragma unroll
      for (int u = 0; u < kChains; ++u) {
        if constexpr (MODE == 0) {
          a[u] = a[u] + b[u];
          b[u] = __vimax3_u16x2(b[u], a[u], c);
        } else if constexpr (MODE == 1) {
          a[u] = a[u] + b[u];
          b[u] = b[u] + a[u];
        } else {
          a[u] = __vimax3_u16x2(a[u], b[u], c);
          b[u] = __vimax3_u16x2(b[u], a[u], c ^ a[u]);
        }
      }
    }
  }
  uint32_t x = 0;
#pragma unroll
  for (int u = 0; u < kChains; ++u) x ^= a[u] ^ b[u];
  if (x == 0x7F4A7C15u) sink[t & 1023] = x;  // keeps every chain live; practically never taken
}

template <int MODE>
void launch_peak(cudaStream_t st, unsigned blocks, int iters, uint32_t seed, uint32_t* sink) {
  k_int_peak<MODE><<<blocks, kPeakThreads, 0, st>>>(iters, seed, sink);
}

}  // namespace
}  // namespace dnb

extern "C" int dnaln_gpu_int_peak(int32_t device, int32_t mode, void* stream, double* thread_ops_per_s,
                                  double* best_ms) {
  using namespace dnb;
  if (mode < 0 || mode > 2 || !thread_ops_per_s) return DNALN_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return DNALN_ERR_NO_DEVICE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint32_t* sink = nullptr;
  if (cudaMalloc(&sink, 1024 * sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();
    return DNALN_ERR_OOM;
  }
  const int sms = device_sm_count();
  const unsigned blocks = static_cast<unsigned>(sms) * 8u;  // 8 blocks of 256 threads: 64 warps per SM
  const int iters = 8192;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = 1e30;
  int rc = DNALN_OK;
  for (int rep = 0; rep < 6 && rc == DNALN_OK; ++rep) {  // the first launch warms up
    cudaEventRecord(e0, st);
    if (mode == 0) launch_peak<0>(st, blocks, iters, 12345u + rep, sink);
    else if (mode == 1) launch_peak<1>(st, blocks, iters, 12345u + rep, sink);
    else launch_peak<2>(st, blocks, iters, 12345u + rep, sink);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = DNALN_ERR_CUDA;
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (rc != DNALN_OK) return rc;
  const double ops = static_cast<double>(blocks) * kPeakThreads * iters * kChains * 2.0;
  *thread_ops_per_s = ops / (best * 1e-3);
  if (best_ms) *best_ms = best;
  return DNALN_OK;
}
