// encode_bulk.cu — codes of both strands of every read (src/mapper.cpp:88-99), staged
// through shared memory by the bulk-copy (TMA) engine.
//
// A block takes tiles of kEncReads consecutive reads, two deep (the next tile's load in
// flight while the current one is converted and stored). When the tile's reads lie back to
// back in the input (the common layout: a batch's reads packed in order) its ASCII bytes
// are one contiguous range, and so are its outputs — read r's forward codes at
// codes[2 pofs[r]], its reverse complement right after them — because the packed offsets
// then differ from the input offsets by a constant. One thread moves the range's 16-byte
// aligned interior into shared memory with a single cp.async.bulk (completion counted on
// an mbarrier), the other threads fetch the at most 15 ragged bytes at either end; the
// warps convert in shared memory (forward code and its complement, a read per warp);
// one thread writes the output range's aligned interior back with a single bulk store
// (cp.async.bulk ... bulk_group) and the threads store its ragged ends. A tile whose reads
// are not back to back, or whose bytes exceed the staging buffer, is encoded read by read
// from global memory, as k_encode_reads does.
//
// Measured against k_encode_reads (one warp per read, byte loads and stores straight to
// and from global memory), CUDA events per 1,000,000 reads: 150 bp, 0.299 against 0.290 ms;
// 50-1000 bp, 1.49 against 0.52 ms (tiles of long reads overflow the staging buffer and
// fall back to a per-read path that has fewer warps than k_encode_reads). The kernel's time
// is the per-byte conversion and the tile phases' latency, not the bytes moved, so staging
// through the copy engine does not pay here: the per-read kernel is the default and this
// one is the option "encode_bulk" 1, tested for identical records.
//
// Waits are bounded: a bulk load not complete after kEncSpinLimit polls of its mbarrier
// sets kErrAsyncCopy and the block stops after one more bounded wait.
#include "common.cuh"
#include "seed.cuh"

namespace dnb {
namespace {

constexpr int kEncThreads = 256;
constexpr int kEncWarps = kEncThreads / 32;
constexpr int kEncReads = 64;      // reads per tile
constexpr int kEncInCap = 16384;   // ASCII bytes a tile may stage
constexpr int kEncOutCap = 2 * kEncInCap;
constexpr int kEncInBytes = kEncInCap + 16;                         // a staging buffer (alignment slack)
constexpr int kEncSmem = 2 * kEncInBytes + kEncOutCap + 16;         // dynamic shared memory of a block
constexpr int kEncSpinLimit = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Arrives on the barrier and announces `bytes` of asynchronous writes it must wait for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n"
      " .reg .b64 st;\n"
      " mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n"
      "}" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for the barrier's phase `parity` to complete.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (int it = 0; it < kEncSpinLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Global -> shared, `bytes` a multiple of 16, both addresses 16-byte aligned; completion
// is counted on `bar` (this CTA's own shared memory: the launch has no cluster).
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst_smem)),
               "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Shared -> global, same alignment rules, as one bulk group.
__device__ __forceinline__ void bulk_store(void* dst_gmem, const void* src_smem, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem), "r"(smem_u32(src_smem)),
               "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Waits until the issued bulk stores have read their shared-memory source.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// Makes this thread's generic-proxy shared-memory writes visible to the bulk-copy engine.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ uintptr_t up16(uintptr_t a) { return (a + 15) & ~static_cast<uintptr_t>(15); }
__device__ __forceinline__ uintptr_t down16(uintptr_t a) { return a & ~static_cast<uintptr_t>(15); }

// Per-tile facts, for the two tiles in flight (the one being converted, the next being loaded).
struct EncTile {
  int64_t r0;       // first read
  int64_t total;    // ASCII bytes of the tile
  uintptr_t a;      // address of its first byte
  int m;            // reads in the tile
  int ok;           // back to back and within the staging capacity
  int bulk;         // a bulk load was issued for it
  int pad_;
};

// Reads the tile's table and, when its reads are back to back and fit, starts staging its
// ASCII into `in`: the 16-byte aligned interior by one bulk load counted on `bar`, the
// ragged ends by the threads. Contains __syncthreads: every thread of the block calls it.
__device__ __forceinline__ void enc_prepare(int64_t tile, int64_t n, const uint8_t* in, const int64_t* seq_off,
                                            int64_t seq_base, const int32_t* seq_len, EncTile& t, int64_t* t_off,
                                            int* t_len, uint8_t* s_in, uint64_t* bar) {
  const int tid = threadIdx.x;
  const int64_t r0 = tile * kEncReads;
  const int m = static_cast<int>(n - r0 < kEncReads ? n - r0 : kEncReads);
  const int64_t off0 = seq_off[r0];
  if (tid < m) {
    t_off[tid] = seq_off[r0 + tid] - off0;
    t_len[tid] = seq_len[r0 + tid];
  }
  if (tid == 0) {
    t.r0 = r0;
    t.m = m;
    t.ok = 1;
    t.bulk = 0;
  }
  __syncthreads();
  if (tid + 1 < m && t_off[tid] + t_len[tid] != t_off[tid + 1]) t.ok = 0;  // not back to back
  const int64_t total = t_off[m - 1] + t_len[m - 1];
  if (tid == 0) {
    if (total > kEncInCap || total < 0) t.ok = 0;
    t.total = total;
    t.a = reinterpret_cast<uintptr_t>(in + (off0 - seq_base));
  }
  __syncthreads();
  if (!t.ok) return;  // block-uniform: every thread returns here
  const uintptr_t a = t.a, b = a + static_cast<uintptr_t>(total);
  const uintptr_t base = down16(a), a16 = up16(a), b16 = down16(b);
  const bool bulk_in = b16 > a16;
  if (bulk_in && tid == 0) {
    // this buffer's earlier generic reads (ordered by the barriers behind us) before the
    // bulk engine writes it
    fence_proxy_async();
    const uint32_t bytes = static_cast<uint32_t>(b16 - a16);
    mbar_arrive_expect_tx(bar, bytes);
    bulk_load(s_in + (a16 - base), reinterpret_cast<const void*>(a16), bytes, bar);
    t.bulk = 1;
  }
  const uintptr_t h_end = bulk_in ? a16 : b, t_beg = bulk_in ? b16 : b;
  for (uintptr_t x = a + tid; x < h_end; x += kEncThreads) s_in[x - base] = *reinterpret_cast<const uint8_t*>(x);
  for (uintptr_t x = t_beg + tid; x < b; x += kEncThreads) s_in[x - base] = *reinterpret_cast<const uint8_t*>(x);
  __syncthreads();  // t.bulk and the ragged bytes are seen by every thread
}

// Dynamic shared memory: two staging buffers of kEncInCap + 16 bytes, one output buffer of
// kEncOutCap + 16. A block works through its tiles two deep: while tile k is converted and
// stored, tile k + 1's ASCII is on its way in.
__global__ void __launch_bounds__(kEncThreads)
    k_encode_tiles(const char* __restrict__ seq, const int64_t* __restrict__ seq_off, int64_t seq_base,
                   const int32_t* __restrict__ seq_len, const int64_t* __restrict__ pofs, int64_t n,
                   uint8_t* __restrict__ codes, uint32_t* __restrict__ err) {
  extern __shared__ __align__(128) uint8_t enc_smem[];
  uint8_t* const s_in0 = enc_smem;
  uint8_t* const s_in1 = enc_smem + kEncInBytes;
  uint8_t* const s_out = enc_smem + 2 * kEncInBytes;
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ EncTile tl[2];
  __shared__ int64_t t_off[2][kEncReads];
  __shared__ int t_len[2][kEncReads];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint8_t* const in = reinterpret_cast<const uint8_t*>(seq);  // read r at in + (seq_off[r] - seq_base)
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
  }
  __syncthreads();
  uint32_t parity[2] = {0u, 0u};
  bool store_pending = false;
  const int64_t tiles = (n + kEncReads - 1) / kEncReads;
  int64_t tile = blockIdx.x;
  if (tile < tiles) enc_prepare(tile, n, in, seq_off, seq_base, seq_len, tl[0], t_off[0], t_len[0], s_in0, &bar[0]);
  for (int k = 0; tile < tiles; ++k, tile += gridDim.x) {
    const int cur = k & 1;
    uint8_t* const s_in = cur ? s_in1 : s_in0;
    const int64_t next = tile + gridDim.x;
    if (next < tiles)  // the next tile's ASCII streams in while this one is converted
      enc_prepare(next, n, in, seq_off, seq_base, seq_len, tl[cur ^ 1], t_off[cur ^ 1], t_len[cur ^ 1],
                  cur ? s_in0 : s_in1, &bar[cur ^ 1]);
    const EncTile t = tl[cur];
    if (!t.ok) {  // read by read from global memory, one warp per read
      for (int j = warp; j < t.m; j += kEncWarps) {
        const int64_t r = t.r0 + j;
        const int len = seq_len[r];
        const uint8_t* si = in + (seq_off[r] - seq_base);
        uint8_t* fw = codes + 2 * pofs[r];
        uint8_t* rc = fw + len;
        for (int i = lane; i < len; i += 32) {
          const uint8_t c = static_cast<uint8_t>(nt4(si[i]));
          fw[i] = c;
          rc[len - 1 - i] = c < 4 ? static_cast<uint8_t>(3 - c) : 4;
        }
      }
      __syncthreads();  // this tile's table is rewritten two tiles on
      continue;
    }
    if (t.bulk) {
      if (!mbar_wait_bounded(&bar[cur], parity[cur])) {
        if (tid == 0) atomicOr(err, kErrAsyncCopy);
        mbar_wait_bounded(&bar[cur], parity[cur]);  // the copy may still be landing: one more bounded wait
        if (tid == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
        return;
      }
      parity[cur] ^= 1u;
    }
    if (store_pending && tid == 0) bulk_wait_read();  // the previous tile's store has read s_out
    __syncthreads();
    // ---- convert: s_out[j] holds the code for address obase + j
    const uintptr_t a = t.a, base = down16(a);
    uint8_t* const oa_p = codes + 2 * pofs[t.r0];
    const uintptr_t oa = reinterpret_cast<uintptr_t>(oa_p), ob = oa + 2 * static_cast<uintptr_t>(t.total);
    const uintptr_t obase = down16(oa), oa16 = up16(oa), ob16 = down16(ob);
    const int ohead = static_cast<int>(oa - obase), ihead = static_cast<int>(a - base);
    for (int j = warp; j < t.m; j += kEncWarps) {
      const int rel = static_cast<int>(t_off[cur][j]), len = t_len[cur][j];
      const uint8_t* si = s_in + ihead + rel;
      uint8_t* fw = s_out + ohead + 2 * rel;
      uint8_t* rc = fw + len;
      for (int i = lane; i < len; i += 32) {
        const uint8_t c = static_cast<uint8_t>(nt4(si[i]));
        fw[i] = c;
        rc[len - 1 - i] = c < 4 ? static_cast<uint8_t>(3 - c) : 4;
      }
    }
    fence_proxy_async();
    __syncthreads();
    // ---- write back: the aligned interior by one bulk store, the ragged ends by the threads
    const bool bulk_out = ob16 > oa16;
    if (bulk_out && tid == 0)
      bulk_store(reinterpret_cast<void*>(oa16), s_out + (oa16 - obase), static_cast<uint32_t>(ob16 - oa16));
    store_pending = bulk_out;
    const uintptr_t h_end = bulk_out ? oa16 : ob, t_beg = bulk_out ? ob16 : ob;
    for (uintptr_t x = oa + tid; x < h_end; x += kEncThreads) *reinterpret_cast<uint8_t*>(x) = s_out[x - obase];
    for (uintptr_t x = t_beg + tid; x < ob; x += kEncThreads) *reinterpret_cast<uint8_t*>(x) = s_out[x - obase];
    __syncthreads();  // the ragged ends read s_out; this tile's table is rewritten two tiles on
  }
  if (tid == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");  // the last stores complete
}

}  // namespace

void launch_encode_reads_bulk(cudaStream_t st, const char* seq, const int64_t* seq_off, int64_t seq_base,
                              const int32_t* seq_len, const int64_t* pofs, int64_t n, uint8_t* codes, uint32_t* err) {
  if (n <= 0) return;
  static std::atomic<bool> attr_set[kMaxDevices];
  if (!set_smem_limit_once(k_encode_tiles, kEncSmem, attr_set)) {  // cannot happen on sm_100: read by read
    launch_encode_reads(st, seq, seq_off, seq_base, seq_len, pofs, n, codes);
    return;
  }
  const int64_t tiles = (n + kEncReads - 1) / kEncReads;
  const int64_t blocks = std::min<int64_t>(tiles, int64_t{3} * device_sm_count());  // 3 resident blocks per SM
  k_encode_tiles<<<static_cast<unsigned>(blocks), kEncThreads, kEncSmem, st>>>(seq, seq_off, seq_base, seq_len, pofs,
                                                                               n, codes, err);
}

}  // namespace dnb
