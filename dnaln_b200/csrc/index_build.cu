// index_build.cu — MinimizerIndex::build (src/index.cpp:10-45) on the device.
//
// The genome is already resident (one code per byte). Steps:
//   1. minimizers of every contig (src/minimizer.cpp:5-68), in tiles of kTile window ends:
//      a block stages its bases, forms the canonical k-mer hashes of the tile plus the w
//      k-mers before it, and each thread decides, for 8 consecutive window ends, whether
//      the window is whole (w consecutive N-free k-mers of one contig) and whether its
//      leftmost minimum is emitted (valid, and not the same position as the previous
//      window's minimum — the reference's `last` can only repeat from the window just
//      before, because minimum positions never decrease inside an N-free run and an
//      all-palindrome window keeps no valid minimum). A count pass and a scan place each
//      tile's minimizers in genome order, so the stable radix sort by hash below leaves
//      positions ascending within a key: the reference's (hash, pos) order.
//   2. stable radix sort of (hash, pos << 1 | strand) by hash;
//   3. distinct keys (run-length encoding), their offsets and counts, the largest count;
//   4. the bucket table: cap = smallest power of two >= max(16, 2 * n_keys), keys placed
//      by linear probing from hash & mask as if inserted one by one in ascending hash
//      order (the reference's loop). In parallel: every key walks from its home bucket and
//      claims buckets with atomicMin on its rank (its place in ascending hash order); a key
//      that takes a bucket from a higher rank sends that key on from the next bucket. A
//      bucket's rank only decreases, so at the end every key sits in the first bucket from
//      its home not held by a lower rank — by induction on the rank, the bucket sequential
//      insertion gives it;
//   5. the maximal runs of non-ACGT codes (used by SW task builders).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_run_length_encode.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <cub/block/block_scan.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <cstdio>
#include <vector>

#include "common.cuh"
#include "index_build.cuh"

namespace dnb {
namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr int kTile = kThreads * kPerThread;  // window ends per block
constexpr int kMaxW = 255;
constexpr int kMaxK = 28;
constexpr uint32_t kEmptyRank = 0xFFFFFFFFu;

struct Tile {
  int64_t t0, t1;  // window ends (k-mer starts) [t0, t1)
  int64_t cs, ce;  // the contig [cs, ce)
};

struct TileSmem {
  uint8_t base[kTile + kMaxW + kMaxK];
  uint64_t hash[kTile + kMaxW];  // kInvalidHash for palindromes
  uint8_t ok[kTile + kMaxW];     // k-mer inside the contig and N-free
  uint8_t strand[kTile + kMaxW];
};

// Window ending at k-mer e (region index x = e - r0): whole, and its leftmost minimum.
__device__ __forceinline__ void window_at(const TileSmem& sm, int x, int w, bool& whole, int& arg) {
  whole = x >= w - 1;
  uint64_t best = kInvalidHash;
  arg = -1;
  for (int y = x - w + 1; y <= x && whole; ++y) {
    if (!sm.ok[y]) whole = false;
    if (sm.hash[y] < best) {  // strict: ties keep the leftmost
      best = sm.hash[y];
      arg = y;
    }
  }
  if (!whole || best == kInvalidHash) arg = -1;
}

// Pass 1 (out == nullptr): per-tile minimizer counts. Pass 2: the minimizers of tile b at
// out_*[tile_off[b] ..], in position order.
__global__ void __launch_bounds__(kThreads)
    k_genome_minimizers(const uint8_t* __restrict__ genome, const Tile* __restrict__ tiles, int k, int w,
                        int64_t* __restrict__ tile_count, const int64_t* __restrict__ tile_off,
                        uint64_t* __restrict__ out_hash, uint32_t* __restrict__ out_val) {
  __shared__ TileSmem sm;
  using BlockScan = cub::BlockScan<int, kThreads>;
  __shared__ typename BlockScan::TempStorage scan_tmp;
  const Tile tl = tiles[blockIdx.x];
  // region of k-mer starts [r0, tl.t1): the tile and the w k-mers before it
  const int64_t r0 = tl.t0 - w;
  const int nk = static_cast<int>(tl.t1 - r0);
  const int nb = nk + k - 1;
  for (int i = threadIdx.x; i < nb; i += kThreads) {
    const int64_t p = r0 + i;
    sm.base[i] = (p >= tl.cs && p < tl.ce) ? genome[p] : 4;
  }
  __syncthreads();
  const uint64_t mask = (1ULL << (2 * k)) - 1;
  for (int i = threadIdx.x; i < nk; i += kThreads) {
    const int64_t s = r0 + i;
    bool ok = s >= tl.cs && s + k <= tl.ce;
    uint64_t fwd = 0, rev = 0;
    for (int m = 0; m < k; ++m) {
      const uint32_t c = sm.base[i + m];
      ok = ok && c <= 3;
      fwd = fwd << 2 | (c & 3u);
      rev |= static_cast<uint64_t>(3u - (c & 3u)) << (2 * m);
    }
    const uint32_t st = rev < fwd;
    sm.ok[i] = ok;
    sm.strand[i] = static_cast<uint8_t>(st);
    sm.hash[i] = (ok && fwd != rev) ? hash64(st ? rev : fwd, mask) : kInvalidHash;
  }
  __syncthreads();
  // this thread's window ends: region indices x in [w + 8t, w + 8t + 8) within the tile
  const int x0 = w + threadIdx.x * kPerThread;
  int cnt = 0;
  uint32_t emit_bits = 0;
  if (x0 < nk) {
    bool whole_prev;
    int arg_prev;
    window_at(sm, x0 - 1, w, whole_prev, arg_prev);
    for (int d = 0; d < kPerThread && x0 + d < nk; ++d) {
      bool whole;
      int arg;
      window_at(sm, x0 + d, w, whole, arg);
      if (arg >= 0 && !(whole_prev && arg_prev == arg)) {
        emit_bits |= 1u << d;
        ++cnt;
      }
      whole_prev = whole;
      arg_prev = arg;
    }
  }
  int before = 0, total = 0;
  BlockScan(scan_tmp).ExclusiveSum(cnt, before, total);
  if (!out_hash) {
    if (threadIdx.x == 0) tile_count[blockIdx.x] = total;
    return;
  }
  int64_t o = tile_off[blockIdx.x] + before;
  for (int d = 0; d < kPerThread; ++d) {
    if (!((emit_bits >> d) & 1u)) continue;
    bool whole;
    int arg;
    window_at(sm, x0 + d, w, whole, arg);
    out_hash[o] = sm.hash[arg];
    out_val[o] = static_cast<uint32_t>(r0 + arg) << 1 | sm.strand[arg];
    ++o;
  }
}

// Bucket placement by rank (see the file comment); err set if a walk passes every bucket.
__global__ void k_place_keys(const uint64_t* __restrict__ keys, int64_t n_keys, uint64_t mask,
                             uint32_t* __restrict__ slot_rank, uint32_t* __restrict__ err) {
  const int64_t r0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r0 >= n_keys) return;
  uint32_t r = static_cast<uint32_t>(r0);
  uint64_t s = keys[r] & mask;
  for (uint64_t steps = 0; steps <= 4 * (mask + 1) + 64; ++steps) {
    const uint32_t old = atomicMin(slot_rank + s, r);
    if (old == kEmptyRank) return;  // placed in an empty bucket
    // old > r: r took the bucket and the displaced key walks on from the next bucket (every
    // bucket from its home up to here holds a lower rank: it walked past them, and a
    // bucket's rank only decreases); old < r: a lower rank holds the bucket, r walks on
    if (old > r) r = old;
    s = (s + 1) & mask;
  }
  atomicOr(err, kErrProbeLoop);
}

__global__ void k_fill_table(const uint32_t* __restrict__ slot_rank, uint64_t n_buckets,
                             const uint64_t* __restrict__ keys, const int64_t* __restrict__ offs,
                             const int32_t* __restrict__ counts, ulonglong2* __restrict__ table) {
  const uint64_t s = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= n_buckets) return;
  const uint32_t r = slot_rank[s];
  table[s] = r == kEmptyRank ? make_ulonglong2(kInvalidHash, 0)
                             : make_ulonglong2(keys[r], static_cast<uint64_t>(offs[r]) |
                                                            static_cast<uint64_t>(static_cast<uint32_t>(counts[r])) << 32);
}

__global__ void k_widen(const int32_t* __restrict__ in, int64_t n, int64_t* __restrict__ out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i];
}

__global__ void k_nrun_flags(const uint8_t* __restrict__ g, int64_t n, uint8_t* __restrict__ is_start,
                             uint8_t* __restrict__ is_end) {
  const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const bool here = g[p] > 3;
  is_start[p] = here && (p == 0 || g[p - 1] <= 3);
  is_end[p] = here && (p == n - 1 || g[p + 1] <= 3);
}

__global__ void k_nrun_pack(const int64_t* __restrict__ starts, const int64_t* __restrict__ ends, int64_t m,
                            uint2* __restrict__ runs) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < m) runs[i] = make_uint2(static_cast<uint32_t>(starts[i]), static_cast<uint32_t>(ends[i] + 1));
}

struct Scratch {  // temporary device buffers of one build, freed on every path out
  std::vector<void*> ptrs;
  ~Scratch() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <class T>
  T* get(size_t count, cudaError_t& e) {
    void* p = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&p, (count ? count : 1) * sizeof(T));
    if (e != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
};

inline unsigned blocks_for(int64_t n, int t = 256) { return static_cast<unsigned>((n + t - 1) / t); }

}  // namespace

int find_n_runs_on_device(cudaStream_t st, const uint8_t* d_genome, uint64_t n_bases, uint2** runs_out,
                          int32_t* n_runs_out, char* err, size_t err_len) {
  *runs_out = nullptr;
  *n_runs_out = 0;
  auto failed = [&](cudaError_t e) {
    snprintf(err, err_len, "index (N runs): %s", cudaGetErrorString(e));
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? DNALN_ERR_OOM : DNALN_ERR_CUDA;
  };
  Scratch tmp;
  cudaError_t e = cudaSuccess;
  uint8_t* is_start = tmp.get<uint8_t>(n_bases, e);
  uint8_t* is_end = tmp.get<uint8_t>(n_bases, e);
  int64_t* d_nr = tmp.get<int64_t>(2, e);
  if (e != cudaSuccess) return failed(e);
  int64_t n_runs = 0;
  int64_t* starts = nullptr;
  int64_t* ends = nullptr;
  if (n_bases) {
    k_nrun_flags<<<blocks_for(static_cast<int64_t>(n_bases)), 256, 0, st>>>(d_genome, static_cast<int64_t>(n_bases),
                                                                            is_start, is_end);
    size_t cb = 0;  // the number of runs first, so that their arrays are sized exactly
    if ((e = cub::DeviceReduce::Sum(nullptr, cb, is_start, d_nr, static_cast<int64_t>(n_bases), st)) != cudaSuccess)
      return failed(e);
    void* d_cb = tmp.get<uint8_t>(cb, e);
    if (e == cudaSuccess) e = cub::DeviceReduce::Sum(d_cb, cb, is_start, d_nr, static_cast<int64_t>(n_bases), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&n_runs, d_nr, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    starts = tmp.get<int64_t>(n_runs, e);
    ends = tmp.get<int64_t>(n_runs, e);
    if (e != cudaSuccess) return failed(e);
    thrust::counting_iterator<int64_t> idx(0);
    size_t fb = 0;
    if ((e = cub::DeviceSelect::Flagged(nullptr, fb, idx, is_start, starts, d_nr, static_cast<int64_t>(n_bases),
                                        st)) != cudaSuccess)
      return failed(e);
    void* d_fb = tmp.get<uint8_t>(fb, e);
    if (e == cudaSuccess)
      e = cub::DeviceSelect::Flagged(d_fb, fb, idx, is_start, starts, d_nr, static_cast<int64_t>(n_bases), st);
    if (e == cudaSuccess)
      e = cub::DeviceSelect::Flagged(d_fb, fb, idx, is_end, ends, d_nr + 1, static_cast<int64_t>(n_bases), st);
    if (e != cudaSuccess) return failed(e);
  }
  uint2* runs = nullptr;
  if ((e = cudaMalloc(&runs, (n_runs ? n_runs : 1) * sizeof(uint2))) != cudaSuccess) return failed(e);
  *runs_out = runs;
  *n_runs_out = static_cast<int32_t>(n_runs);
  if (n_runs) k_nrun_pack<<<blocks_for(n_runs), 256, 0, st>>>(starts, ends, n_runs, runs);
  // the scratch is freed on return: the pack must be done with it first
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess) return failed(e);
  return DNALN_OK;
}

int build_index_on_device(cudaStream_t st, const uint8_t* d_genome, uint64_t n_bases, const uint64_t* contig_off,
                          const uint32_t* contig_len, int32_t n_contigs, int k, int w, DeviceIndexBuild* out,
                          char* err, size_t err_len) {
  *out = DeviceIndexBuild{};
  auto failed = [&](const char* what, cudaError_t e) {
    snprintf(err, err_len, "index build (%s): %s", what, cudaGetErrorString(e));
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? DNALN_ERR_OOM : DNALN_ERR_CUDA;
  };
  if (k < 4 || k > kMaxK || w < 1 || w > kMaxW) {
    snprintf(err, err_len, "index build: k or w out of range");
    return DNALN_ERR_INVALID_ARG;
  }
  Scratch tmp;
  cudaError_t e = cudaSuccess;
  // tiles of window ends, never across a contig
  std::vector<Tile> tiles;
  for (int32_t c = 0; c < n_contigs; ++c) {
    const int64_t cs = static_cast<int64_t>(contig_off[c]), ce = cs + contig_len[c];
    for (int64_t t0 = cs; t0 < ce; t0 += kTile) tiles.push_back(Tile{t0, t0 + kTile < ce ? t0 + kTile : ce, cs, ce});
  }
  const int64_t n_tiles = static_cast<int64_t>(tiles.size());
  Tile* d_tiles = tmp.get<Tile>(n_tiles, e);
  int64_t* d_tcount = tmp.get<int64_t>(n_tiles + 1, e);
  int64_t* d_toff = tmp.get<int64_t>(n_tiles + 1, e);
  uint32_t* d_err = tmp.get<uint32_t>(1, e);
  if (e != cudaSuccess) return failed("scratch", e);
  if (n_tiles) e = cudaMemcpyAsync(d_tiles, tiles.data(), n_tiles * sizeof(Tile), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_tcount, 0, (n_tiles + 1) * sizeof(int64_t), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess) return failed("upload", e);
  // 1. minimizers in genome order
  if (n_tiles)
    k_genome_minimizers<<<static_cast<unsigned>(n_tiles), kThreads, 0, st>>>(d_genome, d_tiles, k, w, d_tcount,
                                                                              nullptr, nullptr, nullptr);
  size_t tb = 0;
  if ((e = cub::DeviceScan::ExclusiveSum(nullptr, tb, d_tcount, d_toff, n_tiles + 1, st)) != cudaSuccess)
    return failed("scan", e);
  void* d_tb = tmp.get<uint8_t>(tb, e);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(d_tb, tb, d_tcount, d_toff, n_tiles + 1, st);
  int64_t n_min = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&n_min, d_toff + n_tiles, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return failed("minimizer count", e);
  uint64_t* h_in = tmp.get<uint64_t>(n_min, e);
  uint32_t* v_in = tmp.get<uint32_t>(n_min, e);
  uint64_t* h_out = tmp.get<uint64_t>(n_min, e);
  uint32_t* v_out = nullptr;
  if (e == cudaSuccess && cudaMalloc(&v_out, (n_min ? n_min : 1) * sizeof(uint32_t)) != cudaSuccess) {
    e = cudaErrorMemoryAllocation;
    v_out = nullptr;
  }
  if (e != cudaSuccess) return failed("minimizer buffers", e);
  out->positions = v_out;  // owned by the caller from here on
  out->n_pos = static_cast<uint64_t>(n_min);
  if (n_tiles && n_min)
    k_genome_minimizers<<<static_cast<unsigned>(n_tiles), kThreads, 0, st>>>(d_genome, d_tiles, k, w, nullptr,
                                                                              d_toff, h_in, v_in);
  // 2. stable sort by hash: positions stay ascending within a key
  if (n_min) {
    size_t sb = 0;
    if ((e = cub::DeviceRadixSort::SortPairs(nullptr, sb, h_in, h_out, v_in, v_out, n_min, 0, 2 * k, st)) !=
        cudaSuccess)
      return failed("sort", e);
    void* d_sb = tmp.get<uint8_t>(sb, e);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(d_sb, sb, h_in, h_out, v_in, v_out, n_min, 0, 2 * k, st);
    if (e != cudaSuccess) return failed("sort", e);
  }
  // 3. distinct keys, counts, offsets, largest count
  uint64_t* keys = tmp.get<uint64_t>(n_min, e);
  int32_t* counts = tmp.get<int32_t>(n_min + 1, e);
  int64_t* offs = tmp.get<int64_t>(n_min + 1, e);
  int64_t* d_nkeys = tmp.get<int64_t>(1, e);
  int32_t* d_maxc = tmp.get<int32_t>(1, e);
  if (e != cudaSuccess) return failed("key buffers", e);
  int64_t n_keys = 0;
  int32_t max_count = 0;
  if (n_min) {
    size_t rb = 0;
    if ((e = cub::DeviceRunLengthEncode::Encode(nullptr, rb, h_out, keys, counts, d_nkeys, n_min, st)) != cudaSuccess)
      return failed("distinct keys", e);
    void* d_rb = tmp.get<uint8_t>(rb, e);
    if (e == cudaSuccess) e = cub::DeviceRunLengthEncode::Encode(d_rb, rb, h_out, keys, counts, d_nkeys, n_min, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&n_keys, d_nkeys, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return failed("distinct keys", e);
    // offsets: exclusive scan of the counts (widened to 64 bits)
    size_t xb = 0;
    int64_t* c64 = tmp.get<int64_t>(n_keys, e);
    if (e != cudaSuccess) return failed("offsets", e);
    k_widen<<<blocks_for(n_keys), 256, 0, st>>>(counts, n_keys, c64);
    if ((e = cub::DeviceScan::ExclusiveSum(nullptr, xb, c64, offs, n_keys, st)) != cudaSuccess)
      return failed("offsets", e);
    void* d_xb = tmp.get<uint8_t>(xb, e);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(d_xb, xb, c64, offs, n_keys, st);
    size_t mb = 0;
    if (e == cudaSuccess) e = cub::DeviceReduce::Max(nullptr, mb, counts, d_maxc, n_keys, st);
    void* d_mb = tmp.get<uint8_t>(mb, e);
    if (e == cudaSuccess) e = cub::DeviceReduce::Max(d_mb, mb, counts, d_maxc, n_keys, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&max_count, d_maxc, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return failed("offsets", e);
  }
  // 4. the bucket table
  uint64_t cap = 16;
  while (cap < static_cast<uint64_t>(n_keys) * 2) cap <<= 1;
  uint32_t* slot_rank = tmp.get<uint32_t>(cap, e);
  ulonglong2* table = nullptr;
  if (e == cudaSuccess && cudaMalloc(&table, cap * sizeof(ulonglong2)) != cudaSuccess) {
    e = cudaErrorMemoryAllocation;
    table = nullptr;
  }
  if (e != cudaSuccess) return failed("table", e);
  out->table = table;
  out->n_buckets = cap;
  if ((e = cudaMemsetAsync(slot_rank, 0xFF, cap * sizeof(uint32_t), st)) != cudaSuccess) return failed("table", e);
  if (n_keys) k_place_keys<<<blocks_for(n_keys), 256, 0, st>>>(keys, n_keys, cap - 1, slot_rank, d_err);
  k_fill_table<<<blocks_for(static_cast<int64_t>(cap)), 256, 0, st>>>(slot_rank, cap, keys, offs, counts, table);
  // 5. runs of non-ACGT codes
  {
    const int en = find_n_runs_on_device(st, d_genome, n_bases, &out->n_runs, &out->n_n_runs, err, err_len);
    if (en != DNALN_OK) return en;
  }
  uint32_t h_err = 0;
  if ((e = cudaMemcpyAsync(&h_err, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess)
    return failed("kernels", e);
  if (h_err) {
    snprintf(err, err_len, "index build: a key walked past every bucket (flags 0x%x)", h_err);
    return DNALN_ERR_DEVICE;
  }
  out->n_keys = static_cast<uint64_t>(n_keys);
  out->max_count = static_cast<uint32_t>(max_count);
  out->mask = cap - 1;
  return DNALN_OK;
}

}  // namespace dnb
