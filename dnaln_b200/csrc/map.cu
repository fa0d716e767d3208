// map.cu — per-read bookkeeping between the pipeline's compute stages: building SW
// tasks from candidate loci, choosing among equally scored candidates, MAPQ and the
// final records with their soft-clipped CIGARs. One thread per read; all integer except
// MAPQ, which is evaluated in FP64 with explicitly rounded operations in the
// reference's operation order (src/mapper.cpp:217-218).
#include "map.cuh"

namespace dnb {

namespace {

constexpr int kThreads = 256;

// SW task of candidate c of read r: query = forward or reverse-complement codes, target
// window = genome[wstart, wstart + len + 2bw) with N outside the candidate's contig
// (src/mapper.cpp:100-121, src/reference.cpp:34-47).
__device__ __forceinline__ SwTask cand_task(int64_t r, int c, const int64_t* pofs, const int32_t* seq_len,
                                            const CandBuf& cb, const DevIndex& ix, const MapConsts& mc) {
  const int64_t ci = r * mc.max_cand + c;
  const int len = seq_len[r];
  const int ctg = cb.contig[ci];
  const int64_t ws = cb.wstart[ci];
  const int64_t cb0 = static_cast<int64_t>(ix.contig_off[ctg]), ce = cb0 + ix.contig_len[ctg];
  const int64_t we = ws + len + 2 * static_cast<int64_t>(mc.bw);
  SwTask t;
  t.q_off = 2 * pofs[r] + (cb.rev[ci] ? len : 0);
  t.qlen = len;
  t.t_start = ws;
  t.t_lo = ws > cb0 ? ws : cb0;
  t.t_hi = we < ce ? we : ce;
  t.slot = 0;
  // the whole window inside the contig and clear of the genome's N runs: no N to score
  t.flags = (t.t_lo == ws && t.t_hi == we && !genome_has_n(ix, ws, we)) ? kTaskNoN : 0;
  t.pad_ = 0;
  return t;
}

__global__ void k_score_tasks(int64_t n, const int64_t* __restrict__ pofs, const int32_t* __restrict__ seq_len,
                              CandBuf cb, DevIndex ix, MapConsts mc, SwTask* __restrict__ tasks,
                              int* __restrict__ counter, unsigned long long* __restrict__ ctr) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int nc = r < n ? cb.n_cand[r] : 0;
  const int want = nc >= 2 ? nc : 0;
  // warp-aggregated slot reservation
  const unsigned lane = threadIdx.x & 31;
  int total;
  const int ex = warp_exclusive_scan(want, &total);
  int base = 0;
  if (lane == 0 && total) base = atomicAdd(counter, total);
  base = __shfl_sync(0xffffffffu, base, 0);
  for (int c = 0; c < want; ++c) {
    SwTask t = cand_task(r, c, pofs, seq_len, cb, ix, mc);
    t.slot = static_cast<int32_t>(r * mc.max_cand + c);
    tasks[base + ex + c] = t;
  }
  // cells of the ranking pass, counted as the reference's MapStats::cells (src/mapper.cpp:139)
  unsigned long long cells = want ? static_cast<unsigned long long>(want) * seq_len[r] * mc.W : 0ull;
  cells = warp_sum(cells);
  if (lane == 0 && cells) atomicAdd(ctr, cells);
}

__global__ void k_choose(int64_t n, const int64_t* __restrict__ pofs, const int32_t* __restrict__ seq_len, CandBuf cb,
                         const SwResult* __restrict__ res_score, const uint32_t* __restrict__ name_hash, DevIndex ix,
                         MapConsts mc, int32_t* __restrict__ chosen, int32_t* __restrict__ s2o,
                         SwTask* __restrict__ tb_tasks, int* __restrict__ tb_counter,
                         unsigned long long* __restrict__ ctr) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  int pick_c = -1, s2 = 0, nc = 0;
  if (r < n) {
    nc = cb.n_cand[r];
    if (nc == 1) {
      pick_c = 0;
    } else if (nc >= 2) {
      const SwResult* rs = res_score + r * mc.max_cand;
      int s1 = -1, ties = 0;
      for (int c = 0; c < nc; ++c) {
        const int sw = rs[c].score;
        if (sw > s1) {
          s1 = sw;
          ties = 1;
        } else if (sw == s1) {
          ++ties;
        }
      }
      if (ties > 1) {
        s2 = s1;
      } else {
        for (int c = 0; c < nc; ++c)
          if (rs[c].score != s1 && rs[c].score > s2) s2 = rs[c].score;
      }
      uint32_t pick = name_hash[r] % static_cast<uint32_t>(ties);
      for (int c = 0; c < nc; ++c)
        if (rs[c].score == s1 && pick-- == 0) {
          pick_c = c;
          break;
        }
    }
    chosen[r] = pick_c;
    s2o[r] = s2;
  }
  const unsigned lane = threadIdx.x & 31;
  const unsigned ball = __ballot_sync(0xffffffffu, pick_c >= 0);
  int base = 0;
  if (lane == 0 && ball) base = atomicAdd(tb_counter, __popc(ball));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (pick_c >= 0) {
    SwTask t = cand_task(r, pick_c, pofs, seq_len, cb, ix, mc);
    t.slot = static_cast<int32_t>(r);
    tb_tasks[base + __popc(ball & ((1u << lane) - 1u))] = t;
  }
  // traceback cells (src/mapper.cpp:186) and candidate count
  unsigned long long cells = pick_c >= 0 ? static_cast<unsigned long long>(seq_len[r]) * mc.W : 0ull;
  unsigned long long cands = static_cast<unsigned long long>(nc);
  cells = warp_sum(cells);
  cands = warp_sum(cands);
  if (lane == 0) {
    if (cells) atomicAdd(ctr, cells);
    if (cands) atomicAdd(ctr + 2, cands);
  }
}

__global__ void k_records(int64_t n, const int32_t* __restrict__ seq_len, CandBuf cb,
                          const int32_t* __restrict__ chosen, const int32_t* __restrict__ s2o,
                          const SwResult* __restrict__ res_tb, DevIndex ix, MapConsts mc,
                          dnaln_map_record* __restrict__ out, int64_t* __restrict__ cig_count,
                          unsigned long long* __restrict__ ctr) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const unsigned ball = __ballot_sync(0xffffffffu, r < n && chosen[r < n ? r : 0] >= 0 &&
                                                       res_tb[r < n ? r : 0].score >= mc.min_aln_score);
  if ((threadIdx.x & 31) == 0 && ball) atomicAdd(ctr + 1, static_cast<unsigned long long>(__popc(ball)));
  if (r > n) return;
  if (r == n) {  // trailing element of the scan input
    cig_count[n] = 0;
    return;
  }
  dnaln_map_record m;
  m.pos = 0;
  m.cigar_off = 0;
  m.contig = -1;
  m.score = 0;
  m.nm = 0;
  m.n_cand = cb.n_cand[r];
  m.cigar_len = 0;
  m.rev = 0;
  m.mapq = 0;
  m.pad_[0] = m.pad_[1] = 0;
  int64_t ops = 0;
  const int c = chosen[r];
  if (c >= 0) {
    const SwResult a = res_tb[r];
    if (a.score >= mc.min_aln_score) {
      const int64_t ci = r * mc.max_cand + c;
      const int ctg = cb.contig[ci];
      m.contig = ctg;
      m.rev = cb.rev[ci];
      m.pos = cb.wstart[ci] + a.tb - static_cast<int64_t>(ix.contig_off[ctg]);
      m.score = a.score;
      m.nm = a.nm;
      if (m.n_cand <= 1) {
        m.mapq = 60;
      } else {
        const int s2 = s2o[r];
        double q = 0.0;
        if (s2 < a.score)
          q = __dadd_rn(__ddiv_rn(__dmul_rn(6.02, static_cast<double>(a.score - s2)), static_cast<double>(mc.match)),
                        0.499);
        m.mapq = static_cast<uint8_t>(static_cast<int>(q < 60.0 ? q : 60.0));
      }
      ops = (a.qb > 0 ? 1 : 0) + a.n_ops + (seq_len[r] > a.qe ? 1 : 0);
    }
  }
  out[r] = m;
  cig_count[r] = ops;
}

__global__ void k_cigar_gather(int64_t n, const int64_t* __restrict__ pofs, const int32_t* __restrict__ seq_len,
                               const SwResult* __restrict__ res_tb, const uint32_t* __restrict__ cig_src,
                               const int64_t* __restrict__ dst_off, int64_t rec_base, dnaln_map_record* __restrict__ out,
                               uint32_t* __restrict__ dst, int64_t cap, uint32_t* __restrict__ err) {
  const int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t o = dst_off[r], cnt = dst_off[r + 1] - o;
  out[r].cigar_off = rec_base + o;
  out[r].cigar_len = static_cast<int32_t>(cnt);
  if (cnt == 0) return;
  if (o + cnt > cap) {  // the caller's buffer is too small: the call reports the size it needs
    atomicOr(err, kErrOutputCapacity);
    return;
  }
  const SwResult a = res_tb[r];
  const uint32_t* src = cig_src + 2 * pofs[r] + r;
  int64_t x = o;
  if (a.qb > 0) dst[x++] = static_cast<uint32_t>(a.qb) << 4 | 4u;  // S
  for (int i = a.n_ops - 1; i >= 0; --i) dst[x++] = src[i];
  if (seq_len[r] > a.qe) dst[x++] = static_cast<uint32_t>(seq_len[r] - a.qe) << 4 | 4u;
}

__global__ void k_align_counts(int64_t n, const SwResult* __restrict__ res, int64_t* __restrict__ counts) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) counts[i] = res[i].n_ops;
  if (i == n) counts[n] = 0;
}

__global__ void k_align_gather(int64_t n, const SwResult* __restrict__ res, const uint32_t* __restrict__ cig_src,
                               const int64_t* __restrict__ src_off, const int64_t* __restrict__ dst_off,
                               dnaln_align_result* __restrict__ out, uint32_t* __restrict__ dst) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SwResult a = res[i];
  dnaln_align_result o;
  o.score = a.score;
  o.qb = a.qb;
  o.qe = a.qe;
  o.tb = a.tb;
  o.te = a.te;
  o.nm = a.nm;
  o.cigar_off = dst_off[i];
  o.cigar_len = a.n_ops;
  o.pad_ = 0;
  out[i] = o;
  const uint32_t* src = cig_src + src_off[i];
  for (int k = 0; k < a.n_ops; ++k) dst[o.cigar_off + k] = src[a.n_ops - 1 - k];
}

inline unsigned blocks_for(int64_t n) { return static_cast<unsigned>((n + kThreads - 1) / kThreads); }

}  // namespace

void launch_score_tasks(cudaStream_t st, int64_t n, const int64_t* pofs, const int32_t* seq_len, CandBuf cb,
                        const DevIndex& ix, const MapConsts& mc, SwTask* tasks, int* counter,
                        unsigned long long* ctr) {
  if (n > 0) k_score_tasks<<<blocks_for(n), kThreads, 0, st>>>(n, pofs, seq_len, cb, ix, mc, tasks, counter, ctr);
}

void launch_choose(cudaStream_t st, int64_t n, const int64_t* pofs, const int32_t* seq_len, CandBuf cb,
                   const SwResult* res_score, const uint32_t* name_hash, const DevIndex& ix, const MapConsts& mc,
                   int32_t* chosen, int32_t* s2, SwTask* tb_tasks, int* tb_counter, unsigned long long* ctr) {
  if (n > 0)
    k_choose<<<blocks_for(n), kThreads, 0, st>>>(n, pofs, seq_len, cb, res_score, name_hash, ix, mc, chosen, s2,
                                                 tb_tasks, tb_counter, ctr);
}

void launch_records(cudaStream_t st, int64_t n, const int32_t* seq_len, CandBuf cb, const int32_t* chosen,
                    const int32_t* s2, const SwResult* res_tb, const DevIndex& ix, const MapConsts& mc,
                    dnaln_map_record* out, int64_t* cig_count, unsigned long long* ctr) {
  k_records<<<blocks_for(n + 1), kThreads, 0, st>>>(n, seq_len, cb, chosen, s2, res_tb, ix, mc, out, cig_count, ctr);
}

void launch_cigar_gather(cudaStream_t st, int64_t n, const int64_t* pofs, const int32_t* seq_len,
                         const SwResult* res_tb, const uint32_t* cig_src, const int64_t* dst_off, int64_t rec_base,
                         dnaln_map_record* out, uint32_t* dst, int64_t cap, uint32_t* err) {
  if (n <= 0) return;
  k_cigar_gather<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(n, pofs, seq_len, res_tb, cig_src, dst_off,
                                                                         rec_base, out, dst, cap, err);
}

void launch_align_counts(cudaStream_t st, int64_t n, const SwResult* res, int64_t* counts) {
  k_align_counts<<<blocks_for(n + 1), kThreads, 0, st>>>(n, res, counts);
}

void launch_align_gather(cudaStream_t st, int64_t n, const SwResult* res, const uint32_t* cig_src,
                         const int64_t* src_off, const int64_t* dst_off, dnaln_align_result* out, uint32_t* dst) {
  if (n > 0) k_align_gather<<<blocks_for(n), kThreads, 0, st>>>(n, res, cig_src, src_off, dst_off, out, dst);
}

namespace {

__global__ void k_task_keys(const SwTask* __restrict__ tasks, int n_max, const int* __restrict__ n_dev,
                            uint32_t* __restrict__ keys, int32_t* __restrict__ idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_max) return;
  const int n = n_dev ? min(n_max, *n_dev) : n_max;
  const int ql = i < n ? min(tasks[i].qlen, 0xFFFF) : 0;
  keys[i] = i < n ? 0xFFFFu - static_cast<uint32_t>(ql) : 0x10000u;  // longest first, unused slots last
  idx[i] = i;
}

__global__ void k_task_gather(const SwTask* __restrict__ tasks, int n_max, const int* __restrict__ n_dev,
                              const int32_t* __restrict__ order, SwTask* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = n_dev ? min(n_max, *n_dev) : n_max;
  if (i < n) out[i] = tasks[order[i]];
}

}  // namespace

void launch_task_keys(cudaStream_t st, const SwTask* tasks, int n_max, const int* n_dev, uint32_t* keys,
                      int32_t* idx) {
  if (n_max > 0) k_task_keys<<<blocks_for(n_max), kThreads, 0, st>>>(tasks, n_max, n_dev, keys, idx);
}

void launch_task_gather(cudaStream_t st, const SwTask* tasks, int n_max, const int* n_dev, const int32_t* order,
                        SwTask* out) {
  if (n_max > 0) k_task_gather<<<blocks_for(n_max), kThreads, 0, st>>>(tasks, n_max, n_dev, order, out);
}

}  // namespace dnb
