// map.cuh — batch bookkeeping kernels of the mapping pipeline (map.cu).
#pragma once

#include "common.cuh"
#include "seed.cuh"

namespace dnb {

struct MapConsts {
  int32_t max_cand, bw, W, min_aln_score, match;
};

// Counters shared by the bookkeeping kernels: ctr[0] SW cells (qlen * (2bw+1) per task,
// as MapStats::cells), ctr[1] mapped reads, ctr[2] candidate loci.

// Score-only tasks for every candidate of reads with >= 2 candidates
// (src/mapper.cpp:125-133); task slot = r * max_cand + c. *counter += tasks.
void launch_score_tasks(cudaStream_t st, int64_t n, const int64_t* pofs, const int32_t* seq_len, CandBuf cb,
                        const DevIndex& ix, const MapConsts& mc, SwTask* tasks, int* counter,
                        unsigned long long* ctr);

// Choice among a read's candidates (src/mapper.cpp:142-174) and its traceback task
// (slot = r). chosen[r] = candidate index or -1; s2[r] = second-best score.
void launch_choose(cudaStream_t st, int64_t n, const int64_t* pofs, const int32_t* seq_len, CandBuf cb,
                   const SwResult* res_score, const uint32_t* name_hash, const DevIndex& ix, const MapConsts& mc,
                   int32_t* chosen, int32_t* s2, SwTask* tb_tasks, int* tb_counter, unsigned long long* ctr);

// Records + MAPQ (src/mapper.cpp:189-222); cig_count[r] = ops including soft clips.
void launch_records(cudaStream_t st, int64_t n, const int32_t* seq_len, CandBuf cb, const int32_t* chosen,
                    const int32_t* s2, const SwResult* res_tb, const DevIndex& ix, const MapConsts& mc,
                    dnaln_map_record* out, int64_t* cig_count, unsigned long long* ctr);

// Writes each mapped read's CIGAR (leading S, the walk's ops reversed, trailing S) at
// dst + dst_off[r] and sets out[r].cigar_off = rec_base + dst_off[r] and cigar_len; a
// CIGAR that would end past cap ops is not written and sets kErrOutputCapacity.
// cig_src slot of read r is 2 * pofs[r] + r.
void launch_cigar_gather(cudaStream_t st, int64_t n, const int64_t* pofs, const int32_t* seq_len,
                         const SwResult* res_tb, const uint32_t* cig_src, const int64_t* dst_off, int64_t rec_base,
                         dnaln_map_record* out, uint32_t* dst, int64_t cap, uint32_t* err);

// GpuAligner: reversed walk ops of task i (slot i, source cig_src + src_off[i]) to
// dst + dst_off[i]; fills out[i].
void launch_align_gather(cudaStream_t st, int64_t n, const SwResult* res, const uint32_t* cig_src,
                         const int64_t* src_off, const int64_t* dst_off, dnaln_align_result* out, uint32_t* dst);

// ops count per align result -> counts[i] (for the scan of dst offsets)
void launch_align_counts(cudaStream_t st, int64_t n, const SwResult* res, int64_t* counts);

// Length order of SW tasks (tasks of similar length share a thread and a warp): sort keys
// (longest first; slots at or past the device count *n_dev last) and identity values.
void launch_task_keys(cudaStream_t st, const SwTask* tasks, int n_max, const int* n_dev, uint32_t* keys,
                      int32_t* idx);
// out[i] = tasks[order[i]] for i below the device count.
void launch_task_gather(cudaStream_t st, const SwTask* tasks, int n_max, const int* n_dev, const int32_t* order,
                        SwTask* out);

}  // namespace dnb
