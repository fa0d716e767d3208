// sw.cuh — launch interface of the banded SW kernels (sw.cu).
#pragma once

#include "common.cuh"

namespace dnb {

// True when match/mismatch/ambig fit the signed-byte score profile of the PRMT path.
bool sw_bytes_ok(const dnaln_score_params& s);
// True when band width W has a register-resident kernel.
bool sw_band_in_registers(int W);
SwParams make_sw_params(const dnaln_score_params& s);
// Direction-nibble scratch per warp of 32 alignments of at most rows_max query rows.
size_t sw_dir_bytes_per_warp(int W, int rows_max);
// True when band width W with these scores runs the generic (scratch-backed) kernel.
bool sw_uses_generic(int W, bool bytes_ok);
// H/E scratch per warp of the generic kernel (0 when a register kernel runs).
size_t sw_band_bytes_per_warp(int W, bool bytes_ok);

// Aligns tasks[base, base + count) that are below the task count min(n, *n_dev) (n_dev
// may be null; it lets a device-side producer size the batch without a host sync).
// Results go to res[task.slot]; with tb, CIGAR ops (walk order) to cig +
// cig_off[task.slot], capacity 2*qlen+1. base must be a multiple of 32; `dir` must hold
// ceil(count/32) warps of sw_dir_bytes_per_warp(W, rows_max) and `band` as many warps of
// sw_band_bytes_per_warp(W, bytes_ok). Returns false, launching nothing, when a needed
// scratch pointer is null.
bool launch_sw(cudaStream_t st, bool tb, bool bytes_ok, const SwTask* tasks, int base, int count, int n,
               const int* n_dev, const uint8_t* qbase, const uint8_t* tbase, const SwParams& p, SwResult* res,
               uint32_t* dir, int rows_max, uint32_t* cig, const int64_t* cig_off, int* band, uint32_t* err);

}  // namespace dnb
