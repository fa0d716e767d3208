// sw.cuh — launch interface of the banded SW kernels (sw.cu).
#pragma once

#include "common.cuh"

namespace dnb {

// Scratch is laid out per group of kSwTaskGroup consecutive tasks (one warp of the
// two-alignments-per-thread kernel); launch bases are multiples of it.
constexpr int kSwTaskGroup = 64;

// True when match/mismatch/ambig fit the signed-byte substitution profile.
bool sw_bytes_ok(const dnaln_score_params& s);
// True when band width W has a register-resident kernel.
bool sw_band_in_registers(int W);
// True when band width W with these scores runs the generic (scratch-backed) kernel.
bool sw_uses_generic(int W, bool bytes_ok);
SwParams make_sw_params(const dnaln_score_params& s);
// Direction-code scratch per task of at most rows_max query rows.
size_t sw_dir_bytes_per_task(int W, int rows_max);
// Band-row scratch per task of the generic kernel (0 when a register kernel runs).
size_t sw_band_bytes_per_task(int W, bool bytes_ok);

// Kernels one launch_sw call issues (for launch accounting).
int sw_launches(int W, bool bytes_ok, bool tb);

// Kernel forms of the register-resident bands, all with the same results: inter-sequence
// (k_sw_u2, a thread holds the whole band row of two alignments; W != 129) and intra-
// sequence (k_sw_wide, the row of a pair spread over lanes in a skewed wavefront: (W - 1) /
// 32 lanes of 32 cells, or, narrow, (W - 1) / 16 lanes of 16 cells; W = 33, 65, 129). The
// generic kernel (other widths or scores) has the inter form only.
enum SwForm : int { kSwInter = 0, kSwIntra = 1, kSwIntraNarrow = 2 };
constexpr int kSwForms = 3;
bool sw_has_form(int W, bool bytes_ok, SwForm form);
int sw_lanes_per_pair(int W, SwForm form);

// Aligns tasks[base, base + count) that are below the task count min(n, *n_dev) (n_dev
// may be null; it lets a device-side producer size the batch without a host sync).
// Results go to res[task.slot]; with tb, CIGAR ops (walk order) to cig +
// cig_off[task.slot], capacity 2*qlen+1. base must be a multiple of kSwTaskGroup; `dir`
// and `band` must hold count rounded up to kSwTaskGroup tasks of
// sw_dir_bytes_per_task(W, rows_max) and sw_band_bytes_per_task(W, bytes_ok); `fb`
// (count + 1 ints) lists the tasks the 16-bit kernel hands to the int32 one; kt (may be
// null) times each kernel. Returns false, launching nothing, when a needed scratch pointer
// is null or base is misaligned.
bool launch_sw(cudaStream_t st, bool tb, bool bytes_ok, const SwTask* tasks, int base, int count, int n,
               const int* n_dev, const uint8_t* qbase, const uint8_t* tbase, const SwParams& p, SwResult* res,
               uint32_t* dir, int rows_max, uint32_t* cig, const int64_t* cig_off, int* band, int* fb,
               uint32_t* err, const KernelTrace* kt, SwForm form = kSwInter);

}  // namespace dnb
