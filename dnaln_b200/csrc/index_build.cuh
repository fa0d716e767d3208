// index_build.cuh — MinimizerIndex::build on the device (index_build.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace dnb {

// Device arrays of a built index; the caller owns them (cudaFree) once the build returns
// DNALN_OK, and on failure whichever are non-null.
struct DeviceIndexBuild {
  ulonglong2* table = nullptr;  // n_buckets buckets: .x key (~0 empty), .y offset | count << 32
  uint64_t n_buckets = 0, mask = 0;
  uint32_t* positions = nullptr;  // pos << 1 | strand, grouped by key, ascending within a key
  uint64_t n_pos = 0;
  uint2* n_runs = nullptr;  // maximal runs of non-ACGT codes [x, y), ascending
  int32_t n_n_runs = 0;
  uint64_t n_keys = 0;
  uint32_t max_count = 0;
};

// Builds the index of the resident genome d_genome[0, n_bases) whose contig c is
// [contig_off[c], contig_off[c] + contig_len[c]) (host arrays), on stream st, bucket for
// bucket as src/index.cpp:10-45 builds it. Returns DNALN_OK or a DNALN_ERR_* code with a
// message in err.
int build_index_on_device(cudaStream_t st, const uint8_t* d_genome, uint64_t n_bases, const uint64_t* contig_off,
                          const uint32_t* contig_len, int32_t n_contigs, int k, int w, DeviceIndexBuild* out,
                          char* err, size_t err_len);

// The maximal runs [x, y) of non-ACGT codes (> 3) of the resident genome d_genome[0,
// n_bases), ascending, into a new device array *runs (the caller frees it, also when the
// call fails after setting it); synchronises st. Returns DNALN_OK or a DNALN_ERR_* code.
int find_n_runs_on_device(cudaStream_t st, const uint8_t* d_genome, uint64_t n_bases, uint2** runs, int32_t* n_runs,
                          char* err, size_t err_len);

}  // namespace dnb
