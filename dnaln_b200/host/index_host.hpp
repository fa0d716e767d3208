// index_host.hpp — host construction of the resident minimizer index (index_host.cpp).
#pragma once

#include <cstdint>
#include <vector>

namespace dnb {

struct HostIndex {
  std::vector<uint64_t> keys;  // n_buckets, ~0 = empty
  std::vector<uint32_t> offs, cnts, pos;
  uint64_t mask = 0, n_keys = 0;
  uint32_t max_count = 0;
  int k = 0, w = 0;
};

bool build_index_host(const uint8_t* genome, const uint64_t* contig_off, const uint32_t* contig_len,
                      int32_t n_contigs, int k, int w, HostIndex& ix);

}  // namespace dnb
