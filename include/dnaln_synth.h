/* dnaln_synth.h — seeded synthetic genomes and reads for the mapping workloads.
 *
 * No counterpart on the reference's mapping path: the closest reference code is its test
 * simulator (src/simulate.cpp:26-152), whose error model and genome differ from the
 * workloads measured here (repeat families, indel cap 8, start range). This generator
 * produces exactly the workloads' inputs from a seed, with the reference's RNG family
 * (xoshiro256** seeded by splitmix64, src/common.hpp:80-107). */
#ifndef DNALN_SYNTH_H
#define DNALN_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t n_contigs;
  uint32_t contig_len;
  double gc;              /* P(G) = P(C) = gc/2, P(A) = P(T) = (1-gc)/2 */
  int32_t n_repeat_units; /* distinct repeat units (0 = none) */
  int32_t repeat_unit_len;
  double repeat_frac;     /* fraction of the genome overwritten by unit copies */
  double repeat_div;      /* per-copy substitution rate */
  double n_frac;          /* fraction of bases in N runs */
  int32_t n_run_min, n_run_max;
} dnaln_synth_genome_spec;

typedef struct {
  int64_t n_reads;
  int32_t len_min, len_max;
  int32_t len_dist;     /* 0: fixed len_min, 1: log-uniform [min, max], 2: uniform [min, max] */
  double sub;           /* per-base substitution rate (to one of the other 3 bases) */
  double indel;         /* per-base indel rate, half insertions, half deletions */
  double indel_geom_p;  /* indel length ~ geometric(p), capped at indel_cap */
  int32_t indel_cap;
  double big_del_frac;  /* fraction of reads carrying one long deletion ... */
  int32_t big_del_min, big_del_max; /* ... of this length range */
  int64_t name_base;    /* read i is named sim_<name_base + i> */
} dnaln_synth_reads_spec;

/* Writes n_contigs * contig_len base codes (A0 C1 G2 T3 N4). */
int dnaln_synth_genome(uint64_t seed, const dnaln_synth_genome_spec* spec, uint8_t* out_codes);

/* Upper bound of the ASCII bytes of a read set (sum of lengths). */
int64_t dnaln_synth_reads_bytes(uint64_t seed, const dnaln_synth_reads_spec* spec);

/* Reads as ASCII (read i = out_seq[out_seq_off[i] .. out_seq_off[i+1])), names likewise,
 * and the truth: contig, 0-based start within the contig (forward strand), strand. */
int dnaln_synth_reads(uint64_t seed, const uint8_t* genome, const uint64_t* contig_off, const uint32_t* contig_len,
                      int32_t n_contigs, const dnaln_synth_reads_spec* spec, char* out_seq, int64_t seq_cap,
                      int64_t* out_seq_off, char* out_names, int64_t names_cap, int64_t* out_name_off,
                      int32_t* truth_contig, int64_t* truth_start, uint8_t* truth_rev);

#ifdef __cplusplus
}
#endif
#endif
