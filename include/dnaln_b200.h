/* dnaln_b200.h — C ABI of the B200 (sm_100a) read-mapping path.
 *
 * Drop-in boundary for dnaln's hot path: minimizer sketching -> minimizer-index probe ->
 * colinear chaining -> banded Smith-Waterman with traceback. Host code (dnaln's C++
 * mapper, or the C++ mirror in dnaln_b200/host/dnaln_gpu.hpp) calls these functions; all
 * arguments are plain pointers and sizes, host memory unless a name says `device`.
 *
 * Every function returns DNALN_OK (0) or a DNALN_ERR_* code; dnaln_gpu_last_error()
 * gives the message of the last failure on a context. The reference reports errors by
 * die() -> exit(1) (src/common.cpp:55-64); the C++ mirror turns a non-zero status into
 * the same message and exit code.
 *
 * Threading: a context serves one host thread at a time (the reference's Mapper and
 * Aligner are not thread-safe either, src/mapper.hpp:78-93). Use one context per thread.
 *
 * Citations (file:line) are to the dnaln sources each entry point replaces. */
#ifndef DNALN_B200_H
#define DNALN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DNALN_OK 0
#define DNALN_ERR_INVALID_ARG 1  /* bad parameter (same checks as src/cli.hpp:93-95, src/index.cpp:11-12) */
#define DNALN_ERR_CUDA 2         /* a CUDA runtime call failed */
#define DNALN_ERR_OOM 3          /* device or pinned memory exhausted / over the context's budget */
#define DNALN_ERR_CAPACITY 4     /* a caller-sized output is too small; the needed size is returned */
#define DNALN_ERR_NO_DEVICE 5    /* no usable CUDA device */
#define DNALN_ERR_DEVICE 6       /* a kernel reported an internal inconsistency (error flag) */
#define DNALN_ERR_NOT_FOUND 7    /* unknown index id */
#define DNALN_ERR_IO 8           /* an index image file could not be written, read or verified */
#define DNALN_ERR_CANCELLED 9    /* a served request was cancelled (dnaln_serve_cancel) */

typedef struct dnaln_ctx dnaln_ctx;

/* Scoring of the banded SW: match, mismatch, gap open/extension (a gap of length L
 * costs gap_open + L*gap_ext), score of any pair involving N, band half-width.
 * Mirrors ScoreParams (src/align.hpp:34-40). */
typedef struct {
  int32_t match, mismatch, gap_open, gap_ext, ambig, bw;
} dnaln_score_params;

/* Mirrors ChainParams (src/chain.hpp:30-36). */
typedef struct {
  int32_t max_gap, band, lookback, min_score, min_anchors;
} dnaln_chain_params;

/* Mirrors MapParams (src/mapper.hpp:25-35) minus the CPU-only simd/prefetch switches. */
typedef struct {
  int32_t k, w;
  uint32_t max_occ;
  int32_t max_cand;
  double pri_ratio;
  int32_t min_aln_score;
  dnaln_score_params sc;
  dnaln_chain_params ch;
} dnaln_map_params;

/* Mirrors AlignResult (src/align.hpp:49-60); its CIGAR (M/I/D ops, BAM encoding
 * (len << 4) | op) is cigar[cigar_off .. cigar_off + cigar_len) of the call's buffer. */
typedef struct {
  int32_t score, qb, qe, tb, te, nm;
  int64_t cigar_off;
  int32_t cigar_len;
  int32_t pad_;
} dnaln_align_result;

/* Mirrors MapRecord (src/mapper.hpp:37-44). contig = -1 for an unmapped read; pos is the
 * 0-based leftmost aligned position within the contig; the CIGAR (soft clips included)
 * is cigar[cigar_off .. cigar_off + cigar_len). */
typedef struct {
  int64_t pos;
  int64_t cigar_off;
  int32_t contig, score, nm, n_cand;
  int32_t cigar_len;
  uint8_t rev, mapq, pad_[2];
} dnaln_map_record;

/* Per-context counters of the last map/align call and running totals, the device
 * counterpart of MapStats (src/mapper.hpp:46-49). Times are CUDA-event milliseconds
 * measured on the context's stream around each stage. */
typedef struct {
  uint64_t reads, mapped, anchors, candidates, cells, sw_tasks_score, sw_tasks_tb, minimizers;
  double ms_seed;     /* encode + sketch + probe */
  double ms_chain;    /* anchors + chaining + candidates */
  double ms_sw_score; /* score-only SW ranking pass */
  double ms_sw_tb;    /* SW with traceback */
  double ms_post;     /* choose, MAPQ, records, CIGAR compaction */
  double ms_h2d, ms_d2h, ms_total;
  uint64_t launches;  /* kernels of this library launched (library scans excluded) */
  /* reads seeded and chained one warp per read (long reads, or past the per-thread
   * budget), their minimizers, anchors and bases */
  uint64_t warp_reads, warp_minimizers, warp_anchors, warp_bases;
  uint64_t long_reads; /* reads seeded and chained by the long-read thread kernel */
  uint64_t graph_launches; /* batches launched as a captured CUDA graph (running total) */
  uint64_t batch_retries;  /* batches mapped again after the chaining pool grew */
} dnaln_stats;

/* ---- context ---------------------------------------------------------------------- */
const char* dnaln_gpu_version(void);
int dnaln_gpu_ctx_create(int device, dnaln_ctx** out);
int dnaln_gpu_ctx_destroy(dnaln_ctx* ctx);
const char* dnaln_gpu_last_error(const dnaln_ctx* ctx);
/* The CUDA device the context runs on. */
int dnaln_gpu_ctx_device(const dnaln_ctx* ctx, int32_t* device);
/* Launch on `stream` (a cudaStream_t) instead of the context's own stream; NULL restores it. */
int dnaln_gpu_set_stream(dnaln_ctx* ctx, void* stream);
int dnaln_gpu_get_stats(const dnaln_ctx* ctx, dnaln_stats* out);
/* Clears the counters and the kernel-time totals. */
int dnaln_gpu_reset_stats(dnaln_ctx* ctx);

/* Per-kernel timing (no reference counterpart; the reference reports stage totals in
 * MapStats, src/mapper.hpp:46-52). When on, every kernel launch of the context is
 * bracketed by a CUDA event pair on its stream and totals accumulate per kernel name;
 * `only` (may be NULL) restricts the trace to the kernel of that name, so that timing one
 * kernel inside a timed loop adds one event pair per launch of it and nothing else. */
typedef struct dnaln_kernel_time {
  char name[48];
  int64_t launches;
  double ms;
} dnaln_kernel_time;
int dnaln_gpu_set_kernel_trace(dnaln_ctx* ctx, int32_t on, const char* only);
/* Writes min(cap, count) entries; *n_out = count of traced kernel names. */
int dnaln_gpu_kernel_times(const dnaln_ctx* ctx, dnaln_kernel_time* out, int32_t cap, int32_t* n_out);
/* Reads per part of a host-buffer batch (default 0: the whole batch is one part; smaller
 * parts let one synchronous call overlap its own copies, at some kernel efficiency). */
int dnaln_gpu_set_sub_batch(dnaln_ctx* ctx, int64_t reads);
/* Tuning switches (none changes any result):
 *   "sub_batch"      same as dnaln_gpu_set_sub_batch;
 *   "warp_seed_only" 1 = seed and chain every read one warp per read (default 0: short
 *                    reads one thread per read, the others one warp per read);
 *   "graphs"         1 = a batch whose size the host knows (the host-buffer calls) and
 *                    whose launches repeat is captured once as a CUDA graph and replayed
 *                    (default); 0 = launched kernel by kernel;
 *   "sw_form"        banded SW kernel form where a band width has several (W = 33, 65,
 *                    129): 0 = tuned per context (default), 1 = inter-sequence, 2 = intra-
 *                    sequence, 3 = intra-sequence narrow (a form the width lacks falls back
 *                    to the width's first form);
 *   "long_thread"    1 = reads the short thread kernel lists go one thread each through
 *                    the long-read kernel first (default); 0 = straight to the warp kernels;
 *   "length_order"   1 = SW tasks of a batch whose reads differ in length run longest
 *                    first (default); 0 = in read order;
 *   "seed_block"     reads per block of the thread-per-read seeding kernel: 0 = tuned
 *                    (default, dnaln_gpu_seed_tuning), 64 or 128;
 *   "encode_bulk"    1 = the codes of both strands are made in shared memory, tiles of
 *                    back-to-back reads moved in and out by bulk (TMA) copies; 0 = read by
 *                    read from global memory (default: 0.290 against 0.299 ms per 1,000,000
 *                    150-bp reads, 0.52 against 1.49 ms for 50-1000 bp reads);
 *   "work_stealing"  1 = the warp-per-read chaining kernel runs on the resident blocks
 *                    only, each warp taking its next read by an atomic claim (default);
 *                    0 = a fixed grid striding over the reads;
 *   "dir_cap_bytes"  traceback direction-code scratch per launch (default 1/32 of the
 *                    device's memory, at least 1 GiB and at most 8 GiB; a launch whose
 *                    tasks need more is split into chunks);
 *   "chain_pool"     entries of the chaining pool that reads seeded one warp each take
 *                    their anchor scratch from (default 65,536, grown from the batches'
 *                    use): a batch that outgrows the pool is mapped again after the pool
 *                    grows to what it asked for (counted in dnaln_stats.batch_retries);
 * Fault injection on the host (tests of the error paths; changes no result):
 *   "fail_alloc_after" N >= 0: the device allocation after N more succeed fails as if the
 *                    device were out of memory (DNALN_ERR_OOM; the context stays usable,
 *                    and the next call allocates again); -1 = off (default). */
int dnaln_gpu_set_option(dnaln_ctx* ctx, const char* name, int64_t value);
/* The SW kernel-form tuner (no reference counterpart; the reference picks its SIMD lane
 * grouping per task group, src/align_simd.cpp:50-70): band widths with more than one
 * register-resident kernel form — inter-sequence (a thread holds the band rows of two
 * alignments; W = 33, 65 and the other register widths) and intra-sequence (a pair's row
 * spread over lanes in a skewed wavefront: (W - 1) / 32 lanes of 32 cells, or narrow,
 * (W - 1) / 16 lanes of 16 cells; W = 33, 65, 129) — have every form timed on the first
 * batch of each (band width, traceback or score-only, read-length bucket <= 256 / <= 1024
 * / longer) a context maps, and the fastest runs from then on (`tasks` says how large the
 * timed sample was; a sample under 4,096 tasks keeps the width's first form, inter-sequence
 * where it has one). All forms give identical results. ms_* = -1 for a form the width
 * lacks. Writes min(cap, count) entries; *n_out = count. */
typedef struct {
  int32_t W, traceback, len_bucket, form; /* form: 0 inter-sequence, 1 intra-sequence, 2 intra narrow */
  double ms_inter, ms_intra;              /* the timed first chunk */
  int64_t tasks;
  double ms_narrow;
  int32_t lanes_per_pair;                 /* lanes of the chosen form per pair of alignments */
  int32_t pad_;
} dnaln_sw_tuning;
int dnaln_gpu_sw_tuning(const dnaln_ctx* ctx, dnaln_sw_tuning* out, int32_t cap, int32_t* n_out);
/* The reads-per-block tuner of the thread-per-read seeding kernel (no reference
 * counterpart): on the first batch of at least 32,768 reads a context maps (option
 * "seed_block" 0, the default), the kernel runs with 64 and with 128 reads per block, each
 * timed, and the faster size is used from then on. Both give identical results. */
typedef struct {
  int32_t tuned;            /* 0 until a batch was timed */
  int32_t reads_per_block;  /* the size chosen */
  double ms_64, ms_128;     /* the timed runs */
  int64_t reads;            /* the timed batch's reads */
} dnaln_seed_tuning;
int dnaln_gpu_seed_tuning(const dnaln_ctx* ctx, dnaln_seed_tuning* out);
/* Page-locked host buffers for fast transfers (pass to the *_batch calls). */
int dnaln_gpu_host_alloc(dnaln_ctx* ctx, size_t bytes, void** out);
int dnaln_gpu_host_free(dnaln_ctx* ctx, void* p);

/* ---- genome + minimizer index: MinimizerIndex::build (src/index.cpp:10-45) ----------
 * genome: one base code (A0 C1 G2 T3 N4) per byte, contigs concatenated; contig c is
 * [contig_off[c], contig_off[c] + contig_len[c]). The index (hash table of 16-byte
 * buckets + position array, the reference's layout, src/index.hpp:3-9,49-56) and the
 * genome stay resident in HBM until dnaln_gpu_index_free. Requires k in [4, 28], w in
 * [1, 255] and fewer than 2^31 bases (src/index.cpp:11-12, src/reference.cpp:21). */
int dnaln_gpu_index_build(dnaln_ctx* ctx, const uint8_t* genome, uint64_t n_bases, const uint64_t* contig_off,
                          const uint32_t* contig_len, int32_t n_contigs, int32_t k, int32_t w, int32_t* index_id);
/* n_keys, n_positions, max_count, memory_bytes (src/index.hpp:43-46), n_buckets, device bytes */
int dnaln_gpu_index_stats(const dnaln_ctx* ctx, int32_t index_id, uint64_t out6[6]);
/* Copies the resident table (n_buckets keys/offsets/counts) and position array to the host. */
int dnaln_gpu_index_export(dnaln_ctx* ctx, int32_t index_id, uint64_t* keys, uint32_t* offsets, uint32_t* counts,
                           uint32_t* positions);
int dnaln_gpu_index_free(dnaln_ctx* ctx, int32_t index_id);
/* A resident index with its genome as an image file at path: a header (k, w, sizes), the
 * contig table, the genome codes, the bucket table, the positions and the N runs, in the
 * device layout, with a 64-bit checksum of the contents. Written to path + ".tmp" and
 * renamed, so a reader never sees half a file. dnaln_gpu_index_load reads an image back
 * into a new resident index (no rebuild: the serving loop's index admission); the header,
 * every bucket's offset + count, every position and the checksum are checked before the
 * index is usable (DNALN_ERR_IO for a file that does not check out). The reference keeps
 * no index on disk (src/main.cpp:33-35 builds it per run); the image is this library's. */
int dnaln_gpu_index_save(dnaln_ctx* ctx, int32_t index_id, const char* path);
int dnaln_gpu_index_load(dnaln_ctx* ctx, const char* path, int32_t* index_id);
/* A new resident index from a table built on the host in the reference's layout
 * (MinimizerIndex after build, src/index.hpp:49-56): n_buckets (a power of two, at least
 * one bucket empty) buckets of keys (~0 = empty) / offsets / counts into positions[n_pos]
 * (pos << 1 | strand), with the genome and contig table as for dnaln_gpu_index_build.
 * The caller that already holds a MinimizerIndex uploads it instead of rebuilding it.
 * Offsets + counts, positions and the contig table are checked (DNALN_ERR_INVALID_ARG);
 * that the table is the one build() makes for (genome, k, w) is the caller's promise. */
int dnaln_gpu_index_upload(dnaln_ctx* ctx, const uint8_t* genome, uint64_t n_bases, const uint64_t* contig_off,
                           const uint32_t* contig_len, int32_t n_contigs, int32_t k, int32_t w, const uint64_t* keys,
                           const uint32_t* offsets, const uint32_t* counts, uint64_t n_buckets,
                           const uint32_t* positions, uint64_t n_pos, int32_t* index_id);
/* Makes index src_id of context src (same device) usable by context dst under the new id
 * *dst_id, without copying it: several contexts (one per host thread, or the lanes of a
 * server below) map against one resident copy. The memory is freed when the last context
 * holding the index frees it or is destroyed. No reference counterpart: the reference
 * builds one MinimizerIndex per process (src/main.cpp:33-35). */
int dnaln_gpu_index_attach(dnaln_ctx* dst, dnaln_ctx* src, int32_t src_id, int32_t* dst_id);

/* ---- per-stage entry points (batched forms of the reference's per-read calls) ------- */

/* sketch (src/minimizer.hpp:34) over n sequences of base codes: sequence s is
 * codes[seq_off[s] .. + seq_len[s]) and its positions are reported + pos_offset[s]
 * (pos_offset may be NULL = 0). Its minimizers go to out_*[seq_off[s] + j], j <
 * out_count[s] (a sequence never has more minimizers than bases). */
int dnaln_gpu_sketch(dnaln_ctx* ctx, const uint8_t* codes, const int64_t* seq_off, const int32_t* seq_len,
                     const uint32_t* pos_offset, int64_t n, int32_t k, int32_t w, uint64_t* out_hash,
                     uint32_t* out_pos, uint32_t* out_strand, int32_t* out_count);

/* MinimizerIndex::lookup (src/index.hpp:24-38) for n hashes: out_count[i] occurrences at
 * positions[out_offset[i] ..] of the resident index (count 0 = absent). */
int dnaln_gpu_lookup(dnaln_ctx* ctx, int32_t index_id, const uint64_t* hashes, int64_t n, uint32_t* out_offset,
                     uint32_t* out_count);

/* Chainer::run (src/chain.hpp:41) over n_sets anchor sets: set s is anchors
 * [set_off[s], set_off[s+1]) of the rpos/qpos/strand columns, which are sorted in place
 * per set as the reference does. Chains of set s go to out_*[set_off[s] + j],
 * j < out_count[s], in the reference's order (score descending, stable). */
int dnaln_gpu_chain(dnaln_ctx* ctx, uint32_t* rpos, int32_t* qpos, uint32_t* strand, const int64_t* set_off,
                    int64_t n_sets, int32_t k, const dnaln_chain_params* p, int32_t* out_score,
                    uint32_t* out_strand, int32_t* out_n, int64_t* out_dmin, int64_t* out_dmax, uint32_t* out_rpos,
                    int32_t* out_count);

/* Aligner::align (src/align.hpp:62-68): task i aligns query q[q_off[i] .. + q_len[i])
 * against target t[t_off[i] .. + t_len[i]) (N-padded to q_len + 2bw, as
 * src/align.cpp:36-39). With traceback = 0 only score is set. CIGARs go to `cigar`
 * (capacity cigar_cap ops; DNALN_ERR_CAPACITY with *cigar_used = needed if short;
 * sum of 2*q_len+1 always suffices). */
int dnaln_gpu_align(dnaln_ctx* ctx, const uint8_t* q, const int64_t* q_off, const int32_t* q_len, const uint8_t* t,
                    const int64_t* t_off, const int32_t* t_len, int64_t n, int32_t traceback,
                    const dnaln_score_params* sp, dnaln_align_result* out, uint32_t* cigar, int64_t cigar_cap,
                    int64_t* cigar_used);

/* Banded SW for callers that cannot allocate device memory (no counterpart in the
 * reference): a host framework that owns every device allocation, or a serving loop that
 * may not allocate per request. Same results as dnaln_gpu_align, but every buffer is the
 * caller's DEVICE memory and the call allocates nothing: its scratch is one fixed 64 MiB
 * static device array in the library, held by each GPU that loads it until exit.
 * Task i aligns d_q[d_q_off[i] ..+ d_q_len[i]) against d_t[d_t_off[i] ..+ d_t_len[i]);
 * every d_q_len[i] must be <= max_qlen. Its result goes to d_out[i] and, with traceback,
 * its CIGAR to d_cigar[i * cigar_stride ..] (cigar_stride >= 2*max_qlen+1; cigar_off =
 * i * cigar_stride). Launches go to `stream` (a cudaStream_t, NULL = default stream) and
 * the call returns after they finish; the stream must belong to the device current at
 * the call. Returns DNALN_ERR_INVALID_ARG when one warp of tasks of max_qlen rows at this
 * band width does not fit the 64 MiB, and also when a task is found on the device to be
 * described wrongly (a query longer than max_qlen, a negative length or offset): that task
 * is aligned as empty and every other task's result stands. DNALN_ERR_DEVICE means a
 * kernel's own consistency check failed. Each call made outside a stream capture looks up
 * the array's address on the current device (cudaGetSymbolAddress); a call inside a
 * capture uses the address the last uncaptured call on that device found, so the first
 * call on each device should come before any stream capture. All calls share the array:
 * calls that overlap on the GPU race, so serialize them. */
int dnaln_gpu_align_noalloc(const uint8_t* d_q, const int64_t* d_q_off, const int32_t* d_q_len, const uint8_t* d_t,
                            const int64_t* d_t_off, const int32_t* d_t_len, int64_t n, int32_t max_qlen,
                            int32_t traceback, const dnaln_score_params* sp, dnaln_align_result* d_out,
                            uint32_t* d_cigar, int64_t cigar_stride, void* stream);

/* Measured issue rate of the integer instructions the banded SW recurrence is made of (no
 * reference counterpart: the denominator of the SW kernels' integer roofline). Runs, on
 * every SM of `device`, independent chains of 32-bit adds and 16x2 DPX three-way maxima:
 * mode 0 one to one (the recurrence's mix), 1 adds only, 2 maxima only; the best of five
 * timed launches on `stream` (a cudaStream_t, NULL = default stream). *thread_ops_per_s =
 * thread instructions of the mode per second; *best_ms (may be NULL) = that launch's time. */
int dnaln_gpu_int_peak(int32_t device, int32_t mode, void* stream, double* thread_ops_per_s, double* best_ms);

/* ---- whole batch: Mapper::map (src/mapper.cpp:75-223) --------------------------------
 * n reads, ASCII, read r = seq[seq_off[r] .. + seq_len[r]); name_hash[r] = FNV-1a of the
 * read name (src/common.hpp:136-140, dnaln_fnv1a below), the tie-break between equal
 * best candidates. Records go to out[r]; CIGARs to `cigar` (capacity cigar_cap ops;
 * the sum over reads of 2*len+3 always suffices; DNALN_ERR_CAPACITY if it is short).
 * Page-locked buffers (dnaln_gpu_host_alloc) make the copies asynchronous. */
int dnaln_gpu_map_batch(dnaln_ctx* ctx, int32_t index_id, const char* seq, const int64_t* seq_off,
                        const int32_t* seq_len, const uint32_t* name_hash, int64_t n, const dnaln_map_params* p,
                        dnaln_map_record* out, uint32_t* cigar, int64_t cigar_cap, int64_t* cigar_used);
/* The same call split in two (no reference counterpart; a streaming caller's form of
 * Mapper::map): submit queues the batch and returns a ticket at once; a worker thread of
 * the context maps queued batches in order, copying the next batch's reads in and the
 * previous batch's results out while the current one computes. Every buffer of a batch
 * must stay valid and unmodified until dnaln_gpu_map_wait returns for its ticket; wait
 * returns the batch's status and sets *cigar_used. Each ticket is waited for once. Other
 * calls on the context wait until the queue is empty. */
int dnaln_gpu_map_submit(dnaln_ctx* ctx, int32_t index_id, const char* seq, const int64_t* seq_off,
                         const int32_t* seq_len, const uint32_t* name_hash, int64_t n, const dnaln_map_params* p,
                         dnaln_map_record* out, uint32_t* cigar, int64_t cigar_cap, int64_t* cigar_used,
                         int64_t* ticket);
int dnaln_gpu_map_wait(dnaln_ctx* ctx, int64_t ticket);

/* Same pipeline with every buffer already in device memory (no host transfers); the
 * CIGAR count is returned through the host pointer cigar_used. */
int dnaln_gpu_map_batch_device(dnaln_ctx* ctx, int32_t index_id, const char* d_seq, const int64_t* d_seq_off,
                               const int32_t* d_seq_len, const uint32_t* d_name_hash, int64_t n,
                               const dnaln_map_params* p, dnaln_map_record* d_out, uint32_t* d_cigar,
                               int64_t cigar_cap, int64_t* cigar_used);

/* ---- serving: continuous batching over resident indexes -------------------------------
 * No reference counterpart: the reference maps one FASTQ per process against one index
 * (src/main.cpp:33-61). A server keeps the indexes of its home context resident and maps
 * requests (read sets of any size, each against one index) submitted from any number of
 * producer threads. Each of its worker lanes is a context of its own (stream, scratch)
 * sharing the home context's indexes (dnaln_gpu_index_attach). A lane that frees up takes
 * the oldest waiting request and, with coalesce = 1, fills its next batch with the reads
 * of the waiting requests for the same index and parameters in arrival order, splitting
 * large requests across batches; requests that arrive while others are on the GPU join
 * the next batch, and the lanes' batches overlap on the device. A batch takes reads while
 * its estimated device footprint fits the lane's share of the HBM budget. Every request's
 * records and CIGARs are those dnaln_gpu_map_batch gives for it alone (mapping is per
 * read, so batch composition cannot change a result). Lanes do not capture CUDA graphs
 * (option "graphs" 0): batch shapes seldom repeat in serving. */
typedef struct dnaln_server dnaln_server;
typedef struct {
  int32_t lanes;             /* concurrent batches on the device (0 = 3) */
  int32_t coalesce;          /* 1 = requests share batches; 0 = each batch holds one request's reads */
  int64_t max_batch_reads;   /* reads per batch (0 = 262,144) */
  int64_t hbm_budget_bytes;  /* device memory for the batches in flight, all lanes together
                                (0 = free device memory at creation minus 2 GiB) */
} dnaln_serve_params;
typedef struct {
  uint64_t requests, reads, bases, batches;  /* completed since creation or the last reset */
  double p50_ms, p99_ms, max_ms, mean_ms;    /* request latency, submit to completion */
  double mean_batch_reads;
  int64_t max_queue_depth;                   /* requests waiting for a lane, at most */
  int64_t budget_bytes, lane_budget_bytes;
  int32_t lanes, pad_;
  /* lane time, summed over lanes: forming batches, gathering reads into the staging
   * buffers, on the device (copies in, mapping, copies out), scattering results, and
   * completing requests (CIGAR layout) */
  double ms_form, ms_gather, ms_device, ms_scatter, ms_complete;
} dnaln_serve_stats;
int dnaln_serve_create(dnaln_ctx* home, const dnaln_serve_params* sp, dnaln_server** out);
/* Same arguments as dnaln_gpu_map_submit; index_id is an index of the home context. The
 * buffers must stay valid until dnaln_serve_wait returns for *request. */
int dnaln_serve_submit(dnaln_server* s, int32_t index_id, const char* seq, const int64_t* seq_off,
                       const int32_t* seq_len, const uint32_t* name_hash, int64_t n, const dnaln_map_params* p,
                       dnaln_map_record* out, uint32_t* cigar, int64_t cigar_cap, int64_t* cigar_used,
                       int64_t* request);
/* Blocks until the request is complete; returns its status, *latency_ms (may be NULL) =
 * submit-to-completion time. Each request is waited for once. */
int dnaln_serve_wait(dnaln_server* s, int64_t request, double* latency_ms);
/* Cancels a request not yet waited for: none of its reads not yet in a batch is mapped, and
 * once the parts already in a batch have finished, dnaln_serve_wait returns
 * DNALN_ERR_CANCELLED for it (its records are then partial and its CIGAR count 0). Its
 * buffers stay the library's until that wait returns. A request already complete keeps its
 * result (the call returns DNALN_OK and changes nothing). Other requests are not affected. */
int dnaln_serve_cancel(dnaln_server* s, int64_t request);
int dnaln_serve_get_stats(dnaln_server* s, dnaln_serve_stats* out);
int dnaln_serve_reset_stats(dnaln_server* s);
const char* dnaln_serve_last_error(const dnaln_server* s);
/* Finishes every submitted request, then releases the lanes. */
int dnaln_serve_destroy(dnaln_server* s);

/* FNV-1a of a read name (src/common.hpp:136-140), and of n names concatenated in
 * names[name_off[i] .. name_off[i+1]) into out[i]. */
uint32_t dnaln_fnv1a(const char* s, int64_t n);
void dnaln_fnv1a_batch(const char* names, const int64_t* name_off, int64_t n, uint32_t* out);

/* ---- host-side helpers of the mapping path ------------------------------------------ */

/* Mapper::append_sam (src/mapper.cpp:231-270) for n records into out (capacity cap
 * bytes); *used = bytes written (or needed, with DNALN_ERR_CAPACITY). Names and
 * qualities are concatenated with offsets name_off/qual_off (n+1 entries; qual may be
 * NULL for '*'); contig names likewise with cname_off. */
int dnaln_sam_format(const char* seq, const int64_t* seq_off, const int32_t* seq_len, const char* names,
                     const int64_t* name_off, const char* qual, const int64_t* qual_off,
                     const dnaln_map_record* rec, const uint32_t* cigar, int64_t n, const char* cnames,
                     const int64_t* cname_off, char* out, int64_t cap, int64_t* used);

/* dnaln_sam_format on `threads` host threads (0 = all hardware threads): each formats a
 * contiguous range of records, the ranges are concatenated in order; the same bytes. */
int dnaln_sam_format_mt(const char* seq, const int64_t* seq_off, const int32_t* seq_len, const char* names,
                        const int64_t* name_off, const char* qual, const int64_t* qual_off,
                        const dnaln_map_record* rec, const uint32_t* cigar, int64_t n, const char* cnames,
                        const int64_t* cname_off, int32_t threads, char* out, int64_t cap, int64_t* used);

/* SeqReader::next (src/seqio.cpp:59-80) over FASTA/FASTQ text already in memory (gzip
 * decoding stays with the caller): records in the layout the mapping calls take, on
 * `threads` host threads (0 = all) when the text is plain four-line FASTQ, else as the
 * reference reads it, line by line. Malformed FASTQ fails with DNALN_ERR_INVALID_ARG and
 * the reference's message in err (capacity err_cap), where the reference would exit. */
typedef struct dnaln_reads dnaln_reads;
int dnaln_parse_reads(const char* text, int64_t len, int32_t threads, dnaln_reads** out, char* err, int64_t err_cap);
/* Views of a parse: n records; sequences, names and qualities concatenated with n + 1
 * offsets each (qual NULL when no record is FASTQ); name_hash[i] = FNV-1a of name i. Valid
 * until dnaln_reads_free. */
int dnaln_reads_view(const dnaln_reads* r, int64_t* n, const char** seq, const int64_t** seq_off,
                     const int32_t** seq_len, const char** names, const int64_t** name_off, const char** qual,
                     const int64_t** qual_off, const uint32_t** name_hash);
void dnaln_reads_free(dnaln_reads* r);

/* The accuracy gate, Evaluator::add (src/evaluate.cpp:57-84) over n records against the
 * simulator's truth (contig index, 0-based start, strand): a mapped record is placed
 * correctly when contig and strand match and its unclipped start (pos minus a leading
 * S/H clip) is within tol of the true start (the reference's default tol is 10); mapped
 * and wrong records are also counted per MAPQ, clamped to [0, 60]. */
typedef struct {
  uint64_t records, mapped, correct;
  uint64_t mapped_at_mapq[61], wrong_at_mapq[61];
} dnaln_eval_counts;
int dnaln_eval_records(const dnaln_map_record* rec, const uint32_t* cigar, const int32_t* truth_contig,
                       const int64_t* truth_start, const uint8_t* truth_rev, int64_t n, int32_t tol,
                       dnaln_eval_counts* out);

#ifdef __cplusplus
}
#endif
#endif
