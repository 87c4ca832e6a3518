/*
 * uc.h — C ABI of the B200 unitig compactor (libuc.so).
 *
 * The reference (euphoricpoptarts/UnitigCoarsening) has no library interface:
 * its driver calls C++ functions that take Kokkos views.  Each entry point
 * below replaces one of those calls with plain pointers and sizes; the
 * comment names the reference function (file:line) it stands in for.
 *
 * Conventions
 *  - Every call returns uc_status; uc_last_error(ctx) gives a one-line reason.
 *  - "d_" pointers are device pointers on the context's device; every call is
 *    enqueued on the context's stream (uc_ctx_set_stream to share a stream
 *    with the caller) and returns after the work is enqueued unless it has to
 *    read a size back, in which case it synchronizes that stream.
 *  - Packed k-mers ("keys") use the reference's bit layout (driver.cpp:236-246:
 *    char x at bits 2x, A=0 C=1 G=2 T=3, any other byte packs as A) stored in
 *    64-bit words: one word per k-mer for k <= 31, two for 32 <= k <= 63.
 *  - Vertex ids are input line numbers (0-based); UC_NONE marks "no vertex".
 *  - A context is not thread safe; use one context per host thread.
 */
#ifndef UC_H
#define UC_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UC_NONE 0xFFFFFFFFu

typedef enum uc_status {
    UC_OK = 0,
    UC_EINPUT = 1,     /* malformed text, count mismatch, k or l out of range */
    UC_ENOMEM = 2,     /* a device or host allocation failed */
    UC_EBUDGET = 3,    /* the job does not fit the context's HBM budget */
    UC_ETIMEOUT = 4,   /* a bounded device wait ran out */
    UC_EINTERNAL = 5,  /* an internal bound or invariant failed */
    UC_ECUDA = 6,      /* a CUDA runtime call failed */
    UC_EBUSY = 7       /* job not finished (uc_job_result before completion) */
} uc_status;

/* Contraction strategies for uc_contract / the stitch step. */
enum { UC_CONTRACT_POINTER_JUMP = 0, UC_CONTRACT_HEC = 1 };

typedef struct uc_ctx uc_ctx;
typedef struct uc_job uc_job;

/* Per-run counters and phase times (milliseconds, CUDA events). */
typedef struct uc_stats {
    uint64_t n_kmers, n_copies, n_cross, n_tiles, n_big_tiles;
    uint64_t n_segments, n_unitigs, n_cycles, out_bytes;
    uint64_t closed_bytes, seg_chars; /* written by the tile kernels: lines, segment chars */
    uint32_t l_used, bucket_bits, tile_capacity, stitch_rounds, launches, graph_nodes;
    float ms_pack, ms_bucket, ms_tiles, ms_stitch, ms_total;
    float ms_tile_warp, ms_tile_block; /* the warp- and block-tile kernels */
} uc_stats;

/* Tuning knobs (0 = automatic).  Filled by the autotuner or by hand. */
typedef struct uc_tuning {
    uint32_t tile_capacity;   /* copies per shared-memory tile (max 8192) */
    uint32_t tile_threads;    /* threads per tile CTA (256 or 512) */
    uint32_t bucket_bits;     /* log2 of the bucket count */
    uint32_t load_factor_pct; /* tile hash slots per 100 copies (150..800; 200) */
    uint32_t contract_method; /* UC_CONTRACT_* for the segment stitch */
    uint32_t warp_capacity;   /* copies per warp tile (32..1024; 1 = no warp tier) */
    uint32_t bucket_fill;     /* buckets per tile when bucket_bits is 0 (1..64; 8) */
} uc_tuning;

/* ---- context --------------------------------------------------------- */

/* Replaces Kokkos::initialize (driver.cpp:433).  hbm_budget 0 = 90% of free. */
uc_status uc_ctx_create(int device, size_t hbm_budget, uc_ctx **out);
uc_status uc_ctx_destroy(uc_ctx *ctx);
uc_status uc_ctx_set_stream(uc_ctx *ctx, void *cuda_stream);
uc_status uc_ctx_sync(uc_ctx *ctx);
/* Deterministic output: with on != 0, uc_compact_device, uc_compact_host,
 * uc_job_* and uc_compact_file leave the lines in byte order, so equal input
 * gives byte-equal output.  The reference appends lines in an order that
 * varies from run to run (compact.h:7-37); sorting costs one radix sort of
 * the lines by their first k-mer and one copy of the output.  Batches
 * (uc_compact_batch) are not reordered. */
uc_status uc_ctx_set_sorted_output(uc_ctx *ctx, int on);
uc_status uc_ctx_set_tuning(uc_ctx *ctx, const uc_tuning *t);
uc_status uc_ctx_get_tuning(const uc_ctx *ctx, uc_tuning *t);
/* Host jobs larger than the device.  The reference runs jobs up to host
 * memory by moving its 64 minimizer buckets to the device one at a time
 * (driver.cpp:479-521, README.md:6-7).  uc_compact_host, uc_job_submit and
 * uc_compact_file instead stream: the text goes to the device in chunks of
 * chunk_lines lines, twice (bucket counts, then the bucketed copies), the
 * tiles run in groups of about group_copies copies whose lines return to
 * host memory group by group, and the cross-tile lines follow; the device
 * holds one chunk, the copies of all k-mers and the segment arrays, so a
 * job of several billion k-mers (64-bit k-mer indices) runs on one B200.
 * mode UC_STREAM_AUTO (the default) streams a job whose resident run does
 * not fit the budget; UC_STREAM_ALWAYS streams every host job;
 * UC_STREAM_NEVER never does.  Streaming needs k chars + '\n' per line and
 * unsorted output.  0 for chunk_lines / group_copies = defaults (2^26
 * lines, 2^28 copies). */
enum { UC_STREAM_AUTO = 0, UC_STREAM_ALWAYS = 1, UC_STREAM_NEVER = 2 };
uc_status uc_ctx_set_streaming(uc_ctx *ctx, int mode, uint64_t chunk_lines,
                               uint64_t group_copies);

/* Failure injection for tests of the error paths; no counterpart in the
 * reference, whose only error handling is exit(1) on a file it cannot open
 * (driver.cpp:262-265, compact.h:12-15).  All zeros (the default) = off.
 *  - fail_alloc_after: the n-th device allocation this context makes from
 *    now on fails as out of memory (1 = the next one); the call returns
 *    UC_ENOMEM and the context stays usable.
 *  - hec_round_cap: at most this many HEC matching rounds (0 = enough for
 *    any list).  The device reports rounds that ran out with lists still
 *    open (the bounded wait of the contraction).
 *  - hec_strict: when the HEC rounds run out, fail with UC_ETIMEOUT instead
 *    of finishing the lists by pointer jumping.
 *  - walk_cap: the line walk of the stitch follows at most this many
 *    segments after a line's head (0 = 1024); longer lines go through list
 *    ranking, so a small cap sends small jobs down that path. */
typedef struct uc_faults {
    uint32_t fail_alloc_after;
    uint32_t hec_round_cap;
    uint32_t hec_strict;
    uint32_t walk_cap;
} uc_faults;
uc_status uc_ctx_set_faults(uc_ctx *ctx, const uc_faults *f);
const char *uc_last_error(const uc_ctx *ctx);
const char *uc_status_str(uc_status s);

/* ---- phases (device memory) ------------------------------------------ */

/* Header line of the k-mer text: the count n and the offset of the first
 * k-mer line.  load_kmers header parse, driver.cpp:296-304. */
uc_status uc_parse_header(uc_ctx *ctx, const char *d_text, size_t bytes,
                          uint64_t *n, uint64_t *body_offset);

/* Text -> packed keys (n * words).  load_kmers line parse + compact_kmers,
 * driver.cpp:257-354 and 227-249.  Fails with UC_EINPUT on a line shorter
 * than k or a count that disagrees with the number of lines. */
uc_status uc_pack(uc_ctx *ctx, const char *d_text, size_t bytes, int k,
                  uint64_t *d_keys, uint64_t *n_out);

/* Prefix/suffix L-minimizer priorities per k-mer.  get_double_lmin,
 * lmin_buckets.h:67-94, with the l-mer priority table of
 * generate_permutation (driver.cpp:356-402) replaced by a seeded bijection of
 * [0, 4^l); d_table (4^l entries) overrides it when not NULL. */
uc_status uc_minimizers(uc_ctx *ctx, const uint64_t *d_keys, uint64_t n,
                        int k, int l, uint64_t seed, const uint32_t *d_table,
                        uint32_t *d_l1, uint32_t *d_l2);

/* Bucketed edge finding: succ[u] = v iff v is u's only (k-1)-overlap
 * successor and u is v's only predecessor; pred is the inverse.
 * find_l_minimizer (lmin_buckets.h:288-433) + generate_hashmap
 * (assembler.h:120-150) + assemble_pruned_graph (assembler.h:164-214). */
uc_status uc_find_edges(uc_ctx *ctx, const uint64_t *d_keys, uint64_t n,
                        int k, int l, uint64_t seed, uint32_t *d_succ,
                        uint32_t *d_pred);

/* Path contraction: head[v] = first vertex of v's unitig, rank[v] = its
 * position (cycles start at their smallest key).  Replaces the round loop
 * coarsen_de_bruijn_full_cycle (coarseners.h:437-485) with its HEC matching
 * (heuristics.h:205-256) and member ordering (coarseners.h:182-235,
 * compact_graph.h:55-112).  method: UC_CONTRACT_*. */
uc_status uc_contract(uc_ctx *ctx, const uint64_t *d_keys,
                      const uint32_t *d_succ, const uint32_t *d_pred,
                      uint64_t n, int k, int method, uint32_t *d_head,
                      uint32_t *d_rank, uint64_t *n_cycles);

/* Unitig lines (first k-mer in full, then the last char of each later
 * k-mer, '\n'), ordered by head id.  write_intra_bucket_outputs,
 * compact.h:161-210.  d_out may be NULL to only size. */
uc_status uc_emit(uc_ctx *ctx, const uint64_t *d_keys, const uint32_t *d_succ,
                  const uint32_t *d_head, const uint32_t *d_rank, uint64_t n,
                  int k, char *d_out, uint64_t cap, uint64_t *out_bytes);

/* uc_emit for callers that cannot allocate device memory (a process whose
 * own pool holds all free HBM, a plugin whose host framework owns the
 * allocator, code whose other streams must not wait on the device-wide
 * synchronisation cudaMalloc/cudaFree may do).  No counterpart in the
 * reference.  Same arguments and output as uc_emit, without a context: the
 * work runs on cuda_stream (NULL = legacy default stream) of the current
 * device.  Calls no cudaMalloc or cudaFree; its scratch is one static device
 * array per device, so n is limited to UC_EMIT_NOALLOC_MAX_KMERS (larger n
 * fails with UC_EINPUT).  The first call in a CUDA context looks that
 * array up and loads the emission kernels; CUDA loads modules lazily, so the
 * array and the kernels take their device memory then.  Make that first
 * call before the caller's own pool takes the rest of the device's memory
 * (or run with CUDA_MODULE_LOADING=EAGER), and before any stream capture;
 * later calls in the context allocate nothing.  A context destroyed and
 * created again (cudaDeviceReset) is set up again at its first call.  All
 * calls in a context share the array: calls that overlap on the GPU race.
 * err (err_len bytes, may be NULL) receives a one-line reason on failure. */
#define UC_EMIT_NOALLOC_MAX_KMERS (1u << 20)
uc_status uc_emit_noalloc(void *cuda_stream, const uint64_t *d_keys,
                          const uint32_t *d_succ, const uint32_t *d_head,
                          const uint32_t *d_rank, uint64_t n, int k,
                          char *d_out, uint64_t cap, uint64_t *out_bytes,
                          char *err, size_t err_len);

/* Autotuner; no counterpart in the reference (its bucket and table sizes
 * are fixed in the code).  Times the fused path (uc_compact_device) on
 * d_text, a representative job already in device memory, for candidate
 * tunings: coordinate descent over warp_capacity, bucket_fill,
 * tile_capacity, tile_threads, load_factor_pct and contract_method, each
 * candidate the median device time of reps runs (0 = 3) after one warm-up.
 * Every candidate must produce the same output size (UC_EINTERNAL if not).
 * Stops after a pass without improvement or after max_ms of device time
 * (0 = 60000).  Leaves the fastest tuning set on ctx and returns it, with its
 * time and the number of candidates timed (best_ms, trials may be NULL). */
uc_status uc_autotune(uc_ctx *ctx, const char *d_text, size_t bytes, int k,
                      int l, int reps, uint32_t max_ms, uc_tuning *best,
                      float *best_ms, uint32_t *trials);

/* ---- fused path ------------------------------------------------------ */

/* Whole path on device-resident text: pack, minimizer bucketing, per-tile
 * edge finding + contraction + emission, cross-tile stitch.  The body of the
 * reference's main (driver.cpp:433-659).  Line order is unspecified (the
 * reference's is too); d_out needs at most bytes(text) bytes.  stats may be
 * NULL. */
uc_status uc_compact_device(uc_ctx *ctx, const char *d_text, size_t bytes,
                            int k, int l, char *d_out, uint64_t cap,
                            uint64_t *out_bytes, uc_stats *stats);

/* Upper bound of the output size of uc_compact_device for this text. */
uint64_t uc_output_bound(size_t text_bytes, int k);

/* Synchronous host-memory form: host text in, lines into the caller's host
 * buffer (pinned memory gives full PCIe bandwidth).  *out_bytes receives the
 * length.  main, driver.cpp:422-662, without the file I/O. */
uc_status uc_compact_host(uc_ctx *ctx, const char *text, size_t bytes, int k,
                          int l, char *out, size_t cap, size_t *out_bytes,
                          uc_stats *stats);

/* Many independent jobs in one pass (same k and l): all their buckets form
 * one tile queue worked by one persistent launch per tier.  Job j's lines land
 * in d_out[out_offsets[j], out_offsets[j] + out_lengths[j]).  d_out needs
 * uc_batch_output_bound bytes.  When a job's lines are not exactly k chars +
 * '\n', or any job is malformed, the jobs are compacted one by one, and a
 * malformed job fails the call with UC_EINPUT and its index in
 * uc_last_error.  (No reference counterpart: the reference runs one job per
 * process; this is the batched form of its main.) */
uc_status uc_compact_batch(uc_ctx *ctx, int njobs, const char *const *d_texts,
                           const size_t *bytes, int k, int l, char *d_out,
                           uint64_t out_cap, uint64_t *out_offsets,
                           uint64_t *out_lengths, uc_stats *stats);
uint64_t uc_batch_output_bound(int njobs, const size_t *bytes, int k);

/* ---- host-memory jobs ------------------------------------------------- */

/* A sequence of host jobs, each from host memory (text) to host memory
 * (outs[j], caps[j] bytes; out_lens[j] receives the length), with the
 * uploads overlapped: job j+1's text goes to the device while job j runs its
 * bucketing, tiles, stitch and result copy (a job's text is not read after
 * its pack phase, so one device text buffer serves all).  Equivalent to
 * uc_compact_host per job.  The reference reads and writes one file per run
 * (driver.cpp:257-354, compact.h:7-37); with pinned buffers the host link
 * carries both directions at once.  stats (may be NULL) sums k-mers, output
 * bytes, device time and launches. */
uc_status uc_compact_host_many(uc_ctx *ctx, int njobs, const char *const *texts,
                               const size_t *bytes, int k, int l,
                               char *const *outs, const size_t *caps,
                               size_t *out_lens, uc_stats *stats);

/* Submit host text (pageable or pinned); the job copies it to the device,
 * runs the fused path and copies the lines back into a buffer the library
 * allocates, all before uc_job_submit returns (poll and wait then report it
 * done; the serving loop below is the asynchronous form).  main,
 * driver.cpp:422-662, without the file I/O. */
uc_status uc_job_submit(uc_ctx *ctx, const char *text, size_t bytes, int k,
                        int l, uc_job **job);
uc_status uc_job_poll(uc_job *job, int *done);
uc_status uc_job_wait(uc_job *job);
/* Owned result buffer (free with uc_free) and its length. */
uc_status uc_job_result(uc_job *job, char **buf, size_t *len,
                        uc_stats *stats);
uc_status uc_job_release(uc_job *job);
void uc_free(void *p);

/* ---- serving loop ------------------------------------------------------
 * No counterpart in the reference, which compacts one file per process.  A
 * server owns one device pool of hbm_budget bytes (0 = the smaller of
 * 160 GiB and 90% of free memory), allocated at creation.  Jobs are admitted
 * in arrival order when a lane (a host thread with its own stream) is idle
 * and a slice of the pool covering the job's footprint bound is free; jobs
 * of at most batch_bytes of text queued behind the admitted one, with the
 * same k and l, join its launch (up to max_batch jobs, uc_compact_batch).
 * Lanes run concurrently, so admitted work overlaps on the GPU.  Results
 * equal uc_compact_host's for the same text, line order aside. */
typedef struct uc_server uc_server;
typedef struct uc_server_config {
    int device;
    int lanes;           /* concurrent device lanes (0 = 4) */
    int max_batch;       /* most jobs in one launch (0 = 64) */
    int reserved;
    size_t hbm_budget;   /* device pool bytes */
    size_t batch_bytes;  /* jobs up to this text size may be batched (0 = 64 MiB) */
    size_t host_budget;  /* pinned host pool for results (0 = 16 GiB) */
    uc_tuning tuning;    /* tuning of every lane (zeros = automatic) */
} uc_server_config;
typedef struct uc_server_job_info {
    uc_status status;
    uint32_t batch;       /* jobs in the launch that served this one */
    uint64_t n_kmers;
    double queue_ms;      /* submit to admission */
    double latency_ms;    /* submit to result on the host */
    char error[128];
} uc_server_job_info;
typedef struct uc_server_totals {
    uint64_t jobs_done, kmers_done, batches, batched_jobs, queued;
    uint64_t pool_bytes, pool_peak_bytes;
    double p50_ms, p99_ms, max_ms, mean_ms; /* job latency over completed jobs */
    double wall_s;                          /* first submit to last completion */
} uc_server_totals;
uc_status uc_server_create(const uc_server_config *cfg, uc_server **out);
/* The text stays owned by the caller and must stay valid until the job's
 * uc_server_wait returns. */
uc_status uc_server_submit(uc_server *srv, const char *text, size_t bytes,
                           int k, int l, uint64_t *ticket);
uc_status uc_server_poll(uc_server *srv, uint64_t ticket, int *done);
/* Blocks until the job is done (timeout_s <= 0: no limit; UC_ETIMEOUT when
 * it runs out).  Hands over the lines and forgets the ticket; returns the
 * job's status.  The lines sit in the server's pinned host pool (or in
 * malloc'd memory when that pool is full); give them back with
 * uc_server_free.  buf NULL: the lines are dropped at once. */
uc_status uc_server_wait(uc_server *srv, uint64_t ticket, double timeout_s,
                         char **buf, size_t *len, uc_server_job_info *info);
uc_status uc_server_free(uc_server *srv, char *buf);
uc_status uc_server_stats(uc_server *srv, uc_server_totals *stats);
/* Finishes the launches in flight; jobs still queued are dropped. */
uc_status uc_server_destroy(uc_server *srv);

/* File to file, appending to out_path like write_to_f (compact.h:7-37).
 * The reference CLI `main <k-mer file> k l <output file>`. */
uc_status uc_compact_file(uc_ctx *ctx, const char *in_path, int k, int l,
                          const char *out_path, uc_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
