/*
 * hera_gpu.h -- C ABI of the B200 (sm_100a) read-alignment hot path for hera.
 *
 * The library replaces, batch-wise, the per-pair front half of hera's
 * alignment worker: for every read pair it produces the two Candidate
 * records exactly as hera leaves them after check_in_transcriptome and the
 * two intersect2 calls (src/hash_align.c:1724-1733), and for every single
 * read the Candidate after its two get_position calls
 * (src/hash_align.c:1819-1823).  The host tail of align_pair_read
 * (src/hash_align.c:1735-1811: pair choice, BAM records, add_class,
 * counters) and everything around it stay hera's own C code -- or, where a
 * caller wants them on the GPU as well, the entry points at the end of this
 * file produce the same bytes: FASTQ chunk parsing, the class table
 * (add_class), the EM over it (estimate_count) and the `-w` BAM records.
 *
 * Plain C types and pointers only.  Every entry point returns 0 on success
 * or a negative HERA_GPU_E* code; hera_gpu_last_error() describes the last
 * failure on a context.  There is no CPU fallback: without a usable CUDA
 * device every entry point fails with HERA_GPU_ENODEV.
 */
#ifndef HERA_GPU_H
#define HERA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HERA_GPU_ABI_VERSION 2

/* status codes */
#define HERA_GPU_OK 0
#define HERA_GPU_ENODEV (-1)      /* no CUDA device / driver */
#define HERA_GPU_ECUDA (-2)       /* a CUDA call failed */
#define HERA_GPU_ENOMEM (-3)      /* device or host allocation failed */
#define HERA_GPU_EINVAL (-4)      /* bad argument (NULL, size, read too long) */
#define HERA_GPU_ECAPACITY (-5)   /* a per-read capacity was exceeded */
#define HERA_GPU_ETIMEOUT (-6)    /* a bounded device wait expired */
#define HERA_GPU_EFORMAT (-7)     /* a chunk the reference's reader rejects
				     ("Wrong format of file") */
#define HERA_GPU_ECANCELED (-8)   /* a served chunk whose sample was cancelled */

/* Longest read the device path accepts (hera itself has no limit; reads
 * longer than this are rejected with HERA_GPU_EINVAL). */
#define HERA_GPU_MAX_READ 320

/* ---- reference-layout types (identical in size and field order) ------- */

/* struct read_inf, src/read.h:16-21 */
typedef struct hera_read_inf {
	char *seq;
	char *name;
	char *qual;
	int32_t len;
} hera_read_inf;

/* Cigar, src/hash_align.h:82-88 (arrays malloc'ed, freed by free_cigar) */
typedef struct hera_cigar {
	unsigned short n_cigar;
	unsigned short n_miss;
	unsigned short *count;
	char *type;
	char *miss;
} hera_cigar;

/* Candidate, src/hash_align.h:90-97 (arrays malloc'ed, freed by
 * destroy_candidate; pos/p are only allocated when n > 0) */
typedef struct hera_candidate {
	int *p[2];
	unsigned int *pos[2];
	unsigned int n[2];
	int err[2];
	hera_cigar *cigar[2];
	int pair;
} hera_candidate;

/* Bucket, src/hash_align.h:138-142 */
typedef struct hera_bucket {
	uint64_t id;
	uint32_t start;
	uint32_t end;
} hera_bucket;

/* The loaded index as hera holds it after load_index
 * (src/hash_align.c:1195-1234): Ref_inf (n, len, find, seq) and
 * Kmer_hash (n[H] per-bucket counts, buckets back to back in bucket order,
 * pos/p occurrence arrays).  Host memory; copied to the device. */
typedef struct hera_gpu_index_view {
	uint32_t n_trans;
	const uint32_t *len;         /* REF_INF->len  [n_trans] */
	const uint32_t *find;        /* REF_INF->find [n_trans] (exclusive ends) */
	const char *seq;             /* REF_INF->seq  [find[n_trans-1]] */
	const uint32_t *bucket_n;    /* KMER_HASH->n  [1<<27] */
	const hera_bucket *buckets;  /* KMER_HASH->sentinel, sum(bucket_n) entries */
	uint64_t n_buckets;
	const uint32_t *pos;         /* KMER_HASH->pos [n_pos] */
	const uint32_t *p;           /* KMER_HASH->p   [n_pos] */
	uint32_t n_pos;
} hera_gpu_index_view;

/* ---- flat results ------------------------------------------------------ */

/* One record per Candidate: two per pair ([2i] = r[0], [2i+1] = r[1]), one
 * per single read.  List i of strand s is pos_pool/p_pool[list_off[s] ..
 * +n[s]); CIGAR ops are op_pool[cig_off[s] .. +n_cigar[s]] encoded
 * (count << 4) | op with op in "MIDNSHP=XB"; miss chars (reference bases of
 * X and D runs) are miss_pool[miss_off[s] .. +n_miss[s]]. */
typedef struct hera_cand_rec {
	int32_t n[2];
	int32_t err[2];
	int32_t pair;
	uint32_t list_off[2];
	uint32_t cig_off[2];
	uint32_t miss_off[2];
	uint16_t n_cigar[2];
	uint16_t n_miss[2];
} hera_cand_rec;

/* Caller-owned host buffers for flat results.  On return *_used hold the
 * pool sizes; if a pool is too small the call returns HERA_GPU_ECAPACITY
 * with *_used set to the sizes needed. */
typedef struct hera_gpu_result {
	hera_cand_rec *recs;
	uint32_t *pos_pool;
	int32_t *p_pool;
	uint32_t *op_pool;
	char *miss_pool;
	uint64_t list_cap, op_cap, miss_cap;
	uint64_t list_used, op_used, miss_used;
} hera_gpu_result;

/* Reads of one batch, back to back in host memory: read i is
 * seq[off[i] .. off[i] + len[i]). */
typedef struct hera_gpu_reads {
	const char *seq;
	const int64_t *off;
	const int32_t *len;
} hera_gpu_reads;

typedef struct hera_gpu_ctx hera_gpu_ctx;

/* Execution forms of the same computation (results are identical).
 * PLAIN: one thread per get_position call and per pair, one pipeline pass
 * per chunk.  BATCHED: get_position split into build / length-binned DP
 * jobs / replay rounds, pair control flow suspended between rounds. */
#define HERA_GPU_PATH_BATCHED 0
#define HERA_GPU_PATH_PLAIN 1

typedef struct hera_gpu_options {
	int device;              /* CUDA device ordinal */
	uint32_t max_batch;      /* pairs (or single reads) per sub-batch; 0 = 1<<18 */
	uint64_t scratch_bytes;  /* unused (the mate-rescue DP works in shared
				    memory); kept for layout compatibility */
	int path;                /* HERA_GPU_PATH_BATCHED (default) or _PLAIN */
	int lanes;               /* concurrent sub-batches (stream + host thread each); 0 = 6 */
} hera_gpu_options;

/* Per-stage device time of the last call, milliseconds (CUDA events,
 * summed over the lanes that ran concurrently); total_ms is wall time. */
typedef struct hera_gpu_timing {
	float h2d_ms, seed_ms, position_ms, resolve_ms, rescue_ms, pack_ms, d2h_ms, total_ms;
	float build_ms, dp_ms;   /* batched form: build and DP+replay parts of position_ms */
	uint32_t launches;       /* kernels launched by the last call */
	uint32_t rescue_rounds;  /* control-flow rounds after the first */
	uint64_t lookups;        /* seed-table lookups issued by seed_probe */
	uint64_t dp_jobs;        /* batched form: gap-DP jobs run (after deduplication) */
	uint64_t dp_calls;       /* batched form: SW_align calls those jobs served */
	/* kernel-level device time (CUDA events around the launches alone) */
	float seed_kernel_ms;    /* seed_probe: the seed-table gathers */
	float dp_kernel_ms;      /* batched form: the gap-DP kernels */
	float rescue_kernel_ms;  /* mate-rescue local SW kernels */
	/* host time inside the call (summed over lane threads) */
	float host_stage_ms;     /* copying reads into pinned staging */
	float host_out_ms;       /* unpacking records into the caller's result */
	/* work counters (device atomics, one per warp) */
	uint64_t probes;         /* bucket records read by the binary searches */
	uint64_t seed_hits;      /* lookups that found their k-mer */
	uint64_t sw_cells;       /* SW_align cells evaluated, counted the way
				    src/hash_align.c:659-681 visits them */
	uint64_t ssw_cells;      /* ssw_align cells: ref_len x read_len per call */
	uint64_t wide_items;     /* pairs (or single reads) aligned again in the
				    wide pass: their first pass met a per-read
				    capacity (more than 256 anchors in one
				    get_position call, 64 hits, 96 CIGAR ops or
				    miss chars) */
} hera_gpu_timing;

/* ---- entry points ------------------------------------------------------ */

/* Library ABI version (HERA_GPU_ABI_VERSION). */
int hera_gpu_abi_version(void);

/* Create a context and copy the index to the device.  Replaces nothing in
 * hera: called once after load_index (src/hash_align.c:1195) with the
 * loaded KMER_HASH / REF_INF arrays.  `opt` may be NULL. */
int hera_gpu_ctx_create(const hera_gpu_index_view *ix, const hera_gpu_options *opt,
			hera_gpu_ctx **out);

/* Release the context and its device memory. */
void hera_gpu_ctx_destroy(hera_gpu_ctx *ctx);

/* Human-readable description of the last failure on `ctx` (never NULL). */
const char *hera_gpu_last_error(const hera_gpu_ctx *ctx);

/* Paired reads -> flat records.  Replaces, for `n` pairs, the calls
 * check_in_transcriptome + intersect2 x2 made per pair by align_pair_read
 * (src/hash_align.c:1728-1733).  write_bam is hera's WRITE_BAM global
 * (src/hash_align.c:32; 1 = no `-w`, score-only gap DP; 0 = `-w`, full
 * traceback).  r1/r2 sequences are read only. */
int hera_gpu_align_pairs_flat(hera_gpu_ctx *ctx, const hera_gpu_reads *r1,
			      const hera_gpu_reads *r2, int32_t n, int write_bam,
			      hera_gpu_result *out);

/* Single reads -> flat records: the two get_position calls of
 * align_single_read (src/hash_align.c:1822-1823). */
int hera_gpu_align_single_flat(hera_gpu_ctx *ctx, const hera_gpu_reads *reads,
			       int32_t n, int write_bam, hera_gpu_result *out);

/* Asynchronous form of hera_gpu_align_pairs_flat, no counterpart in hera:
 * submit starts the call and returns at once with a ticket; complete waits
 * for it and returns its status (out is then filled as the synchronous
 * call fills it; hera_gpu_get_timing then describes that call).  Two calls
 * may be in flight, each on a group of lanes of its own (the second group
 * is made on first use), so one call's copies to and from the host overlap
 * the other's kernels.  r1, r2 and out -- the structs and the memory they
 * point to -- must stay valid and untouched until the call completes; no
 * other call may use the context while asynchronous calls are in flight.
 * A third submit fails with HERA_GPU_EINVAL. */
int hera_gpu_align_pairs_submit(hera_gpu_ctx *ctx, const hera_gpu_reads *r1,
				const hera_gpu_reads *r2, int32_t n, int write_bam,
				hera_gpu_result *out, uint64_t *ticket);
int hera_gpu_align_pairs_complete(hera_gpu_ctx *ctx, uint64_t ticket);

/* Drop-in form of hera_gpu_align_pairs_flat for hera's worker loop
 * (align_pool_pair, src/hash_align.c:1878-1929): reads as struct read_inf,
 * results as heap-allocated Candidate pairs (out[2i] = r[0],
 * out[2i+1] = r[1]) ready for the unchanged host tail; free each with
 * hera's destroy_candidate (src/hash_align.c:973).  Like the reference,
 * lower-case a/c/g/t in r1[i].seq and r2[i].seq become upper-case. */
int hera_gpu_align_pairs(hera_gpu_ctx *ctx, hera_read_inf *r1, hera_read_inf *r2,
			 int32_t n, int write_bam, hera_candidate **out);
/* The two drop-in forms (hera_gpu_align_pairs, hera_gpu_align_single) may be
 * called by several host threads at once on one context, as hera's -t N
 * workers do: calls that meet are combined into one device batch (the
 * first caller runs it, the others wait; each gets its own Candidates),
 * which keeps hera's 1 MB chunks from paying a device call each.  No other
 * entry point may run on the context while they do. */

/* Drop-in form for align_pool_single (src/hash_align.c:1966-1998). */
int hera_gpu_align_single(hera_gpu_ctx *ctx, hera_read_inf *reads, int32_t n,
			  int write_bam, hera_candidate **out);

/* Free n Candidates of the drop-in forms as hera's destroy_candidate
 * (src/hash_align.c:973-989) does, for callers outside hera's C (NULL
 * entries are skipped; each entry is set to NULL). */
void hera_gpu_free_candidates(hera_candidate **c, int64_t n);

/* Device-resident batch (inputs already in HBM): the same computation as
 * hera_gpu_align_pairs_flat on device pointers (seq, off, len for 2n reads:
 * read 2i is mate 1 and read 2i+1 mate 2 of pair i; reads back to back with
 * rising offsets; no read longer than max_read_len <= HERA_GPU_MAX_READ).
 * Results stay on the device; hera_gpu_fetch_result copies them out.
 * `stream` is a cudaStream_t (NULL = the context's own stream). */
int hera_gpu_align_pairs_device(hera_gpu_ctx *ctx, const uint8_t *d_seq,
				const int64_t *d_off, const int32_t *d_len,
				int32_t n, int32_t max_read_len, int write_bam,
				void *stream);

/* Copy the results of the last device-resident call into `out`. */
int hera_gpu_fetch_result(hera_gpu_ctx *ctx, hera_gpu_result *out);

/* Most pairs one hera_gpu_align_pairs_device_noalloc call accepts. */
#define HERA_GPU_NOALLOC_MAX_PAIRS 1024

/* No counterpart in the reference.  The same computation as
 * hera_gpu_align_pairs_device for callers that must not allocate device
 * memory while they align: code that runs inside a memory pool it does not
 * own, or where a cudaMalloc would synchronise the device or fail under a
 * hard memory budget.  This call allocates nothing.  Its working memory
 * (mate-rescue outputs, DP jobs, per-pair state, queues) is one static
 * device array of 17.4 MiB, which every GPU that loads
 * this library holds until the process exits.  The caller passes the reads
 * in device memory (as for hera_gpu_align_pairs_device) and an output in
 * device memory: d_out->recs with room for 2n records and the three pools
 * with their capacities; *_used returns the pool sizes.
 *   - n <= HERA_GPU_NOALLOC_MAX_PAIRS, reads <= HERA_GPU_MAX_READ bytes;
 *     larger batches fail with HERA_GPU_EINVAL.
 *   - A batch whose output outgrows d_out fails with HERA_GPU_ECAPACITY,
 *     and *_used then give the pool sizes needed.  A batch whose internal
 *     work (DP jobs, rescue calls) outgrows the static array also fails
 *     with HERA_GPU_ECAPACITY, with *_used left at 0: align fewer pairs per
 *     call.  So does a pair that passes a per-read capacity (its second,
 *     wide pass would need memory of its own): hera_gpu_align_pairs_device
 *     aligns such pairs.
 *   - The pools are written only below the capacities given, never past.
 *   - Every call reads the batch's byte range back from d_off and waits for
 *     the caller's stream to do so.
 *   - The first call on a device looks up the static array's device
 *     address (cudaGetSymbolAddress); make that first call before any
 *     stream capture.
 *   - Every call shares the one array and its state persists between calls
 *     (each call initialises what it reads).  Calls that overlap on the GPU
 *     -- from two threads, or two contexts on one device -- race. */
int hera_gpu_align_pairs_device_noalloc(hera_gpu_ctx *ctx, const uint8_t *d_seq,
					const int64_t *d_off, const int32_t *d_len,
					int32_t n, int32_t max_read_len, int write_bam,
					hera_gpu_result *d_out, void *stream);

/* Per-stage timing of the last call on `ctx`. */
int hera_gpu_get_timing(const hera_gpu_ctx *ctx, hera_gpu_timing *out);

/* Launch shapes of the batched form, no counterpart in hera.  The library
 * times the candidates on a context's first large batch (at least 16384
 * pairs) and keeps the fastest: the residency of the persistent build
 * kernel (blocks per SM: more blocks hide more gather latency, fewer keep
 * each thread's anchor and chain lists in cache) and the number of
 * mate-rescue calls (warps) per block (shared-memory areas per SM).
 * Results do not depend on these values. */
typedef struct hera_gpu_tuning {
	int build_blocks_per_sm;     /* default 8 until tuned */
	int rescue_warps_per_block;  /* default 4 until tuned */
	int state;                   /* 0 defaults, 1 tuned by the library, 2 set by the caller */
	int n_build, n_rescue;       /* candidates timed */
	int build_cand[8];
	float build_ms[8];           /* build kernel time per candidate (one launch) */
	int rescue_cand[4];
	float rescue_ms[4];          /* rescue kernel time per candidate (one launch) */
} hera_gpu_tuning;

/* The context's launch shapes and, once tuned, the timings they came from. */
int hera_gpu_get_tuning(const hera_gpu_ctx *ctx, hera_gpu_tuning *out);

/* Pin the launch shapes (state becomes 2; the autotuner no longer runs).
 * build_blocks_per_sm in 1..16, rescue_warps_per_block in {1, 2, 4, 8}. */
int hera_gpu_set_tuning(hera_gpu_ctx *ctx, const hera_gpu_tuning *in);

/* Page-lock host memory that is reused across calls (read buffers, result
 * pools), no counterpart in hera.  Calls detect page-locked inputs and
 * outputs by themselves (this or cudaHostAlloc / cudaHostRegister memory):
 * a contiguous mate block then goes to the device without the copy into
 * the library's pinned staging, and records and pools come back straight
 * into the result, their offsets rebased on the device.  Unregister before
 * freeing the memory. */
int hera_gpu_host_register(void *p, size_t bytes);
int hera_gpu_host_unregister(void *p);

/* ---- serving loop (no counterpart in hera) ----------------------------- *
 *
 * hera aligns one sample per process.  The server keeps one context's index
 * resident and aligns FASTQ chunks (read pairs) of many samples as they
 * arrive.  Continuous batching: a device batch is cut from the head of the
 * pending chunks whenever a batch slot frees up, so a batch may hold the
 * tail of one sample's chunk and the head of another's, and chunks that
 * arrive while others run join the next batch instead of waiting for a
 * whole queue to drain.  Slots run concurrently (stream + host thread each);
 * their number is fixed at creation from the free device memory.  Every
 * chunk's records are exactly those hera_gpu_align_pairs_flat returns for
 * it alone.  Per-sample counters are kept on the device. */
typedef struct hera_gpu_server hera_gpu_server;

typedef struct hera_gpu_server_options {
	uint32_t batch_pairs;    /* pairs per device batch; 0 = 131072 */
	int max_slots;           /* batches in flight at most; 0 = 6 */
	uint64_t hbm_reserve;    /* device bytes to leave free; 0 = 4 GiB */
	int write_bam;           /* hera's WRITE_BAM for every chunk */
	uint32_t max_samples;    /* per-sample state slots; 0 = 1024 */
	int borrow_reads;        /* 1: submit keeps pointers to the caller's
				    reads instead of copying them; the caller
				    leaves that memory valid and unchanged until
				    the chunk's wait returns (or the server is
				    destroyed).  The batch slots then stage
				    reads straight from it. */
} hera_gpu_server_options;

typedef struct hera_gpu_chunk_info {
	uint32_t sample;
	int32_t n;               /* pairs */
	double submit_ms;        /* server clock (ms since creation) */
	double admit_ms;         /* first pair of the chunk entered a batch */
	double done_ms;          /* last pair's records were on the host */
	int32_t batches;         /* device batches the chunk was spread over */
} hera_gpu_chunk_info;

typedef struct hera_gpu_sample_stats {   /* kept on the device, per sample */
	uint64_t pairs;          /* pairs aligned */
	uint64_t mapped;         /* pairs with a hit for at least one mate */
	uint64_t paired;         /* pairs whose r[0].pair == 2 (mates agree) */
	uint64_t hits;           /* sum of n[0] + n[1] over both Candidates */
	uint64_t cigar_ops;      /* sum of CIGAR ops over both Candidates */
	uint64_t reserved[3];
} hera_gpu_sample_stats;

typedef struct hera_gpu_server_stats {
	int slots;               /* batch slots (from free device memory) */
	uint64_t slot_bytes;     /* device bytes budgeted per slot */
	uint64_t chunks_done, pairs_done, batches;
	float p50_ms, p99_ms;    /* chunk latency: submit to done */
	float p50_wait_ms, p99_wait_ms;   /* submit to admission */
	double pairs_per_s;      /* pairs_done / (last done - first submit) */
} hera_gpu_server_stats;

/* Start a server on `ctx` (the context must outlive it; do not run other
 * calls on `ctx` while the server is alive).  `opt` may be NULL. */
int hera_gpu_server_create(hera_gpu_ctx *ctx, const hera_gpu_server_options *opt,
			   hera_gpu_server **out);

/* Queue n pairs of `sample` (< max_samples).  The reads are copied, so the
 * caller's buffers are free on return.  *ticket identifies the chunk. */
int hera_gpu_server_submit(hera_gpu_server *s, uint32_t sample, const hera_gpu_reads *r1,
			   const hera_gpu_reads *r2, int32_t n, uint64_t *ticket);

/* Block until the chunk is done and copy its records into `out` (layout as
 * hera_gpu_align_pairs_flat); the chunk is then released.  If a pool of
 * `out` is too small, returns HERA_GPU_ECAPACITY with *_used set and keeps
 * the chunk for another try.  One wait per ticket at a time (a second
 * concurrent wait fails with HERA_GPU_EINVAL).  `info` may be NULL. */
int hera_gpu_server_wait(hera_gpu_server *s, uint64_t ticket, hera_gpu_result *out,
			 hera_gpu_chunk_info *info);

/* Drop the queued work of `sample` (no counterpart in hera: a client that
 * goes away mid-run).  Its chunks not yet fully admitted to a batch stop:
 * their remaining pairs are never aligned, and hera_gpu_server_wait on
 * their tickets returns HERA_GPU_ECANCELED once the pieces already in
 * batches have finished.  Chunks already fully admitted complete normally,
 * and every other sample's chunks are unaffected (their records stay those
 * of the chunk aligned alone).  *n_chunks (may be NULL): chunks cancelled.
 * Later submits for the sample are accepted. */
int hera_gpu_server_cancel(hera_gpu_server *s, uint32_t sample, int32_t *n_chunks);

/* Per-sample counters (read from the device) and server-wide figures. */
int hera_gpu_server_get_sample_stats(hera_gpu_server *s, uint32_t sample, hera_gpu_sample_stats *out);
int hera_gpu_server_get_stats(hera_gpu_server *s, hera_gpu_server_stats *out);

/* Stop the slots after the batches in flight and free everything; chunks
 * not yet waited for are dropped. */
void hera_gpu_server_destroy(hera_gpu_server *s);

/* Kernel-level check, no counterpart in hera: ssw_align (src/ssw.c:81-321)
 * as the mate-rescue kernel computes it, for n (window, read) cases given as
 * ASCII strings back to back (refs[ref_off[i] .. ref_off[i+1]), same for
 * reads; windows up to 1000 bases, reads up to HERA_GPU_MAX_READ).  As in
 * the aligner, a case whose CIGAR passes the first pass's capacities (96
 * ops, 96 miss chars) runs again in the wide pass's form.  Per case: score,
 * skip, and the CIGAR (ops[i*cap ..], n_ops[i]; miss[i*cap ..], n_miss[i]);
 * *flags ORs the flags left after that.  Allocates device memory. */
int hera_gpu_unit_ssw(int device, const char *refs, const int64_t *ref_off, const char *reads,
		      const int64_t *read_off, int32_t n, int32_t *score, int32_t *skip, uint32_t *ops,
		      int32_t *n_ops, char *miss, int32_t *n_miss, int32_t cap, int32_t *flags);

/* Kernel-level check, no counterpart in hera: SW_align
 * (src/hash_align.c:627-760) as the batched form's gap-DP kernels compute
 * it, for n (window, query, err) cases given as ASCII strings back to back
 * (refs[ref_off[i] .. ref_off[i+1]), queries likewise, up to
 * HERA_GPU_MAX_READ bases; err as the reference passes it, negative for a
 * prefix DP).  write_bam is hera's WRITE_BAM (1: score-only, one M op).
 * Per case: score and the CIGAR (ops[i*cap ..], n_ops[i]; miss[i*cap ..],
 * n_miss[i]); *flags ORs capacity flags.  Allocates device memory. */
int hera_gpu_unit_sw(int device, const char *refs, const int64_t *ref_off, const char *qs,
		     const int64_t *q_off, const int32_t *err, int32_t n, int write_bam, int32_t *score,
		     uint32_t *ops, int32_t *n_ops, char *miss, int32_t *n_miss, int32_t cap,
		     int32_t *flags);

/* Measurement helper, no counterpart in hera: the device's throughput of
 * the DPX instruction the gap DP's cell update is built on (packed 16x2
 * add-then-min, __viaddmin_s16x2), measured with independent chains on
 * every SM for about `ms` milliseconds.  *instr_per_s receives thread-level
 * instructions per second (warp instructions x 32; each one updates two
 * 16-bit lanes).  Allocates and frees a small output buffer, so it is not
 * for use inside stream capture. */
int hera_gpu_dpx_peak(int device, float ms, double *instr_per_s);

/* The context's CUDA stream (a cudaStream_t): the default caller stream of
 * hera_gpu_align_pairs_device, for callers that time or order work around
 * the library's launches.  Calls on one context must not overlap. */
void *hera_gpu_stream(hera_gpu_ctx *ctx);

/* ---- FASTQ chunks ---------------------------------------------------------
 * A chunk buffer as hera's reader hands it to a worker (gb_get_pair /
 * gb_get_single, src/get_buffer.c:191-300): whole FASTQ records, bytes
 * [0, n) followed by a NUL.  The caller need not store that NUL; a NUL inside
 * the buffer ends the chunk, as it ends the reference's reader.  Chunks are
 * below 2 GiB (a pair's two together for hera_gpu_align_fastq_pairs). */

/* One read of a chunk, as byte offsets into its buffer. */
typedef struct hera_gpu_fastq_rec {
	int64_t name;      /* the byte after '@' */
	int64_t seq;
	int64_t qual;
	int32_t name_len;  /* bytes of the name line after '@' */
	int32_t len;       /* sequence (and quality) length */
} hera_gpu_fastq_rec;

/* Device time of the last parse (CUDA events): the chunk copies, the parse
 * kernels, and hera_gpu_align_fastq_pairs' gather of the sequences for the
 * aligner. */
typedef struct hera_gpu_fastq_stats {
	float h2d_ms, parse_ms, gather_ms;
	int32_t launches;
	int64_t bytes;     /* chunk bytes parsed */
	int64_t reads;     /* reads of the result */
} hera_gpu_fastq_stats;

/* Parse a pair of chunk buffers on the device: the reads hera's
 * align_pool_pair takes from them (src/hash_align.c:1878-1929), each as
 * get_read_from_fq_buffer reads it (src/read.c:11-63) -- file 1's read,
 * then file 2's, until either file's last read.  recs[2i] and recs[2i+1] are
 * the mates of pair i (room for `cap` pairs).  HERA_GPU_EFORMAT where the
 * reference stops with "Wrong format of file": *bad_file (1 or 2) and
 * *bad_read (0-based read of that file) name the read it rejects.
 * HERA_GPU_ECAPACITY when the chunk holds more than `cap` pairs (*n_pairs
 * is then the count). */
int hera_gpu_parse_fastq_pairs(hera_gpu_ctx *ctx, const char *left, int64_t n_left,
			       const char *right, int64_t n_right, hera_gpu_fastq_rec *recs,
			       int32_t cap, int32_t *n_pairs, int32_t *bad_file,
			       int64_t *bad_read);

/* The same for one chunk of single reads (align_pool_single,
 * src/hash_align.c:1966-1998). */
int hera_gpu_parse_fastq_single(hera_gpu_ctx *ctx, const char *chunk, int64_t n,
				hera_gpu_fastq_rec *recs, int32_t cap, int32_t *n_reads,
				int64_t *bad_read);

/* Parse a pair of chunk buffers and align their pairs on the device: the
 * parsed sequences go to the aligner without leaving the GPU.  `out` gets
 * what hera_gpu_align_pairs_flat gives for the same reads; recs/n_pairs and
 * the errors as for hera_gpu_parse_fastq_pairs (reads longer than
 * HERA_GPU_MAX_READ: HERA_GPU_EINVAL). */
int hera_gpu_align_fastq_pairs(hera_gpu_ctx *ctx, const char *left, int64_t n_left,
			       const char *right, int64_t n_right, int write_bam,
			       hera_gpu_fastq_rec *recs, int32_t cap, int32_t *n_pairs,
			       int32_t *bad_file, int64_t *bad_read, hera_gpu_result *out);

int hera_gpu_get_fastq_stats(hera_gpu_ctx *ctx, hera_gpu_fastq_stats *out);

/* The reader's side effects for hera's host tail: NULs over the newlines
 * that end each read's name, sequence and quality (src/read.c:26, 36, 58),
 * and read_inf views of the reads.  buf/n: the chunk buffer the records came
 * from; recs[i * stride], i < count (stride 2 with recs + 0 or + 1 for one
 * file of a pair). */
int hera_gpu_fastq_read_inf(char *buf, int64_t n, const hera_gpu_fastq_rec *recs,
			    int32_t count, int32_t stride, hera_read_inf *out);

/* ---- equivalence classes ---------------------------------------------------
 * The add_class calls of hera's host tail (src/hash_align.c:1564-1602), made
 * by align_pair_read (:1735-1760) and align_single_read (:1825-1851), run on
 * the device over flat records.  A class table holds, like hera's CLASS and
 * REF_INF->count globals: the classes in first-insertion order (XXH32 id of
 * the transcript list, read count, the list), the per-transcript count of
 * reads with a one-entry list, PAIRED and the running sum behind MEAN_FRAG
 * (before src/main.c:30 divides it).  Adding the records of a run batch by
 * batch, in input order, gives exactly the table hera's `-t 1` worker
 * builds.  With FMINDEX NULL (no `-f`), as everywhere in this library. */
typedef struct hera_gpu_classes hera_gpu_classes;

/* Host buffers for hera_gpu_classes_fetch.  On return n_classes and
 * list_used hold the table's sizes; with class_cap or list_cap too small the
 * call returns HERA_GPU_ECAPACITY and fills only those. */
typedef struct hera_gpu_class_table {
	uint32_t class_cap;
	uint32_t *id;            /* Class.id    [class_cap] */
	double *count;           /* Class.count [class_cap] */
	uint32_t *n;             /* Class.n     [class_cap] */
	uint64_t *list_off;      /* class i's list: list[list_off[i] .. + n[i]) */
	uint64_t list_cap;
	uint32_t *list;          /* Class.ref lists back to back [list_cap] */
	uint32_t *tx_count;      /* REF_INF->count [n_trans]; may be NULL */
	uint32_t n_classes;
	uint64_t list_used;
	uint32_t paired;         /* PAIRED */
	double mean_frag_sum;    /* MEAN_FRAG before the division */
} hera_gpu_class_table;

/* A class table on ctx's device holding at most max_classes classes and
 * max_list list entries in total (device memory: about 24 B a class slot,
 * 28 B a class, 4 B a list entry, 4 B a transcript).  Replaces hera's
 * init_class (src/hash_align.c:1161-1167) and the zeroing of REF_INF->count,
 * PAIRED and MEAN_FRAG. */
int hera_gpu_classes_create(hera_gpu_ctx *ctx, uint32_t max_classes, uint64_t max_list,
			    hera_gpu_classes **out);
void hera_gpu_classes_destroy(hera_gpu_classes *c);

/* add_class for the pairs of the last hera_gpu_align_pairs_device call on
 * ctx, in pair order, without the records leaving the device. */
int hera_gpu_classes_add_last(hera_gpu_classes *c, hera_gpu_ctx *ctx);

/* add_class for n records in device memory (layout of hera_gpu_result:
 * paired = 1, n pairs, d_recs[2i] / [2i+1] = r[0] / r[1]; paired = 0, n
 * single reads).  `stream` (a cudaStream_t, may be NULL) is the stream that
 * wrote the records.  More classes or list entries than the table holds:
 * HERA_GPU_ECAPACITY, and the table is unusable from then on. */
int hera_gpu_classes_add_device(hera_gpu_classes *c, const hera_cand_rec *d_recs,
				const uint32_t *d_pos_pool, const int32_t *d_p_pool, int32_t n,
				int paired, void *stream);

/* add_class for n pairs (paired = 1) or single reads (paired = 0) whose flat
 * records are in host memory, as an align call left them in `res` (records,
 * and the pos/p pools up to res->list_used).  The records are copied to the
 * device first; for results already there use the two calls above. */
int hera_gpu_classes_add_host(hera_gpu_classes *c, const hera_gpu_result *res, int32_t n,
			      int paired);

/* Copy the table out (see hera_gpu_class_table). */
int hera_gpu_classes_fetch(hera_gpu_classes *c, hera_gpu_class_table *out);

/* Replace the table's contents with a class table given in host memory
 * (the layout hera_gpu_classes_fetch fills: n_classes classes with whole-
 * number counts, list_used list entries, tx_count or NULL for zeros, PAIRED
 * and the fragment sum): hera's CLASS and REF_INF->count as its own
 * add_class built them, for callers that keep the tail on the host and run
 * the EM below on the device.  Later adds continue the table. */
int hera_gpu_classes_load(hera_gpu_classes *c, const hera_gpu_class_table *in);

/* hera's EM, estimate_count (src/EM.c:315-387: SQUAREM over M_step with
 * E_step's uniform start, Norm of src/hash_align.c:150-164), over the
 * table's classes, its per-transcript counts and ctx's transcript lengths
 * (REF_INF->len).  grama and overlap (n_trans doubles each, host memory)
 * receive em_val->grama and em_val->overlap bit for bit as the reference
 * leaves them; *rounds the SQUAREM iterations, *em_ms the device time
 * (either may be NULL).  Allocates its working memory per call. */
int hera_gpu_classes_em(hera_gpu_classes *c, hera_gpu_ctx *ctx, double *grama, double *overlap,
			uint32_t *rounds, float *em_ms);

/* ---- BAM records ------------------------------------------------------------
 * With `-w` hera's tail writes each pair's alignment records
 * (align_pair_read's branches, src/hash_align.c:1735-1804, over
 * bam_write_pair, src/bam_write.c:382-416) into the stream it then BGZF-
 * compresses.  hera_gpu_bam_pairs produces those uncompressed bytes for a
 * batch of pairs on the device, identical to hera's; compression stays with
 * the caller (bam_write). */

/* GENE_MAP (src/bam_write.c:22-57): chromosome lengths, each transcript's
 * exons [exon_off[t], exon_off[t+1]) of starts/ends (genome coordinates),
 * and its chromosome and gene.  Host memory; copied at creation. */
typedef struct hera_gpu_gene_map {
	uint32_t n_chr;
	const uint32_t *chr_len;     /* [n_chr] */
	const uint32_t *exon_off;    /* [n_trans + 1] */
	const uint32_t *starts;      /* [exon_off[n_trans]] */
	const uint32_t *ends;
	const uint32_t *chr;         /* [n_trans] */
	const uint32_t *gene;        /* [n_trans] */
} hera_gpu_gene_map;

typedef struct hera_gpu_bam hera_gpu_bam;

/* A BAM record writer for ctx's index with this gene map. */
int hera_gpu_bam_create(hera_gpu_ctx *ctx, const hera_gpu_gene_map *gm, hera_gpu_bam **out);
void hera_gpu_bam_destroy(hera_gpu_bam *b);
const char *hera_gpu_bam_last_error(const hera_gpu_bam *b);

/* The records hera's tail writes for n pairs (host memory throughout):
 * `res` as hera_gpu_align_pairs_flat left it with write_bam = 0; r1/r2 the
 * pairs' sequences and qual1/qual2 their qualities at the same offsets;
 * name1/name2 the NUL-terminated names, pair i's at i * name_stride (a NUL
 * inside each slot).  The inputs are not modified (hera's tail reverses
 * reads and cuts "/1" off names while it writes; the records show that).
 * Pair i's bytes are out[out_off[i] .. out_off[i+1]); out_off has n + 1
 * entries.  With `cap` too small: HERA_GPU_ECAPACITY, out_off[n] = the
 * bytes needed.  *kernel_ms (may be NULL): device time of the call. */
int hera_gpu_bam_pairs(hera_gpu_bam *b, const hera_gpu_result *res, int32_t n,
		       const hera_gpu_reads *r1, const hera_gpu_reads *r2,
		       const char *qual1, const char *qual2, const char *name1,
		       const char *name2, int32_t name_stride, uint8_t *out, uint64_t cap,
		       uint64_t *out_off, float *kernel_ms);

/* The records align_single_read writes for n single reads
 * (src/hash_align.c:1825-1834, bam_write_single src/bam_write.c:418-446):
 * `res` as hera_gpu_align_single_flat left it with write_bam = 0; the rest
 * as for hera_gpu_bam_pairs with one read, quality and name per item. */
int hera_gpu_bam_single(hera_gpu_bam *b, const hera_gpu_result *res, int32_t n,
			const hera_gpu_reads *reads, const char *qual, const char *name,
			int32_t name_stride, uint8_t *out, uint64_t cap, uint64_t *out_off,
			float *kernel_ms);

/* BGZF, the BAM container (hera's bam_write, src/hash_align.c:48-136), on
 * the device: in[0 .. n) (host memory) becomes back-to-back BGZF blocks of
 * at most 65280 input bytes each in out (host, cap bytes); *out_len = the
 * bytes written (or needed, with HERA_GPU_ECAPACITY).  Each block is a
 * gzip member with the BGZF extra field, a DEFLATE stream (greedy LZ77,
 * fixed Huffman codes, or stored when that is not smaller) and the CRC-32
 * and size of its input: the bytes differ from zlib's, the decompressed
 * stream is the input.  No end-of-file block is added (hera's bam_close
 * writes it).  Allocates device memory.  *kernel_ms (may be NULL): device
 * time of the compression and packing. */
int hera_gpu_bgzf(hera_gpu_ctx *ctx, const uint8_t *in, uint64_t n, uint8_t *out, uint64_t cap,
		  uint64_t *out_len, float *kernel_ms);

/* Device time (CUDA events, from the first kernel of the last add call to
 * its end; the call's first-use allocations are not in it) and the
 * kernels it launched. */
int hera_gpu_classes_timing(const hera_gpu_classes *c, float *kernel_ms, uint32_t *launches);
const char *hera_gpu_classes_last_error(const hera_gpu_classes *c);

#ifdef __cplusplus
}
#endif
#endif
