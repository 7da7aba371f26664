/*
 * hera_oracle.h -- CPU restatement of hera's transcriptome read-alignment
 * hot path (k-mer seeding, anchor chaining, SW_align gap fill, ssw_align mate
 * rescue, pairing).  TEST INFRASTRUCTURE ONLY: the parity checker for the
 * CUDA path.  Nothing in the hera_b200 product links, loads or calls this.
 *
 * Parity of this restatement is pinned against the reference program itself
 * (compiled from its own sources into oracle/_ref by oracle/Makefile) through
 * golden vectors committed under tests/golden/ and live comparisons in the
 * CPU test suite.
 *
 * All structures here are the oracle's own; the result record layout matches
 * the product's `hera_cand_rec` field for field so tests can compare them.
 */
#ifndef HERA_ORACLE_H
#define HERA_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HO_KMER 31
#define HO_ERR 7
#define HO_MAX_FRAG 1000
#define HO_HBITS 27

/* One bucket entry, identical in size and order to the reference's Bucket
 * (src/hash_align.h:138-142): 64-bit k-mer id, [start, end) into pos/p. */
typedef struct {
	uint64_t id;
	uint32_t start;
	uint32_t end;
} ho_bucket;

/* Read-only view of a loaded index (src/hash_align.c:1195-1234 layout,
 * with the per-bucket counts n[] replaced by their prefix sums). */
typedef struct {
	uint32_t n_trans;
	const uint32_t *len;        /* transcript lengths */
	const uint32_t *find;       /* exclusive end offset of each transcript in seq */
	const char *seq;            /* concatenated transcripts, >= 8 zero bytes after */
	const uint64_t *bucket_off; /* (1<<27)+1 prefix sums of bucket sizes */
	const ho_bucket *buckets;
	const uint32_t *pos;        /* occurrence transcript ids */
	const uint32_t *p;          /* occurrence offsets (last base of the k-mer) */
} ho_index;

/* Flat result record: one per Candidate (two per read pair, one per single
 * read).  Lists live in pools at list_off; CIGAR ops are (count << 4) | op. */
typedef struct {
	int32_t n[2];
	int32_t err[2];
	int32_t pair;
	uint32_t list_off[2];
	uint32_t cig_off[2];
	uint32_t miss_off[2];
	uint16_t n_cigar[2];
	uint16_t n_miss[2];
} ho_rec;

typedef struct {
	ho_rec *recs;
	uint32_t *pos_pool;
	int32_t *p_pool;
	uint32_t *op_pool;
	char *miss_pool;
	uint64_t list_cap, op_cap, miss_cap;   /* pool capacities (entries) */
	uint64_t list_used, op_used, miss_used;
} ho_result;

/* Batch of reads: read i is seq[off[i] .. off[i]+len[i]). */
typedef struct {
	const char *seq;
	const int64_t *off;
	const int32_t *len;
} ho_reads;

/* Front half of align_pair_read (src/hash_align.c:1724-1733) per pair:
 * check_in_transcriptome then the two intersect2 calls.  write_bam carries
 * the reference's WRITE_BAM global (1 = score-only DP, the no `-w` mode).
 * Returns 0, or -1 when a result pool is too small (nothing is partial:
 * the caller retries with larger pools).  `reads1`/`reads2` are modified
 * exactly as the reference modifies read->seq (lower-case ACGT upper-cased). */
int ho_align_pairs(const ho_index *ix, int write_bam, int n,
		   char *seq1, const int64_t *off1, const int32_t *len1,
		   char *seq2, const int64_t *off2, const int32_t *len2,
		   ho_result *out);

/* Front half of align_single_read (src/hash_align.c:1819-1823). */
int ho_align_single(const ho_index *ix, int write_bam, int n,
		    char *seq, const int64_t *off, const int32_t *len,
		    ho_result *out);

/* Unit entry points (one call of the reference function each). */
int ho_sw_align(const char *ref, uint32_t rstart, const char *q,
		uint32_t ref_len, uint32_t len, int err, int write_bam,
		uint32_t *ops, int *n_ops, char *miss, int *n_miss, int cap);
int ho_ssw_align(const char *ref, int32_t ref_len, const char *read,
		 int32_t read_len, int *skip,
		 uint32_t *ops, int *n_ops, char *miss, int *n_miss, int cap);
uint64_t ho_get_index(const char *seq, uint32_t start);
uint32_t ho_hash_get(const ho_index *ix, uint64_t id, uint32_t *found);

/* Counters of the algorithmic work done by the last ho_align_* call. */
typedef struct {
	uint64_t lookups, hits, probes, occurrences;
	uint64_t sw_calls, sw_cells, ssw_calls, ssw_cells;
} ho_stats;
void ho_get_stats(ho_stats *s);

/* Multi-threaded timing entry: same as ho_align_pairs but splits pairs over
 * nthreads and discards results (used only for the CPU baseline leg). */
int ho_align_pairs_mt(const ho_index *ix, int write_bam, int n,
		      char *seq1, const int64_t *off1, const int32_t *len1,
		      char *seq2, const int64_t *off2, const int32_t *len2,
		      int nthreads);

/* FASTQ chunk parsing as hera's worker loops take a chunk's reads: one
 * read per get_read_from_fq_buffer call (src/read.c:11-63), pairs until
 * either file's READ_END (align_pool_pair, src/hash_align.c:1878-1929),
 * single reads until READ_END (align_pool_single, :1966-1998).  A buffer is
 * bytes [0, n) followed by a NUL; its first NUL ends it.  Offsets are byte
 * offsets into the buffer (name: the byte after '@'). */
typedef struct {
	int64_t name, seq, qual;
	int32_t name_len, len;
} ho_fq_rec;
#define HO_FQ_OK 0
#define HO_FQ_FAIL (-1)   /* READ_FAIL: the reference stops with "Wrong format" */
#define HO_FQ_CAP (-2)    /* more reads than `cap`; *n_reads holds the count */
/* out[2i], out[2i+1]: mates 1 and 2 of pair i (cap pairs); on HO_FQ_FAIL
 * *bad_file is 1 or 2 and *bad_rec the 0-based read of that file. */
int ho_parse_fq_pairs(const char *left, int64_t n_left, const char *right, int64_t n_right,
		      ho_fq_rec *out, int32_t cap, int32_t *n_pairs, int32_t *bad_file,
		      int64_t *bad_rec);
int ho_parse_fq_single(const char *buf, int64_t n, ho_fq_rec *out, int32_t cap,
		       int32_t *n_reads, int64_t *bad_rec);

/* Equivalence classes as the host tail builds them: the add_class calls of
 * align_pair_read (src/hash_align.c:1735-1760) and align_single_read
 * (:1835-1851), applied in input order to records in the flat layout.
 * State: the class table (id = XXH32 of the class's transcript list, count,
 * list), per-transcript counts of single-hit reads (REF_INF->count), PAIRED
 * and MEAN_FRAG's running sum. */
typedef struct ho_classes ho_classes;
ho_classes *ho_classes_new(uint32_t n_trans);
void ho_classes_free(ho_classes *c);
/* paired = 1: n pairs, recs[2i] / recs[2i+1] = r[0] / r[1]; paired = 0: n
 * single reads.  Returns 0, or -1 on a list entry outside the transcripts. */
int ho_classes_add(ho_classes *c, const ho_rec *recs, const uint32_t *pos_pool,
		   const int32_t *p_pool, int n, int paired);
void ho_classes_sizes(const ho_classes *c, uint32_t *n_classes, uint64_t *ref_n);
/* id/count/n/ref_off: n_classes entries; ref: ref_n; tx_count: n_trans. */
void ho_classes_export(const ho_classes *c, uint32_t *id, double *count, uint32_t *n,
		       uint64_t *ref_off, uint32_t *ref, uint32_t *tx_count,
		       uint32_t *paired, double *mean_frag);
/* estimate_count (src/EM.c:315-387): SQUAREM over M_step (:271-302) with
 * E_step's uniform start (:304-313), on a class table given as arrays
 * (class i: count[i], list ref[ref_off[i] .. + n[i])), REF_INF->count
 * (tx_count) and REF_INF->len.  Writes em_val->grama and ->overlap as the
 * reference leaves them; *rounds = the SQUAREM iterations run. */
void ho_em(uint32_t n_trans, const uint32_t *len, const uint32_t *tx_count, uint32_t n_classes,
	   const double *count, const uint32_t *n, const uint64_t *ref_off, const uint32_t *ref,
	   double *grama, double *overlap, uint32_t *rounds);

/* BAM records as the host tail writes them with `-w` (WRITE_BAM = 0):
 * align_pair_read's branches (src/hash_align.c:1735-1804) over bam_write_pair
 * (src/bam_write.c:382-416), write_alignment_pair (:349-380), pack_bam_core,
 * convert_cigar, add_padding, compact_inf and pack_bam_block (:89-310),
 * with the transcript -> genome map of reference.inf (GENE_MAP, :22-57).
 * Per pair, the uncompressed records it appends to the BGZF stream. */
typedef struct {
	uint32_t n_chr;
	const uint32_t *chr_len;     /* [n_chr] */
	const uint32_t *exon_off;    /* [n_trans + 1]: transcript t's exons are [exon_off[t], exon_off[t+1]) */
	const uint32_t *starts, *ends;
	const uint32_t *chr, *gene;  /* [n_trans] */
} ho_gene_map;
/* recs/pools: the pair records of ho_align_pairs with write_bam = 0.  Reads
 * as the tail gets them (seq after the front half, qual, NUL-terminated
 * names at name + i * name_stride); all three are modified in place as the
 * tail modifies them.  out_off[i] .. out_off[i+1]: pair i's bytes.  Returns
 * 0, or -1 if `cap` is too small. */
int ho_bam_pairs(const ho_gene_map *gm, const ho_rec *recs, const uint32_t *pos_pool,
		 const int32_t *p_pool, const uint32_t *op_pool, const char *miss_pool, int n,
		 char *seq1, const int64_t *off1, const int32_t *len1, char *qual1, char *name1,
		 char *seq2, const int64_t *off2, const int32_t *len2, char *qual2, char *name2,
		 int32_t name_stride, uint8_t *out, uint64_t cap, uint64_t *out_off);

/* The same for single reads: align_single_read's writes (src/hash_align.c:
 * 1825-1834) over bam_write_single (src/bam_write.c:418-446); recs from
 * ho_align_single with write_bam = 0. */
int ho_bam_single(const ho_gene_map *gm, const ho_rec *recs, const uint32_t *pos_pool,
		  const int32_t *p_pool, const uint32_t *op_pool, const char *miss_pool, int n,
		  char *seq, const int64_t *off, const int32_t *len, char *qual, char *name,
		  int32_t name_stride, uint8_t *out, uint64_t cap, uint64_t *out_off);

/* XXH32 (the published xxHash 32-bit algorithm) as add_class uses it. */
uint32_t ho_xxh32(const void *buf, size_t len, uint32_t seed);

#ifdef __cplusplus
}
#endif
#endif
