/*
 * ref_harness.c -- ctypes entry points into the reference program, compiled
 * together with the reference's own sources into oracle/_ref/libhera_ref.so
 * by oracle/Makefile.  TEST INFRASTRUCTURE ONLY (golden vectors and the CPU
 * baseline timing); the product never links or loads it.
 *
 * Every alignment result here comes from the reference's functions run
 * unchanged: check_in_transcriptome + intersect2 (the front half of
 * align_pair_read, src/hash_align.c:1724-1733), get_position x2 (front half
 * of align_single_read, src/hash_align.c:1819-1823), SW_align and ssw_align.
 * This file only sets the reference's globals and flattens its Candidate
 * structs into the records the tests compare.
 */
#include "hash_align.h"
#include "ssw.h"
#include "EM.h"

#include <stdint.h>
#include <pthread.h>

/* defined in src/hash_align.c without a header prototype */
void check_in_transcriptome(struct read_inf *r1, struct read_inf *r2, Candidate *r[]);
void intersect2(Candidate *r, struct read_inf *read1, struct read_inf *read2, unsigned int add);
void destroy_candidate(Candidate *read);
Cigar *ssw_align(char *ref_seq, int32_t ref_len, char *read_seq, int32_t read_len,
		 int *score, int *skip);

typedef struct {
	int32_t n[2];
	int32_t err[2];
	int32_t pair;
	uint32_t list_off[2];
	uint32_t cig_off[2];
	uint32_t miss_off[2];
	uint16_t n_cigar[2];
	uint16_t n_miss[2];
} refh_rec;

typedef struct {
	refh_rec *recs;
	uint32_t *pos_pool;
	int32_t *p_pool;
	uint32_t *op_pool;
	char *miss_pool;
	uint64_t list_cap, op_cap, miss_cap;
	uint64_t list_used, op_used, miss_used;
} refh_result;

/* Load <dir>/index with the reference's own loader (src/hash_align.c:1195). */
int refh_load_index(const char *dir)
{
	init_refInf();
	init_hash();
	load_index((char *)dir, NULL);
	return 0;
}

/* Install an index held in caller memory into the reference's globals, in
 * the layout load_hash builds (src/hash_align.c:1169-1193).  `seq` must stay
 * alive and carry zero bytes after the last transcript.  Arrays are
 * borrowed, not copied. */
int refh_set_index(uint32_t n_trans, uint32_t name_len, uint32_t *len,
		   uint32_t *find, char *seq, uint32_t *bucket_n,
		   Bucket *buckets, uint32_t *pos, uint32_t *p, uint32_t n_pos)
{
	uint64_t i, count = 0;

	REF_INF = calloc(1, sizeof(Ref_inf));
	REF_INF->n = n_trans;
	REF_INF->name_len = name_len;
	REF_INF->len = len;
	REF_INF->find = find;
	REF_INF->seq = seq;
	REF_INF->count = calloc(n_trans, sizeof(int));
	REF_INF->eff_len = calloc(n_trans, sizeof(double));

	KMER_HASH = calloc(1, sizeof(Kmer_hash));
	KMER_HASH->n = bucket_n;
	KMER_HASH->bucket = calloc((uint64_t)H + 1, sizeof(Bucket *));
	KMER_HASH->sentinel = buckets;
	for (i = 0; i < H; ++i) {
		KMER_HASH->bucket[i] = buckets + count;
		count += bucket_n[i];
	}
	KMER_HASH->pos = pos;
	KMER_HASH->p = p;
	KMER_HASH->n_pos = n_pos;
	KMER_HASH->is_loaded = 1;
	FMINDEX = NULL;
	return 0;
}

/* Copy the loaded index out (used to check an index builder against
 * `hera index`): sizes first with NULL buffers. */
int refh_index_sizes(uint32_t *n_trans, uint32_t *name_len, uint64_t *seq_len,
		     uint64_t *n_buckets, uint32_t *n_pos)
{
	uint64_t i, count = 0;
	*n_trans = REF_INF->n;
	*name_len = REF_INF->name_len;
	*seq_len = REF_INF->find[REF_INF->n - 1];
	for (i = 0; i < H; ++i)
		count += KMER_HASH->n[i];
	*n_buckets = count;
	*n_pos = KMER_HASH->n_pos;
	return 0;
}

void refh_set_write_bam(int v)
{
	WRITE_BAM = (unsigned)v;
}

static int emit(refh_result *out, uint64_t ri, Candidate *c)
{
	refh_rec *rec = &out->recs[ri];
	int s;

	rec->pair = c->pair;
	for (s = 0; s < 2; ++s) {
		Cigar *g = c->cigar[s];
		int j;
		rec->n[s] = (int32_t)c->n[s];
		rec->err[s] = c->err[s];
		if (out->list_used + c->n[s] > out->list_cap ||
		    out->op_used + g->n_cigar > out->op_cap ||
		    out->miss_used + g->n_miss > out->miss_cap)
			return -1;
		rec->list_off[s] = (uint32_t)out->list_used;
		if (c->n[s]) {
			memcpy(out->pos_pool + out->list_used, c->pos[s], c->n[s] * sizeof(uint32_t));
			memcpy(out->p_pool + out->list_used, c->p[s], c->n[s] * sizeof(int32_t));
		}
		out->list_used += c->n[s];
		rec->cig_off[s] = (uint32_t)out->op_used;
		rec->n_cigar[s] = g->n_cigar;
		for (j = 0; j < g->n_cigar; ++j)
			out->op_pool[out->op_used + j] =
				((uint32_t)g->count[j] << 4) | (uint32_t)(uint8_t)g->type[j];
		out->op_used += g->n_cigar;
		rec->miss_off[s] = (uint32_t)out->miss_used;
		rec->n_miss[s] = g->n_miss;
		if (g->n_miss)
			memcpy(out->miss_pool + out->miss_used, g->miss, g->n_miss);
		out->miss_used += g->n_miss;
	}
	return 0;
}

static void front_half_pair(struct read_inf *a, struct read_inf *b, Candidate *r[2])
{
	r[0] = init_candidate();
	r[1] = init_candidate();
	check_in_transcriptome(a, b, r);
	if (r[0]->n[0] > 0 && r[0]->n[1] > 0)
		intersect2(r[0], a, b, MAX_FRAG);
	if (r[1]->n[0] > 0 && r[1]->n[1] > 0)
		intersect2(r[1], b, a, MAX_FRAG);
}

int refh_align_pairs(int write_bam, int n,
		     char *seq1, const int64_t *off1, const int32_t *len1,
		     char *seq2, const int64_t *off2, const int32_t *len2,
		     refh_result *out)
{
	int i, rc = 0;
	char name[] = "r";

	WRITE_BAM = (unsigned)write_bam;
	out->list_used = out->op_used = out->miss_used = 0;
	for (i = 0; i < n && rc == 0; ++i) {
		struct read_inf a = {seq1 + off1[i], name, NULL, len1[i]};
		struct read_inf b = {seq2 + off2[i], name, NULL, len2[i]};
		Candidate *r[2];
		front_half_pair(&a, &b, r);
		rc = emit(out, 2 * (uint64_t)i, r[0]);
		if (rc == 0)
			rc = emit(out, 2 * (uint64_t)i + 1, r[1]);
		destroy_candidate(r[0]);
		destroy_candidate(r[1]);
	}
	return rc;
}

int refh_align_single(int write_bam, int n, char *seq, const int64_t *off,
		      const int32_t *len, refh_result *out)
{
	int i, rc = 0;
	char name[] = "r";

	WRITE_BAM = (unsigned)write_bam;
	out->list_used = out->op_used = out->miss_used = 0;
	for (i = 0; i < n && rc == 0; ++i) {
		struct read_inf a = {seq + off[i], name, NULL, len[i]};
		Candidate *r = init_candidate();
		get_position(&a, r, 0, 2 * ERR);
		get_position(&a, r, 1, 2 * ERR);
		rc = emit(out, (uint64_t)i, r);
		destroy_candidate(r);
	}
	return rc;
}

static int export_cigar(Cigar *c, uint32_t *ops, int *n_ops, char *miss,
			int *n_miss, int cap)
{
	int j;
	if (c->n_cigar > cap || c->n_miss > cap)
		return -1;
	for (j = 0; j < c->n_cigar; ++j)
		ops[j] = ((uint32_t)c->count[j] << 4) | (uint32_t)(uint8_t)c->type[j];
	*n_ops = c->n_cigar;
	if (c->n_miss)
		memcpy(miss, c->miss, c->n_miss);
	*n_miss = c->n_miss;
	return 0;
}

int refh_sw_align(int write_bam, char *ref, uint32_t rstart, char *q,
		  uint32_t ref_len, uint32_t len, int err,
		  uint32_t *ops, int *n_ops, char *miss, int *n_miss, int cap)
{
	int score = 0, rc;
	Cigar *c;
	WRITE_BAM = (unsigned)write_bam;
	c = SW_align(ref, rstart, q, ref_len, len, &score, (short)err);
	rc = export_cigar(c, ops, n_ops, miss, n_miss, cap);
	free_cigar(c);
	return rc < 0 ? -1000000 : score;
}

int refh_ssw_align(char *ref, int32_t ref_len, char *read, int32_t read_len,
		   int *skip, uint32_t *ops, int *n_ops, char *miss, int *n_miss,
		   int cap)
{
	int score = 0, rc;
	Cigar *c = ssw_align(ref, ref_len, read, read_len, &score, skip);
	rc = export_cigar(c, ops, n_ops, miss, n_miss, cap);
	free_cigar(c);
	return rc < 0 ? -1000000 : score;
}

/* ---- multi-threaded timing (CPU baseline): results are discarded ---- */
typedef struct {
	int lo, hi;
	char *seq1, *seq2;
	const int64_t *off1, *off2;
	const int32_t *len1, *len2;
} refh_job;

static void *refh_worker(void *arg)
{
	refh_job *j = arg;
	char name[] = "r";
	int i;
	for (i = j->lo; i < j->hi; ++i) {
		struct read_inf a = {j->seq1 + j->off1[i], name, NULL, j->len1[i]};
		struct read_inf b = {j->seq2 + j->off2[i], name, NULL, j->len2[i]};
		Candidate *r[2];
		front_half_pair(&a, &b, r);
		destroy_candidate(r[0]);
		destroy_candidate(r[1]);
	}
	return NULL;
}

int refh_align_pairs_mt(int write_bam, int n,
			char *seq1, const int64_t *off1, const int32_t *len1,
			char *seq2, const int64_t *off2, const int32_t *len2,
			int nthreads)
{
	pthread_t *th;
	refh_job *jobs;
	pthread_attr_t attr;
	int t;

	WRITE_BAM = (unsigned)write_bam;
	if (nthreads < 1)
		nthreads = 1;
	th = calloc(nthreads, sizeof(pthread_t));
	jobs = calloc(nthreads, sizeof(refh_job));
	pthread_attr_init(&attr);
	pthread_attr_setstacksize(&attr, THREAD_STACK_SIZE);
	for (t = 0; t < nthreads; ++t) {
		refh_job *j = &jobs[t];
		j->lo = (int)((int64_t)n * t / nthreads);
		j->hi = (int)((int64_t)n * (t + 1) / nthreads);
		j->seq1 = seq1; j->seq2 = seq2;
		j->off1 = off1; j->off2 = off2;
		j->len1 = len1; j->len2 = len2;
		pthread_create(&th[t], &attr, refh_worker, j);
	}
	for (t = 0; t < nthreads; ++t)
		pthread_join(th[t], NULL);
	pthread_attr_destroy(&attr);
	free(th);
	free(jobs);
	return 0;
}

/* ---- FASTQ chunk parsing ------------------------------------------------ */

/* The reference's read loop of align_pool_pair (src/hash_align.c:1878-1929)
 * over two chunk buffers, each a writable NUL-terminated copy: every read
 * comes from the reference's get_read_from_fq_buffer (src/read.c:11-63);
 * a READ_FAIL, where the reference calls _error, is returned with its file
 * (1 or 2) and read index.  rec: per read {name, seq, qual} offsets into its
 * buffer and {name length, len}, as int64 x5; 0 ok, -1 fail, -2 over cap. */
int refh_parse_fq_pairs(char *left, char *right, int64_t *rec, int32_t cap, int32_t *n_pairs,
			int32_t *bad_file, int64_t *bad_rec)
{
	struct read_inf a, b;
	int32_t lp = 0, rp = 0, k = 0;
	*n_pairs = 0;
	*bad_file = 0;
	*bad_rec = -1;
	for (;;) {
		enum read_exit_code c1 = get_read_from_fq_buffer(&a, left, &lp);
		if (c1 == READ_FAIL) {
			*bad_file = 1;
			*bad_rec = k;
			return -1;
		}
		enum read_exit_code c2 = get_read_from_fq_buffer(&b, right, &rp);
		if (c2 == READ_FAIL) {
			*bad_file = 2;
			*bad_rec = k;
			return -1;
		}
		if (k < cap) {
			int64_t *o = rec + 10 * (int64_t)k;
			o[0] = a.name - left;
			o[1] = a.seq - left;
			o[2] = a.qual - left;
			o[3] = (int64_t)strlen(a.name);
			o[4] = a.len;
			o[5] = b.name - right;
			o[6] = b.seq - right;
			o[7] = b.qual - right;
			o[8] = (int64_t)strlen(b.name);
			o[9] = b.len;
		}
		++k;
		if (c1 || c2 == READ_END)
			break;
	}
	*n_pairs = k;
	return k > cap ? -2 : 0;
}

/* align_pool_single's read loop (src/hash_align.c:1966-1998) */
int refh_parse_fq_single(char *buf, int64_t *rec, int32_t cap, int32_t *n_reads, int64_t *bad_rec)
{
	struct read_inf a;
	int32_t p = 0, k = 0;
	*n_reads = 0;
	*bad_rec = -1;
	for (;;) {
		enum read_exit_code c = get_read_from_fq_buffer(&a, buf, &p);
		if (c == READ_FAIL) {
			*bad_rec = k;
			return -1;
		}
		if (k < cap) {
			int64_t *o = rec + 5 * (int64_t)k;
			o[0] = a.name - buf;
			o[1] = a.seq - buf;
			o[2] = a.qual - buf;
			o[3] = (int64_t)strlen(a.name);
			o[4] = a.len;
		}
		++k;
		if (c == READ_END)
			break;
	}
	*n_reads = k;
	return k > cap ? -2 : 0;
}

/* ---- equivalence classes: the reference's whole per-read worker ---------
 * align_pair_read / align_single_read (src/hash_align.c:1717-1853) run
 * unchanged with WRITE_BAM = 1 (no `-w`: bam_write_pair and
 * bam_write_single return at once, src/bam_write.c:386-387, 421-422), on a
 * fresh class table (init_class, :1161-1167) and zeroed REF_INF->count,
 * PAIRED and MEAN_FRAG.  The sequences are modified in place (the tail's
 * reverse_str calls), so callers pass copies.  Afterwards refh_classes_*
 * read the add_class state back. */
void init_class();
void align_pair_read(struct read_inf *r1, struct read_inf *r2, char *stream, unsigned int *slen);
void align_single_read(struct read_inf *read, char *stream, unsigned int *slen);
unsigned int XXH32(const void *input, size_t len, unsigned int seed);

static void classes_reset(void)
{
	uint32_t i;
	if (CLASS) {
		for (i = 0; i < CLASS->n; ++i)
			if (CLASS->cls[i].n)
				free(CLASS->cls[i].ref);
		free(CLASS->cls);
		free(CLASS->map);
		free(CLASS);
		CLASS = NULL;
	}
	init_class();
	memset(REF_INF->count, 0, REF_INF->n * sizeof(int));
	PAIRED = 0;
	MEAN_FRAG = 0;
}

int refh_classes_run(int paired, int n, char *seq1, const int64_t *off1, const int32_t *len1,
		     char *seq2, const int64_t *off2, const int32_t *len2)
{
	int i, max_len = 1;
	char name[] = "r/1";
	unsigned int slen = 0;
	char *q1, *q2;

	/* the tail reverses the quality strings with the sequences */
	for (i = 0; i < n; ++i) {
		if (len1[i] > max_len)
			max_len = len1[i];
		if (paired && len2[i] > max_len)
			max_len = len2[i];
	}
	q1 = malloc(max_len + 1);
	q2 = malloc(max_len + 1);
	WRITE_BAM = 1;
	classes_reset();
	for (i = 0; i < n; ++i) {
		struct read_inf a = {seq1 + off1[i], name, q1, len1[i]};
		if (paired) {
			struct read_inf b = {seq2 + off2[i], name, q2, len2[i]};
			align_pair_read(&a, &b, NULL, &slen);
		} else {
			align_single_read(&a, NULL, &slen);
		}
	}
	free(q1);
	free(q2);
	return 0;
}

void refh_classes_sizes(uint32_t *n_classes, uint64_t *ref_n)
{
	uint64_t s = 0;
	uint32_t i;
	for (i = 0; i < CLASS->n; ++i)
		s += CLASS->cls[i].n;
	*n_classes = CLASS->n;
	*ref_n = s;
}

void refh_classes_export(uint32_t *id, double *count, uint32_t *n, uint64_t *ref_off,
			 uint32_t *ref, uint32_t *tx_count, uint32_t *paired, double *mean_frag)
{
	uint64_t s = 0;
	uint32_t i;
	for (i = 0; i < CLASS->n; ++i) {
		id[i] = CLASS->cls[i].id;
		count[i] = CLASS->cls[i].count;
		n[i] = CLASS->cls[i].n;
		ref_off[i] = s;
		if (CLASS->cls[i].n)
			memcpy(ref + s, CLASS->cls[i].ref, CLASS->cls[i].n * sizeof(uint32_t));
		s += CLASS->cls[i].n;
	}
	memcpy(tx_count, REF_INF->count, REF_INF->n * sizeof(uint32_t));
	*paired = PAIRED;
	*mean_frag = MEAN_FRAG;
}

unsigned int refh_xxh32(const void *buf, size_t len, unsigned int seed)
{
	return XXH32(buf, len, seed);
}

/* ---- the EM: the reference's estimate_count (src/EM.c:315-387) ----------
 * run on a class table given as arrays (installed as CLASS, with the
 * per-transcript counts as REF_INF->count), on the installed index's
 * REF_INF->len; em_val->grama and ->overlap are copied out. */
EM_val *estimate_count(unsigned int *count, unsigned int order);

int refh_em(uint32_t n_classes, const double *count, const uint32_t *n, const uint64_t *ref_off,
	    const uint32_t *ref, const uint32_t *tx_count, double *grama, double *overlap)
{
	uint32_t i;
	Gclass *saved = CLASS;
	Gclass g;
	EM_val *em;

	g.n = n_classes;
	g.map = NULL;
	g.cls = calloc(n_classes ? n_classes : 1, sizeof(Class));
	for (i = 0; i < n_classes; ++i) {
		g.cls[i].n = n[i];
		g.cls[i].ref = (unsigned int *)(ref + ref_off[i]);
		g.cls[i].count = count[i];
		g.cls[i].id = 0;
	}
	CLASS = &g;
	memcpy(REF_INF->count, tx_count, REF_INF->n * sizeof(uint32_t));
	em = estimate_count(REF_INF->count, 0);
	memcpy(grama, em->grama, REF_INF->n * sizeof(double));
	memcpy(overlap, em->overlap, REF_INF->n * sizeof(double));
	free(em->grama);
	free(em->overlap);
	free(em);
	free(g.cls);
	CLASS = saved;
	return 0;
}

/* ---- BAM records: the tail's bam_write_pair calls -----------------------
 * refh_bam_setup loads an index directory written by hera_build + `hera
 * index` with the reference's loader (load_index, src/hash_align.c:1195)
 * and builds GENE_MAP from its reference.inf through init_bam_header
 * (src/bam_write.c:448-495) with WRITE_BAM = 1, so nothing is written.
 * refh_bam_pairs then runs align_pair_read (src/hash_align.c:1717-1812)
 * with WRITE_BAM = 0 (`-w`) for each pair and copies out the uncompressed
 * BAM records the tail appended to the stream (bam_write_pair,
 * src/bam_write.c:382-416), pair by pair.  Names and qualities are
 * modified in place (the writer trims "/1", the tail reverses qualities). */
void init_bam_header(char *idx_dir, int argc, char *argv[]);
void init_class();

int refh_bam_setup(const char *dir)
{
	char *argv[] = {"hera", NULL};
	WRITE_BAM = 1;
	init_refInf();
	init_hash();
	load_index((char *)dir, NULL);
	init_bam_header((char *)dir, 1, argv);
	if (!CLASS)
		init_class();
	return REF_INF->n;
}

int refh_bam_pairs(int n, char *seq1, const int64_t *off1, const int32_t *len1, char *qual1, char *name1,
		   char *seq2, const int64_t *off2, const int32_t *len2, char *qual2, char *name2,
		   int32_t name_stride, uint8_t *out, uint64_t cap, uint64_t *out_off)
{
	int i;
	char *stream = malloc(MAX_COMPRESS + 1);
	uint64_t used = 0;

	WRITE_BAM = 0;
	for (i = 0; i < n; ++i) {
		unsigned int slen = 0;
		struct read_inf a = {seq1 + off1[i], name1 + (int64_t)i * name_stride, qual1 + off1[i], len1[i]};
		struct read_inf b = {seq2 + off2[i], name2 + (int64_t)i * name_stride, qual2 + off2[i], len2[i]};
		out_off[i] = used;
		align_pair_read(&a, &b, stream, &slen);
		if (used + slen > cap) {
			free(stream);
			WRITE_BAM = 1;
			return -1;
		}
		memcpy(out + used, stream, slen);
		used += slen;
	}
	out_off[n] = used;
	free(stream);
	WRITE_BAM = 1;
	return 0;
}

/* The same for single reads: align_single_read (src/hash_align.c:1814-1853)
 * with WRITE_BAM = 0, the records bam_write_single appends, read by read. */
int refh_bam_single(int n, char *seq, const int64_t *off, const int32_t *len, char *qual, char *name,
		    int32_t name_stride, uint8_t *out, uint64_t cap, uint64_t *out_off)
{
	int i;
	char *stream = malloc(MAX_COMPRESS + 1);
	uint64_t used = 0;

	WRITE_BAM = 0;
	for (i = 0; i < n; ++i) {
		unsigned int slen = 0;
		struct read_inf a = {seq + off[i], name + (int64_t)i * name_stride, qual + off[i], len[i]};
		out_off[i] = used;
		align_single_read(&a, stream, &slen);
		if (used + slen > cap) {
			free(stream);
			WRITE_BAM = 1;
			return -1;
		}
		memcpy(out + used, stream, slen);
		used += slen;
	}
	out_off[n] = used;
	free(stream);
	WRITE_BAM = 1;
	return 0;
}
