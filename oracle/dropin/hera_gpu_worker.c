/*
 * hera_gpu_worker.c -- hera's paired-end worker loop on the B200 library,
 * for checking the drop-in end to end inside hera itself.
 *
 * INTEGRATION TEST INFRASTRUCTURE: built by oracle/Makefile into
 * oracle/_ref/hera_gpu from the reference's own sources, unchanged, plus
 * this file.  objcopy makes three definitions of the reference's
 * hash_align.o weak, and this file supplies them:
 *
 *   align_pool_pair (src/hash_align.c:1855-1946): the same chunk loop, but
 *     each chunk's reads are parsed first (get_read_from_fq_buffer /
 *     get_read_from_fa_buffer, as the loop does), aligned in one
 *     hera_gpu_align_pairs call, and then handed one pair at a time, in
 *     input order, to the reference's unchanged align_pair_read
 *     (src/hash_align.c:1716-1812);
 *   check_in_transcriptome (src/hash_align.c:1663-1695): hands
 *     align_pair_read the pair's two Candidates from the device;
 *   intersect2 (src/hash_align.c:1524-1562): nothing -- the device's
 *     Candidates are already the state after align_pair_read's two
 *     intersect2 calls (src/hash_align.c:1730-1733).
 *
 * So align_pair_read's host tail -- pair choice, check_in_genome, the BAM
 * records, add_class, the counters -- runs as the reference's own code on
 * the device's Candidates.  The index, the chunking, the EM and the output
 * files are the reference's.  The library's context is made from the loaded
 * KMER_HASH / REF_INF on the first chunk.  The worker threads call the
 * library without a lock (it combines concurrent calls into one device
 * batch); run with -t 1 for the reference's add_class order.
 */
#include <pthread.h>
#include <time.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hash_align.h"
#include "get_buffer.h"
#include "read.h"
#include "macros.h"

#include "hera_gpu.h"

static hera_gpu_ctx *CTX;
static pthread_mutex_t GPU_LOCK = PTHREAD_MUTEX_INITIALIZER;
static pthread_mutex_t CNT_LOCK = PTHREAD_MUTEX_INITIALIZER;
static __thread Candidate **CUR;      /* the current pair's r[0], r[1] */
static __thread int CUR_TAKEN;
static unsigned long long GPU_PAIRS, GPU_CALLS;
static double CALL_MS, TAIL_MS, PARSE_MS;

static double now_ms(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec * 1e3 + ts.tv_nsec / 1e6;
}

static void report(void)
{
	fprintf(stderr, "hera_gpu: %llu pairs aligned on the device in %llu calls\n", GPU_PAIRS, GPU_CALLS);
	fprintf(stderr, "hera_gpu: worker threads' time: parsing %.1f ms, in hera_gpu_align_pairs %.1f ms "
		"(combined batches included), hera's tail %.1f ms\n", PARSE_MS, CALL_MS, TAIL_MS);
}

static void make_context(void)
{
	unsigned long long nb = 0;
	for (unsigned int i = 0; i < H; ++i)
		nb += KMER_HASH->n[i];
	hera_gpu_index_view v;
	memset(&v, 0, sizeof v);
	v.n_trans = REF_INF->n;
	v.len = REF_INF->len;
	v.find = REF_INF->find;
	v.seq = REF_INF->seq;
	v.bucket_n = KMER_HASH->n;
	v.buckets = (const hera_bucket *)KMER_HASH->sentinel;
	v.n_buckets = nb;
	v.pos = KMER_HASH->pos;
	v.p = KMER_HASH->p;
	v.n_pos = KMER_HASH->n_pos;
	hera_gpu_options o;
	memset(&o, 0, sizeof o);
	if (hera_gpu_ctx_create(&v, &o, &CTX) != HERA_GPU_OK) {
		fprintf(stderr, "hera_gpu: no usable CUDA device\n");
		exit(1);
	}
	atexit(report);
}

void check_in_transcriptome(struct read_inf *r1, struct read_inf *r2, Candidate *r[])
{
	(void)r1;
	(void)r2;
	destroy_candidate(r[0]);
	destroy_candidate(r[1]);
	r[0] = CUR[0];
	r[1] = CUR[1];
	CUR_TAKEN = 1;
}

void intersect2(Candidate *r, struct read_inf *read1, struct read_inf *read2, unsigned int add)
{
	(void)r;
	(void)read1;
	(void)read2;
	(void)add;
}

void *align_pool_pair(void *thr_data)
{
	struct gb_pair_data *data = (struct gb_pair_data *)thr_data;
	struct gb_pair_buf *buffer;
	char *stream = malloc(MAX_COMPRESS);
	uint32_t slen = 0;
	int32_t cap = 0;
	struct read_inf *L = NULL, *R = NULL;

	pthread_mutex_lock(&GPU_LOCK);
	if (!CTX)
		make_context();
	pthread_mutex_unlock(&GPU_LOCK);
	while (1) {
		pthread_mutex_lock(&LOCK);
		buffer = gb_get_pair(data);
		pthread_mutex_unlock(&LOCK);
		if (buffer->left == NULL && buffer->right == NULL)
			break;
		if (buffer->left == NULL || buffer->right == NULL) {
			data->warning_flag = true;
			break;
		}
		/* every read pair of the chunk, with the loop's stop rules */
		double t0 = now_ms();
		int32_t left_pos = 0, right_pos = 0, n = 0, len_read = 0;
		while (1) {
			if (n == cap) {
				cap = cap ? 2 * cap : 16384;
				L = realloc(L, (size_t)cap * sizeof *L);
				R = realloc(R, (size_t)cap * sizeof *R);
			}
			int rc1 = data->format == TYPE_FASTQ ? get_read_from_fq_buffer(&L[n], buffer->left, &left_pos)
							      : get_read_from_fa_buffer(&L[n], buffer->left, &left_pos);
			if (rc1 == READ_FAIL) {
				_verbose("\n");
				_error("Wrong format of file: %s\n", data->left->file_name);
			}
			int rc2 = data->format == TYPE_FASTQ ? get_read_from_fq_buffer(&R[n], buffer->right, &right_pos)
							      : get_read_from_fa_buffer(&R[n], buffer->right, &right_pos);
			if (rc2 == READ_FAIL) {
				_verbose("\n");
				_error("Wrong format of file: %s\n", data->right->file_name);
			}
			if (data->format == TYPE_FASTA) {   /* the loop's fake qualities */
				L[n].qual = malloc(L[n].len + 1);
				R[n].qual = malloc(R[n].len + 1);
				memset(L[n].qual, 'A', L[n].len);
				memset(R[n].qual, 'A', R[n].len);
				L[n].qual[L[n].len] = R[n].qual[R[n].len] = 0;
			}
			len_read += L[n].len + R[n].len;
			++n;
			if (rc1 || rc2 == READ_END)
				break;
		}
		/* one device call for the chunk */
		Candidate **cand = malloc(2 * (size_t)n * sizeof *cand);
		double t1 = now_ms();
		/* no lock: the library combines the calls that the worker threads
		   make at the same time into one device batch */
		int st = hera_gpu_align_pairs(CTX, (hera_read_inf *)L, (hera_read_inf *)R, n, (int)WRITE_BAM,
					      (hera_candidate **)cand);
		double t3 = now_ms();
		pthread_mutex_lock(&CNT_LOCK);
		PARSE_MS += t1 - t0;
		CALL_MS += t3 - t1;
		GPU_PAIRS += (unsigned long long)n;
		GPU_CALLS += 1;
		pthread_mutex_unlock(&CNT_LOCK);
		if (st != HERA_GPU_OK)
			_error("GPU alignment failed: %s\n", hera_gpu_last_error(CTX));
		/* the reference's tail, per pair in input order */
		for (int32_t i = 0; i < n; ++i) {
			CUR = &cand[2 * i];
			CUR_TAKEN = 0;
			align_pair_read(&L[i], &R[i], stream, &slen);
			if (!CUR_TAKEN)   /* align_pair_read returned before its front half */
				hera_gpu_free_candidates((hera_candidate **)&cand[2 * i], 2);
			if (data->format == TYPE_FASTA) {
				free(L[i].qual);
				free(R[i].qual);
			}
		}
		free(cand);
		pthread_mutex_lock(&CNT_LOCK);
		TAIL_MS += now_ms() - t3;
		N_READ += n;
		MEAN_LEN += len_read;
		_verbose("\rNumber of processed read pairs: %u", N_READ);
		pthread_mutex_unlock(&CNT_LOCK);
		gb_destroy_pair_buf(buffer);
	}
	if (slen > 0 && WRITE_BAM == 0)
		bam_write(BAM, stream, slen);
	free(L);
	free(R);
	free(stream);
	pthread_exit(NULL);
	return NULL;
}
