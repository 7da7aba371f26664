/*
 * hera_oracle.c -- CPU restatement of hera's read-alignment hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * path in hera_b200/; the product never links, loads or calls it.  It is
 * written from the reference's behaviour (each function cites the reference
 * file:line it restates) and is itself pinned against the reference program
 * compiled from its own sources (oracle/_ref, built by oracle/Makefile) via
 * tests/golden/ fixtures and live comparisons in the CPU test suite.
 *
 * Behaviour the reference leaves undefined, and what this file does instead:
 *  - SW_align's shrink loop reads r[-1] at column 0 (src/hash_align.c:705).
 *    The term it feeds is ANDed with matrix[k][0] == matrix[k-1][-1]; for
 *    every call the live seed spacings (14 and 31) can make, that equality
 *    is false, so the byte is irrelevant.  Here r[-1] never matches.
 *  - The suffix window may read up to 7 bytes past the last transcript
 *    (src/hash_align.c:1290-1293 with :1223).  The reference's buffer is
 *    mmap-backed at any real size, so those bytes read as zero; the index
 *    view here must carry >= 8 zero bytes after the last transcript.
 *  - Bytes >= 128 index the reference's tables with a negative char; here
 *    they code as 4 (not ACGT).
 */
#include "hera_oracle.h"

#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <pthread.h>

enum { OP_M = 0, OP_I = 1, OP_D = 2, OP_S = 4, OP_X = 8 };

/* ascii_table (src/hash_align.c:6-23) and ascii2int (src/ssw.c:46-56):
 * A/a=0 C/c=1 G/g=2 T/t=3, anything else 4. */
static uint8_t CODE[256];
static const char ACGT[4] = {'A', 'C', 'G', 'T'};

__attribute__((constructor)) static void code_init(void)
{
	int i;
	for (i = 0; i < 256; ++i)
		CODE[i] = 4;
	CODE['A'] = CODE['a'] = 0;
	CODE['C'] = CODE['c'] = 1;
	CODE['G'] = CODE['g'] = 2;
	CODE['T'] = CODE['t'] = 3;
}

#define CD(c) CODE[(uint8_t)(c)]

/* ------------------------------------------------------------------ */
/* work counters                                                      */
/* ------------------------------------------------------------------ */
static __thread ho_stats *ST;
static ho_stats G_STATS;
void ho_get_stats(ho_stats *s) { *s = G_STATS; }
#define COUNT(field, v) do { if (ST) ST->field += (v); } while (0)

/* ------------------------------------------------------------------ */
/* CIGAR algebra                                                      */
/* ------------------------------------------------------------------ */
typedef struct {
	int n, cap;
	uint16_t *cnt;
	uint8_t *op;
	int nm, mcap;
	char *miss;
} ocig;

static void *xrealloc(void *p, size_t sz)
{
	void *q = realloc(p, sz ? sz : 1);
	if (!q)
		abort();
	return q;
}

static void cig_free(ocig *c)
{
	free(c->cnt);
	free(c->op);
	free(c->miss);
	memset(c, 0, sizeof(*c));
}

static void cig_clear(ocig *c)
{
	c->n = 0;
	c->nm = 0;
}

static void cig_swap(ocig *a, ocig *b)
{
	ocig t = *a;
	*a = *b;
	*b = t;
}

/* add_cigar (src/hash_align.c:526-565): merge with an equal last op; once
 * the last op is a soft clip and there are >= 2 ops, every later non-D op
 * is absorbed into the clip and a D is dropped, with no miss chars. */
static void cig_add(ocig *c, int op, unsigned add, const char *mc)
{
	add &= 0xffff;
	if (add == 0)
		return;
	if (c->n > 1 && c->op[c->n - 1] == OP_S) {
		if (op != OP_D)
			c->cnt[c->n - 1] = (uint16_t)(c->cnt[c->n - 1] + add);
		return;
	}
	if (mc) {
		if (c->nm + (int)add > c->mcap) {
			c->mcap = (c->nm + add) * 2 + 8;
			c->miss = xrealloc(c->miss, c->mcap);
		}
		memcpy(c->miss + c->nm, mc, add);
		c->nm += add;
	}
	if (c->n > 0 && c->op[c->n - 1] == op) {
		c->cnt[c->n - 1] = (uint16_t)(c->cnt[c->n - 1] + add);
		return;
	}
	if (c->n == c->cap) {
		c->cap = c->cap * 2 + 8;
		c->cnt = xrealloc(c->cnt, c->cap * sizeof(uint16_t));
		c->op = xrealloc(c->op, c->cap);
	}
	c->op[c->n] = (uint8_t)op;
	c->cnt[c->n] = (uint16_t)add;
	c->n++;
}

/* reverse_cigar (src/hash_align.c:567-587): ops and miss chars reversed. */
static void cig_reverse(ocig *c)
{
	int i;
	for (i = 0; i < c->n / 2; ++i) {
		uint16_t t = c->cnt[i];
		uint8_t o = c->op[i];
		c->cnt[i] = c->cnt[c->n - 1 - i];
		c->op[i] = c->op[c->n - 1 - i];
		c->cnt[c->n - 1 - i] = t;
		c->op[c->n - 1 - i] = o;
	}
	for (i = 0; i < c->nm / 2; ++i) {
		char t = c->miss[i];
		c->miss[i] = c->miss[c->nm - 1 - i];
		c->miss[c->nm - 1 - i] = t;
	}
}

/* concat_cigar (src/hash_align.c:589-603): reverse `t` in place, append
 * its ops to `d`, carrying miss chars for D and X runs. */
static void cig_concat(ocig *d, ocig *t)
{
	int i, k = 0;
	cig_reverse(t);
	for (i = 0; i < t->n; ++i) {
		if (t->op[i] == OP_D || t->op[i] == OP_X) {
			cig_add(d, t->op[i], t->cnt[i], t->miss + k);
			k += t->cnt[i];
		} else {
			cig_add(d, t->op[i], t->cnt[i], NULL);
		}
	}
}

/* ------------------------------------------------------------------ */
/* SW_align: error-capped unit-cost DP (src/hash_align.c:627-760)      */
/* ------------------------------------------------------------------ */
static int o_sw_align(const char *ref, uint32_t rstart, const char *str,
		      uint32_t ref_len, uint32_t len, int err, int write_bam,
		      ocig *cig)
{
	unsigned error = (unsigned)(err < 0 ? -err : err) + 1;
	unsigned s = 0, min = 0, xmin = 0, pen, W = ref_len + 1;
	int i, k, j, ferr = -1, score = 0;
	size_t cells;
	uint16_t *M;
	char *r, *q;

	cig_clear(cig);
	if (len == 0)
		return 0;

	r = malloc(ref_len + 1);
	q = malloc(len + 1);
	memcpy(r, ref + rstart, ref_len);
	memcpy(q, str, len);
	if (err < 0) {   /* prefix DP runs on both strings reversed */
		for (i = 0; i < (int)ref_len / 2; ++i) {
			char t = r[i]; r[i] = r[ref_len - 1 - i]; r[ref_len - 1 - i] = t;
		}
		for (i = 0; i < (int)len / 2; ++i) {
			char t = q[i]; q[i] = q[len - 1 - i]; q[len - 1 - i] = t;
		}
	}

	/* flat (len+1) x (ref_len+1) matrix, zeroed; row 0 holds 0..error+1
	 * and spills into row 1 when ref_len < error + 1 */
	cells = (size_t)(len + 1) * W;
	if (cells < error + 2)
		cells = error + 2;
	M = calloc(cells, sizeof(uint16_t));
	for (i = 0; i <= (int)error + 1; ++i)
		M[i] = (uint16_t)i;
	COUNT(sw_calls, 1);

	for (k = 1; k <= (int)len; ++k) {
		uint16_t *row = M + (size_t)k * W, *up = row - W;
		min = error;
		j = 0;
		row[s] = (uint16_t)(up[s] + 1);
		for (i = s + 1; i <= (int)ref_len; ++i) {
			unsigned d = up[i - 1], v;
			if (d == error + 1) {
				row[i] = (uint16_t)(error + 1);
				break;
			}
			pen = 0;
			if (d < error)
				pen = CD(r[i - 1]) == CD(q[k - 1]) ? 0 : 1;
			v = d + pen;
			if (row[i - 1] + 1u < v)
				v = row[i - 1] + 1u;
			if (up[i] + 1u < v)
				v = up[i] + 1u;
			row[i] = (uint16_t)v;
			COUNT(sw_cells, 1);
			if (row[i] == error && j == 0)
				j = i;
			if (row[i] < error)
				j = 0;
			if (row[i] <= min) {
				min = row[i];
				xmin = i;
			}
			if (ferr == -1 && i == k && row[i] > 0)
				ferr = i;
		}
		if (min == error) {
			++k;
			break;
		}
		while (row[s] >= error && s < (unsigned)i)
			++s;
		if ((unsigned)j > xmin && (unsigned)j < ref_len)
			row[j] = (uint16_t)(error + 1);
	}
	--k;

	if (min >= error) {
		/* early stop: shrink the aligned query prefix (:698-711) */
		while (k >= 5 && (min > (unsigned)(k / 10) ||
				  min * 2 > (unsigned)(k - ferr))) {
			--k;
			for (i = 0, j = 0; (unsigned)i < ref_len; ++i) {
				unsigned v = M[(size_t)k * W + i];
				if (v == error + 1)
					break;
				if (v > 0)
					j = error;
				/* r[-1] at column 0 never matches (see header) */
				if (v <= min && j > 0 && i > 0 &&
				    CD(r[i - 1]) == CD(q[k - 1]) &&
				    v == M[(size_t)k * W + i - W - 1]) {
					min = v;
					xmin = i;
				}
			}
		}
		if (k < 5) {
			cig_add(cig, OP_S, len, NULL);
			free(M); free(r); free(q);
			return (int)len;
		}
		cig_add(cig, OP_S, len - k, NULL);
		score = (int)len - k;
		i = k;
	} else {
		if (xmin < len && k == (int)len) {
			min += len - xmin;
			xmin = len;
		}
		i = (int)len;
	}
	k = (int)xmin;
	score += (int)min;

	if (write_bam == 1) {   /* score-only mode: one M op (:731-734) */
		cig_add(cig, OP_M, (unsigned)k, NULL);
		free(M); free(r); free(q);
		return score;
	}

	while (i > 0 && k > 0) {   /* traceback (:736-758) */
		unsigned cur = M[(size_t)i * W + k];
		pen = CD(r[k - 1]) == CD(q[i - 1]) ? 0 : 1;
		if (cur == M[(size_t)(i - 1) * W + k - 1] + pen) {
			if (pen == 0)
				cig_add(cig, OP_M, 1, NULL);
			else
				cig_add(cig, OP_X, 1, r + k - 1);
			--i;
			--k;
		} else if (cur == M[(size_t)(i - 1) * W + k] + 1u) {
			cig_add(cig, OP_I, 1, NULL);
			--i;
		} else {
			cig_add(cig, OP_D, 1, r + k - 1);
			--k;
		}
	}
	if (i > 0)
		cig_add(cig, OP_I, (unsigned)i, NULL);
	for (i = 1; i <= k; ++i)
		cig_add(cig, OP_D, 1, r + k - i);
	free(M); free(r); free(q);
	return score;
}

/* ------------------------------------------------------------------ */
/* ssw_align: local SW on saturating u8 (src/ssw.c:81-321)             */
/* ------------------------------------------------------------------ */
static int mat_score(uint8_t a, uint8_t b)
{
	/* src/ssw.c:38-44: +1 equal ACGT, -2 different ACGT, 0 with any N */
	if (a == 4 || b == 4)
		return 0;
	return a == b ? 1 : -2;
}

static int o_ssw_align(const char *ref_seq, int32_t ref_len,
		       const char *read_seq, int32_t read_len, int *skip,
		       ocig *cig)
{
	uint8_t *rd, *rf, *H, max = 0;
	int32_t end_read = read_len - 1, end_ref = -1, pos_max = 0;
	int32_t i, x, begin_ref, begin_read, right_sclip, x_pos, y_pos;
	int score = 0, cur, dir;

	cig_clear(cig);
	COUNT(ssw_calls, 1);
	COUNT(ssw_cells, (uint64_t)(ref_len > 0 ? ref_len : 0) * read_len);
	rd = malloc(read_len + 1);
	rf = malloc(ref_len > 0 ? ref_len + 1 : 1);
	for (i = 0; i < read_len; ++i)
		rd[i] = CD(read_seq[i]);
	for (i = 0; i < ref_len; ++i)
		rf[i] = CD(ref_seq[i]);
	/* H[col][x], column 0 all zero */
	H = calloc((size_t)(ref_len + 1) * (read_len > 0 ? read_len : 1), 1);

	for (i = 1; i <= ref_len; ++i) {
		uint8_t *col = H + (size_t)i * read_len;
		const uint8_t *prev = col - read_len;
		uint8_t cmax = 0;
		for (x = 0; x < read_len; ++x) {
			int d = x ? prev[x - 1] : 0;
			int h = d + (rd[x] == rf[i - 1] ? 3 : 0);
			int e = prev[x] >= 4 ? prev[x] - 4 : 0;
			int f = 0, v;
			if (h > 255)
				h = 255;
			h = h >= 2 ? h - 2 : 0;
			if (x)
				f = col[x - 1] >= 4 ? col[x - 1] - 4 : 0;
			v = h > e ? h : e;
			v = v > f ? v : f;
			col[x] = (uint8_t)v;
			if (v > cmax)
				cmax = (uint8_t)v;
		}
		/* first column where the running maximum strictly rises */
		if (cmax > max) {
			max = cmax;
			end_ref = i - 1;
			pos_max = i;
		}
	}

	begin_ref = end_ref;
	/* max == 0 with read_len < 4 leaves the reference tracing back from an
	 * uninitialised column; treated here like the low-score exit. */
	if (max < (read_len >> 2) || max == 0) {
		score = read_len;
		cig_add(cig, OP_S, (unsigned)read_len, NULL);
		goto end;
	}
	for (x = 0; x < read_len; ++x)
		if (H[(size_t)pos_max * read_len + x] == max) {
			if (x < end_read)
				end_read = x;
			break;
		}

	x_pos = end_read;
	y_pos = end_ref + 1;
	begin_read = end_read;
	right_sclip = read_len - end_read - 1;
	if (right_sclip > 0) {
		if (right_sclip < 5) {
			int32_t j;
			for (i = read_len - 1, j = end_ref + right_sclip;
			     i > end_read; i--, j--) {
				if (j >= ref_len) {
					cig_add(cig, OP_S, 1, NULL);
					++score;
				} else if (rd[i] == rf[j]) {
					cig_add(cig, OP_M, 1, NULL);
				} else {
					cig_add(cig, OP_X, 1, ref_seq + j);
					++score;
				}
			}
		} else {
			score += right_sclip;
			cig_add(cig, OP_S, (unsigned)right_sclip, NULL);
		}
	}

#define HV(xx, yy) ((int)H[(size_t)(yy) * read_len + (xx)])
	cur = HV(x_pos, y_pos);
	dir = 0;
	for (;;) {
		int diag, up, left;
		if (dir == 0) {
			if (rd[begin_read] == rf[begin_ref]) {
				cig_add(cig, OP_M, 1, NULL);
			} else {
				cig_add(cig, OP_X, 1, ref_seq + begin_ref);
				++score;
			}
		} else if (dir == 1) {   /* a step along the reference */
			++score;
			cig_add(cig, OP_I, 1, NULL);
		} else {                 /* a step along the read */
			++score;
			cig_add(cig, OP_D, 1, ref_seq + begin_ref);
		}
		if (x_pos == 0 || y_pos == 1)
			break;
		diag = HV(x_pos - 1, y_pos - 1);
		up = HV(x_pos - 1, y_pos);
		left = HV(x_pos, y_pos - 1);
		if (cur == diag + mat_score(rd[begin_read], rf[begin_ref])) {
			if (!diag)
				break;
			cur = diag;
			--begin_read; --begin_ref; --x_pos; --y_pos;
			dir = 0;
		} else if (cur == left - 4) {
			if (!left)
				break;
			cur = left;
			--y_pos; --begin_ref;
			dir = 1;
		} else {
			if (!up)
				break;
			cur = up;
			--x_pos; --begin_read;
			dir = 2;
		}
	}
#undef HV

	if (begin_read < 5) {
		for (--begin_read, --begin_ref; begin_read >= 0;
		     --begin_read, --begin_ref) {
			if (begin_ref < 0) {
				cig_add(cig, OP_S, 1, NULL);
				++score;
			} else if (rd[begin_read] == rf[begin_ref]) {
				cig_add(cig, OP_M, 1, NULL);
			} else {
				cig_add(cig, OP_X, 1, ref_seq + begin_ref);
				++score;
			}
		}
	} else if (begin_read > 0) {
		score += begin_read;
		cig_add(cig, OP_S, (unsigned)begin_read, NULL);
	}
end:
	*skip = begin_ref;
	free(rd); free(rf); free(H);
	return score;
}

/* ------------------------------------------------------------------ */
/* index probes                                                       */
/* ------------------------------------------------------------------ */

/* get_index (src/hash_align.c:997-1006): 31 codes shifted in unmasked,
 * so an N (4) sets the low bit of its left neighbour's field. */
uint64_t ho_get_index(const char *seq, uint32_t start)
{
	uint64_t idx = 0;
	uint32_t i;
	for (i = start; i < start + HO_KMER; ++i)
		idx = (idx << 2) | CD(seq[i]);
	return idx;
}

/* hash_get with add = 0 (src/hash_align.c:862-895): binary search of the
 * bucket id & (2^27-1); returns the slot and sets *found on an exact hit. */
uint32_t ho_hash_get(const ho_index *ix, uint64_t id, uint32_t *found)
{
	uint64_t mod = id & ((1ull << HO_HBITS) - 1);
	uint64_t base = ix->bucket_off[mod];
	uint32_t nb = (uint32_t)(ix->bucket_off[mod + 1] - base);
	uint32_t lo = 0, hi = nb, mid = 0;

	*found = 0;
	COUNT(lookups, 1);
	if (nb == 0)
		return 0;
	while (lo != hi) {
		mid = (lo + hi) >> 1;
		COUNT(probes, 1);
		if (ix->buckets[base + mid].id == id) {
			lo = hi = mid;
			break;
		}
		if (ix->buckets[base + mid].id > id)
			hi = mid;
		else
			lo = mid + 1;
	}
	if (lo < nb && ix->buckets[base + mid].id == id) {
		*found = 1;
		COUNT(hits, 1);
	}
	return lo;
}

/* ------------------------------------------------------------------ */
/* Candidate and anchors                                              */
/* ------------------------------------------------------------------ */
typedef struct {
	uint32_t *pos[2];
	int32_t *p[2];
	uint32_t n[2];
	int err[2];
	ocig cig[2];
	int pair;
} ocand;

typedef struct {
	uint32_t *t, *tp, *off;   /* transcript, transcript pos, read offset */
	uint32_t n, cap;
} anchors;

static void anchors_reserve(anchors *a, uint32_t n)
{
	if (n <= a->cap)
		return;
	a->cap = n * 2 + 16;
	a->t = xrealloc(a->t, a->cap * sizeof(uint32_t));
	a->tp = xrealloc(a->tp, a->cap * sizeof(uint32_t));
	a->off = xrealloc(a->off, a->cap * sizeof(uint32_t));
}

static void anchors_free(anchors *a)
{
	free(a->t); free(a->tp); free(a->off);
	memset(a, 0, sizeof(*a));
}

static void cand_init(ocand *c)
{
	memset(c, 0, sizeof(*c));
}

static void cand_free(ocand *c)
{
	free(c->pos[0]); free(c->pos[1]);
	free(c->p[0]); free(c->p[1]);
	cig_free(&c->cig[0]);
	cig_free(&c->cig[1]);
}

/* merge_sort (src/hash_align.c:257-297): merge a new hit list (all at read
 * offset `idx`) into the anchor list ordered by transcript id.  On equal
 * transcripts the existing anchor goes first when the unsigned wrapped
 * diagonal difference (dp - doff) is < 2*ERR, else the smaller tpos. */
static void merge_hits(anchors *a, const uint32_t *ht, const uint32_t *hp,
		       uint32_t nh, uint32_t idx, anchors *tmp)
{
	uint32_t i = 0, k = 0, n = 0;
	anchors_reserve(tmp, a->n + nh);
#define TAKE_A() do { tmp->t[n] = a->t[i]; tmp->tp[n] = a->tp[i]; tmp->off[n] = a->off[i]; ++n; ++i; } while (0)
#define TAKE_H() do { tmp->t[n] = ht[k]; tmp->tp[n] = hp[k]; tmp->off[n] = idx; ++n; ++k; } while (0)
	while (i < a->n && k < nh) {
		if (a->t[i] < ht[k]) {
			TAKE_A();
		} else if (a->t[i] > ht[k]) {
			TAKE_H();
		} else {
			uint32_t dis = (hp[k] - a->tp[i]) - (idx - a->off[i]);
			if (dis < 2 * HO_ERR)
				TAKE_A();
			else if (a->tp[i] > hp[k])
				TAKE_H();
			else
				TAKE_A();
		}
	}
	while (i < a->n)
		TAKE_A();
	while (k < nh)
		TAKE_H();
#undef TAKE_A
#undef TAKE_H
	tmp->n = n;
	{   /* swap storage */
		anchors t = *a;
		*a = *tmp;
		*tmp = t;
	}
}

/* reverse_str (src/hash_align.c:217-232): in-place reverse complement,
 * non-ACGT bytes kept, complements written upper-case. */
static void o_reverse_str(char *seq, int len)
{
	int i;
	for (i = 0; i < (len >> 1); ++i) {
		char a = seq[i], b = seq[len - 1 - i];
		char ta = CD(a) > 3 ? a : ACGT[3 - CD(a)];
		char tb = CD(b) > 3 ? b : ACGT[3 - CD(b)];
		seq[i] = tb;
		seq[len - 1 - i] = ta;
	}
	if ((len & 1) && CD(seq[len >> 1]) <= 3)
		seq[len >> 1] = ACGT[3 - CD(seq[len >> 1])];
}

typedef struct {
	const ho_index *ix;
	int write_bam;
	anchors tmp;
	ocig c1, c2;
} octx;

static uint32_t tstart(const ho_index *ix, uint32_t t)
{
	return t == 0 ? 0 : ix->find[t - 1];
}

/* get_SWalign (src/hash_align.c:1242-1320): align the chain of n anchors
 * starting at anchor `id`; keep/append/reset the stored hits. */
static void o_get_swalign(octx *cx, const char *rseq, int rlen, anchors *a,
			  uint32_t id, uint32_t n, uint32_t *store,
			  uint32_t *max, ocand *r, int str)
{
	const ho_index *ix = cx->ix;
	uint32_t i, ref_start, len, add;
	int start, score, err, sub;
	ocig *cig = &cx->c1, *tmp = &cx->c2;

	if (n > 1 && a->tp[id + n - 1] - a->tp[id] > (uint32_t)rlen)
		return;
	start = (int)(a->tp[id] - (a->off[id] + HO_KMER - 1));
	if (start < 0 || (uint32_t)(start + rlen) > ix->len[a->t[id]])
		return;
	add = start < HO_ERR ? (uint32_t)start : HO_ERR;
	ref_start = tstart(ix, a->t[id]) + (uint32_t)start;
	err = sub = 0;

	cig_clear(cig);
	if (a->off[id] > 0) {
		score = o_sw_align(ix->seq, ref_start - add, rseq,
				   a->off[id] + add, a->off[id], a->off[id] < 2 * HO_ERR ? -3 : -HO_ERR,
				   cx->write_bam, cig);
		err += score;
		if (err > rlen / 2 || (uint32_t)err > *max)
			return;
		for (i = 0; i < (uint32_t)cig->n; ++i) {
			if (cig->op[i] == OP_I || cig->op[i] == OP_S)
				sub += cig->cnt[i];
			else if (cig->op[i] == OP_D)
				sub -= cig->cnt[i];
		}
	}

	for (i = 0; i < n; ++i) {
		uint32_t s0 = i, seg;
		while (i + 1 < n && a->off[id + i] + HO_KMER >= a->off[id + i + 1])
			++i;
		cig_add(cig, OP_M, a->off[id + i] - a->off[id + s0] + HO_KMER, NULL);
		seg = a->off[id + i] + HO_KMER;
		len = ((i + 1) < n ? a->off[id + i + 1] : (uint32_t)rlen) - seg;
		add = (i + 1) < n ? 0 : HO_ERR;
		score = o_sw_align(ix->seq, ref_start + seg, rseq + seg, len + add,
				   len, len < 2 * HO_ERR ? 3 : HO_ERR, cx->write_bam, tmp);
		err += score;
		if (err > rlen / 2 || (uint32_t)err > *max + 1)
			return;
		cig_concat(cig, tmp);
	}

	if (*max == (uint32_t)(rlen / 2) || (uint32_t)err < *max) {
		cig_swap(&r->cig[str], cig);
		*store = 0;
		*max = (uint32_t)err;
	}
	a->t[*store] = a->t[id];
	a->tp[*store] = a->tp[id] - (a->off[id] + HO_KMER - 1) + (uint32_t)sub;
	++*store;
}

/* chain grows while same transcript, read offset rising, tpos rising from
 * the chain head and span < read length (src/hash_align.c:1378-1384) */
static int chain_next(const anchors *a, uint32_t i, uint32_t n, int rlen,
		      int stop_consumed)
{
	if (i + 1 >= a->n)
		return 0;
	if (a->t[i] != a->t[i + 1] || !(a->off[i + 1] > a->off[i]))
		return 0;
	if (!(a->tp[i + 1] > a->tp[i + 1 - n]))
		return 0;
	if (!(a->tp[i + 1] - a->tp[i + 1 - n] < (uint32_t)rlen))
		return 0;
	if (stop_consumed && a->off[i + 1] == (uint32_t)rlen)
		return 0;
	return 1;
}

/* get_position (src/hash_align.c:1322-1467) */
static void o_get_position(octx *cx, char *rseq, int rlen, ocand *r, int str,
			   int space)
{
	const ho_index *ix = cx->ix;
	anchors a = {0};
	uint32_t i, k, n, n1 = 0, max = 0, step = (uint32_t)(space < 0 ? -space : space);

	if (str == 1)
		o_reverse_str(rseq, rlen);

	/* seed loop (:1331-1362) */
	for (i = 0; i + HO_KMER <= (uint32_t)rlen; i += step) {
		uint32_t found, slot, nh;
		uint64_t id = ho_get_index(rseq, i), mod;
		const ho_bucket *b;
		slot = ho_hash_get(ix, id, &found);
		if (!found)
			continue;
		mod = id & ((1ull << HO_HBITS) - 1);
		b = &ix->buckets[ix->bucket_off[mod] + slot];
		nh = b->end - b->start;
		COUNT(occurrences, nh);
		if (a.n == 0) {
			anchors_reserve(&a, nh);
			memcpy(a.t, ix->pos + b->start, nh * sizeof(uint32_t));
			memcpy(a.tp, ix->p + b->start, nh * sizeof(uint32_t));
			for (k = 0; k < nh; ++k)
				a.off[k] = i;
			a.n = nh;
			continue;
		}
		if (nh == 0)
			continue;
		merge_hits(&a, ix->pos + b->start, ix->p + b->start, nh, i, &cx->tmp);
	}
	if (a.n == 0)
		goto miss;

	/* pass A, mate-guided (:1367-1390) */
	n1 = 0;
	if (r->n[1 - str] > 0 && space < HO_KMER && space > 0) {
		const uint32_t *mt = r->pos[1 - str];
		uint32_t mn = r->n[1 - str];
		for (i = k = 0, max = (uint32_t)(rlen / 2); i < a.n; ++i) {
			if (a.t[i] < mt[k])
				continue;
			while (k < mn && a.t[i] > mt[k])
				++k;
			if (k == mn)
				break;
			n = 1;
			while (chain_next(&a, i, n, rlen, 0)) {
				++i;
				++n;
			}
			o_get_swalign(cx, rseq, rlen, &a, i + 1 - n, n, &n1, &max, r, str);
			for (; n > 0; --n)
				a.off[i + 1 - n] = (uint32_t)rlen;
		}
	}

	/* pass B, chains of >= 2 anchors (:1392-1412) */
	if (n1 == 0) {
		for (i = n1 = 0, max = (uint32_t)(rlen / 2); i < a.n; ++i) {
			if (a.off[i] == (uint32_t)rlen)
				continue;
			n = 1;
			while (chain_next(&a, i, n, rlen, 1)) {
				++i;
				++n;
			}
			if (n < 2 && rlen / HO_KMER > 2)
				continue;
			o_get_swalign(cx, rseq, rlen, &a, i - n + 1, n, &n1, &max, r, str);
		}
	}

	/* pass C, singletons (:1414-1434) */
	if (n1 == 0 && space < HO_KMER) {
		for (i = n1 = 0, max = (uint32_t)(rlen / 2); i < a.n; ++i) {
			if (a.off[i] == (uint32_t)rlen)
				continue;
			n = 1;
			while (chain_next(&a, i, n, rlen, 1)) {
				++i;
				++n;
			}
			if (n >= 2)
				continue;
			o_get_swalign(cx, rseq, rlen, &a, i, n, &n1, &max, r, str);
		}
	}

	if (n1 == 0)
		goto miss;

	/* output (:1443-1459) */
	free(r->pos[str]);
	free(r->p[str]);
	r->pos[str] = xrealloc(NULL, n1 * sizeof(uint32_t));
	r->p[str] = xrealloc(NULL, n1 * sizeof(int32_t));
	memcpy(r->pos[str], a.t, n1 * sizeof(uint32_t));
	memcpy(r->p[str], a.tp, n1 * sizeof(int32_t));
	r->n[str] = n1;
	r->err[str] = (int)max;
	anchors_free(&a);
	if (str == 1)
		o_reverse_str(rseq, rlen);
	return;

miss:
	anchors_free(&a);
	r->n[str] = 0;
	r->err[str] = rlen;
	if (str == 1)
		o_reverse_str(rseq, rlen);
}

/* re_mapSW (src/hash_align.c:762-846): rescue strand `str` with ssw_align
 * in a MAX_FRAG window at each mate hit; min score wins, ties append. */
static uint32_t o_re_mapsw(octx *cx, ocand *r, int str, const char *rseq,
			   int rlen, int type)
{
	const ho_index *ix = cx->ix;
	uint32_t i, new_n = 0, ln, m = 1 - str;
	int range = type > 0 ? 0 : rlen - HO_MAX_FRAG, score1, score2 = 0, start, skip;
	uint32_t *pos = NULL;
	int32_t *p = NULL;
	ocig best = {0}, cur = {0};
	int have = 0;

	for (i = 0; i < r->n[m]; ++i) {
		uint32_t t = r->pos[m][i];
		start = r->p[m][i] + range;
		ln = HO_MAX_FRAG;
		if (start < 0)
			start = 0;
		if ((uint32_t)(start + HO_MAX_FRAG) > ix->len[t])
			ln = ix->len[t] - (uint32_t)start;
		score1 = o_ssw_align(ix->seq + tstart(ix, t) + start, (int32_t)ln,
				     rseq, rlen, &skip, &cur);
		if (score1 > rlen / 2 || start + skip < 0 ||
		    (uint32_t)(start + skip + rlen) > ix->len[t])
			continue;
		if (!have) {
			have = 1;
			cig_swap(&best, &cur);
			score2 = score1;
			r->pos[m][0] = r->pos[m][i];
			r->p[m][0] = r->p[m][i];
			pos = xrealloc(NULL, r->n[m] * sizeof(uint32_t));
			p = xrealloc(NULL, r->n[m] * sizeof(int32_t));
			pos[0] = r->pos[m][i];
			p[0] = start + skip;
			++new_n;
		} else if (score1 == score2) {
			r->pos[m][new_n] = r->pos[m][i];
			r->p[m][new_n] = r->p[m][i];
			pos[new_n] = r->pos[m][i];
			p[new_n] = start + skip;
			++new_n;
		} else if (score1 < score2) {
			cig_swap(&best, &cur);
			score2 = score1;
			r->pos[m][0] = r->pos[m][i];
			r->p[m][0] = r->p[m][i];
			pos[0] = r->pos[m][i];
			p[0] = start + skip;
			new_n = 1;
		}
	}
	cig_free(&cur);
	if (new_n == 0) {
		cig_free(&best);
		return 0;
	}
	free(r->pos[str]);
	free(r->p[str]);
	r->n[m] = r->n[str] = new_n;
	r->pos[str] = pos;
	r->p[str] = p;
	r->err[str] = score2;
	if (type <= 0)
		cig_reverse(&best);
	cig_swap(&r->cig[str], &best);
	cig_free(&best);
	return new_n;
}

/* get_position2 (src/hash_align.c:1469-1502) */
static void o_get_position2(octx *cx, ocand *r, int str, char *rseq, int rlen,
			    int type)
{
	ocig saved = r->cig[str];
	uint32_t n = r->n[str], ret;

	memset(&r->cig[str], 0, sizeof(ocig));
	o_get_position(cx, rseq, rlen, r, str, 2 * HO_ERR);
	ret = r->n[str];
	if (ret == 0) {
		if (type > 0)
			o_reverse_str(rseq, rlen);
		ret = o_re_mapsw(cx, r, str, rseq, rlen, type);
		if (type > 0)
			o_reverse_str(rseq, rlen);
	}
	if (ret > 0) {
		cig_free(&saved);
	} else {
		r->n[str] = n;
		cig_free(&r->cig[str]);
		r->cig[str] = saved;
	}
}

/* re_map (src/hash_align.c:1504-1522) */
static void o_re_map(octx *cx, ocand *r, char *s1, int l1, char *s2, int l2)
{
	uint32_t ret;
	int i = 0;

	o_reverse_str(s2, l2);
	if (r->err[0] < r->err[1])
		i = 1;
	ret = o_re_mapsw(cx, r, i, i == 0 ? s1 : s2, i == 0 ? l1 : l2, i == 0 ? -1 : 1);
	if (ret == 0)
		ret = o_re_mapsw(cx, r, 1 - i, i == 0 ? s2 : s1, i == 0 ? l2 : l1,
				 i == 0 ? 1 : -1);
	if (ret > 0)
		r->pair = 2;
	o_reverse_str(s2, l2);
}

/* intersect2 (src/hash_align.c:1524-1562) */
static void o_intersect2(octx *cx, ocand *r, char *s1, int l1, char *s2, int l2,
			 uint32_t add)
{
	uint32_t i = 0, k = 0, n = 0;

	while (i < r->n[0] && k < r->n[1]) {
		if (r->pos[0][i] < r->pos[1][k]) {
			++i;
		} else if (r->pos[0][i] > r->pos[1][k]) {
			++k;
		} else {
			int d = r->p[0][i] - r->p[1][k];
			uint32_t dis = (uint32_t)(d < 0 ? -d : d);
			if (dis <= add || add == 0) {
				++n;
				r->pos[0][n - 1] = r->pos[0][i];
				r->p[0][n - 1] = r->p[0][i];
				r->pos[1][n - 1] = r->pos[1][k];
				r->p[1][n - 1] = r->p[1][k];
				++i;
				++k;
			} else if (r->p[0][i] < r->p[1][k]) {
				++i;
			} else {
				++k;
			}
		}
	}
	if (n > 0) {
		r->n[0] = r->n[1] = n;
		r->pair = 2;
	} else if (add > 0) {
		o_intersect2(cx, r, s1, l1, s2, l2, 0);
	} else {
		o_re_map(cx, r, s1, l1, s2, l2);
	}
}

/* check_in_transcriptome (src/hash_align.c:1663-1695) */
static void o_check_in_transcriptome(octx *cx, char *s1, int l1, char *s2,
				     int l2, ocand *r0, ocand *r1)
{
	o_get_position(cx, s1, l1, r0, 0, HO_KMER);
	o_get_position(cx, s2, l2, r0, 1, HO_KMER);
	o_get_position(cx, s1, l1, r1, 1, HO_KMER);
	o_get_position(cx, s2, l2, r1, 0, HO_KMER);

	if (r0->n[0] == 0 && r0->n[1] == 0 && r1->err[0] + r1->err[1] > HO_ERR) {
		o_get_position(cx, s1, l1, r0, 0, 2 * HO_ERR);
		o_get_position(cx, s2, l2, r0, 1, 2 * HO_ERR);
	}
	if (r1->n[0] == 0 && r1->n[1] == 0 && r0->err[0] + r0->err[1] > HO_ERR) {
		o_get_position(cx, s1, l1, r1, 1, 2 * HO_ERR);
		o_get_position(cx, s2, l2, r1, 0, 2 * HO_ERR);
	}

	if (r0->n[0] == 0 && r0->n[1] > 0 && r0->err[1] < HO_ERR &&
	    r1->err[0] + r1->err[1] > HO_ERR)
		o_get_position2(cx, r0, 0, s1, l1, -1);
	if (r0->n[1] == 0 && r0->n[0] > 0 && r0->err[0] < HO_ERR &&
	    r1->err[0] + r1->err[1] > HO_ERR)
		o_get_position2(cx, r0, 1, s2, l2, 1);
	if (r1->n[0] == 0 && r1->n[1] > 0 && r1->err[1] < HO_ERR &&
	    r0->err[0] + r0->err[1] > HO_ERR)
		o_get_position2(cx, r1, 0, s2, l2, -1);
	if (r1->n[1] == 0 && r1->n[0] > 0 && r1->err[0] < HO_ERR &&
	    r0->err[0] + r0->err[1] > HO_ERR)
		o_get_position2(cx, r1, 1, s1, l1, 1);
}

/* ------------------------------------------------------------------ */
/* result packing                                                     */
/* ------------------------------------------------------------------ */
static int emit(ho_result *out, uint64_t ri, const ocand *c)
{
	ho_rec *rec = &out->recs[ri];
	int s;

	rec->pair = c->pair;
	for (s = 0; s < 2; ++s) {
		const ocig *g = &c->cig[s];
		int j;
		rec->n[s] = (int32_t)c->n[s];
		rec->err[s] = c->err[s];
		if (out->list_used + c->n[s] > out->list_cap ||
		    out->op_used + (uint64_t)g->n > out->op_cap ||
		    out->miss_used + (uint64_t)g->nm > out->miss_cap)
			return -1;
		rec->list_off[s] = (uint32_t)out->list_used;
		if (c->n[s]) {
			memcpy(out->pos_pool + out->list_used, c->pos[s], c->n[s] * sizeof(uint32_t));
			memcpy(out->p_pool + out->list_used, c->p[s], c->n[s] * sizeof(int32_t));
		}
		out->list_used += c->n[s];
		rec->cig_off[s] = (uint32_t)out->op_used;
		rec->n_cigar[s] = (uint16_t)g->n;
		for (j = 0; j < g->n; ++j)
			out->op_pool[out->op_used + j] = ((uint32_t)g->cnt[j] << 4) | g->op[j];
		out->op_used += g->n;
		rec->miss_off[s] = (uint32_t)out->miss_used;
		rec->n_miss[s] = (uint16_t)g->nm;
		if (g->nm)
			memcpy(out->miss_pool + out->miss_used, g->miss, g->nm);
		out->miss_used += g->nm;
	}
	return 0;
}

static void octx_init(octx *cx, const ho_index *ix, int write_bam)
{
	memset(cx, 0, sizeof(*cx));
	cx->ix = ix;
	cx->write_bam = write_bam;
}

static void octx_free(octx *cx)
{
	anchors_free(&cx->tmp);
	cig_free(&cx->c1);
	cig_free(&cx->c2);
}

/* front half of align_pair_read (src/hash_align.c:1724-1733) */
static void o_align_pair(octx *cx, char *s1, int l1, char *s2, int l2,
			 ocand *r0, ocand *r1)
{
	cand_init(r0);
	cand_init(r1);
	o_check_in_transcriptome(cx, s1, l1, s2, l2, r0, r1);
	if (r0->n[0] > 0 && r0->n[1] > 0)
		o_intersect2(cx, r0, s1, l1, s2, l2, HO_MAX_FRAG);
	if (r1->n[0] > 0 && r1->n[1] > 0)
		o_intersect2(cx, r1, s2, l2, s1, l1, HO_MAX_FRAG);
}

int ho_align_pairs(const ho_index *ix, int write_bam, int n,
		   char *seq1, const int64_t *off1, const int32_t *len1,
		   char *seq2, const int64_t *off2, const int32_t *len2,
		   ho_result *out)
{
	octx cx;
	int i, rc = 0;

	memset(&G_STATS, 0, sizeof(G_STATS));
	ST = &G_STATS;
	octx_init(&cx, ix, write_bam);
	out->list_used = out->op_used = out->miss_used = 0;
	for (i = 0; i < n && rc == 0; ++i) {
		ocand r0, r1;
		o_align_pair(&cx, seq1 + off1[i], len1[i], seq2 + off2[i], len2[i], &r0, &r1);
		rc = emit(out, 2 * (uint64_t)i, &r0);
		if (rc == 0)
			rc = emit(out, 2 * (uint64_t)i + 1, &r1);
		cand_free(&r0);
		cand_free(&r1);
	}
	octx_free(&cx);
	ST = NULL;
	return rc;
}

/* front half of align_single_read (src/hash_align.c:1819-1823) */
int ho_align_single(const ho_index *ix, int write_bam, int n,
		    char *seq, const int64_t *off, const int32_t *len,
		    ho_result *out)
{
	octx cx;
	int i, rc = 0;

	memset(&G_STATS, 0, sizeof(G_STATS));
	ST = &G_STATS;
	octx_init(&cx, ix, write_bam);
	out->list_used = out->op_used = out->miss_used = 0;
	for (i = 0; i < n && rc == 0; ++i) {
		ocand r;
		cand_init(&r);
		o_get_position(&cx, seq + off[i], len[i], &r, 0, 2 * HO_ERR);
		o_get_position(&cx, seq + off[i], len[i], &r, 1, 2 * HO_ERR);
		rc = emit(out, (uint64_t)i, &r);
		cand_free(&r);
	}
	octx_free(&cx);
	ST = NULL;
	return rc;
}

/* ------------------------------------------------------------------ */
/* unit entry points                                                  */
/* ------------------------------------------------------------------ */
static int export_cig(const ocig *c, uint32_t *ops, int *n_ops, char *miss,
		      int *n_miss, int cap)
{
	int j;
	if (c->n > cap || c->nm > cap)
		return -1;
	for (j = 0; j < c->n; ++j)
		ops[j] = ((uint32_t)c->cnt[j] << 4) | c->op[j];
	*n_ops = c->n;
	if (c->nm)
		memcpy(miss, c->miss, c->nm);
	*n_miss = c->nm;
	return 0;
}

int ho_sw_align(const char *ref, uint32_t rstart, const char *q,
		uint32_t ref_len, uint32_t len, int err, int write_bam,
		uint32_t *ops, int *n_ops, char *miss, int *n_miss, int cap)
{
	ocig c = {0};
	int score = o_sw_align(ref, rstart, q, ref_len, len, err, write_bam, &c);
	int rc = export_cig(&c, ops, n_ops, miss, n_miss, cap);
	cig_free(&c);
	return rc < 0 ? -1000000 : score;
}

int ho_ssw_align(const char *ref, int32_t ref_len, const char *read,
		 int32_t read_len, int *skip,
		 uint32_t *ops, int *n_ops, char *miss, int *n_miss, int cap)
{
	ocig c = {0};
	int score = o_ssw_align(ref, ref_len, read, read_len, skip, &c);
	int rc = export_cig(&c, ops, n_ops, miss, n_miss, cap);
	cig_free(&c);
	return rc < 0 ? -1000000 : score;
}

/* ------------------------------------------------------------------ */
/* multi-threaded timing entry (CPU baseline)                          */
/* ------------------------------------------------------------------ */
typedef struct {
	const ho_index *ix;
	int write_bam, lo, hi;
	char *seq1, *seq2;
	const int64_t *off1, *off2;
	const int32_t *len1, *len2;
} mt_job;

static void *mt_worker(void *arg)
{
	mt_job *j = arg;
	octx cx;
	int i;
	octx_init(&cx, j->ix, j->write_bam);
	for (i = j->lo; i < j->hi; ++i) {
		ocand r0, r1;
		o_align_pair(&cx, j->seq1 + j->off1[i], j->len1[i],
			     j->seq2 + j->off2[i], j->len2[i], &r0, &r1);
		cand_free(&r0);
		cand_free(&r1);
	}
	octx_free(&cx);
	return NULL;
}

int ho_align_pairs_mt(const ho_index *ix, int write_bam, int n,
		      char *seq1, const int64_t *off1, const int32_t *len1,
		      char *seq2, const int64_t *off2, const int32_t *len2,
		      int nthreads)
{
	pthread_t *th;
	mt_job *jobs;
	int t;
	if (nthreads < 1)
		nthreads = 1;
	th = calloc(nthreads, sizeof(pthread_t));
	jobs = calloc(nthreads, sizeof(mt_job));
	for (t = 0; t < nthreads; ++t) {
		mt_job *j = &jobs[t];
		j->ix = ix;
		j->write_bam = write_bam;
		j->lo = (int)((int64_t)n * t / nthreads);
		j->hi = (int)((int64_t)n * (t + 1) / nthreads);
		j->seq1 = seq1; j->seq2 = seq2;
		j->off1 = off1; j->off2 = off2;
		j->len1 = len1; j->len2 = len2;
		pthread_create(&th[t], NULL, mt_worker, j);
	}
	for (t = 0; t < nthreads; ++t)
		pthread_join(th[t], NULL);
	free(th);
	free(jobs);
	return 0;
}

/* ---- FASTQ chunk parsing ------------------------------------------------ */

/* byte k of a chunk buffer: bytes [0, n), then the terminating NUL */
static inline char fq_at(const char *b, int64_t n, int64_t k)
{
	return k < n ? b[k] : '\0';
}

/* One get_read_from_fq_buffer call (src/read.c:11-63) at *pos: 0 READ_SUCCESS
 * (*pos moves to the next read), 1 READ_END, 2 READ_FAIL.  The reference also
 * writes NULs over the newlines it passes; no later test reads them. */
static int fq_one(const char *b, int64_t n, int64_t *pos, ho_fq_rec *r)
{
	int64_t i = *pos, prev;
	if (fq_at(b, n, i) != '@')
		return 2;
	prev = i;
	while (fq_at(b, n, i) != '\0' && fq_at(b, n, i) != '\n')
		++i;
	if (fq_at(b, n, i) == '\0')
		return 2;
	r->name = prev + 1;
	r->name_len = (int32_t)(i - prev - 1);
	++i;
	prev = i;
	while (fq_at(b, n, i) != '\0' && fq_at(b, n, i) != '\n')
		++i;
	if (fq_at(b, n, i) == '\0')
		return 2;
	r->seq = prev;
	r->len = (int32_t)(i - prev);
	++i;
	if (r->len == 0)
		return 2;
	if (fq_at(b, n, i) != '+')
		return 2;
	while (fq_at(b, n, i) != '\0' && fq_at(b, n, i) != '\n')
		++i;
	if (fq_at(b, n, i) == '\0')
		return 2;
	++i;
	prev = i;
	while (fq_at(b, n, i) != '\0' && fq_at(b, n, i) != '\n')
		++i;
	if (i - prev != r->len)
		return 2;
	r->qual = prev;
	if (fq_at(b, n, i) == '\0')
		return 1;
	if (fq_at(b, n, i + 1) == '\0')
		return 1;
	*pos = i + 1;
	return 0;
}

/* align_pool_pair's read loop (src/hash_align.c:1878-1929): left read, then
 * right read (a READ_FAIL of either ends the run with its file named), the
 * pair, and a stop when the left read was the last (`ret_code1`, which is
 * READ_END there) or the right one returned READ_END.  An empty buffer is a
 * READ_FAIL at its first read, as the reader gives. */
int ho_parse_fq_pairs(const char *left, int64_t n_left, const char *right, int64_t n_right,
		      ho_fq_rec *out, int32_t cap, int32_t *n_pairs, int32_t *bad_file,
		      int64_t *bad_rec)
{
	int64_t pl = 0, pr = 0;
	int32_t k = 0;
	*n_pairs = 0;
	*bad_file = 0;
	*bad_rec = -1;
	for (;;) {
		ho_fq_rec a, b;
		const int s1 = fq_one(left, n_left, &pl, &a);
		if (s1 == 2) {
			*bad_file = 1;
			*bad_rec = k;
			return HO_FQ_FAIL;
		}
		const int s2 = fq_one(right, n_right, &pr, &b);
		if (s2 == 2) {
			*bad_file = 2;
			*bad_rec = k;
			return HO_FQ_FAIL;
		}
		if (k < cap) {
			out[2 * (int64_t)k] = a;
			out[2 * (int64_t)k + 1] = b;
		}
		++k;
		if (s1 || s2 == 1)
			break;
	}
	*n_pairs = k;
	return k > cap ? HO_FQ_CAP : HO_FQ_OK;
}

/* align_pool_single's read loop (src/hash_align.c:1966-1998) */
int ho_parse_fq_single(const char *buf, int64_t n, ho_fq_rec *out, int32_t cap,
		       int32_t *n_reads, int64_t *bad_rec)
{
	int64_t p = 0;
	int32_t k = 0;
	*n_reads = 0;
	*bad_rec = -1;
	for (;;) {
		ho_fq_rec a;
		const int s = fq_one(buf, n, &p, &a);
		if (s == 2) {
			*bad_rec = k;
			return HO_FQ_FAIL;
		}
		if (k < cap)
			out[k] = a;
		++k;
		if (s == 1)
			break;
	}
	*n_reads = k;
	return k > cap ? HO_FQ_CAP : HO_FQ_OK;
}

/* ===========================================================================
 * Equivalence classes: the host tail's add_class calls
 * ======================================================================== */

/* XXH32, restated from the published xxHash specification (32-bit variant,
 * little-endian input).  hera vendors it as src/xxhash.c and calls it once
 * per class key in add_class (src/hash_align.c:1576). */
#define XP1 2654435761u
#define XP2 2246822519u
#define XP3 3266489917u
#define XP4 668265263u
#define XP5 374761393u
static uint32_t xrotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
static uint32_t xrd32(const uint8_t *p)
{
	return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24;
}
static uint32_t xround(uint32_t acc, uint32_t in) { return xrotl(acc + in * XP2, 13) * XP1; }

uint32_t ho_xxh32(const void *buf, size_t len, uint32_t seed)
{
	const uint8_t *p = (const uint8_t *)buf, *end = p + len;
	uint32_t h;
	if (len >= 16) {
		uint32_t v1 = seed + XP1 + XP2, v2 = seed + XP2, v3 = seed, v4 = seed - XP1;
		const uint8_t *lim = end - 16;
		do {
			v1 = xround(v1, xrd32(p));
			v2 = xround(v2, xrd32(p + 4));
			v3 = xround(v3, xrd32(p + 8));
			v4 = xround(v4, xrd32(p + 12));
			p += 16;
		} while (p <= lim);
		h = xrotl(v1, 1) + xrotl(v2, 7) + xrotl(v3, 12) + xrotl(v4, 18);
	} else {
		h = seed + XP5;
	}
	h += (uint32_t)len;
	for (; p + 4 <= end; p += 4)
		h = xrotl(h + xrd32(p) * XP3, 17) * XP4;
	for (; p < end; ++p)
		h = xrotl(h + *p * XP5, 11) * XP1;
	h ^= h >> 15;
	h *= XP2;
	h ^= h >> 13;
	h *= XP3;
	h ^= h >> 16;
	return h;
}

struct ho_classes {
	uint32_t n_trans;
	uint32_t n, cap;            /* classes in first-insertion order */
	uint32_t *id, *cn;
	double *count;
	uint64_t *ref_off;
	uint32_t *ref;              /* class lists back to back */
	uint64_t ref_n, ref_cap;
	uint32_t *map;              /* open addressing on id: class index + 1 */
	uint64_t map_slots;
	uint32_t *tx_count;         /* REF_INF->count */
	uint32_t paired;            /* PAIRED */
	double mean_frag;           /* MEAN_FRAG before main.c divides it */
};

ho_classes *ho_classes_new(uint32_t n_trans)
{
	ho_classes *c = calloc(1, sizeof *c);
	c->n_trans = n_trans;
	c->tx_count = calloc(n_trans ? n_trans : 1, sizeof(uint32_t));
	c->map_slots = 1024;
	c->map = calloc(c->map_slots, sizeof(uint32_t));
	return c;
}

void ho_classes_free(ho_classes *c)
{
	if (!c)
		return;
	free(c->id); free(c->cn); free(c->count); free(c->ref_off); free(c->ref);
	free(c->map); free(c->tx_count); free(c);
}

/* Slot of `id` in the map: the slot holding it, or the empty slot where it
 * goes.  hera probes a 2^27-slot map the same way (src/hash_align.c:
 * 1576-1584); the class an id lands in depends only on the id, because a
 * class is found by comparing ids, so the map's size is not visible. */
static uint64_t cls_slot(const ho_classes *c, uint32_t id)
{
	uint64_t s = id & (c->map_slots - 1);
	while (c->map[s] && c->id[c->map[s] - 1] != id)
		s = (s + 1) & (c->map_slots - 1);
	return s;
}

static void cls_grow_map(ho_classes *c)
{
	free(c->map);
	c->map_slots *= 2;
	c->map = calloc(c->map_slots, sizeof(uint32_t));
	for (uint32_t i = 0; i < c->n; ++i)
		c->map[cls_slot(c, c->id[i])] = i + 1;
}

/* add_class (src/hash_align.c:1564-1602) for a Candidate whose list 0 is
 * the concatenation a[0..na) ++ b[0..nb) (concate_candidate :1604-1618 and
 * the single-read merges :1842-1850 build such lists). */
static int cls_add(ho_classes *c, const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb,
		   int err_sum, int pair, int32_t p00, int32_t p10)
{
	++c->paired;
	if (pair == 1) {
		int32_t d = p00 - p10;
		c->mean_frag += d < 0 ? -d : d;
	}
	const uint32_t n = na + nb;
	if (n == 1) {
		uint32_t t = na ? a[0] : b[0];
		if (t >= c->n_trans)
			return -1;
		++c->tx_count[t];
		return 0;
	}
	if (err_sum >= HO_ERR)
		return 0;
	uint32_t *key = malloc((n ? n : 1) * sizeof(uint32_t));
	if (na)
		memcpy(key, a, na * sizeof(uint32_t));
	if (nb)
		memcpy(key + na, b, nb * sizeof(uint32_t));
	uint32_t id = ho_xxh32(key, (size_t)n * sizeof(uint32_t), 0);
	uint64_t s = cls_slot(c, id);
	if (c->map[s]) {
		c->count[c->map[s] - 1] += 1;
		free(key);
		return 0;
	}
	if (c->n == c->cap) {
		c->cap = c->cap ? 2 * c->cap : 1024;
		c->id = realloc(c->id, c->cap * sizeof(uint32_t));
		c->cn = realloc(c->cn, c->cap * sizeof(uint32_t));
		c->count = realloc(c->count, c->cap * sizeof(double));
		c->ref_off = realloc(c->ref_off, c->cap * sizeof(uint64_t));
	}
	if (c->ref_n + n > c->ref_cap) {
		while (c->ref_n + n > c->ref_cap)
			c->ref_cap = c->ref_cap ? 2 * c->ref_cap : 4096;
		c->ref = realloc(c->ref, c->ref_cap * sizeof(uint32_t));
	}
	c->id[c->n] = id;
	c->cn[c->n] = n;
	c->count[c->n] = 1;
	c->ref_off[c->n] = c->ref_n;
	memcpy(c->ref + c->ref_n, key, (size_t)n * sizeof(uint32_t));
	c->ref_n += n;
	c->map[s] = ++c->n;
	free(key);
	if (2 * (uint64_t)c->n > c->map_slots)
		cls_grow_map(c);
	return 0;
}

int ho_classes_add(ho_classes *c, const ho_rec *recs, const uint32_t *pos_pool,
		   const int32_t *p_pool, int n, int paired)
{
	for (int i = 0; i < n; ++i) {
		int rc = 0;
		if (paired) {
			/* align_pair_read's tail (src/hash_align.c:1735-1760); with
			 * FMINDEX NULL check_in_genome changes nothing (:1697-1701) */
			const ho_rec *a = &recs[2 * i], *b = &recs[2 * i + 1];
			int pa = a->pair, pb = b->pair;
			const int sa = a->err[0] + a->err[1], sb = b->err[0] + b->err[1];
			if (sa < sb)
				pb = -1;
			else if (sa > sb)
				pa = -1;
			const ho_rec *r = NULL, *m = NULL;   /* class source, appended mate */
			if (pa > 1 && pb > 1) {
				if ((pa & 1) + (pb & 1) == 0) {
					r = a;
					m = b;
				}
			} else if (pa > 1) {
				if ((pa & 1) == 0)
					r = a;
			} else if (pb > 1) {
				if ((pb & 1) == 0)
					r = b;
			}
			if (!r)
				continue;
			const uint32_t *l0 = pos_pool + r->list_off[0];
			const uint32_t *l1 = m ? pos_pool + m->list_off[0] : NULL;
			const uint32_t n0 = (uint32_t)r->n[0], n1 = m ? (uint32_t)m->n[0] : 0;
			/* p[0][0] / p[1][0] after concate_candidate: r's first entry
			 * when r has one, else the appended mate's */
			int32_t p00 = n0 ? p_pool[r->list_off[0]] : (n1 ? p_pool[m->list_off[0]] : 0);
			int32_t p10 = r->n[1] ? p_pool[r->list_off[1]]
					      : (m && m->n[1] ? p_pool[m->list_off[1]] : 0);
			rc = cls_add(c, l0, n0, l1, n1, r->err[0] + r->err[1], 1, p00, p10);
		} else {
			/* align_single_read's tail (src/hash_align.c:1825-1851) */
			const ho_rec *r = &recs[i];
			if (r->n[0] == 0 && r->n[1] == 0)
				continue;
			const uint32_t *l0 = pos_pool + r->list_off[0], *l1 = pos_pool + r->list_off[1];
			const int es = r->err[0] + r->err[1];
			if (r->err[0] > r->err[1])          /* move_candidate(r, 0, 1) */
				rc = cls_add(c, l1, (uint32_t)r->n[1], NULL, 0, es, 0, 0, 0);
			else if (r->err[0] == r->err[1])    /* list 1 appended to list 0 */
				rc = cls_add(c, l0, (uint32_t)r->n[0], l1, (uint32_t)r->n[1], es, 0, 0, 0);
			else
				rc = cls_add(c, l0, (uint32_t)r->n[0], NULL, 0, es, 0, 0, 0);
		}
		if (rc)
			return rc;
	}
	return 0;
}

void ho_classes_sizes(const ho_classes *c, uint32_t *n_classes, uint64_t *ref_n)
{
	*n_classes = c->n;
	*ref_n = c->ref_n;
}

void ho_classes_export(const ho_classes *c, uint32_t *id, double *count, uint32_t *n,
		       uint64_t *ref_off, uint32_t *ref, uint32_t *tx_count,
		       uint32_t *paired, double *mean_frag)
{
	if (c->n) {
		memcpy(id, c->id, c->n * sizeof(uint32_t));
		memcpy(count, c->count, c->n * sizeof(double));
		memcpy(n, c->cn, c->n * sizeof(uint32_t));
		memcpy(ref_off, c->ref_off, c->n * sizeof(uint64_t));
	}
	if (c->ref_n)
		memcpy(ref, c->ref, c->ref_n * sizeof(uint32_t));
	memcpy(tx_count, c->tx_count, c->n_trans * sizeof(uint32_t));
	*paired = c->paired;
	*mean_frag = c->mean_frag;
}

/* ===========================================================================
 * The EM over the class table: estimate_count (src/EM.c:315-387)
 * ======================================================================== */

/* Norm (src/hash_align.c:150-164): the sample standard deviation, two
 * passes in index order. */
static double em_norm(const double *a, uint32_t n)
{
	double sum = 0, total = 0;
	for (uint32_t i = 0; i < n; ++i)
		sum += a[i];
	sum /= n;
	for (uint32_t i = 0; i < n; ++i)
		total += (a[i] - sum) * (a[i] - sum);
	total /= n - 1;
	return sqrt(total);
}

/* M_step (src/EM.c:271-302): per class, its share of the class count
 * goes to each listed transcript in proportion to grama; overlap
 * accumulates in class order and is cleared again. */
static double *em_m_step(uint32_t n_trans, const uint32_t *len, const uint32_t *tx_count,
			 uint32_t n_classes, const double *count, const uint32_t *n,
			 const uint64_t *ref_off, const uint32_t *ref, double *grama, double *overlap,
			 uint32_t *stop)
{
	double *next = calloc(n_trans ? n_trans : 1, sizeof(double));
	for (uint32_t i = 0; i < n_classes; ++i) {
		const uint32_t *l = ref + ref_off[i];
		double total = 0.0;
		for (uint32_t k = 0; k < n[i]; ++k)
			total += grama[l[k]];
		if (total == 0)
			continue;
		for (uint32_t k = 0; k < n[i]; ++k)
			overlap[l[k]] += grama[l[k]] * count[i] / total;
	}
	double max_err = 0.0;
	*stop = 1;
	for (uint32_t i = 0; i < n_trans; ++i) {
		next[i] = (double)(tx_count[i] + overlap[i]) / len[i];
		overlap[i] = 0.0;
		if (next[i] > 1e-3) {
			double d = next[i] - grama[i];
			double err = (d < 0 ? -d : d) / next[i];
			max_err = err > max_err ? err : max_err;
			if (max_err > 0.01)
				*stop = 0;
		}
	}
	return next;
}

void ho_em(uint32_t n_trans, const uint32_t *len, const uint32_t *tx_count, uint32_t n_classes,
	   const double *count, const uint32_t *n, const uint64_t *ref_off, const uint32_t *ref,
	   double *grama_out, double *overlap_out, uint32_t *rounds)
{
	const uint32_t N = n_trans ? n_trans : 1;
	double *grama = calloc(N, sizeof(double));
	double *overlap = calloc(N, sizeof(double));
	double *r = malloc(N * sizeof(double)), *v = malloc(N * sizeof(double));
	for (uint32_t i = 0; i < n_trans; ++i)          /* E_step */
		grama[i] = (double)1 / n_trans;
	uint32_t k = 0, stop = 0;
	while (k < 50 || (k < 1000 && stop == 0)) {
		double *u = grama;
		double *u1 = em_m_step(n_trans, len, tx_count, n_classes, count, n, ref_off, ref, u, overlap, &stop);
		double *u2 = em_m_step(n_trans, len, tx_count, n_classes, count, n, ref_off, ref, u1, overlap, &stop);
		for (uint32_t i = 0; i < n_trans; ++i) {
			r[i] = u1[i] - u[i];
			v[i] = (u2[i] - u1[i]) - r[i];
		}
		double n_r = em_norm(r, n_trans), n_v = em_norm(v, n_trans);
		double alpha = n_v != 0 ? -n_r / n_v : -1;
		if (alpha > -1)
			alpha = -1;
		free(u2);
		for (uint32_t i = 0; i < n_trans; ++i) {
			u1[i] = u[i] - 2 * alpha * r[i] + alpha * alpha * v[i];
			if (u1[i] < 0)
				u1[i] = 0;
		}
		grama = em_m_step(n_trans, len, tx_count, n_classes, count, n, ref_off, ref, u1, overlap, &stop);
		free(u);
		free(u1);
		++k;
	}
	double sum = 0.0;
	for (uint32_t i = 0; i < n_trans; ++i)
		sum += grama[i];
	for (uint32_t i = 0; i < n_trans; ++i) {
		if (sum == 0) {
			overlap_out[i] = 0;
			grama_out[i] = 0;
		} else {
			overlap_out[i] = grama[i] * len[i];
			grama_out[i] = grama[i] * 1000000 / sum;
		}
	}
	*rounds = k;
	free(grama); free(overlap); free(r); free(v);
}

/* ===========================================================================
 * BAM records of the host tail (`-w`)
 * ======================================================================== */

enum { B_MATCH = 0, B_DELETE = 2, B_SKIP = 3, B_DIFF = 8 };

/* bam_nt16_table (src/bam_write.c:3-20): =ACMGRSVTWYHKDBN -> 0..15 */
static unsigned char b_nt16(unsigned char c)
{
	switch (c) {
	case '=': return 0;
	case 'A': case 'a': return 1;
	case 'C': case 'c': return 2;
	case 'M': case 'm': return 3;
	case 'G': case 'g': return 4;
	case 'R': case 'r': return 5;
	case 'S': case 's': return 6;
	case 'V': case 'v': return 7;
	case 'T': case 't': return 8;
	case 'W': case 'w': return 9;
	case 'Y': case 'y': return 10;
	case 'H': case 'h': return 11;
	case 'K': case 'k': return 12;
	case 'D': case 'd': return 13;
	case 'B': case 'b': return 14;
	default: return 15;
	}
}

/* One strand of a Candidate as the tail sees it. */
typedef struct {
	uint32_t n;
	const uint32_t *pos;
	const int32_t *p;
	uint32_t n_cigar, n_miss;
	const uint32_t *ops;    /* (count << 4) | type */
	const char *miss;
} b_strand;

typedef struct {
	b_strand s[2];
	int err[2];
	int pair;
} b_cand;

static void b_swap(b_cand *a, int pa, b_cand *b, int pb)   /* swap_candidate (:1640-1661) */
{
	b_strand t = a->s[pa];
	a->s[pa] = b->s[pb];
	b->s[pb] = t;
}

static uint32_t b_exon_start(const ho_gene_map *g, uint32_t t, uint32_t e) { return g->starts[g->exon_off[t] + e]; }
static uint32_t b_exon_end(const ho_gene_map *g, uint32_t t, uint32_t e) { return g->ends[g->exon_off[t] + e]; }

/* check_overlapGene (src/hash_align.c:395-414) */
static int b_overlap_gene(const ho_gene_map *g, uint32_t t1, uint32_t t2)
{
	if (t1 == t2 || g->gene[t1] == g->gene[t2])
		return 1;
	if (g->chr[t1] != g->chr[t2])
		return 0;
	uint32_t s0 = b_exon_start(g, t1, 0), s1 = b_exon_start(g, t2, 0);
	uint32_t e0 = b_exon_end(g, t1, g->exon_off[t1 + 1] - g->exon_off[t1] - 1);
	uint32_t e1 = b_exon_end(g, t2, g->exon_off[t2 + 1] - g->exon_off[t2] - 1);
	return !(s1 > e0 || s0 > e1);
}

/* check_quanlity (:416-427): genes among the hits, counted by runs */
static unsigned b_genes(const ho_gene_map *g, const b_strand *s)
{
	if (s->n == 0)
		return 0;
	unsigned k = 1;
	for (uint32_t i = 1; i < s->n; ++i)
		if (!b_overlap_gene(g, s->pos[i], s->pos[i - 1]))
			++k;
	return k;
}

/* get_qual (src/bam_write.c:199-205) */
static unsigned int b_qual(unsigned int n)
{
	double error = 1 - (1.0 / n);
	if (error == 0)
		error = 0.0000001;
	return -10 * log10(error);
}

static int b_reg2bin(unsigned int beg, unsigned int end)   /* bam_reg2bin (:59-68) */
{
	--end;
	if (beg >> 14 == end >> 14) return 4681 + (beg >> 14);
	if (beg >> 17 == end >> 17) return 585 + (beg >> 17);
	if (beg >> 20 == end >> 20) return 73 + (beg >> 20);
	if (beg >> 23 == end >> 23) return 9 + (beg >> 23);
	if (beg >> 26 == end >> 26) return 1 + (beg >> 26);
	return 0;
}

static unsigned int b_flag(unsigned pair, unsigned proper, unsigned map, unsigned mmap, unsigned rev,
			   unsigned mrev, unsigned first, unsigned last)   /* make_flag (:70-86) */
{
	return last << 7 | first << 6 | mrev << 5 | rev << 4 | mmap << 3 | map << 2 | proper << 1 | pair;
}

typedef struct {
	int bin, qual, ref, pos, n_cigar;
	unsigned int len, block_len, coord, match, align_len;
	char md[2048];
	uint32_t cig[1024];
	uint8_t data[8192];
} b_core;

/* add_padding (:89-116): a match run over exon junctions gets N ops */
static void b_pad(const ho_gene_map *g, b_core *c, unsigned int *n, unsigned int *l, uint32_t t,
		  unsigned int len, unsigned int type, unsigned int genome)
{
	if ((type != B_MATCH && type != B_DIFF) || genome == 1) {
		c->cig[(*n)++] = len << 4 | type;
		return;
	}
	*l += len;
	while (*l > b_exon_end(g, t, c->coord) + 1) {
		len -= *l - b_exon_end(g, t, c->coord) - 1;
		c->cig[(*n)++] = len << 4 | type;
		len = b_exon_start(g, t, c->coord + 1) - b_exon_end(g, t, c->coord) - 1;
		c->align_len += len;
		c->cig[(*n)++] = len << 4 | B_SKIP;
		len = *l - b_exon_end(g, t, c->coord) - 1;
		*l += b_exon_start(g, t, c->coord + 1) - b_exon_end(g, t, c->coord) - 1;
		++c->coord;
	}
	c->cig[(*n)++] = len << 4 | type;
}

/* convert_cigar (:118-197): position on the genome, MD string, CIGAR */
static void b_convert(const ho_gene_map *g, b_core *c, const b_strand *s, uint32_t hit, unsigned int genome)
{
	const uint32_t t = s->pos[hit];
	if (genome == 0) {
		c->ref = g->chr[t];
		/* gene_coord (src/hash_align.c:320-334) */
		int pos = s->p[hit];
		if (pos <= 0) {
			c->coord = 0;
			c->pos = b_exon_start(g, t, 0);
		} else {
			unsigned int len = 0, i = 0;
			for (; len <= (unsigned int)pos; ++i)
				len += b_exon_end(g, t, i) - b_exon_start(g, t, i) + 1;
			c->coord = i - 1;
			c->pos = b_exon_end(g, t, c->coord) - (len - pos) + 1;
		}
	} else {
		/* chr_coord (src/hash_align.c:307-318) */
		unsigned int sum = 0, i;
		for (i = 0; i < g->n_chr; ++i) {
			if (sum + g->chr_len[i] > t)
				break;
			sum += g->chr_len[i];
		}
		c->ref = i;
		c->pos = t - sum;
	}
	unsigned int match = 0, k = 0;
	for (uint32_t i = 0; i < s->n_cigar; ++i) {
		const unsigned type = s->ops[i] & 15, cnt = s->ops[i] >> 4;
		if (type == B_MATCH) {
			unsigned int n = cnt;
			++i;
			while (i < s->n_cigar && (s->ops[i] & 15) != B_DIFF && (s->ops[i] & 15) != B_DELETE) {
				if ((s->ops[i] & 15) == B_MATCH)
					n += s->ops[i] >> 4;
				++i;
			}
			--i;
			match += n;
			c->len += sprintf(c->md + c->len, "%u", n);
		} else if (type == B_DIFF) {
			c->md[c->len++] = s->miss[k++];
			for (unsigned j = 1; j < cnt; ++j) {
				c->md[c->len++] = '0';
				c->md[c->len++] = s->miss[k++];
			}
			c->md[c->len] = 0;
		} else if (type == B_DELETE) {
			c->md[c->len++] = '^';
			for (unsigned j = 0; j < cnt; ++j)
				c->md[c->len++] = s->miss[k++];
			c->md[c->len] = 0;
		}
		c->len = strlen(c->md);
	}
	unsigned int n = 0, l = c->pos;
	for (uint32_t i = 0; i < s->n_cigar; ++i) {
		unsigned int run = 0;
		while (i < s->n_cigar && ((s->ops[i] & 15) == B_DIFF || (s->ops[i] & 15) == B_MATCH))
			run += s->ops[i++] >> 4;
		if (run > 0)
			b_pad(g, c, &n, &l, t, run, B_MATCH, genome);
		if (i < s->n_cigar)
			b_pad(g, c, &n, &l, t, s->ops[i] >> 4, s->ops[i] & 15, genome);
	}
	c->n_cigar = n;
	c->match = match;
}

/* pack_bam_core + compact_inf (:206-240, 265-283) */
static void b_pack_core(const ho_gene_map *g, b_core *c, const b_cand *r, int p, const char *seq,
			const char *qual, int rlen, const char *name, unsigned int name_len, uint32_t hit)
{
	const unsigned int genome = r->pair & 1;
	const b_strand *s = &r->s[p];
	memset(c, 0, offsetof(b_core, md));
	c->md[0] = 0;
	c->ref = c->pos = -1;
	if (s->n > 0)
		b_convert(g, c, s, hit, genome);
	c->bin = b_reg2bin(c->pos, c->pos + c->match);
	const unsigned int n = genome == 1 ? s->n : b_genes(g, s);
	c->qual = b_qual(n);
	unsigned int len = 36;
	memcpy(c->data + len, name, name_len);
	len += name_len;
	memcpy(c->data + len, c->cig, 4 * c->n_cigar);
	len += 4 * c->n_cigar;
	int i;
	for (i = 0, c->data[len] = 0; i < rlen; ++i) {
		c->data[len] = (uint8_t)(c->data[len] << 4 | b_nt16((unsigned char)seq[i]));
		if (i & 1)
			c->data[++len] = 0;
	}
	if (i & 1) {
		c->data[len] = (uint8_t)(c->data[len] << 4);
		++len;
	}
	for (i = 0; i < rlen; ++i)
		c->data[len + i] = (uint8_t)(qual[i] - 33);
	len += rlen;
	if (c->match > 0) {
		const uint32_t nm = s->n_miss;
		memcpy(c->data + len, "NMi", 3);
		memcpy(c->data + len + 3, &nm, 4);
		len += 7;
		memcpy(c->data + len, "MDZ", 3);
		memcpy(c->data + len + 3, c->md, c->len + 1);
		len += 3 + c->len + 1;
	}
	memcpy(c->data + len, "ASi", 3);
	memcpy(c->data + len + 3, &c->match, 4);
	len += 7;
	c->block_len = len;
}

typedef struct {
	uint8_t *out;
	uint64_t used, cap;
	int full;
} b_stream;

/* pack_bam_block (:285-310) */
static void b_block(b_stream *st, b_core *c, const b_core *mate, unsigned int name_len, int rlen,
		    unsigned int flag, int size)
{
	int x[8];
	x[0] = c->ref;
	x[1] = c->pos;
	x[2] = (unsigned int)c->bin << 16 | c->qual << 8 | name_len;
	x[3] = flag << 16 | c->n_cigar;
	x[4] = rlen;
	x[5] = mate->ref;
	x[6] = mate->pos;
	x[7] = size;
	const unsigned int blen = c->block_len - 4;
	memcpy(c->data, &blen, 4);
	memcpy(c->data + 4, x, 32);
	if (st->used + c->block_len > st->cap) {
		st->full = 1;
		return;
	}
	memcpy(st->out + st->used, c->data, c->block_len);
	st->used += c->block_len;
}

typedef struct {
	char *seq, *qual, *name;
	int len;
} b_read;

/* write_alignment_pair (:349-380): both mates' records of hit `hit` */
static void b_write_alignment(const ho_gene_map *g, b_stream *st, b_read *a, b_read *b, const unsigned int *flag,
			      const b_cand *r, uint32_t hit)
{
	static b_core c0, c1;
	unsigned int name_len = strlen(a->name);
	if (name_len > 2 && a->name[name_len - 2] == '/') {
		a->name[name_len - 2] = 0;
		--name_len;
	} else {
		++name_len;
	}
	b_pack_core(g, &c0, r, 0, a->seq, a->qual, a->len, a->name, name_len, hit);
	/* the mate record takes name_len bytes of the mate's own name */
	b_pack_core(g, &c1, r, 1, b->seq, b->qual, b->len, b->name, name_len, hit);
	int size = 0;
	if (c0.ref >= 0 && c0.ref == c1.ref) {
		if (c0.pos < c1.pos)
			size = c1.pos + b->len + c1.align_len - c0.pos;
		else
			size = c0.pos + a->len + c0.align_len - c1.pos;
	}
	b_block(st, &c0, &c1, name_len, a->len, flag[0], size);
	b_block(st, &c1, &c0, name_len, b->len, flag[1], -size);
}

/* bam_write_pair (:382-416): the primary records, then one secondary pair
 * per further hit that is not in the same gene as the one before it */
static void b_write_pair(const ho_gene_map *g, b_stream *st, b_read *a, b_read *b, const b_cand *r,
			 unsigned proper, unsigned first, unsigned rev, unsigned mrev)
{
	unsigned int flag[2];
	flag[0] = b_flag(1, proper, r->s[0].n == 0, r->s[1].n == 0, rev, mrev, 1, 0);
	flag[1] = b_flag(1, proper, r->s[1].n == 0, r->s[0].n == 0, mrev, rev, 0, 1);
	b_write_alignment(g, st, a, b, flag, r, 0);
	flag[0] |= 1 << 8;
	flag[1] |= 1 << 8;
	if (proper == 0 || r->s[0].n < 2)
		return;
	for (uint32_t i = 1; i < r->s[0].n; ++i) {
		while (i < r->s[0].n && (r->pair & 1) == 0 && b_overlap_gene(g, r->s[0].pos[i], r->s[0].pos[i - 1]))
			++i;
		if (i == r->s[0].n)
			break;
		b_write_alignment(g, st, a, b, flag, r, i);
	}
}

static void b_rev(b_read *x)   /* reverse_str + reverse_qual (:217-245) */
{
	o_reverse_str(x->seq, x->len);
	for (int i = 0; i < (x->len >> 1); ++i) {
		char t = x->qual[i];
		x->qual[i] = x->qual[x->len - 1 - i];
		x->qual[x->len - 1 - i] = t;
	}
}

static b_cand b_from_rec(const ho_rec *rec, const uint32_t *pos_pool, const int32_t *p_pool,
			 const uint32_t *op_pool, const char *miss_pool)
{
	b_cand c;
	for (int s = 0; s < 2; ++s) {
		c.s[s].n = (uint32_t)rec->n[s];
		c.s[s].pos = pos_pool + rec->list_off[s];
		c.s[s].p = p_pool + rec->list_off[s];
		c.s[s].n_cigar = rec->n_cigar[s];
		c.s[s].n_miss = rec->n_miss[s];
		c.s[s].ops = op_pool + rec->cig_off[s];
		c.s[s].miss = miss_pool + rec->miss_off[s];
		c.err[s] = rec->err[s];
	}
	c.pair = rec->pair;
	return c;
}

int ho_bam_pairs(const ho_gene_map *gm, const ho_rec *recs, const uint32_t *pos_pool,
		 const int32_t *p_pool, const uint32_t *op_pool, const char *miss_pool, int n,
		 char *seq1, const int64_t *off1, const int32_t *len1, char *qual1, char *name1,
		 char *seq2, const int64_t *off2, const int32_t *len2, char *qual2, char *name2,
		 int32_t name_stride, uint8_t *out, uint64_t cap, uint64_t *out_off)
{
	b_stream st = {out, 0, cap, 0};
	for (int i = 0; i < n; ++i) {
		out_off[i] = st.used;
		b_read x1 = {seq1 + off1[i], qual1 + off1[i], name1 + (int64_t)i * name_stride, len1[i]};
		b_read x2 = {seq2 + off2[i], qual2 + off2[i], name2 + (int64_t)i * name_stride, len2[i]};
		b_cand r0 = b_from_rec(&recs[2 * i], pos_pool, p_pool, op_pool, miss_pool);
		b_cand r1 = b_from_rec(&recs[2 * i + 1], pos_pool, p_pool, op_pool, miss_pool);
		const int s0 = r0.err[0] + r0.err[1], s1 = r1.err[0] + r1.err[1];
		/* align_pair_read's branches (src/hash_align.c:1735-1804) */
		if (s0 < s1)
			r1.pair = -1;
		else if (s0 > s1)
			r0.pair = -1;
		if (r0.pair > 1 && r1.pair > 1) {
			b_rev(&x2);
			b_write_pair(gm, &st, &x1, &x2, &r0, 1, 1, 0, 1);
			b_rev(&x2);
			b_rev(&x1);
			b_write_pair(gm, &st, &x2, &x1, &r1, 1, 0, 0, 1);
		} else if (r0.pair > 1) {
			b_rev(&x2);
			b_write_pair(gm, &st, &x1, &x2, &r0, 1, 1, 0, 1);
		} else if (r1.pair > 1) {
			b_rev(&x1);
			b_write_pair(gm, &st, &x2, &x1, &r1, 1, 0, 0, 1);
		} else if (r0.s[0].n > 0 && r0.s[1].n > 0 && s0 < s1) {
			b_rev(&x2);
			b_write_pair(gm, &st, &x1, &x2, &r0, 0, 1, 0, 1);
		} else if (r1.s[0].n > 0 && r1.s[1].n > 0) {
			b_rev(&x1);
			b_write_pair(gm, &st, &x2, &x1, &r1, 0, 0, 0, 1);
		} else if (r0.s[0].n > 0 && r1.s[0].n > 0 && (r0.pair & 1) == (r1.pair & 1)) {
			b_swap(&r0, 1, &r1, 0);
			r0.pair = -10;
			b_write_pair(gm, &st, &x1, &x2, &r0, 0, 1, 0, 0);
		} else if (r0.s[1].n > 0 && r1.s[1].n > 0 && (r0.pair & 1) == (r1.pair & 1)) {
			b_rev(&x1);
			b_rev(&x2);
			b_swap(&r0, 0, &r1, 1);
			r0.pair = -20;
			b_write_pair(gm, &st, &x1, &x2, &r0, 0, 0, 1, 1);
		} else if (r0.s[0].n > 0) {
			b_write_pair(gm, &st, &x1, &x2, &r0, 0, 1, 0, 0);
		} else if (r0.s[1].n > 0) {
			b_rev(&x2);
			b_write_pair(gm, &st, &x1, &x2, &r0, 0, 1, 0, 1);
		} else if (r1.s[0].n > 0) {
			b_write_pair(gm, &st, &x2, &x1, &r1, 0, 0, 0, 0);
		} else {
			b_rev(&x1);
			b_write_pair(gm, &st, &x2, &x1, &r1, 0, 0, 0, 1);
		}
		if (st.full)
			return -1;
	}
	out_off[n] = st.used;
	return 0;
}

/* write_alignment_single (src/bam_write.c:314-347) */
static void b_write_alignment_single(const ho_gene_map *g, b_stream *st, b_read *a, unsigned int flag,
				     const b_cand *r, int p, uint32_t hit)
{
	static b_core c0, c1;
	unsigned int name_len = strlen(a->name);
	if (name_len > 2 && a->name[name_len - 2] == '/') {
		a->name[name_len - 2] = 0;
		--name_len;
	} else {
		++name_len;
	}
	b_pack_core(g, &c0, r, p, a->seq, a->qual, a->len, a->name, name_len, hit);
	c1.ref = c1.pos = -1;
	b_block(st, &c0, &c1, name_len, a->len, flag, 0);
}

/* bam_write_single (src/bam_write.c:418-446) */
static void b_write_single(const ho_gene_map *g, b_stream *st, b_read *a, const b_cand *r, unsigned rev, int p)
{
	unsigned int flag = b_flag(0, 0, r->s[p].n == 0, 1, rev, 0, 1, 0);
	b_write_alignment_single(g, st, a, flag, r, p, 0);
	flag |= 1 << 8;
	if (r->s[p].n < 2)
		return;
	for (uint32_t i = 1; i < r->s[p].n; ++i) {
		while (i < r->s[p].n && b_overlap_gene(g, r->s[p].pos[i], r->s[p].pos[i - 1]))
			++i;
		if (i == r->s[p].n)
			break;
		b_write_alignment_single(g, st, a, flag, r, p, i);
	}
}

int ho_bam_single(const ho_gene_map *gm, const ho_rec *recs, const uint32_t *pos_pool,
		  const int32_t *p_pool, const uint32_t *op_pool, const char *miss_pool, int n,
		  char *seq, const int64_t *off, const int32_t *len, char *qual, char *name,
		  int32_t name_stride, uint8_t *out, uint64_t cap, uint64_t *out_off)
{
	b_stream st = {out, 0, cap, 0};
	for (int i = 0; i < n; ++i) {
		out_off[i] = st.used;
		b_read x = {seq + off[i], qual + off[i], name + (int64_t)i * name_stride, len[i]};
		b_cand r = b_from_rec(&recs[i], pos_pool, p_pool, op_pool, miss_pool);
		/* align_single_read (src/hash_align.c:1825-1834) */
		if (r.s[0].n == 0 && r.s[1].n == 0) {
			b_write_single(gm, &st, &x, &r, 0, 0);
		} else if (r.s[0].n > 0) {
			b_write_single(gm, &st, &x, &r, 0, 0);
		} else {
			b_rev(&x);
			b_write_single(gm, &st, &x, &r, 1, 1);
		}
		if (st.full)
			return -1;
	}
	out_off[n] = st.used;
	return 0;
}
