// hera_gpu.cu -- kernels and C ABI of the B200 read-alignment hot path.
//
// Pipeline of one batch (pairs), all on one CUDA stream:
//   k_codes      ASCII reads -> 0..4 codes
//   k_seed       seed_probe: every 31-spaced seed of both strands of every
//                read looked up in the 2^27-bucket table (HBM gathers)
//   k_position   the four independent space-31 get_position calls per pair
//   k_resolve    per-pair control flow (retries, get_position2, intersect2,
//                re_map) up to the point a mate rescue is needed
//   k_rescue_*   re_mapSW: one warp-wide ssw_align per (request, mate hit),
//                then per-request selection; rounds of k_resolve and the
//                rescue alternate until no pair is waiting
//   k_count/k_emit  compact the Candidate records into flat pools
#include "hera_device.cuh"
#include "../../include/hera_gpu.h"

#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace hg;

namespace {

constexpr int TPB = 128;

struct RmReq {
	int32_t pair;
	int16_t c, str;
};

struct Batch {
	DevIndex ix;
	const uint8_t *code;     // read codes
	const uint8_t *code_r;   // reverse-complement codes (read i at the same offset)
	const int64_t *off;      // read offsets (2 per pair: mate 1, mate 2)
	const int32_t *len;
	DPair *P;
	int *flags;
	int score_only;
	int max_len;             // longest read of the batch (seed table stride)
};

__device__ __forceinline__ void flag(int *f, int v)
{
	if (v)
		atomicOr(f, v);
}

// read `ri` in orientation `orient` (1 = reverse complement) into rd
__device__ __forceinline__ int load_read(const Batch &b, int ri, int orient, uint8_t *rd)
{
	const int64_t o = b.off[ri];
	int L = b.len[ri];
	if (L > MAX_READ)
		L = MAX_READ;
	const uint8_t *src = b.code + o;
	if (orient == 0) {
		for (int x = 0; x < L; ++x)
			rd[x] = src[x];
	} else {
		for (int x = 0; x < L; ++x)
			rd[x] = comp_code(src[L - 1 - x]);
	}
	return L;
}

__global__ void k_codes(const uint8_t *__restrict__ ascii, uint8_t *__restrict__ code, int64_t n)
{
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
	     i += (int64_t)gridDim.x * blockDim.x)
		code[i] = code_of(ascii[i]);
}

// reverse-complement codes of every read, at the read's own offset (one
// warp per read, lanes over bases: coalesced)
__global__ void k_rc(const uint8_t *__restrict__ code, const int64_t *__restrict__ off,
		     const int32_t *__restrict__ len, int n_reads, int max_len, uint8_t *__restrict__ rc)
{
	const int r = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
	const int lane = threadIdx.x & 31;
	if (r >= n_reads)
		return;
	const int64_t o = off[r];
	int L = len[r];
	L = L < max_len ? L : max_len;
	for (int x = lane; x < L; x += 32)
		rc[o + x] = comp_code(code[o + L - 1 - x]);
}

// seed_probe: thread per (read, strand, seed) at spacing 31
__global__ void k_seed(DevIndex ix, const uint8_t *__restrict__ code, const int64_t *__restrict__ off,
		       const int32_t *__restrict__ len, int n_reads, int spr, uint2 *__restrict__ hits)
{
	const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
	const int64_t total = (int64_t)n_reads * 2 * spr;
	if (t >= total)
		return;
	const int j = (int)(t % spr);
	const int64_t ro = t / spr;
	const int orient = (int)(ro & 1);
	const int ri = (int)(ro >> 1);
	const int L = len[ri];
	const int i = j * KMER;
	uint2 h = make_uint2(0, 0);
	if (i + KMER <= L && j < spr) {
		const uint8_t *src = code + off[ri];
		uint64_t id = 0;
		if (orient == 0) {
#pragma unroll
			for (int x = 0; x < KMER; ++x)
				id = (id << 2) | src[i + x];
		} else {
#pragma unroll
			for (int x = 0; x < KMER; ++x)
				id = (id << 2) | comp_code(src[L - 1 - i - x]);
		}
		h = probe(ix, id);
	}
	hits[t] = h;
}

__device__ __forceinline__ void slot_reset(DSlot &S)
{
	S.n = 0;
	S.err = 0;
	S.cig.n = 0;
	S.cig.nm = 0;
}

// the four space-31 get_position calls of check_in_transcriptome
// (src/hash_align.c:1667-1670); independent because pass A needs space < 31
__global__ void __launch_bounds__(TPB) k_position(Batch b, int n_pairs, int spr, const uint2 *__restrict__ hits)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n_pairs * 4)
		return;
	const int pi = t >> 2, task = t & 3;
	const int c = task >> 1, str = task & 1;
	const int ri = 2 * pi + ((c ^ str) == 0 ? 0 : 1);
	GpWork w;
	int flags = 0;
	DPair &P = b.P[pi];
	DSlot &S = P.s[c][str];
	slot_reset(S);
	if (str == 0) {
		P.pair[c] = 0;
		if (c == 0) {
			P.stage = 0;
			P.rm_ret = 0;
		}
	}
	if (b.len[ri] > b.max_len) {
		flag(b.flags, F_READ);
		S.err = b.len[ri];
		return;
	}
	const uint2 *pre = hits + ((int64_t)ri * 2 + str) * spr;
	const int L0 = b.len[ri];
	bool any = false;
	for (int j = 0; j * KMER + KMER <= L0; ++j)
		any |= pre[j].y != 0;
	if (!any) {   // no seed hit: get_position's miss exit (src/hash_align.c:1364-1365)
		S.err = L0;
		return;
	}
	const int L = load_read(b, ri, str, w.rd);
	get_position(b.ix, w.rd, L, P, c, str, KMER, pre, b.score_only != 0, w, flags);
	flag(b.flags, flags);
}

// per-pair control flow after the space-31 calls (src/hash_align.c:1672-1695
// and :1730-1733 with intersect2/re_map :1504-1562).  A pair that needs a
// mate rescue enqueues it and stops; it resumes at P.stage next round.
__global__ void __launch_bounds__(TPB) k_resolve(Batch b, const RmReq *__restrict__ resume, int n,
						  RmReq *__restrict__ q, int *__restrict__ qn)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n)
		return;
	const int pi = resume ? resume[t].pair : t;
	DPair &P = b.P[pi];
	GpWork w;
	int flags = 0;
	auto gp = [&](int c, int str) {
		const int ri = 2 * pi + ((c ^ str) == 0 ? 0 : 1);
		const int L = load_read(b, ri, str, w.rd);
		get_position(b.ix, w.rd, L, P, c, str, 2 * ERR, nullptr, b.score_only != 0, w, flags);
	};
	auto rescue = [&](int c, int str, int next) {
		int k = atomicAdd(qn, 1);
		q[k].pair = pi;
		q[k].c = (int16_t)c;
		q[k].str = (int16_t)str;
		P.stage = next;
	};
	if (b.len[2 * pi] > b.max_len || b.len[2 * pi + 1] > b.max_len) {
		P.stage = 7;
		return;
	}
	int st = P.stage;
	for (;;) {
		switch (st) {
		case 0: {   // retries at spacing 14 (:1672-1681)
			if (P.s[0][0].n == 0 && P.s[0][1].n == 0 && P.s[1][0].err + P.s[1][1].err > ERR) {
				gp(0, 0);
				gp(0, 1);
			}
			if (P.s[1][0].n == 0 && P.s[1][1].n == 0 && P.s[0][0].err + P.s[0][1].err > ERR) {
				gp(1, 1);
				gp(1, 0);
			}
			st = 1;
			break;
		}
		case 1: case 2: case 3: case 4: {   // get_position2 x4 (:1683-1694)
			const int c = (st - 1) >> 1, s = (st - 1) & 1;
			const DSlot &X = P.s[c][s], &Y = P.s[c][1 - s];
			const DSlot &O0 = P.s[1 - c][0], &O1 = P.s[1 - c][1];
			if (X.n == 0 && Y.n > 0 && Y.err < ERR && O0.err + O1.err > ERR) {
				gp(c, s);
				if (P.s[c][s].n == 0) {
					rescue(c, s, 10 + st);
					flag(b.flags, flags);
					return;
				}
			}
			st = st + 1;
			break;
		}
		case 11: case 12: case 13: case 14:
			st = st - 10 + 1;
			break;
		case 5: case 6: {   // intersect2 (:1730-1733)
			const int c = st - 5;
			if (P.s[c][0].n > 0 && P.s[c][1].n > 0) {
				if (intersect_lists(P, c, MAX_FRAG) == 0 && intersect_lists(P, c, 0) == 0) {
					const int i = P.s[c][0].err < P.s[c][1].err ? 1 : 0;   // re_map
					P.rm_i = i;
					rescue(c, i, 20 + 2 * c);
					flag(b.flags, flags);
					return;
				}
			}
			st = st + 1;
			break;
		}
		case 20: case 22: {
			const int c = (st - 20) >> 1;
			if (P.rm_ret == 0) {
				rescue(c, 1 - P.rm_i, st + 1);
				flag(b.flags, flags);
				return;
			}
			P.pair[c] = 2;
			st = 6 + c;
			break;
		}
		case 21: case 23: {
			const int c = (st - 21) >> 1;
			if (P.rm_ret > 0)
				P.pair[c] = 2;
			st = 6 + c;
			break;
		}
		default:
			P.stage = 7;
			flag(b.flags, flags);
			return;
		}
	}
}

// re_mapSW (src/hash_align.c:762-846), in three steps.
// 1) one ssw_align call per (queued request, mate hit)
__global__ void k_rescue_expand(Batch b, const RmReq *__restrict__ q, int nq, int2 *__restrict__ calls,
				int *__restrict__ base, int *__restrict__ ncalls)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= nq)
		return;
	const RmReq rq = q[t];
	const int n = b.P[rq.pair].s[rq.c][1 - rq.str].n;
	const int at = atomicAdd(ncalls, n);
	base[t] = at;
	for (int i = 0; i < n; ++i)
		calls[at + i] = make_int2(t, i);
}

// 2) one warp per call: local SW over the MAX_FRAG window at the mate hit
__global__ void __launch_bounds__(128) k_rescue_sw(Batch b, const RmReq *__restrict__ q,
						    const int2 *__restrict__ calls, int c0, int nc,
						    SswOut *__restrict__ out, uint8_t *__restrict__ scratch,
						    size_t per)
{
	const int wl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;   // warp within launch
	if (wl >= nc)
		return;
	const int2 cl = calls[c0 + wl];
	const RmReq rq = q[cl.x];
	const DPair &P = b.P[rq.pair];
	const int c = rq.c, str = rq.str;
	const int type = str == 0 ? -1 : 1;
	const int ri = 2 * rq.pair + ((c ^ str) == 0 ? 0 : 1);
	const int L = b.len[ri];
	const DSlot &M = P.s[c][1 - str];
	const uint32_t tr = M.t[cl.y];
	const uint32_t tl = __ldg(b.ix.tlen + tr);
	int start = M.p[cl.y] + (type > 0 ? 0 : L - MAX_FRAG);
	if (start < 0)
		start = 0;
	int ln = MAX_FRAG;
	if ((uint32_t)(start + MAX_FRAG) > tl)
		ln = (int)tl - start;
	if (ln < 0)
		ln = 0;
	int flags = 0;
	ssw_warp(b.ix, __ldg(b.ix.tstart + tr) + (uint32_t)start, ln, b.code, b.off[ri], L, str, start, tl,
		 scratch + (size_t)wl * per, out[c0 + wl], flags);
	if ((threadIdx.x & 31) == 0)
		flag(b.flags, flags);
}

// 3) per request: min score wins, ties append in hit order; the mate's list
// is compacted to the rescued subset (src/hash_align.c:794-845)
__global__ void k_rescue_fin(Batch b, const RmReq *__restrict__ q, int nq, const int *__restrict__ base,
			     const SswOut *__restrict__ out)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= nq)
		return;
	const RmReq rq = q[t];
	DPair &P = b.P[rq.pair];
	const int c = rq.c, str = rq.str;
	DSlot &S = P.s[c][str];
	DSlot &M = P.s[c][1 - str];
	const int n = M.n, b0 = base[t];
	int new_n = 0, score2 = 0, best = -1;
	for (int i = 0; i < n; ++i) {
		const SswOut &o = out[b0 + i];
		if (!o.ok)
			continue;
		const uint32_t tr = M.t[i];
		const int32_t mp = M.p[i];
		if (new_n == 0 || o.score < score2) {
			best = i;
			score2 = o.score;
			M.t[0] = tr;
			M.p[0] = mp;
			S.t[0] = tr;
			S.p[0] = o.pstart;
			new_n = 1;
		} else if (o.score == score2) {
			M.t[new_n] = tr;
			M.p[new_n] = mp;
			S.t[new_n] = tr;
			S.p[new_n] = o.pstart;
			++new_n;
		}
	}
	P.rm_ret = new_n;
	if (new_n > 0) {
		M.n = S.n = new_n;
		S.err = score2;
		cig_copy(S.cig, out[b0 + best].cig);
		if (str == 0)   // type <= 0: CIGAR reversed (:839-840)
			cig_reverse(S.cig);
	}
}

// align_single_read front half (src/hash_align.c:1822-1823)
__global__ void __launch_bounds__(TPB) k_single(Batch b, int n)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n)
		return;
	DPair &P = b.P[t];
	GpWork w;
	int flags = 0;
	slot_reset(P.s[0][0]);
	slot_reset(P.s[0][1]);
	P.pair[0] = 0;
	if (b.len[t] > b.max_len) {
		flag(b.flags, F_READ);
		P.s[0][0].err = P.s[0][1].err = b.len[t];
		return;
	}
	int L = load_read(b, t, 0, w.rd);
	get_position(b.ix, w.rd, L, P, 0, 0, 2 * ERR, nullptr, b.score_only != 0, w, flags);
	L = load_read(b, t, 1, w.rd);
	get_position(b.ix, w.rd, L, P, 0, 1, 2 * ERR, nullptr, b.score_only != 0, w, flags);
	flag(b.flags, flags);
}

// per record: entries of the list / op / miss pools
__global__ void k_count(const DPair *__restrict__ P, int n_items, int ncand, uint32_t *__restrict__ cl,
			uint32_t *__restrict__ co, uint32_t *__restrict__ cm)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n_items * ncand)
		return;
	const DPair &p = P[t / ncand];
	const int c = t % ncand;
	uint32_t l = 0, o = 0, m = 0;
	for (int s = 0; s < 2; ++s) {
		l += (uint32_t)p.s[c][s].n;
		o += (uint32_t)p.s[c][s].cig.n;
		m += (uint32_t)p.s[c][s].cig.nm;
	}
	cl[t] = l;
	co[t] = o;
	cm[t] = m;
}

__global__ void k_emit(const DPair *__restrict__ P, int n_items, int ncand,
		       const uint32_t *__restrict__ xl, const uint32_t *__restrict__ xo,
		       const uint32_t *__restrict__ xm, hera_cand_rec *__restrict__ recs,
		       uint32_t *__restrict__ pos_pool, int32_t *__restrict__ p_pool,
		       uint32_t *__restrict__ op_pool, uint8_t *__restrict__ miss_pool,
		       uint64_t base_l, uint64_t base_o, uint64_t base_m)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n_items * ncand)
		return;
	const DPair &p = P[t / ncand];
	const int c = t % ncand;
	uint32_t l = xl[t], o = xo[t], m = xm[t];
	hera_cand_rec r;
	r.pair = p.pair[c];
	for (int s = 0; s < 2; ++s) {
		const DSlot &S = p.s[c][s];
		r.n[s] = S.n;
		r.err[s] = S.err;
		r.list_off[s] = (uint32_t)(base_l + l);
		r.cig_off[s] = (uint32_t)(base_o + o);
		r.miss_off[s] = (uint32_t)(base_m + m);
		r.n_cigar[s] = (uint16_t)S.cig.n;
		r.n_miss[s] = (uint16_t)S.cig.nm;
		for (int i = 0; i < S.n; ++i) {
			pos_pool[l + i] = S.t[i];
			p_pool[l + i] = S.p[i];
		}
		for (int i = 0; i < S.cig.n; ++i)
			op_pool[o + i] = S.cig.op[i];
		for (int i = 0; i < S.cig.nm; ++i)
			miss_pool[m + i] = S.cig.miss[i];
		l += (uint32_t)S.n;
		o += (uint32_t)S.cig.n;
		m += (uint32_t)S.cig.nm;
	}
	recs[t] = r;
}

#include "hera_batched.cuh"

}  // namespace

// ===========================================================================
// host side
// ===========================================================================

template <typename T>
struct DBuf {
	T *p = nullptr;
	size_t cap = 0;
	cudaError_t ensure(size_t n)
	{
		if (n <= cap)
			return cudaSuccess;
		if (p)
			cudaFree(p);
		p = nullptr;
		cap = 0;
		size_t want = n + n / 4 + 16;
		cudaError_t e = cudaMalloc(&p, want * sizeof(T));
		if (e == cudaSuccess)
			cap = want;
		return e;
	}
	void release()
	{
		if (p)
			cudaFree(p);
		p = nullptr;
		cap = 0;
	}
};

template <typename T>
struct HBuf {   // pinned host staging
	T *p = nullptr;
	size_t cap = 0;
	cudaError_t ensure(size_t n)
	{
		if (n <= cap)
			return cudaSuccess;
		if (p)
			cudaFreeHost(p);
		p = nullptr;
		cap = 0;
		size_t want = n + n / 4 + 16;
		cudaError_t e = cudaMallocHost(&p, want * sizeof(T));
		if (e == cudaSuccess)
			cap = want;
		return e;
	}
	void release()
	{
		if (p)
			cudaFreeHost(p);
		p = nullptr;
		cap = 0;
	}
};

struct hera_gpu_ctx {
	int device = 0;
	cudaStream_t stream = nullptr;
	DevIndex ix{};
	uint32_t *d_boff = nullptr;
	uint4 *d_bk = nullptr;
	uint2 *d_occ = nullptr;
	uint8_t *d_seq = nullptr, *d_tcode = nullptr;
	uint32_t *d_tlen = nullptr, *d_tstart = nullptr;
	uint32_t max_batch = 1u << 20;
	uint64_t scratch_bytes = 2ull << 30;

	// per-batch device buffers
	DBuf<uint8_t> seq, code;
	DBuf<int64_t> off;
	DBuf<int32_t> len;
	DBuf<uint2> hits;
	DBuf<DPair> pairs;
	DBuf<RmReq> q[2];
	DBuf<int> counters;     // [0] flags, [1..2] queue sizes
	DBuf<uint32_t> cnt;     // 3 * (items+1) counts, then 3 * (items+1) offsets
	DBuf<uint8_t> cub_tmp;
	DBuf<uint8_t> scratch;
	DBuf<uint8_t> code_r;
	DBuf<GpReq> qg[2];
	DBuf<TaskInfo> tinfo;
	DBuf<Chain> chains;
	DBuf<DpJob> jobs;
	DBuf<JobSlot> slots;
	DBuf<uint8_t> res;
	DBuf<int> perm, hist;
	size_t chain_cap = 0, job_cap = 0, slot_cap = 0;
	int batched = 1;
	DBuf<int2> calls;
	DBuf<int> rq_base;
	DBuf<SswOut> ssw_out;
	DBuf<hera_cand_rec> recs;
	DBuf<uint32_t> pos_pool, op_pool;
	DBuf<int32_t> p_pool;
	DBuf<uint8_t> miss_pool;

	// pinned staging
	HBuf<uint8_t> h_seq;
	HBuf<int64_t> h_off;
	HBuf<int32_t> h_len;
	HBuf<int> h_small;

	cudaEvent_t ev[8]{};
	hera_gpu_timing timing{};
	std::string err = "no error";

	// device-resident result of the last hera_gpu_align_pairs_device call
	int32_t last_items = 0, last_ncand = 0;
	uint64_t last_l = 0, last_o = 0, last_m = 0;
};

static int fail(hera_gpu_ctx *c, int code, const char *what, cudaError_t e = cudaSuccess)
{
	if (c) {
		char buf[512];
		if (e != cudaSuccess)
			snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
		else
			snprintf(buf, sizeof buf, "%s", what);
		c->err = buf;
	}
	return code;
}

#define CK(call, what)                                                    \
	do {                                                              \
		cudaError_t e_ = (call);                                  \
		if (e_ != cudaSuccess)                                    \
			return fail(ctx, e_ == cudaErrorMemoryAllocation ? HERA_GPU_ENOMEM : HERA_GPU_ECUDA, what, e_); \
	} while (0)

static unsigned blocks_for(int64_t n, int tpb = TPB)
{
	return (unsigned)((n + tpb - 1) / tpb);
}

extern "C" int hera_gpu_abi_version(void)
{
	return HERA_GPU_ABI_VERSION;
}

extern "C" const char *hera_gpu_last_error(const hera_gpu_ctx *ctx)
{
	return ctx ? ctx->err.c_str() : "null context";
}

extern "C" void *hera_gpu_stream(hera_gpu_ctx *ctx)
{
	return ctx ? (void *)ctx->stream : nullptr;
}

extern "C" int hera_gpu_get_timing(const hera_gpu_ctx *ctx, hera_gpu_timing *out)
{
	if (!ctx || !out)
		return HERA_GPU_EINVAL;
	*out = ctx->timing;
	return HERA_GPU_OK;
}

extern "C" void hera_gpu_ctx_destroy(hera_gpu_ctx *ctx)
{
	if (!ctx)
		return;
	cudaSetDevice(ctx->device);
	if (ctx->stream)
		cudaStreamSynchronize(ctx->stream);
	cudaFree(ctx->d_boff);
	cudaFree(ctx->d_bk);
	cudaFree(ctx->d_occ);
	cudaFree(ctx->d_seq);
	cudaFree(ctx->d_tcode);
	cudaFree(ctx->d_tlen);
	cudaFree(ctx->d_tstart);
	ctx->seq.release(); ctx->code.release(); ctx->off.release(); ctx->len.release();
	ctx->hits.release(); ctx->pairs.release(); ctx->q[0].release(); ctx->q[1].release();
	ctx->counters.release(); ctx->cnt.release(); ctx->cub_tmp.release(); ctx->scratch.release();
	ctx->calls.release(); ctx->rq_base.release(); ctx->ssw_out.release();
	ctx->code_r.release(); ctx->qg[0].release(); ctx->qg[1].release(); ctx->tinfo.release();
	ctx->chains.release(); ctx->jobs.release(); ctx->slots.release(); ctx->res.release(); ctx->perm.release(); ctx->hist.release();
	ctx->recs.release(); ctx->pos_pool.release(); ctx->op_pool.release(); ctx->p_pool.release();
	ctx->miss_pool.release();
	ctx->h_seq.release(); ctx->h_off.release(); ctx->h_len.release(); ctx->h_small.release();
	for (auto &e : ctx->ev)
		if (e)
			cudaEventDestroy(e);
	if (ctx->stream)
		cudaStreamDestroy(ctx->stream);
	delete ctx;
}

extern "C" int hera_gpu_ctx_create(const hera_gpu_index_view *v, const hera_gpu_options *opt,
				   hera_gpu_ctx **out)
{
	hera_gpu_ctx *ctx = nullptr;
	if (!out || !v || !v->len || !v->find || !v->seq || !v->bucket_n || !v->pos || !v->p ||
	    v->n_trans == 0)
		return HERA_GPU_EINVAL;
	*out = nullptr;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
		return HERA_GPU_ENODEV;
	ctx = new hera_gpu_ctx();
	if (opt) {
		ctx->device = opt->device;
		if (opt->max_batch)
			ctx->max_batch = opt->max_batch;
		if (opt->scratch_bytes)
			ctx->scratch_bytes = opt->scratch_bytes;
		ctx->batched = opt->path == HERA_GPU_PATH_PLAIN ? 0 : 1;
	}
	auto bail = [&](int rc) {
		std::string e = ctx->err;
		hera_gpu_ctx_destroy(ctx);
		(void)e;
		return rc;
	};
	if (cudaSetDevice(ctx->device) != cudaSuccess)
		return bail(HERA_GPU_ENODEV);
	if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
		return bail(HERA_GPU_ECUDA);
	for (auto &e : ctx->ev)
		cudaEventCreate(&e);

	const uint64_t H = 1ull << HBITS;
	const uint32_t n = v->n_trans;
	const uint64_t seq_len = v->find[n - 1];
	// bucket offsets: prefix sums of the per-bucket counts
	std::vector<uint32_t> boff(H + 1);
	uint64_t acc = 0;
	for (uint64_t i = 0; i < H; ++i) {
		boff[i] = (uint32_t)acc;
		acc += v->bucket_n[i];
	}
	boff[H] = (uint32_t)acc;
	if (acc != v->n_buckets || acc >= (1ull << 32))
		return bail(fail(ctx, HERA_GPU_EINVAL, "bucket counts do not match n_buckets"));
	std::vector<uint2> occ(v->n_pos);
	for (uint32_t i = 0; i < v->n_pos; ++i)
		occ[i] = make_uint2(v->pos[i], v->p[i]);
	std::vector<uint32_t> tstart(n);
	for (uint32_t i = 0; i < n; ++i)
		tstart[i] = v->find[i] - v->len[i];
	const size_t pad = 64;
	std::vector<uint8_t> seqp(seq_len + pad, 0);
	memcpy(seqp.data(), v->seq, seq_len);

	cudaError_t e;
	if ((e = cudaMalloc(&ctx->d_boff, (H + 1) * 4)) != cudaSuccess ||
	    (e = cudaMalloc(&ctx->d_bk, (acc ? acc : 1) * 16)) != cudaSuccess ||
	    (e = cudaMalloc(&ctx->d_occ, (v->n_pos ? v->n_pos : 1) * 8ull)) != cudaSuccess ||
	    (e = cudaMalloc(&ctx->d_seq, seq_len + pad)) != cudaSuccess ||
	    (e = cudaMalloc(&ctx->d_tcode, seq_len + pad)) != cudaSuccess ||
	    (e = cudaMalloc(&ctx->d_tlen, n * 4ull)) != cudaSuccess ||
	    (e = cudaMalloc(&ctx->d_tstart, n * 4ull)) != cudaSuccess)
		return bail(fail(ctx, HERA_GPU_ENOMEM, "index allocation", e));
	if ((e = cudaMemcpy(ctx->d_boff, boff.data(), (H + 1) * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
	    (acc && (e = cudaMemcpy(ctx->d_bk, v->buckets, acc * 16, cudaMemcpyHostToDevice)) != cudaSuccess) ||
	    (v->n_pos && (e = cudaMemcpy(ctx->d_occ, occ.data(), v->n_pos * 8ull, cudaMemcpyHostToDevice)) != cudaSuccess) ||
	    (e = cudaMemcpy(ctx->d_seq, seqp.data(), seq_len + pad, cudaMemcpyHostToDevice)) != cudaSuccess ||
	    (e = cudaMemcpy(ctx->d_tlen, v->len, n * 4ull, cudaMemcpyHostToDevice)) != cudaSuccess ||
	    (e = cudaMemcpy(ctx->d_tstart, tstart.data(), n * 4ull, cudaMemcpyHostToDevice)) != cudaSuccess)
		return bail(fail(ctx, HERA_GPU_ECUDA, "index upload", e));
	k_codes<<<1184, 256, 0, ctx->stream>>>(ctx->d_seq, ctx->d_tcode, (int64_t)(seq_len + pad));
	// padding after the last transcript codes as 4 (k_codes maps 0 -> 4)
	if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
		return bail(fail(ctx, HERA_GPU_ECUDA, "index codes", e));
	ctx->ix.boff = ctx->d_boff;
	ctx->ix.bk = ctx->d_bk;
	ctx->ix.occ = ctx->d_occ;
	ctx->ix.seq = ctx->d_seq;
	ctx->ix.code = ctx->d_tcode;
	ctx->ix.tlen = ctx->d_tlen;
	ctx->ix.tstart = ctx->d_tstart;
	ctx->ix.n_trans = n;
	*out = ctx;
	return HERA_GPU_OK;
}

// ---- pipeline pieces --------------------------------------------------

// one rescue round (re_mapSW for every queued request)
static int rescue_round(hera_gpu_ctx *ctx, const Batch &b, const RmReq *q, int nq, int max_len,
			cudaStream_t st, uint32_t &launches, float &ms_acc)
{
	CK(ctx->calls.ensure((size_t)nq * LCAP), "rescue calls");
	CK(ctx->rq_base.ensure(nq), "rescue bases");
	int *d_nc = ctx->counters.p + 4;
	CK(cudaMemsetAsync(d_nc, 0, sizeof(int), st), "memset");
	cudaEvent_t e0 = ctx->ev[6], e1 = ctx->ev[7];
	cudaEventRecord(e0, st);
	k_rescue_expand<<<blocks_for(nq, 256), 256, 0, st>>>(b, q, nq, ctx->calls.p, ctx->rq_base.p, d_nc);
	++launches;
	CK(cudaMemcpyAsync(ctx->h_small.p + 1, d_nc, sizeof(int), cudaMemcpyDeviceToHost, st), "calls");
	CK(cudaStreamSynchronize(st), "rescue expand");
	const int ncalls = ctx->h_small.p[1];
	CK(ctx->ssw_out.ensure(ncalls + 1), "rescue outputs");
	const size_t per = ssw_scratch_bytes(max_len);
	size_t slots = ctx->scratch_bytes / per;
	if (slots < 1)
		slots = 1;
	if (slots > (size_t)ncalls)
		slots = (size_t)(ncalls > 0 ? ncalls : 1);
	CK(ctx->scratch.ensure(slots * per), "rescue scratch");
	for (int c0 = 0; c0 < ncalls; c0 += (int)slots) {
		const int m = (int)((size_t)(ncalls - c0) < slots ? (size_t)(ncalls - c0) : slots);
		k_rescue_sw<<<blocks_for((int64_t)m * 32), TPB, 0, st>>>(b, q, ctx->calls.p, c0, m, ctx->ssw_out.p,
									 ctx->scratch.p, per);
		++launches;
	}
	k_rescue_fin<<<blocks_for(nq, 256), 256, 0, st>>>(b, q, nq, ctx->rq_base.p, ctx->ssw_out.p);
	++launches;
	cudaEventRecord(e1, st);
	CK(cudaStreamSynchronize(st), "rescue");
	float ms = 0;
	cudaEventElapsedTime(&ms, e0, e1);
	ms_acc += ms;
	return HERA_GPU_OK;
}

// one round of batched get_position calls: build, bin, DP, replay
static int gp_round(hera_gpu_ctx *ctx, const Batch &b, Round R, cudaStream_t st, uint32_t &launches,
		    float &build_ms, float &dp_ms)
{
	if (R.ntask <= 0)
		return HERA_GPU_OK;
	const int rcap = b.score_only ? 2 : JCAP;
	CK(ctx->tinfo.ensure(R.ntask), "task info");
	if (ctx->chain_cap < 2 * (size_t)R.ntask)
		ctx->chain_cap = 2 * (size_t)R.ntask;
	if (ctx->job_cap < 3 * (size_t)R.ntask)
		ctx->job_cap = 3 * (size_t)R.ntask;
	if (ctx->slot_cap < 4 * (size_t)R.ntask)
		ctx->slot_cap = 4 * (size_t)R.ntask;
	int *d_cnt = ctx->counters.p + 12;
	cudaEvent_t e0 = ctx->ev[6], e1 = ctx->ev[7];
	int nch = 0, nj = 0;
	cudaEventRecord(e0, st);
	for (int attempt = 0; attempt < 2; ++attempt) {
		CK(ctx->chains.ensure(ctx->chain_cap), "chains");
		CK(ctx->jobs.ensure(ctx->job_cap), "dp jobs");
		CK(ctx->slots.ensure(ctx->slot_cap), "job slots");
		R.tinfo = ctx->tinfo.p;
		R.chains = ctx->chains.p;
		R.slots = ctx->slots.p;
		R.jobs = ctx->jobs.p;
		R.cnt = d_cnt;
		R.chain_cap = (int)ctx->chain_cap;
		R.job_cap = (int)ctx->job_cap;
		R.slot_cap = (int)ctx->slot_cap;
		CK(cudaMemsetAsync(d_cnt, 0, 3 * sizeof(int), st), "memset");
		k_build<<<blocks_for(R.ntask), 128, 0, st>>>(b, R);
		++launches;
		CK(cudaMemcpyAsync(ctx->h_small.p + 12, d_cnt, 3 * sizeof(int), cudaMemcpyDeviceToHost, st), "counts");
		CK(cudaStreamSynchronize(st), "build");
		nch = ctx->h_small.p[12];
		nj = ctx->h_small.p[13];
		const int ns = ctx->h_small.p[14];
		ctx->timing.dp_calls += (uint64_t)ns;
		if ((size_t)nch <= ctx->chain_cap && (size_t)nj <= ctx->job_cap && (size_t)ns <= ctx->slot_cap)
			break;
		ctx->timing.dp_calls -= (uint64_t)ns;
		ctx->chain_cap = (size_t)nch + 16;
		ctx->job_cap = (size_t)nj + 16;
		ctx->slot_cap = (size_t)ns + 16;
		if (attempt == 1)
			return fail(ctx, HERA_GPU_ECAPACITY, "dp job buffers");
	}
	cudaEventRecord(e1, st);
	float ms = 0;
	CK(cudaEventSynchronize(e1), "build");
	cudaEventElapsedTime(&ms, e0, e1);
	build_ms += ms;
	cudaEventRecord(e0, st);
	R.res = nullptr;
	R.rcap = rcap;
	if (nj > 0) {
		CK(ctx->res.ensure((size_t)nj * res_stride(rcap)), "dp results");
		CK(ctx->perm.ensure(nj), "dp order");
		CK(ctx->hist.ensure(NBIN), "dp bins");
		CK(cudaMemsetAsync(ctx->hist.p, 0, NBIN * sizeof(int), st), "memset");
		k_bin_count<<<blocks_for(nj, 256), 256, 0, st>>>(ctx->jobs.p, nj, ctx->hist.p);
		k_bin_scan<<<1, 256, 0, st>>>(ctx->hist.p, NBIN);
		k_bin_scatter<<<blocks_for(nj, 256), 256, 0, st>>>(ctx->jobs.p, nj, ctx->hist.p, ctx->perm.p);
		k_dp<<<blocks_for(nj), 128, 0, st>>>(b, ctx->jobs.p, ctx->perm.p, nj, ctx->res.p, rcap);
		launches += 4;
		R.res = ctx->res.p;
	}
	k_replay<<<blocks_for(R.ntask), 128, 0, st>>>(b, R);
	++launches;
	cudaEventRecord(e1, st);
	CK(cudaEventSynchronize(e1), "replay");
	cudaEventElapsedTime(&ms, e0, e1);
	dp_ms += ms;
	ctx->timing.dp_jobs += (uint64_t)nj;
	return HERA_GPU_OK;
}

// Run the device pipeline on staged reads (2 * n reads for pairs, n
// singles otherwise).  Leaves the packed results in the device pools and
// their sizes in last_*.
static int run_batch(hera_gpu_ctx *ctx, const uint8_t *d_seq, const int64_t *d_off,
		     const int32_t *d_len, int32_t n, bool paired, int write_bam, int max_len,
		     int64_t seq_bytes, cudaStream_t st)
{
	const int n_reads = paired ? 2 * n : n;
	const int ncand = paired ? 2 : 1;
	const int items = n * ncand;
	const bool batched = ctx->batched && paired;
	hera_gpu_timing &T = ctx->timing;
	uint32_t launches = 0;

	CK(ctx->code.ensure(seq_bytes + 64), "read code buffer");
	if (batched)
		CK(ctx->code_r.ensure(seq_bytes + 64), "read code buffer");
	CK(ctx->pairs.ensure(n), "pair state");
	CK(ctx->counters.ensure(16), "counters");
	CK(ctx->q[0].ensure(n), "rescue queue");
	CK(ctx->q[1].ensure(n), "rescue queue");
	CK(ctx->cnt.ensure(6 * (size_t)(items + 1)), "count buffer");
	CK(ctx->recs.ensure(items), "records");
	CK(ctx->h_small.ensure(16), "host counters");
	int *d_flags = ctx->counters.p;
	CK(cudaMemsetAsync(ctx->counters.p, 0, 16 * sizeof(int), st), "memset");

	Batch b;
	b.ix = ctx->ix;
	b.code = ctx->code.p;
	b.code_r = batched ? ctx->code_r.p : nullptr;
	b.off = d_off;
	b.len = d_len;
	b.P = ctx->pairs.p;
	b.flags = d_flags;
	b.score_only = write_bam == 1;
	b.max_len = max_len;

	cudaEventRecord(ctx->ev[1], st);
	if (seq_bytes > 0) {
		k_codes<<<1184, 256, 0, st>>>(d_seq, ctx->code.p, seq_bytes);
		++launches;
		if (batched) {
			k_rc<<<blocks_for((int64_t)n_reads * 32, 256), 256, 0, st>>>(ctx->code.p, d_off, d_len, n_reads,
										      max_len, ctx->code_r.p);
			++launches;
		}
	}
	const int spr = max_len >= KMER ? (max_len - KMER) / KMER + 1 : 1;
	if (paired) {
		CK(ctx->hits.ensure((size_t)n_reads * 2 * spr), "seed hits");
		const int64_t ns = (int64_t)n_reads * 2 * spr;
		k_seed<<<blocks_for(ns, 256), 256, 0, st>>>(ctx->ix, ctx->code.p, d_off, d_len, n_reads, spr,
							     ctx->hits.p);
		++launches;
		T.lookups += (uint64_t)ns;
	}
	cudaEventRecord(ctx->ev[2], st);
	float resolve_ms = 0, rescue_ms = 0, build_ms = 0, dp_ms = 0;
	uint32_t rounds = 0;
	if (!paired) {
		k_single<<<blocks_for(n), TPB, 0, st>>>(b, n);
		++launches;
		cudaEventRecord(ctx->ev[3], st);
	} else if (!batched) {
		// plain form: one thread per get_position call / pair
		k_position<<<blocks_for((int64_t)n * 4), TPB, 0, st>>>(b, n, spr, ctx->hits.p);
		++launches;
		cudaEventRecord(ctx->ev[3], st);
		const RmReq *resume = nullptr;
		int nact = n, qi = 0;
		while (nact > 0) {
			int *qn = ctx->counters.p + 1 + qi;
			CK(cudaMemsetAsync(qn, 0, sizeof(int), st), "memset");
			cudaEvent_t e0 = ctx->ev[6], e1 = ctx->ev[7];
			cudaEventRecord(e0, st);
			k_resolve<<<blocks_for(nact), TPB, 0, st>>>(b, resume, nact, ctx->q[qi].p, qn);
			++launches;
			cudaEventRecord(e1, st);
			CK(cudaMemcpyAsync(ctx->h_small.p, qn, sizeof(int), cudaMemcpyDeviceToHost, st), "queue size");
			CK(cudaStreamSynchronize(st), "resolve");
			float ms = 0;
			cudaEventElapsedTime(&ms, e0, e1);
			resolve_ms += ms;
			const int nq = ctx->h_small.p[0];
			if (nq == 0)
				break;
			++rounds;
			int rc = rescue_round(ctx, b, ctx->q[qi].p, nq, max_len, st, launches, rescue_ms);
			if (rc)
				return rc;
			resume = ctx->q[qi].p;
			nact = nq;
			qi ^= 1;
		}
	} else {
		// batched form: rounds of batched get_position calls and rescues
		CK(ctx->qg[0].ensure(n), "gp queue");
		CK(ctx->qg[1].ensure(n), "gp queue");
		Round R{};
		R.req = nullptr;
		R.ntask = 4 * n;
		R.space = KMER;
		R.hits = ctx->hits.p;
		R.spr = spr;
		int rc = gp_round(ctx, b, R, st, launches, build_ms, dp_ms);
		if (rc)
			return rc;
		cudaEventRecord(ctx->ev[3], st);
		int ng = n, nr = 0, qi = 0;
		bool all = true;
		for (;;) {
			int *qng = ctx->counters.p + 8 + 2 * qi, *qnr = qng + 1;
			CK(cudaMemsetAsync(qng, 0, 2 * sizeof(int), st), "memset");
			cudaEvent_t e0 = ctx->ev[6], e1 = ctx->ev[7];
			cudaEventRecord(e0, st);
			k_resolve_b<<<blocks_for(ng + nr), 128, 0, st>>>(b, ctx->qg[qi ^ 1].p, ng, ctx->q[qi ^ 1].p, nr,
									  all ? 1 : 0, ctx->qg[qi].p, qng,
									  ctx->q[qi].p, qnr);
			++launches;
			cudaEventRecord(e1, st);
			CK(cudaMemcpyAsync(ctx->h_small.p + 10, qng, 2 * sizeof(int), cudaMemcpyDeviceToHost, st), "queues");
			CK(cudaStreamSynchronize(st), "resolve");
			float ms = 0;
			cudaEventElapsedTime(&ms, e0, e1);
			resolve_ms += ms;
			all = false;
			ng = ctx->h_small.p[10];
			nr = ctx->h_small.p[11];
			if (ng + nr == 0)
				break;
			++rounds;
			if (ng) {
				Round G{};
				G.req = ctx->qg[qi].p;
				G.ntask = ng;
				G.space = 2 * ERR;
				G.hits = nullptr;
				G.spr = 0;
				rc = gp_round(ctx, b, G, st, launches, build_ms, dp_ms);
				if (rc)
					return rc;
			}
			if (nr) {
				rc = rescue_round(ctx, b, ctx->q[qi].p, nr, max_len, st, launches, rescue_ms);
				if (rc)
					return rc;
			}
			qi ^= 1;
		}
	}
	cudaEventRecord(ctx->ev[4], st);
	// pack
	uint32_t *cl = ctx->cnt.p, *co = cl + (items + 1), *cm = co + (items + 1);
	uint32_t *xl = cm + (items + 1), *xo = xl + (items + 1), *xm = xo + (items + 1);
	CK(cudaMemsetAsync(cl, 0, 3 * sizeof(uint32_t) * (items + 1), st), "memset");
	k_count<<<blocks_for(items, 256), 256, 0, st>>>(ctx->pairs.p, n, ncand, cl, co, cm);
	++launches;
	size_t tmp_bytes = 0;
	cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cl, xl, items + 1, st);
	CK(ctx->cub_tmp.ensure(tmp_bytes), "scan scratch");
	cub::DeviceScan::ExclusiveSum(ctx->cub_tmp.p, tmp_bytes, cl, xl, items + 1, st);
	cub::DeviceScan::ExclusiveSum(ctx->cub_tmp.p, tmp_bytes, co, xo, items + 1, st);
	cub::DeviceScan::ExclusiveSum(ctx->cub_tmp.p, tmp_bytes, cm, xm, items + 1, st);
	CK(cudaMemcpyAsync(ctx->h_small.p + 2, xl + items, 4, cudaMemcpyDeviceToHost, st), "totals");
	CK(cudaMemcpyAsync(ctx->h_small.p + 3, xo + items, 4, cudaMemcpyDeviceToHost, st), "totals");
	CK(cudaMemcpyAsync(ctx->h_small.p + 4, xm + items, 4, cudaMemcpyDeviceToHost, st), "totals");
	CK(cudaMemcpyAsync(ctx->h_small.p + 5, d_flags, 4, cudaMemcpyDeviceToHost, st), "flags");
	CK(cudaStreamSynchronize(st), "scan");
	const uint32_t tl = (uint32_t)ctx->h_small.p[2], to = (uint32_t)ctx->h_small.p[3],
		       tm = (uint32_t)ctx->h_small.p[4];
	const int fl = ctx->h_small.p[5];
	CK(ctx->pos_pool.ensure(tl + 1), "list pool");
	CK(ctx->p_pool.ensure(tl + 1), "list pool");
	CK(ctx->op_pool.ensure(to + 1), "op pool");
	CK(ctx->miss_pool.ensure(tm + 1), "miss pool");
	k_emit<<<blocks_for(items, 256), 256, 0, st>>>(ctx->pairs.p, n, ncand, xl, xo, xm, ctx->recs.p,
							ctx->pos_pool.p, ctx->p_pool.p, ctx->op_pool.p,
							ctx->miss_pool.p, 0, 0, 0);
	++launches;
	cudaEventRecord(ctx->ev[5], st);
	CK(cudaGetLastError(), "kernel launch");
	CK(cudaStreamSynchronize(st), "pack");
	float ms = 0;
	cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
	T.seed_ms += ms;
	if (!batched) {
		cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
		T.position_ms += ms;
	} else {
		T.position_ms += build_ms + dp_ms;
		T.build_ms += build_ms;
		T.dp_ms += dp_ms;
	}
	T.resolve_ms += resolve_ms;
	T.rescue_ms += rescue_ms;
	cudaEventElapsedTime(&ms, ctx->ev[4], ctx->ev[5]);
	T.pack_ms += ms;
	T.launches += launches;
	T.rescue_rounds += rounds;
	ctx->last_items = items;
	ctx->last_ncand = ncand;
	ctx->last_l = tl;
	ctx->last_o = to;
	ctx->last_m = tm;
	if (fl) {
		char buf[160];
		snprintf(buf, sizeof buf, "per-read capacity exceeded (flags 0x%x)", fl);
		return fail(ctx, HERA_GPU_ECAPACITY, buf);
	}
	return HERA_GPU_OK;
}

// copy the packed device results into `out` at record `rec0`, shifting
// pool offsets by what `out` already holds
static int copy_out(hera_gpu_ctx *ctx, hera_gpu_result *out, uint64_t rec0, cudaStream_t st,
		    bool *fits)
{
	const uint64_t bl = out->list_used, bo = out->op_used, bm = out->miss_used;
	const int items = ctx->last_items;
	*fits = bl + ctx->last_l <= out->list_cap && bo + ctx->last_o <= out->op_cap &&
		bm + ctx->last_m <= out->miss_cap;
	if (*fits) {
		CK(cudaMemcpyAsync(out->recs + rec0, ctx->recs.p, items * sizeof(hera_cand_rec),
				   cudaMemcpyDeviceToHost, st), "records D2H");
		if (ctx->last_l) {
			CK(cudaMemcpyAsync(out->pos_pool + bl, ctx->pos_pool.p, ctx->last_l * 4, cudaMemcpyDeviceToHost, st), "D2H");
			CK(cudaMemcpyAsync(out->p_pool + bl, ctx->p_pool.p, ctx->last_l * 4, cudaMemcpyDeviceToHost, st), "D2H");
		}
		if (ctx->last_o)
			CK(cudaMemcpyAsync(out->op_pool + bo, ctx->op_pool.p, ctx->last_o * 4, cudaMemcpyDeviceToHost, st), "D2H");
		if (ctx->last_m)
			CK(cudaMemcpyAsync(out->miss_pool + bm, ctx->miss_pool.p, ctx->last_m, cudaMemcpyDeviceToHost, st), "D2H");
		CK(cudaStreamSynchronize(st), "D2H");
		if (bl | bo | bm) {
			for (int i = 0; i < items; ++i) {
				hera_cand_rec &r = out->recs[rec0 + i];
				for (int s = 0; s < 2; ++s) {
					r.list_off[s] += (uint32_t)bl;
					r.cig_off[s] += (uint32_t)bo;
					r.miss_off[s] += (uint32_t)bm;
				}
			}
		}
	}
	out->list_used = bl + ctx->last_l;
	out->op_used = bo + ctx->last_o;
	out->miss_used = bm + ctx->last_m;
	return HERA_GPU_OK;
}

// stage host reads (pairs interleaved) into pinned memory and the device
static int stage_reads(hera_gpu_ctx *ctx, const hera_gpu_reads *a, const hera_gpu_reads *b,
		       int32_t lo, int32_t n, int64_t *bytes, int *max_len, cudaStream_t st)
{
	const int per = b ? 2 : 1;
	int64_t total = 0;
	int ml = 0;
	for (int32_t i = lo; i < lo + n; ++i) {
		if (a->len[i] < 0 || (b && b->len[i] < 0))
			return fail(ctx, HERA_GPU_EINVAL, "negative read length");
		total += a->len[i] + (b ? b->len[i] : 0);
		ml = a->len[i] > ml ? a->len[i] : ml;
		if (b)
			ml = b->len[i] > ml ? b->len[i] : ml;
	}
	if (ml > MAX_READ)
		return fail(ctx, HERA_GPU_EINVAL, "read longer than HERA_GPU_MAX_READ");
	CK(ctx->h_seq.ensure(total + 1), "pinned reads");
	CK(ctx->h_off.ensure((size_t)n * per), "pinned offsets");
	CK(ctx->h_len.ensure((size_t)n * per), "pinned lengths");
	int64_t o = 0;
	for (int32_t i = 0; i < n; ++i) {
		const hera_gpu_reads *src[2] = {a, b};
		for (int m = 0; m < per; ++m) {
			const hera_gpu_reads *r = src[m];
			const int32_t L = r->len[lo + i];
			memcpy(ctx->h_seq.p + o, r->seq + r->off[lo + i], (size_t)L);
			ctx->h_off.p[(size_t)i * per + m] = o;
			ctx->h_len.p[(size_t)i * per + m] = L;
			o += L;
		}
	}
	CK(ctx->seq.ensure(total + 64), "device reads");
	CK(ctx->off.ensure((size_t)n * per), "device offsets");
	CK(ctx->len.ensure((size_t)n * per), "device lengths");
	CK(cudaMemcpyAsync(ctx->seq.p, ctx->h_seq.p, total, cudaMemcpyHostToDevice, st), "H2D reads");
	CK(cudaMemcpyAsync(ctx->off.p, ctx->h_off.p, (size_t)n * per * 8, cudaMemcpyHostToDevice, st), "H2D");
	CK(cudaMemcpyAsync(ctx->len.p, ctx->h_len.p, (size_t)n * per * 4, cudaMemcpyHostToDevice, st), "H2D");
	*bytes = total;
	*max_len = ml;
	return HERA_GPU_OK;
}

static int align_flat(hera_gpu_ctx *ctx, const hera_gpu_reads *r1, const hera_gpu_reads *r2, int32_t n,
		      int write_bam, hera_gpu_result *out)
{
	if (!ctx || !r1 || !out || n < 0 || (write_bam != 0 && write_bam != 1))
		return fail(ctx, HERA_GPU_EINVAL, "bad argument");
	if (cudaSetDevice(ctx->device) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENODEV, "cudaSetDevice");
	cudaStream_t st = ctx->stream;
	const bool paired = r2 != nullptr;
	const int ncand = paired ? 2 : 1;
	memset(&ctx->timing, 0, sizeof(ctx->timing));
	out->list_used = out->op_used = out->miss_used = 0;
	bool all_fit = true;
	cudaEventRecord(ctx->ev[0], st);
	for (int32_t lo = 0; lo < n; lo += (int32_t)ctx->max_batch) {
		const int32_t m = (n - lo) < (int32_t)ctx->max_batch ? (n - lo) : (int32_t)ctx->max_batch;
		int64_t bytes = 0;
		int max_len = 0;
		int rc = stage_reads(ctx, r1, r2, lo, m, &bytes, &max_len, st);
		if (rc)
			return rc;
		rc = run_batch(ctx, ctx->seq.p, ctx->off.p, ctx->len.p, m, paired, write_bam, max_len, bytes, st);
		if (rc)
			return rc;
		bool fits = true;
		if (all_fit) {
			rc = copy_out(ctx, out, (uint64_t)lo * ncand, st, &fits);
			if (rc)
				return rc;
			all_fit = fits;
		} else {
			out->list_used += ctx->last_l;
			out->op_used += ctx->last_o;
			out->miss_used += ctx->last_m;
		}
	}
	cudaEventRecord(ctx->ev[1], st);
	cudaEventSynchronize(ctx->ev[1]);
	cudaEventElapsedTime(&ctx->timing.total_ms, ctx->ev[0], ctx->ev[1]);
	if (!all_fit)
		return fail(ctx, HERA_GPU_ECAPACITY, "result pools too small (see *_used for the sizes needed)");
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_align_pairs_flat(hera_gpu_ctx *ctx, const hera_gpu_reads *r1,
					 const hera_gpu_reads *r2, int32_t n, int write_bam,
					 hera_gpu_result *out)
{
	if (!r2)
		return fail(ctx, HERA_GPU_EINVAL, "r2 is NULL");
	return align_flat(ctx, r1, r2, n, write_bam, out);
}

extern "C" int hera_gpu_align_single_flat(hera_gpu_ctx *ctx, const hera_gpu_reads *reads, int32_t n,
					  int write_bam, hera_gpu_result *out)
{
	return align_flat(ctx, reads, nullptr, n, write_bam, out);
}

extern "C" int hera_gpu_align_pairs_device(hera_gpu_ctx *ctx, const uint8_t *d_seq, const int64_t *d_off,
					   const int32_t *d_len, int32_t n, int32_t max_read_len, int write_bam,
					   void *stream)
{
	if (!ctx || !d_seq || !d_off || !d_len || n < 0 || (write_bam != 0 && write_bam != 1) ||
	    max_read_len < 1 || max_read_len > MAX_READ)
		return fail(ctx, HERA_GPU_EINVAL, "bad argument");
	if (cudaSetDevice(ctx->device) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENODEV, "cudaSetDevice");
	cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
	memset(&ctx->timing, 0, sizeof(ctx->timing));
	// total bytes and max read length of the device batch
	if (n == 0)
		return HERA_GPU_OK;
	int64_t last_off = 0;
	int32_t last_len = 0;
	CK(cudaMemcpyAsync(&last_off, d_off + 2 * (int64_t)n - 1, 8, cudaMemcpyDeviceToHost, st), "D2H");
	CK(cudaMemcpyAsync(&last_len, d_len + 2 * (int64_t)n - 1, 4, cudaMemcpyDeviceToHost, st), "D2H");
	CK(cudaStreamSynchronize(st), "sync");
	cudaEventRecord(ctx->ev[0], st);
	int rc = run_batch(ctx, d_seq, d_off, d_len, n, true, write_bam, max_read_len, last_off + last_len, st);
	cudaEventRecord(ctx->ev[1], st);
	cudaEventSynchronize(ctx->ev[1]);
	cudaEventElapsedTime(&ctx->timing.total_ms, ctx->ev[0], ctx->ev[1]);
	return rc;
}

extern "C" int hera_gpu_fetch_result(hera_gpu_ctx *ctx, hera_gpu_result *out)
{
	if (!ctx || !out)
		return HERA_GPU_EINVAL;
	out->list_used = out->op_used = out->miss_used = 0;
	bool fits = true;
	int rc = copy_out(ctx, out, 0, ctx->stream, &fits);
	if (rc)
		return rc;
	return fits ? HERA_GPU_OK : fail(ctx, HERA_GPU_ECAPACITY, "result pools too small");
}

// ---- drop-in Candidate form -------------------------------------------

static void upper_acgt(char *s, int32_t L)
{
	for (int32_t i = 0; i < L; ++i) {
		char c = s[i];
		if (c == 'a' || c == 'c' || c == 'g' || c == 't')
			s[i] = (char)(c - 32);
	}
}

static hera_candidate *materialize(const hera_gpu_result *res, uint64_t ri)
{
	const hera_cand_rec &r = res->recs[ri];
	hera_candidate *c = (hera_candidate *)malloc(sizeof(hera_candidate));
	if (!c)
		return nullptr;
	c->pair = r.pair;
	for (int s = 0; s < 2; ++s) {
		c->n[s] = (unsigned)r.n[s];
		c->err[s] = r.err[s];
		c->pos[s] = nullptr;
		c->p[s] = nullptr;
		if (r.n[s] > 0) {
			c->pos[s] = (unsigned *)malloc(sizeof(unsigned) * r.n[s]);
			c->p[s] = (int *)malloc(sizeof(int) * r.n[s]);
			memcpy(c->pos[s], res->pos_pool + r.list_off[s], sizeof(unsigned) * r.n[s]);
			memcpy(c->p[s], res->p_pool + r.list_off[s], sizeof(int) * r.n[s]);
		}
		hera_cigar *g = (hera_cigar *)malloc(sizeof(hera_cigar));
		g->n_cigar = r.n_cigar[s];
		g->n_miss = r.n_miss[s];
		g->count = nullptr;
		g->type = nullptr;
		g->miss = nullptr;
		if (g->n_cigar) {
			g->count = (unsigned short *)malloc(sizeof(unsigned short) * g->n_cigar);
			g->type = (char *)malloc(g->n_cigar);
			for (int i = 0; i < g->n_cigar; ++i) {
				uint32_t o = res->op_pool[r.cig_off[s] + i];
				g->count[i] = (unsigned short)(o >> 4);
				g->type[i] = (char)(o & 15);
			}
		}
		if (g->n_miss) {
			g->miss = (char *)malloc(g->n_miss);
			memcpy(g->miss, res->miss_pool + r.miss_off[s], g->n_miss);
		}
		c->cigar[s] = g;
	}
	return c;
}

static int align_dropin(hera_gpu_ctx *ctx, hera_read_inf *a, hera_read_inf *b, int32_t n, int write_bam,
			hera_candidate **out)
{
	if (!ctx || !a || !out || n < 0)
		return fail(ctx, HERA_GPU_EINVAL, "bad argument");
	const int per = b ? 2 : 1;
	std::vector<int64_t> off[2];
	std::vector<int32_t> len[2];
	std::vector<char> seq;
	int64_t total = 0;
	for (int32_t i = 0; i < n; ++i)
		total += a[i].len + (b ? b[i].len : 0);
	seq.resize((size_t)total + 1);
	int64_t o = 0;
	for (int m = 0; m < per; ++m) {
		hera_read_inf *r = m ? b : a;
		off[m].resize(n);
		len[m].resize(n);
		for (int32_t i = 0; i < n; ++i) {
			if (!r[i].seq || r[i].len < 0)
				return fail(ctx, HERA_GPU_EINVAL, "read without sequence");
			memcpy(seq.data() + o, r[i].seq, (size_t)r[i].len);
			off[m][i] = o;
			len[m][i] = r[i].len;
			o += r[i].len;
		}
	}
	hera_gpu_reads ra{seq.data(), off[0].data(), len[0].data()};
	hera_gpu_reads rb{seq.data(), b ? off[1].data() : nullptr, b ? len[1].data() : nullptr};
	const uint64_t items = (uint64_t)n * per;
	std::vector<hera_cand_rec> recs(items ? items : 1);
	hera_gpu_result res{};
	res.recs = recs.data();
	std::vector<uint32_t> pos, ops;
	std::vector<int32_t> p;
	std::vector<char> miss;
	uint64_t cl = items * 8 + 64, co = items * 8 + 64, cm = items * 8 + 64;
	for (int attempt = 0; attempt < 2; ++attempt) {
		pos.resize(cl);
		p.resize(cl);
		ops.resize(co);
		miss.resize(cm);
		res.pos_pool = pos.data();
		res.p_pool = p.data();
		res.op_pool = ops.data();
		res.miss_pool = miss.data();
		res.list_cap = cl;
		res.op_cap = co;
		res.miss_cap = cm;
		int rc = align_flat(ctx, &ra, b ? &rb : nullptr, n, write_bam, &res);
		if (rc == HERA_GPU_OK)
			break;
		if (rc != HERA_GPU_ECAPACITY || attempt == 1 ||
		    (res.list_used <= cl && res.op_used <= co && res.miss_used <= cm))
			return rc;
		cl = res.list_used + 1;
		co = res.op_used + 1;
		cm = res.miss_used + 1;
	}
	for (uint64_t i = 0; i < items; ++i) {
		out[i] = materialize(&res, i);
		if (!out[i])
			return fail(ctx, HERA_GPU_ENOMEM, "candidate allocation");
	}
	for (int32_t i = 0; i < n; ++i) {
		upper_acgt(a[i].seq, a[i].len);
		if (b)
			upper_acgt(b[i].seq, b[i].len);
	}
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_align_pairs(hera_gpu_ctx *ctx, hera_read_inf *r1, hera_read_inf *r2, int32_t n,
				    int write_bam, hera_candidate **out)
{
	if (!r2)
		return fail(ctx, HERA_GPU_EINVAL, "r2 is NULL");
	return align_dropin(ctx, r1, r2, n, write_bam, out);
}

extern "C" int hera_gpu_align_single(hera_gpu_ctx *ctx, hera_read_inf *reads, int32_t n, int write_bam,
				     hera_candidate **out)
{
	return align_dropin(ctx, reads, nullptr, n, write_bam, out);
}
