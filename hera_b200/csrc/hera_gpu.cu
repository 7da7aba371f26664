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
#include "hera_combine.h"
#include "../../include/hera_gpu.h"

#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <thread>
#include <vector>

using namespace hg;

namespace {

constexpr int TPB = 128;

// bytes of dynamic shared memory the running block was launched with
__device__ __forceinline__ unsigned dyn_smem_bytes()
{
	unsigned r;
	asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(r));
	return r;
}

struct RmReq {
	int32_t pair;
	int16_t c, str;
};

template <class K>
struct BatchT {
	DevIndex ix;
	const uint8_t *code;     // read codes
	const uint8_t *code_r;   // reverse-complement codes (read i at the same offset)
	const int64_t *off;      // read offsets (2 per pair: mate 1, mate 2)
	const int32_t *len;
	DPairT<K> *P;
	int *flags;
	unsigned long long *stats;   // work counters, ST_* slots
	int score_only;
	int max_len;             // longest read of the batch (seed table stride)
	// wide pass only: P[i] is the pair (or single read) pmap[i] of the
	// batch, and thread t of a per-task kernel works in work[t] (the
	// CapsWide working set is too large for local memory)
	const int *pmap;
	GpWorkT<K> *work;
	__device__ __forceinline__ int item(int i) const { return pmap ? pmap[i] : i; }
	// read of candidate c, strand str of the pair in P[i] (c ^ str == 0:
	// mate 1, src/hash_align.c:1667-1670)
	__device__ __forceinline__ int read_of(int i, int c, int str) const
	{
		return 2 * item(i) + ((c ^ str) == 0 ? 0 : 1);
	}
};
using Batch = BatchT<CapsStd>;

// per-task working set: a local variable in the first pass, the task's
// slot of b.work in the wide pass
template <class K, bool GLOBAL = (K::A > CapsStd::A)>
struct TaskWork;
template <class K>
struct TaskWork<K, false> {
	GpWorkT<K> w;
	__device__ __forceinline__ GpWorkT<K> &get(const BatchT<K> &, int) { return w; }
};
template <class K>
struct TaskWork<K, true> {
	__device__ __forceinline__ GpWorkT<K> &get(const BatchT<K> &b, int t) { return b.work[t]; }
};

// the capacity flags a pair met, kept with the pair (the wide pass re-runs
// it); every flag also goes to the batch's word
template <class K>
__device__ __forceinline__ void pair_flags(const BatchT<K> &b, int i, int f)
{
	if (f & F_CAPS)
		atomicOr(&b.P[i].ovf, f & F_CAPS);
}

// work counters (hera_gpu_timing's probes .. ssw_cells)
enum { ST_PROBES = 0, ST_SEED_HITS = 1, ST_SW_CELLS = 2, ST_SSW_CELLS = 3, ST_N = 4 };

__device__ __forceinline__ void flag(int *f, int v)
{
	if (v)
		atomicOr(f, v);
}

// add v over the whole warp to a counter (every lane of the warp calls it)
__device__ __forceinline__ void warp_stat(unsigned long long *c, uint32_t v)
{
	v = __reduce_add_sync(0xffffffffu, v);
	if ((threadIdx.x & 31) == 0 && v)
		atomicAdd(c, (unsigned long long)v);
}

// read `ri` in orientation `orient` (1 = reverse complement) into rd
template <class K>
__device__ __forceinline__ int load_read(const BatchT<K> &b, int ri, int orient, uint8_t *rd)
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

// code_of of four bytes at once: A/a 0, C/c 1, G/g 2, T/t 3, anything else 4
__device__ __forceinline__ uint32_t codes4(uint32_t v)
{
	const uint32_t x = v | 0x20202020u;
	const uint32_t a = __vcmpeq4(x, 0x61616161u), c = __vcmpeq4(x, 0x63636363u),
		       g = __vcmpeq4(x, 0x67676767u), t = __vcmpeq4(x, 0x74747474u);
	return (0x04040404u & ~(a | c | g | t)) | (c & 0x01010101u) | (g & 0x02020202u) | (t & 0x03030303u);
}

// ASCII -> codes, four bytes a thread: one aligned 4-byte store of `code`
// (whose base is 4-byte aligned) from the two aligned input words around
// the four bytes (`ascii` may start anywhere); a group whose second input
// word would reach past byte n - 1 is read byte by byte.
__global__ void k_codes(const uint8_t *__restrict__ ascii, uint8_t *__restrict__ code, int64_t n)
{
	const int s = (int)(reinterpret_cast<uintptr_t>(ascii) & 3);
	const uint32_t *w = reinterpret_cast<const uint32_t *>(ascii - s);
	const int64_t nw = (n + 3) >> 2;
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nw;
	     i += (int64_t)gridDim.x * blockDim.x) {
		const int64_t b0 = 4 * i;
		if (b0 + 7 - s < n) {
			const uint32_t v = s ? __funnelshift_r(__ldg(w + i), __ldg(w + i + 1), 8 * s) : __ldg(w + i);
			reinterpret_cast<uint32_t *>(code)[i] = codes4(v);
		} else {
			for (int64_t k = b0; k < b0 + 4 && k < n; ++k)
				code[k] = code_of(ascii[k]);
		}
	}
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

// seed_probe: thread per (read, strand) over its S seeds at spacing 31.
// The S lookups are independent, so their bucket-offset loads and then
// their binary-search probes are issued together (hash_get,
// src/hash_align.c:862-895; the same search and probe count as probe()).
template <int S>
__global__ void __launch_bounds__(256) k_seed(DevIndex ix, const uint8_t *__restrict__ code,
					       const int64_t *__restrict__ off, const int32_t *__restrict__ len,
					       int n_reads, uint2 *__restrict__ hits,
					       unsigned long long *__restrict__ stats)
{
	const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
	uint32_t np = 0, found = 0;
	if (t < (int64_t)n_reads * 2) {
		const int orient = (int)(t & 1);
		const int ri = (int)(t >> 1);
		const int L = len[ri];
		const uint8_t *src = code + off[ri];
		uint64_t id[S];
		uint32_t lo[S], hi[S];
		uint2 h[S];
#pragma unroll
		for (int j = 0; j < S; ++j) {
			const int i = j * KMER;
			h[j] = make_uint2(0, 0);
			lo[j] = hi[j] = 0;
			id[j] = 0;
			if (i + KMER <= L) {
				// orientation 1: the reverse complement's k-mer at i covers
				// bytes [L-1-i-30, L-1-i] of the read
				id[j] = orient == 0 ? kmer_words(src + i, false) : kmer_words(src + (L - KMER - i), true);
				const uint32_t mod = (uint32_t)(id[j] & HMASK);
				lo[j] = __ldg(ix.boff + mod);
				hi[j] = __ldg(ix.boff + mod + 1);
			}
		}
		bool more = true;
		while (more) {
			more = false;
#pragma unroll
			for (int j = 0; j < S; ++j) {
				if (lo[j] < hi[j]) {
					const uint32_t mid = (lo[j] + hi[j]) >> 1;
					++np;
					const uint4 b = __ldg(ix.bk + mid);
					const uint64_t bid = ((uint64_t)b.y << 32) | b.x;
					if (bid == id[j]) {
						h[j] = make_uint2(b.z, b.w - b.z);
						hi[j] = lo[j];
					} else if (bid > id[j]) {
						hi[j] = mid;
					} else {
						lo[j] = mid + 1;
					}
					more |= lo[j] < hi[j];
				}
			}
		}
#pragma unroll
		for (int j = 0; j < S; ++j) {
			hits[t * S + j] = h[j];
			found += h[j].y > 0;
		}
	}
	warp_stat(stats + ST_PROBES, np);
	warp_stat(stats + ST_SEED_HITS, found);
}

template <class K>
__device__ __forceinline__ void slot_reset(DSlotT<K> &S)
{
	S.n = 0;
	S.err = 0;
	S.cig.n = 0;
	S.cig.nm = 0;
}

// the four space-31 get_position calls of check_in_transcriptome
// (src/hash_align.c:1667-1670); independent because pass A needs space < 31
template <class K>
__global__ void __launch_bounds__(TPB) k_position(BatchT<K> b, int n_pairs, int spr, const uint2 *__restrict__ hits)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n_pairs * 4)
		return;
	const int pi = t >> 2, task = t & 3;
	const int c = task >> 1, str = task & 1;
	const int ri = b.read_of(pi, c, str);
	TaskWork<K> tw;
	GpWorkT<K> &w = tw.get(b, t);
	int flags = 0;
	DPairT<K> &P = b.P[pi];
	DSlotT<K> &S = P.s[c][str];
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
	pair_flags(b, pi, flags);
	flag(b.flags, flags);
}

// per-pair control flow after the space-31 calls (src/hash_align.c:1672-1695
// and :1730-1733 with intersect2/re_map :1504-1562).  A pair that needs a
// mate rescue enqueues it and stops; it resumes at P.stage next round.
template <class K>
__global__ void __launch_bounds__(TPB) k_resolve(BatchT<K> b, const RmReq *__restrict__ resume, int n,
						  RmReq *__restrict__ q, int *__restrict__ qn)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n)
		return;
	const int pi = resume ? resume[t].pair : t;
	DPairT<K> &P = b.P[pi];
	TaskWork<K> tw;
	GpWorkT<K> &w = tw.get(b, t);
	int flags = 0;
	auto gp = [&](int c, int str) {
		const int ri = b.read_of(pi, c, str);
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
	auto done = [&]() {
		pair_flags(b, pi, flags);
		flag(b.flags, flags);
	};
	if (b.len[b.read_of(pi, 0, 0)] > b.max_len || b.len[b.read_of(pi, 0, 1)] > b.max_len) {
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
			const DSlotT<K> &X = P.s[c][s], &Y = P.s[c][1 - s];
			const DSlotT<K> &O0 = P.s[1 - c][0], &O1 = P.s[1 - c][1];
			if (X.n == 0 && Y.n > 0 && Y.err < ERR && O0.err + O1.err > ERR) {
				gp(c, s);
				if (P.s[c][s].n == 0) {
					rescue(c, s, 10 + st);
					done();
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
					done();
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
				done();
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
			done();
			return;
		}
	}
}

// re_mapSW (src/hash_align.c:762-846), in three steps.
// 1) one ssw_align call per (queued request, mate hit)
template <class K>
__global__ void k_rescue_expand(BatchT<K> b, const RmReq *__restrict__ q, int nq, int2 *__restrict__ calls,
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

// 2) one warp per call: local SW over the MAX_FRAG window at the mate hit;
// each warp works in its own `per` bytes of the block's shared memory
constexpr int RESCUE_TPB = 256;   // at most 8 calls (warps) per block
constexpr int WIDE_RESCUE_WPB = 4;   // calls per block in the wide pass (CapsWide areas)
template <class K>
__global__ void __launch_bounds__(RESCUE_TPB) k_rescue_sw(BatchT<K> b, const RmReq *__restrict__ q,
							   const int2 *__restrict__ calls, int c0, int nc,
							   SswOutT<K> *__restrict__ out, int per)
{
	extern __shared__ __align__(16) uint8_t ssw_sm[];
	const int wl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;   // warp within launch
	if (wl >= nc)
		return;
	const int2 cl = calls[c0 + wl];
	const RmReq rq = q[cl.x];
	const DPairT<K> &P = b.P[rq.pair];
	const int c = rq.c, str = rq.str;
	const int type = str == 0 ? -1 : 1;
	const int ri = b.read_of(rq.pair, c, str);
	const int L = b.len[ri];
	const DSlotT<K> &M = P.s[c][1 - str];
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
	if (L < 0 || L > b.max_len || (size_t)((threadIdx.x >> 5) + 1) * per > dyn_smem_bytes()) {
		// longer than the batch's stated maximum, or no room for the area
		if ((threadIdx.x & 31) == 0) {
			out[c0 + wl].ok = 0;
			out[c0 + wl].cig.n = out[c0 + wl].cig.nm = 0;
			flag(b.flags, F_READ);
		}
		return;
	}
	ssw_warp(b.ix, __ldg(b.ix.tstart + tr) + (uint32_t)start, ln, b.code, b.off[ri], L, str, start, tl,
		 ssw_sm + (size_t)(threadIdx.x >> 5) * per, out[c0 + wl], flags);
	if ((threadIdx.x & 31) == 0) {
		pair_flags(b, rq.pair, flags);
		flag(b.flags, flags);
		atomicAdd(b.stats + ST_SSW_CELLS, (unsigned long long)ln * (unsigned long long)L);
	}
}

// 3) per request: min score wins, ties append in hit order; the mate's list
// is compacted to the rescued subset (src/hash_align.c:794-845)
template <class K>
__global__ void k_rescue_fin(BatchT<K> b, const RmReq *__restrict__ q, int nq, const int *__restrict__ base,
			     const SswOutT<K> *__restrict__ out)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= nq)
		return;
	const RmReq rq = q[t];
	DPairT<K> &P = b.P[rq.pair];
	const int c = rq.c, str = rq.str;
	DSlotT<K> &S = P.s[c][str];
	DSlotT<K> &M = P.s[c][1 - str];
	const int n = M.n, b0 = base[t];
	int new_n = 0, score2 = 0, best = -1;
	for (int i = 0; i < n; ++i) {
		const SswOutT<K> &o = out[b0 + i];
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
template <class K>
__global__ void __launch_bounds__(TPB) k_single(BatchT<K> b, int n)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n)
		return;
	DPairT<K> &P = b.P[t];
	const int ri = b.item(t);
	TaskWork<K> tw;
	GpWorkT<K> &w = tw.get(b, t);
	int flags = 0;
	slot_reset(P.s[0][0]);
	slot_reset(P.s[0][1]);
	P.pair[0] = 0;
	P.ovf = 0;
	if (b.len[ri] > b.max_len) {
		flag(b.flags, F_READ);
		P.s[0][0].err = P.s[0][1].err = b.len[ri];
		return;
	}
	int L = load_read(b, ri, 0, w.rd);
	get_position(b.ix, w.rd, L, P, 0, 0, 2 * ERR, nullptr, b.score_only != 0, w, flags);
	L = load_read(b, ri, 1, w.rd);
	get_position(b.ix, w.rd, L, P, 0, 1, 2 * ERR, nullptr, b.score_only != 0, w, flags);
	pair_flags(b, t, flags);
	flag(b.flags, flags);
}

// Records of the pairs that ran the wide pass, already packed (their own
// records and pools); the first pass's state of those pairs is ignored.
struct Side {
	const int *slot;            // per item of the batch: its side index, or -1
	const hera_cand_rec *recs;  // [side index * ncand + c]
	const uint32_t *pos;
	const int32_t *p;
	const uint32_t *op;
	const uint8_t *miss;
};

// per record: entries of the list / op / miss pools
template <class K>
__global__ void k_count(const DPairT<K> *__restrict__ P, int n_items, int ncand, uint32_t *__restrict__ cl,
			uint32_t *__restrict__ co, uint32_t *__restrict__ cm, Side side)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n_items * ncand)
		return;
	const int c = t % ncand;
	const int so = side.slot ? side.slot[t / ncand] : -1;
	uint32_t l = 0, o = 0, m = 0;
	if (so >= 0) {
		const hera_cand_rec &r = side.recs[(size_t)so * ncand + c];
		l = (uint32_t)(r.n[0] + r.n[1]);
		o = (uint32_t)r.n_cigar[0] + r.n_cigar[1];
		m = (uint32_t)r.n_miss[0] + r.n_miss[1];
	} else {
		const DPairT<K> &p = P[t / ncand];
		for (int s = 0; s < 2; ++s) {
			l += (uint32_t)p.s[c][s].n;
			o += (uint32_t)p.s[c][s].cig.n;
			m += (uint32_t)p.s[c][s].cig.nm;
		}
	}
	cl[t] = l;
	co[t] = o;
	cm[t] = m;
}

template <class K>
__global__ void k_emit(const DPairT<K> *__restrict__ P, int n_items, int ncand,
		       const uint32_t *__restrict__ xl, const uint32_t *__restrict__ xo,
		       const uint32_t *__restrict__ xm, hera_cand_rec *__restrict__ recs,
		       uint32_t *__restrict__ pos_pool, int32_t *__restrict__ p_pool,
		       uint32_t *__restrict__ op_pool, uint8_t *__restrict__ miss_pool,
		       uint64_t base_l, uint64_t base_o, uint64_t base_m, Side side)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n_items * ncand)
		return;
	const int c = t % ncand;
	uint32_t l = xl[t], o = xo[t], m = xm[t];
	const int so = side.slot ? side.slot[t / ncand] : -1;
	hera_cand_rec r;
	if (so >= 0) {
		const hera_cand_rec &w = side.recs[(size_t)so * ncand + c];
		r = w;
		for (int s = 0; s < 2; ++s) {
			r.list_off[s] = (uint32_t)(base_l + l);
			r.cig_off[s] = (uint32_t)(base_o + o);
			r.miss_off[s] = (uint32_t)(base_m + m);
			for (int i = 0; i < w.n[s]; ++i) {
				pos_pool[l + i] = side.pos[w.list_off[s] + i];
				p_pool[l + i] = side.p[w.list_off[s] + i];
			}
			for (int i = 0; i < w.n_cigar[s]; ++i)
				op_pool[o + i] = side.op[w.cig_off[s] + i];
			for (int i = 0; i < w.n_miss[s]; ++i)
				miss_pool[m + i] = side.miss[w.miss_off[s] + i];
			l += (uint32_t)w.n[s];
			o += (uint32_t)w.n_cigar[s];
			m += (uint32_t)w.n_miss[s];
		}
		recs[t] = r;
		return;
	}
	const DPairT<K> &p = P[t / ncand];
	r.pair = p.pair[c];
	for (int s = 0; s < 2; ++s) {
		const DSlotT<K> &S = p.s[c][s];
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

// the plain form's pairs start with no capacity flags (k_position's four
// tasks of a pair would race to clear them)
__global__ void k_ovf_reset(DPair *__restrict__ P, int n)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t < n)
		P[t].ovf = 0;
}

// the pairs (items) the first pass flagged: their list, and each item's
// position in it (-1 for the others)
__global__ void k_ovf_list(const DPair *__restrict__ P, int n, int *__restrict__ list, int *__restrict__ nlist,
			   int *__restrict__ slot)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n)
		return;
	int k = -1;
	if (P[t].ovf)
		k = atomicAdd(nlist, 1);
	if (k >= 0)
		list[k] = t;
	slot[t] = k;
}

#include "hera_batched.cuh"

}  // namespace

// ===========================================================================
// host side
// ===========================================================================

template <typename T>
struct DBuf {   // growable device buffer
	T *p = nullptr;
	size_t cap = 0;
	bool fixed = false;   // bound to memory the buffer does not own: never grows
	void bind(void *ptr, size_t n)
	{
		p = static_cast<T *>(ptr);
		cap = n;
		fixed = true;
	}
	cudaError_t ensure(size_t n)
	{
		if (n <= cap)
			return cudaSuccess;
		if (fixed)
			return cudaErrorMemoryAllocation;
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
		if (p && !fixed)
			cudaFree(p);
		p = nullptr;
		cap = 0;
		fixed = false;
	}
};

// an output pool of n entries: an owned pool grows with one spare entry (so
// it is never empty); a bound pool must hold n as it is
template <typename T>
static cudaError_t pool_ensure(DBuf<T> &b, size_t n)
{
	if (b.fixed)
		return n <= b.cap ? cudaSuccess : cudaErrorMemoryAllocation;
	return b.ensure(n + 1);
}

template <typename T>
struct HBuf {   // growable pinned host buffer
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

// One lane: a stream, the per-batch device buffers, pinned staging and a
// host thread of its own.  A call deals its sub-batches to the lanes so the
// copies, kernels and host synchronisations of one sub-batch overlap those
// of the others.
struct Lane {
	cudaStream_t stream = nullptr;
	cudaEvent_t ev[12]{};
	DBuf<uint8_t> seq, code, code_r;
	DBuf<int64_t> off;
	DBuf<int32_t> len;
	// a second set of staged reads, filled on the copy stream while the lane
	// runs the set before (host calls with several sub-batches a lane)
	cudaStream_t cstream = nullptr;
	cudaEvent_t cev[2][2]{};             // per set: copies issued, copies done
	DBuf<uint8_t> seq2;
	DBuf<int64_t> off2;
	DBuf<int32_t> len2;
	DBuf<uint2> hits;
	DBuf<DPair> pairs;
	DBuf<RmReq> q[2];
	DBuf<GpReq> qg[2];
	DBuf<int> counters;
	DBuf<uint32_t> cnt;
	DBuf<uint8_t> cub_tmp;
	DBuf<int2> calls;
	DBuf<int> rq_base;
	DBuf<SswOut> ssw_out;
	// the wide pass (pairs past a first-pass capacity): made on first use
	bool no_wide = false;                // the allocation-free lane has none
	DBuf<int> ovf_list, ovf_slot;
	DBuf<DPairT<CapsWide>> wpairs;
	DBuf<GpWorkT<CapsWide>> wwork;
	DBuf<SswOutT<CapsWide>> wssw_out;
	DBuf<hera_cand_rec> side_recs;
	DBuf<uint32_t> side_pos, side_op;
	DBuf<int32_t> side_p;
	DBuf<uint8_t> side_miss;
	DBuf<TaskInfo> tinfo;
	DBuf<Chain> chains;
	DBuf<JobSlot> slots;
	DBuf<DpJob> jobs;
	DBuf<uint8_t> res;
	DBuf<int> perm, hist, tlist;
	DBuf<uint2> thits;                   // a later round's seeds, looked up before its build
	bool seed_req = true;                // the allocation-free lane's build looks them up itself
	DBuf<int> tval;                      // round 0's calls before the sort by size
	DBuf<uint8_t> tkey;                  // their anchor counts (2 halves: in, out)
	bool sort_tasks = true;              // the allocation-free lane keeps the unsorted list
	size_t chain_cap = 0, job_cap = 0, slot_cap = 0;
	DBuf<hera_cand_rec> recs;
	DBuf<uint32_t> pos_pool, op_pool;
	DBuf<int32_t> p_pool;
	DBuf<uint8_t> miss_pool;
	HBuf<uint8_t> h_seq;
	HBuf<int64_t> h_off;
	HBuf<int32_t> h_len;
	HBuf<int> h_small;
	HBuf<hera_cand_rec> h_recs;
	HBuf<uint32_t> h_pos, h_ops;
	HBuf<int32_t> h_p;
	HBuf<uint8_t> h_miss;
	hera_gpu_timing timing{};
	std::string err;
	// result of the last batch this lane ran (held in its device pools)
	int32_t items = 0, ncand = 0;
	uint64_t nl = 0, no = 0, nm = 0;
	// set while the output pools are sized: a failure then means the pools
	// (not the working buffers) were too small, and nl/no/nm are the sizes
	bool pools_short = false;
	// pool offsets the device records were last rebased by (a fetch into
	// page-locked memory rebases them in place); 0 after each batch
	uint32_t rb_l = 0, rb_o = 0, rb_m = 0;

	void release()
	{
		seq2.release(); off2.release(); len2.release();
		for (auto &s2 : cev)
			for (auto &e : s2)
				if (e)
					cudaEventDestroy(e);
		if (cstream)
			cudaStreamDestroy(cstream);
		seq.release(); code.release(); code_r.release(); off.release(); len.release();
		hits.release(); pairs.release(); q[0].release(); q[1].release(); qg[0].release();
		qg[1].release(); counters.release(); cnt.release(); cub_tmp.release();
		calls.release(); rq_base.release(); ssw_out.release(); tinfo.release(); chains.release();
		ovf_list.release(); ovf_slot.release(); wpairs.release(); wwork.release(); wssw_out.release();
		side_recs.release(); side_pos.release(); side_op.release(); side_p.release(); side_miss.release();
		slots.release(); jobs.release(); res.release(); perm.release(); hist.release(); tlist.release();
		tval.release(); tkey.release(); thits.release();
		recs.release(); pos_pool.release(); op_pool.release(); p_pool.release(); miss_pool.release();
		h_seq.release(); h_off.release(); h_len.release(); h_small.release(); h_recs.release();
		h_pos.release(); h_ops.release(); h_p.release(); h_miss.release();
		for (auto &e : ev)
			if (e)
				cudaEventDestroy(e);
		if (stream)
			cudaStreamDestroy(stream);
	}
};

struct hera_gpu_ctx {
	int device = 0;
	cudaStream_t stream = nullptr;    // the context's default stream
	DevIndex ix{};
	uint32_t *d_boff = nullptr;
	uint4 *d_bk = nullptr;
	uint2 *d_occ = nullptr;
	uint8_t *d_seq = nullptr, *d_tcode = nullptr;
	uint32_t *d_tlen = nullptr, *d_tstart = nullptr;
	uint32_t max_batch = 1u << 18;    // pairs per sub-batch
	uint64_t scratch_bytes = 0;       // accepted for compatibility; unused
	int batched = 1;
	std::vector<Lane *> lanes;
	Lane *na = nullptr;               // lane of hera_gpu_align_pairs_device_noalloc
	hera_gpu_timing timing{};
	std::string err = "no error";
	// device-resident results of the last hera_gpu_align_pairs_device call:
	// sub-batch k is held by lane k
	int nparts = 0;
	// launch shapes (autotuned on the first large batch, or set by the caller)
	int sms = 148;
	std::mutex tune_mu;
	hera_gpu_tuning tune{};
	int build_tuning = 0, rescue_tuning = 0;   // 0 open, 1 claimed by a lane, 2 done
	// lanes run their rounds under a shared lock; the autotuner's trials
	// take it exclusively, so no other lane's kernels share the GPU with them
	std::shared_mutex gate;
	struct FqState *fq = nullptr;     // FASTQ chunk parsing (made on first use)
	// asynchronous flat calls: two in flight at most, each on a lane group
	// of its own (the second group is made on first use)
	struct AsyncCall {
		std::thread th;
		bool busy = false;
		uint64_t ticket = 0;
		int rc = 0;
		std::string err;
		hera_gpu_timing tm{};
		hera_gpu_reads r1{}, r2{};
	};
	std::mutex async_mu;
	AsyncCall async[2];
	std::vector<Lane *> lanes2;
	uint64_t next_async = 1;
	// drop-in calls made at the same time by several host threads run as
	// one device batch (up to 2^20 pairs)
	hcomb::Combiner dropin{1 << 20};
};

struct FqState;
static void fq_release(hera_gpu_ctx *ctx);

// candidate launch shapes the autotuner times
static const int BUILD_BPS[] = {2, 4, 6, 8, 12, 16};
static const int RESCUE_WPB[] = {2, 4, 8};

static int tuned_build_bps(hera_gpu_ctx *ctx)
{
	std::lock_guard<std::mutex> g(ctx->tune_mu);
	return ctx->tune.build_blocks_per_sm;
}

static int tuned_rescue_wpb(hera_gpu_ctx *ctx)
{
	std::lock_guard<std::mutex> g(ctx->tune_mu);
	return ctx->tune.rescue_warps_per_block;
}

// true for the one lane that gets to tune `what` (its flag goes to 1)
static bool claim_tuning(hera_gpu_ctx *ctx, int &flag)
{
	std::lock_guard<std::mutex> g(ctx->tune_mu);
	if (ctx->tune.state == 2 || flag != 0)
		return false;
	flag = 1;
	return true;
}

static int set_err(std::string &dst, int code, const char *what, cudaError_t e = cudaSuccess)
{
	char buf[512];
	if (e != cudaSuccess)
		snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
	else
		snprintf(buf, sizeof buf, "%s", what);
	dst = buf;
	return code;
}

static int fail(hera_gpu_ctx *c, int code, const char *what, cudaError_t e = cudaSuccess)
{
	if (c)
		set_err(c->err, code, what, e);
	return code;
}

// CUDA call inside a lane: record the failure on the lane
#define LK(call, what)                                                                             \
	do {                                                                                       \
		cudaError_t e_ = (call);                                                           \
		if (e_ != cudaSuccess)                                                             \
			return set_err(L.err, e_ == cudaErrorMemoryAllocation ? HERA_GPU_ENOMEM : HERA_GPU_ECUDA, \
				       what, e_);                                                  \
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

extern "C" int hera_gpu_host_register(void *p, size_t bytes)
{
	if (!p || bytes == 0)
		return HERA_GPU_EINVAL;
	return cudaHostRegister(p, bytes, cudaHostRegisterPortable) == cudaSuccess ? HERA_GPU_OK : HERA_GPU_ECUDA;
}

extern "C" int hera_gpu_host_unregister(void *p)
{
	if (!p)
		return HERA_GPU_EINVAL;
	return cudaHostUnregister(p) == cudaSuccess ? HERA_GPU_OK : HERA_GPU_ECUDA;
}

extern "C" int hera_gpu_get_tuning(const hera_gpu_ctx *ctx, hera_gpu_tuning *out)
{
	if (!ctx || !out)
		return HERA_GPU_EINVAL;
	std::lock_guard<std::mutex> g(const_cast<hera_gpu_ctx *>(ctx)->tune_mu);
	*out = ctx->tune;
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_set_tuning(hera_gpu_ctx *ctx, const hera_gpu_tuning *in)
{
	if (!ctx || !in)
		return HERA_GPU_EINVAL;
	const int w = in->rescue_warps_per_block;
	if (in->build_blocks_per_sm < 1 || in->build_blocks_per_sm > 16 || !(w == 1 || w == 2 || w == 4 || w == 8))
		return fail(ctx, HERA_GPU_EINVAL, "tuning values out of range");
	std::lock_guard<std::mutex> g(ctx->tune_mu);
	ctx->tune.build_blocks_per_sm = in->build_blocks_per_sm;
	ctx->tune.rescue_warps_per_block = w;
	ctx->tune.state = 2;
	return HERA_GPU_OK;
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
	for (auto &a : ctx->async)   // asynchronous calls not completed
		if (a.th.joinable())
			a.th.join();
	cudaDeviceSynchronize();
	cudaFree(ctx->d_boff);
	cudaFree(ctx->d_bk);
	cudaFree(ctx->d_occ);
	cudaFree(ctx->d_seq);
	cudaFree(ctx->d_tcode);
	cudaFree(ctx->d_tlen);
	cudaFree(ctx->d_tstart);
	for (Lane *L : ctx->lanes) {
		L->release();
		delete L;
	}
	for (Lane *L : ctx->lanes2) {
		L->release();
		delete L;
	}
	if (ctx->na) {
		ctx->na->release();
		delete ctx->na;
	}
	fq_release(ctx);
	if (ctx->stream)
		cudaStreamDestroy(ctx->stream);
	delete ctx;
}

// n lanes, each with its streams and events
static int make_lanes(std::vector<Lane *> &lanes, int n)
{
	for (int i = 0; i < n; ++i) {
		Lane *L = new Lane();
		lanes.push_back(L);
		if (cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking) != cudaSuccess ||
		    cudaStreamCreateWithFlags(&L->cstream, cudaStreamNonBlocking) != cudaSuccess)
			return HERA_GPU_ECUDA;
		for (auto &e : L->ev)
			cudaEventCreate(&e);
		for (auto &s2 : L->cev)
			for (auto &e : s2)
				cudaEventCreate(&e);
	}
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_ctx_create(const hera_gpu_index_view *v, const hera_gpu_options *opt,
				   hera_gpu_ctx **out)
{
	if (!out || !v || !v->len || !v->find || !v->seq || !v->bucket_n || !v->pos || !v->p ||
	    v->n_trans == 0)
		return HERA_GPU_EINVAL;
	*out = nullptr;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
		return HERA_GPU_ENODEV;
	hera_gpu_ctx *ctx = new hera_gpu_ctx();
	int nlanes = 6;
	if (opt) {
		ctx->device = opt->device;
		if (opt->max_batch)
			ctx->max_batch = opt->max_batch;
		if (opt->scratch_bytes)
			ctx->scratch_bytes = opt->scratch_bytes;
		ctx->batched = opt->path == HERA_GPU_PATH_PLAIN ? 0 : 1;
		if (opt->lanes > 0)
			nlanes = opt->lanes;
	}
	if (nlanes > 8)
		nlanes = 8;
	auto bail = [&](int rc) {
		hera_gpu_ctx_destroy(ctx);
		return rc;
	};
	if (cudaSetDevice(ctx->device) != cudaSuccess)
		return bail(HERA_GPU_ENODEV);
	if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
		return bail(HERA_GPU_ECUDA);
	// the rescue kernel's per-warp shared-memory areas (up to ~177 KiB a block)
	if (cudaFuncSetAttribute(k_rescue_sw<CapsStd>, cudaFuncAttributeMaxDynamicSharedMemorySize,
				 (int)((RESCUE_TPB / 32) * ssw_smem_per_warp(MAX_READ))) != cudaSuccess ||
	    cudaFuncSetAttribute(k_rescue_sw<CapsWide>, cudaFuncAttributeMaxDynamicSharedMemorySize,
				 (int)(WIDE_RESCUE_WPB * ssw_smem_wide())) != cudaSuccess)
		return bail(fail(ctx, HERA_GPU_ECUDA, "rescue kernel shared-memory size"));
	if (cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, ctx->device) != cudaSuccess ||
	    ctx->sms <= 0)
		return bail(fail(ctx, HERA_GPU_ECUDA, "SM count"));
	ctx->tune.build_blocks_per_sm = 8;
	ctx->tune.rescue_warps_per_block = 4;
	if (make_lanes(ctx->lanes, nlanes) != HERA_GPU_OK)
		return bail(HERA_GPU_ECUDA);
	// the allocation-free entry's lane: its stream, events and 32 pinned
	// counters are made here, so that entry point itself allocates nothing
	ctx->na = new Lane();
	ctx->na->no_wide = true;
	ctx->na->sort_tasks = false;
	ctx->na->seed_req = false;
	if (cudaStreamCreateWithFlags(&ctx->na->stream, cudaStreamNonBlocking) != cudaSuccess ||
	    ctx->na->h_small.ensure(32) != cudaSuccess)
		return bail(HERA_GPU_ECUDA);
	for (auto &e : ctx->na->ev)
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
	for (uint32_t i = 0; i < n; ++i) {
		tstart[i] = v->find[i] - v->len[i];
		// the batched form packs transcript positions into 23 bits
		if (ctx->batched && v->len[i] >= (1u << TP_BITS))
			return bail(fail(ctx, HERA_GPU_EINVAL,
					 "a transcript of 2^23 bases or more: use HERA_GPU_PATH_PLAIN"));
	}
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
	// transcript codes; the zero padding after the last transcript codes as 4
	k_codes<<<1184, 256, 0, ctx->stream>>>(ctx->d_seq, ctx->d_tcode, (int64_t)(seq_len + pad));
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
// the lane's rescue outputs for the first pass / the wide pass
template <class K>
static DBuf<SswOutT<K>> &ssw_outputs(Lane &L)
{
	if constexpr (std::is_same<K, CapsStd>::value)
		return L.ssw_out;
	else
		return L.wssw_out;
}

template <class K>
static int rescue_round(hera_gpu_ctx *ctx, Lane &L, const BatchT<K> &b, const RmReq *q, int nq,
			int max_len, uint32_t &launches, float &ms_acc)
{
	constexpr bool wide = !std::is_same<K, CapsStd>::value;
	cudaStream_t st = L.stream;
	std::shared_lock<std::shared_mutex> shared(ctx->gate);
	LK(L.calls.ensure((size_t)nq * K::L), "rescue calls");
	LK(L.rq_base.ensure(nq), "rescue bases");
	int *d_nc = L.counters.p + 4;
	LK(cudaMemsetAsync(d_nc, 0, sizeof(int), st), "memset");
	cudaEvent_t e0 = L.ev[6], e1 = L.ev[7];
	cudaEventRecord(e0, st);
	k_rescue_expand<<<blocks_for(nq, 256), 256, 0, st>>>(b, q, nq, L.calls.p, L.rq_base.p, d_nc);
	++launches;
	LK(cudaMemcpyAsync(L.h_small.p + 1, d_nc, sizeof(int), cudaMemcpyDeviceToHost, st), "calls");
	LK(cudaStreamSynchronize(st), "rescue expand");
	const int ncalls = L.h_small.p[1];
	DBuf<SswOutT<K>> &outs = ssw_outputs<K>(L);
	LK(outs.ensure(ncalls + 1), "rescue outputs");
	const int per = wide ? (int)ssw_smem_wide() : (int)ssw_smem_per_warp(max_len);
	auto launch = [&](int wpb) {
		k_rescue_sw<<<blocks_for((int64_t)ncalls * 32, 32 * wpb), 32 * wpb, wpb * per, st>>>(
			b, q, L.calls.p, 0, ncalls, outs.p, per);
		++launches;
	};
	// autotune: the first large rescue round times each candidate (every
	// run writes the same outputs)
	std::unique_lock<std::shared_mutex> excl(ctx->gate, std::defer_lock);
	if (!wide && ncalls >= 2048 && claim_tuning(ctx, ctx->rescue_tuning)) {
		shared.unlock();   // nothing of this lane is in flight (synchronised above)
		excl.lock();
		int best = 0;
		float best_ms = 0;
		int nc = 0;
		launch(tuned_rescue_wpb(ctx));   // untimed: first-launch costs
		LK(cudaStreamSynchronize(st), "rescue tuning");
		for (int wpb : RESCUE_WPB) {
			cudaEventRecord(L.ev[10], st);
			launch(wpb);
			cudaEventRecord(L.ev[11], st);
			LK(cudaEventSynchronize(L.ev[11]), "rescue tuning");
			float ms = 0;
			cudaEventElapsedTime(&ms, L.ev[10], L.ev[11]);
			if (!best || ms < best_ms) {
				best = wpb;
				best_ms = ms;
			}
			std::lock_guard<std::mutex> g(ctx->tune_mu);
			ctx->tune.rescue_cand[nc] = wpb;
			ctx->tune.rescue_ms[nc] = ms;
			ctx->tune.n_rescue = ++nc;
		}
		std::lock_guard<std::mutex> g(ctx->tune_mu);
		if (ctx->tune.state != 2) {
			ctx->tune.rescue_warps_per_block = best;
			ctx->tune.state = 1;
		}
		ctx->rescue_tuning = 2;
	}
	cudaEventRecord(L.ev[10], st);
	if (ncalls > 0)
		launch(wide ? WIDE_RESCUE_WPB : tuned_rescue_wpb(ctx));
	cudaEventRecord(L.ev[11], st);
	k_rescue_fin<<<blocks_for(nq, 256), 256, 0, st>>>(b, q, nq, L.rq_base.p, outs.p);
	++launches;
	cudaEventRecord(e1, st);
	LK(cudaStreamSynchronize(st), "rescue");
	float ms = 0;
	cudaEventElapsedTime(&ms, e0, e1);
	ms_acc += ms;
	cudaEventElapsedTime(&ms, L.ev[10], L.ev[11]);
	L.timing.rescue_kernel_ms += ms;
	return HERA_GPU_OK;
}

// one round of batched get_position calls: build, bin, DP, replay
static int gp_round(hera_gpu_ctx *ctx, Lane &L, const Batch &b, Round R, uint32_t &launches, float &build_ms, float &dp_ms)
{
	if (R.ntask <= 0)
		return HERA_GPU_OK;
	const bool tune = !R.req && R.ntask >= 4 * 16384 && claim_tuning(ctx, ctx->build_tuning);
	std::shared_lock<std::shared_mutex> shared(ctx->gate, std::defer_lock);
	std::unique_lock<std::shared_mutex> excl(ctx->gate, std::defer_lock);
	if (tune)
		excl.lock();
	else
		shared.lock();
	cudaStream_t st = L.stream;
	const int rcap = b.score_only ? 2 : JCAP;
	LK(L.tinfo.ensure(R.ntask), "task info");
	if (L.chain_cap < 2 * (size_t)R.ntask)
		L.chain_cap = 2 * (size_t)R.ntask;
	if (L.job_cap < 3 * (size_t)R.ntask)
		L.job_cap = 3 * (size_t)R.ntask;
	if (L.slot_cap < 4 * (size_t)R.ntask)
		L.slot_cap = 4 * (size_t)R.ntask;
	int *d_cnt = L.counters.p + 12;
	cudaEvent_t e0 = L.ev[6], e1 = L.ev[7];
	int nch = 0, nj = 0, ns = 0;
	cudaEventRecord(e0, st);
	if (!R.req) {   // round 0: reset the pairs, list the calls with seed hits
		LK(L.tlist.ensure(R.ntask), "task list");
		int *d_nl = L.counters.p + 15;
		LK(cudaMemsetAsync(d_nl, 0, sizeof(int), st), "memset");
		if (L.sort_tasks) {
			// calls largest first (anchor count, descending): a warp of the
			// build then takes calls of like size
			LK(L.tval.ensure(R.ntask), "task list");
			LK(L.tkey.ensure(2 * (size_t)R.ntask), "task keys");
			k_task_list<<<blocks_for(R.ntask, 256), 256, 0, st>>>(b, R.ntask, R.hits, R.spr, L.tinfo.p,
									       L.tval.p, d_nl, L.tkey.p);
			size_t tmp = 0;
			cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, L.tkey.p, L.tkey.p + R.ntask, L.tval.p,
								  L.tlist.p, R.ntask, 0, 8, st);
			LK(L.cub_tmp.ensure(tmp), "sort scratch");
			cub::DeviceRadixSort::SortPairsDescending(L.cub_tmp.p, tmp, L.tkey.p, L.tkey.p + R.ntask, L.tval.p,
								  L.tlist.p, R.ntask, 0, 8, st);
			launches += 2;
		} else {
			k_task_list<<<blocks_for(R.ntask, 256), 256, 0, st>>>(b, R.ntask, R.hits, R.spr, L.tinfo.p,
									       L.tlist.p, d_nl, nullptr);
			++launches;
		}
		R.list = L.tlist.p;
		R.nlist = d_nl;
	} else if (L.seed_req) {
		// a later round: its seeds looked up side by side first (its calls
		// stay in request order: sorted by anchor count, as round 0's are,
		// the build of these rounds measured 70% slower)
		R.tspr = b.max_len >= KMER ? (b.max_len - KMER) / R.space + 1 : 1;
		LK(L.thits.ensure((size_t)R.ntask * R.tspr), "round seeds");
		k_seed_req<<<blocks_for((int64_t)R.ntask * R.tspr, 256), 256, 0, st>>>(b, R, L.thits.p);
		++launches;
		R.thits = L.thits.p;
	}
	for (int attempt = 0; attempt < 2; ++attempt) {
		LK(L.chains.ensure(L.chain_cap), "chains");
		LK(L.jobs.ensure(L.job_cap), "dp jobs");
		LK(L.slots.ensure(L.slot_cap), "job slots");
		R.tinfo = L.tinfo.p;
		R.chains = L.chains.p;
		R.slots = L.slots.p;
		R.jobs = L.jobs.p;
		R.cnt = d_cnt;
		R.chain_cap = (int)L.chain_cap;
		R.job_cap = (int)L.job_cap;
		R.slot_cap = (int)L.slot_cap;
		int *d_queue = L.counters.p + 26;
		auto launch = [&](int bps) {
			cudaMemsetAsync(d_cnt, 0, 3 * sizeof(int), st);
			cudaMemsetAsync(d_queue, 0, sizeof(int), st);
			unsigned grid = (unsigned)(ctx->sms * bps);
			const unsigned need = blocks_for(R.ntask);
			k_build<<<grid < need ? grid : need, 128, 0, st>>>(b, R, d_queue);
			++launches;
		};
		// autotune the persistent build kernel's residency on the first
		// large round 0 (every run writes the same chains and jobs)
		if (tune && ctx->build_tuning == 1) {
			int best = 0, nc = 0;
			float best_ms = 0;
			launch(tuned_build_bps(ctx));   // untimed: first-launch costs
			LK(cudaStreamSynchronize(st), "build tuning");
			for (int bps : BUILD_BPS) {
				cudaEventRecord(L.ev[8], st);
				launch(bps);
				cudaEventRecord(L.ev[9], st);
				LK(cudaEventSynchronize(L.ev[9]), "build tuning");
				float ms = 0;
				cudaEventElapsedTime(&ms, L.ev[8], L.ev[9]);
				if (!best || ms < best_ms) {
					best = bps;
					best_ms = ms;
				}
				std::lock_guard<std::mutex> g(ctx->tune_mu);
				ctx->tune.build_cand[nc] = bps;
				ctx->tune.build_ms[nc] = ms;
				ctx->tune.n_build = ++nc;
			}
			std::lock_guard<std::mutex> g(ctx->tune_mu);
			if (ctx->tune.state != 2) {
				ctx->tune.build_blocks_per_sm = best;
				ctx->tune.state = 1;
			}
			ctx->build_tuning = 2;
		}
		launch(tuned_build_bps(ctx));
		LK(cudaGetLastError(), "build launch");
		LK(cudaMemcpyAsync(L.h_small.p + 12, d_cnt, 3 * sizeof(int), cudaMemcpyDeviceToHost, st), "counts");
		LK(cudaStreamSynchronize(st), "build");
		nch = L.h_small.p[12];
		nj = L.h_small.p[13];
		ns = L.h_small.p[14];
		if ((size_t)nch <= L.chain_cap && (size_t)nj <= L.job_cap && (size_t)ns <= L.slot_cap)
			break;
		L.chain_cap = (size_t)nch + 16;
		L.job_cap = (size_t)nj + 16;
		L.slot_cap = (size_t)ns + 16;
		if (attempt == 1)
			return set_err(L.err, HERA_GPU_ECAPACITY, "dp job buffers");
	}
	L.timing.dp_calls += (uint64_t)ns;
	cudaEventRecord(e1, st);
	float ms = 0;
	LK(cudaEventSynchronize(e1), "build");
	cudaEventElapsedTime(&ms, e0, e1);
	build_ms += ms;
	cudaEventRecord(e0, st);
	R.res = nullptr;
	R.rcap = rcap;
	if (nj > 0) {
		LK(L.res.ensure((size_t)nj * res_stride(rcap)), "dp results");
		LK(L.perm.ensure(nj), "dp order");
		LK(L.hist.ensure(NBIN), "dp bins");
		LK(cudaMemsetAsync(L.hist.p, 0, NBIN * sizeof(int), st), "memset");
		k_bin_count<<<148, 512, 0, st>>>(L.jobs.p, nj, L.hist.p);
		k_bin_scan<<<1, 256, 0, st>>>(L.hist.p, NBIN);
		k_bin_scatter<<<blocks_for(nj, 1024), 1024, 0, st>>>(L.jobs.p, nj, L.hist.p, L.perm.p);
		cudaEventRecord(L.ev[10], st);
		if (b.score_only) {
			k_dp_reg<4, true><<<blocks_for(nj), 128, 0, st>>>(b, L.jobs.p, L.perm.p, nj, L.res.p, rcap);
			k_dp_reg<8, true><<<blocks_for(nj), 128, 0, st>>>(b, L.jobs.p, L.perm.p, nj, L.res.p, rcap);
		} else {
			k_dp_reg<4, false><<<blocks_for(nj), 128, 0, st>>>(b, L.jobs.p, L.perm.p, nj, L.res.p, rcap);
			k_dp_reg<8, false><<<blocks_for(nj), 128, 0, st>>>(b, L.jobs.p, L.perm.p, nj, L.res.p, rcap);
		}
		k_dp_generic<<<blocks_for(nj), 128, 0, st>>>(b, L.jobs.p, nj, L.res.p, rcap);
		cudaEventRecord(L.ev[11], st);
		launches += 6;
		R.res = L.res.p;
	}
	k_replay<<<blocks_for(R.ntask), 128, 0, st>>>(b, R);
	++launches;
	cudaEventRecord(e1, st);
	LK(cudaEventSynchronize(e1), "replay");
	cudaEventElapsedTime(&ms, e0, e1);
	dp_ms += ms;
	if (nj > 0) {
		cudaEventElapsedTime(&ms, L.ev[10], L.ev[11]);
		L.timing.dp_kernel_ms += ms;
	}
	L.timing.dp_jobs += (uint64_t)nj;
	return HERA_GPU_OK;
}

// The plain form's pair control flow after the space-31 calls: rounds of
// k_resolve and mate rescues until no pair waits (n pairs in b.P).
template <class K>
static int plain_rounds(hera_gpu_ctx *ctx, Lane &L, const BatchT<K> &b, int n, int max_len, uint32_t &launches,
			float &resolve_ms, float &rescue_ms, uint32_t &rounds)
{
	cudaStream_t st = L.stream;
	const RmReq *resume = nullptr;
	int nact = n, qi = 0;
	while (nact > 0) {
		int *qn = L.counters.p + 1 + qi;
		LK(cudaMemsetAsync(qn, 0, sizeof(int), st), "memset");
		cudaEvent_t e0 = L.ev[6], e1 = L.ev[7];
		cudaEventRecord(e0, st);
		k_resolve<<<blocks_for(nact), TPB, 0, st>>>(b, resume, nact, L.q[qi].p, qn);
		++launches;
		cudaEventRecord(e1, st);
		LK(cudaMemcpyAsync(L.h_small.p, qn, sizeof(int), cudaMemcpyDeviceToHost, st), "queue size");
		LK(cudaStreamSynchronize(st), "resolve");
		float ms = 0;
		cudaEventElapsedTime(&ms, e0, e1);
		resolve_ms += ms;
		const int nq = L.h_small.p[0];
		if (nq == 0)
			break;
		++rounds;
		int rc = rescue_round(ctx, L, b, L.q[qi].p, nq, max_len, launches, rescue_ms);
		if (rc)
			return rc;
		resume = L.q[qi].p;
		nact = nq;
		qi ^= 1;
	}
	return HERA_GPU_OK;
}

// a device buffer grown to n entries with its first `keep` entries kept
template <typename T>
static cudaError_t grow_keep(DBuf<T> &d, size_t n, size_t keep, cudaStream_t st)
{
	if (n <= d.cap)
		return cudaSuccess;
	DBuf<T> nd;
	cudaError_t e = nd.ensure(n + n / 2);
	if (e == cudaSuccess && keep && d.p)
		e = cudaMemcpyAsync(nd.p, d.p, keep * sizeof(T), cudaMemcpyDeviceToDevice, st);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(st);
	if (e != cudaSuccess) {
		nd.release();
		return e;
	}
	d.release();
	d = nd;
	return cudaSuccess;
}

// The second, wide pass.  Every pair (or single read) whose first pass met
// a per-read capacity (its DPair.ovf) is aligned again from the start with
// CapsWide -- the same code, larger lists, working sets in device memory --
// WIDE_WAVE at a time, and its records are packed into the lane's side
// pools.  A pair's result depends on that pair alone, so this is exactly
// the result an unbounded first pass would have given.  `side` then
// routes the final pack to those records.
constexpr int WIDE_WAVE = 128;

static int wide_pass(hera_gpu_ctx *ctx, Lane &L, const Batch &b, int32_t n, bool paired, int spr, int max_len,
		     uint32_t &launches, float &resolve_ms, float &rescue_ms, uint32_t &rounds, Side &side, int &wflags)
{
	cudaStream_t st = L.stream;
	const int ncand = paired ? 2 : 1;
	LK(L.ovf_list.ensure(n), "wide pass list");
	LK(L.ovf_slot.ensure(n), "wide pass list");
	int *d_nw = L.counters.p + 28, *d_wf = L.counters.p + 29;
	LK(cudaMemsetAsync(d_nw, 0, 2 * sizeof(int), st), "memset");
	k_ovf_list<<<blocks_for(n, 256), 256, 0, st>>>(b.P, n, L.ovf_list.p, d_nw, L.ovf_slot.p);
	++launches;
	LK(cudaMemcpyAsync(L.h_small.p + 28, d_nw, sizeof(int), cudaMemcpyDeviceToHost, st), "wide pass count");
	LK(cudaStreamSynchronize(st), "wide pass list");
	const int nw = L.h_small.p[28];
	if (nw <= 0)
		return set_err(L.err, HERA_GPU_ECAPACITY, "a per-read capacity flag that no pair holds");
	const int wave = nw < WIDE_WAVE ? nw : WIDE_WAVE;
	LK(L.wpairs.ensure(wave), "wide pass state");
	LK(L.wwork.ensure((size_t)(paired ? 4 : 1) * wave), "wide pass working sets");
	LK(L.side_recs.ensure((size_t)nw * ncand), "wide pass records");
	BatchT<CapsWide> bw{};
	bw.ix = b.ix;
	bw.code = b.code;
	bw.code_r = b.code_r;
	bw.off = b.off;
	bw.len = b.len;
	bw.P = L.wpairs.p;
	bw.flags = d_wf;
	bw.stats = b.stats;
	bw.score_only = b.score_only;
	bw.max_len = b.max_len;
	bw.work = L.wwork.p;
	uint64_t fl = 0, fo = 0, fm = 0;   // side pools filled so far
	for (int w0 = 0; w0 < nw; w0 += wave) {
		const int nv = nw - w0 < wave ? nw - w0 : wave;
		bw.pmap = L.ovf_list.p + w0;
		if (paired) {
			k_position<<<blocks_for((int64_t)nv * 4), TPB, 0, st>>>(bw, nv, spr, L.hits.p);
			++launches;
			const int rc = plain_rounds(ctx, L, bw, nv, max_len, launches, resolve_ms, rescue_ms, rounds);
			if (rc)
				return rc;
		} else {
			k_single<<<blocks_for(nv), TPB, 0, st>>>(bw, nv);
			++launches;
		}
		// pack the wave's records into the side pools
		const int items = nv * ncand;
		uint32_t *cl = L.cnt.p, *co = cl + (items + 1), *cm = co + (items + 1);
		uint32_t *xl = cm + (items + 1), *xo = xl + (items + 1), *xm = xo + (items + 1);
		LK(cudaMemsetAsync(cl, 0, 3 * sizeof(uint32_t) * (items + 1), st), "memset");
		k_count<<<blocks_for(items, 256), 256, 0, st>>>(bw.P, nv, ncand, cl, co, cm, Side{});
		size_t tmp_bytes = 0;
		cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cl, xl, items + 1, st);
		LK(L.cub_tmp.ensure(tmp_bytes), "scan scratch");
		cub::DeviceScan::ExclusiveSum(L.cub_tmp.p, tmp_bytes, cl, xl, items + 1, st);
		cub::DeviceScan::ExclusiveSum(L.cub_tmp.p, tmp_bytes, co, xo, items + 1, st);
		cub::DeviceScan::ExclusiveSum(L.cub_tmp.p, tmp_bytes, cm, xm, items + 1, st);
		LK(cudaMemcpyAsync(L.h_small.p + 2, xl + items, 4, cudaMemcpyDeviceToHost, st), "totals");
		LK(cudaMemcpyAsync(L.h_small.p + 3, xo + items, 4, cudaMemcpyDeviceToHost, st), "totals");
		LK(cudaMemcpyAsync(L.h_small.p + 4, xm + items, 4, cudaMemcpyDeviceToHost, st), "totals");
		LK(cudaStreamSynchronize(st), "wide pass scan");
		const uint64_t tl = (uint32_t)L.h_small.p[2], to = (uint32_t)L.h_small.p[3], tm = (uint32_t)L.h_small.p[4];
		LK(grow_keep(L.side_pos, fl + tl + 1, fl, st), "wide pass pools");
		LK(grow_keep(L.side_p, fl + tl + 1, fl, st), "wide pass pools");
		LK(grow_keep(L.side_op, fo + to + 1, fo, st), "wide pass pools");
		LK(grow_keep(L.side_miss, fm + tm + 1, fm, st), "wide pass pools");
		k_emit<<<blocks_for(items, 256), 256, 0, st>>>(bw.P, nv, ncand, xl, xo, xm, L.side_recs.p + (size_t)w0 * ncand,
								L.side_pos.p + fl, L.side_p.p + fl, L.side_op.p + fo,
								L.side_miss.p + fm, fl, fo, fm, Side{});
		launches += 5;
		fl += tl;
		fo += to;
		fm += tm;
		if (fl >= (1ull << 32) || fo >= (1ull << 32) || fm >= (1ull << 32))
			return set_err(L.err, HERA_GPU_ECAPACITY, "wide pass pools beyond 2^32 entries");
	}
	LK(cudaMemcpyAsync(L.h_small.p + 29, d_wf, sizeof(int), cudaMemcpyDeviceToHost, st), "wide pass flags");
	LK(cudaStreamSynchronize(st), "wide pass");
	wflags = L.h_small.p[29];
	side.slot = L.ovf_slot.p;
	side.recs = L.side_recs.p;
	side.pos = L.side_pos.p;
	side.p = L.side_p.p;
	side.op = L.side_op.p;
	side.miss = L.side_miss.p;
	return HERA_GPU_OK;
}

// Run the device pipeline for one sub-batch on lane L.  Reads: d_seq holds
// seq_bytes bytes, d_off/d_len are lane-local (offsets into d_seq), 2n
// reads for pairs (mates interleaved), n for singles.  Leaves the packed
// records in L's device pools and their sizes in L.items/nl/no/nm.
static int run_batch(hera_gpu_ctx *ctx, Lane &L, const uint8_t *d_seq, const int64_t *d_off,
		     const int32_t *d_len, int32_t n, bool paired, int write_bam, int max_len,
		     int64_t seq_bytes)
{
	cudaStream_t st = L.stream;
	const int n_reads = paired ? 2 * n : n;
	const int ncand = paired ? 2 : 1;
	const int items = n * ncand;
	const bool batched = ctx->batched && paired;
	hera_gpu_timing &T = L.timing;
	uint32_t launches = 0;

	LK(L.code.ensure(seq_bytes + 64), "read code buffer");
	if (batched)
		LK(L.code_r.ensure(seq_bytes + 64), "read code buffer");
	LK(L.pairs.ensure(n), "pair state");
	LK(L.counters.ensure(32), "counters");
	LK(L.q[0].ensure(n), "rescue queue");
	LK(L.q[1].ensure(n), "rescue queue");
	LK(L.cnt.ensure(6 * (size_t)(items + 1)), "count buffer");
	LK(L.recs.ensure(items), "records");
	LK(L.h_small.ensure(32), "host counters");
	int *d_flags = L.counters.p;
	unsigned long long *d_stats = reinterpret_cast<unsigned long long *>(L.counters.p + 16);
	LK(cudaMemsetAsync(L.counters.p, 0, 32 * sizeof(int), st), "memset");

	Batch b{};   // value-initialised: no pair map, no per-task work areas
	b.ix = ctx->ix;
	b.code = L.code.p;
	b.code_r = batched ? L.code_r.p : nullptr;
	b.off = d_off;
	b.len = d_len;
	b.P = L.pairs.p;
	b.flags = d_flags;
	b.stats = d_stats;
	b.score_only = write_bam == 1;
	b.max_len = max_len;

	cudaEventRecord(L.ev[1], st);
	if (seq_bytes > 0) {
		k_codes<<<592, 256, 0, st>>>(d_seq, L.code.p, seq_bytes);
		++launches;
		if (batched) {
			k_rc<<<blocks_for((int64_t)n_reads * 32, 256), 256, 0, st>>>(L.code.p, d_off, d_len, n_reads,
										      max_len, L.code_r.p);
			++launches;
		}
	}
	const int spr = max_len >= KMER ? (max_len - KMER) / KMER + 1 : 1;
	if (paired) {
		LK(L.hits.ensure((size_t)n_reads * 2 * spr), "seed hits");
		const int64_t ns = (int64_t)n_reads * 2 * spr;
		cudaEventRecord(L.ev[8], st);
		const unsigned g = blocks_for((int64_t)n_reads * 2, 256);
		switch (spr) {
#define SEED_CASE(S)                                                                                              \
	case S:                                                                                                   \
		k_seed<S><<<g, 256, 0, st>>>(ctx->ix, L.code.p, d_off, d_len, n_reads, L.hits.p, d_stats);       \
		break;
		SEED_CASE(1) SEED_CASE(2) SEED_CASE(3) SEED_CASE(4) SEED_CASE(5)
		SEED_CASE(6) SEED_CASE(7) SEED_CASE(8) SEED_CASE(9) SEED_CASE(10)
#undef SEED_CASE
		default:
			return set_err(L.err, HERA_GPU_EINVAL, "seeds per read beyond HERA_GPU_MAX_READ");
		}
		cudaEventRecord(L.ev[9], st);
		++launches;
		T.lookups += (uint64_t)ns;
	}
	cudaEventRecord(L.ev[2], st);
	float resolve_ms = 0, rescue_ms = 0, build_ms = 0, dp_ms = 0;
	uint32_t rounds = 0;
	if (!paired) {
		k_single<<<blocks_for(n), TPB, 0, st>>>(b, n);
		++launches;
		cudaEventRecord(L.ev[3], st);
	} else if (!batched) {
		// plain form: one thread per get_position call / pair
		k_ovf_reset<<<blocks_for(n, 256), 256, 0, st>>>(L.pairs.p, n);
		k_position<<<blocks_for((int64_t)n * 4), TPB, 0, st>>>(b, n, spr, L.hits.p);
		launches += 2;
		cudaEventRecord(L.ev[3], st);
		const int rc = plain_rounds(ctx, L, b, n, max_len, launches, resolve_ms, rescue_ms, rounds);
		if (rc)
			return rc;
	} else {
		// batched form: rounds of batched get_position calls and rescues
		LK(L.qg[0].ensure(n), "gp queue");
		LK(L.qg[1].ensure(n), "gp queue");
		Round R{};
		R.req = nullptr;
		R.ntask = 4 * n;
		R.space = KMER;
		R.hits = L.hits.p;
		R.spr = spr;
		int rc = gp_round(ctx, L, b, R, launches, build_ms, dp_ms);
		if (rc)
			return rc;
		cudaEventRecord(L.ev[3], st);
		int ng = n, nr = 0, qi = 0;
		bool all = true;
		for (;;) {
			int *qng = L.counters.p + 8 + 2 * qi, *qnr = qng + 1;
			LK(cudaMemsetAsync(qng, 0, 2 * sizeof(int), st), "memset");
			cudaEvent_t e0 = L.ev[6], e1 = L.ev[7];
			cudaEventRecord(e0, st);
			k_resolve_b<<<blocks_for(ng + nr), 128, 0, st>>>(b, L.qg[qi ^ 1].p, ng, L.q[qi ^ 1].p, nr,
									  all ? 1 : 0, L.qg[qi].p, qng, L.q[qi].p, qnr);
			++launches;
			cudaEventRecord(e1, st);
			LK(cudaMemcpyAsync(L.h_small.p + 10, qng, 2 * sizeof(int), cudaMemcpyDeviceToHost, st), "queues");
			LK(cudaStreamSynchronize(st), "resolve");
			float ms = 0;
			cudaEventElapsedTime(&ms, e0, e1);
			resolve_ms += ms;
			all = false;
			ng = L.h_small.p[10];
			nr = L.h_small.p[11];
			if (ng + nr == 0)
				break;
			++rounds;
			if (ng) {
				Round G{};
				G.req = L.qg[qi].p;
				G.ntask = ng;
				G.space = 2 * ERR;
				rc = gp_round(ctx, L, b, G, launches, build_ms, dp_ms);
				if (rc)
					return rc;
			}
			if (nr) {
				rc = rescue_round(ctx, L, b, L.q[qi].p, nr, max_len, launches, rescue_ms);
				if (rc)
					return rc;
			}
			qi ^= 1;
		}
	}
	cudaEventRecord(L.ev[4], st);
	// pack: per-record pool sizes, their offsets and totals (and the
	// batch's flags and work counters)
	uint32_t *cl = L.cnt.p, *co = cl + (items + 1), *cm = co + (items + 1);
	uint32_t *xl = cm + (items + 1), *xo = xl + (items + 1), *xm = xo + (items + 1);
	auto count_scan = [&](const Side &side) -> int {
		LK(cudaMemsetAsync(cl, 0, 3 * sizeof(uint32_t) * (items + 1), st), "memset");
		k_count<<<blocks_for(items, 256), 256, 0, st>>>(L.pairs.p, n, ncand, cl, co, cm, side);
		++launches;
		size_t tmp_bytes = 0;
		cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cl, xl, items + 1, st);
		LK(L.cub_tmp.ensure(tmp_bytes), "scan scratch");
		cub::DeviceScan::ExclusiveSum(L.cub_tmp.p, tmp_bytes, cl, xl, items + 1, st);
		cub::DeviceScan::ExclusiveSum(L.cub_tmp.p, tmp_bytes, co, xo, items + 1, st);
		cub::DeviceScan::ExclusiveSum(L.cub_tmp.p, tmp_bytes, cm, xm, items + 1, st);
		LK(cudaMemcpyAsync(L.h_small.p + 2, xl + items, 4, cudaMemcpyDeviceToHost, st), "totals");
		LK(cudaMemcpyAsync(L.h_small.p + 3, xo + items, 4, cudaMemcpyDeviceToHost, st), "totals");
		LK(cudaMemcpyAsync(L.h_small.p + 4, xm + items, 4, cudaMemcpyDeviceToHost, st), "totals");
		LK(cudaMemcpyAsync(L.h_small.p + 5, d_flags, 4, cudaMemcpyDeviceToHost, st), "flags");
		LK(cudaMemcpyAsync(L.h_small.p + 16, d_stats, ST_N * sizeof(unsigned long long),
				   cudaMemcpyDeviceToHost, st),
		   "counters");
		LK(cudaStreamSynchronize(st), "scan");
		return HERA_GPU_OK;
	};
	Side side{};
	int rc = count_scan(side);
	if (rc)
		return rc;
	int fl = L.h_small.p[5];
	if ((fl & F_CAPS) && !L.no_wide) {
		// pairs past a first-pass capacity: aligned again in the wide pass,
		// then the records packed with theirs in place
		int wf = 0;
		rc = wide_pass(ctx, L, b, n, paired, spr, max_len, launches, resolve_ms, rescue_ms, rounds, side, wf);
		if (rc)
			return rc;
		T.wide_items += (uint64_t)L.h_small.p[28];
		fl = (fl & ~F_CAPS) | (wf & ~F_CAPS) | ((wf & F_CAPS) ? F_WIDE : 0);
		rc = count_scan(side);
		if (rc)
			return rc;
	}
	const uint32_t tl = (uint32_t)L.h_small.p[2], to = (uint32_t)L.h_small.p[3],
		       tm = (uint32_t)L.h_small.p[4];
	L.items = items;
	L.rb_l = L.rb_o = L.rb_m = 0;
	L.nl = tl;
	L.no = to;
	L.nm = tm;
	// owned pools keep one spare entry; pools bound to a caller's buffers
	// are held to exactly the capacity the caller gave (nothing is ever
	// written at index tl / to / tm)
	L.pools_short = true;
	LK(pool_ensure(L.pos_pool, tl), "list pool");
	LK(pool_ensure(L.p_pool, tl), "list pool");
	LK(pool_ensure(L.op_pool, to), "op pool");
	LK(pool_ensure(L.miss_pool, tm), "miss pool");
	L.pools_short = false;
	k_emit<<<blocks_for(items, 256), 256, 0, st>>>(L.pairs.p, n, ncand, xl, xo, xm, L.recs.p, L.pos_pool.p,
							L.p_pool.p, L.op_pool.p, L.miss_pool.p, 0, 0, 0, side);
	++launches;
	cudaEventRecord(L.ev[5], st);
	LK(cudaGetLastError(), "kernel launch");
	LK(cudaStreamSynchronize(st), "pack");
	float ms = 0;
	cudaEventElapsedTime(&ms, L.ev[1], L.ev[2]);
	T.seed_ms += ms;
	if (paired) {
		cudaEventElapsedTime(&ms, L.ev[8], L.ev[9]);
		T.seed_kernel_ms += ms;
	}
	{
		const unsigned long long *hs = reinterpret_cast<const unsigned long long *>(L.h_small.p + 16);
		T.probes += hs[ST_PROBES];
		T.seed_hits += hs[ST_SEED_HITS];
		T.sw_cells += hs[ST_SW_CELLS];
		T.ssw_cells += hs[ST_SSW_CELLS];
	}
	if (!batched) {
		cudaEventElapsedTime(&ms, L.ev[2], L.ev[3]);
		T.position_ms += ms;
	} else {
		T.position_ms += build_ms + dp_ms;
		T.build_ms += build_ms;
		T.dp_ms += dp_ms;
	}
	T.resolve_ms += resolve_ms;
	T.rescue_ms += rescue_ms;
	cudaEventElapsedTime(&ms, L.ev[4], L.ev[5]);
	T.pack_ms += ms;
	T.launches += launches;
	T.rescue_rounds += rounds;
	L.items = items;
	L.rb_l = L.rb_o = L.rb_m = 0;
	L.ncand = ncand;
	L.nl = tl;
	L.no = to;
	L.nm = tm;
	if (fl) {
		char buf[200];
		if (fl & F_WIDE)
			snprintf(buf, sizeof buf, "a read passed the wide pass's capacities (%d anchors or hits of one "
				 "get_position call; flags 0x%x)", CapsWide::A, fl);
		else if ((fl & F_CAPS) && L.no_wide)
			snprintf(buf, sizeof buf, "per-read capacity exceeded (flags 0x%x); this entry has no wide pass",
				 fl);
		else
			snprintf(buf, sizeof buf, "per-read capacity exceeded (flags 0x%x)", fl);
		return set_err(L.err, HERA_GPU_ECAPACITY, buf);
	}
	return HERA_GPU_OK;
}

// ---- host copy pool ------------------------------------------------------
//
// One host thread copies pageable memory at a few GB/s, far below what the
// PCIe copies and the kernels sustain, so the large host copies of a call
// (reads into pinned staging, records and pools out of it) are cut into
// pieces that a process-wide pool of threads and the calling thread share.
// Lanes submit concurrently; each waits for its own job only.
class CopyPool {
public:
	static CopyPool &get()
	{
		static CopyPool p;
		return p;
	}
	// run fn(0 .. n-1), the caller taking part
	void run(size_t n, const std::function<void(size_t)> &fn)
	{
		if (n == 0)
			return;
		if (n == 1 || th_.empty()) {
			for (size_t i = 0; i < n; ++i)
				fn(i);
			return;
		}
		auto j = std::make_shared<Job>();
		j->fn = &fn;
		j->n = n;
		{
			std::lock_guard<std::mutex> g(mu_);
			q_.push_back(j);
		}
		cv_.notify_all();
		work(*j);
		std::unique_lock<std::mutex> g(j->mu);
		j->cv.wait(g, [&] { return j->done.load() == j->n; });
	}
	~CopyPool()
	{
		{
			std::lock_guard<std::mutex> g(mu_);
			stop_ = true;
		}
		cv_.notify_all();
		for (auto &t : th_)
			t.join();
	}

private:
	struct Job {
		const std::function<void(size_t)> *fn = nullptr;
		size_t n = 0;
		std::atomic<size_t> next{0}, done{0};
		std::mutex mu;
		std::condition_variable cv;
	};
	CopyPool()
	{
		unsigned n = std::thread::hardware_concurrency();
		n = n > 16 ? 16 : n;
		for (unsigned i = 1; i < n; ++i)
			th_.emplace_back([this] { loop(); });
	}
	static void work(Job &j)
	{
		for (;;) {
			const size_t i = j.next.fetch_add(1);
			if (i >= j.n)
				return;
			(*j.fn)(i);
			if (j.done.fetch_add(1) + 1 == j.n) {
				std::lock_guard<std::mutex> g(j.mu);
				j.cv.notify_all();
			}
		}
	}
	void loop()
	{
		for (;;) {
			std::shared_ptr<Job> j;
			{
				std::unique_lock<std::mutex> g(mu_);
				cv_.wait(g, [&] {
					while (!q_.empty() && q_.front()->next.load() >= q_.front()->n)
						q_.pop_front();
					return stop_ || !q_.empty();
				});
				if (stop_)
					return;
				j = q_.front();
			}
			work(*j);
		}
	}
	std::vector<std::thread> th_;
	std::mutex mu_;
	std::condition_variable cv_;
	std::deque<std::shared_ptr<Job>> q_;
	bool stop_ = false;
};

// memcpy in pieces of at most 4 MiB over the pool
static void pcopy(void *dst, const void *src, size_t bytes)
{
	const size_t piece = 4u << 20;
	const size_t n = (bytes + piece - 1) / piece;
	CopyPool::get().run(n, [&](size_t i) {
		const size_t a = i * piece, b = a + piece < bytes ? a + piece : bytes;
		memcpy(static_cast<char *>(dst) + a, static_cast<const char *>(src) + a, b - a);
	});
}

// true if host range [p, p + bytes) is page-locked (cudaHostAlloc, or
// cudaHostRegister / hera_gpu_host_register): copies can then use it
// directly instead of going through the lane's pinned staging
static bool host_pinned(const void *p, size_t bytes)
{
	if (!p || bytes == 0)
		return false;
	cudaPointerAttributes a{}, e{};
	if (cudaPointerGetAttributes(&a, p) != cudaSuccess ||
	    cudaPointerGetAttributes(&e, static_cast<const char *>(p) + bytes - 1) != cudaSuccess) {
		cudaGetLastError();
		return false;
	}
	return a.type == cudaMemoryTypeHost && e.type == cudaMemoryTypeHost;
}

// records of a sub-batch rebased to the caller's pool offsets on the device
// (by the difference to the offsets they were last rebased to; u32 wrap-around)
__global__ void k_rebase_recs(hera_cand_rec *__restrict__ r, int n, uint32_t bl, uint32_t bo, uint32_t bm)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	for (int s = 0; s < 2; ++s) {
		r[i].list_off[s] += bl;
		r[i].cig_off[s] += bo;
		r[i].miss_off[s] += bm;
	}
}

// D2H of lane L's packed records into `out` at record rec0 and pool
// offsets (bl, bo, bm), through the lane's pinned staging
static int copy_out(Lane &L, hera_gpu_result *out, uint64_t rec0, uint64_t bl, uint64_t bo, uint64_t bm)
{
	cudaStream_t st = L.stream;
	const int items = L.items;
	// caller buffers that are page-locked take the records straight from
	// the device (offsets rebased there); otherwise through the staging
	if (host_pinned(out->recs + rec0, (size_t)items * sizeof(hera_cand_rec)) &&
	    (!L.nl || (host_pinned(out->pos_pool + bl, L.nl * 4) && host_pinned(out->p_pool + bl, L.nl * 4))) &&
	    (!L.no || host_pinned(out->op_pool + bo, L.no * 4)) && (!L.nm || host_pinned(out->miss_pool + bm, L.nm))) {
		cudaEventRecord(L.ev[6], st);
		if (items > 0)
			k_rebase_recs<<<blocks_for(items, 256), 256, 0, st>>>(L.recs.p, items, (uint32_t)bl - L.rb_l,
									       (uint32_t)bo - L.rb_o, (uint32_t)bm - L.rb_m);
		L.rb_l = (uint32_t)bl;
		L.rb_o = (uint32_t)bo;
		L.rb_m = (uint32_t)bm;
		LK(cudaMemcpyAsync(out->recs + rec0, L.recs.p, items * sizeof(hera_cand_rec), cudaMemcpyDeviceToHost, st),
		   "D2H");
		if (L.nl) {
			LK(cudaMemcpyAsync(out->pos_pool + bl, L.pos_pool.p, L.nl * 4, cudaMemcpyDeviceToHost, st), "D2H");
			LK(cudaMemcpyAsync(out->p_pool + bl, L.p_pool.p, L.nl * 4, cudaMemcpyDeviceToHost, st), "D2H");
		}
		if (L.no)
			LK(cudaMemcpyAsync(out->op_pool + bo, L.op_pool.p, L.no * 4, cudaMemcpyDeviceToHost, st), "D2H");
		if (L.nm)
			LK(cudaMemcpyAsync(out->miss_pool + bm, L.miss_pool.p, L.nm, cudaMemcpyDeviceToHost, st), "D2H");
		cudaEventRecord(L.ev[7], st);
		LK(cudaStreamSynchronize(st), "D2H");
		float ms = 0;
		cudaEventElapsedTime(&ms, L.ev[6], L.ev[7]);
		L.timing.d2h_ms += ms;
		return HERA_GPU_OK;
	}
	LK(L.h_recs.ensure(items + 1), "pinned records");
	LK(L.h_pos.ensure(L.nl + 1), "pinned pools");
	LK(L.h_p.ensure(L.nl + 1), "pinned pools");
	LK(L.h_ops.ensure(L.no + 1), "pinned pools");
	LK(L.h_miss.ensure(L.nm + 1), "pinned pools");
	cudaEventRecord(L.ev[6], st);
	LK(cudaMemcpyAsync(L.h_recs.p, L.recs.p, items * sizeof(hera_cand_rec), cudaMemcpyDeviceToHost, st), "D2H");
	if (L.nl) {
		LK(cudaMemcpyAsync(L.h_pos.p, L.pos_pool.p, L.nl * 4, cudaMemcpyDeviceToHost, st), "D2H");
		LK(cudaMemcpyAsync(L.h_p.p, L.p_pool.p, L.nl * 4, cudaMemcpyDeviceToHost, st), "D2H");
	}
	if (L.no)
		LK(cudaMemcpyAsync(L.h_ops.p, L.op_pool.p, L.no * 4, cudaMemcpyDeviceToHost, st), "D2H");
	if (L.nm)
		LK(cudaMemcpyAsync(L.h_miss.p, L.miss_pool.p, L.nm, cudaMemcpyDeviceToHost, st), "D2H");
	cudaEventRecord(L.ev[7], st);
	LK(cudaStreamSynchronize(st), "D2H");
	float ms = 0;
	cudaEventElapsedTime(&ms, L.ev[6], L.ev[7]);
	L.timing.d2h_ms += ms;
	const auto h0 = std::chrono::steady_clock::now();
	hera_cand_rec *dst = out->recs + rec0;
	const int per = 65536;   // records per piece
	CopyPool::get().run(((size_t)items + per - 1) / per, [&](size_t k) {
		const int a = (int)k * per, e = a + per < items ? a + per : items;
		for (int i = a; i < e; ++i) {
			hera_cand_rec r = L.h_recs.p[i];
			for (int s = 0; s < 2; ++s) {
				r.list_off[s] += (uint32_t)bl;
				r.cig_off[s] += (uint32_t)bo;
				r.miss_off[s] += (uint32_t)bm;
			}
			dst[i] = r;
		}
	});
	if (L.nl) {
		pcopy(out->pos_pool + bl, L.h_pos.p, L.nl * 4);
		pcopy(out->p_pool + bl, L.h_p.p, L.nl * 4);
	}
	if (L.no)
		pcopy(out->op_pool + bo, L.h_ops.p, L.no * 4);
	if (L.nm)
		pcopy(out->miss_pool + bm, L.h_miss.p, L.nm);
	L.timing.host_out_ms +=
		std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - h0).count();
	return HERA_GPU_OK;
}

// stage host reads of [lo, lo+n) into lane L's pinned memory and device
// buffers; mates interleaved in the offset table, sequences as blocks
// Stage reads [lo, lo + n) into the lane's buffer set `set` (0: seq/off/len,
// 1: seq2/off2/len2).  Synchronous on the lane's stream, or (async) on its
// copy stream with cev[set][1] recorded when the copies are done; stage_wait
// then waits for them.
static int stage_reads_to(Lane &L, const hera_gpu_reads *a, const hera_gpu_reads *b, int32_t lo, int32_t n,
			  int64_t *bytes, int *max_len, int set, bool async)
{
	cudaStream_t st = async ? L.cstream : L.stream;
	DBuf<uint8_t> &dseq = set ? L.seq2 : L.seq;
	DBuf<int64_t> &doff = set ? L.off2 : L.off;
	DBuf<int32_t> &dlen = set ? L.len2 : L.len;
	cudaEvent_t e0 = async ? L.cev[set][0] : L.ev[0], e1 = async ? L.cev[set][1] : L.ev[1];
	const int per = b ? 2 : 1;
	const hera_gpu_reads *src[2] = {a, b};
	int64_t total = 0;
	int ml = 0;
	bool contig[2] = {true, true};
	for (int m = 0; m < per; ++m) {
		const hera_gpu_reads *r = src[m];
		for (int32_t i = lo; i < lo + n; ++i) {
			if (r->len[i] < 0)
				return set_err(L.err, HERA_GPU_EINVAL, "negative read length");
			total += r->len[i];
			ml = r->len[i] > ml ? r->len[i] : ml;
			if (i > lo && r->off[i] != r->off[i - 1] + r->len[i - 1])
				contig[m] = false;
		}
	}
	if (ml > MAX_READ)
		return set_err(L.err, HERA_GPU_EINVAL, "read longer than HERA_GPU_MAX_READ");
	LK(L.h_seq.ensure(total + 1), "pinned reads");
	LK(L.h_off.ensure((size_t)n * per), "pinned offsets");
	LK(L.h_len.ensure((size_t)n * per), "pinned lengths");
	const auto h0 = std::chrono::steady_clock::now();
	int64_t o = 0;
	// a contiguous, page-locked mate block goes to the device directly
	int64_t reg_o[2] = {0, 0}, reg_len[2] = {0, 0};
	const char *direct[2] = {nullptr, nullptr};
	for (int m = 0; m < per; ++m) {
		const hera_gpu_reads *r = src[m];
		reg_o[m] = o;
		if (contig[m] && n > 0) {
			const int64_t len_m = r->off[lo + n - 1] + r->len[lo + n - 1] - r->off[lo];
			if (host_pinned(r->seq + r->off[lo], (size_t)len_m))
				direct[m] = r->seq + r->off[lo];
			else
				pcopy(L.h_seq.p + o, r->seq + r->off[lo], (size_t)len_m);
			const int64_t shift = o - r->off[lo];
			for (int32_t i = 0; i < n; ++i) {
				L.h_off.p[(size_t)i * per + m] = r->off[lo + i] + shift;
				L.h_len.p[(size_t)i * per + m] = r->len[lo + i];
			}
			o += len_m;
		} else {
			for (int32_t i = 0; i < n; ++i) {
				const int32_t Ln = r->len[lo + i];
				memcpy(L.h_seq.p + o, r->seq + r->off[lo + i], (size_t)Ln);
				L.h_off.p[(size_t)i * per + m] = o;
				L.h_len.p[(size_t)i * per + m] = Ln;
				o += Ln;
			}
		}
		reg_len[m] = o - reg_o[m];
	}
	L.timing.host_stage_ms +=
		std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - h0).count();
	LK(dseq.ensure(total + 64), "device reads");
	LK(doff.ensure((size_t)n * per), "device offsets");
	LK(dlen.ensure((size_t)n * per), "device lengths");
	cudaEventRecord(e0, st);
	if (!direct[0] && !direct[1]) {
		LK(cudaMemcpyAsync(dseq.p, L.h_seq.p, total, cudaMemcpyHostToDevice, st), "H2D reads");
	} else {   // per mate block: from the caller's memory or from the staging
		for (int m = 0; m < per; ++m) {
			const void *from = direct[m] ? (const void *)direct[m] : (const void *)(L.h_seq.p + reg_o[m]);
			if (reg_len[m] > 0)
				LK(cudaMemcpyAsync(dseq.p + reg_o[m], from, (size_t)reg_len[m], cudaMemcpyHostToDevice, st),
				   "H2D reads");
		}
	}
	LK(cudaMemcpyAsync(doff.p, L.h_off.p, (size_t)n * per * 8, cudaMemcpyHostToDevice, st), "H2D");
	LK(cudaMemcpyAsync(dlen.p, L.h_len.p, (size_t)n * per * 4, cudaMemcpyHostToDevice, st), "H2D");
	cudaEventRecord(e1, st);
	if (!async) {
		LK(cudaEventSynchronize(e1), "H2D");
		float ms = 0;
		cudaEventElapsedTime(&ms, e0, e1);
		L.timing.h2d_ms += ms;
	}
	*bytes = total;
	*max_len = ml;
	return HERA_GPU_OK;
}

// wait for an async stage_reads_to into `set`
static int stage_wait(Lane &L, int set)
{
	LK(cudaEventSynchronize(L.cev[set][1]), "H2D");
	float ms = 0;
	cudaEventElapsedTime(&ms, L.cev[set][0], L.cev[set][1]);
	L.timing.h2d_ms += ms;
	return HERA_GPU_OK;
}

// ---- sub-batch scheduling over the lanes --------------------------------

struct Sched {
	std::mutex mu;
	std::condition_variable cv;
	std::vector<int> ready;             // sub-batch k's sizes are known
	std::vector<uint64_t> nl, no, nm;
	bool abort = false;
	int rc = HERA_GPU_OK;
	std::string err;
	void publish(int k, uint64_t l, uint64_t o, uint64_t m)
	{
		std::lock_guard<std::mutex> g(mu);
		nl[k] = l;
		no[k] = o;
		nm[k] = m;
		ready[k] = 1;
		cv.notify_all();
	}
	void failed(int k, int code, const std::string &e)
	{
		std::lock_guard<std::mutex> g(mu);
		if (!abort) {
			abort = true;
			rc = code;
			err = e;
		}
		ready[k] = 1;
		cv.notify_all();
	}
	// wait for the sizes of every sub-batch before k; false on abort
	bool prefix(int k, uint64_t &bl, uint64_t &bo, uint64_t &bm)
	{
		std::unique_lock<std::mutex> g(mu);
		cv.wait(g, [&] {
			if (abort)
				return true;
			for (int q = 0; q < k; ++q)
				if (!ready[q])
					return false;
			return true;
		});
		if (abort)
			return false;
		bl = bo = bm = 0;
		for (int q = 0; q < k; ++q) {
			bl += nl[q];
			bo += no[q];
			bm += nm[q];
		}
		return true;
	}
};

static hera_gpu_timing sum_lanes(const std::vector<Lane *> &lanes)
{
	hera_gpu_timing t{};
	for (Lane *L : lanes) {
		const hera_gpu_timing &a = L->timing;
		t.h2d_ms += a.h2d_ms;
		t.seed_ms += a.seed_ms;
		t.position_ms += a.position_ms;
		t.resolve_ms += a.resolve_ms;
		t.rescue_ms += a.rescue_ms;
		t.pack_ms += a.pack_ms;
		t.d2h_ms += a.d2h_ms;
		t.build_ms += a.build_ms;
		t.dp_ms += a.dp_ms;
		t.launches += a.launches;
		t.rescue_rounds += a.rescue_rounds;
		t.lookups += a.lookups;
		t.dp_jobs += a.dp_jobs;
		t.dp_calls += a.dp_calls;
		t.seed_kernel_ms += a.seed_kernel_ms;
		t.dp_kernel_ms += a.dp_kernel_ms;
		t.rescue_kernel_ms += a.rescue_kernel_ms;
		t.host_stage_ms += a.host_stage_ms;
		t.host_out_ms += a.host_out_ms;
		t.probes += a.probes;
		t.seed_hits += a.seed_hits;
		t.sw_cells += a.sw_cells;
		t.ssw_cells += a.ssw_cells;
		t.wide_items += a.wide_items;
	}
	return t;
}

static void sum_timing(hera_gpu_ctx *ctx)
{
	hera_gpu_timing t = sum_lanes(ctx->lanes);
	t.total_ms = ctx->timing.total_ms;
	ctx->timing = t;
}

// One flat call on a group of lanes; its status, error text and timing go
// to rc / err / tm (the context's own fields are left to the caller).
static int align_flat_on(hera_gpu_ctx *ctx, const std::vector<Lane *> &lanes, const hera_gpu_reads *r1,
			 const hera_gpu_reads *r2, int32_t n, int write_bam, hera_gpu_result *out, std::string &err,
			 hera_gpu_timing &tm)
{
	if (cudaSetDevice(ctx->device) != cudaSuccess) {
		err = "cudaSetDevice";
		return HERA_GPU_ENODEV;
	}
	const auto t0 = std::chrono::steady_clock::now();
	const bool paired = r2 != nullptr;
	const int ncand = paired ? 2 : 1;
	for (Lane *L : lanes)
		L->timing = hera_gpu_timing{};
	// sub-batches of at most max_batch pairs, as many as a multiple of the
	// lane count (each lane then carries an equal share of the call)
	const int64_t nlanes = (int64_t)lanes.size();
	int64_t ns = (n + (int64_t)ctx->max_batch - 1) / ctx->max_batch;
	if (ns > 0 && n >= nlanes * 4096)
		ns = (ns + nlanes - 1) / nlanes * nlanes;

	const int32_t sub = ns > 0 ? (int32_t)((n + ns - 1) / ns) : 1;
	const int nsub = (int)((n + (int64_t)sub - 1) / sub);
	Sched S;
	S.ready.assign(nsub, 0);
	S.nl.assign(nsub, 0);
	S.no.assign(nsub, 0);
	S.nm.assign(nsub, 0);
	const int nl = (int)lanes.size() < nsub ? (int)lanes.size() : nsub;
	const int dev = ctx->device;
	auto worker = [&](int li) {
		cudaSetDevice(dev);
		Lane &L = *lanes[li];
		// a lane's sub-batches alternate between its two buffer sets: the
		// next one is staged on the copy stream while this one runs
		int b = 0;
		int64_t sbytes[2] = {0, 0};
		int smax[2] = {0, 0};
		bool pending = false;   // an async stage into set b is in flight
		auto drain = [&] {      // nothing left reading the caller's memory
			if (pending)
				cudaStreamSynchronize(L.cstream);
			pending = false;
		};
		for (int k = li; k < nsub; k += nl) {
			const int32_t lo = (int32_t)((int64_t)k * sub);
			const int32_t m = (n - lo) < sub ? (n - lo) : sub;
			int rc = HERA_GPU_OK;
			if (k == li)
				rc = stage_reads_to(L, r1, r2, lo, m, &sbytes[b], &smax[b], b, false);
			else if (pending)
				rc = stage_wait(L, b);
			pending = false;
			const int kn = k + nl;
			if (!rc && kn < nsub) {
				const int32_t lon = (int32_t)((int64_t)kn * sub);
				const int32_t mn = (n - lon) < sub ? (n - lon) : sub;
				rc = stage_reads_to(L, r1, r2, lon, mn, &sbytes[b ^ 1], &smax[b ^ 1], b ^ 1, true);
				pending = rc == HERA_GPU_OK;
			}
			if (!rc)
				rc = run_batch(ctx, L, b ? L.seq2.p : L.seq.p, b ? L.off2.p : L.off.p, b ? L.len2.p : L.len.p, m,
					       paired, write_bam, smax[b], sbytes[b]);
			if (rc) {
				drain();
				S.failed(k, rc, L.err);
				return;
			}
			S.publish(k, L.nl, L.no, L.nm);
			uint64_t bl, bo, bm;
			if (!S.prefix(k, bl, bo, bm)) {
				drain();
				return;
			}
			if (bl + L.nl <= out->list_cap && bo + L.no <= out->op_cap && bm + L.nm <= out->miss_cap) {
				rc = copy_out(L, out, (uint64_t)lo * ncand, bl, bo, bm);
				if (rc) {
					drain();
					S.failed(k, rc, L.err);
					return;
				}
			}
			b ^= 1;
		}
		drain();
	};
	std::vector<std::thread> th;
	for (int i = 1; i < nl; ++i)
		th.emplace_back(worker, i);
	if (nl > 0)
		worker(0);
	for (auto &t : th)
		t.join();
	tm = sum_lanes(lanes);
	tm.total_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
	if (S.abort) {
		err = S.err;
		return S.rc;
	}
	uint64_t tl = 0, to = 0, tmm = 0;
	for (int k = 0; k < nsub; ++k) {
		tl += S.nl[k];
		to += S.no[k];
		tmm += S.nm[k];
	}
	out->list_used = tl;
	out->op_used = to;
	out->miss_used = tmm;
	if (tl > out->list_cap || to > out->op_cap || tmm > out->miss_cap) {
		err = "result pools too small (see *_used for the sizes needed)";
		return HERA_GPU_ECAPACITY;
	}
	return HERA_GPU_OK;
}

static int align_flat(hera_gpu_ctx *ctx, const hera_gpu_reads *r1, const hera_gpu_reads *r2, int32_t n,
		      int write_bam, hera_gpu_result *out)
{
	if (!ctx || !r1 || !out || n < 0 || (write_bam != 0 && write_bam != 1))
		return fail(ctx, HERA_GPU_EINVAL, "bad argument");
	std::string err;
	hera_gpu_timing tm{};
	const int rc = align_flat_on(ctx, ctx->lanes, r1, r2, n, write_bam, out, err, tm);
	ctx->timing = tm;
	return rc ? fail(ctx, rc, err.c_str()) : HERA_GPU_OK;
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

// ---- asynchronous flat calls --------------------------------------------

extern "C" int hera_gpu_align_pairs_submit(hera_gpu_ctx *ctx, const hera_gpu_reads *r1, const hera_gpu_reads *r2,
					   int32_t n, int write_bam, hera_gpu_result *out, uint64_t *ticket)
{
	if (!ctx || !r1 || !r2 || !out || !ticket || n < 0 || (write_bam != 0 && write_bam != 1))
		return fail(ctx, HERA_GPU_EINVAL, "bad argument");
	std::lock_guard<std::mutex> g(ctx->async_mu);
	int k = -1;
	for (int i = 0; i < 2 && k < 0; ++i)
		if (!ctx->async[i].busy)
			k = i;
	if (k < 0)
		return fail(ctx, HERA_GPU_EINVAL, "two asynchronous calls in flight: complete one first");
	if (k == 1 && ctx->lanes2.empty()) {
		if (cudaSetDevice(ctx->device) != cudaSuccess)
			return fail(ctx, HERA_GPU_ENODEV, "cudaSetDevice");
		if (make_lanes(ctx->lanes2, (int)ctx->lanes.size()) != HERA_GPU_OK)
			return fail(ctx, HERA_GPU_ECUDA, "lanes of the second asynchronous call");
	}
	auto &a = ctx->async[k];
	if (a.th.joinable())
		a.th.join();
	a.busy = true;
	a.ticket = ctx->next_async++;
	a.r1 = *r1;
	a.r2 = *r2;
	a.rc = HERA_GPU_OK;
	a.err.clear();
	const std::vector<Lane *> *group = k == 0 ? &ctx->lanes : &ctx->lanes2;
	a.th = std::thread([ctx, &a, group, n, write_bam, out] {
		a.rc = align_flat_on(ctx, *group, &a.r1, &a.r2, n, write_bam, out, a.err, a.tm);
	});
	*ticket = a.ticket;
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_align_pairs_complete(hera_gpu_ctx *ctx, uint64_t ticket)
{
	if (!ctx)
		return HERA_GPU_EINVAL;
	hera_gpu_ctx::AsyncCall *a = nullptr;
	{
		std::lock_guard<std::mutex> g(ctx->async_mu);
		for (auto &c : ctx->async)
			if (c.busy && c.ticket == ticket)
				a = &c;
	}
	if (!a)
		return fail(ctx, HERA_GPU_EINVAL, "unknown or completed ticket");
	a->th.join();
	std::lock_guard<std::mutex> g(ctx->async_mu);
	a->busy = false;
	ctx->timing = a->tm;
	return a->rc ? fail(ctx, a->rc, a->err.c_str()) : HERA_GPU_OK;
}

// lane-local offsets of a device-resident sub-batch
__global__ void k_rebase(const int64_t *__restrict__ in, int64_t n, int64_t base, int64_t *__restrict__ out)
{
	const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
	if (t < n)
		out[t] = in[t] - base;
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
	const auto t0 = std::chrono::steady_clock::now();
	cudaStream_t caller = stream ? (cudaStream_t)stream : ctx->stream;
	for (Lane *L : ctx->lanes)
		L->timing = hera_gpu_timing{};
	ctx->nparts = 0;
	if (n == 0)
		return HERA_GPU_OK;
	// one contiguous sub-batch per lane (results stay in the lane's pools)
	const int nl = (int)ctx->lanes.size();
	int parts = nl;
	while (parts > 1 && n / parts < 4096)
		--parts;
	std::vector<int32_t> lo(parts + 1);
	for (int k = 0; k <= parts; ++k)
		lo[k] = (int32_t)((int64_t)n * k / parts);
	// the sub-batches' byte ranges: [off of first read, end of last read)
	std::vector<int64_t> first(parts), last(parts);
	std::vector<int32_t> last_len(parts);
	cudaEvent_t start_ev;
	cudaEventCreateWithFlags(&start_ev, cudaEventDisableTiming);
	cudaEventRecord(start_ev, caller);
	for (int k = 0; k < parts; ++k) {
		cudaMemcpyAsync(&first[k], d_off + 2 * (int64_t)lo[k], 8, cudaMemcpyDeviceToHost, caller);
		cudaMemcpyAsync(&last[k], d_off + 2 * (int64_t)lo[k + 1] - 1, 8, cudaMemcpyDeviceToHost, caller);
		cudaMemcpyAsync(&last_len[k], d_len + 2 * (int64_t)lo[k + 1] - 1, 4, cudaMemcpyDeviceToHost, caller);
	}
	if (cudaStreamSynchronize(caller) != cudaSuccess) {
		cudaEventDestroy(start_ev);
		return fail(ctx, HERA_GPU_ECUDA, "offsets");
	}
	std::vector<int> rcs(parts, HERA_GPU_OK);
	const int dev = ctx->device;
	auto worker = [&](int k) {
		cudaSetDevice(dev);
		Lane &L = *ctx->lanes[k];
		cudaStreamWaitEvent(L.stream, start_ev, 0);
		const int32_t m = lo[k + 1] - lo[k];
		const int64_t base = first[k];
		const int64_t bytes = last[k] + last_len[k] - base;
		int rc = HERA_GPU_OK;
		if (L.off.ensure((size_t)2 * m) != cudaSuccess || L.len.ensure(1) != cudaSuccess) {
			rcs[k] = set_err(L.err, HERA_GPU_ENOMEM, "offsets");
			return;
		}
		k_rebase<<<blocks_for(2 * (int64_t)m, 256), 256, 0, L.stream>>>(d_off + 2 * (int64_t)lo[k], 2 * (int64_t)m,
										 base, L.off.p);
		rc = run_batch(ctx, L, d_seq + base, L.off.p, d_len + 2 * (int64_t)lo[k], m, true, write_bam,
			       max_read_len, bytes);
		rcs[k] = rc;
	};
	std::vector<std::thread> th;
	for (int k = 1; k < parts; ++k)
		th.emplace_back(worker, k);
	worker(0);
	for (auto &t : th)
		t.join();
	cudaEventDestroy(start_ev);
	ctx->timing.total_ms =
		std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
	sum_timing(ctx);
	for (int k = 0; k < parts; ++k)
		if (rcs[k] != HERA_GPU_OK)
			return fail(ctx, rcs[k], ctx->lanes[k]->err.c_str());
	// order later work on the caller's stream after the lanes
	for (int k = 0; k < parts; ++k) {
		cudaEventRecord(ctx->lanes[k]->ev[5], ctx->lanes[k]->stream);
		cudaStreamWaitEvent(caller, ctx->lanes[k]->ev[5], 0);
	}
	ctx->nparts = parts;
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_fetch_result(hera_gpu_ctx *ctx, hera_gpu_result *out)
{
	if (!ctx || !out)
		return HERA_GPU_EINVAL;
	uint64_t bl = 0, bo = 0, bm = 0, rec = 0;
	bool fits = true;
	for (int k = 0; k < ctx->nparts; ++k) {
		Lane &L = *ctx->lanes[k];
		if (fits && bl + L.nl <= out->list_cap && bo + L.no <= out->op_cap && bm + L.nm <= out->miss_cap) {
			int rc = copy_out(L, out, rec, bl, bo, bm);
			if (rc)
				return fail(ctx, rc, L.err.c_str());
		} else {
			fits = false;
		}
		rec += (uint64_t)L.items;
		bl += L.nl;
		bo += L.no;
		bm += L.nm;
	}
	out->list_used = bl;
	out->op_used = bo;
	out->miss_used = bm;
	return fits ? HERA_GPU_OK : fail(ctx, HERA_GPU_ECAPACITY, "result pools too small");
}

// ---- allocation-free variant of the device-resident entry ---------------
//
// For callers that cannot allocate device memory while they align (see
// include/hera_gpu.h).  Every per-batch buffer -- the mate-rescue calls'
// outputs, the DP jobs and results, the per-pair Candidate state, the
// queues -- is carved from one file-scope device array; records go straight
// into the caller's device buffers.  Sized for HERA_GPU_NOALLOC_MAX_PAIRS
// pairs of reads up to HERA_GPU_MAX_READ.

namespace na {
constexpr size_t A(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t PAIRS = HERA_GPU_NOALLOC_MAX_PAIRS;
constexpr size_t READS = 2 * PAIRS;
constexpr size_t TASKS = 4 * PAIRS;
constexpr size_t ITEMS = 2 * PAIRS;
constexpr size_t SPR = (MAX_READ - KMER) / KMER + 1;
constexpr size_t SEQ = READS * MAX_READ + 64;
constexpr size_t CHAINS = 32 * PAIRS;
constexpr size_t JOBS = 32 * PAIRS;
constexpr size_t SLOTS = 64 * PAIRS;
constexpr size_t CALLS = 8 * PAIRS;
constexpr size_t CUB = 64 << 10;
constexpr size_t BYTES =
	2 * A(SEQ) + A(READS * 8) + A(READS * 2 * SPR * sizeof(uint2)) + A(PAIRS * sizeof(DPair)) +
	2 * A(PAIRS * sizeof(RmReq)) + 2 * A(PAIRS * sizeof(GpReq)) + A(32 * sizeof(int)) +
	A(6 * (ITEMS + 1) * sizeof(uint32_t)) + A(CUB) + A(TASKS * sizeof(TaskInfo)) + A(TASKS * sizeof(int)) +
	A(CHAINS * sizeof(Chain)) + A(JOBS * sizeof(DpJob)) + A(SLOTS * sizeof(JobSlot)) +
	A(JOBS * (size_t)res_stride(JCAP)) + A(JOBS * sizeof(int)) + A(NBIN * sizeof(int)) +
	A(PAIRS * LCAP * sizeof(int2)) + A(PAIRS * sizeof(int)) + A(CALLS * sizeof(SswOut));
}  // namespace na

// the scratch: every GPU that loads this library holds it until exit
static __device__ __align__(256) uint8_t g_noalloc_scratch[na::BYTES];

static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[64];   // device address of the scratch, per device

// once per device, with that device current: the scratch's device address
// (the host-side symbol is only a stand-in and must never reach a kernel)
static int noalloc_scratch(int dev, uint8_t **out)
{
	std::lock_guard<std::mutex> g(g_noalloc_mu);
	if (dev < 0 || dev >= 64)
		return HERA_GPU_EINVAL;
	if (!g_noalloc_ptr[dev]) {
		void *p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess || !p)
			return HERA_GPU_ECUDA;
		g_noalloc_ptr[dev] = p;
	}
	*out = static_cast<uint8_t *>(g_noalloc_ptr[dev]);
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_align_pairs_device_noalloc(hera_gpu_ctx *ctx, const uint8_t *d_seq,
						   const int64_t *d_off, const int32_t *d_len, int32_t n,
						   int32_t max_read_len, int write_bam,
						   hera_gpu_result *d_out, void *stream)
{
	if (!ctx || !ctx->na || !d_seq || !d_off || !d_len || !d_out || !d_out->recs ||
	    (write_bam != 0 && write_bam != 1) || max_read_len < 1 || max_read_len > MAX_READ)
		return fail(ctx, HERA_GPU_EINVAL, "bad argument");
	if (n < 0 || n > (int32_t)na::PAIRS)
		return fail(ctx, HERA_GPU_EINVAL,
			    "allocation-free entry: more than HERA_GPU_NOALLOC_MAX_PAIRS (1024) pairs");
	d_out->list_used = d_out->op_used = d_out->miss_used = 0;
	if (n == 0)
		return HERA_GPU_OK;
	if (cudaSetDevice(ctx->device) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENODEV, "cudaSetDevice");
	uint8_t *arena = nullptr;
	if (noalloc_scratch(ctx->device, &arena) != HERA_GPU_OK)
		return fail(ctx, HERA_GPU_ECUDA, "cudaGetSymbolAddress of the allocation-free scratch");
	Lane &L = *ctx->na;
	cudaStream_t caller = stream ? (cudaStream_t)stream : ctx->stream;
	// byte range of the batch's reads (pinned counters of the lane)
	int64_t *hb = reinterpret_cast<int64_t *>(L.h_small.p);
	cudaMemcpyAsync(hb, d_off, 8, cudaMemcpyDeviceToHost, caller);
	cudaMemcpyAsync(hb + 1, d_off + 2 * (int64_t)n - 1, 8, cudaMemcpyDeviceToHost, caller);
	cudaMemcpyAsync(L.h_small.p + 4, d_len + 2 * (int64_t)n - 1, 4, cudaMemcpyDeviceToHost, caller);
	if (cudaStreamSynchronize(caller) != cudaSuccess)
		return fail(ctx, HERA_GPU_ECUDA, "read offsets");
	const int64_t base = hb[0];
	const int64_t bytes = hb[1] + L.h_small.p[4] - base;
	if (bytes < 0 || (size_t)bytes + 64 > na::SEQ)
		return fail(ctx, HERA_GPU_EINVAL, "allocation-free entry: reads exceed 2048 x HERA_GPU_MAX_READ bytes");

	// carve the scratch
	uint8_t *q = arena;
	auto take = [&](size_t b) {
		uint8_t *r = q;
		q += na::A(b);
		return r;
	};
	L.code.bind(take(na::SEQ), na::SEQ);
	L.code_r.bind(take(na::SEQ), na::SEQ);
	L.off.bind(take(na::READS * 8), na::READS);
	L.hits.bind(take(na::READS * 2 * na::SPR * sizeof(uint2)), na::READS * 2 * na::SPR);
	L.pairs.bind(take(na::PAIRS * sizeof(DPair)), na::PAIRS);
	for (int k = 0; k < 2; ++k)
		L.q[k].bind(take(na::PAIRS * sizeof(RmReq)), na::PAIRS);
	for (int k = 0; k < 2; ++k)
		L.qg[k].bind(take(na::PAIRS * sizeof(GpReq)), na::PAIRS);
	L.counters.bind(take(32 * sizeof(int)), 32);
	L.cnt.bind(take(6 * (na::ITEMS + 1) * sizeof(uint32_t)), 6 * (na::ITEMS + 1));
	L.cub_tmp.bind(take(na::CUB), na::CUB);
	L.tinfo.bind(take(na::TASKS * sizeof(TaskInfo)), na::TASKS);
	L.tlist.bind(take(na::TASKS * sizeof(int)), na::TASKS);
	L.chains.bind(take(na::CHAINS * sizeof(Chain)), na::CHAINS);
	L.jobs.bind(take(na::JOBS * sizeof(DpJob)), na::JOBS);
	L.slots.bind(take(na::SLOTS * sizeof(JobSlot)), na::SLOTS);
	L.res.bind(take(na::JOBS * (size_t)res_stride(JCAP)), na::JOBS * (size_t)res_stride(JCAP));
	L.perm.bind(take(na::JOBS * sizeof(int)), na::JOBS);
	L.hist.bind(take(NBIN * sizeof(int)), NBIN);
	L.calls.bind(take(na::PAIRS * LCAP * sizeof(int2)), na::PAIRS * LCAP);
	L.rq_base.bind(take(na::PAIRS * sizeof(int)), na::PAIRS);
	L.ssw_out.bind(take(na::CALLS * sizeof(SswOut)), na::CALLS);
	L.chain_cap = na::CHAINS;
	L.job_cap = na::JOBS;
	L.slot_cap = na::SLOTS;
	// outputs: the caller's device buffers (records: 2 n entries)
	L.recs.bind(d_out->recs, 2 * (size_t)n);
	// exactly the caller's capacities: the pools are written below the
	// sizes the count pass found and nowhere else
	L.pos_pool.bind(d_out->pos_pool, d_out->pos_pool ? d_out->list_cap : 0);
	L.p_pool.bind(d_out->p_pool, d_out->p_pool ? d_out->list_cap : 0);
	L.op_pool.bind(d_out->op_pool, d_out->op_pool ? d_out->op_cap : 0);
	L.miss_pool.bind(d_out->miss_pool, d_out->miss_pool ? d_out->miss_cap : 0);

	L.timing = hera_gpu_timing{};
	L.err.clear();
	L.nl = L.no = L.nm = 0;
	L.pools_short = false;
	cudaEventRecord(L.ev[0], caller);
	cudaStreamWaitEvent(L.stream, L.ev[0], 0);
	k_rebase<<<blocks_for(2 * (int64_t)n, 256), 256, 0, L.stream>>>(d_off, 2 * (int64_t)n, base, L.off.p);
	const int rc = run_batch(ctx, L, d_seq + base, L.off.p, d_len, n, true, write_bam, max_read_len, bytes);
	cudaEventRecord(L.ev[5], L.stream);
	cudaStreamWaitEvent(caller, L.ev[5], 0);
	ctx->timing = L.timing;
	if (rc == HERA_GPU_ENOMEM && L.pools_short) {
		// the batch ran; only the caller's pools were too small
		d_out->list_used = L.nl;
		d_out->op_used = L.no;
		d_out->miss_used = L.nm;
		return fail(ctx, HERA_GPU_ECAPACITY,
			    (std::string("allocation-free entry: output pools too small (") + L.err +
			     "); *_used hold the pool sizes needed")
				    .c_str());
	}
	if (rc == HERA_GPU_ENOMEM) {
		// the batch's working set outgrew the fixed scratch: *_used stay 0
		return fail(ctx, HERA_GPU_ECAPACITY,
			    (std::string("allocation-free entry: the batch's working set outgrew the fixed scratch (") +
			     L.err + "); align fewer pairs per call")
				    .c_str());
	}
	if (rc != HERA_GPU_OK)
		return fail(ctx, rc, L.err.c_str());
	d_out->list_used = L.nl;
	d_out->op_used = L.no;
	d_out->miss_used = L.nm;
	return HERA_GPU_OK;
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

// f(lo, hi) over [0, n) in contiguous parts on up to 16 host threads
template <class F>
static void par_for(int64_t n, F f)
{
	const int64_t T = std::max<int64_t>(1, std::min<int64_t>({16, (int64_t)std::thread::hardware_concurrency(),
								   n / 4096 + 1}));
	std::vector<std::thread> th;
	for (int64_t t = 1; t < T; ++t)
		th.emplace_back([&, t] { f(n * t / T, n * (t + 1) / T); });
	f(0, n / T);
	for (auto &x : th)
		x.join();
}

// one drop-in call's arguments, queued for a combined batch
struct DropinArgs {
	hera_read_inf *a, *b;
	int32_t n;
	int write_bam;
	hera_candidate **out;
};

// A batch of drop-in calls of one kind (pairs or single reads, one
// WRITE_BAM) as one flat call: the calls' reads gathered back to back, the
// records of call k at its pairs' place, each call's Candidates made from
// its own records (host threads over all of the batch's items).
static void dropin_batch(hera_gpu_ctx *ctx, std::vector<hcomb::Request *> &batch)
{
	const DropinArgs &first = *static_cast<DropinArgs *>(batch[0]->user);
	const bool paired = first.b != nullptr;
	const int per = paired ? 2 : 1;
	const int write_bam = first.write_bam;
	const size_t nk = batch.size();
	std::vector<int64_t> pair0(nk + 1, 0);   // first pair of call k in the batch
	for (size_t k = 0; k < nk; ++k)
		pair0[k + 1] = pair0[k] + static_cast<DropinArgs *>(batch[k]->user)->n;
	const int64_t n = pair0[nk];
	auto finish = [&](int rc) {
		for (hcomb::Request *r : batch)
			r->rc = rc;
	};
	std::vector<int64_t> off[2];
	std::vector<int32_t> len[2];
	int64_t total = 0;
	for (int m = 0; m < per; ++m) {
		off[m].resize(n);
		len[m].resize(n);
		for (size_t k = 0; k < nk; ++k) {
			const DropinArgs &c = *static_cast<DropinArgs *>(batch[k]->user);
			const hera_read_inf *r = m ? c.b : c.a;
			for (int32_t i = 0; i < c.n; ++i) {
				off[m][pair0[k] + i] = total;
				len[m][pair0[k] + i] = r[i].len;
				total += r[i].len;
			}
		}
	}
	// the reads gathered back to back (host threads), then one flat call
	std::unique_ptr<char[]> seq(new char[(size_t)total + 1]);
	for (int m = 0; m < per; ++m)
		for (size_t k = 0; k < nk; ++k) {
			const DropinArgs &c = *static_cast<DropinArgs *>(batch[k]->user);
			const hera_read_inf *r = m ? c.b : c.a;
			const int64_t p0 = pair0[k];
			par_for(c.n, [&](int64_t lo, int64_t hi) {
				for (int64_t i = lo; i < hi; ++i)
					memcpy(seq.get() + off[m][p0 + i], r[i].seq, (size_t)r[i].len);
			});
		}
	hera_gpu_reads ra{seq.get(), off[0].data(), len[0].data()};
	hera_gpu_reads rb{seq.get(), paired ? off[1].data() : nullptr, paired ? len[1].data() : nullptr};
	const uint64_t items = (uint64_t)n * per;
	std::unique_ptr<hera_cand_rec[]> recs(new hera_cand_rec[items ? items : 1]);
	hera_gpu_result res{};
	res.recs = recs.get();
	std::unique_ptr<uint32_t[]> pos, ops;
	std::unique_ptr<int32_t[]> p;
	std::unique_ptr<char[]> miss;
	uint64_t cl = items * 8 + 64, co = items * 8 + 64, cm = items * 8 + 64;
	for (int attempt = 0; attempt < 2; ++attempt) {
		pos.reset(new uint32_t[cl]);
		p.reset(new int32_t[cl]);
		ops.reset(new uint32_t[co]);
		miss.reset(new char[cm]);
		res.pos_pool = pos.get();
		res.p_pool = p.get();
		res.op_pool = ops.get();
		res.miss_pool = miss.get();
		res.list_cap = cl;
		res.op_cap = co;
		res.miss_cap = cm;
		int rc = align_flat(ctx, &ra, paired ? &rb : nullptr, (int32_t)n, write_bam, &res);
		if (rc == HERA_GPU_OK)
			break;
		if (rc != HERA_GPU_ECAPACITY || attempt == 1 ||
		    (res.list_used <= cl && res.op_used <= co && res.miss_used <= cm))
			return finish(rc);
		cl = res.list_used + 1;
		co = res.op_used + 1;
		cm = res.miss_used + 1;
	}
	// hera's malloc'd Candidates, and the reads upper-cased as hera leaves
	// them, on host threads: item j of the batch is item j - per * pair0[k]
	// of call k
	std::atomic<int> nomem{0};
	par_for((int64_t)items, [&](int64_t lo, int64_t hi) {
		size_t k = std::upper_bound(pair0.begin(), pair0.end(), lo / per) - pair0.begin() - 1;
		for (int64_t j = lo; j < hi; ++j) {
			while (j >= per * pair0[k + 1])
				++k;
			const DropinArgs &c = *static_cast<DropinArgs *>(batch[k]->user);
			hera_candidate *x = materialize(&res, (uint64_t)j);
			c.out[j - per * pair0[k]] = x;
			if (!x)
				nomem = 1;
		}
	});
	if (nomem) {
		for (size_t k = 0; k < nk; ++k) {
			const DropinArgs &c = *static_cast<DropinArgs *>(batch[k]->user);
			hera_gpu_free_candidates(c.out, (int64_t)c.n * per);
		}
		finish(fail(ctx, HERA_GPU_ENOMEM, "candidate allocation"));
		return;
	}
	for (size_t k = 0; k < nk; ++k) {
		const DropinArgs &c = *static_cast<DropinArgs *>(batch[k]->user);
		par_for(c.n, [&](int64_t lo, int64_t hi) {
			for (int64_t i = lo; i < hi; ++i) {
				upper_acgt(c.a[i].seq, c.a[i].len);
				if (c.b)
					upper_acgt(c.b[i].seq, c.b[i].len);
			}
		});
	}
	finish(HERA_GPU_OK);
}

static int align_dropin(hera_gpu_ctx *ctx, hera_read_inf *a, hera_read_inf *b, int32_t n, int write_bam,
			hera_candidate **out)
{
	if (!ctx || !a || !out || n < 0 || (write_bam != 0 && write_bam != 1))
		return fail(ctx, HERA_GPU_EINVAL, "bad argument");
	for (int m = 0; m < (b ? 2 : 1); ++m) {
		const hera_read_inf *r = m ? b : a;
		for (int32_t i = 0; i < n; ++i)
			if (!r[i].seq || r[i].len < 0)
				return fail(ctx, HERA_GPU_EINVAL, "read without sequence");
	}
	if (n == 0)
		return HERA_GPU_OK;
	DropinArgs args{a, b, n, write_bam, out};
	hcomb::Request req;
	req.kind = (b ? 1 : 0) | (write_bam << 1);
	req.items = n;
	req.user = &args;
	return ctx->dropin.call(req, [ctx](std::vector<hcomb::Request *> &batch) { dropin_batch(ctx, batch); });
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

extern "C" void hera_gpu_free_candidates(hera_candidate **c, int64_t n)
{
	if (!c)
		return;
	for (int64_t i = 0; i < n; ++i) {
		hera_candidate *x = c[i];
		if (!x)
			continue;
		for (int s = 0; s < 2; ++s) {
			free(x->pos[s]);
			free(x->p[s]);
			if (x->cigar[s]) {
				free(x->cigar[s]->count);
				free(x->cigar[s]->type);
				free(x->cigar[s]->miss);
				free(x->cigar[s]);
			}
		}
		free(x);
		c[i] = nullptr;
	}
}

// ---- kernel-level check of the gap DP ------------------------------------
//
// One SW_align call (src/hash_align.c:627-760) per (window, query, err),
// run by the batched form's own DP kernels: the register form k_dp_reg<4|8>
// for the live error caps, k_dp_generic for everything else (empty queries,
// windows shorter than error + 1 whose row 0 spills into row 1).  Windows
// are laid out 16 zero bytes apart, like the reference's zero-padded calls.

namespace {
__global__ void k_unit_jobs(const int64_t *__restrict__ ref_at, const int64_t *__restrict__ ref_off,
			    const int64_t *__restrict__ q_off, const int32_t *__restrict__ err, int n,
			    DpJob *__restrict__ jobs, int *__restrict__ perm)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n)
		return;
	DpJob j{};
	j.rstart = (uint32_t)ref_at[t];
	j.ref_len = (uint16_t)(ref_off[t + 1] - ref_off[t]);
	j.len = (uint16_t)(q_off[t + 1] - q_off[t]);
	j.qoff = 0;
	j.err = (int8_t)err[t];
	j.orient = 0;
	j.read = t;
	jobs[t] = j;
	perm[t] = t;
}
}  // namespace

extern "C" int hera_gpu_unit_sw(int device, const char *refs, const int64_t *ref_off, const char *qs,
				const int64_t *q_off, const int32_t *err, int32_t n, int write_bam, int32_t *score,
				uint32_t *ops, int32_t *n_ops, char *miss, int32_t *n_miss, int32_t cap,
				int32_t *flags)
{
	if (!refs || !ref_off || !qs || !q_off || !err || n < 0 || !score || !ops || !n_ops || !miss || !n_miss ||
	    !flags || cap < 1 || (write_bam != 0 && write_bam != 1))
		return HERA_GPU_EINVAL;
	*flags = 0;
	if (n == 0)
		return HERA_GPU_OK;
	if (cudaSetDevice(device) != cudaSuccess)
		return HERA_GPU_ENODEV;
	std::vector<int64_t> at((size_t)n);
	int64_t rb = 0;
	for (int i = 0; i < n; ++i) {
		const int64_t rl = ref_off[i + 1] - ref_off[i], ql = q_off[i + 1] - q_off[i];
		const int e = err[i] < 0 ? -err[i] : err[i];
		if (rl < 0 || rl > 65535 || ql < 0 || ql > MAX_DP_ROWS || e < 1 || e > 12)
			return HERA_GPU_EINVAL;
		at[i] = rb;
		rb += rl + 16;
	}
	const int64_t qb = q_off[n];
	std::vector<uint8_t> seq((size_t)rb + 64, 0);
	for (int i = 0; i < n; ++i)
		memcpy(seq.data() + at[i], refs + ref_off[i], (size_t)(ref_off[i + 1] - ref_off[i]));
	const int rcap = write_bam == 1 ? 2 : JCAP;
	const size_t stride = (size_t)res_stride(rcap);
	auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
	const size_t o_rcode = al((size_t)rb + 64), o_q = o_rcode + al((size_t)rb + 64),
		     o_qc = o_q + al((size_t)qb + 64), o_at = o_qc + al((size_t)qb + 64),
		     o_roff = o_at + al((size_t)n * 8), o_qoff = o_roff + al((size_t)(n + 1) * 8),
		     o_err = o_qoff + al((size_t)(n + 1) * 8), o_jobs = o_err + al((size_t)n * 4),
		     o_perm = o_jobs + al((size_t)n * sizeof(DpJob)), o_res = o_perm + al((size_t)n * 4),
		     o_cnt = o_res + al((size_t)n * stride), need = o_cnt + 256;
	uint8_t *d = nullptr;
	if (cudaMalloc(&d, need) != cudaSuccess)
		return HERA_GPU_ENOMEM;
	int rc = HERA_GPU_OK;
	int *d_cnt = reinterpret_cast<int *>(d + o_cnt);
	cudaGetLastError();
	if (cudaMemcpy(d, seq.data(), (size_t)rb + 64, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(d + o_q, qs, (size_t)qb, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemset(d + o_q + qb, 0, 64) != cudaSuccess ||
	    cudaMemcpy(d + o_at, at.data(), (size_t)n * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(d + o_roff, ref_off, (size_t)(n + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(d + o_qoff, q_off, (size_t)(n + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(d + o_err, err, (size_t)n * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemset(d_cnt, 0, 256) != cudaSuccess)
		rc = HERA_GPU_ECUDA;
	if (rc == HERA_GPU_OK) {
		k_codes<<<64, 256>>>(d, d + o_rcode, rb + 64);
		k_codes<<<64, 256>>>(d + o_q, d + o_qc, qb + 64);
		DpJob *jobs = reinterpret_cast<DpJob *>(d + o_jobs);
		int *perm = reinterpret_cast<int *>(d + o_perm);
		k_unit_jobs<<<blocks_for(n, 256), 256>>>(reinterpret_cast<int64_t *>(d + o_at),
							 reinterpret_cast<int64_t *>(d + o_roff),
							 reinterpret_cast<int64_t *>(d + o_qoff),
							 reinterpret_cast<int32_t *>(d + o_err), n, jobs, perm);
		Batch b{};
		b.ix.code = d + o_rcode;
		b.ix.seq = d;
		b.code = d + o_qc;
		b.code_r = d + o_qc;
		b.off = reinterpret_cast<int64_t *>(d + o_qoff);
		b.flags = d_cnt;
		b.stats = reinterpret_cast<unsigned long long *>(d_cnt + 16);
		b.score_only = write_bam == 1;
		b.max_len = MAX_READ;
		uint8_t *res = d + o_res;
		if (write_bam == 1) {   // the score-only mode, as the aligner runs it
			k_dp_reg<4, true><<<blocks_for(n), 128>>>(b, jobs, perm, n, res, rcap);
			k_dp_reg<8, true><<<blocks_for(n), 128>>>(b, jobs, perm, n, res, rcap);
		} else {
			k_dp_reg<4, false><<<blocks_for(n), 128>>>(b, jobs, perm, n, res, rcap);
			k_dp_reg<8, false><<<blocks_for(n), 128>>>(b, jobs, perm, n, res, rcap);
		}
		k_dp_generic<<<blocks_for(n), 128>>>(b, jobs, n, res, rcap);
		std::vector<uint8_t> h((size_t)n * stride);
		cudaError_t e = cudaGetLastError();
		if (e == cudaSuccess)
			e = cudaDeviceSynchronize();
		if (e == cudaSuccess)
			e = cudaMemcpy(h.data(), res, h.size(), cudaMemcpyDeviceToHost);
		if (e == cudaSuccess)
			e = cudaMemcpy(flags, d_cnt, 4, cudaMemcpyDeviceToHost);
		if (e != cudaSuccess) {
			fprintf(stderr, "hera_gpu_unit_sw: %s\n", cudaGetErrorString(e));
			rc = HERA_GPU_ECUDA;
		} else {
			for (int i = 0; i < n; ++i) {
				const uint8_t *o = h.data() + (size_t)i * stride;
				DpResHdr hd;
				memcpy(&hd, o, sizeof hd);
				score[i] = hd.score;
				n_ops[i] = hd.n;
				n_miss[i] = hd.nm;
				if (hd.caps)
					*flags |= F_CCAP;
				for (int k = 0; k < hd.n && k < cap; ++k)
					memcpy(ops + (size_t)i * cap + k, o + sizeof(DpResHdr) + 4 * k, 4);
				for (int k = 0; k < hd.nm && k < cap; ++k)
					miss[(size_t)i * cap + k] = (char)o[sizeof(DpResHdr) + 4 * rcap + k];
			}
		}
	}
	cudaFree(d);
	return rc;
}

// ---- kernel-level check of the mate-rescue DP ----------------------------

// As in the aligner, a call whose CIGAR passes the first pass's capacities
// runs again in the wide pass's form.
namespace {
template <class K>
__global__ void __launch_bounds__(RESCUE_TPB) k_unit_ssw(DevIndex ix, const int *__restrict__ which,
							  const int64_t *__restrict__ ref_off,
							  const uint8_t *__restrict__ rcode, const int64_t *__restrict__ read_off,
							  int n, SswOutT<K> *__restrict__ out, int per, int *__restrict__ flags)
{
	extern __shared__ __align__(16) uint8_t ssw_sm[];
	const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (w >= n)
		return;
	const int i = which ? which[w] : w;
	const int ln = (int)(ref_off[i + 1] - ref_off[i]), L = (int)(read_off[i + 1] - read_off[i]);
	int f = 0;
	const size_t need = std::is_same<K, CapsStd>::value ? ssw_smem_per_warp(L) : ssw_smem_wide();
	if ((size_t)((threadIdx.x >> 5) + 1) * per > dyn_smem_bytes() || (size_t)per < need) {
		if ((threadIdx.x & 31) == 0)
			flags[w] = F_SCRATCH;
		return;
	}
	ssw_warp(ix, (uint32_t)ref_off[i], ln, rcode, read_off[i], L, 0, 0, 0xffffffffu,
		 ssw_sm + (size_t)(threadIdx.x >> 5) * per, out[w], f);
	if ((threadIdx.x & 31) == 0)
		flags[w] = f;
}
}  // namespace

extern "C" int hera_gpu_unit_ssw(int device, const char *refs, const int64_t *ref_off, const char *reads,
				 const int64_t *read_off, int32_t n, int32_t *score, int32_t *skip, uint32_t *ops,
				 int32_t *n_ops, char *miss, int32_t *n_miss, int32_t cap, int32_t *flags)
{
	if (!refs || !ref_off || !reads || !read_off || n < 0 || !score || !skip || !ops || !n_ops || !miss ||
	    !n_miss || !flags || cap < 1)
		return HERA_GPU_EINVAL;
	*flags = 0;
	if (n == 0)
		return HERA_GPU_OK;
	if (cudaSetDevice(device) != cudaSuccess)
		return HERA_GPU_ENODEV;
	int max_len = 1;
	for (int i = 0; i < n; ++i) {
		const int64_t ln = ref_off[i + 1] - ref_off[i], L = read_off[i + 1] - read_off[i];
		if (ln < 0 || ln > MAX_FRAG || L < 0 || L > MAX_READ)
			return HERA_GPU_EINVAL;
		max_len = L > max_len ? (int)L : max_len;
	}
	const int64_t rb = ref_off[n], qb = read_off[n];
	std::vector<uint8_t> seq((size_t)rb + 64, 0);
	memcpy(seq.data(), refs, (size_t)rb);
	auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
	const size_t o_rcode = al((size_t)rb + 64), o_read = o_rcode + al((size_t)rb + 64),
		     o_qcode = o_read + al((size_t)qb + 64), o_roff = o_qcode + al((size_t)qb + 64),
		     o_qoff = o_roff + al((size_t)(n + 1) * 8), o_flags = o_qoff + al((size_t)(n + 1) * 8),
		     o_which = o_flags + al((size_t)n * 4), o_out = o_which + al((size_t)n * 4),
		     o_wout = o_out + al((size_t)n * sizeof(SswOut));
	uint8_t *d = nullptr;
	if (cudaMalloc(&d, o_wout) != cudaSuccess)
		return HERA_GPU_ENOMEM;
	int64_t *d_roff = reinterpret_cast<int64_t *>(d + o_roff), *d_qoff = reinterpret_cast<int64_t *>(d + o_qoff);
	int *d_flags = reinterpret_cast<int *>(d + o_flags), *d_which = reinterpret_cast<int *>(d + o_which);
	SswOut *d_out = reinterpret_cast<SswOut *>(d + o_out);
	SswOutT<CapsWide> *d_wout = nullptr;
	int rc = HERA_GPU_OK;
	cudaGetLastError();
	if (cudaMemcpy(d, seq.data(), rb + 64, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(d + o_read, reads, qb, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemset(d + o_read + qb, 0, 64) != cudaSuccess ||
	    cudaMemcpy(d_roff, ref_off, (n + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(d_qoff, read_off, (n + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemset(d_flags, 0, (size_t)n * 4) != cudaSuccess)
		rc = HERA_GPU_ECUDA;
	std::vector<int> hf((size_t)n), wide;
	std::vector<SswOut> h((size_t)n);
	std::vector<SswOutT<CapsWide>> hw;
	DevIndex ix{};
	ix.code = d + o_rcode;
	ix.seq = d;
	auto check = [&](const char *what, cudaError_t e) {
		if (e != cudaSuccess && rc == HERA_GPU_OK) {
			fprintf(stderr, "hera_gpu_unit_ssw: %s: %s\n", what, cudaGetErrorString(e));
			rc = HERA_GPU_ECUDA;
		}
	};
	if (rc == HERA_GPU_OK) {
		k_codes<<<64, 256>>>(d, d + o_rcode, rb + 64);
		k_codes<<<64, 256>>>(d + o_read, d + o_qcode, qb + 64);
		const int wpb = 4;
		const size_t per = ssw_smem_per_warp(max_len);
		check("shared-memory size",
		      cudaFuncSetAttribute(k_unit_ssw<CapsStd>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(wpb * per)));
		k_unit_ssw<CapsStd><<<(n + wpb - 1) / wpb, 32 * wpb, wpb * per>>>(ix, nullptr, d_roff, d + o_qcode, d_qoff, n,
										  d_out, (int)per, d_flags);
		check("launch", cudaGetLastError());
		check("run", cudaDeviceSynchronize());
		check("copy", cudaMemcpy(h.data(), d_out, n * sizeof(SswOut), cudaMemcpyDeviceToHost));
		check("copy", cudaMemcpy(hf.data(), d_flags, (size_t)n * 4, cudaMemcpyDeviceToHost));
		for (int i = 0; i < n; ++i)
			if (hf[i] & F_CAPS)
				wide.push_back(i);
	}
	if (rc == HERA_GPU_OK && !wide.empty()) {
		const int nw = (int)wide.size();
		const size_t per = ssw_smem_wide();
		hw.resize((size_t)nw);
		check("wide outputs", cudaMalloc(&d_wout, (size_t)nw * sizeof(SswOutT<CapsWide>)));
		if (rc == HERA_GPU_OK) {
			check("copy", cudaMemcpy(d_which, wide.data(), (size_t)nw * 4, cudaMemcpyHostToDevice));
			check("copy", cudaMemset(d_flags, 0, (size_t)nw * 4));
			check("shared-memory size",
			      cudaFuncSetAttribute(k_unit_ssw<CapsWide>, cudaFuncAttributeMaxDynamicSharedMemorySize,
						   (int)(WIDE_RESCUE_WPB * per)));
			k_unit_ssw<CapsWide><<<(nw + WIDE_RESCUE_WPB - 1) / WIDE_RESCUE_WPB, 32 * WIDE_RESCUE_WPB,
					       WIDE_RESCUE_WPB * per>>>(ix, d_which, d_roff, d + o_qcode, d_qoff, nw, d_wout,
									 (int)per, d_flags);
			check("launch", cudaGetLastError());
			check("run", cudaDeviceSynchronize());
			check("copy", cudaMemcpy(hw.data(), d_wout, (size_t)nw * sizeof(SswOutT<CapsWide>),
						 cudaMemcpyDeviceToHost));
			std::vector<int> wf((size_t)nw);
			check("copy", cudaMemcpy(wf.data(), d_flags, (size_t)nw * 4, cudaMemcpyDeviceToHost));
			for (int k = 0; k < nw; ++k)
				hf[wide[k]] = wf[k] ? (wf[k] | F_WIDE) : 0;
		}
	}
	if (rc == HERA_GPU_OK) {
		auto put = [&](int i, const auto &o) {
			score[i] = o.score;
			skip[i] = o.skip;
			n_ops[i] = o.cig.n;
			n_miss[i] = o.cig.nm;
			for (int k = 0; k < o.cig.n && k < cap; ++k)
				ops[(size_t)i * cap + k] = o.cig.op[k];
			for (int k = 0; k < o.cig.nm && k < cap; ++k)
				miss[(size_t)i * cap + k] = (char)o.cig.miss[k];
		};
		std::vector<int> wpos((size_t)n, -1);
		for (size_t k = 0; k < wide.size(); ++k)
			wpos[wide[k]] = (int)k;
		for (int i = 0; i < n; ++i) {
			if (wpos[i] >= 0)
				put(i, hw[wpos[i]]);
			else
				put(i, h[i]);
			*flags |= hf[i];
		}
	}
	if (d_wout)
		cudaFree(d_wout);
	cudaFree(d);
	return rc;
}

// ---- DPX throughput probe ----------------------------------------------
//
// Eight independent chains of packed 16x2 add-then-min per thread, on
// 8 resident blocks of 256 threads per SM: the instruction rate that bounds
// a DP cell update built from __viaddmin_s16x2.

namespace {
constexpr int DPX_CHAINS = 8;

__global__ void __launch_bounds__(256) k_dpx_peak(const unsigned *__restrict__ seed, int iters,
						   unsigned *__restrict__ out)
{
	const unsigned b = seed[32], c = seed[33];
	unsigned a[DPX_CHAINS];
#pragma unroll
	for (int k = 0; k < DPX_CHAINS; ++k)
		a[k] = seed[(threadIdx.x + k) & 31];
	for (int i = 0; i < iters; ++i) {
#pragma unroll
		for (int k = 0; k < DPX_CHAINS; ++k)
			a[k] = __viaddmin_s16x2(a[k], b, c ^ (unsigned)k);
	}
	unsigned x = 0;
#pragma unroll
	for (int k = 0; k < DPX_CHAINS; ++k)
		x ^= a[k];
	out[blockIdx.x * blockDim.x + threadIdx.x] = x;
}
}  // namespace

extern "C" int hera_gpu_dpx_peak(int device, float ms, double *instr_per_s)
{
	if (!instr_per_s || !(ms > 0))
		return HERA_GPU_EINVAL;
	*instr_per_s = 0;
	if (cudaSetDevice(device) != cudaSuccess)
		return HERA_GPU_ENODEV;
	int sms = 0;
	if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0)
		return HERA_GPU_ENODEV;
	const int tpb = 256, blocks = sms * 8;
	unsigned *d = nullptr;
	const size_t n_out = (size_t)blocks * tpb;
	if (cudaMalloc(&d, (n_out + 64) * sizeof(unsigned)) != cudaSuccess)
		return HERA_GPU_ENOMEM;
	unsigned *seed = d + n_out;
	unsigned h_seed[64];
	for (int i = 0; i < 64; ++i)
		h_seed[i] = 0x00070003u * (unsigned)(i + 1);
	h_seed[32] = 0x00010001u;   // +1 in both lanes
	h_seed[33] = 0x7f007f00u;
	cudaStream_t st = nullptr;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	int rc = HERA_GPU_OK;
	if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
	    cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
	    cudaMemcpyAsync(seed, h_seed, sizeof h_seed, cudaMemcpyHostToDevice, st) != cudaSuccess)
		rc = HERA_GPU_ECUDA;
	int iters = 1024;
	float t = 0;
	for (int pass = 0; pass < 3 && rc == HERA_GPU_OK; ++pass) {
		cudaEventRecord(e0, st);
		k_dpx_peak<<<blocks, tpb, 0, st>>>(seed, iters, d);
		cudaEventRecord(e1, st);
		if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
			rc = HERA_GPU_ECUDA;
			break;
		}
		cudaEventElapsedTime(&t, e0, e1);
		if (pass < 2) {   // scale the loop to the requested duration
			double f = t > 0 ? ms / t : 64.0;
			f = f < 0.5 ? 0.5 : (f > 64.0 ? 64.0 : f);
			double ni = iters * f;
			iters = ni > 1e8 ? 100000000 : (ni < 64 ? 64 : (int)ni);
		}
	}
	if (rc == HERA_GPU_OK && t > 0)
		*instr_per_s = (double)n_out * iters * DPX_CHAINS / (t * 1e-3);
	if (e0)
		cudaEventDestroy(e0);
	if (e1)
		cudaEventDestroy(e1);
	if (st)
		cudaStreamDestroy(st);
	cudaFree(d);
	return rc;
}

#include "hera_server.cuh"
#include "hera_fastq.cuh"
#include "hera_classes.cuh"
#include "hera_bam.cuh"
#include "hera_bgzf.cuh"
