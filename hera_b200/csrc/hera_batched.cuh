// hera_batched.cuh -- the batched form of get_position.
//
// In hera, one get_position call (src/hash_align.c:1322-1467) seeds the
// read, merges the hit lists into anchors, forms chains in up to three
// passes, and for every chain runs get_SWalign (:1242-1320): a prefix
// SW_align plus one SW_align per gap, with early exits and a keep / append /
// reset rule on the running best error.  The inputs of every SW_align call
// are fixed by the chain structure; only the bookkeeping around them is
// sequential.  So the batched form splits a round of get_position calls
// into:
//   k_build   per call: seeds, anchor merge, chain enumeration of all
//             passes, one DP job per SW_align the call could make;
//   k_bin_*   counting sort of the jobs by (error cap, gap length);
//   k_dp      one thread per job, neighbouring threads on equal-shaped DPs
//             (register form of SW_align);
//   k_replay  per call: the reference's pass / early-exit / keep rules
//             over the job results, then the kept chain's CIGAR.
// Pair-level control flow (k_resolve_b) requests get_position calls and
// mate rescues and suspends until the round that serves them has run.
#pragma once

// (included inside hera_gpu.cu's unnamed namespace, after Batch/RmReq)

constexpr int JCAP = 32;          // CIGAR ops kept per DP job (traceback mode)
constexpr int NBIN = 2 * (MAX_READ + 1);

struct GpReq {
	int32_t pair;
	int16_t c, str;
};

struct TaskInfo {
	int32_t chain0;
	int32_t nch;              // -1: no anchors (miss), -2: buffers overflowed
};

struct Chain {
	uint32_t t, tp, off;      // head anchor
	int32_t js0;              // first job slot (slots of a chain are contiguous)
	int16_t njs;              // job slots: prefix (if any) then one per gap
	int8_t pass;              // 0 mate-guided, 1 chains, 2 singletons
	int8_t viable;            // 0: get_SWalign returns before any DP
	int8_t has_prefix;
	int8_t pad[3];
};

struct JobSlot {              // one SW_align call of a chain
	int32_t job;              // the (deduplicated) DP job computing it
	uint16_t mrun;            // M run added before this gap (0 for the prefix)
	uint16_t pad;
};

struct DpJob {
	uint32_t rstart;          // reference window start (offset in seq)
	uint16_t ref_len, len;
	uint16_t qoff, pad0;      // query offset in the oriented read
	int8_t err, orient;
	int16_t pad;
	int32_t read;
};

struct DpResHdr {
	int16_t score, sub;
	uint8_t n, nm;
	uint8_t caps;             // 1: the CIGAR passed a capacity (the job's pairs go to the wide pass)
	uint8_t pad;
};

__host__ __device__ constexpr int res_stride(int cap)
{
	return (int)sizeof(DpResHdr) + 4 * cap + ((cap + 3) & ~3);
}

struct Round {
	const GpReq *req;         // null: round 0 (task t = pair t>>2, c (t>>1)&1, str t&1)
	const int *list;          // round 0: the tasks k_build runs (those with seed hits)
	const int *nlist;         // ... and their number (device)
	int ntask;
	int space;
	const uint2 *hits;        // precomputed seeds (round 0) or null
	int spr;
	const uint2 *thits;       // precomputed seeds per task (later rounds: k_seed_req) or null
	int tspr;
	TaskInfo *tinfo;
	Chain *chains;
	JobSlot *slots;
	DpJob *jobs;
	int *cnt;                 // [0] chains, [1] jobs, [2] job slots
	int chain_cap, job_cap, slot_cap;
	uint8_t *res;
	int rcap;                 // CIGAR ops per job result
};

// Anchors of the batched form, 8 bytes each: {transcript, position |
// read offset << 23}; one load per anchor.  Transcripts must be shorter
// than 2^23 bases (checked when the context is created).
constexpr int TP_BITS = 23;
constexpr uint32_t TP_MASK = (1u << TP_BITS) - 1;
struct __align__(8) PA {
	uint32_t t, w;
	__device__ __forceinline__ uint32_t tp() const { return w & TP_MASK; }
	__device__ __forceinline__ uint32_t off() const { return w >> TP_BITS; }
};
struct PAnchors {
	PA a[ACAP];
};
__device__ __forceinline__ PA pa_make(uint32_t t, uint32_t tp, uint32_t off)
{
	return PA{t, tp | (off << TP_BITS)};
}

// merge_sort / add_sort (src/hash_align.c:247-297) of a k-mer's occurrence
// list (read offset idx) into the anchors, as merge_hits does for the
// plain form
__device__ inline int merge_packed(const PAnchors &A, int na, PAnchors &B, const uint2 *occ, uint32_t nh,
				   uint32_t idx, int &flags)
{
	if (na + (int)nh > ACAP) {
		flags |= F_ACAP;
		nh = (uint32_t)(ACAP - na);
	}
	int i = 0, n = 0;
	uint32_t k = 0;
	uint2 h = nh ? __ldg(occ) : make_uint2(0, 0);
	PA a = na ? A.a[0] : PA{0, 0};
	while (i < na && k < nh) {
		bool take_a;
		if (a.t < h.x) {
			take_a = true;
		} else if (a.t > h.x) {
			take_a = false;
		} else {
			const uint32_t dis = (h.y - a.tp()) - (idx - a.off());
			take_a = dis < 2 * ERR ? true : !(a.tp() > h.y);
		}
		if (take_a) {
			B.a[n] = a;
			if (++i < na)
				a = A.a[i];
		} else {
			B.a[n] = pa_make(h.x, h.y, idx);
			if (++k < nh)
				h = __ldg(occ + k);
		}
		++n;
	}
	for (; i < na; ++i, ++n)
		B.a[n] = A.a[i];
	for (; k < nh; ++k, ++n) {
		h = __ldg(occ + k);
		B.a[n] = pa_make(h.x, h.y, idx);
	}
	return n;
}

// round 0: reset every pair's Candidate state and list the get_position
// calls that have at least one seed hit (the others take the miss exit).
// With `key`, every call gets its anchor count (the seeds' hits, capped at
// 255; 0 for a call with none) and `list` the identity, for a sort that
// hands the build its calls largest first, so that a warp's 32 calls are of
// like size; without, `list` holds the calls with hits in no set order.
__global__ void k_task_list(Batch b, int ntask, const uint2 *__restrict__ hits, int spr,
			    TaskInfo *__restrict__ tinfo, int *__restrict__ list, int *__restrict__ nlist,
			    uint8_t *__restrict__ key)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= ntask)
		return;
	const int pi = t >> 2, c = (t >> 1) & 1, str = t & 1;
	DPair &P = b.P[pi];
	DSlot &S = P.s[c][str];
	S.n = 0;
	S.err = 0;
	S.cig.n = S.cig.nm = 0;
	if (str == 0)
		P.pair[c] = 0;
	if ((t & 3) == 0) {
		P.stage = 0;
		P.rm_ret = 0;
		P.ovf = 0;
	}
	tinfo[t].chain0 = 0;
	tinfo[t].nch = -1;
	const int ri = 2 * pi + ((c ^ str) == 0 ? 0 : 1);
	const int L = b.len[ri];
	if (key) {
		key[t] = 0;
		list[t] = t;
	}
	if (L > b.max_len) {
		flag(b.flags, F_READ);
		return;
	}
	const uint2 *h = hits + ((int64_t)ri * 2 + str) * spr;
	uint32_t w = 0;
	for (int j = 0; j * KMER + KMER <= L; ++j)
		w += h[j].y;
	if (w == 0)
		return;
	if (key) {
		key[t] = (uint8_t)(w < 255 ? w : 255);
		atomicAdd(nlist, 1);
	} else {
		list[atomicAdd(nlist, 1)] = t;
	}
}

__device__ __forceinline__ void task_of(const Round &R, int t, int &pi, int &c, int &str)
{
	if (R.req) {
		pi = R.req[t].pair;
		c = R.req[t].c;
		str = R.req[t].str;
	} else {
		pi = t >> 2;
		c = (t >> 1) & 1;
		str = t & 1;
	}
}

// The seeds of a later round's get_position calls (space 2*ERR on the
// oriented read, :1322-1344), one thread per (call, seed): the hash
// lookups the build would make one after another, made side by side so
// that their latencies overlap.  A seed past the read's end, or a read
// longer than the batch's maximum, gets no hits (the build never reads it).
__global__ void __launch_bounds__(256) k_seed_req(Batch b, Round R, uint2 *__restrict__ thits)
{
	const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= (int64_t)R.ntask * R.tspr)
		return;
	const int t = (int)(idx / R.tspr), sj = (int)(idx % R.tspr);
	int pi, c, str;
	task_of(R, t, pi, c, str);
	const int ri = 2 * pi + ((c ^ str) == 0 ? 0 : 1);
	const int L = b.len[ri];
	const int i = sj * R.space;
	uint2 h = make_uint2(0, 0);
	if (L <= b.max_len && i + KMER <= L)
		h = probe(b.ix, kmer_words((str ? b.code_r : b.code) + b.off[ri] + i, false));
	thits[idx] = h;
}

__device__ __forceinline__ void prefetch_l2(const void *p)
{
	asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Enumerate the chains of one get_position call in the reference's order
// (pass A :1367-1390, pass B :1392-1412, pass C :1414-1434); pass A's
// consumed marks are kept in a bitmask so the walk can be repeated.
template <class Emit>
__device__ inline void enum_chains(const PAnchors &A, int na, const DSlot &Mt, int space, int rlen,
				   uint32_t *used, Emit emit)
{
	for (int w = 0; w < ACAP / 32; ++w)
		used[w] = 0;
	auto is_used = [&](uint32_t i) { return (used[i >> 5] >> (i & 31)) & 1u; };
	auto next = [&](uint32_t i, uint32_t n, bool stop_used) -> bool {
		if (i + 1 >= (uint32_t)na)
			return false;
		const PA a0 = A.a[i], a1 = A.a[i + 1];
		if (a0.t != a1.t)
			return false;
		// read offsets of used anchors read as rlen in the reference
		const uint32_t o0 = is_used(i) ? (uint32_t)rlen : a0.off();
		const uint32_t o1 = is_used(i + 1) ? (uint32_t)rlen : a1.off();
		if (!(o1 > o0))
			return false;
		const uint32_t tp1 = a1.tp(), tph = A.a[i + 1 - n].tp();
		if (!(tp1 > tph))
			return false;
		if (!(tp1 - tph < (uint32_t)rlen))
			return false;
		if (stop_used && o1 == (uint32_t)rlen)
			return false;
		return true;
	};
	// (the spacing first: at spacing 31 pass A never runs, and the mate's
	// slot, a random read of the pair state, is not touched)
	bool passA = space < KMER && space > 0 && Mt.n > 0;
	if (passA) {
		const uint32_t mn = (uint32_t)Mt.n;
		uint32_t k = 0;
		for (uint32_t i = 0; i < (uint32_t)na; ++i) {
			if (A.a[i].t < Mt.t[k])
				continue;
			while (k < mn && A.a[i].t > Mt.t[k])
				++k;
			if (k == mn)
				break;
			uint32_t n = 1;
			while (next(i, n, false)) {
				++i;
				++n;
			}
			emit(0, i + 1 - n, n);
			for (uint32_t q = i + 1 - n; q <= i; ++q)
				used[q >> 5] |= 1u << (q & 31);
		}
	}
	for (uint32_t i = 0; i < (uint32_t)na; ++i) {
		if (is_used(i) || A.a[i].off() == (uint32_t)rlen)
			continue;
		uint32_t n = 1;
		while (next(i, n, true)) {
			++i;
			++n;
		}
		if (n < 2 && rlen / KMER > 2)
			continue;
		emit(1, i - n + 1, n);
	}
	if (space < KMER) {
		for (uint32_t i = 0; i < (uint32_t)na; ++i) {
			if (is_used(i) || A.a[i].off() == (uint32_t)rlen)
				continue;
			uint32_t n = 1;
			while (next(i, n, true)) {
				++i;
				++n;
			}
			if (n >= 2)
				continue;
			emit(2, i, n);
		}
	}
}

constexpr int LCH = 128;       // chains of one get_position call
constexpr int LJS = 256;       // SW_align calls of one get_position call
constexpr int LJ = 256;        // distinct DP jobs of one get_position call

struct BuildWork {
	PAnchors a[2];
	uint32_t used[ACAP / 32];
	Chain ch[LCH];
	JobSlot js[LJS];
	DpJob jb[LJ];
	uint64_t jkey[LJ];   // a job's (query offset, lengths, error cap) in one word, for the dedup scan
};

// one get_position call of the round (list position t)
__device__ void build_one(const Batch &b, const Round &R, int t)
{
	if (R.list)
		t = R.list[t];
	int pi, c, str;
	task_of(R, t, pi, c, str);
	DPair &P = b.P[pi];
	const int ri = 2 * pi + ((c ^ str) == 0 ? 0 : 1);
	const int L = b.len[ri];
	int flags = 0;
	R.tinfo[t].chain0 = 0;
	R.tinfo[t].nch = -1;
	if (L > b.max_len) {
		flag(b.flags, F_READ);
		return;
	}
	const uint8_t *rd = (str ? b.code_r : b.code) + b.off[ri];
	const uint32_t step = (uint32_t)R.space;
	// the seeds' hits, when a kernel before this one looked them up
	const uint2 *pre = R.hits ? R.hits + ((int64_t)ri * 2 + str) * R.spr
				  : (R.thits ? R.thits + (int64_t)t * R.tspr : nullptr);
	if (pre) {   // their hit lists' first lines on their way to L2 before the merge
		int j = 0;
		for (uint32_t i = 0; i + KMER <= (uint32_t)L; i += step, ++j) {
			const uint2 h = pre[j];
			if (h.y)
				prefetch_l2(b.ix.occ + h.x);
		}
	}
	BuildWork w;
	int cur = 0, na = 0, sj = 0;
	for (uint32_t i = 0; i + KMER <= (uint32_t)L; i += step, ++sj) {
		uint2 h = pre ? pre[sj] : probe(b.ix, kmer_words(rd + i, false));
		if (h.y == 0)
			continue;
		const uint2 *occ = b.ix.occ + h.x;
		if (na == 0) {
			uint32_t nh = h.y;
			if (nh > (uint32_t)ACAP) {
				flags |= F_ACAP;
				nh = ACAP;
			}
			for (uint32_t k = 0; k < nh; ++k) {
				const uint2 o = __ldg(occ + k);
				w.a[cur].a[k] = pa_make(o.x, o.y, i);
			}
			na = (int)nh;
			continue;
		}
		na = merge_packed(w.a[cur], na, w.a[cur ^ 1], occ, h.y, i, flags);
		cur ^= 1;
	}
	if (na == 0) {
		pair_flags(b, pi, flags);
		flag(b.flags, flags);
		return;
	}
	const PAnchors &A = w.a[cur];
	const DSlot &Mt = P.s[c][1 - str];
	int nch = 0, ns = 0, nj = 0;
	// one SW_align call -> a job slot; identical calls (same query span,
	// caps and reference bytes) share one DP job
	auto add_job = [&](const DpJob &j, uint16_t mrun) {
		if (ns >= LJS) {
			flags |= F_ACAP;
			return;
		}
		const uint64_t key = (uint64_t)j.qoff | (uint64_t)j.len << 16 | (uint64_t)j.ref_len << 32 |
				     (uint64_t)(uint8_t)j.err << 48;
		int hit = -1;
		for (int q = 0; q < nj && hit < 0; ++q)
			if (w.jkey[q] == key && bytes_equal(b.ix.seq, w.jb[q].rstart, j.rstart, j.ref_len))
				hit = q;
		if (hit < 0) {
			if (nj >= LJ) {
				flags |= F_ACAP;
				return;
			}
			w.jb[nj] = j;
			w.jkey[nj] = key;
			hit = nj++;
		}
		w.js[ns].job = hit;
		w.js[ns].mrun = mrun;
		w.js[ns].pad = 0;
		++ns;
	};
	enum_chains(A, na, Mt, R.space, L, w.used, [&](int pass, uint32_t id, uint32_t n) {
		if (nch >= LCH) {
			flags |= F_ACAP;
			return;
		}
		Chain &ch = w.ch[nch++];
		ch.t = A.a[id].t;
		ch.tp = A.a[id].tp();
		ch.off = A.a[id].off();
		ch.pass = (int8_t)pass;
		ch.viable = 0;
		ch.has_prefix = 0;
		ch.js0 = ns;
		ch.njs = 0;
		// get_SWalign's early returns before any DP (:1250-1256)
		if (n > 1 && A.a[id + n - 1].tp() - A.a[id].tp() > (uint32_t)L)
			return;
		const int start = (int)(A.a[id].tp() - (A.a[id].off() + KMER - 1));
		if (start < 0 || (uint32_t)(start + L) > __ldg(b.ix.tlen + A.a[id].t))
			return;
		ch.viable = 1;
		const uint32_t add = start < ERR ? (uint32_t)start : (uint32_t)ERR;
		const uint32_t ref_start = __ldg(b.ix.tstart + A.a[id].t) + (uint32_t)start;
		DpJob j;
		j.orient = (int8_t)str;
		j.read = ri;
		j.pad = 0;
		j.pad0 = 0;
		const int ns0 = ns;
		if (A.a[id].off() > 0) {   // prefix DP on the reversed strings (:1262-1266)
			const uint32_t o0 = A.a[id].off();
			ch.has_prefix = 1;
			j.rstart = ref_start - add;
			j.ref_len = (uint16_t)(o0 + add);
			j.len = (uint16_t)o0;
			j.qoff = 0;
			j.err = (int8_t)(o0 < 2 * ERR ? -3 : -ERR);
			add_job(j, 0);
		}
		for (uint32_t i = 0; i < n; ++i) {   // merged runs and their gaps (:1282-1305)
			const uint32_t s0 = i;
			while (i + 1 < n && A.a[id + i].off() + KMER >= A.a[id + i + 1].off())
				++i;
			const uint32_t seg = A.a[id + i].off() + KMER;
			const uint32_t len = ((i + 1) < n ? A.a[id + i + 1].off() : (uint32_t)L) - seg;
			const uint32_t ad = (i + 1) < n ? 0u : (uint32_t)ERR;
			j.rstart = ref_start + seg;
			j.ref_len = (uint16_t)(len + ad);
			j.len = (uint16_t)len;
			j.qoff = (uint16_t)seg;
			j.err = (int8_t)(len < 2 * ERR ? 3 : ERR);
			add_job(j, (uint16_t)(A.a[id + i].off() - A.a[id + s0].off() + KMER));
		}
		ch.njs = (int16_t)(ns - ns0);
	});
	const int at = atomicAdd(R.cnt, nch);
	const int jt = atomicAdd(R.cnt + 1, nj);
	const int st = atomicAdd(R.cnt + 2, ns);
	if (at + nch > R.chain_cap || jt + nj > R.job_cap || st + ns > R.slot_cap) {
		R.tinfo[t].nch = -2;
		pair_flags(b, pi, flags);
		flag(b.flags, flags);
		return;
	}
	R.tinfo[t].chain0 = at;
	R.tinfo[t].nch = nch;
	for (int q = 0; q < nj; ++q)
		R.jobs[jt + q] = w.jb[q];
	for (int q = 0; q < ns; ++q) {
		JobSlot js = w.js[q];
		js.job += jt;
		R.slots[st + q] = js;
	}
	for (int q = 0; q < nch; ++q) {
		Chain ch = w.ch[q];
		ch.js0 += st;
		R.chains[at + q] = ch;
	}
	pair_flags(b, pi, flags);
	flag(b.flags, flags);
}

// Persistent work-queue form: a grid of a few blocks per SM (the residency
// the autotuner picked) whose warps take the round's calls 32 at a time
// from `queue`; a warp held up by a heavy call delays only its own 32.
__global__ void __launch_bounds__(128) k_build(Batch b, Round R, int *__restrict__ queue)
{
	const int n = R.list ? *R.nlist : R.ntask;
	const int lane = threadIdx.x & 31;
	for (;;) {
		int base = 0;
		if (lane == 0)
			base = atomicAdd(queue, 32);
		base = __shfl_sync(0xffffffffu, base, 0);
		if (base >= n)
			break;
		if (base + lane < n)
			build_one(b, R, base + lane);
	}
}

__device__ __forceinline__ int job_bin(const DpJob &j)
{
	const int e = j.err < 0 ? -j.err : j.err;
	return (e == 7 ? 1 : 0) * (MAX_READ + 1) + (j.len <= MAX_READ ? j.len : MAX_READ);
}

// histogram of job bins: per-block shared counts, one global atomic per bin
__global__ void k_bin_count(const DpJob *__restrict__ jobs, int n, int *__restrict__ hist)
{
	__shared__ int h[NBIN];
	for (int i = threadIdx.x; i < NBIN; i += blockDim.x)
		h[i] = 0;
	__syncthreads();
	for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
		atomicAdd(h + job_bin(jobs[t]), 1);
	__syncthreads();
	for (int i = threadIdx.x; i < NBIN; i += blockDim.x)
		if (h[i])
			atomicAdd(hist + i, h[i]);
}

// exclusive scan of the (small) histogram, one block
__global__ void k_bin_scan(int *__restrict__ hist, int nbin)
{
	__shared__ int part[1024];
	const int tid = threadIdx.x;
	const int per = (nbin + blockDim.x - 1) / blockDim.x;
	int s = 0;
	for (int i = tid * per; i < (tid + 1) * per && i < nbin; ++i)
		s += hist[i];
	part[tid] = s;
	__syncthreads();
	if (tid == 0) {
		int acc = 0;
		for (int i = 0; i < (int)blockDim.x; ++i) {
			const int v = part[i];
			part[i] = acc;
			acc += v;
		}
	}
	__syncthreads();
	int acc = part[tid];
	for (int i = tid * per; i < (tid + 1) * per && i < nbin; ++i) {
		const int v = hist[i];
		hist[i] = acc;
		acc += v;
	}
}

// scatter jobs into bin order: per-block shared counts reserve a range of
// each bin with one global atomic, then threads take slots in shared memory
__global__ void k_bin_scatter(const DpJob *__restrict__ jobs, int n, int *__restrict__ cursor,
			      int *__restrict__ perm)
{
	__shared__ int h[NBIN];
	__shared__ int base[NBIN];
	for (int i = threadIdx.x; i < NBIN; i += blockDim.x)
		h[i] = 0;
	__syncthreads();
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	int bin = -1, rank = 0;
	if (t < n) {
		bin = job_bin(jobs[t]);
		rank = atomicAdd(h + bin, 1);
	}
	__syncthreads();
	for (int i = threadIdx.x; i < NBIN; i += blockDim.x)
		if (h[i])
			base[i] = atomicAdd(cursor + i, h[i]);
	__syncthreads();
	if (t < n)
		perm[base[bin] + rank] = t;
}

__device__ inline void store_res(const DCig &cig, int score, uint8_t *o, int rcap, int &flags)
{
	DpResHdr h;
	int sub = 0;
	for (int k = 0; k < cig.n; ++k) {
		const int ty = op_type(cig.op[k]);
		if (ty == OP_I || ty == OP_S)
			sub += (int)op_cnt(cig.op[k]);
		else if (ty == OP_D)
			sub -= (int)op_cnt(cig.op[k]);
	}
	if (cig.n > rcap || cig.nm > rcap)
		flags |= F_CCAP;
	h.score = (int16_t)score;
	h.sub = (int16_t)sub;
	h.n = (uint8_t)(cig.n < rcap ? cig.n : rcap);
	h.nm = (uint8_t)(cig.nm < rcap ? cig.nm : rcap);
	h.caps = (flags & F_CAPS) ? 1 : 0;
	h.pad = 0;
	*reinterpret_cast<DpResHdr *>(o) = h;
	uint32_t *ops = reinterpret_cast<uint32_t *>(o + sizeof(DpResHdr));
	for (int k = 0; k < h.n; ++k)
		ops[k] = cig.op[k];
	uint8_t *miss = o + sizeof(DpResHdr) + 4 * rcap;
	for (int k = 0; k < h.nm; ++k)
		miss[k] = cig.miss[k];
}

// which kernel computes a job: the register form for the two live error
// caps (when no row-0 spill can occur), the general banded form otherwise
__device__ __forceinline__ int job_form(const DpJob &j)
{
	const int e = j.err < 0 ? -j.err : j.err;
	if (j.len == 0)
		return 0;
	if (e == 7 && j.ref_len >= 9)
		return 8;
	if (e == 3 && j.ref_len >= 5)
		return 4;
	return 0;
}

// one thread per job, jobs in (error cap, length) order; threads whose job
// is not of cap E leave at once (whole warps, the order is by cap).  The
// DP runs in the bit-plane form (sw_align_bits).  With traceback every row
// is kept (4 bits a slot, in local memory).  In the score-only mode (SUM)
// rows serve only the shrink loop of a DP that stops early (18% of the
// error-8 calls, nearly every warp holds one), so each row keeps the
// loop's 2-byte summary instead and the loop reads one summary a row.  (A
// score-only first pass keeping no rows, with the early stops run again,
// measured 40% slower on config-2s: the reruns redid most of the DP.)
template <int E, bool SUM>
__global__ void __launch_bounds__(128, 8)
k_dp_reg(Batch b, const DpJob *__restrict__ jobs, const int *__restrict__ perm, int n, uint8_t *__restrict__ res,
	 int rcap)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	uint32_t cells = 0;
	const int id = t < n ? perm[t] : 0;
	if (t < n && job_form(jobs[id]) == E) {
		const DpJob jb = jobs[id];
		typename DpRow<E, SUM>::T rows[MAX_DP_ROWS + 1];
		DCig cig;
		int flags = 0;
		cig.n = cig.nm = 0;
		const bool rev = jb.err < 0;
		const uint8_t *q = (jb.orient ? b.code_r : b.code) + b.off[jb.read] + jb.qoff;
		RefWin r{b.ix.code, b.ix.seq, jb.rstart, jb.ref_len, rev};
		QView qv{rev ? q + (jb.len - 1) : q, rev ? -1 : 1};
		const int score = sw_align_bits<E, SUM>(r, qv, jb.ref_len, jb.len, b.score_only != 0, cig, rows, flags,
							cells);
		store_res(cig, score, res + (size_t)id * res_stride(rcap), rcap, flags);
		flag(b.flags, flags & ~F_CAPS);   // capacity: in the result header, for k_replay
	}
	warp_stat(b.stats + ST_SW_CELLS, cells);
}

// the jobs outside the register form (empty gaps, spill cases)
__global__ void __launch_bounds__(128) k_dp_generic(Batch b, const DpJob *__restrict__ jobs, int n,
						    uint8_t *__restrict__ res, int rcap)
{
	const int id = blockIdx.x * blockDim.x + threadIdx.x;
	uint32_t cells = 0;
	if (id < n && job_form(jobs[id]) == 0) {
		const DpJob jb = jobs[id];
		SwWork sw;
		DCig cig;
		int flags = 0;
		cig.n = cig.nm = 0;
		int score = 0;
		if (jb.len > 0) {
			const uint8_t *q = (jb.orient ? b.code_r : b.code) + b.off[jb.read] + jb.qoff;
			score = sw_align(b.ix, jb.rstart, q, jb.ref_len, jb.len, jb.err, b.score_only != 0, cig, sw,
					 flags, &cells);
		}
		store_res(cig, score, res + (size_t)id * res_stride(rcap), rcap, flags);
		flag(b.flags, flags & ~F_CAPS);   // capacity: in the result header, for k_replay
	}
	warp_stat(b.stats + ST_SW_CELLS, cells);
}

__device__ inline void load_res_cig(const uint8_t *o, int rcap, DCig &c, int &flags)
{
	const DpResHdr h = *reinterpret_cast<const DpResHdr *>(o);
	if (h.caps)
		flags |= F_CCAP;
	const uint32_t *ops = reinterpret_cast<const uint32_t *>(o + sizeof(DpResHdr));
	const uint8_t *miss = o + sizeof(DpResHdr) + 4 * rcap;
	c.n = h.n;
	c.nm = h.nm;
	for (int k = 0; k < h.n; ++k)
		c.op[k] = ops[k];
	for (int k = 0; k < h.nm; ++k)
		c.miss[k] = miss[k];
}

// get_position's pass / early-exit / keep rules over the job results
__global__ void __launch_bounds__(128) k_replay(Batch b, Round R)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= R.ntask)
		return;
	int pi, c, str;
	task_of(R, t, pi, c, str);
	DPair &P = b.P[pi];
	DSlot &S = P.s[c][str];
	const int ri = 2 * pi + ((c ^ str) == 0 ? 0 : 1);
	const int L = b.len[ri];
	const TaskInfo ti = R.tinfo[t];
	if (ti.nch == -2)
		return;
	int flags = 0;
	uint32_t n1 = 0, max = 0;
	int keep = -1;
	const int stride = res_stride(R.rcap);
	for (int pass = 0; pass < 3 && ti.nch > 0; ++pass) {
		bool runs;
		if (pass == 0)
			runs = R.space < KMER && R.space > 0 && P.s[c][1 - str].n > 0;
		else if (pass == 1)
			runs = n1 == 0;
		else
			runs = n1 == 0 && R.space < KMER;
		if (!runs)
			continue;
		n1 = 0;
		max = (uint32_t)(L / 2);
		for (int q = 0; q < ti.nch; ++q) {
			const Chain ch = R.chains[ti.chain0 + q];
			if (ch.pass != pass || !ch.viable)
				continue;
			int err = 0, sub = 0, j = ch.js0;
			bool ok = true;
			if (ch.has_prefix) {
				const DpResHdr h = *reinterpret_cast<const DpResHdr *>(R.res + (size_t)R.slots[j].job * stride);
				if (h.caps)
					flags |= F_CCAP;
				err += h.score;
				if (err > L / 2 || (uint32_t)err > max)
					ok = false;
				sub = h.sub;
				++j;
			}
			for (; ok && j < ch.js0 + ch.njs; ++j) {
				const DpResHdr h = *reinterpret_cast<const DpResHdr *>(R.res + (size_t)R.slots[j].job * stride);
				if (h.caps)
					flags |= F_CCAP;
				err += h.score;
				if (err > L / 2 || (uint32_t)err > max + 1)
					ok = false;
			}
			if (!ok)
				continue;
			if (max == (uint32_t)(L / 2) || (uint32_t)err < max) {
				keep = ti.chain0 + q;
				n1 = 0;
				max = (uint32_t)err;
			}
			if (n1 < (uint32_t)LCAP) {
				S.t[n1] = ch.t;
				S.p[n1] = (int32_t)(ch.tp - (ch.off + KMER - 1) + (uint32_t)sub);
			} else {
				flags |= F_LCAP;
			}
			++n1;
		}
	}
	if (n1 == 0) {   // miss exit (src/hash_align.c:1461-1466)
		S.n = 0;
		S.err = L;
		pair_flags(b, pi, flags);
		flag(b.flags, flags);
		return;
	}
	S.n = (int32_t)(n1 < (uint32_t)LCAP ? n1 : (uint32_t)LCAP);
	S.err = (int32_t)max;
	// the kept chain's CIGAR: prefix DP, then an M run and the gap DP per
	// segment (get_SWalign :1262-1305)
	DCig cig, tmp;
	const Chain ch = R.chains[keep];
	int j = ch.js0;
	cig.n = cig.nm = 0;
	if (ch.has_prefix) {
		load_res_cig(R.res + (size_t)R.slots[j].job * stride, R.rcap, cig, flags);
		++j;
	}
	for (; j < ch.js0 + ch.njs; ++j) {
		const JobSlot js = R.slots[j];
		cig_add(cig, OP_M, js.mrun, nullptr, flags);
		load_res_cig(R.res + (size_t)js.job * stride, R.rcap, tmp, flags);
		cig_concat(cig, tmp, flags);
	}
	cig_copy(S.cig, cig);
	pair_flags(b, pi, flags);
	flag(b.flags, flags);
}

// pair control flow of the batched form: the same decisions as k_resolve,
// but every get_position at spacing 14 is requested (GpReq) like a rescue
__global__ void __launch_bounds__(128) k_resolve_b(Batch b, const GpReq *__restrict__ res_g, int ng,
						    const RmReq *__restrict__ res_r, int nr, int all,
						    GpReq *__restrict__ qg, int *__restrict__ qng,
						    RmReq *__restrict__ qr, int *__restrict__ qnr)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= ng + nr)
		return;
	const int pi = all ? t : (t < ng ? res_g[t].pair : res_r[t - ng].pair);
	DPair &P = b.P[pi];
	auto gp = [&](int c, int str, int next) {
		const int k = atomicAdd(qng, 1);
		qg[k].pair = pi;
		qg[k].c = (int16_t)c;
		qg[k].str = (int16_t)str;
		P.stage = next;
	};
	auto rm = [&](int c, int str, int next) {
		const int k = atomicAdd(qnr, 1);
		qr[k].pair = pi;
		qr[k].c = (int16_t)c;
		qr[k].str = (int16_t)str;
		P.stage = next;
	};
	if (b.len[2 * pi] > b.max_len || b.len[2 * pi + 1] > b.max_len) {
		P.stage = 8;
		return;
	}
	int st = P.stage;
	for (;;) {
		switch (st) {
		case 0:   // retry r[0] at spacing 14 (:1672-1676)
			if (P.s[0][0].n == 0 && P.s[0][1].n == 0 && P.s[1][0].err + P.s[1][1].err > ERR) {
				gp(0, 0, 100);
				return;
			}
			st = 1;
			break;
		case 100:
			gp(0, 1, 101);
			return;
		case 101:
			st = 1;
			break;
		case 1:   // retry r[1] (:1677-1681)
			if (P.s[1][0].n == 0 && P.s[1][1].n == 0 && P.s[0][0].err + P.s[0][1].err > ERR) {
				gp(1, 1, 110);
				return;
			}
			st = 2;
			break;
		case 110:
			gp(1, 0, 111);
			return;
		case 111:
			st = 2;
			break;
		case 2: case 3: case 4: case 5: {   // get_position2 x4 (:1683-1694)
			const int c = (st - 2) >> 1, s = (st - 2) & 1;
			const DSlot &X = P.s[c][s], &Y = P.s[c][1 - s];
			const DSlot &O0 = P.s[1 - c][0], &O1 = P.s[1 - c][1];
			if (X.n == 0 && Y.n > 0 && Y.err < ERR && O0.err + O1.err > ERR) {
				gp(c, s, 200 + st);
				return;
			}
			st = st + 1;
			break;
		}
		case 202: case 203: case 204: case 205: {
			const int k = st - 200, c = (k - 2) >> 1, s = (k - 2) & 1;
			if (P.s[c][s].n == 0) {
				rm(c, s, 210 + k);
				return;
			}
			st = k + 1;
			break;
		}
		case 212: case 213: case 214: case 215:
			st = st - 210 + 1;
			break;
		case 6: case 7: {   // intersect2 (:1730-1733)
			const int c = st - 6;
			if (P.s[c][0].n > 0 && P.s[c][1].n > 0) {
				if (intersect_lists(P, c, MAX_FRAG) == 0 && intersect_lists(P, c, 0) == 0) {
					const int i = P.s[c][0].err < P.s[c][1].err ? 1 : 0;   // re_map
					P.rm_i = i;
					rm(c, i, 20 + 2 * c);
					return;
				}
			}
			st = st + 1;
			break;
		}
		case 20: case 22: {
			const int c = (st - 20) >> 1;
			if (P.rm_ret == 0) {
				rm(c, 1 - P.rm_i, st + 1);
				return;
			}
			P.pair[c] = 2;
			st = 7 + c;
			break;
		}
		case 21: case 23: {
			const int c = (st - 21) >> 1;
			if (P.rm_ret > 0)
				P.pair[c] = 2;
			st = 7 + c;
			break;
		}
		default:
			P.stage = 8;
			return;
		}
	}
}

