// hera_classes.cuh -- equivalence classes on the device: the add_class calls
// of hera's host tail (src/hash_align.c:1564-1602), applied to the flat
// records in input order.
//
// A read pair (or single read) that the tail hands to add_class either
// counts towards one transcript (a one-entry list: REF_INF->count), or, when
// its errors sum below ERR, towards the class whose key is XXH32 of its
// transcript list.  hera numbers classes by first insertion and compares
// classes by that 32-bit id only.  On the device a batch runs as:
//   k_cls_items  thread per item: the tail's branch (:1735-1760 for pairs,
//                :1825-1851 for single reads), PAIRED / MEAN_FRAG sums,
//                REF_INF->count, XXH32, and the id's slot in an
//                open-addressing table (atomicCAS on the key; a class made
//                by an earlier batch takes its count at once, a new id
//                records the smallest item index that holds it);
//   k_cls_mark   the item that first holds a new id marks (1, list length);
//   scan         exclusive sum of the marks: each new class's number and
//                list offset, in item order = the reference's insertion order;
//   k_cls_assign the new classes' ids, counts and lists;
//   k_cls_commit class and list totals.
// Identical to the sequential add_class for any split of the input into
// batches, because a class made by an earlier batch is numbered before any
// made by a later one.

namespace cls {

constexpr uint32_t P1 = 2654435761u, P2 = 2246822519u, P3 = 3266489917u, P4 = 668265263u,
		   P5 = 374761393u;
constexpr uint32_t NONE = 0xffffffffu;
constexpr uint64_t OFF_MASK = (1ull << 40) - 1;
constexpr int ERR_CAP = 7;   // ERR, src/hash_align.h:36

// flag bits
constexpr uint32_t F_TX = 1;      // a one-entry list names no transcript of the index
constexpr uint32_t F_MAP = 2;     // the id table is full
constexpr uint32_t F_CAP = 4;     // more classes or list entries than the table holds

struct State {
	uint32_t n_classes;
	uint32_t flags;
	unsigned long long ref_used;
	unsigned long long paired;
	unsigned long long frag;
};

struct Table {
	unsigned long long *keys;     // id + 1, 0 = empty
	uint32_t *cls_of;             // class number + 1, 0 = not numbered yet
	uint32_t *first;              // smallest item index holding a new id
	uint32_t *pend;               // items of a new id in the current batch
	uint32_t mask;                // slots - 1
	uint32_t *id;                 // per class
	unsigned long long *count;
	uint32_t *n;
	unsigned long long *ref_off;
	uint32_t *ref;
	uint32_t max_classes;
	unsigned long long ref_cap;
	uint32_t *tx_count;
	uint32_t n_trans;
	State *st;
};

// The add_class call an item makes, if any: list 0 of the Candidate it is
// given is a[0..na) ++ b[0..nb).
struct Call {
	const uint32_t *a, *b;
	uint32_t na, nb;
	int err_sum;
	int pair;            // add_class's `pair` argument (1 for read pairs)
	int32_t p00, p10;    // p[0][0], p[1][0] after the list merges
	bool on;
};

// lbase: the pool offset the records' list_off values start from.
__device__ __forceinline__ Call decide(const hera_cand_rec *recs, const uint32_t *pos, const int32_t *pp,
				       int64_t i, int paired, uint32_t lbase)
{
	pos -= lbase;
	pp -= lbase;
	Call c{};
	c.on = false;
	if (paired) {
		const hera_cand_rec a = recs[2 * i], b = recs[2 * i + 1];
		int pa = a.pair, pb = b.pair;
		const int sa = a.err[0] + a.err[1], sb = b.err[0] + b.err[1];
		if (sa < sb)
			pb = -1;
		else if (sa > sb)
			pa = -1;
		const hera_cand_rec *r = nullptr, *m = nullptr;
		if (pa > 1 && pb > 1) {
			if ((pa & 1) + (pb & 1) == 0) {   // concate_candidate(r[0], r[1])
				r = &recs[2 * i];
				m = &recs[2 * i + 1];
			}
		} else if (pa > 1) {
			if ((pa & 1) == 0)
				r = &recs[2 * i];
		} else if (pb > 1) {
			if ((pb & 1) == 0)
				r = &recs[2 * i + 1];
		}
		if (!r)
			return c;
		const hera_cand_rec R = *r;
		c.on = true;
		c.pair = 1;
		c.a = pos + R.list_off[0];
		c.na = (uint32_t)R.n[0];
		c.b = m ? pos + m->list_off[0] : nullptr;
		c.nb = m ? (uint32_t)m->n[0] : 0;
		c.err_sum = R.err[0] + R.err[1];
		c.p00 = c.na ? pp[R.list_off[0]] : (c.nb ? pp[m->list_off[0]] : 0);
		c.p10 = R.n[1] ? pp[R.list_off[1]] : (m && m->n[1] ? pp[m->list_off[1]] : 0);
		return c;
	}
	const hera_cand_rec R = recs[i];
	if (R.n[0] == 0 && R.n[1] == 0)
		return c;
	c.on = true;
	c.pair = 0;
	c.err_sum = R.err[0] + R.err[1];
	c.p00 = c.p10 = 0;
	c.b = nullptr;
	c.nb = 0;
	if (R.err[0] > R.err[1]) {            // move_candidate(r, 0, 1)
		c.a = pos + R.list_off[1];
		c.na = (uint32_t)R.n[1];
	} else {
		c.a = pos + R.list_off[0];
		c.na = (uint32_t)R.n[0];
		if (R.err[0] == R.err[1]) {   // list 1 appended to list 0
			c.b = pos + R.list_off[1];
			c.nb = (uint32_t)R.n[1];
		}
	}
	return c;
}

__device__ __forceinline__ uint32_t word(const Call &c, uint32_t k)
{
	return k < c.na ? c.a[k] : c.b[k - c.na];
}

__device__ __forceinline__ uint32_t rnd(uint32_t acc, uint32_t in)
{
	return __funnelshift_l(acc + in * P2, acc + in * P2, 13) * P1;
}

__device__ __forceinline__ uint32_t rotl(uint32_t x, int r)
{
	return __funnelshift_l(x, x, r);
}

// XXH32 with seed 0 over the list's bytes (4 per entry, little-endian), the
// published xxHash 32-bit algorithm; hera calls its vendored copy
// (src/xxhash.c) at src/hash_align.c:1576.
__device__ uint32_t xxh32_list(const Call &c)
{
	const uint32_t nw = c.na + c.nb;
	const uint32_t len = nw * 4;
	uint32_t h, k = 0;
	if (len >= 16) {
		uint32_t v1 = P1 + P2, v2 = P2, v3 = 0, v4 = 0u - P1;
		for (; k + 4 <= nw; k += 4) {
			v1 = rnd(v1, word(c, k));
			v2 = rnd(v2, word(c, k + 1));
			v3 = rnd(v3, word(c, k + 2));
			v4 = rnd(v4, word(c, k + 3));
		}
		h = rotl(v1, 1) + rotl(v2, 7) + rotl(v3, 12) + rotl(v4, 18);
	} else {
		h = P5;
	}
	h += len;
	for (; k < nw; ++k)
		h = rotl(h + word(c, k) * P3, 17) * P4;
	h ^= h >> 15;
	h *= P2;
	h ^= h >> 13;
	h *= P3;
	h ^= h >> 16;
	return h;
}

// Pass 1.  slot[i] = the id's table slot for an item that adds to a class,
// NONE otherwise; ids[i], nl[i] = its id and list length.
__global__ void k_cls_items(const hera_cand_rec *recs, const uint32_t *pos, const int32_t *pp, int64_t n,
			    int paired, uint32_t lbase, uint32_t base, Table T, uint32_t *slot, uint32_t *ids,
			    uint32_t *nl)
{
	const int64_t stride = (int64_t)gridDim.x * blockDim.x;
	const int64_t end = (n + 31) / 32 * 32;
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < end; i += stride) {
		unsigned long long frag = 0;
		uint32_t called = 0;
		uint32_t at = NONE, k = 0, tx = NONE;   // id slot, its class + 1; one-entry transcript
		if (i < n) {
			const Call c = decide(recs, pos, pp, i, paired, lbase);
			if (c.on) {
				called = 1;
				if (c.pair == 1) {
					const int32_t d = c.p00 - c.p10;
					frag = (unsigned long long)(d < 0 ? -(int64_t)d : (int64_t)d);
				}
				const uint32_t nw = c.na + c.nb;
				if (nw == 1) {
					const uint32_t t = c.na ? c.a[0] : c.b[0];
					if (t < T.n_trans)
						tx = t;
					else
						atomicOr(&T.st->flags, F_TX);
				} else if (c.err_sum < ERR_CAP) {
					const uint32_t id = xxh32_list(c);
					const unsigned long long key = (unsigned long long)id + 1;
					uint32_t a = id & T.mask;
					bool got = false;
					// a key already in place is read, not CASed: common
					// classes are read by many threads at once
					for (uint32_t probe = 0; probe <= T.mask; ++probe) {
						unsigned long long cur = *(volatile unsigned long long *)&T.keys[a];
						if (cur == 0ull)
							cur = atomicCAS(&T.keys[a], 0ull, key);
						if (cur == 0ull || cur == key) {
							got = true;
							break;
						}
						a = (a + 1) & T.mask;
					}
					if (!got) {
						atomicOr(&T.st->flags, F_MAP);
					} else {
						at = a;
						k = T.cls_of[a];
					}
					ids[i] = id;
					nl[i] = nw;
				}
			}
			slot[i] = (at != NONE && k == 0) ? at : NONE;
		}
		// one atomic per distinct slot (and transcript) in the warp: lanes
		// holding the same one combine, the lowest lane -- the smallest
		// item index of the group -- adds for all of them
		const uint32_t lane = threadIdx.x & 31;
		const unsigned g = __match_any_sync(0xffffffffu, at);
		if (at != NONE && lane == (uint32_t)(__ffs(g) - 1)) {
			if (k) {
				atomicAdd(&T.count[k - 1], (unsigned long long)__popc(g));
			} else {
				atomicMin(&T.first[at], base + (uint32_t)i);
				atomicAdd(&T.pend[at], (uint32_t)__popc(g));
			}
		}
		const unsigned gt = __match_any_sync(0xffffffffu, tx);
		if (tx != NONE && lane == (uint32_t)(__ffs(gt) - 1))
			atomicAdd(&T.tx_count[tx], (uint32_t)__popc(gt));
		// PAIRED and MEAN_FRAG's sum: one atomic a warp
		for (int o = 16; o; o >>= 1)
			frag += __shfl_down_sync(0xffffffffu, frag, o);
		called = __reduce_add_sync(0xffffffffu, called);
		if ((threadIdx.x & 31) == 0 && (called || frag)) {
			atomicAdd(&T.st->paired, (unsigned long long)called);
			atomicAdd(&T.st->frag, frag);
		}
	}
}

// Pass 2.  mark[i] = (1 << 40) | list length for the first item of a new id.
__global__ void k_cls_mark(int64_t n, uint32_t base, Table T, const uint32_t *slot, const uint32_t *nl,
			   unsigned long long *mark)
{
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i > n)
		return;
	unsigned long long v = 0;
	if (i < n) {
		const uint32_t s = slot[i];
		if (s != NONE && T.first[s] == base + (uint32_t)i)
			v = (1ull << 40) | nl[i];
	}
	mark[i] = v;
}

// Pass 3.  Number the new classes in item order and copy their lists.
__global__ void k_cls_assign(const hera_cand_rec *recs, const uint32_t *pos, const int32_t *pp, int64_t n,
			     int paired, uint32_t lbase, Table T, const uint32_t *slot, const uint32_t *ids,
			     const unsigned long long *mark, const unsigned long long *xs)
{
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n || !mark[i])
		return;
	const uint32_t s = slot[i];
	const uint64_t k = (uint64_t)T.st->n_classes + (xs[i] >> 40);
	const unsigned long long r = T.st->ref_used + (xs[i] & OFF_MASK);
	const uint32_t nw = (uint32_t)(mark[i] & OFF_MASK);
	if (k >= T.max_classes || r + nw > T.ref_cap) {
		atomicOr(&T.st->flags, F_CAP);
		return;
	}
	T.cls_of[s] = (uint32_t)k + 1;
	T.id[k] = ids[i];
	T.count[k] = T.pend[s];
	T.n[k] = nw;
	T.ref_off[k] = r;
	const Call c = decide(recs, pos, pp, i, paired, lbase);
	for (uint32_t j = 0; j < nw; ++j)
		T.ref[r + j] = word(c, j);
}

__global__ void k_cls_commit(Table T, const unsigned long long *xs, int64_t n)
{
	const unsigned long long t = xs[n];
	const uint64_t nc = (uint64_t)T.st->n_classes + (t >> 40);
	const unsigned long long nr = T.st->ref_used + (t & OFF_MASK);
	if (nc > T.max_classes || nr > T.ref_cap) {   // sizes stay within the arrays
		atomicOr(&T.st->flags, F_CAP);
		return;
	}
	T.st->n_classes = (uint32_t)nc;
	T.st->ref_used = nr;
}

}   // namespace cls

struct hera_gpu_classes {
	int device = 0;
	cudaStream_t stream = nullptr;
	cls::Table T{};
	uint32_t slots = 0;
	uint32_t items_done = 0;         // items added so far (first-insertion keys)
	bool broken = false;
	DBuf<uint32_t> slot, ids, nl;
	DBuf<unsigned long long> mark, xs;
	DBuf<uint8_t> cub_tmp;
	DBuf<hera_cand_rec> in_recs;     // hera_gpu_classes_add_host's copies
	DBuf<uint32_t> in_pos;
	DBuf<int32_t> in_p;
	cudaEvent_t ev0 = nullptr, ev1 = nullptr;
	float kernel_ms = 0;
	uint32_t launches = 0;
	bool timed = false;              // ev0 recorded for the current add call
	std::string err = "no error";
	std::vector<void *> owned;
};

static int cls_fail(hera_gpu_classes *c, int code, const char *what, cudaError_t e = cudaSuccess)
{
	return set_err(c->err, code, what, e);
}

extern "C" void hera_gpu_classes_destroy(hera_gpu_classes *c)
{
	if (!c)
		return;
	cudaSetDevice(c->device);
	if (c->stream)
		cudaStreamSynchronize(c->stream);
	for (void *p : c->owned)
		cudaFree(p);
	c->slot.release(); c->ids.release(); c->nl.release(); c->mark.release(); c->xs.release();
	c->cub_tmp.release();
	c->in_recs.release(); c->in_pos.release(); c->in_p.release();
	if (c->ev0)
		cudaEventDestroy(c->ev0);
	if (c->ev1)
		cudaEventDestroy(c->ev1);
	if (c->stream)
		cudaStreamDestroy(c->stream);
	delete c;
}

extern "C" int hera_gpu_classes_create(hera_gpu_ctx *ctx, uint32_t max_classes, uint64_t max_list,
				       hera_gpu_classes **out)
{
	if (!ctx || !out || max_classes == 0 || max_classes > (1u << 30) || max_list == 0 ||
	    max_list > cls::OFF_MASK)
		return fail(ctx, HERA_GPU_EINVAL, "bad argument");
	*out = nullptr;
	if (cudaSetDevice(ctx->device) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENODEV, "cudaSetDevice");
	auto *c = new hera_gpu_classes;
	c->device = ctx->device;
	uint32_t slots = 1024;
	while (slots < 2 * max_classes)
		slots *= 2;
	c->slots = slots;
	auto grab = [&](void **p, size_t bytes) {
		cudaError_t e = cudaMalloc(p, bytes);
		if (e == cudaSuccess)
			c->owned.push_back(*p);
		return e;
	};
	cls::Table &T = c->T;
	T.mask = slots - 1;
	T.max_classes = max_classes;
	T.ref_cap = max_list;
	T.n_trans = ctx->ix.n_trans;
	cudaError_t e = cudaSuccess;
	if ((e = grab((void **)&T.keys, (size_t)slots * 8)) != cudaSuccess ||
	    (e = grab((void **)&T.cls_of, (size_t)slots * 4)) != cudaSuccess ||
	    (e = grab((void **)&T.first, (size_t)slots * 4)) != cudaSuccess ||
	    (e = grab((void **)&T.pend, (size_t)slots * 4)) != cudaSuccess ||
	    (e = grab((void **)&T.id, (size_t)max_classes * 4)) != cudaSuccess ||
	    (e = grab((void **)&T.count, (size_t)max_classes * 8)) != cudaSuccess ||
	    (e = grab((void **)&T.n, (size_t)max_classes * 4)) != cudaSuccess ||
	    (e = grab((void **)&T.ref_off, (size_t)max_classes * 8)) != cudaSuccess ||
	    (e = grab((void **)&T.ref, (size_t)max_list * 4)) != cudaSuccess ||
	    (e = grab((void **)&T.tx_count, (size_t)(T.n_trans ? T.n_trans : 1) * 4)) != cudaSuccess ||
	    (e = grab((void **)&T.st, sizeof(cls::State))) != cudaSuccess) {
		hera_gpu_classes_destroy(c);
		return fail(ctx, HERA_GPU_ENOMEM, "class table", e);
	}
	if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
	    (e = cudaEventCreate(&c->ev0)) != cudaSuccess || (e = cudaEventCreate(&c->ev1)) != cudaSuccess) {
		hera_gpu_classes_destroy(c);
		return fail(ctx, HERA_GPU_ECUDA, "class table stream", e);
	}
	cudaMemsetAsync(T.keys, 0, (size_t)slots * 8, c->stream);
	cudaMemsetAsync(T.cls_of, 0, (size_t)slots * 4, c->stream);
	cudaMemsetAsync(T.first, 0xff, (size_t)slots * 4, c->stream);
	cudaMemsetAsync(T.pend, 0, (size_t)slots * 4, c->stream);
	cudaMemsetAsync(T.tx_count, 0, (size_t)(T.n_trans ? T.n_trans : 1) * 4, c->stream);
	cudaMemsetAsync(T.st, 0, sizeof(cls::State), c->stream);
	if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) {
		hera_gpu_classes_destroy(c);
		return fail(ctx, HERA_GPU_ECUDA, "class table init", e);
	}
	*out = c;
	return HERA_GPU_OK;
}

// One batch of records (device pointers) on the table's stream.
static int cls_add_part(hera_gpu_classes *c, const hera_cand_rec *recs, const uint32_t *pos, const int32_t *pp,
			int64_t n, int paired, uint32_t lbase)
{
	if (n <= 0)
		return HERA_GPU_OK;
	if ((uint64_t)c->items_done + (uint64_t)n >= (uint64_t)cls::NONE)
		return cls_fail(c, HERA_GPU_ECAPACITY, "more than 2^32 - 1 items on one class table");
	cudaError_t e;
	if ((e = c->slot.ensure(n)) != cudaSuccess || (e = c->ids.ensure(n)) != cudaSuccess ||
	    (e = c->nl.ensure(n)) != cudaSuccess || (e = c->mark.ensure(n + 1)) != cudaSuccess ||
	    (e = c->xs.ensure(n + 1)) != cudaSuccess)
		return cls_fail(c, HERA_GPU_ENOMEM, "class scratch", e);
	size_t tmp = 0;
	cub::DeviceScan::ExclusiveSum(nullptr, tmp, c->mark.p, c->xs.p, n + 1, c->stream);
	if ((e = c->cub_tmp.ensure(tmp + 16)) != cudaSuccess)
		return cls_fail(c, HERA_GPU_ENOMEM, "class scan", e);
	const cudaStream_t st = c->stream;
	if (!c->timed) {   // the device time of an add call starts after its allocations
		cudaEventRecord(c->ev0, st);
		c->timed = true;
	}
	const uint32_t base = c->items_done;
	const int sms = 148;
	const unsigned g1 = (unsigned)std::min<int64_t>(blocks_for(n, 256), (int64_t)sms * 8);
	cls::k_cls_items<<<g1, 256, 0, st>>>(recs, pos, pp, n, paired, lbase, base, c->T, c->slot.p, c->ids.p, c->nl.p);
	cls::k_cls_mark<<<blocks_for(n + 1, 256), 256, 0, st>>>(n, base, c->T, c->slot.p, c->nl.p, c->mark.p);
	cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tmp, c->mark.p, c->xs.p, n + 1, st);
	cls::k_cls_assign<<<blocks_for(n, 256), 256, 0, st>>>(recs, pos, pp, n, paired, lbase, c->T, c->slot.p, c->ids.p,
							       c->mark.p, c->xs.p);
	cls::k_cls_commit<<<1, 1, 0, st>>>(c->T, c->xs.p, n);
	c->launches += 5;
	c->items_done += (uint32_t)n;
	if ((e = cudaGetLastError()) != cudaSuccess)
		return cls_fail(c, HERA_GPU_ECUDA, "class kernels", e);
	return HERA_GPU_OK;
}

// Reads the table's flags; a set flag leaves the table unusable.
static int cls_check(hera_gpu_classes *c)
{
	cls::State s{};
	cudaError_t e = cudaMemcpyAsync(&s, c->T.st, sizeof s, cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(c->stream);
	if (e != cudaSuccess)
		return cls_fail(c, HERA_GPU_ECUDA, "class table state", e);
	if (s.flags) {
		c->broken = true;
		if (s.flags & cls::F_TX)
			return cls_fail(c, HERA_GPU_EINVAL, "a one-entry hit list names no transcript of the index");
		return cls_fail(c, HERA_GPU_ECAPACITY, "class table full (max_classes / max_list)");
	}
	return HERA_GPU_OK;
}

static int cls_begin(hera_gpu_classes *c)
{
	if (c->broken)
		return cls_fail(c, HERA_GPU_ECAPACITY, "class table overflowed earlier");
	if (cudaSetDevice(c->device) != cudaSuccess)
		return cls_fail(c, HERA_GPU_ENODEV, "cudaSetDevice");
	c->launches = 0;
	c->timed = false;
	c->kernel_ms = 0;
	return HERA_GPU_OK;
}

static int cls_end(hera_gpu_classes *c, int rc)
{
	cudaEventRecord(c->ev1, c->stream);
	if (rc != HERA_GPU_OK)
		return rc;
	rc = cls_check(c);
	if (rc == HERA_GPU_OK && c->timed)
		cudaEventElapsedTime(&c->kernel_ms, c->ev0, c->ev1);
	return rc;
}

extern "C" int hera_gpu_classes_add_last(hera_gpu_classes *c, hera_gpu_ctx *ctx)
{
	if (!c || !ctx || ctx->device != c->device)
		return c ? cls_fail(c, HERA_GPU_EINVAL, "bad argument") : HERA_GPU_EINVAL;
	int rc = cls_begin(c);
	if (rc)
		return rc;
	for (int k = 0; k < ctx->nparts && rc == HERA_GPU_OK; ++k) {
		Lane &L = *ctx->lanes[k];
		cudaEventRecord(L.ev[5], L.stream);
		cudaStreamWaitEvent(c->stream, L.ev[5], 0);
		rc = cls_add_part(c, L.recs.p, L.pos_pool.p, L.p_pool.p, L.items / 2, 1, L.rb_l);
	}
	return cls_end(c, rc);
}

extern "C" int hera_gpu_classes_add_device(hera_gpu_classes *c, const hera_cand_rec *d_recs,
					   const uint32_t *d_pos_pool, const int32_t *d_p_pool, int32_t n,
					   int paired, void *stream)
{
	if (!c)
		return HERA_GPU_EINVAL;
	if (n < 0 || (n > 0 && (!d_recs || !d_pos_pool || !d_p_pool)) || (paired != 0 && paired != 1))
		return cls_fail(c, HERA_GPU_EINVAL, "bad argument");
	int rc = cls_begin(c);
	if (rc)
		return rc;
	if (stream) {   // order after the caller's work that wrote the records
		cudaEventRecord(c->ev1, (cudaStream_t)stream);
		cudaStreamWaitEvent(c->stream, c->ev1, 0);
	}
	rc = cls_add_part(c, d_recs, d_pos_pool, d_p_pool, n, paired, 0);
	return cls_end(c, rc);
}

extern "C" int hera_gpu_classes_add_host(hera_gpu_classes *c, const hera_gpu_result *res, int32_t n,
					 int paired)
{
	if (!c)
		return HERA_GPU_EINVAL;
	if (!res || n < 0 || (paired != 0 && paired != 1) || (n > 0 && !res->recs) ||
	    (res->list_used > 0 && (!res->pos_pool || !res->p_pool)))
		return cls_fail(c, HERA_GPU_EINVAL, "bad argument");
	int rc = cls_begin(c);
	if (rc)
		return rc;
	const size_t nr = (size_t)n * (paired ? 2 : 1);
	const size_t nl = (size_t)res->list_used;
	cudaError_t e;
	if ((e = c->in_recs.ensure(nr + 1)) != cudaSuccess || (e = c->in_pos.ensure(nl + 1)) != cudaSuccess ||
	    (e = c->in_p.ensure(nl + 1)) != cudaSuccess)
		return cls_fail(c, HERA_GPU_ENOMEM, "class input copies", e);
	if ((nr && (e = cudaMemcpyAsync(c->in_recs.p, res->recs, nr * sizeof(hera_cand_rec), cudaMemcpyHostToDevice,
					c->stream)) != cudaSuccess) ||
	    (nl && (e = cudaMemcpyAsync(c->in_pos.p, res->pos_pool, nl * 4, cudaMemcpyHostToDevice, c->stream)) !=
			   cudaSuccess) ||
	    (nl && (e = cudaMemcpyAsync(c->in_p.p, res->p_pool, nl * 4, cudaMemcpyHostToDevice, c->stream)) !=
			   cudaSuccess))
		return cls_fail(c, HERA_GPU_ECUDA, "class input copies", e);
	rc = cls_add_part(c, c->in_recs.p, c->in_pos.p, c->in_p.p, n, paired, 0);
	return cls_end(c, rc);
}

extern "C" int hera_gpu_classes_fetch(hera_gpu_classes *c, hera_gpu_class_table *out)
{
	if (!c || !out)
		return HERA_GPU_EINVAL;
	if (cudaSetDevice(c->device) != cudaSuccess)
		return cls_fail(c, HERA_GPU_ENODEV, "cudaSetDevice");
	cls::State s{};
	cudaError_t e = cudaMemcpyAsync(&s, c->T.st, sizeof s, cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(c->stream);
	if (e != cudaSuccess)
		return cls_fail(c, HERA_GPU_ECUDA, "class table state", e);
	if (c->broken || s.flags)
		return cls_fail(c, HERA_GPU_ECAPACITY, "class table overflowed; its contents are incomplete");
	out->n_classes = s.n_classes;
	out->list_used = s.ref_used;
	out->paired = (uint32_t)s.paired;               // PAIRED is an unsigned int
	out->mean_frag_sum = (double)s.frag;             // exact below 2^53, as hera's double sum
	if (s.n_classes > out->class_cap || s.ref_used > out->list_cap)
		return cls_fail(c, HERA_GPU_ECAPACITY, "class output buffers too small");
	const uint32_t nc = s.n_classes;
	std::vector<unsigned long long> cnt(nc), off(nc);
	if (nc) {
		if ((e = cudaMemcpyAsync(out->id, c->T.id, (size_t)nc * 4, cudaMemcpyDeviceToHost, c->stream)) ||
		    (e = cudaMemcpyAsync(cnt.data(), c->T.count, (size_t)nc * 8, cudaMemcpyDeviceToHost, c->stream)) ||
		    (e = cudaMemcpyAsync(out->n, c->T.n, (size_t)nc * 4, cudaMemcpyDeviceToHost, c->stream)) ||
		    (e = cudaMemcpyAsync(off.data(), c->T.ref_off, (size_t)nc * 8, cudaMemcpyDeviceToHost, c->stream)))
			return cls_fail(c, HERA_GPU_ECUDA, "class table copy", e);
	}
	if (s.ref_used &&
	    (e = cudaMemcpyAsync(out->list, c->T.ref, (size_t)s.ref_used * 4, cudaMemcpyDeviceToHost, c->stream)))
		return cls_fail(c, HERA_GPU_ECUDA, "class list copy", e);
	if (out->tx_count && c->T.n_trans &&
	    (e = cudaMemcpyAsync(out->tx_count, c->T.tx_count, (size_t)c->T.n_trans * 4, cudaMemcpyDeviceToHost,
				 c->stream)))
		return cls_fail(c, HERA_GPU_ECUDA, "transcript count copy", e);
	if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess)
		return cls_fail(c, HERA_GPU_ECUDA, "class table copy", e);
	for (uint32_t i = 0; i < nc; ++i) {
		out->count[i] = (double)cnt[i];
		out->list_off[i] = off[i];
	}
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_classes_timing(const hera_gpu_classes *c, float *kernel_ms, uint32_t *launches)
{
	if (!c)
		return HERA_GPU_EINVAL;
	if (kernel_ms)
		*kernel_ms = c->kernel_ms;
	if (launches)
		*launches = c->launches;
	return HERA_GPU_OK;
}

extern "C" const char *hera_gpu_classes_last_error(const hera_gpu_classes *c)
{
	return c ? c->err.c_str() : "null class table";
}
