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

namespace cls {
// hera_gpu_classes_load: class i's id into the table (ids are distinct in
// a table add_class built; a repeated id keeps its first class)
__global__ void k_cls_load_keys(Table T, uint32_t nc)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nc)
		return;
	const uint32_t id = T.id[i];
	const unsigned long long key = (unsigned long long)id + 1;
	uint32_t a = id & T.mask;
	for (uint32_t probe = 0; probe <= T.mask; ++probe) {
		const unsigned long long cur = atomicCAS(&T.keys[a], 0ull, key);
		if (cur == 0ull || cur == key) {
			atomicMin(&T.first[a], i);
			return;
		}
		a = (a + 1) & T.mask;
	}
	atomicOr(&T.st->flags, F_MAP);
}

__global__ void k_cls_load_number(Table T, uint32_t nc)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nc)
		return;
	const uint32_t id = T.id[i];
	const unsigned long long key = (unsigned long long)id + 1;
	uint32_t a = id & T.mask;
	for (uint32_t probe = 0; probe <= T.mask; ++probe) {
		if (T.keys[a] == key) {
			if (T.first[a] == i)
				T.cls_of[a] = i + 1;
			return;
		}
		a = (a + 1) & T.mask;
	}
}

__global__ void k_cls_load_reset(Table T)
{
	const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
	if (a > T.mask)
		return;
	T.first[a] = NONE;   // the load used first[] for its own numbering
}
}   // namespace cls

extern "C" int hera_gpu_classes_load(hera_gpu_classes *c, const hera_gpu_class_table *in)
{
	if (!c)
		return HERA_GPU_EINVAL;
	if (!in || (in->n_classes && (!in->id || !in->count || !in->n || !in->list_off)) ||
	    (in->list_used && !in->list))
		return cls_fail(c, HERA_GPU_EINVAL, "bad argument");
	if (in->n_classes > c->T.max_classes || in->list_used > c->T.ref_cap)
		return cls_fail(c, HERA_GPU_ECAPACITY, "class table too small for the classes loaded");
	const uint32_t nc = in->n_classes;
	std::vector<unsigned long long> cnt(nc), off(nc);
	for (uint32_t i = 0; i < nc; ++i) {
		const double x = in->count[i];
		if (!(x >= 0) || x != (double)(unsigned long long)x || x >= 9007199254740992.0)
			return cls_fail(c, HERA_GPU_EINVAL, "class counts must be whole numbers below 2^53");
		if (in->list_off[i] + in->n[i] > in->list_used)
			return cls_fail(c, HERA_GPU_EINVAL, "a class list lies outside the list entries");
		cnt[i] = (unsigned long long)x;
		off[i] = in->list_off[i];
	}
	if (!(in->mean_frag_sum >= 0) || in->mean_frag_sum >= 9007199254740992.0)
		return cls_fail(c, HERA_GPU_EINVAL, "bad fragment sum");
	if (cudaSetDevice(c->device) != cudaSuccess)
		return cls_fail(c, HERA_GPU_ENODEV, "cudaSetDevice");
	cls::Table &T = c->T;
	const cudaStream_t st = c->stream;
	cls::State s{};
	s.n_classes = nc;
	s.ref_used = in->list_used;
	s.paired = in->paired;
	s.frag = (unsigned long long)in->mean_frag_sum;
	const size_t slots = (size_t)T.mask + 1;
	cudaError_t e;
	if ((e = cudaMemsetAsync(T.keys, 0, slots * 8, st)) != cudaSuccess ||
	    (e = cudaMemsetAsync(T.cls_of, 0, slots * 4, st)) != cudaSuccess ||
	    (e = cudaMemsetAsync(T.first, 0xff, slots * 4, st)) != cudaSuccess ||
	    (e = cudaMemsetAsync(T.pend, 0, slots * 4, st)) != cudaSuccess ||
	    (nc && (e = cudaMemcpyAsync(T.id, in->id, (size_t)nc * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) ||
	    (nc && (e = cudaMemcpyAsync(T.count, cnt.data(), (size_t)nc * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess) ||
	    (nc && (e = cudaMemcpyAsync(T.n, in->n, (size_t)nc * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) ||
	    (nc && (e = cudaMemcpyAsync(T.ref_off, off.data(), (size_t)nc * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess) ||
	    (in->list_used && (e = cudaMemcpyAsync(T.ref, in->list, (size_t)in->list_used * 4, cudaMemcpyHostToDevice,
						   st)) != cudaSuccess) ||
	    (e = (in->tx_count ? cudaMemcpyAsync(T.tx_count, in->tx_count, (size_t)T.n_trans * 4,
						 cudaMemcpyHostToDevice, st)
			       : cudaMemsetAsync(T.tx_count, 0, (size_t)T.n_trans * 4, st))) != cudaSuccess ||
	    (e = cudaMemcpyAsync(T.st, &s, sizeof s, cudaMemcpyHostToDevice, st)) != cudaSuccess)
		return cls_fail(c, HERA_GPU_ECUDA, "class table load", e);
	if (nc) {
		cls::k_cls_load_keys<<<blocks_for(nc, 256), 256, 0, st>>>(T, nc);
		cls::k_cls_load_number<<<blocks_for(nc, 256), 256, 0, st>>>(T, nc);
	}
	cls::k_cls_load_reset<<<blocks_for((int64_t)slots, 256), 256, 0, st>>>(T);
	c->broken = false;
	c->items_done = 0;
	return cls_check(c);
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

// ---------------------------------------------------------------------------
// The EM over the class table: hera's estimate_count (src/EM.c:315-387),
// SQUAREM over M_step (:271-302), bit for bit.
//
// Every floating-point operation is the reference's, in its order, with
// explicit round-to-nearest intrinsics (nothing is contracted into an FMA):
//   - a class's total (sum of grama over its list) is summed in list order
//     by one thread per class;
//   - a transcript's overlap is summed in class order by one thread per
//     transcript over the table's list entries sorted stably by transcript
//     (a radix sort keeps entry order, which is class order);
//   - the two Norm sums (src/hash_align.c:150-164) and the final sum run in
//     index order in one warp each (seq_sum) -- a sequential double sum has
//     only one rounding sequence;
//   - the convergence flag is an "any transcript moved > 1%", which does
//     not depend on order.
namespace em {

__global__ void k_em_entries(const unsigned long long *ref_off, const uint32_t *n, uint32_t nc, uint32_t *ecls)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nc)
		return;
	const unsigned long long o = ref_off[i];
	for (uint32_t k = 0; k < n[i]; ++k)
		ecls[o + k] = i;
}

__global__ void k_em_hist(const uint32_t *ref, int64_t L, uint32_t nt, uint32_t *hist, uint32_t *flags)
{
	const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (e >= L)
		return;
	const uint32_t t = ref[e];
	if (t < nt)
		atomicAdd(&hist[t], 1u);
	else
		atomicOr(flags, 1u);
}

__global__ void k_em_prep(const unsigned long long *cnt, uint32_t nc, double *dc, double *g, uint32_t nt)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < nc)
		dc[i] = (double)cnt[i];
	if (i < nt)
		g[i] = __ddiv_rn(1.0, (double)nt);            // E_step (src/EM.c:304-313)
}

__global__ void k_em_total(const unsigned long long *ref_off, const uint32_t *n, const uint32_t *ref, uint32_t nc,
			   const double *g, double *tot)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nc)
		return;
	const uint32_t *l = ref + ref_off[i];
	double total = 0.0;
	for (uint32_t k = 0; k < n[i]; ++k)
		total = __dadd_rn(total, g[l[k]]);
	tot[i] = total;
}

__global__ void k_em_tx(const uint32_t *seg, const uint32_t *ecls, const double *dc, const double *tot,
			const double *g, const uint32_t *txc, const uint32_t *len, uint32_t nt, double *next,
			int *busy)
{
	const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= nt)
		return;
	const double gt = g[t];
	double acc = 0.0;
	for (uint32_t e = seg[t]; e < seg[t + 1]; ++e) {
		const uint32_t i = ecls[e];
		const double total = tot[i];
		if (total == 0)
			continue;
		acc = __dadd_rn(acc, __ddiv_rn(__dmul_rn(gt, dc[i]), total));
	}
	const double x = __ddiv_rn(__dadd_rn((double)txc[t], acc), (double)len[t]);
	next[t] = x;
	if (x > 1e-3) {
		const double d = __dsub_rn(x, gt);
		const double err = __ddiv_rn(d < 0 ? -d : d, x);
		if (err > 0.01)
			*busy = 1;
	}
}

__global__ void k_em_rv(const double *u, const double *u1, const double *u2, double *r, double *v, uint32_t nt)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nt)
		return;
	const double ri = __dsub_rn(u1[i], u[i]);
	r[i] = ri;
	v[i] = __dsub_rn(__dsub_rn(u2[i], u1[i]), ri);
}

// Sum of f(a[0]), f(a[1]), ... in index order, rounded after every add, as
// a C loop does it.  One warp: 256 elements at a time go through shared
// memory (8 coalesced loads a lane), the next 256 are loaded into registers
// while these are added, and every lane runs the same add chain over the
// staged values (broadcast reads), so every lane ends with the same sum.
// The chain of dependent adds is the bound.
template <typename F>
__device__ double seq_sum(const double *a, uint32_t n, F f, double *sm)
{
	const uint32_t lane = threadIdx.x & 31;
	double nxt[8];
#pragma unroll
	for (int u = 0; u < 8; ++u) {
		const uint32_t i = u * 32 + lane;
		sm[i] = i < n ? a[i] : 0.0;
	}
	__syncwarp();
	double s = 0.0;
	for (uint32_t base = 0; base < n; base += 256) {
#pragma unroll
		for (int u = 0; u < 8; ++u) {
			const uint64_t i = (uint64_t)base + 256 + u * 32 + lane;
			nxt[u] = i < n ? a[i] : 0.0;
		}
		const uint32_t m = n - base < 256 ? n - base : 256;
		if (m == 256) {
#pragma unroll 32
			for (int j = 0; j < 256; ++j)
				s = __dadd_rn(s, f(sm[j]));
		} else {
			for (uint32_t j = 0; j < m; ++j)
				s = __dadd_rn(s, f(sm[j]));
		}
		__syncwarp();
#pragma unroll
		for (int u = 0; u < 8; ++u)
			sm[u * 32 + lane] = nxt[u];
		__syncwarp();
	}
	return s;
}

// Norm (src/hash_align.c:150-164), one warp a vector: block 0 r -> scal[0],
// block 1 v -> scal[1]
__global__ void k_em_norms(const double *r, const double *v, uint32_t nt, double *scal)
{
	__shared__ double sm[256];
	const double *a = blockIdx.x ? v : r;
	double mean = seq_sum(a, nt, [](double x) { return x; }, sm);
	mean = __ddiv_rn(mean, (double)nt);
	double total = seq_sum(a, nt, [mean](double x) {
		const double d = __dsub_rn(x, mean);
		return __dmul_rn(d, d);
	}, sm);
	total = __ddiv_rn(total, (double)(nt - 1));
	if (threadIdx.x == 0)
		scal[blockIdx.x] = __dsqrt_rn(total);
}

__global__ void k_em_step(const double *u, const double *r, const double *v, const double *scal, double *u1,
			  uint32_t nt)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nt)
		return;
	const double n_r = scal[0], n_v = scal[1];
	double alpha = n_v != 0 ? __ddiv_rn(-n_r, n_v) : -1.0;
	if (alpha > -1)
		alpha = -1.0;
	double x = __dadd_rn(__dsub_rn(u[i], __dmul_rn(__dmul_rn(2.0, alpha), r[i])),
			     __dmul_rn(__dmul_rn(alpha, alpha), v[i]));
	if (x < 0)
		x = 0;
	u1[i] = x;
}

__global__ void k_em_sum(const double *g, uint32_t nt, double *sum)
{
	__shared__ double sm[256];
	const double s = seq_sum(g, nt, [](double x) { return x; }, sm);
	if (threadIdx.x == 0)
		*sum = s;
}

__global__ void k_em_final(const double *g, const uint32_t *len, const double *sum, double *grama, double *overlap,
			   uint32_t nt)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= nt)
		return;
	const double s = *sum;
	if (s == 0) {
		grama[i] = 0;
		overlap[i] = 0;
	} else {
		overlap[i] = __dmul_rn(g[i], (double)len[i]);
		grama[i] = __ddiv_rn(__dmul_rn(g[i], 1000000.0), s);
	}
}

}   // namespace em

extern "C" int hera_gpu_classes_em(hera_gpu_classes *c, hera_gpu_ctx *ctx, double *grama, double *overlap,
				   uint32_t *rounds, float *em_ms)
{
	if (!c)
		return HERA_GPU_EINVAL;
	if (!ctx || ctx->device != c->device || !grama || !overlap || ctx->ix.n_trans != c->T.n_trans ||
	    c->T.n_trans < 1)
		return cls_fail(c, HERA_GPU_EINVAL, "bad argument");
	if (c->broken)
		return cls_fail(c, HERA_GPU_ECAPACITY, "class table overflowed earlier");
	if (cudaSetDevice(c->device) != cudaSuccess)
		return cls_fail(c, HERA_GPU_ENODEV, "cudaSetDevice");
	cls::State s{};
	cudaError_t e = cudaMemcpyAsync(&s, c->T.st, sizeof s, cudaMemcpyDeviceToHost, c->stream);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(c->stream);
	if (e != cudaSuccess)
		return cls_fail(c, HERA_GPU_ECUDA, "class table state", e);
	const uint32_t nt = c->T.n_trans, nc = s.n_classes;
	const int64_t L = (int64_t)s.ref_used;
	if (L >= (1ll << 31))
		return cls_fail(c, HERA_GPU_ECAPACITY, "more than 2^31 list entries");
	const cudaStream_t st = c->stream;
	// buffers: 6 transcript vectors, 2 class vectors, entries x3, segments, flags
	double *d = nullptr, *dc = nullptr;
	uint32_t *ecls = nullptr, *keys = nullptr, *vals = nullptr, *seg = nullptr;
	int *busy = nullptr;
	void *tmp = nullptr;
	size_t tmp_sort = 0, tmp_scan = 0;
	cub::DeviceRadixSort::SortPairs(nullptr, tmp_sort, (const uint32_t *)nullptr, (uint32_t *)nullptr,
					(const uint32_t *)nullptr, (uint32_t *)nullptr, (int)std::max<int64_t>(L, 1), 0, 32,
					st);
	cub::DeviceScan::ExclusiveSum(nullptr, tmp_scan, (uint32_t *)nullptr, (uint32_t *)nullptr, nt + 1, st);
	const size_t tmp_bytes = std::max(tmp_sort, tmp_scan) + 16;
	int rc = HERA_GPU_OK;
	auto grab = [&](void **p, size_t bytes) {
		if (rc != HERA_GPU_OK)
			return;
		cudaError_t ee = cudaMalloc(p, bytes);
		if (ee != cudaSuccess)
			rc = cls_fail(c, HERA_GPU_ENOMEM, "EM buffers", ee);
	};
	grab((void **)&d, (size_t)8 * nt * 7 + 16);      // u, A, B, C, r, v, scalars
	grab((void **)&dc, (size_t)16 * (nc ? nc : 1));  // class counts as double, class totals
	grab((void **)&ecls, (size_t)4 * (L ? L : 1));
	grab((void **)&keys, (size_t)4 * (L ? L : 1));
	grab((void **)&vals, (size_t)4 * (L ? L : 1));
	grab((void **)&seg, (size_t)8 * (nt + 2));      // per-transcript counts, then their offsets
	grab((void **)&busy, 16);
	grab(&tmp, tmp_bytes);
	auto release = [&]() {
		cudaFree(d); cudaFree(dc); cudaFree(ecls); cudaFree(keys); cudaFree(vals); cudaFree(seg);
		cudaFree(busy); cudaFree(tmp);
	};
	if (rc != HERA_GPU_OK) {
		release();
		return rc;
	}
	double *vec[4] = {d, d + nt, d + 2 * (size_t)nt, d + 3 * (size_t)nt};   // u, A, B, C
	double *r = d + 4 * (size_t)nt, *v = d + 5 * (size_t)nt, *scal = d + 6 * (size_t)nt;
	double *tot = dc + (nc ? nc : 1);
	const unsigned bt = blocks_for(nt, 256), bc = blocks_for(nc ? nc : 1, 256);
	cudaEventRecord(c->ev0, st);
	// transcript-major view of the lists, entries in class order
	uint32_t *hist = seg + (nt + 2);
	cudaMemsetAsync(hist, 0, (size_t)4 * (nt + 2), st);
	cudaMemsetAsync(busy, 0, 16, st);
	if (L > 0) {
		em::k_em_entries<<<bc, 256, 0, st>>>(c->T.ref_off, c->T.n, nc, ecls);
		em::k_em_hist<<<blocks_for(L, 256), 256, 0, st>>>(c->T.ref, L, nt, hist, (uint32_t *)(busy + 2));
		size_t tb = tmp_bytes;
		cub::DeviceRadixSort::SortPairs(tmp, tb, c->T.ref, keys, ecls, vals, (int)L, 0, 32, st);
	}
	{
		size_t tb = tmp_bytes;
		cub::DeviceScan::ExclusiveSum(tmp, tb, hist, seg, nt + 1, st);
	}
	em::k_em_prep<<<std::max(bt, bc), 256, 0, st>>>(c->T.count, nc, dc, vec[0], nt);
	auto m_step = [&](const double *g, double *next, int *flag) {
		if (nc)
			em::k_em_total<<<bc, 256, 0, st>>>(c->T.ref_off, c->T.n, c->T.ref, nc, g, tot);
		em::k_em_tx<<<bt, 256, 0, st>>>(seg, vals, dc, tot, g, c->T.tx_count, ctx->d_tlen, nt, next, flag);
	};
	uint32_t k = 0;
	int host_busy = 1;
	while (k < 50 || (k < 1000 && host_busy)) {
		double *u = vec[0], *A = vec[1], *B = vec[2], *C = vec[3];
		m_step(u, A, busy + 1);
		m_step(A, B, busy + 1);
		em::k_em_rv<<<bt, 256, 0, st>>>(u, A, B, r, v, nt);
		em::k_em_norms<<<2, 32, 0, st>>>(r, v, nt, scal);
		em::k_em_step<<<bt, 256, 0, st>>>(u, r, v, scal, A, nt);
		cudaMemsetAsync(busy, 0, 4, st);
		m_step(A, C, busy);
		vec[0] = C;
		vec[3] = u;
		++k;
		if (k >= 50) {   // the loop test reads the last M_step's flag
			if ((e = cudaMemcpyAsync(&host_busy, busy, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
			    (e = cudaStreamSynchronize(st)) != cudaSuccess) {
				rc = cls_fail(c, HERA_GPU_ECUDA, "EM", e);
				break;
			}
		}
	}
	if (rc == HERA_GPU_OK) {
		em::k_em_sum<<<1, 32, 0, st>>>(vec[0], nt, scal + 2);
		// results into r and v, then to the host
		em::k_em_final<<<bt, 256, 0, st>>>(vec[0], ctx->d_tlen, scal + 2, r, v, nt);
		cudaEventRecord(c->ev1, st);
		int hflags = 0;
		if ((e = cudaMemcpyAsync(grama, r, (size_t)8 * nt, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
		    (e = cudaMemcpyAsync(overlap, v, (size_t)8 * nt, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
		    (e = cudaMemcpyAsync(&hflags, busy + 2, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
		    (e = cudaStreamSynchronize(st)) != cudaSuccess)
			rc = cls_fail(c, HERA_GPU_ECUDA, "EM results", e);
		else if (hflags)
			rc = cls_fail(c, HERA_GPU_EINVAL, "a class list names no transcript of the index");
		float ms = 0;
		cudaEventElapsedTime(&ms, c->ev0, c->ev1);
		if (em_ms)
			*em_ms = ms;
		if (rounds)
			*rounds = k;
	}
	release();
	return rc;
}
