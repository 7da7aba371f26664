// hera_server.cuh -- the serving loop of include/hera_gpu.h (included at
// the end of hera_gpu.cu; uses its Lane, run_batch and copy_out).
//
// Chunks wait in a FIFO.  Each batch slot has a Lane (stream, device
// buffers, pinned staging) and a host thread that loops: cut a batch of up
// to batch_pairs pairs from the head of the FIFO (pieces of one or more
// chunks), stage it, run the batched pipeline, tally the per-sample
// counters on the device, bring the records back and file each piece's
// records under its chunk.  A chunk is done when all its pieces are filed;
// hera_gpu_server_wait then lays its pieces out in pair order.
#pragma once

#include <algorithm>
#include <deque>
#include <memory>
#include <unordered_map>

namespace {

constexpr int SRV_MAX_PIECES = 32;   // chunks (pieces) in one device batch
constexpr int SRV_FIELDS = 8;        // u64 counters per sample

struct PieceTable {
	int n;
	int32_t lo[SRV_MAX_PIECES + 1];  // first pair of piece k in the batch; lo[n] = batch size
	uint32_t sample[SRV_MAX_PIECES];
};

// per-sample counters over one batch's records (two per pair)
__global__ void k_tally(const hera_cand_rec *__restrict__ recs, PieceTable pt,
			unsigned long long *__restrict__ samples)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= pt.lo[pt.n])
		return;
	int k = 0;
	while (k + 1 < pt.n && i >= pt.lo[k + 1])
		++k;
	const hera_cand_rec a = recs[2 * i], b = recs[2 * i + 1];
	unsigned long long *S = samples + (size_t)pt.sample[k] * SRV_FIELDS;
	const unsigned long long hits = (unsigned long long)(a.n[0] + a.n[1] + b.n[0] + b.n[1]);
	atomicAdd(S + 0, 1ull);
	if (hits)
		atomicAdd(S + 1, 1ull);
	if (a.pair == 2)
		atomicAdd(S + 2, 1ull);
	atomicAdd(S + 3, hits);
	atomicAdd(S + 4, (unsigned long long)(a.n_cigar[0] + a.n_cigar[1] + b.n_cigar[0] + b.n_cigar[1]));
}

struct SrvBatchOut {   // one batch's records and pools on the host
	std::vector<hera_cand_rec> recs;
	std::vector<uint32_t> pos, ops;
	std::vector<int32_t> p;
	std::vector<char> miss;
};

struct SrvSeg {   // one piece: its ranges in a batch's output
	int32_t lo = 0, cnt = 0;
	std::shared_ptr<SrvBatchOut> out;
	size_t r0 = 0, r1 = 0;                 // records
	uint32_t l0 = 0, l1 = 0, o0 = 0, o1 = 0, m0 = 0, m1 = 0;   // pools
};

// host array without value-initialisation, reused across chunks (fresh
// memory for every chunk would cost a page fault per 4 KiB on first touch)
template <typename T>
struct RawBuf {
	std::unique_ptr<T[]> p;
	size_t cap = 0;
	void need(size_t n)
	{
		if (n > cap) {
			p.reset(new T[n]);
			cap = n;
		}
	}
	T *data() { return p.get(); }
	const T *data() const { return p.get(); }
	T &operator[](size_t i) { return p[i]; }
	const T &operator[](size_t i) const { return p[i]; }
};

struct SrvChunk {
	uint64_t ticket = 0;
	uint32_t sample = 0;
	int32_t n = 0;
	RawBuf<char> seq[2];          // mate 1 and mate 2 reads, back to back
	const char *src[2] = {nullptr, nullptr};   // borrowed: the caller's reads (off[] index it)
	RawBuf<int64_t> off[2];       // n each, into seq[m]
	RawBuf<int32_t> len[2];
	int max_len = 0;
	int32_t handed = 0, done = 0;
	int32_t inflight = 0;         // pieces handed to batches and not filed yet
	bool waited = false;          // a hera_gpu_server_wait holds the chunk
	int32_t batches = 0;
	double t_submit = 0, t_admit = -1, t_done = -1;
	std::vector<SrvSeg> segs;
	int rc = HERA_GPU_OK;
	std::string err;
	// on a failure, done once no batch holds a piece of it any more
	bool finished() const { return done == n || (rc != HERA_GPU_OK && inflight == 0); }
};

struct SrvPiece {
	SrvChunk *c;
	int32_t lo, cnt;
};

}  // namespace

struct hera_gpu_server {
	hera_gpu_ctx *ctx = nullptr;
	int write_bam = 1;
	uint32_t batch_pairs = 131072;
	uint32_t max_samples = 1024;
	bool borrow = false;             // submit keeps the caller's read pointers
	uint64_t slot_bytes = 0;
	std::vector<Lane *> slots;
	std::vector<std::thread> workers;
	std::mutex mu;
	std::condition_variable cv_work, cv_done;
	std::deque<SrvChunk *> pending;
	std::unordered_map<uint64_t, SrvChunk *> chunks;
	std::vector<SrvChunk *> spare;   // released chunks whose buffers are reused
	uint64_t next_ticket = 1;
	bool stop = false;
	unsigned long long *d_samples = nullptr;
	std::mutex sample_mu;          // d_samples reads vs tallies
	std::chrono::steady_clock::time_point t0;
	std::vector<float> lat, wait;
	uint64_t chunks_done = 0, pairs_done = 0, batches = 0;
	double first_submit = -1, last_done = 0;
	std::string err;

	double now() const
	{
		return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
	}
};

// device bytes one slot holds for a batch of P pairs of reads up to
// MAX_READ (the lane's buffers at their usual high-water marks)
static uint64_t srv_slot_bytes(uint64_t P)
{
	const uint64_t spr = (MAX_READ - KMER) / KMER + 1;
	uint64_t b = 0;
	b += 3 * 2 * P * MAX_READ;                // reads, codes, reverse codes
	b += 2 * P * 12 + 2 * P * 2 * spr * 8;    // offsets, lengths, seed hits
	b += P * sizeof(DPair);                   // per-pair Candidate state
	b += 4 * P * (sizeof(TaskInfo) + 2 * sizeof(Chain) + 3 * sizeof(DpJob) + 4 * sizeof(JobSlot));
	b += 12 * P * ((uint64_t)res_stride(JCAP) + 12);   // DP results, order, reruns
	b += 2 * P * (sizeof(hera_cand_rec) + 24) + 2 * P * 16 * 8;   // records, counts, pools
	b += P / 8 * LCAP * (sizeof(int2) + sizeof(SswOut));          // rescue calls
	return b + (64ull << 20);
}

// a released chunk's state cleared for reuse (its buffers are kept)
static void srv_reset(SrvChunk &c)
{
	c.ticket = 0;
	c.handed = c.done = c.inflight = c.batches = 0;
	c.waited = false;
	c.max_len = 0;
	c.t_admit = c.t_done = -1;
	c.segs.clear();
	c.rc = HERA_GPU_OK;
	c.err.clear();
}

// keep a released chunk's buffers for the next submit (a bounded number)
static void srv_release(hera_gpu_server *S, SrvChunk *c)
{
	c->segs.clear();   // drop the batch outputs now
	std::lock_guard<std::mutex> g(S->mu);
	if (S->spare.size() < 4 * S->slots.size() + 8)
		S->spare.push_back(c);
	else
		delete c;
}

// stage a batch's pieces into lane L: per piece the mate-1 and mate-2
// byte ranges, offsets interleaved (read 2i = mate 1 of pair i)
static int srv_stage(Lane &L, const std::vector<SrvPiece> &pc, int32_t npairs, int64_t *bytes, int *max_len)
{
	cudaStream_t st = L.stream;
	int64_t total = 0;
	int ml = 0;
	auto range = [](const SrvChunk &c, int m, int32_t lo, int32_t cnt, int64_t &a, int64_t &e) {
		a = c.off[m][lo];
		e = c.off[m][lo + cnt - 1] + c.len[m][lo + cnt - 1];
	};
	for (const SrvPiece &q : pc) {
		for (int m = 0; m < 2; ++m) {
			int64_t a, e;
			range(*q.c, m, q.lo, q.cnt, a, e);
			total += e - a;
		}
		ml = q.c->max_len > ml ? q.c->max_len : ml;
	}
	LK(L.h_seq.ensure(total + 1), "pinned reads");
	LK(L.h_off.ensure(2 * (size_t)npairs), "pinned offsets");
	LK(L.h_len.ensure(2 * (size_t)npairs), "pinned lengths");
	const auto h0 = std::chrono::steady_clock::now();
	int64_t o = 0;
	size_t r = 0;
	for (const SrvPiece &q : pc) {
		const SrvChunk &c = *q.c;
		for (int m = 0; m < 2; ++m) {
			int64_t a, e;
			range(c, m, q.lo, q.cnt, a, e);
			pcopy(L.h_seq.p + o, (c.src[m] ? c.src[m] : c.seq[m].data()) + a, (size_t)(e - a));
			for (int32_t i = 0; i < q.cnt; ++i) {
				L.h_off.p[2 * (r + i) + m] = c.off[m][q.lo + i] - a + o;
				L.h_len.p[2 * (r + i) + m] = c.len[m][q.lo + i];
			}
			o += e - a;
		}
		r += (size_t)q.cnt;
	}
	L.timing.host_stage_ms +=
		std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - h0).count();
	LK(L.seq.ensure(total + 64), "device reads");
	LK(L.off.ensure(2 * (size_t)npairs), "device offsets");
	LK(L.len.ensure(2 * (size_t)npairs), "device lengths");
	LK(cudaMemcpyAsync(L.seq.p, L.h_seq.p, total, cudaMemcpyHostToDevice, st), "H2D reads");
	LK(cudaMemcpyAsync(L.off.p, L.h_off.p, 2 * (size_t)npairs * 8, cudaMemcpyHostToDevice, st), "H2D");
	LK(cudaMemcpyAsync(L.len.p, L.h_len.p, 2 * (size_t)npairs * 4, cudaMemcpyHostToDevice, st), "H2D");
	*bytes = total;
	*max_len = ml;
	return HERA_GPU_OK;
}

// one batch on slot L: stage, align, tally, bring back, file per piece
static int srv_batch(hera_gpu_server *S, Lane &L, const std::vector<SrvPiece> &pc)
{
	int32_t np = 0;
	PieceTable pt{};
	pt.n = (int)pc.size();
	for (int k = 0; k < pt.n; ++k) {
		pt.lo[k] = np;
		pt.sample[k] = pc[k].c->sample;
		np += pc[k].cnt;
	}
	pt.lo[pt.n] = np;
	int64_t bytes = 0;
	int max_len = 0;
	int rc = srv_stage(L, pc, np, &bytes, &max_len);
	if (rc)
		return rc;
	rc = run_batch(S->ctx, L, L.seq.p, L.off.p, L.len.p, np, true, S->write_bam, max_len, bytes);
	if (rc)
		return rc;
	{
		std::lock_guard<std::mutex> g(S->sample_mu);
		k_tally<<<blocks_for(np, 256), 256, 0, L.stream>>>(L.recs.p, pt, S->d_samples);
		LK(cudaGetLastError(), "tally");
	}
	// the batch's records into host vectors; pieces refer to their ranges
	auto bo = std::make_shared<SrvBatchOut>();
	bo->recs.resize((size_t)L.items);
	bo->pos.resize(L.nl + 1);
	bo->p.resize(L.nl + 1);
	bo->ops.resize(L.no + 1);
	bo->miss.resize(L.nm + 1);
	hera_gpu_result out{bo->recs.data(), bo->pos.data(), bo->p.data(), bo->ops.data(), bo->miss.data(),
			    L.nl + 1, L.no + 1, L.nm + 1, 0, 0, 0};
	rc = copy_out(L, &out, 0, 0, 0, 0);
	if (rc)
		return rc;
	std::vector<SrvSeg> segs(pc.size());
	for (size_t k = 0; k < pc.size(); ++k) {
		SrvSeg &g = segs[k];
		g.lo = pc[k].lo;
		g.cnt = pc[k].cnt;
		g.out = bo;
		g.r0 = 2 * (size_t)pt.lo[k];
		g.r1 = 2 * (size_t)pt.lo[k + 1];
		const hera_cand_rec &f = bo->recs[g.r0], &l = bo->recs[g.r1 - 1];
		g.l0 = f.list_off[0];
		g.l1 = l.list_off[1] + (uint32_t)l.n[1];
		g.o0 = f.cig_off[0];
		g.o1 = l.cig_off[1] + l.n_cigar[1];
		g.m0 = f.miss_off[0];
		g.m1 = l.miss_off[1] + l.n_miss[1];
	}
	std::lock_guard<std::mutex> g(S->mu);
	const double t = S->now();
	++S->batches;
	for (size_t k = 0; k < pc.size(); ++k) {
		SrvChunk &c = *pc[k].c;
		c.segs.push_back(std::move(segs[k]));
		c.done += pc[k].cnt;
		--c.inflight;
		++c.batches;
		if (c.done == c.n) {
			c.t_done = t;
			S->lat.push_back((float)(t - c.t_submit));
			S->wait.push_back((float)(c.t_admit - c.t_submit));
			++S->chunks_done;
			S->pairs_done += (uint64_t)c.n;
			S->last_done = t;
		}
	}
	S->cv_done.notify_all();
	return HERA_GPU_OK;
}

static void srv_worker(hera_gpu_server *S, int k)
{
	cudaSetDevice(S->ctx->device);
	Lane &L = *S->slots[k];
	for (;;) {
		std::vector<SrvPiece> pc;
		{
			std::unique_lock<std::mutex> g(S->mu);
			S->cv_work.wait(g, [&] { return S->stop || !S->pending.empty(); });
			if (S->stop)
				return;
			int32_t room = (int32_t)S->batch_pairs;
			const double t = S->now();
			while (room > 0 && !S->pending.empty() && (int)pc.size() < SRV_MAX_PIECES) {
				SrvChunk *c = S->pending.front();
				const int32_t take = std::min(room, c->n - c->handed);
				if (c->handed == 0)
					c->t_admit = t;
				pc.push_back({c, c->handed, take});
				c->handed += take;
				++c->inflight;
				room -= take;
				if (c->handed == c->n)
					S->pending.pop_front();
			}
			if (!S->pending.empty())
				S->cv_work.notify_one();
		}
		L.err.clear();
		const int rc = srv_batch(S, L, pc);
		if (rc) {
			std::lock_guard<std::mutex> g(S->mu);
			for (const SrvPiece &q : pc) {
				q.c->rc = rc;
				q.c->err = L.err;
				--q.c->inflight;
				// no further pieces of a failed chunk
				auto it = std::find(S->pending.begin(), S->pending.end(), q.c);
				if (it != S->pending.end())
					S->pending.erase(it);
			}
			S->cv_done.notify_all();
		}
	}
}

extern "C" int hera_gpu_server_create(hera_gpu_ctx *ctx, const hera_gpu_server_options *opt,
				      hera_gpu_server **out)
{
	if (!ctx || !out)
		return HERA_GPU_EINVAL;
	*out = nullptr;
	if (cudaSetDevice(ctx->device) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENODEV, "cudaSetDevice");
	hera_gpu_server *S = new hera_gpu_server();
	S->ctx = ctx;
	S->t0 = std::chrono::steady_clock::now();
	int max_slots = 6;
	uint64_t reserve = 4ull << 30;
	if (opt) {
		if (opt->batch_pairs)
			S->batch_pairs = opt->batch_pairs;
		if (opt->max_slots > 0)
			max_slots = opt->max_slots;
		if (opt->hbm_reserve)
			reserve = opt->hbm_reserve;
		if (opt->write_bam != 0 && opt->write_bam != 1) {
			delete S;
			return fail(ctx, HERA_GPU_EINVAL, "write_bam must be 0 or 1");
		}
		S->write_bam = opt->write_bam;
		if (opt->max_samples)
			S->max_samples = opt->max_samples;
		S->borrow = opt->borrow_reads != 0;
	}
	if (S->batch_pairs > (1u << 20))
		S->batch_pairs = 1u << 20;
	if (max_slots > 16)
		max_slots = 16;
	// admission by free device memory: as many slots as fit
	size_t free_b = 0, total_b = 0;
	if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
		delete S;
		return fail(ctx, HERA_GPU_ECUDA, "cudaMemGetInfo");
	}
	S->slot_bytes = srv_slot_bytes(S->batch_pairs);
	const uint64_t avail = free_b > reserve ? free_b - reserve : 0;
	int nslots = (int)std::min<uint64_t>((uint64_t)max_slots, avail / S->slot_bytes);
	if (nslots < 1) {
		delete S;
		return fail(ctx, HERA_GPU_ENOMEM, "not enough free device memory for one batch slot");
	}
	const size_t sbytes = (size_t)S->max_samples * SRV_FIELDS * sizeof(unsigned long long);
	if (cudaMalloc(&S->d_samples, sbytes) != cudaSuccess ||
	    cudaMemset(S->d_samples, 0, sbytes) != cudaSuccess) {
		if (S->d_samples)
			cudaFree(S->d_samples);
		delete S;
		return fail(ctx, HERA_GPU_ENOMEM, "per-sample state");
	}
	for (int i = 0; i < nslots; ++i) {
		Lane *L = new Lane();
		S->slots.push_back(L);
		if (cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking) != cudaSuccess) {
			hera_gpu_server_destroy(S);
			return fail(ctx, HERA_GPU_ECUDA, "slot stream");
		}
		for (auto &e : L->ev)
			cudaEventCreate(&e);
	}
	for (int i = 0; i < nslots; ++i)
		S->workers.emplace_back(srv_worker, S, i);
	*out = S;
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_server_submit(hera_gpu_server *S, uint32_t sample, const hera_gpu_reads *r1,
				      const hera_gpu_reads *r2, int32_t n, uint64_t *ticket)
{
	if (!S || !r1 || !r2 || !ticket || n < 0)
		return HERA_GPU_EINVAL;
	if (sample >= S->max_samples)
		return fail(S->ctx, HERA_GPU_EINVAL, "sample id beyond max_samples");
	SrvChunk *c = nullptr;
	{
		std::lock_guard<std::mutex> g(S->mu);
		if (!S->spare.empty()) {
			c = S->spare.back();
			S->spare.pop_back();
		}
	}
	if (c)
		srv_reset(*c);
	else
		c = new SrvChunk();
	c->sample = sample;
	c->n = n;
	const hera_gpu_reads *src[2] = {r1, r2};
	for (int m = 0; m < 2; ++m) {
		const hera_gpu_reads &R = *src[m];
		c->off[m].need((size_t)n);
		c->len[m].need((size_t)n);
		int64_t total = 0;
		bool contig = true;
		for (int32_t i = 0; i < n; ++i) {
			const int32_t Ln = R.len[i];
			if (Ln < 0 || Ln > MAX_READ) {
				delete c;
				return fail(S->ctx, HERA_GPU_EINVAL, "read length outside 0..HERA_GPU_MAX_READ");
			}
			if (i > 0 && R.off[i] != R.off[i - 1] + R.len[i - 1])
				contig = false;
			c->max_len = Ln > c->max_len ? Ln : c->max_len;
			total += Ln;
		}
		c->src[m] = nullptr;
		if (S->borrow) {   // the caller's memory, read by the slots at staging
			// a piece is staged as one byte range: reads in rising order
			for (int32_t i = 1; i < n; ++i)
				if (R.off[i] < R.off[i - 1] + R.len[i - 1]) {
					delete c;
					return fail(S->ctx, HERA_GPU_EINVAL,
						    "borrowed reads must lie in rising order without overlap");
				}
			c->src[m] = R.seq;
			for (int32_t i = 0; i < n; ++i) {
				c->off[m][i] = R.off[i];
				c->len[m][i] = R.len[i];
			}
			continue;
		}
		c->seq[m].need((size_t)total + 1);
		if (contig && n > 0) {   // one copy of the block
			pcopy(c->seq[m].data(), R.seq + R.off[0], (size_t)total);
			for (int32_t i = 0; i < n; ++i) {
				c->off[m][i] = R.off[i] - R.off[0];
				c->len[m][i] = R.len[i];
			}
		} else {
			int64_t o = 0;
			for (int32_t i = 0; i < n; ++i) {
				memcpy(c->seq[m].data() + o, R.seq + R.off[i], (size_t)R.len[i]);
				c->off[m][i] = o;
				c->len[m][i] = R.len[i];
				o += R.len[i];
			}
		}
	}
	std::lock_guard<std::mutex> g(S->mu);
	c->ticket = S->next_ticket++;
	c->t_submit = S->now();
	if (S->first_submit < 0)
		S->first_submit = c->t_submit;
	S->chunks[c->ticket] = c;
	if (n > 0) {
		S->pending.push_back(c);
		S->cv_work.notify_one();
	} else {
		c->t_admit = c->t_done = c->t_submit;
	}
	*ticket = c->ticket;
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_server_wait(hera_gpu_server *S, uint64_t ticket, hera_gpu_result *out,
				    hera_gpu_chunk_info *info)
{
	if (!S || !out)
		return HERA_GPU_EINVAL;
	std::unique_lock<std::mutex> g(S->mu);
	auto it = S->chunks.find(ticket);
	if (it == S->chunks.end())
		return fail(S->ctx, HERA_GPU_EINVAL, "unknown ticket");
	SrvChunk *c = it->second;
	if (c->waited)
		return fail(S->ctx, HERA_GPU_EINVAL, "ticket already being waited for");
	c->waited = true;
	S->cv_done.wait(g, [&] { return c->finished(); });
	if (c->rc != HERA_GPU_OK) {
		const int rc = c->rc;
		const std::string e = c->err;
		S->chunks.erase(it);
		delete c;
		g.unlock();
		return fail(S->ctx, rc, e.c_str());
	}
	// finished: no slot touches the chunk any more, so the copy runs unlocked
	g.unlock();
	std::sort(c->segs.begin(), c->segs.end(), [](const SrvSeg &a, const SrvSeg &b) { return a.lo < b.lo; });
	uint64_t tl = 0, to = 0, tm = 0;
	for (const SrvSeg &s : c->segs) {
		tl += s.l1 - s.l0;
		to += s.o1 - s.o0;
		tm += s.m1 - s.m0;
	}
	out->list_used = tl;
	out->op_used = to;
	out->miss_used = tm;
	if (tl > out->list_cap || to > out->op_cap || tm > out->miss_cap) {
		g.lock();
		c->waited = false;   // kept for another try
		g.unlock();
		return fail(S->ctx, HERA_GPU_ECAPACITY, "result pools too small (see *_used for the sizes needed)");
	}
	uint64_t bl = 0, bo = 0, bm = 0;
	for (const SrvSeg &s : c->segs) {
		const SrvBatchOut &B = *s.out;
		hera_cand_rec *dst = out->recs + 2 * (size_t)s.lo;
		for (size_t i = s.r0; i < s.r1; ++i) {
			hera_cand_rec r = B.recs[i];
			for (int k = 0; k < 2; ++k) {
				r.list_off[k] = r.list_off[k] - s.l0 + (uint32_t)bl;
				r.cig_off[k] = r.cig_off[k] - s.o0 + (uint32_t)bo;
				r.miss_off[k] = r.miss_off[k] - s.m0 + (uint32_t)bm;
			}
			*dst++ = r;
		}
		if (s.l1 > s.l0) {
			memcpy(out->pos_pool + bl, B.pos.data() + s.l0, (size_t)(s.l1 - s.l0) * 4);
			memcpy(out->p_pool + bl, B.p.data() + s.l0, (size_t)(s.l1 - s.l0) * 4);
		}
		if (s.o1 > s.o0)
			memcpy(out->op_pool + bo, B.ops.data() + s.o0, (size_t)(s.o1 - s.o0) * 4);
		if (s.m1 > s.m0)
			memcpy(out->miss_pool + bm, B.miss.data() + s.m0, (size_t)(s.m1 - s.m0));
		bl += s.l1 - s.l0;
		bo += s.o1 - s.o0;
		bm += s.m1 - s.m0;
	}
	if (info) {
		info->sample = c->sample;
		info->n = c->n;
		info->submit_ms = c->t_submit;
		info->admit_ms = c->t_admit;
		info->done_ms = c->t_done;
		info->batches = c->batches;
	}
	g.lock();
	S->chunks.erase(ticket);
	g.unlock();
	srv_release(S, c);
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_server_cancel(hera_gpu_server *S, uint32_t sample, int32_t *n_chunks)
{
	if (!S)
		return HERA_GPU_EINVAL;
	if (sample >= S->max_samples)
		return fail(S->ctx, HERA_GPU_EINVAL, "sample id beyond max_samples");
	int32_t k = 0;
	{
		std::lock_guard<std::mutex> g(S->mu);
		// queued chunks of the sample: the parts not yet in a batch are
		// dropped; pieces already in a batch finish (they share it with
		// other samples' pieces) and are then discarded with the chunk
		for (auto it = S->pending.begin(); it != S->pending.end();) {
			SrvChunk *c = *it;
			if (c->sample == sample) {
				c->rc = HERA_GPU_ECANCELED;
				c->err = "the chunk's sample was cancelled";
				it = S->pending.erase(it);
				++k;
			} else {
				++it;
			}
		}
		S->cv_done.notify_all();
	}
	if (n_chunks)
		*n_chunks = k;
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_server_get_sample_stats(hera_gpu_server *S, uint32_t sample, hera_gpu_sample_stats *out)
{
	if (!S || !out || sample >= S->max_samples)
		return HERA_GPU_EINVAL;
	if (cudaSetDevice(S->ctx->device) != cudaSuccess)
		return HERA_GPU_ENODEV;
	unsigned long long v[SRV_FIELDS];
	{
		// every tally launched so far is ordered before this copy
		std::lock_guard<std::mutex> g(S->sample_mu);
		for (Lane *L : S->slots)
			if (cudaStreamSynchronize(L->stream) != cudaSuccess)
				return fail(S->ctx, HERA_GPU_ECUDA, "slot stream");
		if (cudaMemcpy(v, S->d_samples + (size_t)sample * SRV_FIELDS, sizeof v, cudaMemcpyDeviceToHost) !=
		    cudaSuccess)
			return fail(S->ctx, HERA_GPU_ECUDA, "per-sample state");
	}
	out->pairs = v[0];
	out->mapped = v[1];
	out->paired = v[2];
	out->hits = v[3];
	out->cigar_ops = v[4];
	out->reserved[0] = out->reserved[1] = out->reserved[2] = 0;
	return HERA_GPU_OK;
}

static float srv_quantile(std::vector<float> v, double q)
{
	if (v.empty())
		return 0;
	std::sort(v.begin(), v.end());
	size_t i = (size_t)(q * (double)(v.size() - 1) + 0.5);
	return v[std::min(i, v.size() - 1)];
}

extern "C" int hera_gpu_server_get_stats(hera_gpu_server *S, hera_gpu_server_stats *out)
{
	if (!S || !out)
		return HERA_GPU_EINVAL;
	std::lock_guard<std::mutex> g(S->mu);
	out->slots = (int)S->slots.size();
	out->slot_bytes = S->slot_bytes;
	out->chunks_done = S->chunks_done;
	out->pairs_done = S->pairs_done;
	out->batches = S->batches;
	out->p50_ms = srv_quantile(S->lat, 0.50);
	out->p99_ms = srv_quantile(S->lat, 0.99);
	out->p50_wait_ms = srv_quantile(S->wait, 0.50);
	out->p99_wait_ms = srv_quantile(S->wait, 0.99);
	const double span = S->last_done - S->first_submit;
	out->pairs_per_s = span > 0 ? (double)S->pairs_done / (span * 1e-3) : 0.0;
	return HERA_GPU_OK;
}

extern "C" void hera_gpu_server_destroy(hera_gpu_server *S)
{
	if (!S)
		return;
	{
		std::lock_guard<std::mutex> g(S->mu);
		S->stop = true;
	}
	S->cv_work.notify_all();
	for (auto &t : S->workers)
		t.join();
	cudaSetDevice(S->ctx->device);
	for (Lane *L : S->slots) {
		if (L->stream)
			cudaStreamSynchronize(L->stream);
		L->release();
		delete L;
	}
	for (auto &kv : S->chunks)
		delete kv.second;
	for (SrvChunk *c : S->spare)
		delete c;
	if (S->d_samples)
		cudaFree(S->d_samples);
	delete S;
}
