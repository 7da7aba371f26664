// hera_bam.cuh -- the host tail's BAM records (`-w`) on the device: one
// thread per read pair (or single read) runs hera_bam_core.h's writer
// twice, first for the item's byte count, then -- after a scan of the
// counts -- into its place in the output.  The records leave uncompressed
// (BGZF: hera's bam_write, or hera_gpu_bgzf).

#include "hera_bam_core.h"

namespace bamk {

struct Inputs {
	const hera_cand_rec *recs;
	const uint32_t *pos, *ops;
	const int32_t *pp;
	const char *miss;
	const char *seq1, *seq2, *qual1, *qual2, *name1, *name2;
	const int64_t *off1, *off2;
	const int32_t *len1, *len2;
	int32_t stride;
	int64_t ext1, ext2;     // bytes of seq1/qual1 and seq2/qual2 on the device
	uint64_t nl, no, nm;    // entries of the list, op and miss pools
	bamw::GeneMap g;
	const uint32_t *qual_table;
};

// an item's inputs lie inside the device copies (the host checked the
// same on its side; this re-checks what arrived, so that a bad copy is an
// error bit rather than a stray read)
constexpr uint32_t E_INPUT = 1u << 30;

__device__ __forceinline__ bool rec_ok(const Inputs &in, const hera_cand_rec &r)
{
	for (int s = 0; s < 2; ++s)
		if (r.n[s] < 0 || (uint64_t)r.list_off[s] + (uint32_t)r.n[s] > in.nl ||
		    (uint64_t)r.cig_off[s] + r.n_cigar[s] > in.no || (uint64_t)r.miss_off[s] + r.n_miss[s] > in.nm)
			return false;
	return true;
}

template <bool PAIRED>
__device__ __forceinline__ bool item_ok(const Inputs &in, int64_t i)
{
	if (in.off1[i] < 0 || in.len1[i] < 0 || in.off1[i] + in.len1[i] > in.ext1)
		return false;
	if (PAIRED) {
		if (in.off2[i] < 0 || in.len2[i] < 0 || in.off2[i] + in.len2[i] > in.ext2)
			return false;
		return rec_ok(in, in.recs[2 * i]) && rec_ok(in, in.recs[2 * i + 1]);
	}
	return rec_ok(in, in.recs[i]);
}

// the records of item i (a pair: align_pair_read's writes; a single read:
// align_single_read's, src/hash_align.c:1825-1834); size pass: out null
template <bool PAIRED>
__device__ __forceinline__ uint32_t one_item(const Inputs &in, int64_t i, uint8_t *out, uint64_t at,
					     uint64_t end, uint64_t *bytes)
{
	*bytes = 0;
	if (!item_ok<PAIRED>(in, i))
		return E_INPUT;
	bamw::Ctx x{in.g, in.qual_table, 0};
	bamw::Core cc[2];
	bamw::Sink o{out, at, end};
	bamw::Read a{in.seq1 + in.off1[i], in.qual1 + in.off1[i], in.name1 + i * in.stride, in.len1[i], false, 0, -1};
	a.name_l = bamw::name_length(a.name, in.stride);
	if constexpr (PAIRED) {
		bamw::Read b{in.seq2 + in.off2[i], in.qual2 + in.off2[i], in.name2 + i * in.stride, in.len2[i], false, 0,
			     -1};
		b.name_l = bamw::name_length(b.name, in.stride);
		const bamw::Cand r0 = bamw::cand(in.recs[2 * i], in.pos, in.pp, in.ops, in.miss);
		const bamw::Cand r1 = bamw::cand(in.recs[2 * i + 1], in.pos, in.pp, in.ops, in.miss);
		bamw::tail(x, o, cc, r0, r1, a, b);
	} else {
		const bamw::Cand r = bamw::cand(in.recs[i], in.pos, in.pp, in.ops, in.miss);
		bamw::tail_single(x, o, cc, r, a);
	}
	*bytes = o.at - at;
	return x.err;
}

template <bool PAIRED>
__global__ void k_bam_size(Inputs in, int64_t n, unsigned long long *size, uint32_t *err)
{
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i > n)
		return;
	if (i == n) {
		size[n] = 0;
		return;
	}
	uint64_t bytes = 0;
	const uint32_t e = one_item<PAIRED>(in, i, nullptr, 0, 0, &bytes);
	size[i] = bytes;
	if (e)
		atomicOr(err, e);
}

// the write pass, into the places the scan of the sizes gave; no byte
// lands past an item's place, and an item whose bytes differ from its size
// pass is an error
template <bool PAIRED>
__global__ void k_bam_write(Inputs in, int64_t n, const unsigned long long *off, uint8_t *out, uint32_t *err)
{
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	uint64_t bytes = 0;
	const uint32_t e = one_item<PAIRED>(in, i, out, off[i], off[i + 1], &bytes);
	if ((e & E_INPUT) || off[i] + bytes != off[i + 1])
		atomicOr(err, E_INPUT);
}

}   // namespace bamk

struct hera_gpu_bam {
	int device = 0;
	uint32_t n_trans = 0;
	cudaStream_t stream = nullptr;
	uint32_t n_chr = 0;
	uint32_t *d_map = nullptr;   // chr_len | exon_off | starts | ends | chr | gene | qual table
	size_t off_chr_len = 0, off_exon_off = 0, off_starts = 0, off_ends = 0, off_chr = 0, off_gene = 0,
	       off_qual = 0;
	float kernel_ms = 0;
	cudaEvent_t ev0 = nullptr, ev1 = nullptr;
	std::string err = "no error";
};

static int bam_fail(hera_gpu_bam *b, int code, const char *what, cudaError_t e = cudaSuccess)
{
	return set_err(b->err, code, what, e);
}

extern "C" void hera_gpu_bam_destroy(hera_gpu_bam *b)
{
	if (!b)
		return;
	cudaSetDevice(b->device);
	if (b->stream)
		cudaStreamSynchronize(b->stream);
	cudaFree(b->d_map);
	if (b->ev0)
		cudaEventDestroy(b->ev0);
	if (b->ev1)
		cudaEventDestroy(b->ev1);
	if (b->stream)
		cudaStreamDestroy(b->stream);
	delete b;
}

extern "C" int hera_gpu_bam_create(hera_gpu_ctx *ctx, const hera_gpu_gene_map *gm, hera_gpu_bam **out)
{
	if (!ctx || !gm || !out || !gm->chr_len || !gm->exon_off || !gm->starts || !gm->ends || !gm->chr || !gm->gene)
		return fail(ctx, HERA_GPU_EINVAL, "bad argument");
	*out = nullptr;
	const uint32_t nt = ctx->ix.n_trans;
	const uint32_t n_ex = gm->exon_off[nt];
	for (uint32_t t = 0; t < nt; ++t)
		if (gm->exon_off[t + 1] <= gm->exon_off[t] || gm->chr[t] >= gm->n_chr)
			return fail(ctx, HERA_GPU_EINVAL, "gene map: a transcript without exons or on no chromosome");
	if (cudaSetDevice(ctx->device) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENODEV, "cudaSetDevice");
	auto *b = new hera_gpu_bam;
	b->device = ctx->device;
	b->n_trans = nt;
	b->n_chr = gm->n_chr;
	std::vector<uint32_t> h;
	auto put = [&](const uint32_t *p, size_t k) {
		const size_t at = h.size();
		h.insert(h.end(), p, p + k);
		return at;
	};
	b->off_chr_len = put(gm->chr_len, gm->n_chr);
	b->off_exon_off = put(gm->exon_off, (size_t)nt + 1);
	b->off_starts = put(gm->starts, n_ex);
	b->off_ends = put(gm->ends, n_ex);
	b->off_chr = put(gm->chr, nt);
	b->off_gene = put(gm->gene, nt);
	uint32_t qt[bamw::QUAL_TABLE];
	bamw::qual_table_host(qt);
	b->off_qual = put(qt, bamw::QUAL_TABLE);
	cudaError_t e;
	if ((e = cudaMalloc(&b->d_map, h.size() * 4)) != cudaSuccess ||
	    (e = cudaMemcpy(b->d_map, h.data(), h.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
	    (e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess ||
	    (e = cudaEventCreate(&b->ev0)) != cudaSuccess || (e = cudaEventCreate(&b->ev1)) != cudaSuccess) {
		hera_gpu_bam_destroy(b);
		return fail(ctx, HERA_GPU_ENOMEM, "gene map", e);
	}
	*out = b;
	return HERA_GPU_OK;
}

extern "C" const char *hera_gpu_bam_last_error(const hera_gpu_bam *b)
{
	return b ? b->err.c_str() : "null BAM writer";
}

// the records of n pairs (r2 given) or n single reads (r2, qual2 and
// name2 null): inputs copied to the device, size pass, scan, write pass
static int bam_run(hera_gpu_bam *b, const hera_gpu_result *res, int32_t n, const hera_gpu_reads *r1,
		   const hera_gpu_reads *r2, const char *qual1, const char *qual2, const char *name1,
		   const char *name2, int32_t name_stride, uint8_t *out, uint64_t cap, uint64_t *out_off,
		   float *kernel_ms)
{
	const bool paired = r2 != nullptr;
	if (!res || n < 0 || !r1 || !qual1 || !name1 || name_stride < 1 || !out_off ||
	    (paired && (!qual2 || !name2)) ||
	    (n > 0 && (!res->recs || !r1->seq || !r1->off || !r1->len ||
		       (paired && (!r2->seq || !r2->off || !r2->len)))))
		return bam_fail(b, HERA_GPU_EINVAL, "bad argument");
	out_off[0] = 0;
	if (n == 0)
		return HERA_GPU_OK;
	if (cudaSetDevice(b->device) != cudaSuccess)
		return bam_fail(b, HERA_GPU_ENODEV, "cudaSetDevice");
	// the extents of the host inputs
	const int per = paired ? 2 : 1;
	int64_t ext1 = 0, ext2 = 0;
	for (int32_t i = 0; i < n; ++i) {
		if (r1->len[i] < 0 || r1->off[i] < 0 || (paired && (r2->len[i] < 0 || r2->off[i] < 0)))
			return bam_fail(b, HERA_GPU_EINVAL, "negative read offset or length");
		ext1 = std::max<int64_t>(ext1, r1->off[i] + r1->len[i]);
		if (paired)
			ext2 = std::max<int64_t>(ext2, r2->off[i] + r2->len[i]);
	}
	for (int64_t k = 0; k < per * (int64_t)n; ++k)
		for (int s = 0; s < 2; ++s)
			if ((uint64_t)res->recs[k].list_off[s] + (uint32_t)res->recs[k].n[s] > res->list_used ||
			    (uint64_t)res->recs[k].cig_off[s] + res->recs[k].n_cigar[s] > res->op_used ||
			    (uint64_t)res->recs[k].miss_off[s] + res->recs[k].n_miss[s] > res->miss_used ||
			    res->recs[k].n[s] < 0)
				return bam_fail(b, HERA_GPU_EINVAL, "a record points outside its pools");
	for (int64_t k = 0; k < per * (int64_t)n; ++k)
		for (int s = 0; s < 2; ++s)
			for (int32_t j = 0; j < res->recs[k].n[s]; ++j)
				if (res->pos_pool[res->recs[k].list_off[s] + j] >= b->n_trans)
					return bam_fail(b, HERA_GPU_EINVAL, "a hit names no transcript of the gene map");
	for (int32_t i = 0; i < n; ++i)   // names end within their slots
		if (bamw::name_length(name1 + (int64_t)i * name_stride, name_stride) >= name_stride ||
		    (paired && bamw::name_length(name2 + (int64_t)i * name_stride, name_stride) >= name_stride))
			return bam_fail(b, HERA_GPU_EINVAL, "a read name without a NUL inside its slot");
	const cudaStream_t st = b->stream;
	const size_t nrec = (size_t)per * n, nl = res->list_used, no = res->op_used, nm = res->miss_used;
	const size_t names = (size_t)n * name_stride, names2 = paired ? names : 0;
	// one device block for the inputs, 16-byte aligned pieces
	size_t sz[12] = {nrec * sizeof(hera_cand_rec), nl * 4 + 4, nl * 4 + 4, no * 4 + 4, nm + 1,
			 (size_t)ext1 + 1, (size_t)ext2 + 1, (size_t)ext1 + 1, (size_t)ext2 + 1, names, names2,
			 (size_t)n * 2 * 8 + (size_t)n * 2 * 4};
	size_t at[12], total = 0;
	for (int k = 0; k < 12; ++k) {
		at[k] = total;
		total += (sz[k] + 15) & ~(size_t)15;
	}
	uint8_t *d_in = nullptr;
	unsigned long long *d_size = nullptr, *d_off = nullptr;
	uint32_t *d_err = nullptr;
	uint8_t *d_out = nullptr;
	void *d_tmp = nullptr;
	size_t tmp_bytes = 0;
	cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, (unsigned long long *)nullptr, (unsigned long long *)nullptr,
				      n + 1, st);
	cudaError_t e;
	int rc = HERA_GPU_OK;
	auto release = [&]() {
		cudaFree(d_in); cudaFree(d_size); cudaFree(d_off); cudaFree(d_err); cudaFree(d_out); cudaFree(d_tmp);
	};
	if ((e = cudaMalloc(&d_in, total)) != cudaSuccess || (e = cudaMalloc(&d_size, (n + 1) * 8ull)) != cudaSuccess ||
	    (e = cudaMalloc(&d_off, (n + 1) * 8ull)) != cudaSuccess || (e = cudaMalloc(&d_err, 16)) != cudaSuccess ||
	    (e = cudaMalloc(&d_tmp, tmp_bytes + 16)) != cudaSuccess) {
		release();
		return bam_fail(b, HERA_GPU_ENOMEM, "BAM inputs", e);
	}
	std::vector<int64_t> offs(2 * (size_t)n);
	std::vector<int32_t> lens(2 * (size_t)n);
	std::memcpy(offs.data(), r1->off, n * 8ull);
	std::memcpy(lens.data(), r1->len, n * 4ull);
	if (paired) {
		std::memcpy(offs.data() + n, r2->off, n * 8ull);
		std::memcpy(lens.data() + n, r2->len, n * 4ull);
	}
	const void *src[11] = {res->recs, res->pos_pool, res->p_pool, res->op_pool, res->miss_pool, r1->seq,
			       paired ? r2->seq : nullptr, qual1, qual2, name1, name2};
	const size_t len_src[11] = {nrec * sizeof(hera_cand_rec), nl * 4, nl * 4, no * 4, nm, (size_t)ext1,
				    (size_t)ext2, (size_t)ext1, (size_t)ext2, names, names2};
	cudaEventRecord(b->ev0, st);
	for (int k = 0; k < 11 && rc == HERA_GPU_OK; ++k)
		if (len_src[k] && (e = cudaMemcpyAsync(d_in + at[k], src[k], len_src[k], cudaMemcpyHostToDevice, st)) !=
				      cudaSuccess)
			rc = bam_fail(b, HERA_GPU_ECUDA, "BAM input copies", e);
	if (rc == HERA_GPU_OK &&
	    ((e = cudaMemcpyAsync(d_in + at[11], offs.data(), n * 16ull, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
	     (e = cudaMemcpyAsync(d_in + at[11] + n * 16ull, lens.data(), n * 8ull, cudaMemcpyHostToDevice, st)) !=
		     cudaSuccess ||
	     (e = cudaMemsetAsync(d_err, 0, 16, st)) != cudaSuccess))
		rc = bam_fail(b, HERA_GPU_ECUDA, "BAM input copies", e);
	if (rc != HERA_GPU_OK) {
		cudaStreamSynchronize(st);
		release();
		return rc;
	}
	bamk::Inputs in{};
	in.recs = (const hera_cand_rec *)(d_in + at[0]);
	in.pos = (const uint32_t *)(d_in + at[1]);
	in.pp = (const int32_t *)(d_in + at[2]);
	in.ops = (const uint32_t *)(d_in + at[3]);
	in.miss = (const char *)(d_in + at[4]);
	in.seq1 = (const char *)(d_in + at[5]);
	in.seq2 = (const char *)(d_in + at[6]);
	in.qual1 = (const char *)(d_in + at[7]);
	in.qual2 = (const char *)(d_in + at[8]);
	in.name1 = (const char *)(d_in + at[9]);
	in.name2 = (const char *)(d_in + at[10]);
	in.off1 = (const int64_t *)(d_in + at[11]);
	in.off2 = in.off1 + n;
	in.len1 = (const int32_t *)(d_in + at[11] + n * 16ull);
	in.len2 = in.len1 + n;
	in.stride = name_stride;
	in.ext1 = ext1;
	in.ext2 = ext2;
	in.nl = nl;
	in.no = no;
	in.nm = nm;
	const uint32_t *m = b->d_map;
	in.g = bamw::GeneMap{b->n_chr, m + b->off_chr_len, m + b->off_exon_off, m + b->off_starts, m + b->off_ends,
			     m + b->off_chr, m + b->off_gene};
	in.qual_table = m + b->off_qual;
	if (paired)
		bamk::k_bam_size<true><<<blocks_for((int64_t)n + 1, 128), 128, 0, st>>>(in, n, d_size, d_err);
	else
		bamk::k_bam_size<false><<<blocks_for((int64_t)n + 1, 128), 128, 0, st>>>(in, n, d_size, d_err);
	cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_size, d_off, n + 1, st);
	unsigned long long used = 0;
	uint32_t herr = 0;
	if ((e = cudaMemcpyAsync(&used, d_off + n, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
	    (e = cudaMemcpyAsync(&herr, d_err, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
	    (e = cudaStreamSynchronize(st)) != cudaSuccess) {
		release();
		return bam_fail(b, HERA_GPU_ECUDA, "BAM sizes", e);
	}
	if (herr & bamk::E_INPUT) {
		release();
		return bam_fail(b, HERA_GPU_EINVAL, "BAM inputs on the device outside their copies");
	}
	if (herr) {
		release();
		return bam_fail(b, HERA_GPU_ECAPACITY,
				herr & bamw::E_NAME ? "a read name the writer would cut twice"
						    : "a record beyond the writer's capacity or its gene map");
	}
	out_off[n] = used;
	if (used > cap) {
		release();
		return bam_fail(b, HERA_GPU_ECAPACITY, "BAM output buffer too small (out_off[n] holds the size)");
	}
	if ((e = cudaMalloc(&d_out, used + 16)) != cudaSuccess) {
		release();
		return bam_fail(b, HERA_GPU_ENOMEM, "BAM output", e);
	}
	if (paired)
		bamk::k_bam_write<true><<<blocks_for((int64_t)n, 128), 128, 0, st>>>(in, n, d_off, d_out, d_err);
	else
		bamk::k_bam_write<false><<<blocks_for((int64_t)n, 128), 128, 0, st>>>(in, n, d_off, d_out, d_err);
	cudaEventRecord(b->ev1, st);
	if ((e = cudaMemcpyAsync(out, d_out, used, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
	    (e = cudaMemcpyAsync(out_off, d_off, (n + 1) * 8ull, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
	    (e = cudaMemcpyAsync(&herr, d_err, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
	    (e = cudaStreamSynchronize(st)) != cudaSuccess) {
		release();
		return bam_fail(b, HERA_GPU_ECUDA, "BAM records", e);
	}
	if (herr) {
		release();
		return bam_fail(b, HERA_GPU_EINVAL, "BAM write pass: a pair's bytes differ from its size pass");
	}
	cudaEventElapsedTime(&b->kernel_ms, b->ev0, b->ev1);
	if (kernel_ms)
		*kernel_ms = b->kernel_ms;
	release();
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_bam_pairs(hera_gpu_bam *b, const hera_gpu_result *res, int32_t n, const hera_gpu_reads *r1,
				  const hera_gpu_reads *r2, const char *qual1, const char *qual2, const char *name1,
				  const char *name2, int32_t name_stride, uint8_t *out, uint64_t cap, uint64_t *out_off,
				  float *kernel_ms)
{
	if (!b)
		return HERA_GPU_EINVAL;
	if (!r2 || !qual2 || !name2)
		return bam_fail(b, HERA_GPU_EINVAL, "bad argument");
	return bam_run(b, res, n, r1, r2, qual1, qual2, name1, name2, name_stride, out, cap, out_off, kernel_ms);
}

extern "C" int hera_gpu_bam_single(hera_gpu_bam *b, const hera_gpu_result *res, int32_t n,
				   const hera_gpu_reads *reads, const char *qual, const char *name,
				   int32_t name_stride, uint8_t *out, uint64_t cap, uint64_t *out_off, float *kernel_ms)
{
	if (!b)
		return HERA_GPU_EINVAL;
	return bam_run(b, res, n, reads, nullptr, qual, nullptr, name, nullptr, name_stride, out, cap, out_off,
		       kernel_ms);
}
