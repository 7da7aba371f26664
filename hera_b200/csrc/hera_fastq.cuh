// hera_fastq.cuh -- FASTQ chunk parsing on the device.
//
// hera's worker loops take the reads of a chunk buffer one at a time with
// get_read_from_fq_buffer (src/read.c:11-63): a read is four lines -- '@'
// name, sequence, '+' line, a quality of the sequence's length -- and the
// chunk ends at its first NUL.  The device form finds every line at once and
// then judges every read independently:
//   k_fq_count   per 8 KiB tile: newlines (an exact SWAR zero-byte test on
//                16-byte loads) and the first NUL;
//   k_fq_scan    tile offsets (one block);
//   k_fq_lines   the newline positions, in order;
//   k_fq_ends    per file: the newlines before its end and where they start;
//   k_fq_recs    one thread per read: its line ends give the read's fields
//                and the reader's verdict (another read follows / the last
//                read / READ_FAIL); the first read not followed by another
//                is a min over the reads;
//   k_fq_pack    pairs interleaved in file order, and their lengths;
//   k_fq_gather  the sequences back to back for the aligner (warp a read).
// The host reads four ints per file to settle the read (pair) count the
// reference's loop reaches, or the read it rejects.
#pragma once

// (included at the end of hera_gpu.cu, outside its unnamed namespace)

namespace {
namespace fq {

constexpr int TILE = 8192;   // bytes per block
constexpr int TPB = 256;     // 32 bytes a thread
constexpr int SCAN_TPB = 1024;
constexpr int64_t MAX_BYTES = (int64_t)INT32_MAX - 4 * TILE;   // positions are int32

// info[] of a file: [0] first NUL (or n), [1] its newlines' base in nl[],
// [2] newlines before [0], [3] 4 * first read not followed by another +
// its verdict (1 last read, 2 READ_FAIL), [4] longest read of the result
constexpr int NINFO = 8;

struct File {
	const uint8_t *text;   // 256-byte aligned, readable up to a whole tile
	int64_t n;
	int32_t tiles, tile0;
	int32_t *info;
	hera_gpu_fastq_rec *rec;
	int32_t max_rec;       // reads a thread grid covers (n / 8 + 1)
};

struct Files {
	File f[2];
	int nf;
};

__device__ __forceinline__ uint32_t zero_bytes(uint32_t x)
{
	// 0x80 in every byte of x that is 0x00, nothing elsewhere
	return ~(((x & 0x7f7f7f7fu) + 0x7f7f7f7fu) | x | 0x7f7f7f7fu);
}

// newline and NUL flags (0x80 per byte) of the 32 bytes at p; bytes at or
// past n carry none
__device__ __forceinline__ void masks(const File &f, int64_t p, uint32_t (&nlm)[8], uint32_t (&nul)[8])
{
	const uint4 a = __ldg(reinterpret_cast<const uint4 *>(f.text + p));
	const uint4 b = __ldg(reinterpret_cast<const uint4 *>(f.text + p + 16));
	const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
	for (int k = 0; k < 8; ++k) {
		const int64_t left = f.n - (p + 4 * k);
		const uint32_t valid = left >= 4 ? 0x80808080u : (left <= 0 ? 0u : ((1u << (8 * left)) - 1u) & 0x80808080u);
		nlm[k] = zero_bytes(w[k] ^ 0x0a0a0a0au) & valid;
		nul[k] = zero_bytes(w[k]) & valid;
	}
}

__device__ __forceinline__ int file_of(const Files &F, int block)
{
	return F.nf > 1 && block >= F.f[1].tile0 ? 1 : 0;
}

// exclusive block scan of one int a thread (blockDim.x <= 1024); returns the
// block total in *total
__device__ __forceinline__ int block_excl(int v, int *sh, int *total)
{
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
	int x = v;
#pragma unroll
	for (int d = 1; d < 32; d <<= 1) {
		const int y = __shfl_up_sync(0xffffffffu, x, d);
		if (lane >= d)
			x += y;
	}
	if (lane == 31)
		sh[w] = x;
	__syncthreads();
	if (w == 0) {
		int s = lane < nw ? sh[lane] : 0;
#pragma unroll
		for (int d = 1; d < 32; d <<= 1) {
			const int y = __shfl_up_sync(0xffffffffu, s, d);
			if (lane >= d)
				s += y;
		}
		if (lane < nw)
			sh[lane] = s;   // inclusive
	}
	__syncthreads();
	const int before = w ? sh[w - 1] : 0;
	*total = sh[nw - 1];
	__syncthreads();
	return before + x - v;
}

__global__ void __launch_bounds__(TPB) k_fq_count(Files F, int32_t *__restrict__ tile_cnt)
{
	__shared__ int sh[32];
	const int fi = file_of(F, blockIdx.x);
	const File &f = F.f[fi];
	const int64_t p = (int64_t)(blockIdx.x - f.tile0) * TILE + threadIdx.x * 32;
	uint32_t nlm[8], nul[8];
	masks(f, p, nlm, nul);
	int c = 0, z = INT32_MAX;
#pragma unroll
	for (int k = 0; k < 8; ++k) {
		c += __popc(nlm[k]);
		if (nul[k] && z == INT32_MAX)
			z = (int)(p + 4 * k + ((__ffs(nul[k]) - 1) >> 3));
	}
	if (z != INT32_MAX)
		atomicMin(f.info + 0, z);
	int total;
	block_excl(c, sh, &total);
	if (threadIdx.x == 0)
		tile_cnt[blockIdx.x] = total;
}

// exclusive scan of cnt[0, n) into off[0, n]; one block of SCAN_TPB threads
__global__ void __launch_bounds__(SCAN_TPB) k_fq_scan(const int32_t *__restrict__ cnt, int n,
						       int32_t *__restrict__ off)
{
	__shared__ int sh[32];
	constexpr int PER = 8;
	int carry = 0;
	for (int base = 0; base < n; base += SCAN_TPB * PER) {
		int v[PER], s = 0;
		const int i0 = base + threadIdx.x * PER;
#pragma unroll
		for (int k = 0; k < PER; ++k) {
			v[k] = i0 + k < n ? cnt[i0 + k] : 0;
			s += v[k];
		}
		int total;
		int x = carry + block_excl(s, sh, &total);
#pragma unroll
		for (int k = 0; k < PER; ++k) {
			if (i0 + k < n)
				off[i0 + k] = x;
			x += v[k];
		}
		carry += total;
	}
	if (threadIdx.x == 0)
		off[n] = carry;
}

__global__ void __launch_bounds__(TPB) k_fq_lines(Files F, const int32_t *__restrict__ tile_off,
						   int32_t *__restrict__ nl)
{
	__shared__ int sh[32];
	const int fi = file_of(F, blockIdx.x);
	const File &f = F.f[fi];
	const int64_t p = (int64_t)(blockIdx.x - f.tile0) * TILE + threadIdx.x * 32;
	uint32_t nlm[8], nul[8];
	masks(f, p, nlm, nul);
	int c = 0;
#pragma unroll
	for (int k = 0; k < 8; ++k)
		c += __popc(nlm[k]);
	int total;
	int at = tile_off[blockIdx.x] + block_excl(c, sh, &total);
#pragma unroll
	for (int k = 0; k < 8; ++k) {
		uint32_t m = nlm[k];
		while (m) {
			nl[at++] = (int32_t)(p + 4 * k + ((__ffs(m) - 1) >> 3));
			m &= m - 1;
		}
	}
}

// per file: where its newlines start in nl[] and how many lie before its end
__global__ void k_fq_ends(Files F, const int32_t *__restrict__ tile_off, const int32_t *__restrict__ nl)
{
	const int fi = threadIdx.x;
	if (fi >= F.nf)
		return;
	const File &f = F.f[fi];
	const int32_t base = tile_off[f.tile0], cnt = tile_off[f.tile0 + f.tiles] - base;
	const int32_t z = f.info[0];
	int lo = 0, hi = cnt;   // first newline at or past z
	while (lo < hi) {
		const int mid = (lo + hi) >> 1;
		if (nl[base + mid] < z)
			lo = mid + 1;
		else
			hi = mid;
	}
	f.info[1] = base;
	f.info[2] = lo;
}

// One read (get_read_from_fq_buffer, src/read.c:11-63) per thread: read r
// of a file is lines 4r .. 4r+3 while every earlier read was followed by
// another.  Line j ends at the j-th newline before the file's end z, or at z
// (a NUL, or the end of the buffer) past the last one.  Verdicts: 0 another
// read follows, 1 READ_END (the quality ends at z, or z follows its
// newline), 2 READ_FAIL.  A read the reference reaches follows reads of 8
// bytes at least, so the first read not followed by another lies below
// n / 8 + 1 (max_rec); the reads judged are r <= min(newlines / 4,
// max_rec - 1), a grid-stride loop per file.
__device__ __forceinline__ void fq_rec(const File &f, const int32_t *__restrict__ L, int32_t m, int64_t r)
{
	const int64_t z = f.info[0];
	auto at = [&](int64_t k) -> uint8_t { return k < z ? f.text[k] : (uint8_t)0; };
	const int j = (int)(4 * r);
	int verdict = 2;
	hera_gpu_fastq_rec o{};
	do {
		const int64_t s0 = j == 0 ? 0 : (int64_t)L[j - 1] + 1;
		if (at(s0) != '@' || j >= m)
			break;
		o.name = s0 + 1;
		o.name_len = (int32_t)(L[j] - s0 - 1);
		if (j + 1 >= m)
			break;
		o.seq = (int64_t)L[j] + 1;
		o.len = (int32_t)(L[j + 1] - o.seq);
		if (o.len == 0)
			break;
		const int64_t s2 = (int64_t)L[j + 1] + 1;
		if (at(s2) != '+' || j + 2 >= m)
			break;
		o.qual = (int64_t)L[j + 2] + 1;
		const int64_t e3 = j + 3 < m ? (int64_t)L[j + 3] : z;
		if (e3 - o.qual != o.len)
			break;
		verdict = (j + 3 >= m || e3 + 1 == z) ? 1 : 0;
	} while (false);
	f.rec[r] = o;
	if (verdict)
		atomicMin(f.info + 3, (int32_t)(4 * r + verdict));
}

__global__ void __launch_bounds__(TPB) k_fq_recs(Files F, const int32_t *__restrict__ nl)
{
	const int64_t stride = (int64_t)gridDim.x * blockDim.x;
	for (int fi = 0; fi < F.nf; ++fi) {
		const File &f = F.f[fi];
		const int32_t m = f.info[2];
		const int64_t nrec = min((int64_t)m / 4 + 1, (int64_t)f.max_rec);
		const int32_t *L = nl + f.info[1];
		for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrec; r += stride)
			fq_rec(f, L, m, r);
	}
}

// reads of the result, interleaved by pair (mate 1, mate 2) or as they are
__global__ void k_fq_pack(Files F, int n, hera_gpu_fastq_rec *__restrict__ out, int32_t *__restrict__ len)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	int mx = 0;
	for (int fi = 0; fi < F.nf; ++fi) {
		const hera_gpu_fastq_rec o = F.f[fi].rec[i];
		out[(int64_t)F.nf * i + fi] = o;
		len[(int64_t)F.nf * i + fi] = o.len;
		mx = max(mx, o.len);
	}
	atomicMax(F.f[0].info + 4, mx);
}

// exclusive scan of 2n lengths into int64 offsets: per-block sums, a scan of
// those (k_fq_scan), then the blocks again
__global__ void __launch_bounds__(SCAN_TPB) k_fq_lsum(const int32_t *__restrict__ len, int64_t n,
						       int32_t *__restrict__ bsum)
{
	__shared__ int sh[32];
	const int64_t i = (int64_t)blockIdx.x * SCAN_TPB + threadIdx.x;
	int total;
	block_excl(i < n ? len[i] : 0, sh, &total);
	if (threadIdx.x == 0)
		bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_TPB) k_fq_loff(const int32_t *__restrict__ len, int64_t n,
						       const int32_t *__restrict__ boff, int64_t *__restrict__ off)
{
	__shared__ int sh[32];
	const int64_t i = (int64_t)blockIdx.x * SCAN_TPB + threadIdx.x;
	int total;
	const int x = block_excl(i < n ? len[i] : 0, sh, &total);
	if (i < n)
		off[i] = (int64_t)boff[blockIdx.x] + x;
}

// warp per read: its sequence to seq + off[i]
__global__ void k_fq_gather(Files F, const hera_gpu_fastq_rec *__restrict__ recs, int64_t n,
			    const int64_t *__restrict__ off, uint8_t *__restrict__ seq)
{
	const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (i >= n)
		return;
	const hera_gpu_fastq_rec o = recs[i];
	const uint8_t *src = F.f[F.nf > 1 ? (int)(i & 1) : 0].text + o.seq;
	uint8_t *dst = seq + off[i];
	for (int k = lane; k < o.len; k += 32)
		dst[k] = src[k];
}

}  // namespace fq
}  // namespace

struct FqState {
	std::mutex mu;
	cudaStream_t stream = nullptr;
	DBuf<uint8_t> text;                 // file 1 at 0, file 2 at a tile boundary
	DBuf<int32_t> tile_cnt, tile_off, nl, info, len, bsum, boff;
	DBuf<hera_gpu_fastq_rec> rec, out;  // per file (file 2 after file 1's max_rec), result
	DBuf<int64_t> off;
	DBuf<uint8_t> seq;
	HBuf<int32_t> h_info;
	fq::Files F{};                      // the last parse's files
	cudaEvent_t ev[7] = {};
	hera_gpu_fastq_stats stats{};
	void release()
	{
		text.release(); tile_cnt.release(); tile_off.release(); nl.release(); info.release();
		len.release(); bsum.release(); boff.release(); rec.release(); out.release(); off.release();
		seq.release(); h_info.release();
		for (auto &e : ev)
			if (e)
				cudaEventDestroy(e);
		if (stream)
			cudaStreamDestroy(stream);
	}
};

static void fq_release(hera_gpu_ctx *ctx)
{
	if (ctx->fq) {
		ctx->fq->release();
		delete ctx->fq;
		ctx->fq = nullptr;
	}
}

static int fq_state(hera_gpu_ctx *ctx, FqState **out)
{
	std::lock_guard<std::mutex> g(ctx->tune_mu);
	if (!ctx->fq) {
		FqState *s = new FqState();
		if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
			delete s;
			return HERA_GPU_ECUDA;
		}
		for (auto &e : s->ev)
			if (cudaEventCreate(&e) != cudaSuccess) {
				s->release();
				delete s;
				return HERA_GPU_ECUDA;
			}
		ctx->fq = s;
	}
	*out = ctx->fq;
	return HERA_GPU_OK;
}

// Parse nf chunk buffers on the device.  On HERA_GPU_OK, *n is the read
// (pair) count the reference's loop reaches and S.out / S.len hold the reads
// interleaved; HERA_GPU_EFORMAT gives the rejected file and read.
static int fq_parse(hera_gpu_ctx *ctx, FqState &S, const char *const *buf, const int64_t *bytes, int nf,
		    int32_t *n, int32_t *bad_file, int64_t *bad_read)
{
	using namespace fq;
	cudaStream_t st = S.stream;
	S.stats = hera_gpu_fastq_stats{};
	fq::Files F{};
	F.nf = nf;
	int64_t tb = 0, all = 0;
	int32_t tiles = 0, recs = 0;
	int64_t start[2] = {0, 0};
	for (int k = 0; k < nf; ++k) {
		if (bytes[k] < 0 || bytes[k] > MAX_BYTES || (bytes[k] > 0 && !buf[k]))
			return fail(ctx, HERA_GPU_EINVAL, "chunk buffer size");
		start[k] = tb;
		F.f[k].n = bytes[k];
		F.f[k].tiles = (int32_t)((bytes[k] + TILE - 1) / TILE);
		if (F.f[k].tiles == 0)
			F.f[k].tiles = 1;
		F.f[k].tile0 = tiles;
		F.f[k].max_rec = (int32_t)(bytes[k] / 8 + 1);
		tiles += F.f[k].tiles;
		tb += (int64_t)F.f[k].tiles * TILE;
		recs += F.f[k].max_rec;
		all += bytes[k];
	}
	// newlines: at most one a byte
	if (S.text.ensure((size_t)tb) != cudaSuccess || S.tile_cnt.ensure(tiles) != cudaSuccess ||
	    S.tile_off.ensure(tiles + 1) != cudaSuccess || S.info.ensure(NINFO * 2) != cudaSuccess ||
	    S.rec.ensure((size_t)recs) != cudaSuccess || S.h_info.ensure(NINFO * 2) != cudaSuccess ||
	    S.nl.ensure((size_t)all + 16) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENOMEM, "FASTQ parse buffers");
	int64_t rb = 0;
	for (int k = 0; k < nf; ++k) {
		F.f[k].text = S.text.p + start[k];
		F.f[k].info = S.info.p + NINFO * k;
		F.f[k].rec = S.rec.p + rb;
		rb += F.f[k].max_rec;
	}
	for (int k = 0; k < nf; ++k) {
		int32_t *I = S.h_info.p + NINFO * k;
		I[0] = (int32_t)bytes[k];
		I[1] = I[2] = 0;
		I[3] = INT32_MAX;
		for (int q = 4; q < NINFO; ++q)
			I[q] = 0;
	}
	S.F = F;
	cudaEventRecord(S.ev[0], st);
	for (int k = 0; k < nf; ++k)
		if (bytes[k] > 0)
			cudaMemcpyAsync(S.text.p + start[k], buf[k], (size_t)bytes[k], cudaMemcpyHostToDevice, st);
	cudaMemcpyAsync(S.info.p, S.h_info.p, sizeof(int32_t) * NINFO * nf, cudaMemcpyHostToDevice, st);
	cudaEventRecord(S.ev[1], st);
	k_fq_count<<<tiles, fq::TPB, 0, st>>>(F, S.tile_cnt.p);
	k_fq_scan<<<1, SCAN_TPB, 0, st>>>(S.tile_cnt.p, tiles, S.tile_off.p);
	k_fq_lines<<<tiles, fq::TPB, 0, st>>>(F, S.tile_off.p, S.nl.p);
	k_fq_ends<<<1, 32, 0, st>>>(F, S.tile_off.p, S.nl.p);
	{
		const int64_t want = (recs + fq::TPB - 1) / fq::TPB;
		k_fq_recs<<<(unsigned)std::min<int64_t>(want, (int64_t)ctx->sms * 16), fq::TPB, 0, st>>>(F, S.nl.p);
	}
	S.stats.launches = 5;
	cudaEventRecord(S.ev[2], st);
	cudaMemcpyAsync(S.h_info.p, S.info.p, sizeof(int32_t) * NINFO * nf, cudaMemcpyDeviceToHost, st);
	cudaError_t e = cudaStreamSynchronize(st);
	if (e != cudaSuccess)
		return fail(ctx, HERA_GPU_ECUDA, "FASTQ parse", e);
	S.stats.bytes = all;
	// the reference's loop: file 1's read, then file 2's, stop after a pair
	// with a last read; a READ_FAIL of file 1 is met before file 2's
	int32_t k_stop[2], v[2];
	for (int k = 0; k < nf; ++k) {
		const int32_t key = S.h_info.p[NINFO * k + 3];
		if (key == INT32_MAX)
			return fail(ctx, HERA_GPU_ECUDA, "FASTQ parse: no last read");
		k_stop[k] = key >> 2;
		v[k] = key & 3;
	}
	int32_t kk = k_stop[0];
	for (int k = 1; k < nf; ++k)
		kk = k_stop[k] < kk ? k_stop[k] : kk;
	for (int k = 0; k < nf; ++k)
		if (k_stop[k] == kk && v[k] == 2) {
			*bad_file = k + 1;
			*bad_read = kk;
			*n = 0;
			return HERA_GPU_EFORMAT;
		}
	*n = kk + 1;
	*bad_file = 0;
	*bad_read = -1;
	if (S.out.ensure((size_t)nf * *n) != cudaSuccess || S.len.ensure((size_t)nf * *n) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENOMEM, "FASTQ parse outputs");
	cudaEventRecord(S.ev[3], st);
	k_fq_pack<<<(*n + 255) / 256, 256, 0, st>>>(F, *n, S.out.p, S.len.p);
	++S.stats.launches;
	cudaEventRecord(S.ev[4], st);
	S.stats.reads = (int64_t)nf * *n;
	return HERA_GPU_OK;
}

// device times: chunk copies; the parse kernels (the host's look at the
// read counts between them left out); the sequence gather
static void fq_times(FqState &S, bool gather)
{
	cudaEventSynchronize(gather ? S.ev[6] : S.ev[4]);
	float a = 0, b = 0;
	cudaEventElapsedTime(&S.stats.h2d_ms, S.ev[0], S.ev[1]);
	cudaEventElapsedTime(&a, S.ev[1], S.ev[2]);
	cudaEventElapsedTime(&b, S.ev[3], S.ev[4]);
	S.stats.parse_ms = a + b;
	S.stats.gather_ms = 0;
	if (gather)
		cudaEventElapsedTime(&S.stats.gather_ms, S.ev[5], S.ev[6]);
}

static int fq_parse_host(hera_gpu_ctx *ctx, const char *const *buf, const int64_t *bytes, int nf,
			 hera_gpu_fastq_rec *recs, int32_t cap, int32_t *n, int32_t *bad_file, int64_t *bad_read)
{
	FqState *S = nullptr;
	if (int rc = fq_state(ctx, &S))
		return fail(ctx, rc, "FASTQ parse state");
	std::lock_guard<std::mutex> g(S->mu);
	if (cudaSetDevice(ctx->device) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENODEV, "cudaSetDevice");
	int rc = fq_parse(ctx, *S, buf, bytes, nf, n, bad_file, bad_read);
	if (rc != HERA_GPU_OK)
		return rc == HERA_GPU_EFORMAT ? fail(ctx, rc, "chunk not in hera's FASTQ form") : rc;
	fq_times(*S, false);
	if (*n > cap)
		return fail(ctx, HERA_GPU_ECAPACITY, "more reads than the record array holds");
	cudaError_t e = cudaMemcpyAsync(recs, S->out.p, sizeof(hera_gpu_fastq_rec) * nf * (size_t)*n,
					cudaMemcpyDeviceToHost, S->stream);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(S->stream);
	if (e != cudaSuccess)
		return fail(ctx, HERA_GPU_ECUDA, "FASTQ records", e);
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_parse_fastq_pairs(hera_gpu_ctx *ctx, const char *left, int64_t n_left, const char *right,
					  int64_t n_right, hera_gpu_fastq_rec *recs, int32_t cap, int32_t *n_pairs,
					  int32_t *bad_file, int64_t *bad_read)
{
	if (!ctx || !recs || cap < 0 || !n_pairs || !bad_file || !bad_read)
		return HERA_GPU_EINVAL;
	const char *buf[2] = {left, right};
	const int64_t bytes[2] = {n_left, n_right};
	return fq_parse_host(ctx, buf, bytes, 2, recs, cap, n_pairs, bad_file, bad_read);
}

extern "C" int hera_gpu_parse_fastq_single(hera_gpu_ctx *ctx, const char *chunk, int64_t n, hera_gpu_fastq_rec *recs,
					   int32_t cap, int32_t *n_reads, int64_t *bad_read)
{
	if (!ctx || !recs || cap < 0 || !n_reads || !bad_read)
		return HERA_GPU_EINVAL;
	const char *buf[1] = {chunk};
	const int64_t bytes[1] = {n};
	int32_t bf = 0;
	return fq_parse_host(ctx, buf, bytes, 1, recs, cap, n_reads, &bf, bad_read);
}

extern "C" int hera_gpu_align_fastq_pairs(hera_gpu_ctx *ctx, const char *left, int64_t n_left, const char *right,
					  int64_t n_right, int write_bam, hera_gpu_fastq_rec *recs, int32_t cap,
					  int32_t *n_pairs, int32_t *bad_file, int64_t *bad_read,
					  hera_gpu_result *out)
{
	using namespace fq;
	if (!ctx || !recs || cap < 0 || !n_pairs || !bad_file || !bad_read || !out ||
	    (write_bam != 0 && write_bam != 1))
		return HERA_GPU_EINVAL;
	if (n_left < 0 || n_right < 0 || n_left + n_right > MAX_BYTES)
		return fail(ctx, HERA_GPU_EINVAL, "chunk buffer size");
	FqState *S = nullptr;
	if (int rc = fq_state(ctx, &S))
		return fail(ctx, rc, "FASTQ parse state");
	std::lock_guard<std::mutex> g(S->mu);
	if (cudaSetDevice(ctx->device) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENODEV, "cudaSetDevice");
	const char *buf[2] = {left, right};
	const int64_t bytes[2] = {n_left, n_right};
	int rc = fq_parse(ctx, *S, buf, bytes, 2, n_pairs, bad_file, bad_read);
	if (rc != HERA_GPU_OK)
		return rc == HERA_GPU_EFORMAT ? fail(ctx, rc, "chunk not in hera's FASTQ form") : rc;
	const int32_t n = *n_pairs;
	if (n > cap)
		return fail(ctx, HERA_GPU_ECAPACITY, "more pairs than the record array holds");
	cudaStream_t st = S->stream;
	// sequences back to back for the aligner (read 2i mate 1, 2i+1 mate 2)
	const int64_t nr = 2 * (int64_t)n;
	const int nb = (int)((nr + SCAN_TPB - 1) / SCAN_TPB);
	if (S->bsum.ensure(nb + 1) != cudaSuccess || S->boff.ensure(nb + 1) != cudaSuccess ||
	    S->off.ensure((size_t)nr + 1) != cudaSuccess || S->seq.ensure((size_t)(n_left + n_right) + 64) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENOMEM, "FASTQ gather buffers");
	const fq::Files &F = S->F;
	cudaEventRecord(S->ev[5], st);
	k_fq_lsum<<<nb, SCAN_TPB, 0, st>>>(S->len.p, nr, S->bsum.p);
	k_fq_scan<<<1, SCAN_TPB, 0, st>>>(S->bsum.p, nb, S->boff.p);
	k_fq_loff<<<nb, SCAN_TPB, 0, st>>>(S->len.p, nr, S->boff.p, S->off.p);
	k_fq_gather<<<(unsigned)((nr * 32 + 255) / 256), 256, 0, st>>>(F, S->out.p, nr, S->off.p, S->seq.p);
	S->stats.launches += 4;
	cudaEventRecord(S->ev[6], st);
	int32_t max_len = 0;
	cudaError_t e = cudaMemcpyAsync(&max_len, S->info.p + 4, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(recs, S->out.p, sizeof(hera_gpu_fastq_rec) * nr, cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(st);
	if (e != cudaSuccess)
		return fail(ctx, HERA_GPU_ECUDA, "FASTQ gather", e);
	fq_times(*S, true);
	if (max_len > MAX_READ)
		return fail(ctx, HERA_GPU_EINVAL, "a read is longer than HERA_GPU_MAX_READ");
	rc = hera_gpu_align_pairs_device(ctx, S->seq.p, S->off.p, S->len.p, n, max_len < 1 ? 1 : max_len, write_bam,
					 st);
	if (rc != HERA_GPU_OK)
		return rc;
	return hera_gpu_fetch_result(ctx, out);
}

extern "C" int hera_gpu_get_fastq_stats(hera_gpu_ctx *ctx, hera_gpu_fastq_stats *out)
{
	if (!ctx || !out)
		return HERA_GPU_EINVAL;
	*out = ctx->fq ? ctx->fq->stats : hera_gpu_fastq_stats{};
	return HERA_GPU_OK;
}

extern "C" int hera_gpu_fastq_read_inf(char *buf, int64_t n, const hera_gpu_fastq_rec *recs, int32_t count,
				       int32_t stride, hera_read_inf *out)
{
	if ((!buf && count > 0) || n < 0 || count < 0 || stride < 1 || (count > 0 && (!recs || !out)))
		return HERA_GPU_EINVAL;
	for (int32_t i = 0; i < count; ++i) {
		const hera_gpu_fastq_rec &r = recs[(int64_t)i * stride];
		if (r.name < 1 || r.name + r.name_len >= n || r.seq + r.len >= n || r.qual + r.len > n || r.len < 1)
			return HERA_GPU_EINVAL;
	}
	for (int32_t i = 0; i < count; ++i) {
		const hera_gpu_fastq_rec &r = recs[(int64_t)i * stride];
		// the reader's NULs: over the newlines ending the name, the sequence
		// and the quality (src/read.c:26, 36, 58)
		buf[r.name + r.name_len] = '\0';
		buf[r.seq + r.len] = '\0';
		if (r.qual + r.len < n)
			buf[r.qual + r.len] = '\0';
		out[i].name = buf + r.name;
		out[i].seq = buf + r.seq;
		out[i].qual = buf + r.qual;
		out[i].len = r.len;
	}
	return HERA_GPU_OK;
}
