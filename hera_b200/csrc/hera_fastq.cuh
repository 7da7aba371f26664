// hera_fastq.cuh -- FASTQ chunk parsing on the device.
//
// hera's worker loops take the reads of a chunk buffer one at a time with
// get_read_from_fq_buffer (src/read.c:11-63): a read is four lines -- '@'
// name, sequence, '+' line, a quality of the sequence's length -- and the
// chunk ends at its first NUL.  The device form finds every line at once and
// then judges every read independently:
//   k_fq_count   per 8 KiB tile: newlines (an exact SWAR zero-byte test on
//                16-byte loads) as one bit a byte, with bits for a newline
//                followed by '@' or by '+', their count, and the first NUL
//                -- the one pass over the text;
//   k_fq_scan    tile offsets (one block);
//   k_fq_lines   from the bits: the newline positions, in order, and the
//                class of the line each one starts ('@', '+', other);
//   k_fq_ends    per file: the newlines before its end and where they start;
//   k_fq_recs    one thread per read: its line ends give the read's fields
//                and the reader's verdict (another read follows / the last
//                read / READ_FAIL), written interleaved by pair; the first
//                read not followed by another is a min over the reads;
//   k_fq_gather  the sequences for the aligner, each in a 16-byte aligned
//                slot (warp a read, 4-byte words).
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
// its verdict (1 last read, 2 READ_FAIL); info[4] of file 1: the longest
// read of the result (set by the gather's length scan)
constexpr int NINFO = 8;

struct File {
	const uint8_t *text;   // 256-byte aligned, readable up to a whole tile
	int64_t n;
	int32_t tiles, tile0;
	int32_t *info;
	int32_t max_rec;       // reads that can be judged (n / 8 + 1)
};

struct Files {
	File f[2];
	int nf;
	uint32_t *bits;            // three planes of a bit a byte (see k_fq_count)
	size_t plane;              // words a plane
	hera_gpu_fastq_rec *out;   // reads interleaved by pair (nf * max max_rec)
	int32_t *len;              // their lengths
};

__device__ __forceinline__ uint32_t zero_bytes(uint32_t x)
{
	// 0x80 in every byte of x that is 0x00, nothing elsewhere
	return ~(((x & 0x7f7f7f7fu) + 0x7f7f7f7fu) | x | 0x7f7f7f7fu);
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

// 0x80 byte flags (bits 7, 15, 23, 31) -> 4 bits: after the shift the flags
// sit at bits 0, 8, 16, 24; the multiply by 1 + 2^7 + 2^14 + 2^21 lands them
// at 21, 22, 23, 24 with no other term there (so no carries)
__device__ __forceinline__ uint32_t flags4(uint32_t x)
{
	return (((x >> 7) * 0x00204081u) >> 21) & 15u;
}

// A tile per block of PASS_TPB threads, 128 bytes (eight 16-byte loads issued
// together) a thread.  Bit planes of the tile, one word per 32 bytes:
// newlines; newlines followed by '@'; newlines followed by '+' (bytes at or
// past n carry none; a line class is checked against the file's end too).
constexpr int PASS_TPB = TPB / 4;
constexpr int WORDS = TILE / 32;   // bit words of a tile

__global__ void __launch_bounds__(PASS_TPB) k_fq_count(Files F, int32_t *__restrict__ tile_cnt)
{
	__shared__ int sh[32];
	const int fi = file_of(F, blockIdx.x);
	const File f = fi ? F.f[1] : F.f[0];
	const int64_t p = (int64_t)(blockIdx.x - f.tile0) * TILE + threadIdx.x * 128;
	uint32_t w[33];
#pragma unroll
	for (int k = 0; k < 8; ++k) {
		const uint4 q = __ldg(reinterpret_cast<const uint4 *>(f.text + p) + k);
		w[4 * k] = q.x;
		w[4 * k + 1] = q.y;
		w[4 * k + 2] = q.z;
		w[4 * k + 3] = q.w;
	}
	w[32] = p + 128 < f.n ? f.text[p + 128] : 0u;   // the byte after the 128
	const bool whole = p + 128 <= f.n;
	int z = INT32_MAX, c = 0;
#pragma unroll
	for (int g = 0; g < 4; ++g) {   // 32-byte groups: one word of each plane
		uint32_t nlb = 0, atb = 0, plb = 0;
#pragma unroll
		for (int e = 0; e < 8; ++e) {
			const int k = 8 * g + e;
			uint32_t valid = 0x80808080u;
			if (!whole) {
				const int64_t left = f.n - (p + 4 * k);
				valid = left >= 4 ? 0x80808080u
						  : (left <= 0 ? 0u : ((1u << (8 * left)) - 1u) & 0x80808080u);
			}
			const uint32_t nlf = zero_bytes(w[k] ^ 0x0a0a0a0au) & valid;
			const uint32_t nul = zero_bytes(w[k]) & valid;
			if (nul && z == INT32_MAX)
				z = (int)(p + 4 * k + ((__ffs(nul) - 1) >> 3));
			if (nlf) {
				// each byte's next byte, and whether it is '@' / '+'
				const uint32_t nx = __funnelshift_r(w[k], w[k + 1], 8);
				nlb |= flags4(nlf) << (4 * e);
				atb |= flags4(nlf & zero_bytes(nx ^ 0x40404040u)) << (4 * e);
				plb |= flags4(nlf & zero_bytes(nx ^ 0x2b2b2b2bu)) << (4 * e);
			}
		}
		const size_t wi = (size_t)blockIdx.x * WORDS + 4 * threadIdx.x + g;
		F.bits[wi] = nlb;
		F.bits[F.plane + wi] = atb;
		F.bits[2 * F.plane + wi] = plb;
		c += __popc(nlb);
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

// a tile per block of PASS_TPB threads, 128 bytes (four bit words) a thread;
// cls of the line a newline starts: 1 '@', 2 '+', 0 other
__global__ void __launch_bounds__(PASS_TPB) k_fq_lines(Files F, const int32_t *__restrict__ tile_off,
							int32_t *__restrict__ nl, uint8_t *__restrict__ cls)
{
	__shared__ int sh[32];
	const int fi = file_of(F, blockIdx.x);
	const File f = fi ? F.f[1] : F.f[0];
	const size_t w0 = (size_t)blockIdx.x * WORDS + 4 * threadIdx.x;
	const int64_t p = (int64_t)(blockIdx.x - f.tile0) * TILE + threadIdx.x * 128;
	const uint4 m4 = *reinterpret_cast<const uint4 *>(F.bits + w0);
	const uint4 a4 = *reinterpret_cast<const uint4 *>(F.bits + F.plane + w0);
	const uint4 p4 = *reinterpret_cast<const uint4 *>(F.bits + 2 * F.plane + w0);
	const uint32_t m[4] = {m4.x, m4.y, m4.z, m4.w}, ma[4] = {a4.x, a4.y, a4.z, a4.w},
		       mp[4] = {p4.x, p4.y, p4.z, p4.w};
	const int c = __popc(m[0]) + __popc(m[1]) + __popc(m[2]) + __popc(m[3]);
	int total;
	int at = tile_off[blockIdx.x] + block_excl(c, sh, &total);
#pragma unroll
	for (int k = 0; k < 4; ++k) {
		uint32_t x = m[k];
		while (x) {
			const uint32_t lo = x & (0u - x);
			nl[at] = (int32_t)(p + 32 * k + __ffs(x) - 1);
			cls[at] = (ma[k] & lo) ? 1 : ((mp[k] & lo) ? 2 : 0);
			++at;
			x &= x - 1;
		}
	}
}

// per file: where its newlines start in nl[] and how many lie before its end
__global__ void k_fq_ends(Files F, const int32_t *__restrict__ tile_off, const int32_t *__restrict__ nl)
{
	const int fi = threadIdx.x;
	if (fi >= F.nf)
		return;
	const File f = fi ? F.f[1] : F.f[0];
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
__device__ __forceinline__ void fq_rec(const Files &F, int fi, const int32_t *__restrict__ L,
				       const uint8_t *__restrict__ cls, int32_t m, int64_t r)
{
	const File f = fi ? F.f[1] : F.f[0];
	const int64_t z = f.info[0];
	// line j's first byte is '@' / '+' (the file's first line read from the text)
	auto first_is = [&](int j, int64_t s, uint8_t ch, uint8_t c) -> bool {
		if (s >= z)
			return false;
		return j == 0 ? f.text[0] == ch : cls[j - 1] == c;
	};
	const int j = (int)(4 * r);
	int verdict = 2;
	hera_gpu_fastq_rec o{};
	do {
		const int64_t s0 = j == 0 ? 0 : (int64_t)L[j - 1] + 1;
		if (!first_is(j, s0, '@', 1) || j >= m)
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
		if (!first_is(j + 2, s2, '+', 2) || j + 2 >= m)
			break;
		o.qual = (int64_t)L[j + 2] + 1;
		const int64_t e3 = j + 3 < m ? (int64_t)L[j + 3] : z;
		if (e3 - o.qual != o.len)
			break;
		verdict = (j + 3 >= m || e3 + 1 == z) ? 1 : 0;
	} while (false);
	F.out[(int64_t)F.nf * r + fi] = o;
	F.len[(int64_t)F.nf * r + fi] = o.len;
	if (verdict)
		atomicMin(f.info + 3, (int32_t)(4 * r + verdict));
}

__global__ void __launch_bounds__(TPB) k_fq_recs(Files F, const int32_t *__restrict__ nl,
						  const uint8_t *__restrict__ cls)
{
	const int64_t stride = (int64_t)gridDim.x * blockDim.x;
	for (int fi = 0; fi < F.nf; ++fi) {
		const File f = fi ? F.f[1] : F.f[0];
		const int32_t m = f.info[2];
		const int64_t nrec = min((int64_t)m / 4 + 1, (int64_t)f.max_rec);
		const int32_t *L = nl + f.info[1];
		const uint8_t *C = cls + f.info[1];
		for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nrec; r += stride)
			fq_rec(F, fi, L, C, m, r);
	}
}

// Offsets of the aligner's read slots: an exclusive scan of the lengths
// rounded up to 16 bytes (per-block sums, a scan of those with k_fq_scan,
// the blocks again); the first pass also takes the longest read.
__device__ __forceinline__ int slot_bytes(int len) { return (len + 15) & ~15; }

__global__ void __launch_bounds__(SCAN_TPB) k_fq_lsum(const int32_t *__restrict__ len, int64_t n,
						       int32_t *__restrict__ bsum, int32_t *__restrict__ max_len)
{
	__shared__ int sh[32];
	const int64_t i = (int64_t)blockIdx.x * SCAN_TPB + threadIdx.x;
	const int L = i < n ? len[i] : 0;
	int total;
	block_excl(slot_bytes(L), sh, &total);
	if (threadIdx.x == 0)
		bsum[blockIdx.x] = total;
	const int mx = __reduce_max_sync(0xffffffffu, L);
	if ((threadIdx.x & 31) == 0 && mx > 0)
		atomicMax(max_len, mx);
}

__global__ void __launch_bounds__(SCAN_TPB) k_fq_loff(const int32_t *__restrict__ len, int64_t n,
						       const int32_t *__restrict__ boff, int64_t *__restrict__ off)
{
	__shared__ int sh[32];
	const int64_t i = (int64_t)blockIdx.x * SCAN_TPB + threadIdx.x;
	int total;
	const int x = block_excl(i < n ? slot_bytes(len[i]) : 0, sh, &total);
	if (i < n)
		off[i] = (int64_t)boff[blockIdx.x] + x;
}

// warp per read: its sequence into its 16-byte aligned slot, lane k on the
// slot's 4-byte words k, k + 32, ... (two aligned source words and a
// funnel shift each; the slot's bytes past the read are don't-care)
__global__ void k_fq_gather(Files F, const hera_gpu_fastq_rec *__restrict__ recs, int64_t n,
			    const int64_t *__restrict__ off, uint8_t *__restrict__ seq)
{
	const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	const int lane = threadIdx.x & 31;
	if (i >= n)
		return;
	const hera_gpu_fastq_rec o = recs[i];
	const uint8_t *src = (F.nf > 1 && (i & 1) ? F.f[1].text : F.f[0].text) + o.seq;
	uint32_t *dst = reinterpret_cast<uint32_t *>(seq + off[i]);
	const uintptr_t sa = reinterpret_cast<uintptr_t>(src);
	const uint32_t *sw = reinterpret_cast<const uint32_t *>(sa & ~(uintptr_t)3);
	const unsigned sh = 8u * (unsigned)(sa & 3);
	const int words = (o.len + 3) >> 2;
	for (int k = lane; k < words; k += 32)
		dst[k] = __funnelshift_r(sw[k], sw[k + 1], sh);
}

}  // namespace fq
}  // namespace

struct FqState {
	std::mutex mu;
	cudaStream_t stream = nullptr;
	DBuf<uint8_t> text;                 // file 1 at 0, file 2 at a tile boundary
	DBuf<int32_t> tile_cnt, tile_off, nl, info, len, bsum, boff;
	DBuf<uint32_t> bits;
	DBuf<uint8_t> cls;
	DBuf<hera_gpu_fastq_rec> out;       // reads interleaved by pair
	DBuf<int64_t> off;
	DBuf<uint8_t> seq;
	HBuf<int32_t> h_info;
	fq::Files F{};                      // the last parse's files
	cudaEvent_t ev[7] = {};
	hera_gpu_fastq_stats stats{};
	void release()
	{
		text.release(); tile_cnt.release(); tile_off.release(); nl.release(); info.release();
		len.release(); bsum.release(); boff.release(); bits.release(); cls.release(); out.release();
		off.release();
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
// (pair) count the reference's loop reaches and the first nf * n entries of
// S.out / S.len hold its reads interleaved; HERA_GPU_EFORMAT gives the
// rejected file and read.
static int fq_parse(hera_gpu_ctx *ctx, FqState &S, const char *const *buf, const int64_t *bytes, int nf,
		    int32_t *n, int32_t *bad_file, int64_t *bad_read)
{
	using namespace fq;
	cudaStream_t st = S.stream;
	S.stats = hera_gpu_fastq_stats{};
	fq::Files F{};
	F.nf = nf;
	int64_t tb = 0, all = 0;
	int32_t tiles = 0, recs = 0, most = 0;
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
		most = std::max(most, F.f[k].max_rec);
		all += bytes[k];
	}
	// text: whole tiles and 64 bytes the gather's word loads may pass over;
	// newlines: at most one a byte
	if (S.text.ensure((size_t)tb + 64) != cudaSuccess || S.tile_cnt.ensure(tiles) != cudaSuccess ||
	    S.tile_off.ensure(tiles + 1) != cudaSuccess || S.info.ensure(NINFO * 2) != cudaSuccess ||
	    S.bits.ensure((size_t)tiles * fq::WORDS * 3) != cudaSuccess || S.h_info.ensure(NINFO * 2) != cudaSuccess ||
	    S.nl.ensure((size_t)all + 16) != cudaSuccess || S.cls.ensure((size_t)all + 16) != cudaSuccess ||
	    S.out.ensure((size_t)nf * most) != cudaSuccess ||
	    S.len.ensure((size_t)nf * most) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENOMEM, "FASTQ parse buffers");
	F.bits = S.bits.p;
	F.plane = (size_t)tiles * fq::WORDS;
	F.out = S.out.p;
	F.len = S.len.p;
	for (int k = 0; k < nf; ++k) {
		F.f[k].text = S.text.p + start[k];
		F.f[k].info = S.info.p + NINFO * k;
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
	k_fq_count<<<tiles, fq::PASS_TPB, 0, st>>>(F, S.tile_cnt.p);
	k_fq_scan<<<1, SCAN_TPB, 0, st>>>(S.tile_cnt.p, tiles, S.tile_off.p);
	k_fq_lines<<<tiles, fq::PASS_TPB, 0, st>>>(F, S.tile_off.p, S.nl.p, S.cls.p);
	k_fq_ends<<<1, 32, 0, st>>>(F, S.tile_off.p, S.nl.p);
	{
		const int64_t want = (recs + fq::TPB - 1) / fq::TPB;
		k_fq_recs<<<(unsigned)std::min<int64_t>(want, (int64_t)ctx->sms * 16), fq::TPB, 0, st>>>(F, S.nl.p,
													     S.cls.p);
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
	S.stats.reads = (int64_t)nf * *n;
	return HERA_GPU_OK;
}

// device times: chunk copies, parse kernels, sequence gather
static void fq_times(FqState &S, bool gather)
{
	cudaEventSynchronize(gather ? S.ev[6] : S.ev[2]);
	cudaEventElapsedTime(&S.stats.h2d_ms, S.ev[0], S.ev[1]);
	cudaEventElapsedTime(&S.stats.parse_ms, S.ev[1], S.ev[2]);
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
	// sequences in rising 16-byte slots for the aligner (read 2i mate 1,
	// 2i+1 mate 2)
	const int64_t nr = 2 * (int64_t)n;
	const int nb = (int)((nr + SCAN_TPB - 1) / SCAN_TPB);
	if (S->bsum.ensure(nb + 1) != cudaSuccess || S->boff.ensure(nb + 1) != cudaSuccess ||
	    S->off.ensure((size_t)nr + 1) != cudaSuccess ||
	    S->seq.ensure((size_t)(n_left + n_right) + 16 * (size_t)nr + 64) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENOMEM, "FASTQ gather buffers");
	const fq::Files &F = S->F;
	cudaEventRecord(S->ev[5], st);
	k_fq_lsum<<<nb, SCAN_TPB, 0, st>>>(S->len.p, nr, S->bsum.p, S->info.p + 4);
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
