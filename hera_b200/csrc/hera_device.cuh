// hera_device.cuh -- device-side algorithms of the hera read-alignment hot
// path for sm_100a.  One CUDA thread runs one task (a get_position call, a
// pair's control flow, or one mate rescue); per-task working sets live in
// local memory (L1-backed), per-pair Candidate state in HBM.
//
// Each routine restates one reference function; the cited file:line is the
// behaviour it must reproduce bit for bit (reference = bioturing/hera).
#pragma once

#include <cstdint>

namespace hg {

constexpr int KMER = 31;
constexpr int ERR = 7;
constexpr int MAX_FRAG = 1000;
constexpr int HBITS = 27;
constexpr uint64_t HMASK = (1ull << HBITS) - 1;
constexpr int MAX_READ = 320;          // HERA_GPU_MAX_READ
constexpr int MAX_DP_ROWS = MAX_READ;  // rows of one gap DP (<= read length)
constexpr int BW = 24;                 // gap-DP band width (bound: 2*error+2 = 18)
// Per-read capacities.  The reference grows every list without bound; the
// device keeps fixed-size per-task state, in two sizes.  The first pass
// (every pair) uses CapsStd.  A pair that passes one of its capacities is
// flagged and aligned again, alone, in a second pass with CapsWide, whose
// CIGAR and miss bounds hold for any read up to MAX_READ (a traceback takes
// at most read + window steps, 320 + 1000) and whose anchor and list bounds
// are 32x the first pass's.
struct CapsStd {
	static constexpr int A = 256;     // anchors of one get_position call
	static constexpr int L = 64;      // hits kept per Candidate strand
	static constexpr int C = 96;      // CIGAR ops per Candidate strand
	static constexpr int M = 96;      // miss chars per Candidate strand
};
struct CapsWide {
	static constexpr int A = 8192;
	static constexpr int L = 8192;
	static constexpr int C = 1344;
	static constexpr int M = 1344;
};
constexpr int ACAP = CapsStd::A;
constexpr int LCAP = CapsStd::L;
constexpr int CCAP = CapsStd::C;
constexpr int MCAP = CapsStd::M;

enum : int { OP_M = 0, OP_I = 1, OP_D = 2, OP_S = 4, OP_X = 8 };

// capacity / consistency flags (OR-ed into one word per batch)
enum : int {
	F_ACAP = 1, F_LCAP = 2, F_CCAP = 4, F_MCAP = 8, F_BAND = 16, F_READ = 32,
	F_SCRATCH = 64, F_QUEUE = 128, F_SSW = 256,
	F_WIDE = 512    // (host) a capacity was met again in the wide pass
};
// the flags a second, wide pass clears (per-read list capacities)
constexpr int F_CAPS = F_ACAP | F_LCAP | F_CCAP | F_MCAP;

struct DevIndex {
	const uint32_t *boff;    // [2^27 + 1] bucket start offsets
	const uint4 *bk;         // buckets {id lo, id hi, start, end}
	const uint2 *occ;        // occurrences {transcript, offset}
	const uint8_t *seq;      // transcript ASCII, zero padded
	const uint8_t *code;     // transcript codes 0..4, padded with 4
	const uint32_t *tlen;    // transcript lengths
	const uint32_t *tstart;  // transcript start offsets in seq
	uint32_t n_trans;
};

// ascii_table (src/hash_align.c:6-23): A/a 0, C/c 1, G/g 2, T/t 3, else 4
__device__ __forceinline__ uint8_t code_of(uint8_t c)
{
	uint8_t x = c | 0x20;
	return x == 'a' ? 0 : x == 'c' ? 1 : x == 'g' ? 2 : x == 't' ? 3 : 4;
}

__device__ __forceinline__ uint8_t comp_code(uint8_t c)
{
	return c < 4 ? (uint8_t)(3 - c) : c;
}

// ---------------------------------------------------------------------
// CIGAR algebra
// ---------------------------------------------------------------------
template <class K>
struct DCigT {
	static constexpr int CC = K::C, MC = K::M;
	int n, nm;
	uint32_t op[K::C];       // (count << 4) | op
	uint8_t miss[K::M];
};
using DCig = DCigT<CapsStd>;

__device__ __forceinline__ int op_type(uint32_t o) { return (int)(o & 15u); }
__device__ __forceinline__ unsigned op_cnt(uint32_t o) { return o >> 4; }

// add_cigar (src/hash_align.c:526-565)
template <class Cig>
__device__ inline void cig_add(Cig &c, int type, unsigned add, const uint8_t *mc, int &flags)
{
	constexpr int MCAP = Cig::MC, CCAP = Cig::CC;
	add &= 0xffffu;
	if (add == 0)
		return;
	if (c.n > 1 && op_type(c.op[c.n - 1]) == OP_S) {
		if (type != OP_D)
			c.op[c.n - 1] = (((op_cnt(c.op[c.n - 1]) + add) & 0xffffu) << 4) | OP_S;
		return;
	}
	if (mc) {
		if (c.nm + (int)add > MCAP) {
			flags |= F_MCAP;
		} else {
			for (unsigned t = 0; t < add; ++t)
				c.miss[c.nm + t] = mc[t];
			c.nm += (int)add;
		}
	}
	if (c.n > 0 && op_type(c.op[c.n - 1]) == type) {
		c.op[c.n - 1] = (((op_cnt(c.op[c.n - 1]) + add) & 0xffffu) << 4) | (uint32_t)type;
		return;
	}
	if (c.n == CCAP) {
		flags |= F_CCAP;
		return;
	}
	c.op[c.n++] = (add << 4) | (uint32_t)type;
}

// reverse_cigar (src/hash_align.c:567-587)
template <class Cig>
__device__ inline void cig_reverse(Cig &c)
{
	for (int i = 0; i < c.n / 2; ++i) {
		uint32_t t = c.op[i];
		c.op[i] = c.op[c.n - 1 - i];
		c.op[c.n - 1 - i] = t;
	}
	for (int i = 0; i < c.nm / 2; ++i) {
		uint8_t t = c.miss[i];
		c.miss[i] = c.miss[c.nm - 1 - i];
		c.miss[c.nm - 1 - i] = t;
	}
}

// concat_cigar (src/hash_align.c:589-603)
template <class Cig>
__device__ inline void cig_concat(Cig &d, Cig &t, int &flags)
{
	cig_reverse(t);
	int k = 0;
	for (int i = 0; i < t.n; ++i) {
		int ty = op_type(t.op[i]);
		unsigned cnt = op_cnt(t.op[i]);
		if (ty == OP_D || ty == OP_X) {
			cig_add(d, ty, cnt, t.miss + k, flags);
			k += (int)cnt;
		} else {
			cig_add(d, ty, cnt, nullptr, flags);
		}
	}
}

template <class Cig>
__device__ inline void cig_copy(Cig &d, const Cig &s)
{
	d.n = s.n;
	d.nm = s.nm;
	for (int i = 0; i < s.n; ++i)
		d.op[i] = s.op[i];
	for (int i = 0; i < s.nm; ++i)
		d.miss[i] = s.miss[i];
}

// ---------------------------------------------------------------------
// Gap DP: SW_align (src/hash_align.c:627-760), banded.
//
// The reference fills a zeroed (len+1) x (ref_len+1) u16 matrix; row k only
// ever writes columns [s_k, b_k] plus one marker, and every computed cell
// satisfies |k - c| <= M[k][c] <= error, so b_k - s_k <= 2*error + 1.  Here
// each row keeps just its written band (lo = s_k, width); any other cell
// reads as the zeroed matrix would, including row 0 (M[0][c] = c for
// c <= error+1) and its spill into later rows of the flat array.
// ---------------------------------------------------------------------
struct SwWork {
	uint8_t band[(MAX_DP_ROWS + 1) * BW];
	uint16_t lo[MAX_DP_ROWS + 1];
	uint8_t wid[MAX_DP_ROWS + 1];
};

struct SwView {
	const SwWork *w;
	unsigned W, error;
	__device__ __forceinline__ unsigned get(int k, int c) const
	{
		unsigned rel = (unsigned)(c - (int)w->lo[k]);
		if (rel < w->wid[k])
			return w->band[k * BW + rel];
		long long flat = (long long)k * W + c;
		return flat <= (long long)error + 1 ? (unsigned)flat : 0u;
	}
};

// Reference window accessor: x in [0, ref_len), reversed for prefix DPs.
struct RefWin {
	const uint8_t *code;
	const uint8_t *ascii;
	uint32_t start, len;
	bool rev;
	__device__ __forceinline__ uint32_t at(int x) const { return rev ? start + len - 1 - x : start + x; }
	__device__ __forceinline__ uint8_t c(int x) const { return code[at(x)]; }
	__device__ __forceinline__ const uint8_t *a(int x) const { return ascii + at(x); }
};

// q: query codes (already oriented), qlen; qrev: read q backwards (prefix DP)
template <class Cig>
__device__ inline int sw_align(const DevIndex &ix, uint32_t rstart, const uint8_t *q,
			       uint32_t ref_len, uint32_t len, int err, bool score_only,
			       Cig &cig, SwWork &w, int &flags, uint32_t *cells = nullptr)
{
	cig.n = 0;
	cig.nm = 0;
	if (len == 0)
		return 0;
	if (len > (uint32_t)MAX_DP_ROWS) {
		flags |= F_READ;
		return 0;
	}
	const unsigned error = (unsigned)(err < 0 ? -err : err) + 1;
	const bool rev = err < 0;
	RefWin r{ix.code, ix.seq, rstart, ref_len, rev};
	auto qc = [&](int x) -> uint8_t { return rev ? q[len - 1 - x] : q[x]; };
	SwView M{&w, ref_len + 1, error};

	// row 0: M[0][c] = c for c <= error+1 (the rest of the row is zero)
	{
		unsigned wd = (ref_len < error + 1 ? ref_len : error + 1) + 1;
		w.lo[0] = 0;
		w.wid[0] = (uint8_t)wd;
		for (unsigned c = 0; c < wd; ++c)
			w.band[c] = (uint8_t)c;
	}

	unsigned s = 0, min = 0, xmin = 0;
	int i = 0, k, j, ferr = -1, score = 0;
	for (k = 1; k <= (int)len; ++k) {
		uint8_t *cb = w.band + k * BW;
		const int plo = w.lo[k - 1];
		const unsigned pwd = w.wid[k - 1];
		const uint8_t *pb = w.band + (k - 1) * BW;
		auto pget = [&](int c) -> unsigned {
			unsigned rel = (unsigned)(c - plo);
			if (rel < pwd)
				return pb[rel];
			long long flat = (long long)(k - 1) * (ref_len + 1) + c;
			return flat <= (long long)error + 1 ? (unsigned)flat : 0u;
		};
		const uint8_t qk = qc(k - 1);
		min = error;
		j = 0;
		w.lo[k] = (uint16_t)s;
		unsigned left = pget((int)s) + 1;
		cb[0] = (uint8_t)left;
		unsigned wd = 1;
		unsigned d = pget((int)s);
		for (i = (int)s + 1; i <= (int)ref_len; ++i) {
			unsigned rel = (unsigned)i - s;
			if (rel >= (unsigned)BW) {
				flags |= F_BAND;
				break;
			}
			unsigned up = pget(i);
			if (d == error + 1) {
				cb[rel] = (uint8_t)(error + 1);
				wd = rel + 1;
				break;
			}
			unsigned pen = 0;
			if (d < error)
				pen = r.c(i - 1) == qk ? 0u : 1u;
			unsigned v = d + pen;
			if (left + 1 < v)
				v = left + 1;
			if (up + 1 < v)
				v = up + 1;
			cb[rel] = (uint8_t)v;
			wd = rel + 1;
			if (v == error && j == 0)
				j = i;
			if (v < error)
				j = 0;
			if (v <= min) {
				min = v;
				xmin = (unsigned)i;
			}
			if (ferr == -1 && i == k && v > 0)
				ferr = i;
			left = v;
			d = up;
		}
		w.wid[k] = (uint8_t)wd;
		if (cells && i > (int)s + 1)
			*cells += (uint32_t)(i - (int)s - 1);
		if (min == error) {
			++k;
			break;
		}
		while (M.get(k, (int)s) >= error && s < (unsigned)i)
			++s;
		if ((unsigned)j > xmin && (unsigned)j < ref_len)
			cb[(unsigned)j - w.lo[k]] = (uint8_t)(error + 1);
	}
	--k;

	if (min >= error) {
		// early stop: shrink the aligned query prefix (:698-711); the
		// reference's r[-1] read at column 0 cannot change the outcome
		while (k >= 5 && (min > (unsigned)(k / 10) || min * 2 > (unsigned)(k - ferr))) {
			--k;
			int jj = 0;
			for (int c = 0; (unsigned)c < ref_len; ++c) {
				unsigned v = M.get(k, c);
				if (v == error + 1)
					break;
				if (v > 0)
					jj = (int)error;
				if (v <= min && jj > 0 && c > 0 && r.c(c - 1) == qc(k - 1) &&
				    v == M.get(k - 1, c - 1)) {
					min = v;
					xmin = (unsigned)c;
				}
			}
		}
		if (k < 5) {
			cig_add(cig, OP_S, len, nullptr, flags);
			return (int)len;
		}
		cig_add(cig, OP_S, len - (unsigned)k, nullptr, flags);
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

	if (score_only) {   // WRITE_BAM == 1 (:731-734)
		cig_add(cig, OP_M, (unsigned)k, nullptr, flags);
		return score;
	}
	while (i > 0 && k > 0) {   // traceback (:736-758)
		unsigned cur = M.get(i, k);
		unsigned pen = r.c(k - 1) == qc(i - 1) ? 0u : 1u;
		if (cur == M.get(i - 1, k - 1) + pen) {
			if (pen == 0)
				cig_add(cig, OP_M, 1, nullptr, flags);
			else
				cig_add(cig, OP_X, 1, r.a(k - 1), flags);
			--i;
			--k;
		} else if (cur == M.get(i - 1, k) + 1) {
			cig_add(cig, OP_I, 1, nullptr, flags);
			--i;
		} else {
			cig_add(cig, OP_D, 1, r.a(k - 1), flags);
			--k;
		}
	}
	if (i > 0)
		cig_add(cig, OP_I, (unsigned)i, nullptr, flags);
	for (int t = 1; t <= k; ++t)
		cig_add(cig, OP_D, 1, r.a(k - t), flags);
	return score;
}

// ---------------------------------------------------------------------
// Gap DP, register form.  Same semantics as sw_align above, for the two
// error caps the live calls use (err = +-3 -> error 4, err = +-7 ->
// error 8) when ref_len >= error + 1 (no row-0 spill).
//
// Every written cell of row k lies on a diagonal d = c - k in
// [-error, error + 1] (computed cells satisfy |d| <= M <= error; the break
// and j markers sit at most one diagonal further), so a row is held as
// W = 2*error + 2 diagonal slots in registers.  In slot terms the diag,
// up and left neighbours are the fixed offsets P[q], P[q+1], V[q-1]: each
// row is one fully unrolled, predicated pass with no dynamic indexing, and
// the reference bases slide through a register window (one load per row).
// Rows are written to local memory only for the early-stop shrink loop and
// the traceback.
// ---------------------------------------------------------------------
struct QView {   // query codes: q(x) = p[x * step]
	const uint8_t *p;
	int step;
	__device__ __forceinline__ uint8_t operator()(int x) const { return p[x * step]; }
};

template <int E, bool STORE, class Cig>
__device__ inline int sw_align_reg(const RefWin &r, QView qc, uint32_t ref_len, uint32_t len,
				   bool score_only, Cig &cig, uint8_t *__restrict__ rows, int &flags,
				   uint32_t &cells)
{
	constexpr int W = 2 * E + 2;
	constexpr unsigned error = E;
	constexpr int NW = (W + 7) / 8;        // 32-bit words per stored row (4 bits a slot)
	// reference code at window position x, clamped (values outside the
	// window are never used, the clamp only keeps the address valid)
	auto rcode = [&](int x) -> int {
		x = x < 0 ? 0 : (x >= (int)ref_len ? (int)ref_len - 1 : x);
		return r.c(x);
	};
	// P: the previous row, updated in place into the current row (slot q
	// reads P[q] and P[q+1] before it is overwritten)
	int P[W], RC[W];
#pragma unroll
	for (int q = 0; q < W; ++q) {
		const int d = q - E;
		P[q] = (d >= 0) ? d : 0;          // row 0: M[0][c] = c, c <= error+1
		RC[q] = rcode(q - E);             // row 1 needs r[c-1], c = 1 + q - E
	}
	// rows are kept 4 bits a slot (values <= error + 1 <= 9)
	uint32_t *rw = reinterpret_cast<uint32_t *>(rows);
	auto store_row = [&](int k) {
#pragma unroll
		for (int w = 0; w < NW; ++w) {
			uint32_t pk = 0;
#pragma unroll
			for (int b = 0; b < 8; ++b)
				if (w * 8 + b < W)
					pk |= (uint32_t)P[w * 8 + b] << (4 * b);
			rw[k * NW + w] = pk;
		}
	};
	if (STORE)
		store_row(0);
	auto get = [&](int k, int c) -> unsigned {
		const int q = c - k + E;
		return (q >= 0 && q < W) ? (rw[k * NW + (q >> 3)] >> (4 * (q & 7))) & 15u : 0u;
	};

	int s = 0, ferr = -1, k, i = 0;
	unsigned min = 0, xmin = 0;
	for (k = 1; k <= (int)len; ++k) {
		if (k > 1) {
#pragma unroll
			for (int q = 0; q < W - 1; ++q)
				RC[q] = RC[q + 1];
			RC[W - 1] = rcode(k + W - 2 - E);
		}
		const int qk = qc(k - 1);
		min = error;
		int j = 0, left = 0, brk = -1;
		bool broken = false;
		if (s - k < -E) {   // outside the proven band: cannot happen
			flags |= F_BAND;
			return 0;
		}
#pragma unroll
		for (int q = 0; q < W; ++q) {
			const int c = k + q - E;
			const int up = (q + 1 < W) ? P[q + 1] : 0;
			const int dg = P[q];
			int v = 0;
			if (c == s) {
				v = up + 1;   // left edge: M[k-1][s] + 1
			} else if (c > s && !broken && c <= (int)ref_len) {
				if (dg == (int)error + 1) {
					v = error + 1;
					broken = true;
					brk = c;
				} else {
					const int pen = (dg < (int)error && RC[q] != qk) ? 1 : 0;
					v = dg + pen;
					v = (left + 1 < v) ? left + 1 : v;
					v = (up + 1 < v) ? up + 1 : v;
					if (v == (int)error && j == 0)
						j = c;
					if (v < (int)error)
						j = 0;
					if ((unsigned)v <= min) {
						min = (unsigned)v;
						xmin = (unsigned)c;
					}
					if (q == E && ferr == -1 && v > 0)
						ferr = c;
				}
			}
			P[q] = v;
			left = v;
		}
		i = broken ? brk : (int)ref_len + 1;
		cells += i > s + 1 ? (uint32_t)(i - s - 1) : 0u;   // the cells the reference visits
		if (min != error) {
			// while (M[k][s] >= error && s < i) ++s
			bool go = true;
#pragma unroll
			for (int q = 0; q < W; ++q) {
				const int c = k + q - E;
				if (go && c == s) {
					if (P[q] >= (int)error && s < i)
						++s;
					else
						go = false;
				}
			}
			if ((unsigned)j > xmin && (unsigned)j < ref_len) {
#pragma unroll
				for (int q = 0; q < W; ++q)
					if (k + q - E == j)
						P[q] = error + 1;
			}
		}
		if (STORE)
			store_row(k);
		if (min == error) {
			if (!STORE)
				return -1;   // early stop: the shrink loop needs the rows
			++k;
			break;
		}
	}
	--k;

	int score = 0;
	if (min >= error) {
		while (k >= 5 && (min > (unsigned)(k / 10) || min * 2 > (unsigned)(k - ferr))) {
			--k;
			// The reference scans row k from column 0 to its break.  Cells
			// left of the window are zero there and here (no effect: jj
			// stays 0), and the break marker or ref_len lies inside the
			// window, so the scan covers the window only.
			int jj = 0;
			const int c_lo = k - E > 0 ? k - E : 0;
			const int c_hi = k - E + W < (int)ref_len ? k - E + W : (int)ref_len;
			for (int c = c_lo; c < c_hi; ++c) {
				const unsigned v = get(k, c);
				if (v == error + 1)
					break;
				if (v > 0)
					jj = (int)error;
				if (v <= min && jj > 0 && c > 0 && r.c(c - 1) == qc(k - 1) && v == get(k - 1, c - 1)) {
					min = v;
					xmin = (unsigned)c;
				}
			}
		}
		if (k < 5) {
			cig_add(cig, OP_S, len, nullptr, flags);
			return (int)len;
		}
		cig_add(cig, OP_S, len - (unsigned)k, nullptr, flags);
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
	if (score_only) {
		cig_add(cig, OP_M, (unsigned)k, nullptr, flags);
		return score;
	}
	if constexpr (!STORE)
		return -1;
	else {
	while (i > 0 && k > 0) {
		const unsigned cur = get(i, k);
		const unsigned pen = r.c(k - 1) == qc(i - 1) ? 0u : 1u;
		if (cur == get(i - 1, k - 1) + pen) {
			if (pen == 0)
				cig_add(cig, OP_M, 1, nullptr, flags);
			else
				cig_add(cig, OP_X, 1, r.a(k - 1), flags);
			--i;
			--k;
		} else if (cur == get(i - 1, k) + 1) {
			cig_add(cig, OP_I, 1, nullptr, flags);
			--i;
		} else {
			cig_add(cig, OP_D, 1, r.a(k - 1), flags);
			--k;
		}
	}
	if (i > 0)
		cig_add(cig, OP_I, (unsigned)i, nullptr, flags);
	for (int t = 1; t <= k; ++t)
		cig_add(cig, OP_D, 1, r.a(k - t), flags);
	return score;
	}
}

// ---------------------------------------------------------------------
// Gap DP, bit-plane form.  Same semantics as sw_align_reg (and so as
// SW_align) for the two live error caps, with a row's W = 2*error + 2
// diagonal slots held as thermometer bit planes: bit q of plane t is set
// when slot q's value is >= t.  Values never exceed error + 2 (the left
// edge, one more than a break or j marker above it), so planes t = 1 ..
// error + 2 hold a row exactly.  In this form a cell's min is an AND, +1
// renames planes, and the left-neighbour term of the recurrence,
// V[q] = min(T[q], V[q-1] + 1), unrolls plane by plane to
// A_t = T_t & ((A_{t-1} << 1) | 1): a whole row is a few word operations
// per plane instead of ~20 predicated operations per slot.  The left edge,
// the break marker, the row's min / rightmost xmin, the j marker, ferr and
// the advance of s are masks and bit scans over single words.  Rows are
// kept in binary (as planes of the 4-bit values) for the early-stop shrink
// loop and the traceback.
// ---------------------------------------------------------------------
template <int E>
struct BitRows;
template <>
struct BitRows<8> {            // W = 18: planes b0..b3 of 18 bits, 16 bytes a row
	using T = uint4;
	static __device__ __forceinline__ T pack(uint32_t b0, uint32_t b1, uint32_t b2, uint32_t b3)
	{
		return make_uint4(b0, b1, b2, b3);
	}
	static __device__ __forceinline__ unsigned at(const T &r, int q)
	{
		return ((r.x >> q) & 1u) | (((r.y >> q) & 1u) << 1) | (((r.z >> q) & 1u) << 2) | (((r.w >> q) & 1u) << 3);
	}
};
template <>
struct BitRows<4> {            // W = 10, values <= 6: planes b0..b2 in one word, 4 bytes a row
	using T = uint32_t;
	static __device__ __forceinline__ T pack(uint32_t b0, uint32_t b1, uint32_t b2, uint32_t)
	{
		return b0 | (b1 << 10) | (b2 << 20);
	}
	static __device__ __forceinline__ unsigned at(const T &r, int q)
	{
		return ((r >> q) & 1u) | (((r >> (q + 10)) & 1u) << 1) | (((r >> (q + 20)) & 1u) << 2);
	}
};

// What the bit-plane DP keeps of each row: the whole row (4 binary planes)
// for the traceback, or, in the score-only mode (SUM), the 2-byte summary
// the shrink loop needs (below).
template <int E, bool SUM>
struct DpRow {
	using T = typename BitRows<E>::T;
};
template <int E>
struct DpRow<E, true> {
	using T = uint16_t;
};

template <int E, bool SUM, class Cig>
__device__ inline int sw_align_bits(const RefWin &r, QView qc, uint32_t ref_len, uint32_t len,
				    bool score_only, Cig &cig, typename DpRow<E, SUM>::T *__restrict__ rows, int &flags,
				    uint32_t &cells)
{
	constexpr int W = 2 * E + 2;
	constexpr int NT = E + 2;              // planes t = 1 .. error + 2
	constexpr uint32_t FULL = (1u << W) - 1;
	constexpr unsigned error = E;
	using RB = BitRows<E>;
	// reference code at window position x, clamped (values outside the
	// window are never used, the clamp only keeps the address valid)
	auto rcode = [&](int x) -> uint32_t {
		x = x < 0 ? 0 : (x >= (int)ref_len ? (int)ref_len - 1 : x);
		return r.c(x);
	};
	// a thermometer row stored as planes of its binary values (traceback mode)
	auto store = [&](int k, const uint32_t (&G)[NT + 1]) {
		if constexpr (SUM)
			return;
		uint32_t b0 = 0, b1 = 0, b2 = 0, b3 = 0;
#pragma unroll
		for (int t = 1; t <= NT; ++t) {
			const uint32_t only = G[t] & ~(t < NT ? G[t + 1] : 0u);   // value == t
			if (t & 1) b0 |= only;
			if (t & 2) b1 |= only;
			if (t & 4) b2 |= only;
			if (t & 8) b3 |= only;
		}
		if constexpr (!SUM)
			rows[k] = RB::pack(b0, b1, b2, b3);
	};
	auto get = [&](int k, int c) -> unsigned {
		if constexpr (SUM) {
			return 0u;   // not used: the score-only mode keeps summaries
		} else {
			const int q = c - k + E;
			return (q >= 0 && q < W) ? RB::at(rows[k], q) : 0u;
		}
	};
	// reference codes of row k's slots (x = k + q - error - 1) as three
	// planes; row 1 first
	uint32_t R0 = 0, R1 = 0, R2 = 0;
#pragma unroll
	for (int q = 0; q < W; ++q) {
		const uint32_t c = rcode(q - E);
		R0 |= (c & 1u) << q;
		R1 |= ((c >> 1) & 1u) << q;
		R2 |= ((c >> 2) & 1u) << q;
	}
	// row 0: slot q holds q - error (M[0][c] = c for c <= error + 1), 0 left of it
	uint32_t G[NT + 1];
	G[0] = FULL;
#pragma unroll
	for (int t = 1; t <= NT; ++t)
		G[t] = (E + t < W) ? (FULL & ~((1u << (E + t)) - 1)) : 0u;
	store(0, G);

	int s = 0, ferr = -1, k, i = 0;
	unsigned min = 0, xmin = 0;
	for (k = 1; k <= (int)len; ++k) {
		if (k > 1) {   // slide the reference planes one slot
			const uint32_t c = rcode(k + W - E - 2);
			R0 = (R0 >> 1) | ((c & 1u) << (W - 1));
			R1 = (R1 >> 1) | (((c >> 1) & 1u) << (W - 1));
			R2 = (R2 >> 1) | (((c >> 2) & 1u) << (W - 1));
		}
		const uint32_t qk = qc(k - 1);
		const int qs = s - k + E;              // slot of the left edge
		if (qs < 0) {   // outside the proven band: cannot happen
			flags |= F_BAND;
			return 0;
		}
		const uint32_t EQ = 1u << qs;
		const uint32_t LT = EQ - 1, LE = (EQ << 1) - 1;
		const int qr = (int)ref_len - k + E;   // last slot with c <= ref_len
		const uint32_t RL = qr >= W - 1 ? FULL : (qr < 0 ? 0u : (2u << qr) - 1);
		// the break: first slot past the left edge (within the window) whose
		// diagonal neighbour is error + 1
		const uint32_t BR = G[E + 1] & ~LE & RL;
		const uint32_t BM = BR & (0u - BR);
		const uint32_t COMP = ~LE & RL & (BM ? BM - 1 : FULL);   // the cells the row computes
		// mismatch slots; the penalty only where the diagonal is < error
		const uint32_t MM = (R0 ^ (0u - (qk & 1u))) | (R1 ^ (0u - ((qk >> 1) & 1u))) |
				    (R2 ^ (0u - ((qk >> 2) & 1u)));
		const uint32_t PEN = MM & ~G[E];
		// T = min(diag + pen, up + 1); slots left of the edge infinite, the
		// edge up + 1; then the left-neighbour prefix, plane by plane
		uint32_t V[NT + 1];
		V[0] = FULL;
		uint32_t A = FULL;
#pragma unroll
		for (int t = 1; t <= NT; ++t) {
			const uint32_t DG = t <= E ? (G[t] | (PEN & G[t - 1])) : G[t];
			const uint32_t U = t == 1 ? FULL : ((G[t - 1] >> 1) & FULL);
			const uint32_t T = (DG | LE) & (U | LT);
			A = T & ((A << 1) | 1u);
			V[t] = A;
		}
		// the written row: the edge and the computed cells, the break
		// marker error + 1, zero elsewhere
		const uint32_t LIVE = COMP | EQ;
#pragma unroll
		for (int t = 1; t <= NT; ++t)
			V[t] = (V[t] & LIVE) | (t <= E + 1 ? BM : 0u);
		i = BM ? k + (__ffs(BM) - 1) - E : (int)ref_len + 1;
		cells += i > s + 1 ? (uint32_t)(i - s - 1) : 0u;   // the cells the reference visits
		// min (from error) and the rightmost slot holding it, over the
		// computed cells (their values are <= error)
		min = error;
		uint32_t XM = COMP;
#pragma unroll
		for (int t = E; t >= 1; --t) {
			const uint32_t X = ~V[t] & COMP;   // cells < t
			if (X) {
				min = (unsigned)(t - 1);
				XM = X;
			}
		}
		if (COMP)
			xmin = (unsigned)(k + (31 - __clz(XM)) - E);
		// j: the first cell == error after the last cell < error
		const uint32_t LTE = ~V[E] & COMP, EQE = V[E] & COMP;
		const uint32_t above = LTE ? ~((2u << (31 - __clz(LTE))) - 1) : 0xffffffffu;
		const uint32_t JC = EQE & above;
		const int j = JC ? k + (__ffs(JC) - 1) - E : 0;
		if (ferr == -1 && ((COMP & V[1]) >> E) & 1u)   // slot error is column k
			ferr = k;
		if (min != error) {
			// while (M[k][s] >= error && s < i) ++s
			const uint32_t run = ~(V[E] >> qs);
			const int n = __ffs(run) - 1;
			s = s + n < i ? s + n : (i > s ? i : s);
			if ((unsigned)j > xmin && (unsigned)j < ref_len) {
				const uint32_t JM = 1u << (j - k + E);
#pragma unroll
				for (int t = 1; t <= NT; ++t)
					V[t] = t <= E + 1 ? (V[t] | JM) : (V[t] & ~JM);
			}
		}
		if constexpr (SUM) {
			// The shrink loop's scan of row k (below), as one summary: the
			// scan runs over the window's columns up to the first cell ==
			// error + 1; a cell is a candidate from the first cell > 0 on,
			// at a column > 0, where the diagonal codes match and the cell
			// equals its up-left neighbour (same slot of row k - 1, still in
			// G).  Scanning in column order with `v <= min`, the scan ends
			// with min = the smallest candidate value m (when m <= min) and
			// xmin = the last candidate column holding m: the summary keeps
			// m and that slot.
			const int qlo = E - k > 0 ? E - k : 0;
			const int qhi = (int)ref_len - k + E < W ? (int)ref_len - k + E : W;
			const uint32_t SR = qhi > qlo ? ((1u << qhi) - 1u) & ~((1u << qlo) - 1u) : 0u;
			const uint32_t E1 = V[E + 1] & ~V[E + 2] & SR;
			const uint32_t SCAN = SR & (E1 ? (E1 & (0u - E1)) - 1u : 0xffffffffu);
			const uint32_t NZ = V[1] & SCAN;
			const uint32_t ALW = NZ ? ~((NZ & (0u - NZ)) - 1u) : 0u;
			const int q0 = E - k + 1;                 // column > 0
			const uint32_t C0 = q0 <= 0 ? 0xffffffffu : ~((1u << q0) - 1u);
			uint32_t DIFF = 0;
#pragma unroll
			for (int t = 1; t <= NT; ++t)
				DIFF |= V[t] ^ G[t];
			const uint32_t CAND = SCAN & ALW & C0 & ~MM & ~DIFF;
			uint32_t X = 0, m = 0;
#pragma unroll
			for (int t = E + 1; t >= 1; --t) {
				const uint32_t Y = CAND & ~V[t];   // candidates < t
				if (Y) {
					X = Y;
					m = (uint32_t)(t - 1);
				}
			}
			rows[k] = X ? (uint16_t)(0x8000u | (m << 8) | (uint32_t)(31 - __clz(X))) : (uint16_t)0;
		}
#pragma unroll
		for (int t = 1; t <= NT; ++t)
			G[t] = V[t];
		store(k, G);
		if (min == error) {
			++k;
			break;
		}
	}
	--k;

	int score = 0;
	if (min >= error) {
		if constexpr (SUM) {
			while (k >= 5 && (min > (unsigned)(k / 10) || min * 2 > (unsigned)(k - ferr))) {
				--k;
				const uint32_t sm = rows[k];   // the row's scan, summarised as it was computed
				if ((sm & 0x8000u) && ((sm >> 8) & 15u) <= min) {
					min = (sm >> 8) & 15u;
					xmin = (unsigned)(k + (int)(sm & 31u) - E);
				}
			}
		}
		while (!SUM && k >= 5 && (min > (unsigned)(k / 10) || min * 2 > (unsigned)(k - ferr))) {
			--k;
			// The reference scans row k from column 0 to its break.  Cells
			// left of the window are zero there and here (no effect: jj
			// stays 0), and the break marker or ref_len lies inside the
			// window, so the scan covers the window only.
			int jj = 0;
			const int c_lo = k - E > 0 ? k - E : 0;
			const int c_hi = k - E + W < (int)ref_len ? k - E + W : (int)ref_len;
			for (int c = c_lo; c < c_hi; ++c) {
				const unsigned v = get(k, c);
				if (v == error + 1)
					break;
				if (v > 0)
					jj = (int)error;
				if (v <= min && jj > 0 && c > 0 && r.c(c - 1) == qc(k - 1) && v == get(k - 1, c - 1)) {
					min = v;
					xmin = (unsigned)c;
				}
			}
		}
		if (k < 5) {
			cig_add(cig, OP_S, len, nullptr, flags);
			return (int)len;
		}
		cig_add(cig, OP_S, len - (unsigned)k, nullptr, flags);
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
	if (SUM || score_only) {
		cig_add(cig, OP_M, (unsigned)k, nullptr, flags);
		return score;
	}
	if constexpr (!SUM) {   // the traceback over the kept rows
		while (i > 0 && k > 0) {
			const unsigned cur = get(i, k);
			const unsigned pen = r.c(k - 1) == qc(i - 1) ? 0u : 1u;
			if (cur == get(i - 1, k - 1) + pen) {
				if (pen == 0)
					cig_add(cig, OP_M, 1, nullptr, flags);
				else
					cig_add(cig, OP_X, 1, r.a(k - 1), flags);
				--i;
				--k;
			} else if (cur == get(i - 1, k) + 1) {
				cig_add(cig, OP_I, 1, nullptr, flags);
				--i;
			} else {
				cig_add(cig, OP_D, 1, r.a(k - 1), flags);
				--k;
			}
		}
		if (i > 0)
			cig_add(cig, OP_I, (unsigned)i, nullptr, flags);
		for (int t = 1; t <= k; ++t)
			cig_add(cig, OP_D, 1, r.a(k - t), flags);
	}
	return score;
}

// Entry used by the per-task (plain) path: the banded form, which keeps the
// register footprint small where neighbouring threads diverge.  The batched
// path runs sw_align_reg on length-sorted jobs instead.  q: oriented read
// codes of the gap.
template <class Cig>
__device__ inline int gap_dp(const DevIndex &ix, uint32_t rstart, const uint8_t *q, int qstep,
			     uint32_t ref_len, uint32_t len, int err, bool score_only, Cig &cig,
			     SwWork &w, int &flags)
{
	cig.n = 0;
	cig.nm = 0;
	if (len == 0)
		return 0;
	if (len > (uint32_t)MAX_DP_ROWS) {
		flags |= F_READ;
		return 0;
	}
	(void)qstep;
	return sw_align(ix, rstart, q, ref_len, len, err, score_only, cig, w, flags);
}

// ---------------------------------------------------------------------
// Seed-table probe: hash_get with add = 0 (src/hash_align.c:862-895).
// Returns {start, count} of the k-mer's occurrence list, count 0 on a miss.
// Buckets are sorted by id, so any search that finds the equal id returns
// the reference's slot.
// ---------------------------------------------------------------------
__device__ __forceinline__ uint2 probe(const DevIndex &ix, uint64_t id, uint32_t *n_probes = nullptr)
{
	const uint32_t mod = (uint32_t)(id & HMASK);
	uint32_t lo = __ldg(ix.boff + mod);
	uint32_t hi = __ldg(ix.boff + mod + 1);
	while (lo < hi) {
		uint32_t mid = (lo + hi) >> 1;
		if (n_probes)
			++*n_probes;
		uint4 b = __ldg(ix.bk + mid);
		uint64_t bid = ((uint64_t)b.y << 32) | b.x;
		if (bid == id)
			return make_uint2(b.z, b.w - b.z);
		if (bid > id)
			hi = mid;
		else
			lo = mid + 1;
	}
	return make_uint2(0, 0);
}

// 8 bytes at any address p, from the two aligned words around it (the
// buffers this reads carry at least 16 bytes of padding past their data)
__device__ __forceinline__ uint64_t load8(const uint8_t *p)
{
	const uintptr_t a = reinterpret_cast<uintptr_t>(p);
	const unsigned long long *w = reinterpret_cast<const unsigned long long *>(a & ~(uintptr_t)7);
	const int s = (int)(a & 7) * 8;
	const uint64_t lo = __ldg(w);
	if (s == 0)
		return lo;
	return (lo >> s) | ((uint64_t)__ldg(w + 1) << (64 - s));
}

// get_index (src/hash_align.c:997-1006) over 31 codes at p, read as four
// 8-byte words: id = OR of code[x] << 2*(30-x) (the reference shifts codes
// in unmasked, so code 4 sets the low bit of the previous slot).  rev: the
// reverse complement of the same 31 bytes (the k-mer that starts at the
// last byte and runs backwards), id = OR of comp(code[x]) << 2*x.
__device__ __forceinline__ uint64_t kmer_words(const uint8_t *p, bool rev)
{
	uint64_t W[4];
#pragma unroll
	for (int k = 0; k < 4; ++k)
		W[k] = load8(p + 8 * k);
	uint64_t id = 0;
#pragma unroll
	for (int x = 0; x < KMER; ++x) {
		const uint8_t c = (uint8_t)(W[x >> 3] >> (8 * (x & 7)));
		if (rev)
			id |= (uint64_t)comp_code(c) << (2 * x);
		else
			id |= (uint64_t)c << (2 * (KMER - 1 - x));
	}
	return id;
}

// true if the n bytes at s+a and s+b are equal (8 at a time)
__device__ __forceinline__ bool bytes_equal(const uint8_t *s, uint32_t a, uint32_t b, uint32_t n)
{
	if (a == b)
		return true;
	// 32 bytes a step: the five aligned words around each string's piece
	// are loaded together (one load latency a step, not one per 8 bytes),
	// then shifted into place; the buffers carry 64 bytes of padding past
	// their data, so the last step's extra words are readable
	const unsigned long long *wa = reinterpret_cast<const unsigned long long *>((uintptr_t)(s + a) & ~(uintptr_t)7);
	const unsigned long long *wb = reinterpret_cast<const unsigned long long *>((uintptr_t)(s + b) & ~(uintptr_t)7);
	const int sa = (int)((a & 7) * 8), sb = (int)((b & 7) * 8);
	for (uint32_t x = 0; x < n; x += 32) {
		uint64_t A[5], B[5];
#pragma unroll
		for (int k = 0; k < 5; ++k) {
			A[k] = __ldg(wa + x / 8 + k);
			B[k] = __ldg(wb + x / 8 + k);
		}
		bool same = true;
#pragma unroll
		for (int k = 0; k < 4; ++k) {
			uint64_t u = sa ? (A[k] >> sa) | (A[k + 1] << (64 - sa)) : A[k];
			uint64_t v = sb ? (B[k] >> sb) | (B[k + 1] << (64 - sb)) : B[k];
			const uint32_t at = x + 8 * k;
			if (at < n && n - at < 8) {
				const uint64_t m = (1ull << (8 * (n - at))) - 1;
				u &= m;
				v &= m;
			}
			same = same && (at >= n || u == v);
		}
		if (!same)
			return false;
	}
	return true;
}

// get_index (src/hash_align.c:997-1006): codes shifted in unmasked
__device__ __forceinline__ uint64_t kmer_at(const uint8_t *rd, int i)
{
	uint64_t id = 0;
#pragma unroll
	for (int t = 0; t < KMER; ++t)
		id = (id << 2) | rd[i + t];
	return id;
}

// ---------------------------------------------------------------------
// Per-pair Candidate state in HBM
// ---------------------------------------------------------------------
template <class K>
struct DSlotT {             // one strand of a Candidate (src/hash_align.h:90-97)
	static constexpr int LC = K::L;
	int32_t n, err;
	uint32_t t[K::L];       // transcript ids   (Candidate.pos)
	int32_t p[K::L];        // positions        (Candidate.p)
	DCigT<K> cig;
};
using DSlot = DSlotT<CapsStd>;

template <class K>
struct DPairT {
	DSlotT<K> s[2][2];      // [candidate r[0]/r[1]][strand]
	int32_t pair[2];
	int32_t stage;
	int32_t rm_ret;
	int32_t rm_i;
	int32_t ovf;            // F_CAPS flags met by this pair (first pass)
};
using DPair = DPairT<CapsStd>;

// Anchors of one get_position call: pos2[0..2] of the reference, one
// 12-byte record per anchor so a call's few anchors share cache lines.
struct Anc {
	uint32_t t, tp, off;    // transcript, transcript position, read offset
};
template <class K>
struct AnchorsT {
	Anc a[K::A];
};

template <class K>
struct GpWorkT {
	AnchorsT<K> a[2];
	DCigT<K> c1, c2;
	SwWork sw;
	uint8_t rd[MAX_READ];
};
using GpWork = GpWorkT<CapsStd>;

// merge_sort (src/hash_align.c:257-297): new hit list (all at read offset
// idx) merged into the anchors by transcript; on an equal transcript the
// existing anchor goes first when the unsigned wrapped diagonal difference
// is < 2*ERR, else the smaller tpos.
template <class K>
__device__ inline int merge_hits(const AnchorsT<K> &A, int na, AnchorsT<K> &B, const uint2 *occ,
				 uint32_t nh, uint32_t idx, int &flags)
{
	constexpr int ACAP = K::A;
	if (na + (int)nh > ACAP) {
		flags |= F_ACAP;
		nh = (uint32_t)(ACAP - na);
	}
	int i = 0, n = 0;
	uint32_t k = 0;
	uint2 h = nh ? __ldg(occ) : make_uint2(0, 0);
	while (i < na && k < nh) {
		bool take_a;
		if (A.a[i].t < h.x) {
			take_a = true;
		} else if (A.a[i].t > h.x) {
			take_a = false;
		} else {
			uint32_t dis = (h.y - A.a[i].tp) - (idx - A.a[i].off);
			take_a = dis < 2 * ERR ? true : !(A.a[i].tp > h.y);
		}
		if (take_a) {
			B.a[n].t = A.a[i].t; B.a[n].tp = A.a[i].tp; B.a[n].off = A.a[i].off;
			++i;
		} else {
			B.a[n].t = h.x; B.a[n].tp = h.y; B.a[n].off = idx;
			++k;
			if (k < nh)
				h = __ldg(occ + k);
		}
		++n;
	}
	while (i < na) {
		B.a[n].t = A.a[i].t; B.a[n].tp = A.a[i].tp; B.a[n].off = A.a[i].off;
		++i; ++n;
	}
	while (k < nh) {
		h = __ldg(occ + k);
		B.a[n].t = h.x; B.a[n].tp = h.y; B.a[n].off = idx;
		++k; ++n;
	}
	return n;
}

// get_SWalign (src/hash_align.c:1242-1320)
template <class K>
__device__ inline void get_swalign(const DevIndex &ix, const uint8_t *rd, int rlen, AnchorsT<K> &A,
				   uint32_t id, uint32_t n, uint32_t &store, uint32_t &max,
				   DSlotT<K> &S, bool score_only, GpWorkT<K> &w, int &flags)
{
	if (n > 1 && A.a[id + n - 1].tp - A.a[id].tp > (uint32_t)rlen)
		return;
	const uint32_t tr = A.a[id].t;
	int start = (int)(A.a[id].tp - (A.a[id].off + KMER - 1));
	if (start < 0 || (uint32_t)(start + rlen) > __ldg(ix.tlen + tr))
		return;
	uint32_t add = start < ERR ? (uint32_t)start : (uint32_t)ERR;
	const uint32_t ref_start = __ldg(ix.tstart + tr) + (uint32_t)start;
	int err = 0, sub = 0, score;
	DCigT<K> &cig = w.c1;
	DCigT<K> &tmp = w.c2;
	cig.n = cig.nm = 0;
	if (A.a[id].off > 0) {
		const uint32_t o0 = A.a[id].off;
		score = gap_dp(ix, ref_start - add, rd, 1, o0 + add, o0, o0 < 2 * ERR ? -3 : -ERR,
			       score_only, cig, w.sw, flags);
		err += score;
		if (err > rlen / 2 || (uint32_t)err > max)
			return;
		for (int t = 0; t < cig.n; ++t) {
			int ty = op_type(cig.op[t]);
			if (ty == OP_I || ty == OP_S)
				sub += (int)op_cnt(cig.op[t]);
			else if (ty == OP_D)
				sub -= (int)op_cnt(cig.op[t]);
		}
	}
	for (uint32_t i = 0; i < n; ++i) {
		uint32_t s0 = i;
		while (i + 1 < n && A.a[id + i].off + KMER >= A.a[id + i + 1].off)
			++i;
		cig_add(cig, OP_M, A.a[id + i].off - A.a[id + s0].off + KMER, nullptr, flags);
		uint32_t seg = A.a[id + i].off + KMER;
		uint32_t len = ((i + 1) < n ? A.a[id + i + 1].off : (uint32_t)rlen) - seg;
		uint32_t ad = (i + 1) < n ? 0u : (uint32_t)ERR;
		score = gap_dp(ix, ref_start + seg, rd + seg, 1, len + ad, len, len < 2 * ERR ? 3 : ERR,
			       score_only, tmp, w.sw, flags);
		err += score;
		if (err > rlen / 2 || (uint32_t)err > max + 1)
			return;
		cig_concat(cig, tmp, flags);
	}
	if (max == (uint32_t)(rlen / 2) || (uint32_t)err < max) {
		cig_copy(S.cig, cig);
		store = 0;
		max = (uint32_t)err;
	}
	A.a[store].t = A.a[id].t;
	A.a[store].tp = A.a[id].tp - (A.a[id].off + KMER - 1) + (uint32_t)sub;
	++store;
}

template <class K>
__device__ __forceinline__ bool chain_next(const AnchorsT<K> &A, int na, uint32_t i, uint32_t n,
					   int rlen, bool stop_consumed)
{
	if (i + 1 >= (uint32_t)na)
		return false;
	if (A.a[i].t != A.a[i + 1].t || !(A.a[i + 1].off > A.a[i].off))
		return false;
	if (!(A.a[i + 1].tp > A.a[i + 1 - n].tp))
		return false;
	if (!(A.a[i + 1].tp - A.a[i + 1 - n].tp < (uint32_t)rlen))
		return false;
	if (stop_consumed && A.a[i + 1].off == (uint32_t)rlen)
		return false;
	return true;
}

// get_position (src/hash_align.c:1322-1467).  `rd` holds the read already
// in the strand's orientation (reverse complement for str 1).  Seed hits
// come from `pre` (one {start, count} per seed) when given, else are probed.
template <class K>
__device__ inline void get_position(const DevIndex &ix, const uint8_t *rd, int rlen, DPairT<K> &P,
				    int c, int str, int space, const uint2 *pre, bool score_only,
				    GpWorkT<K> &w, int &flags)
{
	constexpr int ACAP = K::A, LCAP = K::L;
	DSlotT<K> &S = P.s[c][str];
	const DSlotT<K> &Mt = P.s[c][1 - str];
	int cur = 0, na = 0;
	const uint32_t step = (uint32_t)(space < 0 ? -space : space);

	int sj = 0;
	for (uint32_t i = 0; i + KMER <= (uint32_t)rlen; i += step, ++sj) {
		uint2 h = pre ? pre[sj] : probe(ix, kmer_at(rd, (int)i));
		if (h.y == 0)
			continue;
		const uint2 *occ = ix.occ + h.x;
		if (na == 0) {
			uint32_t nh = h.y;
			if (nh > (uint32_t)ACAP) {
				flags |= F_ACAP;
				nh = ACAP;
			}
			AnchorsT<K> &A = w.a[cur];
			for (uint32_t k = 0; k < nh; ++k) {
				uint2 o = __ldg(occ + k);
				A.a[k].t = o.x;
				A.a[k].tp = o.y;
				A.a[k].off = i;
			}
			na = (int)nh;
			continue;
		}
		na = merge_hits(w.a[cur], na, w.a[cur ^ 1], occ, h.y, i, flags);
		cur ^= 1;
	}
	AnchorsT<K> &A = w.a[cur];
	uint32_t n1 = 0, max = 0, n;
	if (na == 0)
		goto miss;

	// pass A, mate-guided (:1367-1390)
	if (space < KMER && space > 0 && Mt.n > 0) {
		const uint32_t mn = (uint32_t)Mt.n;
		uint32_t k = 0;
		max = (uint32_t)(rlen / 2);
		for (uint32_t i = 0; i < (uint32_t)na; ++i) {
			if (A.a[i].t < Mt.t[k])
				continue;
			while (k < mn && A.a[i].t > Mt.t[k])
				++k;
			if (k == mn)
				break;
			n = 1;
			while (chain_next(A, na, i, n, rlen, false)) {
				++i;
				++n;
			}
			get_swalign(ix, rd, rlen, A, i + 1 - n, n, n1, max, S, score_only, w, flags);
			for (; n > 0; --n)
				A.a[i + 1 - n].off = (uint32_t)rlen;
		}
	}
	// pass B, chains of >= 2 anchors (:1392-1412)
	if (n1 == 0) {
		max = (uint32_t)(rlen / 2);
		for (uint32_t i = 0; i < (uint32_t)na; ++i) {
			if (A.a[i].off == (uint32_t)rlen)
				continue;
			n = 1;
			while (chain_next(A, na, i, n, rlen, true)) {
				++i;
				++n;
			}
			if (n < 2 && rlen / KMER > 2)
				continue;
			get_swalign(ix, rd, rlen, A, i - n + 1, n, n1, max, S, score_only, w, flags);
		}
	}
	// pass C, singletons (:1414-1434)
	if (n1 == 0 && space < KMER) {
		max = (uint32_t)(rlen / 2);
		for (uint32_t i = 0; i < (uint32_t)na; ++i) {
			if (A.a[i].off == (uint32_t)rlen)
				continue;
			n = 1;
			while (chain_next(A, na, i, n, rlen, true)) {
				++i;
				++n;
			}
			if (n >= 2)
				continue;
			get_swalign(ix, rd, rlen, A, i, n, n1, max, S, score_only, w, flags);
		}
	}
	if (n1 == 0)
		goto miss;
	if (n1 > (uint32_t)LCAP) {
		flags |= F_LCAP;
		n1 = LCAP;
	}
	for (uint32_t t = 0; t < n1; ++t) {
		S.t[t] = A.a[t].t;
		S.p[t] = (int32_t)A.a[t].tp;
	}
	S.n = (int32_t)n1;
	S.err = (int32_t)max;
	return;
miss:
	S.n = 0;
	S.err = rlen;
}

// intersect2 list step (src/hash_align.c:1528-1556): returns the number of
// pairs kept (lists compacted in place), 0 if none.
template <class K>
__device__ inline int intersect_lists(DPairT<K> &P, int c, uint32_t add)
{
	DSlotT<K> &X = P.s[c][0];
	DSlotT<K> &Y = P.s[c][1];
	int i = 0, k = 0, n = 0;
	while (i < X.n && k < Y.n) {
		if (X.t[i] < Y.t[k]) {
			++i;
		} else if (X.t[i] > Y.t[k]) {
			++k;
		} else {
			int d = X.p[i] - Y.p[k];
			uint32_t dis = (uint32_t)(d < 0 ? -d : d);
			if (dis <= add || add == 0) {
				++n;
				X.t[n - 1] = X.t[i];
				X.p[n - 1] = X.p[i];
				Y.t[n - 1] = Y.t[k];
				Y.p[n - 1] = Y.p[k];
				++i;
				++k;
			} else if (X.p[i] < Y.p[k]) {
				++i;
			} else {
				++k;
			}
		}
	}
	if (n > 0) {
		X.n = Y.n = n;
		P.pair[c] = 2;
	}
	return n;
}

// ---------------------------------------------------------------------
// Mate rescue DP: ssw_align (src/ssw.c:81-321), one warp per call.
//
// Local SW on saturating u8: H = max(0, min(255, diag + 3*[codes equal]) - 2,
// left - 4, up - 4) (+1 match incl. N==N, -2 mismatch, linear gap 4), which
// is what the reference's striped SSE2 loop with lazy-F converges to.  The
// warp sweeps anti-diagonally: lane l owns read rows [l*R, l*R+R) and works
// on column y = t - l + 1 at step t; the row above its block comes from lane
// l-1 by shuffle one step later.
//
// The sweep keeps no matrix.  It finds the maximum and its cell, and every
// SSW_CK columns it saves the whole column in shared memory.  The
// reference's traceback then walks back from the maximum; the warp
// recomputes the SSW_CK-column block the walk is in from the checkpoint at
// its left edge (exact: a column depends only on the column before it), so
// the walk reads shared memory only.  The reference window, the read and the
// CIGAR under construction also live in the warp's shared-memory area.
// ---------------------------------------------------------------------
constexpr int SSW_RMAX = (MAX_READ + 31) / 32;   // rows per lane, <= 10
constexpr int SSW_CK = 32;                       // checkpoint spacing (columns)
constexpr int SSW_NCK = MAX_FRAG / SSW_CK + 1;   // checkpoints at columns j*SSW_CK

__device__ __forceinline__ int mat_score(uint8_t a, uint8_t b)
{
	if (a == 4 || b == 4)
		return 0;
	return a == b ? 1 : -2;
}

template <class K>
struct SswOutT {
	int32_t score, skip, pstart, ok;
	DCigT<K> cig;
};
using SswOut = SswOutT<CapsStd>;

// oriented read code x of read (o, L)
__device__ __forceinline__ uint8_t read_code(const uint8_t *code, int64_t o, int L, int orient, int x)
{
	return orient ? comp_code(code[o + L - 1 - x]) : code[o + x];
}

// rows per lane used for a read of length L (instantiated widths only)
__host__ __device__ inline int ssw_rows(int L)
{
	const int R = (L + 31) / 32;
	return R <= 6 ? (R < 1 ? 1 : R) : (R <= 8 ? 8 : 10);
}

// shared-memory layout of one warp's area
constexpr int SSW_REF_B = ((MAX_FRAG + 32 + 15) / 16) * 16;
constexpr int SSW_RD_B = ((MAX_READ + 15) / 16) * 16;
template <class K>
__host__ __device__ constexpr int ssw_cig_b()
{
	return (int)((sizeof(DCigT<K>) + 15) / 16) * 16;
}
// an area for R rows a lane and a CIGAR of capacities K
template <class K>
__host__ __device__ inline size_t ssw_smem_rows(int R)
{
	const size_t col = (size_t)32 * R;   // bytes of one saved column
	return SSW_REF_B + SSW_RD_B + ssw_cig_b<K>() + SSW_NCK * col + (((SSW_CK + 1) * col + 15) / 16) * 16;
}
__host__ __device__ inline size_t ssw_smem_per_warp(int max_len)
{
	return ssw_smem_rows<CapsStd>(ssw_rows(max_len));
}
// the wide pass runs every call with the widest row layout (rows past the
// read take code 5 and feed no row of the read, so results do not change)
constexpr int SSW_WIDE_R = 10;
__host__ __device__ inline size_t ssw_smem_wide()
{
	return ssw_smem_rows<CapsWide>(SSW_WIDE_R);
}

// Score + 2 (3 for equal codes, N == N included, else 0) of every code
// against code q, as the two words of a byte permute: bytes 0-4 codes 0-4,
// byte 5 the code no sequence has (5), bytes 6-7 zero.
struct ScoreT {
	uint32_t lo, hi;
};
__device__ __forceinline__ ScoreT score_table(uint32_t q)
{
	return ScoreT{q < 4 ? 3u << (8 * q) : 0u, q == 4 ? 3u : 0u};
}
// byte-permute selector of code k: byte k, then three zero bytes
__device__ __forceinline__ uint32_t score_sel(uint32_t k) { return k | 0x7770u; }

// The DP keeps G = H - 4 (the value a gap step out of a cell gives), so a
// cell is: a = G(diag) + score + 4 (capped at 253 when CAP: only reads
// longer than 253 reach it), H = max(a, G(up), G(left), 0) in one DPX
// three-way max, G = H - 4.

// One block of the sweep, lanes over the read rows: columns nb+1 .. nb+ncol,
// starting from column nb's values in Hl (H of the lane's rows); lane l holds
// rows x0 = l*R .. x0+R-1 (their codes as score_sel selectors in `sel`) and
// works on column y = nb + t - l + 1 at step t.
// Each column's values go to `store(y, lane's H)`.  Rows past the read take
// code 5 and are not masked: they feed no row of the read.
template <int R, bool CAP, typename Store>
__device__ __forceinline__ void ssw_sweep(const uint8_t *__restrict__ ref_s, const uint32_t (&sel)[R], int nb,
					  int ncol, int nact, const int (&Hl)[R], Store store)
{
	const unsigned FULL = 0xffffffffu;
	const int lane = threadIdx.x & 31;
	int G[R], H[R];
#pragma unroll
	for (int r = 0; r < R; ++r)
		G[r] = Hl[r] - 4;
	// `bot` as of step -1: lane 0 then stands on the left-edge column nb
	// (its saved last row feeds lane 1's first diagonal), the others before it
	int bot = lane == 0 ? G[R - 1] : -4, up_prev = -4;
	const int steps = ncol > 0 ? ncol + nact - 1 : 0;
	for (int t = 0; t < steps; ++t) {
		const int y = nb + t - lane + 1;
		int up_in = __shfl_up_sync(FULL, bot, 1);
		if (lane == 0)
			up_in = -4;
		const int diag_in = up_prev;
		up_prev = up_in;
		if (y > nb && y <= nb + ncol) {
			const ScoreT T = score_table(ref_s[y - 1]);
			int d = diag_in, up = up_in;
#pragma unroll
			for (int r = 0; r < R; ++r) {
				const int s2 = (int)__byte_perm(T.lo, T.hi, sel[r]);
				const int a = CAP ? __viaddmin_s32(d + s2, 2, 253) : d + s2 + 2;
				const int v = __vimax3_s32_relu(a, up, G[r]);
				d = G[r];
				H[r] = v;
				G[r] = v - 4;
				up = G[r];
			}
			bot = G[R - 1];
			store(y, H);
		} else {
			// column nb is the block's left edge: the lane's saved last row
			bot = y == nb ? G[R - 1] : -4;
		}
	}
}

// Stage a call's window and read codes into its shared-memory area.
__device__ inline void ssw_stage(const DevIndex &ix, uint32_t wstart, int ln, const uint8_t *code, int64_t roff,
				 int L, int orient, uint8_t *__restrict__ sm)
{
	const int lane = threadIdx.x & 31;
	uint8_t *ref_s = sm;
	uint8_t *rd_s = sm + SSW_REF_B;
	int *cig_n = reinterpret_cast<int *>(sm + SSW_REF_B + SSW_RD_B);   // DCigT's n, nm
	for (int i = lane; i < ln; i += 32)
		ref_s[i] = __ldg(ix.code + wstart + i);
	for (int i = lane; i < L; i += 32)
		rd_s[i] = read_code(code, roff, L, orient, i);
	if (lane == 0)
		cig_n[0] = cig_n[1] = 0;
}

// Pass 1 of one call with the lanes over the window: lane l owns columns
// y = 32l+1 .. 32l+32 (one checkpoint block, SSW_CK == 32) and steps down
// the read rows, row x = t - l at step t; its left edge (column 32l) comes
// from lane l-1 a step earlier.  A cell is a byte permute for the score, an
// add, one DPX three-way max and the G add.  Columns past the window take code 5, which equals no read code;
// as every value there stays below one of the window's own values, they can
// neither be the maximum nor tie it.  Writes the checkpoint columns
// (y = 32(l+1) <= ln) and returns the end cell by the reference's rule:
// maximum value, then first column, then first row.
template <bool CAP>
__device__ void ssw_pass1_cols(const uint8_t *__restrict__ ref_s, const uint8_t *__restrict__ rd_s, int ln, int L,
			       uint8_t *__restrict__ ck, int COL, int &max_v, int &min_y, int &min_x)
{
	static_assert(SSW_CK == 32, "one checkpoint block per lane");
	const unsigned FULL = 0xffffffffu;
	const int lane = threadIdx.x & 31;
	const int y0 = 32 * lane;
	uint32_t sel[32];
	int G[32];   // G of row x-1 (row -1: H = 0)
#pragma unroll
	for (int c = 0; c < 32; ++c) {
		sel[c] = score_sel(y0 + c < ln ? ref_s[y0 + c] : 5u);
		G[c] = -4;
	}
	uint8_t *ckl = y0 + 32 <= ln ? ck + (size_t)(lane + 1) * COL : nullptr;
	int bv = 0, by = 0, bx = 0, last = -4, dprev = -4;
	const int steps = ln > 0 && L > 0 ? L + 31 : 0;
	for (int t = 0; t < steps; ++t) {
		int lin = __shfl_up_sync(FULL, last, 1);   // G(x, y0) from lane l-1
		if (lane == 0)
			lin = -4;
		const int diag0 = dprev;                   // G(x-1, y0)
		dprev = lin;
		const int x = t - lane;
		if (x >= 0 && x < L) {
			const ScoreT T = score_table(rd_s[x]);
			int d = diag0, left = lin, cm = 0;
#pragma unroll
			for (int c = 0; c < 32; ++c) {
				const int s2 = (int)__byte_perm(T.lo, T.hi, sel[c]);
				const int a = CAP ? __viaddmin_s32(d + s2, 2, 253) : d + s2 + 2;
				const int v = __vimax3_s32_relu(a, G[c], left);
				d = G[c];
				G[c] = v - 4;
				left = G[c];
				cm = max(cm, v);
			}
			if (cm >= bv && cm > 0) {
				int fc = 0;
#pragma unroll
				for (int c = 31; c >= 0; --c)
					if (G[c] == cm - 4)
						fc = c;
				const int yy = y0 + fc + 1;
				if (cm > bv || yy < by) {
					bv = cm;
					by = yy;
					bx = x;
				}
			}
			if (ckl)
				ckl[x] = (uint8_t)(G[31] + 4);
			last = G[31];
		}
	}
	max_v = __reduce_max_sync(FULL, bv);
	min_y = __reduce_min_sync(FULL, bv == max_v ? by : 0x7fffffff);
	min_x = __reduce_min_sync(FULL, (bv == max_v && by == min_y) ? bx : 0x7fffffff);
	__syncwarp();
}

// The reference's traceback and output of one call whose sweep has run
// (end cell max_v / min_y / min_x; checkpoints in its area).
template <int R, bool CAP, class K>
__device__ void ssw_walk(const DevIndex &ix, uint32_t wstart, int ln, int L, int start, uint32_t tl,
			 uint8_t *__restrict__ sm, SswOutT<K> &out, int &flags, int max_v, int min_y, int min_x)
{
	constexpr int MCAP = K::M, CCAP = K::C;
	const unsigned FULL = 0xffffffffu;
	const int lane = threadIdx.x & 31;
	const int x0 = lane * R;
	const int COL = 32 * R;
	uint8_t *ref_s = sm;
	uint8_t *rd_s = sm + SSW_REF_B;
	DCigT<K> &cig = *reinterpret_cast<DCigT<K> *>(sm + SSW_REF_B + SSW_RD_B);
	uint8_t *ck = sm + SSW_REF_B + SSW_RD_B + ssw_cig_b<K>();
	uint8_t *tb = ck + (size_t)SSW_NCK * COL;
	uint32_t rsel[R];   // the lane's read rows as score selectors
#pragma unroll
	for (int r = 0; r < R; ++r)
		rsel[r] = score_sel(x0 + r < L ? rd_s[x0 + r] : 5u);
	const int nact = (L + R - 1) / R;
	// self-check of the end cell before the walk (a bad one reports flag
	// F_SSW instead of reading outside the warp's area)
	if (max_v > 0 && (min_y < 1 || min_y > ln || min_x < 0 || min_x >= L)) {
		if (lane == 0) {
			out.score = -1002;
			out.skip = min_y;
			out.pstart = min_x;
			out.ok = 0;
			out.cig.n = out.cig.nm = 0;
			flags |= F_SSW;
		}
		return;
	}

	const uint8_t *ra = ix.seq + wstart;
	const bool w0 = lane == 0;
	// cig_add with the CIGAR's counts and last op kept in registers (the
	// same in every lane; lane 0 stores to the shared-memory CIGAR), so the
	// serial walk does not reload them from shared memory at each step
	int cn = 0, cnm = 0;
	uint32_t clast = 0;   // op[cn - 1] when cn > 0
	auto add = [&](int type, unsigned cnt, const uint8_t *mc) {
		cnt &= 0xffffu;
		if (cnt == 0)
			return;
		if (cn > 1 && op_type(clast) == OP_S) {
			if (type != OP_D) {
				clast = (((op_cnt(clast) + cnt) & 0xffffu) << 4) | OP_S;
				if (w0)
					cig.op[cn - 1] = clast;
			}
			return;
		}
		if (mc) {
			if (cnm + (int)cnt > MCAP) {
				flags |= F_MCAP;
			} else {
				if (w0)
					for (unsigned t = 0; t < cnt; ++t)
						cig.miss[cnm + t] = mc[t];
				cnm += (int)cnt;
			}
		}
		if (cn > 0 && op_type(clast) == type) {
			clast = (((op_cnt(clast) + cnt) & 0xffffu) << 4) | (uint32_t)type;
			if (w0)
				cig.op[cn - 1] = clast;
			return;
		}
		if (cn == CCAP) {
			flags |= F_CCAP;
			return;
		}
		clast = (cnt << 4) | (uint32_t)type;
		if (w0)
			cig.op[cn] = clast;
		++cn;
	};
	// block of saved columns [nb, nb + SSW_CK] around the walk
	int nb = -1, bad_walk = 0;
	// (rows 0 .. xmax only: the walk never goes down again)
	auto load_block = [&](int b, int xmax) {
		if (b < 0 || b >= ln || (b & (SSW_CK - 1)) || b / SSW_CK >= SSW_NCK) {
			bad_walk = 3;
			return;
		}
		nb = b;
		__syncwarp();
		int H0[R];
		const uint8_t *c0 = ck + (size_t)(b / SSW_CK) * COL;
#pragma unroll
		for (int r = 0; r < R; ++r) {
			H0[r] = b == 0 ? 0 : c0[x0 + r];
			tb[x0 + r] = (uint8_t)H0[r];
		}
		const int ncol = ln - b < SSW_CK ? ln - b : SSW_CK;
		const int nrow = xmax / R + 1;
		ssw_sweep<R, CAP>(ref_s, rsel, b, ncol, nrow < nact ? nrow : nact, H0, [&](int y, const int (&H)[R]) {
			uint8_t *c = tb + (size_t)(y - b) * COL + x0;
#pragma unroll
			for (int r = 0; r < R; ++r)
				c[r] = (uint8_t)H[r];
		});
		__syncwarp();
	};
	auto HV = [&](int x, int yy) -> int {
		if (yy == 0)
			return 0;
		if (yy - nb < 0 || yy - nb > SSW_CK || x < 0 || x >= COL) {
			bad_walk = 5;
			return 0;
		}
		return tb[(size_t)(yy - nb) * COL + x];
	};
	const int end_ref = max_v > 0 ? min_y - 1 : -1;
	int begin_ref = end_ref, score = 0, end_read = L - 1;
	if (max_v < (L >> 2) || max_v == 0) {
		score = L;
		add(OP_S, (unsigned)L, nullptr);
	} else {
		if (min_x < end_read)
			end_read = min_x;
		int x_pos = end_read, y_pos = end_ref + 1, begin_read = end_read;
		const int right = L - end_read - 1;
		if (right > 0) {
			if (right < 5) {
				for (int i = L - 1, j = end_ref + right; i > end_read; --i, --j) {
					if (j >= ln) {
						add(OP_S, 1, nullptr);
						++score;
					} else if (rd_s[i] == ref_s[j]) {
						add(OP_M, 1, nullptr);
					} else {
						add(OP_X, 1, ra + j);
						++score;
					}
				}
			} else {
				score += right;
				add(OP_S, (unsigned)right, nullptr);
			}
		}
		load_block((y_pos - 1) / SSW_CK * SSW_CK, x_pos);
		int cur = HV(x_pos, y_pos), dir = 0;
		// the op of the walk's current cell, by the move that reached it
		auto emit = [&](uint8_t qb, uint8_t rb) {
			if (dir == 0) {
				if (qb == rb) {
					add(OP_M, 1, nullptr);
				} else {
					add(OP_X, 1, ra + begin_ref);
					++score;
				}
			} else if (dir == 1) {   // a step along the reference
				++score;
				add(OP_I, 1, nullptr);
			} else {                 // a step along the read
				++score;
				add(OP_D, 1, ra + begin_ref);
			}
		};
		for (;;) {
			// Diagonal runs, up to 32 cells at once: lane k takes the cell k
			// steps down the diagonal and tells whether the walk, there,
			// moves diagonally again (inside the block, away from the
			// walk's ends and bounds).  The leading run of such cells is the
			// walk's next steps; their ops are M/X (the first cell's by the
			// move that reached it).  The cell after the run takes the
			// single step below.
			if (!bad_walk) {
				const int xk = x_pos - lane, yk = y_pos - lane;
				bool go = false, mis = false;
				int hd = 0;
				if (xk >= 1 && xk < L && yk >= 2 && yk - 1 < ln && yk - 1 >= nb && yk - nb <= SSW_CK) {
					const int hc = lane == 0 ? cur : tb[(size_t)(yk - nb) * COL + xk];
					hd = tb[(size_t)(yk - 1 - nb) * COL + xk - 1];
					const uint8_t q = rd_s[xk], r = ref_s[yk - 1];
					mis = q != r;
					go = hd != 0 && hc == hd + mat_score(q, r);
				}
				const unsigned run = __ballot_sync(FULL, go);
				const int m = run == FULL ? 32 : __ffs(~run) - 1;
				if (m > 0) {
					const unsigned xm = __ballot_sync(FULL, mis);
					emit(rd_s[begin_read], ref_s[begin_ref]);
					for (int k = 1; k < m;) {
						const unsigned rest = (xm >> k) << k;
						int nx = rest ? __ffs(rest) - 1 : m;
						nx = nx < m ? nx : m;
						if (nx > k)
							add(OP_M, (unsigned)(nx - k), nullptr);
						if (nx < m) {
							add(OP_X, 1, ra + (begin_ref - nx));
							++score;
						}
						k = nx + 1;
					}
					cur = __shfl_sync(FULL, hd, m - 1);
					x_pos -= m;
					y_pos -= m;
					begin_read -= m;
					begin_ref -= m;
					dir = 0;
				}
			}
			if (bad_walk || begin_read < 0 || begin_read >= L || begin_ref < 0 || begin_ref >= ln) {
				bad_walk = bad_walk ? bad_walk : 6;
				break;
			}
			const uint8_t qb = rd_s[begin_read], rb = ref_s[begin_ref];
			emit(qb, rb);
			if (x_pos == 0 || y_pos == 1)
				break;
			if (y_pos - 1 < nb)   // the walk left the block: recompute the one before
				load_block(nb - SSW_CK, x_pos);
			const int diag = HV(x_pos - 1, y_pos - 1);
			const int up = HV(x_pos - 1, y_pos);
			const int left = HV(x_pos, y_pos - 1);
			if (cur == diag + mat_score(qb, rb)) {
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
		if (begin_read < 5) {
			for (--begin_read, --begin_ref; begin_read >= 0; --begin_read, --begin_ref) {
				if (begin_ref < 0) {
					add(OP_S, 1, nullptr);
					++score;
				} else if (rd_s[begin_read] == ref_s[begin_ref]) {
					add(OP_M, 1, nullptr);
				} else {
					add(OP_X, 1, ra + begin_ref);
					++score;
				}
			}
		} else if (begin_read > 0) {
			score += begin_read;
			add(OP_S, (unsigned)begin_read, nullptr);
		}
	}
	__syncwarp();
	if (__reduce_max_sync(FULL, bad_walk)) {
		if (lane == 0) {
			out.score = -2000 - bad_walk;
			out.ok = 0;
			out.cig.n = out.cig.nm = 0;
			flags |= F_SSW;
		}
		return;
	}
	__syncwarp();   // lane 0's CIGAR stores before the copy
	const int n = cn, nm = cnm;
	for (int k = lane; k < n; k += 32)
		out.cig.op[k] = cig.op[k];
	for (int k = lane; k < nm; k += 32)
		out.cig.miss[k] = cig.miss[k];
	if (w0) {
		const int skip = begin_ref;
		out.cig.n = n;
		out.cig.nm = nm;
		out.score = score;
		out.skip = skip;
		out.pstart = start + skip;
		// acceptance test of re_mapSW (src/hash_align.c:788-792)
		out.ok = !(score > L / 2 || start + skip < 0 || (uint32_t)(start + skip + L) > tl);
	}
}

// One call: stage, pass 1 over the window columns, walk.  Called by all
// 32 lanes of a warp; `sm` is the warp's shared-memory area
// (ssw_smem_per_warp(L) bytes at least).  Fills `out` (lane 0 writes the
// scalars; the CIGAR is copied by the warp).
template <int R, class K = CapsStd>
__device__ void ssw_warp_r(const DevIndex &ix, uint32_t wstart, int ln, const uint8_t *code, int64_t roff, int L,
			   int orient, int start, uint32_t tl, uint8_t *__restrict__ sm, SswOutT<K> &out, int &flags)
{
	ssw_stage(ix, wstart, ln, code, roff, L, orient, sm);
	__syncwarp();
	uint8_t *ck = sm + SSW_REF_B + SSW_RD_B + ssw_cig_b<K>();
	int max_v, min_y, min_x;
	if (L > 253) {
		ssw_pass1_cols<true>(sm, sm + SSW_REF_B, ln, L, ck, 32 * R, max_v, min_y, min_x);
		ssw_walk<R, true, K>(ix, wstart, ln, L, start, tl, sm, out, flags, max_v, min_y, min_x);
	} else {
		ssw_pass1_cols<false>(sm, sm + SSW_REF_B, ln, L, ck, 32 * R, max_v, min_y, min_x);
		ssw_walk<R, false, K>(ix, wstart, ln, L, start, tl, sm, out, flags, max_v, min_y, min_x);
	}
}

// the call's read length picks the rows-per-lane instantiation
__device__ inline void ssw_warp(const DevIndex &ix, uint32_t wstart, int ln, const uint8_t *code, int64_t roff,
				int L, int orient, int start, uint32_t tl, uint8_t *__restrict__ sm, SswOut &out,
				int &flags)
{
	switch (ssw_rows(L)) {
	case 1: ssw_warp_r<1>(ix, wstart, ln, code, roff, L, orient, start, tl, sm, out, flags); break;
	case 2: ssw_warp_r<2>(ix, wstart, ln, code, roff, L, orient, start, tl, sm, out, flags); break;
	case 3: ssw_warp_r<3>(ix, wstart, ln, code, roff, L, orient, start, tl, sm, out, flags); break;
	case 4: ssw_warp_r<4>(ix, wstart, ln, code, roff, L, orient, start, tl, sm, out, flags); break;
	case 5: ssw_warp_r<5>(ix, wstart, ln, code, roff, L, orient, start, tl, sm, out, flags); break;
	case 6: ssw_warp_r<6>(ix, wstart, ln, code, roff, L, orient, start, tl, sm, out, flags); break;
	case 8: ssw_warp_r<8>(ix, wstart, ln, code, roff, L, orient, start, tl, sm, out, flags); break;
	default: ssw_warp_r<10>(ix, wstart, ln, code, roff, L, orient, start, tl, sm, out, flags); break;
	}
}

// The wide pass's form: every read length in the widest row layout, the
// CIGAR in a CapsWide area (ssw_smem_wide() bytes).
__device__ inline void ssw_warp(const DevIndex &ix, uint32_t wstart, int ln, const uint8_t *code, int64_t roff,
				int L, int orient, int start, uint32_t tl, uint8_t *__restrict__ sm,
				SswOutT<CapsWide> &out, int &flags)
{
	ssw_warp_r<SSW_WIDE_R, CapsWide>(ix, wstart, ln, code, roff, L, orient, start, tl, sm, out, flags);
}

}  // namespace hg
