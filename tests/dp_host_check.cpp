// Test-only: the batched form's gap DP (sw_align_bits in
// hera_b200/csrc/hera_device.cuh) compiled for the host and called the way
// k_dp_reg calls it: row summaries in the score-only mode (WRITE_BAM 1),
// whole rows with traceback (WRITE_BAM 0).  Built and driven by
// tests/test_dp_host.py.
#include "dp_host_shim.h"
#include "../hera_b200/csrc/hera_device.cuh"

#include <random>
#include <string>
#include <vector>

using namespace hg;

namespace {

uint8_t code_of_host(uint8_t c)
{
	const uint8_t x = c | 0x20;
	return x == 'a' ? 0 : x == 'c' ? 1 : x == 'g' ? 2 : x == 't' ? 3 : 4;
}

struct Call {
	std::vector<uint8_t> asc, code, qc;
	RefWin r;
	QView qv;
	int E;
};

// the job as k_build makes it: the window's ASCII and codes (padded as the
// device copy is), the query's codes, reversed for a prefix DP (err < 0)
bool setup(const char *ref, int rl, const char *q, int ql, int err, Call &c)
{
	c.E = (err < 0 ? -err : err) + 1;
	if (ql <= 0 || (c.E == 8 && rl < 9) || (c.E == 4 && rl < 5) || (c.E != 8 && c.E != 4))
		return false;   // k_dp_generic's jobs
	c.asc.assign((size_t)rl + 64, 0);
	c.code.assign((size_t)rl + 64, 4);
	c.qc.resize((size_t)ql);
	for (int i = 0; i < rl; ++i) {
		c.asc[i] = (uint8_t)ref[i];
		c.code[i] = code_of_host((uint8_t)ref[i]);
	}
	for (int i = 0; i < ql; ++i)
		c.qc[i] = code_of_host((uint8_t)q[i]);
	const bool rev = err < 0;
	c.r = RefWin{c.code.data(), c.asc.data(), 0, (uint32_t)rl, rev};
	c.qv = QView{rev ? c.qc.data() + (ql - 1) : c.qc.data(), rev ? -1 : 1};
	return true;
}

template <bool SUM>
int run(Call &c, int rl, int ql, bool score_only, DCig &cig, int &flags)
{
	uint32_t cells = 0;
	cig.n = cig.nm = 0;
	if (c.E == 8) {
		std::vector<typename DpRow<8, SUM>::T> rows(MAX_DP_ROWS + 1);
		return sw_align_bits<8, SUM>(c.r, c.qv, (uint32_t)rl, (uint32_t)ql, score_only, cig, rows.data(), flags,
					     cells);
	}
	std::vector<typename DpRow<4, SUM>::T> rows(MAX_DP_ROWS + 1);
	return sw_align_bits<4, SUM>(c.r, c.qv, (uint32_t)rl, (uint32_t)ql, score_only, cig, rows.data(), flags, cells);
}

}   // namespace

// One call as k_dp_reg runs it.  Returns 1 when the register form handles
// the job (0: a k_dp_generic job, nothing written).
extern "C" int dp_bits(const char *ref, int rl, const char *q, int ql, int err, int write_bam, int *score,
		       uint32_t *ops, int *n_ops, char *miss, int *n_miss, int *flags)
{
	Call c;
	if (!setup(ref, rl, q, ql, err, c))
		return 0;
	DCig cig;
	*flags = 0;
	*score = write_bam == 1 ? run<true>(c, rl, ql, true, cig, *flags) : run<false>(c, rl, ql, false, cig, *flags);
	*n_ops = cig.n;
	*n_miss = cig.nm;
	for (int k = 0; k < cig.n; ++k)
		ops[k] = cig.op[k];
	for (int k = 0; k < cig.nm; ++k)
		miss[k] = (char)cig.miss[k];
	return 1;
}

// Random score-only calls, row summaries against whole rows (the same
// algorithm with the rows kept): reads with N's, mutation rates 2-42%,
// both error caps and both orientations.  Returns the calls that differ;
// *n and *clipped count the calls made and those ending in a soft clip
// (the shrink loop's path).
extern "C" long dp_summaries_vs_rows(int iters, unsigned seed, long *n, long *clipped)
{
	std::mt19937 rng(seed);
	const char *B = "ACGTN";
	long bad = 0;
	*n = *clipped = 0;
	for (int it = 0; it < iters; ++it) {
		const int len = 1 + (int)(rng() % 120);
		const int e = (rng() & 1) ? 7 : 3;
		const int err = (rng() & 1) ? e : -e;
		const int rate = 2 + (int)(rng() % 40);
		std::string q, ref;
		for (int i = 0; i < len; ++i)
			q += B[rng() % (rng() % 30 ? 4 : 5)];
		for (int i = 0; i < len; ++i) {
			const int x = (int)(rng() % 100);
			if (x < rate / 2) {
				ref += B[rng() % 4];
			} else if (x < rate * 3 / 4) {
				ref += q[i];
				ref += B[rng() % 4];
			} else if (x >= rate) {
				ref += q[i];
			}
		}
		const int extra = (int)(rng() % 16);
		for (int i = 0; i < extra; ++i)
			ref += B[rng() % 4];
		if (ref.size() < q.size())
			continue;
		Call c;
		if (!setup(ref.data(), (int)ref.size(), q.data(), (int)q.size(), err, c))
			continue;
		DCig a, b;
		int fa = 0, fb = 0;
		const int sa = run<true>(c, (int)ref.size(), (int)q.size(), true, a, fa);
		const int sb = run<false>(c, (int)ref.size(), (int)q.size(), true, b, fb);
		bool same = sa == sb && a.n == b.n && a.nm == b.nm && fa == fb;
		for (int k = 0; same && k < a.n; ++k)
			same = a.op[k] == b.op[k];
		++*n;
		if (a.n && op_type(a.op[0]) == OP_S)
			++*clipped;
		bad += same ? 0 : 1;
	}
	return bad;
}
