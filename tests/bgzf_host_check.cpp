// The device's BGZF encoder (hera_b200/csrc/hera_bgzf_core.h) compiled for
// the host, for the CPU suite: blocks of a buffer, back to back.
#include "../hera_b200/csrc/hera_bgzf_core.h"

#include <stdint.h>
#include <vector>

extern "C" long long bgzf_host(const uint8_t *in, long long n, uint8_t *out, long long cap)
{
	uint32_t t[256];
	bgzf::crc_table(t);
	std::vector<uint16_t> table(bgzf::HASH_SIZE);
	std::vector<uint8_t> blk(bgzf::BLOCK_MAX);
	long long o = 0;
	for (long long a = 0; a < n; a += bgzf::BLOCK_IN) {
		const int k = n - a < bgzf::BLOCK_IN ? (int)(n - a) : bgzf::BLOCK_IN;
		const int z = bgzf::block(in + a, k, blk.data(), table.data(), t);
		if (o + z > cap)
			return -1;
		for (int i = 0; i < z; ++i)
			out[o + i] = blk[i];
		o += z;
	}
	return o;
}
