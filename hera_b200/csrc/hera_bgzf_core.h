// hera_bgzf_core.h -- BGZF blocks (the BAM container hera's bam_write
// writes, src/hash_align.c:48-136) from plain bytes: each block is a gzip
// member with the BGZF "BC" extra field, one raw DEFLATE stream (RFC 1951)
// and the CRC-32 and size of its input.  The DEFLATE stream here is greedy
// LZ77 (one candidate per 4-byte hash, window 32 KiB, matches 3..258) coded
// with the fixed Huffman codes of RFC 1951 3.2.6, or a stored block when
// that would not be smaller than the input.  The bytes differ from zlib's;
// what they decompress to is the input, which is what a BAM reader sees.
//
// Plain C++ usable on the device (one thread per block) and on the host (the
// CPU checks compile this header alone).
#pragma once

#include <stdint.h>
#include <string.h>

#ifdef __CUDACC__
#define BGZF_HD __host__ __device__
#else
#define BGZF_HD
#endif

namespace bgzf {

constexpr int BLOCK_IN = 0xff00;          // input bytes per block (as htslib's writer)
constexpr int BLOCK_MAX = 0x10000;        // a BGZF block's size limit (BSIZE is 16 bits)
constexpr int HEADER = 18, FOOTER = 8;
constexpr int HASH_BITS = 13;             // default table: 2^13 uint16 positions + 1 (0 = empty)
constexpr int HASH_SIZE = 1 << HASH_BITS;
constexpr int WINDOW = 32768;
constexpr int MIN_MATCH = 3, MAX_MATCH = 258;

// CRC-32 (ISO 3309 / gzip: reflected polynomial 0xEDB88320), byte-wise
// with a 256-entry table the caller makes once (crc_table)
BGZF_HD inline void crc_table(uint32_t *t)
{
	for (uint32_t n = 0; n < 256; ++n) {
		uint32_t c = n;
		for (int k = 0; k < 8; ++k)
			c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
		t[n] = c;
	}
}

BGZF_HD inline uint32_t crc32(const uint32_t *t, const uint8_t *p, int n)
{
	uint32_t c = 0xffffffffu;
	for (int i = 0; i < n; ++i)
		c = t[(c ^ p[i]) & 0xff] ^ (c >> 8);
	return c ^ 0xffffffffu;
}

// LSB-first bit writer into out[0 .. cap)
struct Bits {
	uint8_t *out;
	int cap, pos;
	uint64_t acc;
	int n;
	bool full;
	BGZF_HD void put(uint32_t v, int k)   // k <= 32 bits, LSB first
	{
		acc |= (uint64_t)v << n;
		n += k;
		while (n >= 8) {
			if (pos < cap)
				out[pos] = (uint8_t)acc;
			else
				full = true;
			++pos;
			acc >>= 8;
			n -= 8;
		}
	}
	BGZF_HD void flush()
	{
		if (n > 0)
			put(0, 8 - n);
	}
};

// a Huffman code of `len` bits, MSB first (RFC 1951 3.1.1), as LSB-first bits
BGZF_HD inline uint32_t rev(uint32_t code, int len)
{
	uint32_t r = 0;
	for (int i = 0; i < len; ++i)
		r |= ((code >> i) & 1u) << (len - 1 - i);
	return r;
}

// fixed literal/length code of symbol s (RFC 1951 3.2.6)
BGZF_HD inline void put_litlen(Bits &b, int s)
{
	if (s < 144)
		b.put(rev(0x30 + s, 8), 8);
	else if (s < 256)
		b.put(rev(0x190 + (s - 144), 9), 9);
	else if (s < 280)
		b.put(rev(s - 256, 7), 7);
	else
		b.put(rev(0xC0 + (s - 280), 8), 8);
}

BGZF_HD inline void put_match(Bits &b, int len, int dist)
{
	// length: codes 257..285 (RFC 1951 3.2.5)
	static const uint16_t lbase[29] = {3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 15, 17, 19, 23, 27, 31,
					   35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
	static const uint8_t lext[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2,
					 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
	static const uint16_t dbase[30] = {1, 2, 3, 4, 5, 7, 9, 13, 17, 25, 33, 49, 65, 97, 129,
					   193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097,
					   6145, 8193, 12289, 16385, 24577};
	static const uint8_t dext[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8,
					 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
	int li = 28;
	while (li > 0 && lbase[li] > len)
		--li;
	if (len == 258)
		li = 28;
	else if (li == 28)
		li = 27;
	put_litlen(b, 257 + li);
	if (lext[li])
		b.put((uint32_t)(len - lbase[li]), lext[li]);
	int di = 29;
	while (di > 0 && dbase[di] > dist)
		--di;
	b.put(rev((uint32_t)di, 5), 5);
	if (dext[di])
		b.put((uint32_t)(dist - dbase[di]), dext[di]);
}

BGZF_HD inline uint32_t load4(const uint8_t *p)
{
	return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

// One fixed-Huffman DEFLATE block (BFINAL set) of in[0 .. n) into
// out[0 .. cap); returns its bytes, or -1 if it does not fit.  `table`:
// 2^HB uint16 of scratch (cleared here).
template <int HB = HASH_BITS>
BGZF_HD inline int deflate_fixed(const uint8_t *in, int n, uint8_t *out, int cap, uint16_t *table)
{
	for (int i = 0; i < (1 << HB); ++i)
		table[i] = 0;
	Bits b{out, cap, 0, 0, 0, false};
	b.put(1, 1);   // BFINAL
	b.put(1, 2);   // BTYPE = 01, fixed codes
	int p = 0;
	while (p < n) {
		int len = 0, dist = 0;
		if (p + 4 <= n) {
			const uint32_t h = (load4(in + p) * 2654435761u) >> (32 - HB);
			const int cand = (int)table[h] - 1;
			table[h] = (uint16_t)(p + 1);
			if (cand >= 0 && p - cand <= WINDOW) {
				const int lim = n - p < MAX_MATCH ? n - p : MAX_MATCH;
				while (len < lim && in[cand + len] == in[p + len])
					++len;
				dist = p - cand;
			}
		}
		if (len >= MIN_MATCH) {
			put_match(b, len, dist);
			// index the positions the match covers
			for (int q = p + 1; q < p + len && q + 4 <= n; ++q)
				table[(load4(in + q) * 2654435761u) >> (32 - HB)] = (uint16_t)(q + 1);
			p += len;
		} else {
			put_litlen(b, in[p]);
			++p;
		}
		if (b.full)
			return -1;
	}
	put_litlen(b, 256);   // end of block
	b.flush();
	return b.full ? -1 : b.pos;
}

// One BGZF block of in[0 .. n) (n <= BLOCK_IN) into out (BLOCK_MAX bytes);
// returns its size.
template <int HB = HASH_BITS>
BGZF_HD inline int block(const uint8_t *in, int n, uint8_t *out, uint16_t *table, const uint32_t *crc_t)
{
	static const uint8_t head[HEADER - 2] = {31, 139, 8, 4, 0, 0, 0, 0, 0, 255, 6, 0, 66, 67, 2, 0};
	for (int i = 0; i < HEADER - 2; ++i)
		out[i] = head[i];
	int body = deflate_fixed<HB>(in, n, out + HEADER, n, table);   // only if smaller than the input
	if (body < 0) {   // a stored block: BFINAL, BTYPE 00, LEN, NLEN, the bytes
		uint8_t *o = out + HEADER;
		o[0] = 1;
		o[1] = (uint8_t)n;
		o[2] = (uint8_t)(n >> 8);
		o[3] = (uint8_t)~n;
		o[4] = (uint8_t)(~n >> 8);
		memcpy(o + 5, in, (size_t)n);
		body = n + 5;
	}
	const int total = HEADER + body + FOOTER;
	out[16] = (uint8_t)(total - 1);
	out[17] = (uint8_t)((total - 1) >> 8);
	const uint32_t crc = crc32(crc_t, in, n);
	uint8_t *f = out + HEADER + body;
	for (int i = 0; i < 4; ++i) {
		f[i] = (uint8_t)(crc >> (8 * i));
		f[4 + i] = (uint8_t)((uint32_t)n >> (8 * i));
	}
	return total;
}

}  // namespace bgzf
