// hera_bam_core.h -- the host tail's BAM records (`-w`), one read pair at a
// time, in code that compiles for the device (the kernels of hera_bam.cuh)
// and for the host alike.
//
// For pair i the writer reproduces the records hera's align_pair_read
// appends to its BGZF stream (src/hash_align.c:1735-1804): the branch and
// flags it picks, bam_write_pair's primary and secondary record pairs
// (src/bam_write.c:382-416), write_alignment_pair (:349-380), and per record
// pack_bam_core / convert_cigar / add_padding / compact_inf / pack_bam_block
// (:89-310) with the transcript -> genome map (GENE_MAP).
//
// hera mutates the reads while it writes (reverse_str / reverse_qual around
// each call, and the writer cuts "/1" off a name with a NUL).  Here the
// inputs stay read-only: a read view carries "reversed" and "cut at"
// state and applies it on access.
#pragma once

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define BAM_HD __host__ __device__
#else
#define BAM_HD
#endif

namespace bamw {

constexpr int MAX_CIG = 256;    // CIGAR ops of one record after intron padding
constexpr int MAX_MD = 640;     // MD string bytes of one record
constexpr int QUAL_TABLE = 65;  // mapping qualities for 0..64 hits (get_qual)

// error bits of a pair
constexpr uint32_t E_CIG = 1;   // more CIGAR ops than MAX_CIG
constexpr uint32_t E_MD = 2;    // MD string longer than MAX_MD
constexpr uint32_t E_NAME = 4;  // a name the writer would cut twice
constexpr uint32_t E_HITS = 8;  // more hits than the quality table covers, or a hit index past a list
constexpr uint32_t E_MAP = 16;  // a position or alignment past the transcript's last exon
constexpr uint32_t E_MISS = 32; // a CIGAR asking for more mismatch bytes than the record holds

enum { B_MATCH = 0, B_DELETE = 2, B_SKIP = 3, B_DIFF = 8 };

struct GeneMap {
	uint32_t n_chr;
	const uint32_t *chr_len;    // [n_chr]
	const uint32_t *exon_off;   // [n_trans + 1]
	const uint32_t *starts, *ends;
	const uint32_t *chr, *gene; // [n_trans]
	BAM_HD uint32_t start(uint32_t t, uint32_t e) const { return starts[exon_off[t] + e]; }
	BAM_HD uint32_t end(uint32_t t, uint32_t e) const { return ends[exon_off[t] + e]; }
	BAM_HD uint32_t last(uint32_t t) const { return ends[exon_off[t + 1] - 1]; }
	BAM_HD uint32_t exons(uint32_t t) const { return exon_off[t + 1] - exon_off[t]; }
};

// One strand of a Candidate, as flat records hold it.
struct Strand {
	uint32_t n;
	const uint32_t *pos;
	const int32_t *p;
	uint32_t n_cigar, n_miss;
	const uint32_t *ops;        // (count << 4) | type
	const char *miss;
};

struct Cand {
	Strand s[2];
	int err[2];
	int pair;
};

// ascii_table of src/hash_align.c:6-23: A/a 0, C/c 1, G/g 2, T/t 3, else 4
BAM_HD inline int code(unsigned char c)
{
	switch (c) {
	case 'A': case 'a': return 0;
	case 'C': case 'c': return 1;
	case 'G': case 'g': return 2;
	case 'T': case 't': return 3;
	default: return 4;
	}
}

// bam_nt16_table, src/bam_write.c:3-20 (=ACMGRSVTWYHKDBN)
BAM_HD inline unsigned char nt16(unsigned char c)
{
	switch (c) {
	case '=': return 0;
	case 'A': case 'a': return 1;
	case 'C': case 'c': return 2;
	case 'M': case 'm': return 3;
	case 'G': case 'g': return 4;
	case 'R': case 'r': return 5;
	case 'S': case 's': return 6;
	case 'V': case 'v': return 7;
	case 'T': case 't': return 8;
	case 'W': case 'w': return 9;
	case 'Y': case 'y': return 10;
	case 'H': case 'h': return 11;
	case 'K': case 'k': return 12;
	case 'D': case 'd': return 13;
	case 'B': case 'b': return 14;
	default: return 15;
	}
}

BAM_HD inline char upper_acgt(unsigned char c)   // what the front half's two reverse_str calls leave
{
	const int k = code(c);
	return k > 3 ? (char)c : "ACGT"[k];
}

BAM_HD inline char comp(char c)                 // reverse_str's complement (src/hash_align.c:217-232)
{
	const int k = code((unsigned char)c);
	return k > 3 ? c : "ACGT"[3 - k];
}

// A read as the tail sees it at the moment of a write.
struct Read {
	const char *seq, *qual, *name;
	int len;
	bool rev;       // reverse_str + reverse_qual applied an odd number of times
	int name_l;     // strlen of the name now
	int cut;        // where the writer's NUL went (-1: nowhere yet)
	BAM_HD char base(int j) const
	{
		if (!rev)
			return upper_acgt((unsigned char)seq[j]);
		// reverse_str: mirrored position, complemented; an odd length's
		// middle base is complemented too
		return comp(upper_acgt((unsigned char)seq[len - 1 - j]));
	}
	BAM_HD char q(int j) const { return rev ? qual[len - 1 - j] : qual[j]; }
	BAM_HD char name_byte(int j) const { return j == cut ? 0 : name[j]; }
};

// The bytes of a pair's records go to `out` from `at` (size pass: out null).
struct Sink {
	uint8_t *out;
	uint64_t at;
	uint64_t end = ~0ull;   // no byte is stored at or past end
	BAM_HD void put(uint8_t b)
	{
		if (out && at < end)
			out[at] = b;
		++at;
	}
	BAM_HD void u32(uint32_t v)
	{
		put(v & 255); put(v >> 8 & 255); put(v >> 16 & 255); put(v >> 24);
	}
};

BAM_HD inline int overlap_gene(const GeneMap &g, uint32_t t1, uint32_t t2)   // check_overlapGene
{
	if (t1 == t2 || g.gene[t1] == g.gene[t2])
		return 1;
	if (g.chr[t1] != g.chr[t2])
		return 0;
	const uint32_t s0 = g.start(t1, 0), s1 = g.start(t2, 0), e0 = g.last(t1), e1 = g.last(t2);
	return !(s1 > e0 || s0 > e1);
}

BAM_HD inline int reg2bin(unsigned int beg, unsigned int end)   // bam_reg2bin
{
	--end;
	if (beg >> 14 == end >> 14) return 4681 + (beg >> 14);
	if (beg >> 17 == end >> 17) return 585 + (beg >> 17);
	if (beg >> 20 == end >> 20) return 73 + (beg >> 20);
	if (beg >> 23 == end >> 23) return 9 + (beg >> 23);
	if (beg >> 26 == end >> 26) return 1 + (beg >> 26);
	return 0;
}

BAM_HD inline unsigned int make_flag(unsigned pair, unsigned proper, unsigned map, unsigned mmap, unsigned rev,
				     unsigned mrev, unsigned first, unsigned last)
{
	return last << 7 | first << 6 | mrev << 5 | rev << 4 | mmap << 3 | map << 2 | proper << 1 | pair;
}

// What pack_bam_core computes for one record before the bytes.
struct Core {
	int bin, qual, ref, pos, n_cigar;
	unsigned int md_len, coord, match, align_len;
	uint32_t cig[MAX_CIG];
	char md[MAX_MD + 16];
};

struct Ctx {
	GeneMap g;
	const uint32_t *qual_table;   // get_qual(n), n < QUAL_TABLE, computed on the host
	uint32_t err;
};

BAM_HD inline void cig_push(Ctx &x, Core &c, unsigned int *n, uint32_t v)
{
	if (*n < (unsigned)MAX_CIG)
		c.cig[*n] = v;
	else
		x.err |= E_CIG;
	++*n;
}

// add_padding (src/bam_write.c:89-116)
BAM_HD inline void pad(Ctx &x, Core &c, unsigned int *n, unsigned int *l, uint32_t t, unsigned int len,
		       unsigned int type, unsigned int genome)
{
	if ((type != B_MATCH && type != B_DIFF) || genome == 1) {
		cig_push(x, c, n, len << 4 | type);
		return;
	}
	*l += len;
	while (*l > x.g.end(t, c.coord) + 1) {
		if (c.coord + 1 >= x.g.exons(t)) {   // hera would read past the exon arrays
			x.err |= E_MAP;
			break;
		}
		len -= *l - x.g.end(t, c.coord) - 1;
		cig_push(x, c, n, len << 4 | type);
		len = x.g.start(t, c.coord + 1) - x.g.end(t, c.coord) - 1;
		c.align_len += len;
		cig_push(x, c, n, len << 4 | B_SKIP);
		len = *l - x.g.end(t, c.coord) - 1;
		*l += x.g.start(t, c.coord + 1) - x.g.end(t, c.coord) - 1;
		++c.coord;
	}
	cig_push(x, c, n, len << 4 | type);
}

BAM_HD inline void md_put(Ctx &x, Core &c, char ch)
{
	if (c.md_len < (unsigned)MAX_MD)
		c.md[c.md_len] = ch;
	else
		x.err |= E_MD;
	++c.md_len;
}

BAM_HD inline char miss_at(Ctx &x, const Strand &s, unsigned int k)
{
	if (k < s.n_miss)
		return s.miss[k];
	x.err |= E_MISS;
	return 0;
}

// convert_cigar (src/bam_write.c:118-197)
BAM_HD inline void convert(Ctx &x, Core &c, const Strand &s, uint32_t hit, unsigned int genome)
{
	const GeneMap &g = x.g;
	if (hit >= s.n) {   // a mate list shorter than the hit index hera walks
		x.err |= E_HITS;
		return;
	}
	const uint32_t t = s.pos[hit];
	if (genome == 0) {
		c.ref = (int)g.chr[t];
		const int pos = s.p[hit];   // gene_coord (src/hash_align.c:320-334)
		if (pos <= 0) {
			c.coord = 0;
			c.pos = (int)g.start(t, 0);
		} else {
			unsigned int len = 0, i = 0;
			for (; len <= (unsigned int)pos; ++i) {
				if (i >= g.exons(t)) {
					x.err |= E_MAP;
					break;
				}
				len += g.end(t, i) - g.start(t, i) + 1;
			}
			c.coord = i - 1;
			c.pos = (int)(g.end(t, c.coord) - (len - pos) + 1);
		}
	} else {
		unsigned int sum = 0, i;   // chr_coord (src/hash_align.c:307-318)
		for (i = 0; i < g.n_chr; ++i) {
			if (sum + g.chr_len[i] > t)
				break;
			sum += g.chr_len[i];
		}
		c.ref = (int)i;
		c.pos = (int)(t - sum);
	}
	unsigned int match = 0, k = 0;
	for (uint32_t i = 0; i < s.n_cigar; ++i) {
		const unsigned type = s.ops[i] & 15, cnt = s.ops[i] >> 4;
		if (type == B_MATCH) {
			unsigned int n = cnt;
			++i;
			while (i < s.n_cigar && (s.ops[i] & 15) != B_DIFF && (s.ops[i] & 15) != B_DELETE) {
				if ((s.ops[i] & 15) == B_MATCH)
					n += s.ops[i] >> 4;
				++i;
			}
			--i;
			match += n;
			char dig[12];
			int nd = 0;
			do {
				dig[nd++] = (char)('0' + n % 10);
				n /= 10;
			} while (n);
			while (nd)
				md_put(x, c, dig[--nd]);
		} else if (type == B_DIFF) {
			md_put(x, c, miss_at(x, s, k++));
			for (unsigned j = 1; j < cnt; ++j) {
				md_put(x, c, '0');
				md_put(x, c, miss_at(x, s, k++));
			}
		} else if (type == B_DELETE) {
			md_put(x, c, '^');
			for (unsigned j = 0; j < cnt; ++j)
				md_put(x, c, miss_at(x, s, k++));
		}
		// hera continues at strlen(miss): a NUL miss byte cuts the string
		for (unsigned int j = 0; j < c.md_len && j < (unsigned)MAX_MD; ++j)
			if (!c.md[j]) {
				c.md_len = j;
				break;
			}
	}
	unsigned int n = 0, l = (unsigned int)c.pos;
	for (uint32_t i = 0; i < s.n_cigar; ++i) {
		unsigned int run = 0;
		while (i < s.n_cigar && ((s.ops[i] & 15) == B_DIFF || (s.ops[i] & 15) == B_MATCH))
			run += s.ops[i++] >> 4;
		if (run > 0)
			pad(x, c, &n, &l, t, run, B_MATCH, genome);
		if (i < s.n_cigar)
			pad(x, c, &n, &l, t, s.ops[i] >> 4, s.ops[i] & 15, genome);
	}
	c.n_cigar = (int)n;
	c.match = match;
}

// pack_bam_core (src/bam_write.c:265-283) up to the bytes
BAM_HD inline void core(Ctx &x, Core &c, const Cand &r, int p, uint32_t hit)
{
	const unsigned int genome = (unsigned int)r.pair & 1;
	const Strand &s = r.s[p];
	c.bin = c.qual = c.n_cigar = 0;
	c.md_len = c.coord = c.match = c.align_len = 0;
	c.ref = c.pos = -1;
	if (s.n > 0)
		convert(x, c, s, hit, genome);
	c.bin = reg2bin((unsigned int)c.pos, (unsigned int)c.pos + c.match);
	unsigned int n;
	if (genome == 1) {
		n = s.n;
	} else {   // check_quanlity (src/hash_align.c:416-427)
		n = s.n ? 1 : 0;
		for (uint32_t i = 1; i < s.n; ++i)
			if (!overlap_gene(x.g, s.pos[i], s.pos[i - 1]))
				++n;
	}
	if (n >= (unsigned)QUAL_TABLE) {
		x.err |= E_HITS;
		n = 0;
	}
	c.qual = (int)x.qual_table[n];
}

// compact_inf + pack_bam_block (src/bam_write.c:207-240, 285-310): one record
BAM_HD inline void emit(Sink &o, const Core &c, const Core &mate, const Read &rd, unsigned int name_len,
			unsigned int flag, int size, uint32_t n_miss)
{
	const unsigned int tags = c.match > 0 ? 7 + 3 + c.md_len + 1 : 0;
	const unsigned int block = 36 + name_len + 4 * c.n_cigar + (rd.len + 1) / 2 + rd.len + tags + 7;
	o.u32(block - 4);
	o.u32((uint32_t)c.ref);
	o.u32((uint32_t)c.pos);
	o.u32((unsigned int)c.bin << 16 | (unsigned int)(c.qual << 8) | name_len);
	o.u32(flag << 16 | (unsigned int)c.n_cigar);
	o.u32((uint32_t)rd.len);
	o.u32((uint32_t)mate.ref);
	o.u32((uint32_t)mate.pos);
	o.u32((uint32_t)size);
	for (unsigned int j = 0; j < name_len; ++j)
		o.put((uint8_t)rd.name_byte((int)j));
	for (int j = 0; j < c.n_cigar; ++j)   // past MAX_CIG the call fails (E_CIG); the bytes only keep the count
		o.u32(j < MAX_CIG ? c.cig[j] : 0u);
	for (int j = 0; j < rd.len; j += 2) {
		const uint8_t hi = nt16((unsigned char)rd.base(j));
		const uint8_t lo = j + 1 < rd.len ? nt16((unsigned char)rd.base(j + 1)) : 0;
		o.put((uint8_t)(hi << 4 | lo));
	}
	for (int j = 0; j < rd.len; ++j)
		o.put((uint8_t)(rd.q(j) - 33));
	if (c.match > 0) {
		o.put('N'); o.put('M'); o.put('i');
		o.u32(n_miss);
		o.put('M'); o.put('D'); o.put('Z');
		for (unsigned int j = 0; j < c.md_len; ++j)   // likewise past MAX_MD (E_MD)
			o.put(j < (unsigned)MAX_MD ? (uint8_t)c.md[j] : (uint8_t)0);
		o.put(0);
	}
	o.put('A'); o.put('S'); o.put('i');
	o.u32(c.match);
}

// write_alignment_pair (src/bam_write.c:349-380)
BAM_HD inline void write_alignment(Ctx &x, Sink &o, Core *cc, Read &a, Read &b, const unsigned int *flag,
				   const Cand &r, uint32_t hit)
{
	unsigned int name_len = (unsigned int)a.name_l;
	if (name_len > 2 && a.name_byte((int)name_len - 2) == '/') {
		if (a.cut >= 0)
			x.err |= E_NAME;
		a.cut = (int)name_len - 2;
		a.name_l = (int)name_len - 2;
		--name_len;
	} else {
		++name_len;
	}
	core(x, cc[0], r, 0, hit);
	core(x, cc[1], r, 1, hit);
	int size = 0;
	if (cc[0].ref >= 0 && cc[0].ref == cc[1].ref) {
		if (cc[0].pos < cc[1].pos)
			size = (int)((unsigned int)cc[1].pos + (unsigned int)b.len + cc[1].align_len - (unsigned int)cc[0].pos);
		else
			size = (int)((unsigned int)cc[0].pos + (unsigned int)a.len + cc[0].align_len - (unsigned int)cc[1].pos);
	}
	// the mate's record takes name_len bytes of the mate's own name
	emit(o, cc[0], cc[1], a, name_len, flag[0], size, r.s[0].n_miss);
	emit(o, cc[1], cc[0], b, name_len, flag[1], -size, r.s[1].n_miss);
}

// bam_write_pair (src/bam_write.c:382-416)
BAM_HD inline void write_pair(Ctx &x, Sink &o, Core *cc, Read &a, Read &b, const Cand &r, unsigned proper,
			      unsigned first, unsigned rev, unsigned mrev)
{
	unsigned int flag[2];
	flag[0] = make_flag(1, proper, r.s[0].n == 0, r.s[1].n == 0, rev, mrev, 1, 0);
	flag[1] = make_flag(1, proper, r.s[1].n == 0, r.s[0].n == 0, mrev, rev, 0, 1);
	write_alignment(x, o, cc, a, b, flag, r, 0);
	flag[0] |= 1 << 8;
	flag[1] |= 1 << 8;
	if (proper == 0 || r.s[0].n < 2)
		return;
	for (uint32_t i = 1; i < r.s[0].n; ++i) {
		while (i < r.s[0].n && (r.pair & 1) == 0 && overlap_gene(x.g, r.s[0].pos[i], r.s[0].pos[i - 1]))
			++i;
		if (i == r.s[0].n)
			break;
		write_alignment(x, o, cc, a, b, flag, r, i);
	}
}

BAM_HD inline void swap(Cand &a, int pa, Cand &b, int pb)   // swap_candidate (src/hash_align.c:1640-1661)
{
	const Strand t = a.s[pa];
	a.s[pa] = b.s[pb];
	b.s[pb] = t;
}

// The tail's branches (src/hash_align.c:1735-1804) for one pair.
BAM_HD inline void tail(Ctx &x, Sink &o, Core *cc, Cand r0, Cand r1, Read x1, Read x2)
{
	const int s0 = r0.err[0] + r0.err[1], s1 = r1.err[0] + r1.err[1];
	if (s0 < s1)
		r1.pair = -1;
	else if (s0 > s1)
		r0.pair = -1;
	if (r0.pair > 1 && r1.pair > 1) {
		x2.rev = !x2.rev;
		write_pair(x, o, cc, x1, x2, r0, 1, 1, 0, 1);
		x2.rev = !x2.rev;
		x1.rev = !x1.rev;
		write_pair(x, o, cc, x2, x1, r1, 1, 0, 0, 1);
	} else if (r0.pair > 1) {
		x2.rev = !x2.rev;
		write_pair(x, o, cc, x1, x2, r0, 1, 1, 0, 1);
	} else if (r1.pair > 1) {
		x1.rev = !x1.rev;
		write_pair(x, o, cc, x2, x1, r1, 1, 0, 0, 1);
	} else if (r0.s[0].n > 0 && r0.s[1].n > 0 && s0 < s1) {
		x2.rev = !x2.rev;
		write_pair(x, o, cc, x1, x2, r0, 0, 1, 0, 1);
	} else if (r1.s[0].n > 0 && r1.s[1].n > 0) {
		x1.rev = !x1.rev;
		write_pair(x, o, cc, x2, x1, r1, 0, 0, 0, 1);
	} else if (r0.s[0].n > 0 && r1.s[0].n > 0 && (r0.pair & 1) == (r1.pair & 1)) {
		swap(r0, 1, r1, 0);
		r0.pair = -10;
		write_pair(x, o, cc, x1, x2, r0, 0, 1, 0, 0);
	} else if (r0.s[1].n > 0 && r1.s[1].n > 0 && (r0.pair & 1) == (r1.pair & 1)) {
		x1.rev = !x1.rev;
		x2.rev = !x2.rev;
		swap(r0, 0, r1, 1);
		r0.pair = -20;
		write_pair(x, o, cc, x1, x2, r0, 0, 0, 1, 1);
	} else if (r0.s[0].n > 0) {
		write_pair(x, o, cc, x1, x2, r0, 0, 1, 0, 0);
	} else if (r0.s[1].n > 0) {
		x2.rev = !x2.rev;
		write_pair(x, o, cc, x1, x2, r0, 0, 1, 0, 1);
	} else if (r1.s[0].n > 0) {
		write_pair(x, o, cc, x2, x1, r1, 0, 0, 0, 0);
	} else {
		x1.rev = !x1.rev;
		write_pair(x, o, cc, x2, x1, r1, 0, 0, 0, 1);
	}
}

// write_alignment_single (src/bam_write.c:312-347): one record, no mate
BAM_HD inline void write_alignment_single(Ctx &x, Sink &o, Core *cc, Read &a, unsigned int flag, const Cand &r,
					  int p, uint32_t hit)
{
	unsigned int name_len = (unsigned int)a.name_l;
	if (name_len > 2 && a.name_byte((int)name_len - 2) == '/') {
		if (a.cut >= 0)
			x.err |= E_NAME;
		a.cut = (int)name_len - 2;
		a.name_l = (int)name_len - 2;
		--name_len;
	} else {
		++name_len;
	}
	core(x, cc[0], r, p, hit);
	cc[1].ref = cc[1].pos = -1;
	emit(o, cc[0], cc[1], a, name_len, flag, 0, r.s[p].n_miss);
}

// bam_write_single (src/bam_write.c:418-446)
BAM_HD inline void write_single(Ctx &x, Sink &o, Core *cc, Read &a, const Cand &r, unsigned rev, int p)
{
	unsigned int flag = make_flag(0, 0, r.s[p].n == 0, 1, rev, 0, 1, 0);
	write_alignment_single(x, o, cc, a, flag, r, p, 0);
	flag |= 1 << 8;
	if (r.s[p].n < 2)
		return;
	for (uint32_t i = 1; i < r.s[p].n; ++i) {
		while (i < r.s[p].n && overlap_gene(x.g, r.s[p].pos[i], r.s[p].pos[i - 1]))
			++i;
		if (i == r.s[p].n)
			break;
		write_alignment_single(x, o, cc, a, flag, r, p, i);
	}
}

// align_single_read's writes (src/hash_align.c:1825-1834) for one read.
BAM_HD inline void tail_single(Ctx &x, Sink &o, Core *cc, const Cand &r, Read a)
{
	if (r.s[0].n == 0 && r.s[1].n == 0) {
		write_single(x, o, cc, a, r, 0, 0);
		return;
	}
	if (r.s[0].n > 0) {
		write_single(x, o, cc, a, r, 0, 0);
	} else {
		a.rev = !a.rev;
		write_single(x, o, cc, a, r, 1, 1);
	}
}

// Candidate view of a flat record (hera_cand_rec layout).
template <typename Rec>
BAM_HD inline Cand cand(const Rec &rec, const uint32_t *pos, const int32_t *pp, const uint32_t *ops, const char *miss)
{
	Cand c;
	for (int s = 0; s < 2; ++s) {
		c.s[s].n = (uint32_t)rec.n[s];
		c.s[s].pos = pos + rec.list_off[s];
		c.s[s].p = pp + rec.list_off[s];
		c.s[s].n_cigar = rec.n_cigar[s];
		c.s[s].n_miss = rec.n_miss[s];
		c.s[s].ops = ops + rec.cig_off[s];
		c.s[s].miss = miss + rec.miss_off[s];
		c.err[s] = rec.err[s];
	}
	c.pair = rec.pair;
	return c;
}

// get_qual (src/bam_write.c:199-205) for 0..QUAL_TABLE-1 hits, evaluated on
// the host as hera evaluates it (libm's log10, then the conversion to
// unsigned int), so the device only looks the values up.
inline void qual_table_host(uint32_t *t)
{
	for (unsigned int n = 0; n < (unsigned)QUAL_TABLE; ++n) {
		volatile unsigned int nn = n;   // evaluated at run time, as in hera
		double error = 1 - (1.0 / nn);
		if (error == 0)
			error = 0.0000001;
		t[n] = (unsigned int)(-10 * log10(error));
	}
}

BAM_HD inline int name_length(const char *name, int stride)
{
	int l = 0;
	while (l < stride && name[l])
		++l;
	return l;
}

}   // namespace bamw
