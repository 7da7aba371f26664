// Test-only: hera_b200/csrc/hera_bam_core.h -- the BAM record writer the
// device kernels run -- compiled for the host and driven pair by pair the
// way the kernels drive it, so the CPU suite can hold its bytes against the
// reference's before any GPU is involved.  Built by tests/test_bam.py.
#include "../hera_b200/csrc/hera_bam_core.h"

struct Rec {   // hera_cand_rec
	int32_t n[2];
	int32_t err[2];
	int32_t pair;
	uint32_t list_off[2];
	uint32_t cig_off[2];
	uint32_t miss_off[2];
	uint16_t n_cigar[2];
	uint16_t n_miss[2];
};

static bamw::Core cc[2];

extern "C" int bam_host_pairs(uint32_t n_chr, const uint32_t *chr_len, const uint32_t *exon_off,
			      const uint32_t *starts, const uint32_t *ends, const uint32_t *chr, const uint32_t *gene,
			      const Rec *recs, const uint32_t *pos, const int32_t *pp, const uint32_t *ops,
			      const char *miss, int n, const char *seq1, const int64_t *off1, const int32_t *len1,
			      const char *qual1, const char *name1, const char *seq2, const int64_t *off2,
			      const int32_t *len2, const char *qual2, const char *name2, int32_t stride, uint8_t *out,
			      uint64_t *out_off, uint32_t *err)
{
	uint32_t qt[bamw::QUAL_TABLE];
	bamw::qual_table_host(qt);
	bamw::GeneMap g{n_chr, chr_len, exon_off, starts, ends, chr, gene};
	uint64_t at = 0;
	*err = 0;
	for (int i = 0; i < n; ++i) {
		bamw::Ctx x{g, qt, 0};
		bamw::Sink o{out, at};
		bamw::Read a{seq1 + off1[i], qual1 + off1[i], name1 + (int64_t)i * stride, len1[i], false, 0, -1};
		bamw::Read b{seq2 + off2[i], qual2 + off2[i], name2 + (int64_t)i * stride, len2[i], false, 0, -1};
		a.name_l = bamw::name_length(a.name, stride);
		b.name_l = bamw::name_length(b.name, stride);
		out_off[i] = at;
		bamw::tail(x, o, cc, bamw::cand(recs[2 * i], pos, pp, ops, miss),
			   bamw::cand(recs[2 * i + 1], pos, pp, ops, miss), a, b);
		at = o.at;
		*err |= x.err;
	}
	out_off[n] = at;
	return 0;
}

extern "C" int bam_host_single(uint32_t n_chr, const uint32_t *chr_len, const uint32_t *exon_off,
			       const uint32_t *starts, const uint32_t *ends, const uint32_t *chr, const uint32_t *gene,
			       const Rec *recs, const uint32_t *pos, const int32_t *pp, const uint32_t *ops,
			       const char *miss, int n, const char *seq, const int64_t *off, const int32_t *len,
			       const char *qual, const char *name, int32_t stride, uint8_t *out, uint64_t *out_off,
			       uint32_t *err)
{
	uint32_t qt[bamw::QUAL_TABLE];
	bamw::qual_table_host(qt);
	bamw::GeneMap g{n_chr, chr_len, exon_off, starts, ends, chr, gene};
	uint64_t at = 0;
	*err = 0;
	for (int i = 0; i < n; ++i) {
		bamw::Ctx x{g, qt, 0};
		bamw::Sink o{out, at};
		bamw::Read a{seq + off[i], qual + off[i], name + (int64_t)i * stride, len[i], false, 0, -1};
		a.name_l = bamw::name_length(a.name, stride);
		out_off[i] = at;
		bamw::tail_single(x, o, cc, bamw::cand(recs[i], pos, pp, ops, miss), a);
		at = o.at;
		*err |= x.err;
	}
	out_off[n] = at;
	return 0;
}
