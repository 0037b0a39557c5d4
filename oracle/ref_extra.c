/*
 * ref_extra.c -- test infrastructure: the reference's own mp_extra_cal
 * (align.c:148-269, static there) exposed through plain arrays, so that the
 * device version (extra.cu) is checked against the reference itself.  Compiled
 * with the rest of the reference sources by oracle/Makefile (`extra`).
 */
#include "align.c"

int ref_extra_cal(const uint32_t *cigar, int32_t n_cigar, const uint8_t *nt, int32_t l_nt, const char *aa,
		int64_t vs, int64_t ve, int32_t qs, int32_t qe, int32_t has_stop, const int8_t *pssm,
		int32_t go, int32_t ge, int32_t fs, const int8_t *mat, int32_t *stats, mp_feat_t *feats, int32_t feat_cap)
{
	static int tables = 0;
	mp_reg1_t r;
	mp_mapopt_t opt;
	int32_t k;
	if (!tables) ns_make_tables(1), tables = 1;
	memset(&r, 0, sizeof(r));
	memset(&opt, 0, sizeof(opt));
	r.p = (mp_extra_t*)calloc(1, sizeof(mp_extra_t) + sizeof(uint32_t) * (size_t)(n_cigar > 0 ? n_cigar : 1));
	r.p->n_cigar = r.p->m_cigar = n_cigar;
	memcpy(r.p->cigar, cigar, sizeof(uint32_t) * (size_t)n_cigar);
	r.p->dist_stop = has_stop ? 0 : 1;
	r.vs = vs, r.ve = ve, r.qs = qs, r.qe = qe;
	opt.go = go, opt.ge = ge, opt.fs = fs, opt.asize = 22;
	memcpy(opt.mat, mat, 22 * 22);
	/* has_stop in mp_extra_cal is r->qe == qlen && dist_stop == 0 */
	mp_extra_cal(&r, &opt, nt, l_nt, aa, has_stop ? qe : qe + 1, 0, pssm);
	if (!r.p) {
		stats[8] = 0;
		return 1;
	}
	stats[0] = r.p->blen, stats[1] = r.p->n_iden, stats[2] = r.p->n_plus, stats[3] = r.p->n_fs;
	stats[4] = r.p->n_stop, stats[5] = r.p->dp_max, stats[6] = r.n_exon, stats[7] = r.n_feat, stats[8] = 1;
	for (k = 0; k < r.n_feat && k < feat_cap; ++k) feats[k] = r.feat[k];
	free(r.p), free(r.feat);
	return 1;
}
