/*
 * map_learned_hook.c -- libplgpu's learned candidate selector at the reference mapper's
 * candidate selection, as a maintainer would add it to map.c.
 *
 * oracle/Makefile (target progs) copies the reference's map.c, includes this file right
 * before mp_gpu_prefilter_batch (map.c:1014-1089) and makes that function's first
 * statement `if (pl_learned_select(s)) return;`; the result is oracle/_ref/protlocus_learned,
 * test infrastructure for tests/test_gpu_program.py (the product is libplgpu; this is its
 * caller).  With the environment variable PL_PF_MODEL naming a model file -- one text line
 * "hidden tau margin tau_fb n_params" followed by n_params float32, written by the test from
 * protlocus_b200/data/prefilter.npz -- every coarse candidate of the mini-batch goes through
 * pl_pf_select_device: the protein and the genomic window mp_align would align, on the
 * candidate's strand.  The candidates it drops leave the query's set the way
 * mp_select_gapless's do (hit.c:217-263), then the set is sorted and its parents set again
 * as mp_gpu_prefilter_select does (map.c:511-532); the kept ones are aligned by the mapper
 * exactly as before.  Without PL_PF_MODEL the reference's gapless selection runs.
 */
#include <cuda_runtime_api.h>
#include "plgpu.h"

static int pl_pf_state = -1;  /* -1: not loaded yet, 0: off, 1: ready */
static pl_engine_t *pl_pf_eng;
static pl_pf_model_t *pl_pf_m;
static double pl_pf_tau, pl_pf_tau_fb;
static int32_t pl_pf_margin;

static int pl_learned_load(void)
{
	const char *path = getenv("PL_PF_MODEL");
	FILE *f;
	int hidden, margin, ok = 0;
	double tau, tau_fb;
	long long n;
	if (!path || !*path) return 0;
	if ((f = fopen(path, "rb")) == 0) {
		fprintf(stderr, "[E::%s] cannot open %s\n", __func__, path);
		return 0;
	}
	if (fscanf(f, "%d %lf %d %lf %lld", &hidden, &tau, &margin, &tau_fb, &n) == 5 && fgetc(f) == '\n' && n > 0) {
		float *w = (float*)malloc((size_t)n * sizeof(float));
		if (w && fread(w, sizeof(float), (size_t)n, f) == (size_t)n) {
			pl_pf_eng = pl_engine_create(0, 0);
			pl_pf_m = pl_pf_eng ? pl_pf_model_create(0, PL_PF_FDIM, hidden, 0) : 0;
			ok = pl_pf_m && pl_pf_model_set(pl_pf_m, w, n);
		}
		free(w);
	}
	fclose(f);
	if (!ok) fprintf(stderr, "[E::%s] learned selector unavailable: %s\n", __func__, pl_last_error());
	pl_pf_tau = tau, pl_pf_tau_fb = tau_fb, pl_pf_margin = margin;
	return ok;
}

/* the window mp_align aligns a candidate in: its span widened by max_ext, or by
 * max_intron/2 on a side where the protein is not covered to within 10 residues
 * (mp_align_start, align.c:437-452), cut to the contig */
static void pl_learned_window(const mp_mapopt_t *opt, const mp_idx_t *mi, int32_t qlen, const mp_reg1_t *r,
		int64_t *as, int64_t *ae)
{
	const int64_t ctg_len = mi->nt->ctg[r->vid >> 1].len;
	const int32_t extl = r->qs >= 10 ? opt->max_intron / 2 : opt->max_ext;
	const int32_t extr = qlen - r->qe >= 10 ? opt->max_intron / 2 : opt->max_ext;
	*as = r->vs > extl ? r->vs - extl : 0;
	*ae = r->ve + extr < ctg_len ? r->ve + extr : ctg_len;
}

/* the learned selection for a mini-batch; returns 0 when the reference's own selection
 * should run instead (no model) */
static int pl_learned_select(step_t *s)
{
	static int warned = 0;
	const mp_idx_t *mi = s->p->mi;
	const mp_mapopt_t *opt = s->p->opt;
	mp_tbuf_t *b = s->buf[0];
	mp_profile_t *prof = (opt->flag & MP_F_PROFILE) ? &b->profile : 0;
	int64_t n_nt = 0, n_aa = 0, off_nt = 0, off_aa = 0;
	int32_t i, j, n = 0, k = 0, ok = 0;
	pl_splice_job_t *jobs = 0, *tight = 0;
	uint8_t *nt = 0, *aa = 0, *keep = 0, *fb = 0, *d_nt = 0, *d_aa = 0;
	ns_opt_t no;

	if (pl_pf_state < 0) pl_pf_state = pl_learned_load();
	if (!pl_pf_state) return 0;
	for (i = 0; i < s->n_seq; ++i) {  /* the queries mp_gpu_prefilter_batch scores: >1 coarse candidate */
		const mp_coarse_map_t *c = &s->coarse[i];
		if (c->a == 0 || c->n_reg <= 1) continue;
		n_aa += s->seq[i].l_seq;
		for (j = 0; j < c->n_reg; ++j) {
			int64_t as, ae;
			pl_learned_window(opt, mi, s->seq[i].l_seq, &c->reg[j], &as, &ae);
			n_nt += ae - as, ++n;
		}
	}
	if (n == 0) return 1;
	jobs = (pl_splice_job_t*)calloc(n, sizeof(*jobs)), tight = (pl_splice_job_t*)calloc(n, sizeof(*tight));
	nt = (uint8_t*)malloc(n_nt + 16), aa = (uint8_t*)malloc(n_aa + 16);
	keep = (uint8_t*)calloc(n, 1), fb = (uint8_t*)calloc(n, 1);
	if (!jobs || !tight || !nt || !aa || !keep || !fb) goto end;
	for (i = 0; i < s->n_seq; ++i) {
		const mp_coarse_map_t *c = &s->coarse[i];
		const mp_bseq1_t *q = &s->seq[i];
		if (c->a == 0 || c->n_reg <= 1) continue;
		memcpy(aa + off_aa, q->seq, q->l_seq);
		for (j = 0; j < c->n_reg; ++j, ++k) {
			int64_t as, ae;
			pl_learned_window(opt, mi, q->l_seq, &c->reg[j], &as, &ae);
			mp_ntseq_get_by_v(mi->nt, c->reg[j].vid, as, ae, nt + off_nt);  /* 0-3 codes on the candidate's strand */
			jobs[k].nt_off = off_nt, jobs[k].aa_off = off_aa, jobs[k].ss_off = -1;
			jobs[k].nl = (int32_t)(ae - as), jobs[k].al = q->l_seq;
			off_nt += ae - as;
		}
		off_aa += q->l_seq;
	}
	if (cudaMalloc((void**)&d_nt, n_nt + 16) != cudaSuccess || cudaMalloc((void**)&d_aa, n_aa + 16) != cudaSuccess ||
			cudaMemcpy(d_nt, nt, n_nt, cudaMemcpyHostToDevice) != cudaSuccess ||
			cudaMemcpy(d_aa, aa, n_aa, cudaMemcpyHostToDevice) != cudaSuccess)
		goto end;
	ns_opt_init(&no);  /* the residue and codon tables the features read */
	ok = pl_pf_select_device(pl_pf_m, pl_pf_eng, &no, jobs, n, d_nt, d_aa, pl_pf_tau, pl_pf_margin, pl_pf_tau_fb,
			keep, fb, tight, 0, 0);
end:
	if (ok) {
		for (i = 0, k = 0; i < s->n_seq; ++i) {
			mp_coarse_map_t *c = &s->coarse[i];
			int32_t n_before = c->n_reg, m = 0;
			if (c->a == 0 || c->n_reg <= 1) continue;
			for (j = 0; j < c->n_reg; ++j, ++k)
				if (keep[k]) c->reg[m++] = c->reg[j];
			c->n_reg = m;
			mp_sort_reg(b->km, &c->n_reg, c->reg, 0);
			mp_set_parent(b->km, opt->mask_level, opt->mask_len, c->n_reg, c->reg, mi->opt.kmer, 0);
			if (prof) prof->n_prefilter_candidate += n_before, prof->n_prefilter_survivor += c->n_reg;
		}
	} else if (!warned) {  /* every candidate stays, as the reference does when its GPU selection fails */
		warned = 1;
		fprintf(stderr, "[WARNING] learned selector failed (%s); keeping all candidates\n", pl_last_error());
	}
	if (d_nt) cudaFree(d_nt);
	if (d_aa) cudaFree(d_aa);
	free(jobs), free(tight), free(nt), free(aa), free(keep), free(fb);
	return 1;
}
