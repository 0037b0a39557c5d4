/*
 * plfeat.c -- host side of the batched alignment statistics / exon features
 * (extra.cu): uploads a batch of alignments, runs one warp per alignment and
 * returns the mp_extra_cal results (align.c:148-269) with their features.
 */
#define _POSIX_C_SOURCE 200809L
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "plhost.h"

/* accumulates the recorded kernel events of this call into the engine's timers (phase 1) */
static void pl_feat_times(pl_engine_t *e, int64_t cells)
{
	int k;
	float ms;
	if (!e->timing) return;
	for (k = 0; k + 1 < e->n_ev; k += 2) {
		cudaEventElapsedTime(&ms, e->ev[k], e->ev[k + 1]);
		e->acc_ms[e->ev_kind[k]] += ms;
	}
	e->acc_dp_launches += e->n_ev / 2, e->acc_cells += cells;
}

void pl_feat_engine_free(pl_engine_t *e)
{
	dbuf_free(&e->f_jobs), dbuf_free(&e->f_cig), dbuf_free(&e->f_nt), dbuf_free(&e->f_aa), dbuf_free(&e->f_pssm);
	dbuf_free(&e->f_mat), dbuf_free(&e->f_res), dbuf_free(&e->f_feat);
}

PL_EXPORT int pl_extra_cal_host(pl_engine_t *e, int32_t go, int32_t ge, int32_t fs, int32_t asize, const int8_t *mat,
		const uint8_t *codon, const uint8_t *aa20, const pl_extra_job_t *jobs, int32_t n,
		const uint32_t *cigar, int64_t n_cigar_words, const uint8_t *nt, int64_t l_nt, const uint8_t *aa, int64_t l_aa,
		const int8_t *pssm, int64_t l_pssm, pl_extra_result_t *results, pl_feat_t *feats, int64_t n_feat_slots)
{
	plk_extra_args_t a;
	cudaStream_t st;
	int32_t q;
	if (!e || !mat || !codon || !aa20 || asize <= 0 || asize > 32) { pl_set_error("extra: missing tables"); return 0; }
	if (n <= 0) return 1;
	for (q = 0; q < n; ++q) { /* every read of the device kernel stays inside the given buffers */
		const pl_extra_job_t *J = &jobs[q];
		if (J->n_cigar < 0 || J->cigar_off < 0 || J->cigar_off + J->n_cigar > n_cigar_words || J->nt_off < 0 ||
				J->l_nt < 0 || J->nt_off + J->l_nt > l_nt || J->aa_off < 0 || J->qe < J->qs ||
				J->aa_off + (J->qe - J->qs) > l_aa || J->feat_off < 0 || J->feat_cap < 0 ||
				J->feat_off + J->feat_cap > n_feat_slots ||
				(J->pssm_off >= 0 && (!pssm || J->pssm_off + (int64_t)(J->qe - J->qs) * asize > l_pssm))) {
			pl_set_error("alignment %d: offsets outside the buffers", q);
			return 0;
		}
	}
	CK(cudaSetDevice(e->device));
	st = e->stream;
	if (!dbuf_ensure(&e->f_jobs, sizeof(plk_extra_job_t) * (size_t)n) ||
			!dbuf_ensure(&e->f_cig, sizeof(uint32_t) * (size_t)(n_cigar_words > 0 ? n_cigar_words : 1)) ||
			!dbuf_ensure(&e->f_nt, (size_t)(l_nt > 0 ? l_nt : 1)) || !dbuf_ensure(&e->f_aa, (size_t)(l_aa > 0 ? l_aa : 1)) ||
			!dbuf_ensure(&e->f_pssm, (size_t)(l_pssm > 0 ? l_pssm : 1)) || !dbuf_ensure(&e->f_mat, (size_t)asize * asize) ||
			!dbuf_ensure(&e->f_res, sizeof(plk_extra_res_t) * (size_t)n) ||
			!dbuf_ensure(&e->f_feat, sizeof(plk_feat_t) * (size_t)(n_feat_slots > 0 ? n_feat_slots : 1)))
		goto fail;
	/* the public and kernel records are layout-identical */
	CK(cudaMemcpyAsync(e->f_jobs.p, jobs, sizeof(plk_extra_job_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	if (n_cigar_words > 0) CK(cudaMemcpyAsync(e->f_cig.p, cigar, sizeof(uint32_t) * (size_t)n_cigar_words, cudaMemcpyHostToDevice, st));
	if (l_nt > 0) CK(cudaMemcpyAsync(e->f_nt.p, nt, (size_t)l_nt, cudaMemcpyHostToDevice, st));
	if (l_aa > 0) CK(cudaMemcpyAsync(e->f_aa.p, aa, (size_t)l_aa, cudaMemcpyHostToDevice, st));
	if (pssm && l_pssm > 0) CK(cudaMemcpyAsync(e->f_pssm.p, pssm, (size_t)l_pssm, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->f_mat.p, mat, (size_t)asize * asize, cudaMemcpyHostToDevice, st));
	memset(&a, 0, sizeof(a));
	a.jobs = (const plk_extra_job_t*)e->f_jobs.p, a.n = n, a.cigar = (const uint32_t*)e->f_cig.p;
	a.nt = (const uint8_t*)e->f_nt.p, a.aa = (const uint8_t*)e->f_aa.p, a.pssm = (const int8_t*)e->f_pssm.p;
	a.mat = (const int8_t*)e->f_mat.p, a.go = go, a.ge = ge, a.fs = fs, a.asize = asize;
	memcpy(a.codon, codon, 64), memcpy(a.aa20, aa20, 256);
	a.res = (plk_extra_res_t*)e->f_res.p, a.feat = (plk_feat_t*)e->f_feat.p;
	e->n_ev = 0;
	PL_TIME(e, st, 1);
	CKK(plk_extra(&a, st));
	PL_TIME(e, st, 1);
	CK(cudaMemcpyAsync(results, e->f_res.p, sizeof(plk_extra_res_t) * (size_t)n, cudaMemcpyDeviceToHost, st));
	if (n_feat_slots > 0) CK(cudaMemcpyAsync(feats, e->f_feat.p, sizeof(plk_feat_t) * (size_t)n_feat_slots, cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	{
		int64_t codons = 0;
		for (q = 0; q < n; ++q) codons += jobs[q].qe - jobs[q].qs;
		pl_feat_times(e, codons);
	}
	return 1;
fail:
	return 0;
}

void pl_ps_engine_free(pl_engine_t *e)
{
	dbuf_free(&e->s_jobs), dbuf_free(&e->s_pssm), dbuf_free(&e->s_orf), dbuf_free(&e->s_scr), dbuf_free(&e->s_score);
	dbuf_free(&e->s_order);
}

/* The candidates the band kernel takes (plk_ps_band_ok), longest profile first (a counting
 * sort on the profile length in 16-row buckets) so that the two candidates sharing a warp run
 * about as many rows; key holds n int64 of host scratch and must outlive the upload (the
 * callers free it after their final synchronisation). */
#define PL_PS_BUCKETS 1024
static int pl_ps_band_plan(pl_engine_t *e, const plk_ps_job_t *hj, int32_t n, int32_t go, int32_t ge, int64_t *key,
		cudaStream_t st, plk_ps_args_t *a)
{
	int32_t q, m = 0, *ord = (int32_t*)key, cnt[PL_PS_BUCKETS + 1];
	memset(cnt, 0, sizeof(cnt));
	for (q = 0; q < n; ++q)
		if (plk_ps_band_ok(hj[q].L, hj[q].n, hj[q].band, go, ge)) {
			const int32_t b = hj[q].L >> 4 < PL_PS_BUCKETS - 1 ? hj[q].L >> 4 : PL_PS_BUCKETS - 1;
			++cnt[PL_PS_BUCKETS - 1 - b + 1], ++m;
		}
	a->band_order = 0, a->n_band = m;
	if (m == 0) return 1;
	for (q = 0; q < PL_PS_BUCKETS; ++q) cnt[q + 1] += cnt[q];
	for (q = 0; q < n; ++q)
		if (plk_ps_band_ok(hj[q].L, hj[q].n, hj[q].band, go, ge)) {
			const int32_t b = hj[q].L >> 4 < PL_PS_BUCKETS - 1 ? hj[q].L >> 4 : PL_PS_BUCKETS - 1;
			ord[cnt[PL_PS_BUCKETS - 1 - b]++] = q;
		}
	if (!dbuf_ensure(&e->s_order, sizeof(int32_t) * (size_t)m)) return 0;
	CK(cudaMemcpyAsync(e->s_order.p, ord, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice, st));
	a->band_order = (const int32_t*)e->s_order.p;
	return 1;
fail:
	return 0;
}

/* Cells of one candidate's banded DP: rows i in [0, L) cover ORF positions
 * [max(i + diag - band, 0), min(i + diag + band, n - 1)] (every position when band <= 0),
 * summed in closed form: with x = i + diag the width is linear in x between the two
 * breakpoints x = band and x = n - 1 - band, and positive exactly on [-band, n - 1 + band]. */
PL_EXPORT int64_t pl_ps_band_cells(int32_t L, int32_t n, int32_t diag, int32_t band)
{
	int64_t x0, x1, cut[2], tot = 0;
	int k;
	if (L <= 0 || n <= 0) return 0;
	if (band <= 0) return (int64_t)L * n;
	x0 = diag > -(int64_t)band ? diag : -(int64_t)band;
	x1 = (int64_t)diag + L - 1 < (int64_t)n - 1 + band ? (int64_t)diag + L - 1 : (int64_t)n - 1 + band;
	cut[0] = band < (int64_t)n - 1 - band ? band : (int64_t)n - 1 - band;
	cut[1] = band < (int64_t)n - 1 - band ? (int64_t)n - 1 - band : band;
	for (k = 0; k < 3 && x0 <= x1; ++k) {
		const int64_t s = x0, t = k < 2 && cut[k] < x1 ? cut[k] : x1;
		if (t >= s) {
			/* lo = 0 (x <= band) or x - band; hi = x + band (x <= n - 1 - band) or n - 1 */
			const int64_t la = s <= band ? 0 : 1, lc = s <= band ? 0 : -(int64_t)band;
			const int64_t ha = s <= (int64_t)n - 1 - band ? 1 : 0, hc = s <= (int64_t)n - 1 - band ? band : (int64_t)n - 1;
			const int64_t a = ha - la, c = hc - lc + 1, m = t - s + 1;
			tot += a * (s + t) * m / 2 + c * m;
			x0 = t + 1;
		}
	}
	return tot;
}

PL_EXPORT int pl_ps_gapped_host(pl_engine_t *e, const pl_ps_job_t *jobs, int32_t n, const int8_t *pssm, int64_t l_pssm,
		const uint8_t *orf, int64_t l_orf, int32_t go, int32_t ge, int32_t *scores)
{
	plk_ps_job_t *hj = 0;
	plk_ps_args_t a;
	cudaStream_t st;
	int64_t scr = 0;
	int32_t q;
	int ok = 0;
	if (!e) { pl_set_error("no engine"); return 0; }
	if (n <= 0) return 1;
	hj = (plk_ps_job_t*)malloc((sizeof(*hj) + sizeof(int64_t)) * (size_t)n);  /* the job table, then the band plan's keys */
	if (!hj) { pl_set_error("out of host memory"); return 0; }
	for (q = 0; q < n; ++q) {
		const pl_ps_job_t *J = &jobs[q];
		int64_t k;
		if (J->L < 0 || J->n < 0 || J->pssm_off < 0 || J->orf_off < 0 || J->pssm_off + (int64_t)J->L * 22 > l_pssm ||
				J->orf_off + J->n > l_orf) {
			pl_set_error("candidate %d: profile or ORF outside the buffers", q);
			goto fail;
		}
		for (k = 0; k < J->n; ++k) /* every residue code indexes a 22-wide score row */
			if (orf[J->orf_off + k] > 21) { pl_set_error("candidate %d: residue code %d", q, orf[J->orf_off + k]); goto fail; }
		hj[q].pssm_off = J->pssm_off, hj[q].orf_off = J->orf_off, hj[q].scratch_off = scr;
		hj[q].L = J->L, hj[q].n = J->n, hj[q].diag = J->diag, hj[q].band = J->band;
		scr += (int64_t)J->n + 1;
	}
	CK(cudaSetDevice(e->device));
	st = e->stream;
	if (!dbuf_ensure(&e->s_jobs, sizeof(*hj) * (size_t)n) || !dbuf_ensure(&e->s_pssm, (size_t)(l_pssm > 0 ? l_pssm : 1)) ||
			!dbuf_ensure(&e->s_orf, (size_t)(l_orf > 0 ? l_orf : 1)) ||
			!dbuf_ensure(&e->s_scr, sizeof(int) * 2 * (size_t)(scr > 0 ? scr : 1)) ||
			!dbuf_ensure(&e->s_score, sizeof(int32_t) * (size_t)n))
		goto fail;
	CK(cudaMemcpyAsync(e->s_jobs.p, hj, sizeof(*hj) * (size_t)n, cudaMemcpyHostToDevice, st));
	if (l_pssm > 0) CK(cudaMemcpyAsync(e->s_pssm.p, pssm, (size_t)l_pssm, cudaMemcpyHostToDevice, st));
	if (l_orf > 0) CK(cudaMemcpyAsync(e->s_orf.p, orf, (size_t)l_orf, cudaMemcpyHostToDevice, st));
	memset(&a, 0, sizeof(a));
	a.jobs = (const plk_ps_job_t*)e->s_jobs.p, a.n = n, a.pssm = (const int8_t*)e->s_pssm.p;
	a.orf = (const uint8_t*)e->s_orf.p, a.go = go, a.ge = ge, a.scratch = (int*)e->s_scr.p, a.score = (int32_t*)e->s_score.p;
	if (!pl_ps_band_plan(e, hj, n, go, ge, (int64_t*)(hj + n), st, &a)) goto fail;
	e->n_ev = 0;
	PL_TIME(e, st, 1);
	CKK(plk_ps_gapped(&a, st));
	PL_TIME(e, st, 1);
	CK(cudaMemcpyAsync(scores, e->s_score.p, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	{ /* cells: the banded (or full) rows inside the ORF */
		int64_t cells = 0;
		for (q = 0; q < n; ++q) cells += pl_ps_band_cells(jobs[q].L, jobs[q].n, jobs[q].diag, jobs[q].band);
		pl_feat_times(e, cells);
	}
	ok = 1;
fail:
	free(hj);
	return ok;
}

/* ------------------------------------------------------------------ device-resident variants */

PL_EXPORT int pl_extra_cal_device(pl_engine_t *e, int32_t go, int32_t ge, int32_t fs, int32_t asize, const int8_t *mat,
		const uint8_t *codon, const uint8_t *aa20, const pl_extra_job_t *jobs, int32_t n, const uint32_t *cigar,
		const uint8_t *nt, const uint8_t *aa, const int8_t *pssm, pl_extra_result_t *results, pl_feat_t *feats,
		void *stream)
{
	plk_extra_args_t a;
	cudaStream_t st;
	int32_t q;
	if (!e || !mat || !codon || !aa20 || asize <= 0 || asize > 32) { pl_set_error("extra: missing tables"); return 0; }
	if (n <= 0) return 1;
	for (q = 0; q < n; ++q) {
		const pl_extra_job_t *J = &jobs[q];
		if (J->n_cigar < 0 || J->cigar_off < 0 || J->nt_off < 0 || J->l_nt < 0 || J->aa_off < 0 || J->qe < J->qs ||
				J->feat_off < 0 || J->feat_cap < 0 || (J->pssm_off >= 0 && !pssm)) {
			pl_set_error("alignment %d: negative offsets or sizes", q);
			return 0;
		}
	}
	CK(cudaSetDevice(e->device));
	st = stream ? (cudaStream_t)stream : e->stream;
	if (!dbuf_ensure(&e->f_jobs, sizeof(plk_extra_job_t) * (size_t)n) || !dbuf_ensure(&e->f_mat, (size_t)asize * asize))
		goto fail;
	CK(cudaMemcpyAsync(e->f_jobs.p, jobs, sizeof(plk_extra_job_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->f_mat.p, mat, (size_t)asize * asize, cudaMemcpyHostToDevice, st));
	memset(&a, 0, sizeof(a));
	a.jobs = (const plk_extra_job_t*)e->f_jobs.p, a.n = n, a.cigar = cigar, a.nt = nt, a.aa = aa, a.pssm = pssm;
	a.mat = (const int8_t*)e->f_mat.p, a.go = go, a.ge = ge, a.fs = fs, a.asize = asize;
	memcpy(a.codon, codon, 64), memcpy(a.aa20, aa20, 256);
	a.res = (plk_extra_res_t*)results, a.feat = (plk_feat_t*)feats;
	e->n_ev = 0;
	PL_TIME(e, st, 1);
	CKK(plk_extra(&a, st));
	PL_TIME(e, st, 1);
	CK(cudaStreamSynchronize(st));  /* the job table is reused by the next call */
	{
		int64_t codons = 0;
		for (q = 0; q < n; ++q) codons += jobs[q].qe - jobs[q].qs;
		pl_feat_times(e, codons);
	}
	return 1;
fail:
	return 0;
}

PL_EXPORT int pl_ps_gapped_device(pl_engine_t *e, const pl_ps_job_t *jobs, int32_t n, const int8_t *pssm,
		const uint8_t *orf, int32_t go, int32_t ge, int32_t *scores, void *stream)
{
	plk_ps_job_t *hj = 0;
	plk_ps_args_t a;
	cudaStream_t st;
	int64_t scr = 0, cells = 0;
	int32_t q;
	int ok = 0;
	if (!e) { pl_set_error("no engine"); return 0; }
	if (n <= 0) return 1;
	hj = (plk_ps_job_t*)malloc((sizeof(*hj) + sizeof(int64_t)) * (size_t)n);  /* the job table, then the band plan's keys */
	if (!hj) { pl_set_error("out of host memory"); return 0; }
	for (q = 0; q < n; ++q) {
		const pl_ps_job_t *J = &jobs[q];
		if (J->L < 0 || J->n < 0 || J->pssm_off < 0 || J->orf_off < 0) {
			pl_set_error("candidate %d: negative offsets or sizes", q);
			goto fail;
		}
		hj[q].pssm_off = J->pssm_off, hj[q].orf_off = J->orf_off, hj[q].scratch_off = scr;
		hj[q].L = J->L, hj[q].n = J->n, hj[q].diag = J->diag, hj[q].band = J->band;
		scr += (int64_t)J->n + 1;
		cells += pl_ps_band_cells(J->L, J->n, J->diag, J->band);
	}
	CK(cudaSetDevice(e->device));
	st = stream ? (cudaStream_t)stream : e->stream;
	if (!dbuf_ensure(&e->s_jobs, sizeof(*hj) * (size_t)n) || !dbuf_ensure(&e->s_scr, sizeof(int) * 2 * (size_t)(scr > 0 ? scr : 1)))
		goto fail;
	CK(cudaMemcpyAsync(e->s_jobs.p, hj, sizeof(*hj) * (size_t)n, cudaMemcpyHostToDevice, st));
	memset(&a, 0, sizeof(a));
	a.jobs = (const plk_ps_job_t*)e->s_jobs.p, a.n = n, a.pssm = pssm, a.orf = orf, a.go = go, a.ge = ge;
	a.scratch = (int*)e->s_scr.p, a.score = scores;
	if (!pl_ps_band_plan(e, hj, n, go, ge, (int64_t*)(hj + n), st, &a)) goto fail;
	e->n_ev = 0;
	PL_TIME(e, st, 1);
	CKK(plk_ps_gapped(&a, st));
	PL_TIME(e, st, 1);
	CK(cudaStreamSynchronize(st));  /* the job table and scratch are reused by the next call */
	pl_feat_times(e, cells);
	ok = 1;
fail:
	free(hj);
	return ok;
}
