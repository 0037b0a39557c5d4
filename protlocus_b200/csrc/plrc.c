/*
 * plrc.c -- host layer of the recheck Forward score (the device replacement of
 * recheck.c's rc_score and its kt_for worker, recheck.c:283-440 and :546-568).
 *
 * Profiles are the search profiles recheck.c builds (rc_prof_t's msc / tsc,
 * recheck.c:66-72 and :197-249), uploaded once with pl_rc_profile_create.  A
 * batch scores peptides against their own profiles, one peptide per lane: the
 * peptides of a profile, longest first, go in groups of up to 32 (one warp each),
 * and the groups run longest first.  A group's DP matrices are interleaved by lane
 * in one scratch region (plk_rc_group_floats: with null2 the Forward and Backward
 * M/I rows of every row, 4*(lmax+1)*(M+1) floats per lane, else two rows), and a
 * batch whose groups exceed the engine's budget runs in waves on the stream.  As
 * in recheck.c, the null2 correction is skipped for a pair above 2^25 DP cells
 * (RC_NULL2_MAXCELLS, recheck.c:273).
 */
#define _POSIX_C_SOURCE 200809L
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "plhost.h"

#define RC_NULL2_MAXCELLS 33554432LL

struct pl_rc_profile_s {
	int device;
	plk_rc_prof_t k;
};

PL_EXPORT pl_rc_profile_t *pl_rc_profile_create(int32_t device, int32_t M, const float *msc, const float *tsc)
{
	pl_rc_profile_t *p;
	if (M < 1 || M > PLK_RC_MAX_M || !msc || !tsc) {
		pl_set_error("recheck profile of length %d (1..%d supported)", M, PLK_RC_MAX_M);
		return 0;
	}
	p = (pl_rc_profile_t*)calloc(1, sizeof(*p));
	if (!p) { pl_set_error("out of host memory"); return 0; }
	p->device = device, p->k.M = M;
	CK(cudaSetDevice(device));
	CK(cudaMalloc((void**)&p->k.msc, sizeof(float) * 21 * (size_t)M));
	CK(cudaMalloc((void**)&p->k.tsc, sizeof(float) * 8 * (size_t)M));
	CK(cudaMemcpy((void*)p->k.msc, msc, sizeof(float) * 21 * (size_t)M, cudaMemcpyHostToDevice));
	CK(cudaMemcpy((void*)p->k.tsc, tsc, sizeof(float) * 8 * (size_t)M, cudaMemcpyHostToDevice));
	return p;
fail:
	if (p->k.msc) cudaFree((void*)p->k.msc);
	if (p->k.tsc) cudaFree((void*)p->k.tsc);
	free(p);
	return 0;
}

PL_EXPORT void pl_rc_profile_destroy(pl_rc_profile_t *p)
{
	if (!p) return;
	cudaSetDevice(p->device);
	cudaFree((void*)p->k.msc), cudaFree((void*)p->k.tsc);
	free(p);
}

void pl_rc_engine_free(pl_engine_t *e)
{
	dbuf_free(&e->r_prof), dbuf_free(&e->r_pep), dbuf_free(&e->r_dsq), dbuf_free(&e->r_order);
	dbuf_free(&e->r_grp), dbuf_free(&e->r_err), dbuf_free(&e->r_scratch), dbuf_free(&e->r_bits), dbuf_free(&e->r_bias);
}

/* the limit of the waits between a group's warps (pl_rc_debug_wait_limit), 0: the kernel's default */
static int64_t g_rc_wait_limit = 0;

PL_EXPORT int pl_rc_debug_wait_limit(int64_t cycles)
{
	__atomic_store_n(&g_rc_wait_limit, cycles > 0 ? cycles : 0, __ATOMIC_RELAXED);
	return 1;
}

typedef struct { int64_t key; int32_t idx; } pl_rkey_t;
static int pl_rkey_cmp(const void *a, const void *b)
{
	const pl_rkey_t *x = (const pl_rkey_t*)a, *y = (const pl_rkey_t*)b;
	if (x->key != y->key) return x->key > y->key ? -1 : 1;
	return x->idx - y->idx;
}

/* peptides by profile, longest first within a profile (the lanes of a group then run
 * about as many rows) */
typedef struct { int32_t prof, len, idx; } pl_rpep_t;
static int pl_rpep_cmp(const void *a, const void *b)
{
	const pl_rpep_t *x = (const pl_rpep_t*)a, *y = (const pl_rpep_t*)b;
	if (x->prof != y->prof) return x->prof - y->prof;
	if (x->len != y->len) return y->len - x->len;
	return x->idx - y->idx;
}

PL_EXPORT int pl_rc_score_host(pl_engine_t *e, const pl_rc_profile_t *const *profiles, int32_t n_prof, int32_t n,
		const int32_t *prof_id, const uint8_t *dsq, int64_t dsq_len, const int64_t *off, const int32_t *len,
		int32_t do_null2, float *bits, float *bias)
{
	plk_rc_prof_t *hp = 0;
	plk_rc_pep_t *pep = 0;
	pl_rpep_t *rp = 0;
	pl_rkey_t *gk = 0;
	plk_rc_grp_t *grp = 0, *gs = 0;
	int32_t *order = 0, q, n_grp = 0;
	int64_t budget, cells_total = 0;
	cudaStream_t st;
	int ok = 0;
	if (!e) { pl_set_error("no engine"); return 0; }
	if (n <= 0) return 1;
	st = e->stream;
	CK(cudaSetDevice(e->device));
	hp = (plk_rc_prof_t*)malloc(sizeof(*hp) * (size_t)(n_prof > 0 ? n_prof : 1));
	pep = (plk_rc_pep_t*)calloc((size_t)n, sizeof(*pep));
	rp = (pl_rpep_t*)malloc(sizeof(*rp) * (size_t)n);
	order = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
	grp = (plk_rc_grp_t*)calloc((size_t)n, sizeof(*grp));
	gs = (plk_rc_grp_t*)calloc((size_t)n, sizeof(*gs));
	gk = (pl_rkey_t*)malloc(sizeof(*gk) * (size_t)n);
	if (!hp || !pep || !rp || !order || !grp || !gs || !gk) { pl_set_error("out of host memory"); goto fail; }
	for (q = 0; q < n_prof; ++q) {
		if (!profiles[q] || profiles[q]->device != e->device) { pl_set_error("profile %d missing or on another device", q); goto fail; }
		hp[q] = profiles[q]->k;
	}
	for (q = 0; q < n; ++q) {
		const int32_t pid = prof_id[q], L = len[q];
		int64_t cells;
		if (pid < 0 || pid >= n_prof) { pl_set_error("peptide %d: profile %d of %d", q, pid, n_prof); goto fail; }
		if (L < 1 || off[q] < 0 || off[q] + L > dsq_len) { pl_set_error("peptide %d: length %d at %lld", q, L, (long long)off[q]); goto fail; }
		cells = (int64_t)(L + 1) * (hp[pid].M + 1);
		pep[q].dsq_off = off[q], pep[q].len = L, pep[q].prof = pid;
		pep[q].null2 = do_null2 && cells <= RC_NULL2_MAXCELLS;
		{ /* the length model's logarithms, with the expressions of recheck.c:289-290, :321 and :433-434
		   * evaluated by the host's libm, so the device starts from the bits the reference computes */
			const float pmove = (2.0f + 1.0f) / ((float)L + 2.0f + 1.0f);
			const float p1 = (float)L / (float)(L + 1);
			const float lp1 = logf(p1), l1p1 = logf(1.0f - p1);
			const float l_term = (float)L * lp1;
			pep[q].lmove = logf(pmove), pep[q].lloop = logf(1.0f - pmove);
			pep[q].logL = logf((float)L);
			pep[q].null1 = l_term + l1p1;
		}
		rp[q].prof = pid, rp[q].len = L, rp[q].idx = q;
		cells_total += (int64_t)L * hp[pid].M;
	}
	{ /* residue codes index the 21-column score rows */
		int64_t j;
		for (j = 0; j < dsq_len; ++j)
			if (dsq[j] > 20) { pl_set_error("residue code %d at %lld (0-20 expected)", dsq[j], (long long)j); goto fail; }
	}
	/* groups: up to 32 consecutive peptides of one profile, in the longest-first order */
	qsort(rp, (size_t)n, sizeof(*rp), pl_rpep_cmp);
	for (q = 0; q < n; ++q) order[q] = rp[q].idx;
	for (q = 0; q < n;) {
		plk_rc_grp_t *G = &grp[n_grp];
		int32_t j = q;
		G->first = q, G->prof = rp[q].prof, G->lmax = rp[q].len, G->full = 0;
		while (j < n && j - q < 32 && rp[j].prof == G->prof) G->full |= pep[rp[j].idx].null2, ++j;
		G->count = j - q;
		gk[n_grp].key = (int64_t)G->lmax * hp[G->prof].M, gk[n_grp].idx = n_grp;
		++n_grp, q = j;
	}
	qsort(gk, (size_t)n_grp, sizeof(*gk), pl_rkey_cmp);  /* the longest groups first */
	for (q = 0; q < n_grp; ++q) gs[q] = grp[gk[q].idx];
	if (!dbuf_ensure(&e->r_prof, sizeof(*hp) * (size_t)(n_prof > 0 ? n_prof : 1)) ||
			!dbuf_ensure(&e->r_pep, sizeof(*pep) * (size_t)n) || !dbuf_ensure(&e->r_dsq, (size_t)dsq_len) ||
			!dbuf_ensure(&e->r_order, sizeof(int32_t) * (size_t)n) ||
			!dbuf_ensure(&e->r_grp, sizeof(*gs) * (size_t)n_grp) || !dbuf_ensure(&e->r_err, 64) ||
			!dbuf_ensure(&e->r_bits, sizeof(float) * (size_t)n) || !dbuf_ensure(&e->r_bias, sizeof(float) * (size_t)n))
		goto fail;
	/* waves of groups, each within the scratch budget (the first group of a wave always
	 * goes, so the budget only has to hold the largest group) */
	budget = e->trace_budget;
	{
		int32_t w0 = 0;
		int64_t peak = 0;
		while (w0 < n_grp) {
			int32_t w1 = w0;
			int64_t used = 0;
			while (w1 < n_grp) {
				const int64_t need = plk_rc_group_floats(gs[w1].lmax, hp[gs[w1].prof].M, gs[w1].full);
				if (w1 > w0 && (used + need) * (int64_t)sizeof(float) > budget) break;
				gs[w1].scratch_off = used, used += need;
				++w1;
			}
			if (used > peak) peak = used;
			w0 = w1;
		}
		if (!dbuf_ensure(&e->r_scratch, (size_t)(peak > 0 ? peak : 4) * sizeof(float))) goto fail;
	}
	CK(cudaMemcpyAsync(e->r_prof.p, hp, sizeof(*hp) * (size_t)n_prof, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->r_dsq.p, dsq, (size_t)dsq_len, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->r_pep.p, pep, sizeof(*pep) * (size_t)n, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->r_order.p, order, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->r_grp.p, gs, sizeof(*gs) * (size_t)n_grp, cudaMemcpyHostToDevice, st));
	CK(cudaMemsetAsync(e->r_err.p, 0, sizeof(int), st));
	e->n_ev = 0;
	{
		int32_t w0 = 0;
		while (w0 < n_grp) {
			int32_t w1 = w0 + 1;
			while (w1 < n_grp && gs[w1].scratch_off > 0) ++w1;  /* a wave ends where the offsets restart */
			PL_TIME(e, st, 1);
			CKK(plk_rc_forward((const plk_rc_prof_t*)e->r_prof.p, (const plk_rc_pep_t*)e->r_pep.p,
					(const uint8_t*)e->r_dsq.p, (const int32_t*)e->r_order.p, (const plk_rc_grp_t*)e->r_grp.p + w0,
					w1 - w0, (float*)e->r_scratch.p, (float*)e->r_bits.p, (float*)e->r_bias.p, (int*)e->r_err.p,
					__atomic_load_n(&g_rc_wait_limit, __ATOMIC_RELAXED), st));
			PL_TIME(e, st, 1);
			w0 = w1;  /* waves run in stream order, so the next one may reuse the scratch */
		}
	}
	CK(cudaMemcpyAsync(bits, e->r_bits.p, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, st));
	CK(cudaMemcpyAsync(bias, e->r_bias.p, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, st));
	{
		int derr = 0;
		CK(cudaMemcpyAsync(&derr, e->r_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
		if (derr) { pl_set_error("recheck Forward: a wait between the warps of a group ran out"); goto fail; }
	}
	if (e->timing) {
		int k;
		float ms;
		for (k = 0; k + 1 < e->n_ev; k += 2) {
			cudaEventElapsedTime(&ms, e->ev[k], e->ev[k + 1]);
			e->acc_ms[e->ev_kind[k]] += ms;
		}
		e->acc_dp_launches += e->n_ev / 2, e->acc_cells += cells_total;
	}
	e->r_last_cells = cells_total;
	ok = 1;
fail:
	free(hp), free(pep), free(rp), free(order), free(grp), free(gs), free(gk);
	return ok;
}

PL_EXPORT int64_t pl_rc_last_cells(const pl_engine_t *e) { return e ? e->r_last_cells : 0; }
