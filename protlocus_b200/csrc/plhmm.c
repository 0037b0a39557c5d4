/*
 * plhmm.c -- host layer of the integer profile DP (the device replacement of
 * hmm-gpu.c; semantics of mp_hmm_dp_score, hmm.c:252-291).
 *
 * Bulk entry points take the profile as plain tables (pl_hmm_profile_create);
 * the reference's entry points (mppriv.h:128-134) take its opaque mp_hmm_t and
 * read the tables through hmm.c's accessors, caching the device copy in the
 * profile's GPU slot (mp_hmm_gpu_slot) until mp_hmm_gpu_release().  Those
 * accessors and the codon tables live in the host program (hmm.c, nasw-tab.c);
 * they are weak references here, so a caller without them (Python, tests) uses
 * the bulk entry points and the reference entry points report "not taken".
 * No CPU fallback: a failed batch returns 0 with the reason in pl_last_error().
 */
#define _POSIX_C_SOURCE 200809L
#include <limits.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "plhost.h"

struct pl_hmm_profile_s {
	int device;
	plk_hmm_prof_t k;      /* device tables */
	uint8_t *codon_dev;    /* codon index -> HMMER column, 20 = no emission */
	uint8_t codon[64];     /* the same, on the host */
};

PL_EXPORT pl_hmm_profile_t *pl_hmm_profile_create(int32_t device, int32_t m, const int16_t *emit,
		const int16_t *trans, const uint8_t *codon_alpha)
{
	pl_hmm_profile_t *p;
	int16_t *e = 0;
	int32_t *t = 0;
	int32_t mpad, j, k;
	if (m <= 0 || !emit || !trans || !codon_alpha) { pl_set_error("pl_hmm_profile_create: empty profile"); return 0; }
	for (k = 0; k < 64; ++k)
		if (codon_alpha[k] > 20) { pl_set_error("codon_alpha[%d] = %d (HMMER columns 0-19, 20 = none)", k, codon_alpha[k]); return 0; }
	mpad = (m + PLK_HMM_TILE - 1) / PLK_HMM_TILE * PLK_HMM_TILE;
	p = (pl_hmm_profile_t*)calloc(1, sizeof(*p));
	e = (int16_t*)calloc((size_t)21 * mpad, sizeof(int16_t));
	t = (int32_t*)malloc(sizeof(int32_t) * 7 * (size_t)mpad);
	if (!p || !e || !t) { pl_set_error("out of host memory"); goto fail; }
	for (j = 0; j < m; ++j) /* column j holds profile position j (the DP's column j+1) */
		for (k = 0; k < 20; ++k) e[(size_t)k * mpad + j] = emit[(size_t)j * 20 + k];
	for (k = 0; k < 7; ++k)
		for (j = 0; j < mpad; ++j) t[(size_t)k * mpad + j] = j < m ? trans[(size_t)j * 7 + k] : -(1 << 28);
	p->device = device, p->k.m = m, p->k.mpad = mpad;
	memcpy(p->codon, codon_alpha, 64);
	CK(cudaSetDevice(device));
	CK(cudaMalloc((void**)&p->k.emit_t, sizeof(int16_t) * 21 * (size_t)mpad));
	CK(cudaMalloc((void**)&p->k.trans_t, sizeof(int32_t) * 7 * (size_t)mpad));
	CK(cudaMalloc((void**)&p->codon_dev, 64));
	CK(cudaMemcpy((void*)p->k.emit_t, e, sizeof(int16_t) * 21 * (size_t)mpad, cudaMemcpyHostToDevice));
	CK(cudaMemcpy((void*)p->k.trans_t, t, sizeof(int32_t) * 7 * (size_t)mpad, cudaMemcpyHostToDevice));
	CK(cudaMemcpy(p->codon_dev, codon_alpha, 64, cudaMemcpyHostToDevice));
	free(e), free(t);
	return p;
fail:
	free(e), free(t);
	if (p) {
		if (p->k.emit_t) cudaFree((void*)p->k.emit_t);
		if (p->k.trans_t) cudaFree((void*)p->k.trans_t);
		if (p->codon_dev) cudaFree(p->codon_dev);
		free(p);
	}
	return 0;
}

PL_EXPORT void pl_hmm_profile_destroy(pl_hmm_profile_t *p)
{
	if (!p) return;
	cudaSetDevice(p->device);
	cudaFree((void*)p->k.emit_t), cudaFree((void*)p->k.trans_t), cudaFree(p->codon_dev);
	free(p);
}

void pl_hmm_engine_free(pl_engine_t *e)
{
	dbuf_free(&e->h_off), dbuf_free(&e->h_len), dbuf_free(&e->h_rowoff), dbuf_free(&e->h_rows);
	dbuf_free(&e->h_order), dbuf_free(&e->h_counter), dbuf_free(&e->h_edge), dbuf_free(&e->h_nt);
	dbuf_free(&e->h_score);
	{
		int s;
		for (s = 0; s < PL_HMM_STREAMS; ++s) {
			dbuf_free(&e->h_edge_s[s]);
			if (e->h_st[s]) cudaStreamDestroy(e->h_st[s]), e->h_st[s] = 0;
		}
		for (s = 0; s <= PL_HMM_STREAMS; ++s)
			if (e->h_ev[s]) cudaEventDestroy(e->h_ev[s]), e->h_ev[s] = 0;
	}
	free(e->h_hbuf);
	e->h_hbuf = 0, e->h_hcap = 0;
}

/* longest region first; one counting pass over the length (bounded buckets) */
static int pl_hmm_plan(pl_engine_t *e, int32_t n, const int32_t *len, int64_t **row_off, int32_t **order,
		int64_t *rows_total, int32_t *max_rows)
{
	const size_t need = sizeof(int64_t) * (size_t)n + sizeof(int32_t) * (size_t)n + sizeof(int32_t) * 4097;
	int32_t q, *cnt;
	int64_t acc = 0;
	if (need > e->h_hcap) {
		free(e->h_hbuf);
		e->h_hbuf = malloc(need);
		e->h_hcap = e->h_hbuf ? need : 0;
		if (!e->h_hbuf) { pl_set_error("out of host memory"); return 0; }
	}
	*row_off = (int64_t*)e->h_hbuf;
	*order = (int32_t*)(*row_off + n);
	cnt = *order + n;
	memset(cnt, 0, sizeof(int32_t) * 4097);
	*max_rows = 0;
	for (q = 0; q < n; ++q) {
		const int32_t r = len[q] >= 3 ? len[q] / 3 : 0;
		int b;
		if (len[q] < 0) { pl_set_error("region %d: negative length", q); return 0; }
		(*row_off)[q] = acc, acc += (r + 15) / 16 * 16;
		if (r > *max_rows) *max_rows = r;
		b = 4095 - (r >> 4 > 4095 ? 4095 : r >> 4);
		++cnt[b + 1];
	}
	for (q = 0; q < 4096; ++q) cnt[q + 1] += cnt[q];
	for (q = 0; q < n; ++q) {
		const int32_t r = len[q] >= 3 ? len[q] / 3 : 0;
		(*order)[cnt[4095 - (r >> 4 > 4095 ? 4095 : r >> 4)]++] = q;
	}
	*rows_total = acc;
	return 1;
}

static int pl_hmm_run(pl_engine_t *e, const pl_hmm_profile_t *p, int32_t n, const uint8_t *nt_dev,
		const int32_t *off, const int32_t *len, int32_t *score_dev, cudaStream_t st)
{
	int64_t *row_off, rows_total, cells = 0;
	int32_t *order, max_rows, ctas, q;
	if (n <= 0) return 1;
	if (!p) { pl_set_error("no profile"); return 0; }
	if (p->device != e->device) { pl_set_error("profile on device %d, engine on device %d", p->device, e->device); return 0; }
	if (!pl_hmm_plan(e, n, len, &row_off, &order, &rows_total, &max_rows)) return 0;
	for (q = 0; q < n; ++q) cells += (int64_t)(len[q] >= 3 ? len[q] / 3 : 0) * p->k.m;
	ctas = plk_hmm_ctas_per_sm(p->k.mpad);
	if (ctas < 1) { pl_set_error("HMM DP kernel does not fit on an SM"); return 0; }
	ctas *= e->n_sm;
	if ((int64_t)ctas * plk_hmm_warps_per_cta() > n) ctas = (n + plk_hmm_warps_per_cta() - 1) / plk_hmm_warps_per_cta();
	if (!dbuf_ensure(&e->h_off, sizeof(int32_t) * (size_t)n) || !dbuf_ensure(&e->h_len, sizeof(int32_t) * (size_t)n) ||
			!dbuf_ensure(&e->h_rowoff, sizeof(int64_t) * (size_t)n) || !dbuf_ensure(&e->h_order, sizeof(int32_t) * (size_t)n) ||
			!dbuf_ensure(&e->h_rows, (size_t)(rows_total > 0 ? rows_total : 16)) || !dbuf_ensure(&e->h_counter, 64) ||
			!dbuf_ensure(&e->h_edge, (size_t)16 * 2 * (size_t)(max_rows + 1) * (size_t)ctas * plk_hmm_warps_per_cta()))
		return 0;
	CK(cudaMemcpyAsync(e->h_off.p, off, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->h_len.p, len, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->h_rowoff.p, row_off, sizeof(int64_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->h_order.p, order, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	e->n_ev = 0;
	PL_TIME(e, st, 0);
	CKK(plk_hmm_codons(nt_dev, (const int32_t*)e->h_off.p, (const int32_t*)e->h_len.p, (const int64_t*)e->h_rowoff.p, n,
			p->codon_dev, (uint8_t*)e->h_rows.p, st));
	PL_TIME(e, st, 0);
	PL_TIME(e, st, 1);
	CKK(plk_hmm_dp(&p->k, (const uint8_t*)e->h_rows.p, (const int64_t*)e->h_rowoff.p, (const int32_t*)e->h_len.p,
			(const int32_t*)e->h_order.p, n, (int32_t*)e->h_counter.p, e->h_edge.p, (int64_t)max_rows + 1, ctas,
			score_dev, st));
	PL_TIME(e, st, 1);
	CK(cudaStreamSynchronize(st));
	if (e->timing) {
		int k;
		float ms;
		for (k = 0; k + 1 < e->n_ev; k += 2) {
			cudaEventElapsedTime(&ms, e->ev[k], e->ev[k + 1]);
			e->acc_ms[e->ev_kind[k]] += ms;
		}
		e->acc_dp_launches += 1, e->acc_cells += cells;
	}
	e->h_last_cells = cells;
	return 1;
fail:
	return 0;
}

PL_EXPORT int pl_hmm_score_device(pl_engine_t *e, const pl_hmm_profile_t *p, int32_t n, const uint8_t *nt,
		const int32_t *off, const int32_t *len, int32_t *score_dev, void *stream)
{
	if (!e) { pl_set_error("no engine"); return 0; }
	if (cudaSetDevice(e->device) != cudaSuccess) { pl_set_error("cudaSetDevice failed"); return 0; }
	return pl_hmm_run(e, p, n, nt, off, len, score_dev, stream ? (cudaStream_t)stream : e->stream);
}

/* Many profiles against one region set: the planning, the upload of the region tables and
 * the codon translation once (again only when a profile's codon table differs from the
 * previous one's), then one DP launch per profile, round-robin on PL_HMM_STREAMS streams
 * with their own queue counters and edge buffers, so that the launches of a region set too
 * small to fill the GPU run side by side. */
PL_EXPORT int pl_hmm_score_many_device(pl_engine_t *e, const pl_hmm_profile_t *const *ps, int32_t n_prof, int32_t n,
		const uint8_t *nt, const int32_t *off, const int32_t *len, int32_t *score_dev, void *stream)
{
	int64_t *row_off, rows_total, cells = 0, rows_sum = 0;
	int32_t *order, max_rows, q, k, s, warps;
	const uint8_t *codon = 0;
	cudaStream_t st;
	if (!e) { pl_set_error("no engine"); return 0; }
	if (n <= 0 || n_prof <= 0) return 1;
	if (!ps || !off || !len || !nt || !score_dev) { pl_set_error("pl_hmm_score_many_device: missing argument"); return 0; }
	for (k = 0; k < n_prof; ++k)
		if (!ps[k] || ps[k]->device != e->device) { pl_set_error("profile %d missing or on another device", k); return 0; }
	CK(cudaSetDevice(e->device));
	st = stream ? (cudaStream_t)stream : e->stream;
	if (!pl_hmm_plan(e, n, len, &row_off, &order, &rows_total, &max_rows)) return 0;
	for (q = 0; q < n; ++q) rows_sum += len[q] >= 3 ? len[q] / 3 : 0;
	warps = plk_hmm_warps_per_cta();
	for (s = 0; s < PL_HMM_STREAMS; ++s)
		if (!e->h_st[s]) CK(cudaStreamCreateWithFlags(&e->h_st[s], cudaStreamNonBlocking));
	for (s = 0; s <= PL_HMM_STREAMS; ++s)
		if (!e->h_ev[s]) CK(cudaEventCreateWithFlags(&e->h_ev[s], cudaEventDisableTiming));
	if (!dbuf_ensure(&e->h_off, sizeof(int32_t) * (size_t)n) || !dbuf_ensure(&e->h_len, sizeof(int32_t) * (size_t)n) ||
			!dbuf_ensure(&e->h_rowoff, sizeof(int64_t) * (size_t)n) || !dbuf_ensure(&e->h_order, sizeof(int32_t) * (size_t)n) ||
			!dbuf_ensure(&e->h_rows, (size_t)(rows_total > 0 ? rows_total : 16)) ||
			!dbuf_ensure(&e->h_counter, 64 * PL_HMM_STREAMS))
		return 0;
	CK(cudaMemcpyAsync(e->h_off.p, off, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->h_len.p, len, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->h_rowoff.p, row_off, sizeof(int64_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->h_order.p, order, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	e->n_ev = 0;
	PL_TIME(e, st, 1);
	for (k = 0; k < n_prof; ++k) {
		const pl_hmm_profile_t *p = ps[k];
		int32_t ctas = plk_hmm_ctas_per_sm(p->k.mpad);
		cudaStream_t sk;
		if (ctas < 1) { pl_set_error("HMM DP kernel does not fit on an SM"); return 0; }
		ctas *= e->n_sm;
		if ((int64_t)ctas * warps > n) ctas = (n + warps - 1) / warps;
		if (!codon || memcmp(codon, p->codon, 64) != 0) {  /* the rows of this codon table, then fork again */
			if (codon) {  /* every launch reading the previous rows has finished */
				for (s = 0; s < PL_HMM_STREAMS; ++s) {
					CK(cudaEventRecord(e->h_ev[s], e->h_st[s]));
					CK(cudaStreamWaitEvent(st, e->h_ev[s], 0));
				}
			}
			CKK(plk_hmm_codons(nt, (const int32_t*)e->h_off.p, (const int32_t*)e->h_len.p, (const int64_t*)e->h_rowoff.p,
					n, p->codon_dev, (uint8_t*)e->h_rows.p, st));
			CK(cudaEventRecord(e->h_ev[PL_HMM_STREAMS], st));
			for (s = 0; s < PL_HMM_STREAMS; ++s) CK(cudaStreamWaitEvent(e->h_st[s], e->h_ev[PL_HMM_STREAMS], 0));
			codon = p->codon;
		}
		s = k % PL_HMM_STREAMS, sk = e->h_st[s];
		if (!dbuf_ensure(&e->h_edge_s[s], (size_t)16 * 2 * (size_t)(max_rows + 1) * (size_t)ctas * warps)) return 0;
		CKK(plk_hmm_dp(&p->k, (const uint8_t*)e->h_rows.p, (const int64_t*)e->h_rowoff.p, (const int32_t*)e->h_len.p,
				(const int32_t*)e->h_order.p, n, (int32_t*)e->h_counter.p + 16 * s, e->h_edge_s[s].p,
				(int64_t)max_rows + 1, ctas, score_dev + (int64_t)k * n, sk));
		cells += rows_sum * p->k.m;
	}
	for (s = 0; s < PL_HMM_STREAMS; ++s) {  /* join */
		CK(cudaEventRecord(e->h_ev[s], e->h_st[s]));
		CK(cudaStreamWaitEvent(st, e->h_ev[s], 0));
	}
	PL_TIME(e, st, 1);
	CK(cudaStreamSynchronize(st));
	if (e->timing) {
		float ms;
		if (e->n_ev >= 2 && cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]) == cudaSuccess) e->acc_ms[1] += ms;
		e->acc_dp_launches += n_prof, e->acc_cells += cells;
	}
	e->h_last_cells = cells;
	return 1;
fail:
	return 0;
}

/* pl_hmm_score_many_device from host buffers: the region set uploaded once, the
 * n_prof x n scores copied back. */
PL_EXPORT int pl_hmm_score_many_host(pl_engine_t *e, const pl_hmm_profile_t *const *ps, int32_t n_prof, int32_t n,
		const uint8_t *nt, int64_t l_nt, const int32_t *off, const int32_t *len, int32_t *score)
{
	cudaStream_t st;
	int32_t q;
	if (!e) { pl_set_error("no engine"); return 0; }
	if (n <= 0 || n_prof <= 0) return 1;
	for (q = 0; q < n; ++q)
		if (off[q] < 0 || len[q] < 0 || (int64_t)off[q] + len[q] > l_nt) {
			pl_set_error("region %d [%d, +%d) outside the %lld-byte buffer", q, off[q], len[q], (long long)l_nt);
			return 0;
		}
	st = e->stream;
	CK(cudaSetDevice(e->device));
	if (!dbuf_ensure(&e->h_nt, (size_t)(l_nt > 0 ? l_nt : 1)) ||
			!dbuf_ensure(&e->h_score, sizeof(int32_t) * (size_t)n * (size_t)n_prof))
		return 0;
	if (l_nt > 0) CK(cudaMemcpyAsync(e->h_nt.p, nt, (size_t)l_nt, cudaMemcpyHostToDevice, st));
	if (!pl_hmm_score_many_device(e, ps, n_prof, n, (const uint8_t*)e->h_nt.p, off, len, (int32_t*)e->h_score.p, st))
		return 0;
	CK(cudaMemcpyAsync(score, e->h_score.p, sizeof(int32_t) * (size_t)n * (size_t)n_prof, cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	return 1;
fail:
	return 0;
}

PL_EXPORT int pl_hmm_score_host(pl_engine_t *e, const pl_hmm_profile_t *p, int32_t n, const uint8_t *nt,
		int64_t l_nt, const int32_t *off, const int32_t *len, int32_t *score)
{
	cudaStream_t st;
	int32_t q;
	if (!e) { pl_set_error("no engine"); return 0; }
	if (n <= 0) return 1;
	for (q = 0; q < n; ++q)
		if (off[q] < 0 || len[q] < 0 || (int64_t)off[q] + len[q] > l_nt) {
			pl_set_error("region %d [%d, +%d) outside the %lld-byte buffer", q, off[q], len[q], (long long)l_nt);
			return 0;
		}
	st = e->stream;
	CK(cudaSetDevice(e->device));
	if (!dbuf_ensure(&e->h_nt, (size_t)(l_nt > 0 ? l_nt : 1)) || !dbuf_ensure(&e->h_score, sizeof(int32_t) * (size_t)n)) return 0;
	if (l_nt > 0) CK(cudaMemcpyAsync(e->h_nt.p, nt, (size_t)l_nt, cudaMemcpyHostToDevice, st));
	if (!pl_hmm_run(e, p, n, (const uint8_t*)e->h_nt.p, off, len, (int32_t*)e->h_score.p, st)) return 0;
	CK(cudaMemcpyAsync(score, e->h_score.p, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	return 1;
fail:
	return 0;
}

PL_EXPORT int64_t pl_hmm_last_cells(const pl_engine_t *e) { return e ? e->h_last_cells : 0; }

/* ------------------------------------------------------------------ reference entry points (mppriv.h:128-134) */

typedef struct mp_hmm_s mp_hmm_t;
/* provided by the host program's hmm.c and nasw-tab.c */
extern int32_t mp_hmm_length(const mp_hmm_t *h) __attribute__((weak));
extern const int16_t *mp_hmm_emissions(const mp_hmm_t *h) __attribute__((weak));
extern const int16_t *mp_hmm_transitions(const mp_hmm_t *h) __attribute__((weak));
extern void **mp_hmm_gpu_slot(const mp_hmm_t *h, int which) __attribute__((weak));
extern const int8_t *mp_hmm_aa20_to_alpha_table(void) __attribute__((weak));
extern uint8_t ns_tab_codon[64] __attribute__((weak));

static pthread_mutex_t hm_mu = PTHREAD_MUTEX_INITIALIZER;
static pl_engine_t *hm_engine;
static int hm_ready = -1;

static int hm_init(void)
{ /* called with hm_mu held */
	const char *env = getenv("PLGPU_DEVICE");
	int count = 0, dev = env ? atoi(env) : 0;
	if (hm_ready >= 0) return hm_ready;
	hm_ready = 0;
	if (!mp_hmm_length || !mp_hmm_emissions || !mp_hmm_transitions || !mp_hmm_gpu_slot ||
			!mp_hmm_aa20_to_alpha_table || !ns_tab_codon) {
		pl_set_error("the host program provides no hmm.c accessors: use pl_hmm_profile_create");
		return 0;
	}
	if (cudaGetDeviceCount(&count) != cudaSuccess || dev < 0 || dev >= count) { cudaGetLastError(); return 0; }
	hm_engine = pl_engine_create(dev, 0);
	hm_ready = hm_engine != 0;
	return hm_ready;
}

/* the device copy of h's tables, built once and kept in h's GPU slot 0 (called with hm_mu held) */
static pl_hmm_profile_t *hm_profile(const mp_hmm_t *h)
{
	void **slot = mp_hmm_gpu_slot(h, 0);
	uint8_t codon[64];
	const int8_t *alpha;
	int k;
	if (!slot) return 0;
	if (*slot) return (pl_hmm_profile_t*)*slot;
	alpha = mp_hmm_aa20_to_alpha_table();
	for (k = 0; k < 64; ++k) { /* hmm.c:269-270 */
		const int a = ns_tab_codon[k];
		codon[k] = a < 20 && alpha[a] >= 0 ? (uint8_t)alpha[a] : 20;
	}
	*slot = pl_hmm_profile_create(hm_engine->device, mp_hmm_length(h), mp_hmm_emissions(h), mp_hmm_transitions(h), codon);
	return (pl_hmm_profile_t*)*slot;
}

/* mppriv.h:132 -- 1 = every score filled, exactly mp_hmm_dp_score() of each region. */
PL_EXPORT int mp_hmm_dp_score_gpu_batch(const mp_hmm_t *h, int32_t n, const uint8_t *nt, int64_t l_nt,
		const int32_t *off, const int32_t *len, int32_t *score)
{
	pl_hmm_profile_t *p;
	int ok = 0;
	if (!h || n <= 0 || !nt || !off || !len || !score) return 0;
	pthread_mutex_lock(&hm_mu);
	if (hm_init() && mp_hmm_length(h) > 0 && (p = hm_profile(h)) != 0)
		ok = pl_hmm_score_host(hm_engine, p, n, nt, l_nt, off, len, score);
	pthread_mutex_unlock(&hm_mu);
	return ok;
}

/* mppriv.h:129 -- INT32_MIN when not taken (the caller then runs the CPU). */
PL_EXPORT int32_t mp_hmm_dp_score_gpu(const mp_hmm_t *h, const uint8_t *nt, int32_t nlen)
{
	int32_t off = 0, score = INT32_MIN;
	if (nlen < 3) return INT32_MIN;
	return mp_hmm_dp_score_gpu_batch(h, 1, nt, nlen, &off, &nlen, &score) ? score : INT32_MIN;
}

/* mppriv.h:134 -- drop the cached device tables (called from mp_hmm_destroy, hmm.c:207-212). */
PL_EXPORT void mp_hmm_gpu_release(mp_hmm_t *h)
{
	void **slot;
	if (!h || !mp_hmm_gpu_slot) return;
	slot = mp_hmm_gpu_slot(h, 0);
	if (!slot || !*slot) return;
	pthread_mutex_lock(&hm_mu);
	pl_hmm_profile_destroy((pl_hmm_profile_t*)*slot);
	*slot = 0;
	pthread_mutex_unlock(&hm_mu);
}
