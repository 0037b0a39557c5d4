/*
 * plgroup.c -- one batch of global spliced DPs sharded over several GPUs.
 *
 * Every DP job is independent (nasw-cuda.cu runs one job per block, :935-943),
 * so a caller's job table splits over devices with no exchange inside a DP: the
 * planner assigns jobs to devices by decreasing DP cells, each job to the device
 * with the fewest cells so far (longest-processing-time order, so the length
 * bins spread round-robin and the loads even out); one host thread per device
 * packs its jobs' sequences, runs pl_splice_batch_host on that device's engine
 * and keeps its results; the gather then writes results and CIGARs back in the
 * caller's job order, CIGARs dense, exactly as one engine would have.
 *
 * The planner (pl_group_plan) and the gather (pl_group_gather) are plain host
 * functions: they are exported so that the partition and the reassembly can be
 * tested without a device.
 */
#define _POSIX_C_SOURCE 200809L
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "plhost.h"

#define PL_GROUP_MAX 64

struct pl_group_s {
	int32_t n_dev;
	pl_engine_t *eng[PL_GROUP_MAX];
};

typedef struct { int64_t cells; int32_t q; } pl_gkey_t;

static int pl_gkey_cmp(const void *a, const void *b)
{ /* decreasing cells, then increasing job index */
	const pl_gkey_t *x = (const pl_gkey_t*)a, *y = (const pl_gkey_t*)b;
	if (x->cells != y->cells) return x->cells > y->cells ? -1 : 1;
	return x->q - y->q;
}

PL_EXPORT int pl_group_plan(const pl_splice_job_t *jobs, int32_t n, int32_t n_dev, int32_t *dev_of_job,
		int64_t *cells_of_dev)
{
	pl_gkey_t *key;
	int64_t load[PL_GROUP_MAX];
	int32_t q, d;
	if (n < 0 || n_dev < 1 || n_dev > PL_GROUP_MAX || (n > 0 && (!jobs || !dev_of_job))) {
		pl_set_error("group plan: %d jobs over %d devices (1..%d)", n, n_dev, PL_GROUP_MAX);
		return 0;
	}
	memset(load, 0, sizeof(load));
	key = (pl_gkey_t*)malloc(sizeof(*key) * (size_t)(n > 0 ? n : 1));
	if (!key) { pl_set_error("out of host memory"); return 0; }
	for (q = 0; q < n; ++q)
		key[q].cells = (int64_t)(jobs[q].nl > 2 ? jobs[q].nl - 2 : 1) * (jobs[q].al > 0 ? jobs[q].al : 1), key[q].q = q;
	qsort(key, (size_t)n, sizeof(*key), pl_gkey_cmp);
	for (q = 0; q < n; ++q) {
		int32_t best = 0;
		for (d = 1; d < n_dev; ++d) if (load[d] < load[best]) best = d;
		dev_of_job[key[q].q] = best;
		load[best] += key[q].cells;
	}
	if (cells_of_dev) for (d = 0; d < n_dev; ++d) cells_of_dev[d] = load[d];
	free(key);
	return 1;
}

PL_EXPORT int pl_group_gather(int32_t n, const int32_t *dev_of_job, int32_t n_dev,
		const pl_splice_result_t *const *dev_results, const uint32_t *const *dev_cigar,
		pl_splice_result_t *results, uint32_t *cigar, int64_t cigar_cap, int64_t *total_cigar)
{
	int32_t pos[PL_GROUP_MAX], q;
	int64_t off = 0;
	if (n < 0 || n_dev < 1 || n_dev > PL_GROUP_MAX) { pl_set_error("group gather: bad sizes"); return 0; }
	memset(pos, 0, sizeof(pos));
	for (q = 0; q < n; ++q) {
		const int32_t d = dev_of_job[q];
		const pl_splice_result_t *r;
		if (d < 0 || d >= n_dev) { pl_set_error("group gather: job %d on device slot %d", q, d); return 0; }
		r = &dev_results[d][pos[d]++];  /* a device's results are in the order of its jobs */
		results[q] = *r;
		if (r->status != 0 || r->n_cigar < 0) { results[q].n_cigar = 0, results[q].cigar_off = off; continue; }
		results[q].cigar_off = off;
		if (off + r->n_cigar > cigar_cap) {  /* the caller's buffer is full: as one engine reports it */
			results[q].status = -2;
		} else if (r->n_cigar > 0) {
			memcpy(cigar + off, dev_cigar[d] + r->cigar_off, sizeof(uint32_t) * (size_t)r->n_cigar);
		}
		off += r->n_cigar;
	}
	if (total_cigar) *total_cigar = off;
	return 1;
}

PL_EXPORT pl_group_t *pl_group_create(const int32_t *devices, int32_t n_dev, int64_t trace_budget_bytes)
{
	pl_group_t *g;
	int32_t d;
	if (!devices || n_dev < 1 || n_dev > PL_GROUP_MAX) { pl_set_error("group of %d devices (1..%d)", n_dev, PL_GROUP_MAX); return 0; }
	g = (pl_group_t*)calloc(1, sizeof(*g));
	if (!g) { pl_set_error("out of host memory"); return 0; }
	g->n_dev = n_dev;
	for (d = 0; d < n_dev; ++d) {
		g->eng[d] = pl_engine_create(devices[d], trace_budget_bytes);
		if (!g->eng[d]) { pl_group_destroy(g); return 0; }
	}
	return g;
}

PL_EXPORT void pl_group_destroy(pl_group_t *g)
{
	int32_t d;
	if (!g) return;
	for (d = 0; d < g->n_dev; ++d) pl_engine_destroy(g->eng[d]);
	free(g);
}

PL_EXPORT pl_engine_t *pl_group_engine(pl_group_t *g, int32_t slot)
{
	return g && slot >= 0 && slot < g->n_dev ? g->eng[slot] : 0;
}

typedef struct {
	pl_engine_t *e;
	const ns_opt_t *opt;
	const pl_splice_job_t *jobs;    /* caller's table */
	const int32_t *dev_of_job;
	int32_t n, slot, n_mine;
	const uint8_t *nt, *aa, *ss;
	pl_splice_result_t *res;        /* n_mine results, in the order of the slot's jobs */
	uint32_t *cig;
	int ok;
	char err[512];
} pl_gwork_t;

static void *pl_group_worker(void *arg)
{
	pl_gwork_t *w = (pl_gwork_t*)arg;
	pl_splice_job_t *sub = 0;
	uint8_t *nt = 0, *aa = 0, *ss = 0;
	int64_t l_nt = 0, l_aa = 0, l_ss = 0, cap = 0, p_nt = 0, p_aa = 0, p_ss = 0;
	int32_t q, k = 0;
	w->ok = 0;
	for (q = 0; q < w->n; ++q) {
		if (w->dev_of_job[q] != w->slot) continue;
		l_nt += w->jobs[q].nl, l_aa += w->jobs[q].al, cap += (int64_t)w->jobs[q].nl + w->jobs[q].al + 8;
		if (w->ss && w->jobs[q].ss_off >= 0) l_ss += w->jobs[q].nl;
	}
	if (w->n_mine == 0) { w->ok = 1; return 0; }
	sub = (pl_splice_job_t*)malloc(sizeof(*sub) * (size_t)w->n_mine);
	nt = (uint8_t*)malloc((size_t)l_nt + 1), aa = (uint8_t*)malloc((size_t)l_aa + 1);
	ss = l_ss ? (uint8_t*)malloc((size_t)l_ss) : 0;
	w->cig = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)cap);
	if (!sub || !nt || !aa || (l_ss && !ss) || !w->cig) { snprintf(w->err, sizeof(w->err), "out of host memory"); goto out; }
	for (q = 0; q < w->n; ++q) { /* this device's jobs, their spans packed back to back */
		const pl_splice_job_t *x = &w->jobs[q];
		if (w->dev_of_job[q] != w->slot) continue;
		sub[k] = *x;
		memcpy(nt + p_nt, w->nt + x->nt_off, (size_t)x->nl), sub[k].nt_off = p_nt, p_nt += x->nl;
		memcpy(aa + p_aa, w->aa + x->aa_off, (size_t)x->al), sub[k].aa_off = p_aa, p_aa += x->al;
		if (w->ss && x->ss_off >= 0) memcpy(ss + p_ss, w->ss + x->ss_off, (size_t)x->nl), sub[k].ss_off = p_ss, p_ss += x->nl;
		else sub[k].ss_off = -1;
		++k;
	}
	if (!pl_splice_batch_host(w->e, w->opt, sub, w->n_mine, nt, l_nt, aa, l_aa, ss, l_ss, w->res, w->cig, cap)) {
		snprintf(w->err, sizeof(w->err), "%s", pl_last_error());
		goto out;
	}
	w->ok = 1;
out:
	free(sub), free(nt), free(aa), free(ss);
	return 0;
}

PL_EXPORT int pl_group_splice_host(pl_group_t *g, const ns_opt_t *opt, const pl_splice_job_t *jobs, int32_t n,
		const uint8_t *nt, int64_t nt_len, const uint8_t *aa, int64_t aa_len, const uint8_t *ss, int64_t ss_len,
		pl_splice_result_t *results, uint32_t *cigar, int64_t cigar_cap, int64_t *total_cigar)
{
	pl_gwork_t w[PL_GROUP_MAX];
	pthread_t th[PL_GROUP_MAX];
	const pl_splice_result_t *dres[PL_GROUP_MAX];
	const uint32_t *dcig[PL_GROUP_MAX];
	int32_t *dev_of_job = 0, q, d;
	int ok = 0, started[PL_GROUP_MAX];
	if (!g) { pl_set_error("no group"); return 0; }
	if (n < 0 || (n > 0 && (!jobs || !nt || !aa || !results))) { pl_set_error("invalid batch arguments"); return 0; }
	if (n == 0) { if (total_cigar) *total_cigar = 0; return 1; }
	for (q = 0; q < n; ++q) /* spans inside the caller's buffers before any thread packs them */
		if (!pl_span_ok("job", q, "nt", jobs[q].nt_off, jobs[q].nl, nt_len) ||
				!pl_span_ok("job", q, "aa", jobs[q].aa_off, jobs[q].al, aa_len) ||
				(ss && jobs[q].ss_off >= 0 && !pl_span_ok("job", q, "ss", jobs[q].ss_off, jobs[q].nl, ss_len)))
			return 0;
	memset(w, 0, sizeof(w));
	memset(started, 0, sizeof(started));
	dev_of_job = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
	if (!dev_of_job) { pl_set_error("out of host memory"); return 0; }
	if (!pl_group_plan(jobs, n, g->n_dev, dev_of_job, 0)) goto out;
	for (d = 0; d < g->n_dev; ++d) {
		w[d].e = g->eng[d], w[d].opt = opt, w[d].jobs = jobs, w[d].dev_of_job = dev_of_job, w[d].n = n, w[d].slot = d;
		w[d].nt = nt, w[d].aa = aa, w[d].ss = ss;
		for (q = 0; q < n; ++q) w[d].n_mine += dev_of_job[q] == d;
		w[d].res = (pl_splice_result_t*)malloc(sizeof(pl_splice_result_t) * (size_t)(w[d].n_mine > 0 ? w[d].n_mine : 1));
		if (!w[d].res) { pl_set_error("out of host memory"); goto out; }
	}
	for (d = 0; d < g->n_dev; ++d) { /* one host thread per device */
		if (pthread_create(&th[d], 0, pl_group_worker, &w[d]) != 0) { pl_set_error("thread creation failed"); break; }
		started[d] = 1;
	}
	for (d = 0; d < g->n_dev; ++d) if (started[d]) pthread_join(th[d], 0);
	for (d = 0; d < g->n_dev; ++d) {
		if (!started[d]) goto out;
		if (!w[d].ok) { pl_set_error("device slot %d: %s", d, w[d].err); goto out; }
		dres[d] = w[d].res, dcig[d] = w[d].cig;
	}
	ok = pl_group_gather(n, dev_of_job, g->n_dev, dres, dcig, results, cigar, cigar_cap, total_cigar);
out:
	for (d = 0; d < g->n_dev; ++d) free(w[d].res), free(w[d].cig);
	free(dev_of_job);
	return ok;
}
