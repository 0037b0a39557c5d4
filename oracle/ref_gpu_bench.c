/*
 * ref_gpu_bench.c -- ORACLE build helper (test infrastructure only): timing driver
 * for the reference's own CUDA global DP (nasw-cuda.cu, compiled for sm_100a into
 * oracle/_ref/libnscuda_ref.so by oracle/Makefile's refcuda target).
 *
 * ref_gpu_queue_bench submits n jobs through the reference's request queue
 * (ns_gpu_submit from n_threads host threads, as its kt_for workers would) and
 * then waits for each (ns_gpu_wait, which also runs its host backtrack); it
 * returns the wall seconds and sets taken[q] (1 when the queue accepted job q)
 * and score[q].  ref_gpu_global_latency times single ns_gpu_global calls on one
 * job (the queue collects for up to 2 ms before dispatching, nasw-cuda.cu:423).
 */
#define _POSIX_C_SOURCE 200809L
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "nasw.h"

typedef struct {
	const char *nt, *aa;
	const int64_t *nt_off, *aa_off;
	const int32_t *nl, *al;
	int32_t n, t, n_threads;
	const ns_opt_t *opt;
	ns_gpu_request_t **req;
	int32_t *score, *taken;
} rgb_ctx_t;

static double rgb_now(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void *rgb_submit(void *arg)
{
	rgb_ctx_t *c = (rgb_ctx_t*)arg;
	int32_t q;
	for (q = c->t; q < c->n; q += c->n_threads) {
		c->req[q] = ns_gpu_submit(0, c->nt + c->nt_off[q], c->nl[q], c->aa + c->aa_off[q], c->al[q], c->opt, 0);
		c->taken[q] = c->req[q] != 0;
	}
	return 0;
}

static void *rgb_wait(void *arg)
{
	rgb_ctx_t *c = (rgb_ctx_t*)arg;
	int32_t q;
	for (q = c->t; q < c->n; q += c->n_threads) {
		ns_rst_t r;
		memset(&r, 0, sizeof(r));
		c->score[q] = INT32_MIN;
		if (c->req[q] && ns_gpu_wait(c->req[q], &r)) c->score[q] = r.score;
		free(r.cigar);
	}
	return 0;
}

double ref_gpu_queue_bench(int32_t device, int32_t n_threads, const ns_opt_t *opt, int32_t n, const char *nt,
		const int64_t *nt_off, const int32_t *nl, const char *aa, const int64_t *aa_off, const int32_t *al,
		int32_t *score, int32_t *taken)
{
	rgb_ctx_t *ctx;
	pthread_t *th;
	ns_gpu_request_t **req;
	double t0, t1;
	int32_t t;
	if (n_threads < 1) n_threads = 1;
	if (!ns_gpu_init(device)) return -1.0;
	ctx = (rgb_ctx_t*)calloc((size_t)n_threads, sizeof(*ctx));
	th = (pthread_t*)calloc((size_t)n_threads, sizeof(*th));
	req = (ns_gpu_request_t**)calloc((size_t)(n > 0 ? n : 1), sizeof(*req));
	if (!ctx || !th || !req) { free(ctx), free(th), free(req); return -1.0; }
	for (t = 0; t < n_threads; ++t) {
		rgb_ctx_t *c = &ctx[t];
		c->nt = nt, c->aa = aa, c->nt_off = nt_off, c->aa_off = aa_off, c->nl = nl, c->al = al;
		c->n = n, c->t = t, c->n_threads = n_threads, c->opt = opt, c->req = req, c->score = score, c->taken = taken;
	}
	t0 = rgb_now();
	for (t = 0; t < n_threads; ++t) pthread_create(&th[t], 0, rgb_submit, &ctx[t]);
	for (t = 0; t < n_threads; ++t) pthread_join(th[t], 0);
	for (t = 0; t < n_threads; ++t) pthread_create(&th[t], 0, rgb_wait, &ctx[t]);
	for (t = 0; t < n_threads; ++t) pthread_join(th[t], 0);
	t1 = rgb_now();
	free(ctx), free(th), free(req);
	return t1 - t0;
}

/* seconds of each of `reps` ns_gpu_global calls on one job, into secs[]; returns the score */
int32_t ref_gpu_global_latency(int32_t device, const ns_opt_t *opt, const char *nt, int32_t nl, const char *aa,
		int32_t al, int32_t reps, double *secs)
{
	int32_t k, score = INT32_MIN;
	if (!ns_gpu_init(device)) return INT32_MIN;
	for (k = 0; k < reps; ++k) {
		ns_rst_t r;
		double t0;
		memset(&r, 0, sizeof(r));
		t0 = rgb_now();
		if (ns_gpu_global(0, nt, nl, aa, al, opt, 0, &r)) score = r.score;
		secs[k] = rgb_now() - t0;
		free(r.cigar);
	}
	return score;
}
