/*
 * port_bench.c -- ORACLE timing driver for the restatement (test/bench infrastructure only).
 * Same contract as ref_bench.c, for machines where the reference build is absent:
 * port_global_gs_auto over a job list on a plain pthread pool.
 */
#define _POSIX_C_SOURCE 200809L
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <time.h>
#include "../include/plgpu.h"

void port_global_gs_auto(const char *ns, int32_t nl, const char *as, int32_t al, const ns_opt_t *opt,
		const uint8_t *ss, ns_rst_t *r, int32_t avx2);

typedef struct {
	const char *nt, *aa;
	const int64_t *nt_off, *aa_off;
	const int32_t *nl, *al;
	const ns_opt_t *opt;
	int32_t *score, *n_cigar, n_jobs;
	long next;
} port_bench_t;

static void *port_bench_worker(void *data)
{
	port_bench_t *b = (port_bench_t*)data;
	for (;;) {
		long i = __sync_fetch_and_add(&b->next, 1);
		ns_rst_t r = {0, 0, 0, 0, 0, 0};
		if (i >= b->n_jobs) break;
		port_global_gs_auto(b->nt + b->nt_off[i], b->nl[i], b->aa + b->aa_off[i], b->al[i], b->opt, 0, &r, 1);
		b->score[i] = r.score, b->n_cigar[i] = r.n_cigar;
		free(r.cigar);
	}
	return 0;
}

__attribute__((visibility("default")))
double port_bench_global(int32_t n_threads, int32_t n_jobs, const char *nt, const int64_t *nt_off, const int32_t *nl,
		const char *aa, const int64_t *aa_off, const int32_t *al, const ns_opt_t *opt, int32_t *score, int32_t *n_cigar)
{
	port_bench_t b;
	pthread_t *th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
	struct timespec t0, t1;
	int32_t k;
	b.nt = nt, b.aa = aa, b.nt_off = nt_off, b.aa_off = aa_off, b.nl = nl, b.al = al, b.opt = opt;
	b.score = score, b.n_cigar = n_cigar, b.n_jobs = n_jobs, b.next = 0;
	clock_gettime(CLOCK_MONOTONIC, &t0);
	for (k = 0; k < n_threads; ++k) pthread_create(&th[k], 0, port_bench_worker, &b);
	for (k = 0; k < n_threads; ++k) pthread_join(th[k], 0);
	clock_gettime(CLOCK_MONOTONIC, &t1);
	free(th);
	return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}
