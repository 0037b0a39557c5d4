/*
 * ref_bench.c -- ORACLE timing driver (test/bench infrastructure only).
 *
 * Linked into oracle/_ref/libnsref.so next to the reference's nasw-sse.c,
 * nasw-tab.c, kalloc.c and kthread.c.  Runs the reference CPU path
 * ns_global_gs_auto (nasw-sse.c:980-999) with NS_F_CIGAR over a list of jobs,
 * spread over host threads with the reference's own kt_for (kthread.c:54), the
 * way the mapping pipeline drives it.  Used as bench.py's CPU baseline and by
 * `bench.py --impl reference`.
 */
#define _POSIX_C_SOURCE 200809L
#include <stdint.h>
#include <stdlib.h>
#include <time.h>
#include "nasw.h"
#include "kthread.h"

typedef struct {
	const char *nt, *aa;
	const int64_t *nt_off, *aa_off;
	const int32_t *nl, *al;
	const ns_opt_t *opt;
	int32_t *score, *n_cigar;
} ref_bench_t;

static void ref_bench_worker(void *data, long i, int tid)
{
	ref_bench_t *b = (ref_bench_t*)data;
	ns_rst_t r;
	(void)tid;
	ns_rst_init(&r);
	ns_global_gs_auto(0, b->nt + b->nt_off[i], b->nl[i], b->aa + b->aa_off[i], b->al[i], b->opt, 0, &r);
	b->score[i] = r.score, b->n_cigar[i] = r.n_cigar;
	free(r.cigar);
}

/* returns wall seconds */
double ref_bench_global(int32_t n_threads, int32_t n_jobs, const char *nt, const int64_t *nt_off, const int32_t *nl,
		const char *aa, const int64_t *aa_off, const int32_t *al, const ns_opt_t *opt, int32_t *score, int32_t *n_cigar)
{
	ref_bench_t b;
	struct timespec t0, t1;
	b.nt = nt, b.aa = aa, b.nt_off = nt_off, b.aa_off = aa_off, b.nl = nl, b.al = al, b.opt = opt;
	b.score = score, b.n_cigar = n_cigar;
	clock_gettime(CLOCK_MONOTONIC, &t0);
	kt_for(n_threads, ref_bench_worker, &b, n_jobs);
	clock_gettime(CLOCK_MONOTONIC, &t1);
	return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}

/* Extension DPs: the reference's ns_global_gs16b (nasw-sse.c:763-772) with each
 * job's NS_F_EXT_LEFT / NS_F_EXT_RIGHT flag, no CIGAR, over kt_for -- the CPU
 * path ns_ext_batch_* replaces (nasw-ext-gpu.c:118-122). */
typedef struct {
	const char *nt, *aa;
	const int64_t *nt_off, *aa_off;
	const int32_t *nl, *al, *flag;
	const ns_opt_t *opt;
	int32_t *score, *nt_len, *aa_len;
} ref_bench_ext_t;

static void ref_bench_ext_worker(void *data, long i, int tid)
{
	ref_bench_ext_t *b = (ref_bench_ext_t*)data;
	ns_opt_t o = *b->opt;
	ns_rst_t r;
	(void)tid;
	o.flag = (o.flag & ~(NS_F_CIGAR | NS_F_EXT_LEFT | NS_F_EXT_RIGHT)) | b->flag[i];
	ns_rst_init(&r);
	ns_global_gs16b(0, b->nt + b->nt_off[i], b->nl[i], b->aa + b->aa_off[i], b->al[i], &o, 0, &r);
	b->score[i] = r.score, b->nt_len[i] = r.nt_len, b->aa_len[i] = r.aa_len;
	free(r.cigar);
}

double ref_bench_ext(int32_t n_threads, int32_t n_jobs, const char *nt, const int64_t *nt_off, const int32_t *nl,
		const char *aa, const int64_t *aa_off, const int32_t *al, const int32_t *flag, const ns_opt_t *opt,
		int32_t *score, int32_t *nt_len, int32_t *aa_len)
{
	ref_bench_ext_t b;
	struct timespec t0, t1;
	b.nt = nt, b.aa = aa, b.nt_off = nt_off, b.aa_off = aa_off, b.nl = nl, b.al = al, b.flag = flag, b.opt = opt;
	b.score = score, b.nt_len = nt_len, b.aa_len = aa_len;
	clock_gettime(CLOCK_MONOTONIC, &t0);
	kt_for(n_threads, ref_bench_ext_worker, &b, n_jobs);
	clock_gettime(CLOCK_MONOTONIC, &t1);
	return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}

/* Profile-HMM regions: the reference's mp_hmm_dp_score (hmm.c:252-291) over kt_for,
 * the CPU path of mp_hmm_batch_flush (hmm.c:319-335). */
typedef struct mp_hmm_s mp_hmm_t;
int32_t mp_hmm_dp_score(const mp_hmm_t *h, const uint8_t *nt, int32_t nlen);
typedef struct {
	const mp_hmm_t *h;
	const uint8_t *nt;
	const int32_t *off, *len;
	int32_t *score;
} ref_bench_hmm_t;

static void ref_bench_hmm_worker(void *data, long i, int tid)
{
	ref_bench_hmm_t *b = (ref_bench_hmm_t*)data;
	(void)tid;
	b->score[i] = mp_hmm_dp_score(b->h, b->nt + b->off[i], b->len[i]);
}

double ref_bench_hmm(int32_t n_threads, const mp_hmm_t *h, int32_t n, const uint8_t *nt, const int32_t *off,
		const int32_t *len, int32_t *score)
{
	ref_bench_hmm_t b;
	struct timespec t0, t1;
	b.h = h, b.nt = nt, b.off = off, b.len = len, b.score = score;
	clock_gettime(CLOCK_MONOTONIC, &t0);
	kt_for(n_threads, ref_bench_hmm_worker, &b, n);
	clock_gettime(CLOCK_MONOTONIC, &t1);
	return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}
