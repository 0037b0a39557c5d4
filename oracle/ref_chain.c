/*
 * ref_chain.c -- test infrastructure: the reference's own mp_chain (chain.c:160)
 * behind plain arrays, so that the batched chaining (chain.cu + plchain.c) is
 * checked against the reference itself.  Compiled with the reference sources by
 * oracle/Makefile (`extra`).
 */
#include <stdlib.h>
#include <string.h>
#include "mppriv.h"

/* chains of n anchors a[]: u_out (n_u words) and the chained anchors a_out (the sum
 * of the chains' counts); both hold up to n words.  Returns the chained anchor count. */
int64_t ref_chain(int32_t max_dist_x, int32_t max_dist_y, int32_t bw, int32_t max_skip, int32_t max_iter,
		int32_t min_cnt, int32_t min_sc, float chn_coef_log, int32_t is_spliced, int32_t kmer, int32_t bbit,
		int64_t n, const uint64_t *a_in, uint64_t *u_out, int32_t *n_u, uint64_t *a_out)
{
	uint64_t *a = 0, *u = 0, *r;
	int32_t i, nu = 0;
	int64_t tot = 0;
	if (n > 0) {
		a = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
		memcpy(a, a_in, sizeof(uint64_t) * (size_t)n);
	}
	r = mp_chain(max_dist_x, max_dist_y, bw, max_skip, max_iter, min_cnt, min_sc, chn_coef_log, is_spliced, kmer, bbit,
			n, a, &nu, &u, 0);
	for (i = 0; i < nu; ++i) tot += (uint32_t)u[i];
	if (nu > 0) memcpy(u_out, u, sizeof(uint64_t) * (size_t)nu);
	if (tot > 0) memcpy(a_out, r, sizeof(uint64_t) * (size_t)tot);
	*n_u = nu;
	free(u), free(r);
	return tot;
}

/* the reference's mp_chain over a batch of queries on n_threads host threads (the
 * reference's kt_for); returns the total number of chained anchors */
typedef struct {
	int32_t arg[7], is_spliced, kmer, bbit;
	float coef;
	const int64_t *off;
	const int32_t *n;
	const uint64_t *a;
	int64_t *tot;
} ref_chain_batch_t;

void kt_for(int n_threads, void (*func)(void*, long, int), void *data, long n);

static void ref_chain_one(void *data, long q, int tid)
{
	ref_chain_batch_t *B = (ref_chain_batch_t*)data;
	uint64_t *a = 0, *u = 0, *r;
	int32_t nu = 0, i;
	int64_t n = B->n[q], tot = 0;
	(void)tid;
	if (n > 0) {
		a = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
		memcpy(a, B->a + B->off[q], sizeof(uint64_t) * (size_t)n);
	}
	r = mp_chain(B->arg[0], B->arg[1], B->arg[2], B->arg[3], B->arg[4], B->arg[5], B->arg[6], B->coef, B->is_spliced,
			B->kmer, B->bbit, n, a, &nu, &u, 0);
	for (i = 0; i < nu; ++i) tot += (uint32_t)u[i];
	B->tot[q] = tot;
	free(u), free(r);
}

int64_t ref_chain_batch(int32_t max_dist_x, int32_t max_dist_y, int32_t bw, int32_t max_skip, int32_t max_iter,
		int32_t min_cnt, int32_t min_sc, float chn_coef_log, int32_t is_spliced, int32_t kmer, int32_t bbit,
		int32_t n_q, const int64_t *off, const int32_t *n, const uint64_t *a, int32_t n_threads)
{
	ref_chain_batch_t B;
	int64_t q, tot = 0;
	B.arg[0] = max_dist_x, B.arg[1] = max_dist_y, B.arg[2] = bw, B.arg[3] = max_skip, B.arg[4] = max_iter;
	B.arg[5] = min_cnt, B.arg[6] = min_sc, B.coef = chn_coef_log, B.is_spliced = is_spliced, B.kmer = kmer, B.bbit = bbit;
	B.off = off, B.n = n, B.a = a;
	B.tot = (int64_t*)calloc((size_t)(n_q > 0 ? n_q : 1), sizeof(int64_t));
	kt_for(n_threads, ref_chain_one, &B, n_q);
	for (q = 0; q < n_q; ++q) tot += B.tot[q];
	free(B.tot);
	return tot;
}
