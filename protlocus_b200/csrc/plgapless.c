/*
 * plgapless.c -- host layer of the gapless X-drop candidate prefilter: the
 * reference's entry points (ns_gpu_gapless_*, nasw.h:169-184; semantics of
 * nasw-cuda.cu:1316-1395) and bulk entry points on an engine.
 *
 * As in the reference, ns_gpu_gapless_score_batch needs ns_gpu_init() first,
 * keeps the packed genome resident across calls (re-uploaded only when the
 * caller's pointer or length changes, or after ns_gpu_gapless_reset_target),
 * is serialised by a mutex (mapping worker threads call it concurrently), and
 * counts batches, candidates, anchors and seed positions.
 */
#define _POSIX_C_SOURCE 200809L
#include <limits.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "plhost.h"

void pl_gapless_engine_free(pl_engine_t *e)
{
	dbuf_free(&e->g_packed), dbuf_free(&e->g_queries), dbuf_free(&e->g_cand), dbuf_free(&e->g_anchors);
	dbuf_free(&e->g_mat), dbuf_free(&e->g_codon), dbuf_free(&e->g_scores), dbuf_free(&e->g_steps);
	e->g_cached_src = 0, e->g_cached_bases = 0;
}

static int pl_gapless_check(int32_t n, int64_t n_anchors, int32_t block_width, int32_t kmer, int32_t xdrop,
		int32_t asize)
{
	if (n < 0 || n_anchors < 0) { pl_set_error("negative candidate or anchor count"); return 0; }
	if (block_width < 1 || block_width > 8192) { pl_set_error("block_width %d outside 1..8192", block_width); return 0; }
	if (kmer < 1 || kmer > 64) { pl_set_error("kmer %d outside 1..64", kmer); return 0; }
	if (xdrop < 0) { pl_set_error("xdrop %d < 0", xdrop); return 0; }
	if (asize < 21 || asize > 32) { pl_set_error("asize %d outside 21..32", asize); return 0; }
	return 1;
}

/* device-resident inputs; matrix and codon table from the host */
static int pl_gapless_run(pl_engine_t *e, const uint8_t *packed, int64_t bases, const uint8_t *queries,
		int64_t query_aa, const void *cand, int32_t n, const void *anchors, int64_t n_anchors, int32_t block_width,
		int32_t kmer, int32_t xdrop, const int8_t *mat, int32_t asize, const uint8_t *codon, int32_t *scores_dev,
		cudaStream_t st)
{
	unsigned long long steps = 0;
	if (!pl_gapless_check(n, n_anchors, block_width, kmer, xdrop, asize)) return 0;
	if (n == 0) return 1;
	if (!dbuf_ensure(&e->g_mat, (size_t)asize * asize) || !dbuf_ensure(&e->g_codon, 64) || !dbuf_ensure(&e->g_steps, 16))
		return 0;
	CK(cudaMemcpyAsync(e->g_mat.p, mat, (size_t)asize * asize, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->g_codon.p, codon, 64, cudaMemcpyHostToDevice, st));
	CK(cudaMemsetAsync(e->g_steps.p, 0, 16, st));
	e->n_ev = 0;
	PL_TIME(e, st, 1);
	CKK(plk_gapless(packed, bases, queries, query_aa, cand, n, anchors, n_anchors, block_width, kmer, xdrop,
			(const int8_t*)e->g_mat.p, asize, (const uint8_t*)e->g_codon.p, scores_dev,
			(unsigned long long*)e->g_steps.p, e->n_sm, st));
	PL_TIME(e, st, 1);
	CK(cudaMemcpyAsync(&steps, e->g_steps.p, sizeof(steps), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	e->g_last_steps = (int64_t)steps;
	if (e->timing && e->n_ev >= 2) {
		float ms;
		cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]);
		e->acc_ms[1] += ms, e->acc_dp_launches += 1, e->acc_cells += n_anchors * block_width;
	}
	return 1;
fail:
	return 0;
}

PL_EXPORT int pl_gapless_score_device(pl_engine_t *e, const uint8_t *packed_nt, int64_t packed_nt_bases,
		const uint8_t *queries, int64_t query_aa, const ns_gpu_gapless_candidate_t *candidates, int32_t n_candidates,
		const ns_gpu_gapless_anchor_t *anchors, int64_t n_anchors, int32_t block_width, int32_t kmer, int32_t xdrop,
		const int8_t *score_matrix, int32_t asize, const uint8_t *codon, int32_t *scores_dev, void *stream)
{
	if (!e) { pl_set_error("no engine"); return 0; }
	if (cudaSetDevice(e->device) != cudaSuccess) { pl_set_error("cudaSetDevice failed"); return 0; }
	return pl_gapless_run(e, packed_nt, packed_nt_bases, queries, query_aa, candidates, n_candidates, anchors,
			n_anchors, block_width, kmer, xdrop, score_matrix, asize, codon, scores_dev,
			stream ? (cudaStream_t)stream : e->stream);
}

/* host buffers; the genome is uploaded unless the same pointer and length are resident */
static int pl_gapless_host(pl_engine_t *e, int cache_genome, const uint8_t *packed_nt, int64_t bases,
		const uint8_t *queries, int64_t query_aa, const ns_gpu_gapless_candidate_t *cand, int32_t n,
		const ns_gpu_gapless_anchor_t *anchors, int64_t n_anchors, int32_t block_width, int32_t kmer, int32_t xdrop,
		const int8_t *mat, int32_t asize, const uint8_t *codon, int32_t *scores)
{
	cudaStream_t st = e->stream;
	const size_t packed_bytes = (size_t)((bases + 1) >> 1);
	if (!pl_gapless_check(n, n_anchors, block_width, kmer, xdrop, asize)) return 0;
	if (n == 0) return 1;
	CK(cudaSetDevice(e->device));
	if (!dbuf_ensure(&e->g_queries, (size_t)(query_aa > 0 ? query_aa : 1)) ||
			!dbuf_ensure(&e->g_cand, sizeof(*cand) * (size_t)n) ||
			!dbuf_ensure(&e->g_anchors, sizeof(*anchors) * (size_t)(n_anchors > 0 ? n_anchors : 1)) ||
			!dbuf_ensure(&e->g_scores, sizeof(int32_t) * (size_t)n))
		return 0;
	if (!cache_genome || e->g_cached_src != packed_nt || e->g_cached_bases != bases) {
		e->g_cached_src = 0;
		if (!dbuf_ensure(&e->g_packed, packed_bytes > 0 ? packed_bytes : 1)) return 0;
		if (packed_bytes) CK(cudaMemcpyAsync(e->g_packed.p, packed_nt, packed_bytes, cudaMemcpyHostToDevice, st));
		if (cache_genome) e->g_cached_src = packed_nt, e->g_cached_bases = bases;
	}
	if (query_aa > 0) CK(cudaMemcpyAsync(e->g_queries.p, queries, (size_t)query_aa, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->g_cand.p, cand, sizeof(*cand) * (size_t)n, cudaMemcpyHostToDevice, st));
	if (n_anchors > 0) CK(cudaMemcpyAsync(e->g_anchors.p, anchors, sizeof(*anchors) * (size_t)n_anchors, cudaMemcpyHostToDevice, st));
	if (!pl_gapless_run(e, (const uint8_t*)e->g_packed.p, bases, (const uint8_t*)e->g_queries.p, query_aa, e->g_cand.p, n,
			e->g_anchors.p, n_anchors, block_width, kmer, xdrop, mat, asize, codon, (int32_t*)e->g_scores.p, st))
		return 0;
	CK(cudaMemcpyAsync(scores, e->g_scores.p, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	return 1;
fail:
	return 0;
}

PL_EXPORT int pl_gapless_score_host(pl_engine_t *e, const uint8_t *packed_nt, int64_t packed_nt_bases,
		const uint8_t *queries, int64_t query_aa, const ns_gpu_gapless_candidate_t *candidates, int32_t n_candidates,
		const ns_gpu_gapless_anchor_t *anchors, int64_t n_anchors, int32_t block_width, int32_t kmer, int32_t xdrop,
		const int8_t *score_matrix, int32_t asize, const uint8_t *codon, int32_t *scores)
{
	if (!e) { pl_set_error("no engine"); return 0; }
	return pl_gapless_host(e, 0, packed_nt, packed_nt_bases, queries, query_aa, candidates, n_candidates, anchors,
			n_anchors, block_width, kmer, xdrop, score_matrix, asize, codon, scores);
}

PL_EXPORT int64_t pl_gapless_last_steps(const pl_engine_t *e) { return e ? e->g_last_steps : 0; }

/* ------------------------------------------------------------------ reference entry points (nasw.h:169-184) */

static pthread_mutex_t gl_mu = PTHREAD_MUTEX_INITIALIZER;
static pl_engine_t *gl_engine;
static uint64_t gl_batches, gl_candidates, gl_anchors, gl_seed_positions;

PL_EXPORT void ns_gpu_gapless_profile(ns_gpu_gapless_profile_t *p)
{ /* nasw-cuda.cu:1316-1322 */
	p->batches = __sync_fetch_and_add(&gl_batches, 0ull);
	p->candidates = __sync_fetch_and_add(&gl_candidates, 0ull);
	p->anchors = __sync_fetch_and_add(&gl_anchors, 0ull);
	p->seed_positions = __sync_fetch_and_add(&gl_seed_positions, 0ull);
}

PL_EXPORT int ns_gpu_gapless_supported(void) { return 1; }

PL_EXPORT void ns_gpu_gapless_reset_target(void)
{
	pthread_mutex_lock(&gl_mu);
	if (gl_engine) gl_engine->g_cached_src = 0, gl_engine->g_cached_bases = 0;
	pthread_mutex_unlock(&gl_mu);
}

PL_EXPORT int ns_gpu_gapless_score_batch(const uint8_t *packed_nt, int64_t packed_nt_bases,
		const uint8_t *queries, int64_t query_aa, const ns_gpu_gapless_candidate_t *candidates, int32_t n_candidates,
		const ns_gpu_gapless_anchor_t *anchors, int64_t n_anchors, int32_t block_width, int32_t kmer, int32_t xdrop,
		const int8_t *score_matrix, int32_t asize, const uint8_t *codon, int32_t *scores)
{
	const int dev = pl_ns_device();
	int ok;
	/* the preconditions of nasw-cuda.cu:1340-1344 */
	if (dev < 0 || !packed_nt || packed_nt_bases < 1 || !queries || query_aa < 1 || !candidates || n_candidates < 1 ||
			!anchors || n_anchors < 1 || block_width < 1 || kmer < 1 || xdrop < 0 || !score_matrix || asize < 1 ||
			!codon || !scores)
		return 0;
	pthread_mutex_lock(&gl_mu);
	if (!gl_engine && !(gl_engine = pl_engine_create(dev, 0))) {
		pl_ns_set_error(pl_last_error());
		pthread_mutex_unlock(&gl_mu);
		return 0;
	}
	ok = pl_gapless_host(gl_engine, 1, packed_nt, packed_nt_bases, queries, query_aa, candidates, n_candidates,
			anchors, n_anchors, block_width, kmer, xdrop, score_matrix, asize, codon, scores);
	if (ok) {
		__sync_fetch_and_add(&gl_batches, 1ull);
		__sync_fetch_and_add(&gl_candidates, (uint64_t)n_candidates);
		__sync_fetch_and_add(&gl_anchors, (uint64_t)n_anchors);
		__sync_fetch_and_add(&gl_seed_positions, (uint64_t)n_anchors * (uint64_t)block_width);
	} else {
		char msg[1100];
		snprintf(msg, sizeof(msg), "gapless GPU batch: %s", pl_last_error());
		pl_ns_set_error(msg);
	}
	pthread_mutex_unlock(&gl_mu);
	return ok;
}
