/*
 * plchain.c -- host side of batched anchor chaining (mp_chain, chain.c:160-219).
 *
 * The chaining DP (f, p, v of every anchor) runs on the device (chain.cu); the
 * backtrack that extracts chains best score first (chain.c:8-75) and the compaction
 * that orders them by target position (chain.c:77-110) run here, one query per
 * task over the host's cores.  Both sorts are the reference's in-place MSD radix
 * sort (ksort.h:112-162 as instantiated in misc.c:8): it is not stable, and the
 * order it leaves among equal scores decides which chain claims a shared anchor,
 * so it is restated step for step.
 */
#define _POSIX_C_SOURCE 200809L
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include "plhost.h"

typedef struct { uint64_t x, y; } pl_kv_t;

/* ------------------------------------------------------------------ radix sort on x */

static void pl_kv_insertsort(pl_kv_t *beg, pl_kv_t *end)
{
	pl_kv_t *i, *j, tmp;
	for (i = beg + 1; i < end; ++i)
		if (i->x < (i - 1)->x) {
			tmp = *i;
			for (j = i; j > beg && tmp.x < (j - 1)->x; --j) *j = *(j - 1);
			*j = tmp;
		}
}

/* one pass on the byte of x at shift s: buckets placed in place by following
 * displacement cycles, then each bucket sorted on the next byte (more than 64
 * elements) or by insertion (2 to 64).  A pass whose keys all share the byte
 * leaves the order as it is and hands the whole range to the next byte, so the
 * passes above the highest byte in which the range's keys differ are skipped
 * (identical permutation, without the 256-bucket work). */
static void pl_kv_rsort(pl_kv_t *beg, pl_kv_t *end, int s)
{
	pl_kv_t *bb[256], *be[256], *i, tmp, swap;
	int k, l;
	{
		uint64_t lo = beg->x, hi = beg->x, d;
		for (i = beg + 1; i != end; ++i) lo = i->x < lo ? i->x : lo, hi = i->x > hi ? i->x : hi;
		if (lo == hi) return; /* every pass is the identity */
		d = lo ^ hi;
		k = 63 - __builtin_clzll(d);  /* highest differing bit */
		if (k / 8 * 8 < s) s = k / 8 * 8;
	}
	for (k = 0; k < 256; ++k) bb[k] = be[k] = beg;
	for (i = beg; i != end; ++i) ++be[i->x >> s & 255];
	for (k = 1; k < 256; ++k) be[k] += be[k - 1] - beg, bb[k] = be[k - 1];
	for (k = 0; k < 256;) {
		if (bb[k] != be[k]) {
			if ((l = (int)(bb[k]->x >> s & 255)) != k) {
				tmp = *bb[k];
				do {
					swap = tmp, tmp = *bb[l], *bb[l]++ = swap;
					l = (int)(tmp.x >> s & 255);
				} while (l != k);
				*bb[k]++ = tmp;
			} else ++bb[k];
		} else ++k;
	}
	for (bb[0] = beg, k = 1; k < 256; ++k) bb[k] = be[k - 1];
	if (s) {
		s = s > 8 ? s - 8 : 0;
		for (k = 0; k < 256; ++k)
			if (be[k] - bb[k] > 64) pl_kv_rsort(bb[k], be[k], s);
			else if (be[k] - bb[k] > 1) pl_kv_insertsort(bb[k], be[k]);
	}
}

static void pl_kv_sort(pl_kv_t *beg, pl_kv_t *end)
{
	if (end - beg <= 64) pl_kv_insertsort(beg, end);
	else pl_kv_rsort(beg, end, 56);
}

/* ------------------------------------------------------------------ backtrack + compaction */

typedef struct {
	pl_kv_t *z, *w;
	int32_t *t, *v;
	uint64_t *b, *u2;
	int64_t cap;
} pl_chain_scr_t;

static int pl_chain_scr_grow(pl_chain_scr_t *S, int64_t n)
{
	if (n <= S->cap) return 1;
	free(S->z), free(S->w), free(S->t), free(S->v), free(S->b), free(S->u2);
	S->z = (pl_kv_t*)malloc(sizeof(pl_kv_t) * (size_t)n), S->w = (pl_kv_t*)malloc(sizeof(pl_kv_t) * (size_t)n);
	S->t = (int32_t*)malloc(sizeof(int32_t) * (size_t)n), S->v = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
	S->b = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n), S->u2 = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
	S->cap = n;
	if (!S->z || !S->w || !S->t || !S->v || !S->b || !S->u2) { S->cap = 0; return 0; }
	return 1;
}

static void pl_chain_scr_free(pl_chain_scr_t *S)
{
	free(S->z), free(S->w), free(S->t), free(S->v), free(S->b), free(S->u2);
	memset(S, 0, sizeof(*S));
}

/* walks back from the anchor of z[k] while the chain score keeps its peak within
 * max_drop, marking the walk; returns where the chain starts (chain.c:8-24) */
static int64_t pl_chain_bk_end(int32_t max_drop, const pl_kv_t *z, const int32_t *f, const int32_t *p, int32_t *t,
		int64_t k)
{
	int64_t i = (int64_t)z[k].y, end_i = -1, max_i = i;
	int32_t max_s = 0;
	if (i < 0 || t[i] != 0) return i;
	do {
		int32_t s;
		t[i] = 2;
		if (p[i] >= i) return -2; /* predecessors precede: anything else is a corrupt fill */
		end_i = i = p[i];
		s = i < 0 ? (int32_t)z[k].x : (int32_t)z[k].x - f[i];
		if (s > max_s) max_s = s, max_i = i;
		else if (max_s - s > max_drop) break;
	} while (i >= 0 && t[i] == 0);
	for (i = (int64_t)z[k].y; i >= 0 && i != end_i; i = p[i]) t[i] = 0;
	return max_i;
}

/* chains of one query from its fill: u[] (score << 32 | #anchors, by target position
 * of the first anchor) and the chained anchors in that order; returns #chains */
static int32_t pl_chain_finish1(const pl_chain_opt_t *o, int64_t n, const uint64_t *a, const int32_t *f,
		const int32_t *p, pl_chain_scr_t *S, uint64_t *u, uint64_t *a_out)
{
	const int32_t max_drop = o->is_spliced ? INT32_MAX : o->bw;
	int64_t i, k, n_z = 0, n_v = 0;
	int32_t n_u = 0;
	for (i = 0; i < n; ++i)
		if (f[i] >= o->min_sc) S->z[n_z].x = (uint64_t)(int64_t)f[i], S->z[n_z++].y = (uint64_t)i;
	if (n_z == 0) return 0;
	pl_kv_sort(S->z, S->z + n_z);
	memset(S->t, 0, sizeof(int32_t) * (size_t)n);
	for (k = n_z - 1; k >= 0; --k) { /* best score first (chain.c:56-70) */
		if (S->t[S->z[k].y] == 0) {
			const int64_t n_v0 = n_v, end_i = pl_chain_bk_end(max_drop, S->z, f, p, S->t, k);
			int32_t sc;
			if (end_i < -1) return -1;
			for (i = (int64_t)S->z[k].y; i != end_i; i = p[i]) {
				if (i < 0 || n_v >= n) return -1; /* walked past the chain start: corrupt fill */
				S->v[n_v++] = (int32_t)i, S->t[i] = 1;
			}
			sc = i < 0 ? (int32_t)S->z[k].x : (int32_t)S->z[k].x - f[i];
			if (sc >= o->min_sc && n_v > n_v0 && n_v - n_v0 >= o->min_cnt)
				u[n_u++] = (uint64_t)(int64_t)sc << 32 | (uint64_t)(n_v - n_v0);
			else n_v = n_v0;
		}
	}
	if (n_u == 0) return 0;
	{ /* compaction (chain.c:77-110): anchors of each chain in ascending order, chains
	   * ordered by the target block of their first anchor */
		int64_t kk = 0;
		for (i = 0; i < n_u; ++i) {
			const int64_t k0 = kk, ni = (int32_t)u[i];
			int64_t j;
			for (j = 0; j < ni; ++j) S->b[kk++] = a[S->v[k0 + (ni - j - 1)]];
		}
		for (i = kk = 0; i < n_u; ++i) {
			S->w[i].x = S->b[kk] >> 32, S->w[i].y = (uint64_t)kk << 32 | (uint64_t)i;
			kk += (int32_t)u[i];
		}
		pl_kv_sort(S->w, S->w + n_u);
		for (i = kk = 0; i < n_u; ++i) {
			const int32_t j = (int32_t)S->w[i].y, nj = (int32_t)u[j];
			S->u2[i] = u[j];
			memcpy(&a_out[kk], &S->b[S->w[i].y >> 32], (size_t)nj * sizeof(uint64_t));
			kk += nj;
		}
		memcpy(u, S->u2, (size_t)n_u * sizeof(uint64_t));
	}
	return n_u;
}

PL_EXPORT int pl_chain_finish(const pl_chain_opt_t *opt, int64_t n, const uint64_t *a, const int32_t *f,
		const int32_t *p, uint64_t *u, int32_t *n_u, uint64_t *a_out)
{
	pl_chain_scr_t S;
	memset(&S, 0, sizeof(S));
	*n_u = 0;
	if (n <= 0) return 1;
	if (!pl_chain_scr_grow(&S, n)) { pl_set_error("out of host memory"); pl_chain_scr_free(&S); return 0; }
	*n_u = pl_chain_finish1(opt, n, a, f, p, &S, u, a_out);
	pl_chain_scr_free(&S);
	if (*n_u < 0) { *n_u = 0; pl_set_error("chaining: predecessor array is not a forest of backward links"); return 0; }
	return 1;
}

/* ------------------------------------------------------------------ batch */

void pl_chain_engine_free(pl_engine_t *e)
{
	dbuf_free(&e->c_off), dbuf_free(&e->c_n), dbuf_free(&e->c_order), dbuf_free(&e->c_a), dbuf_free(&e->c_f);
	dbuf_free(&e->c_p), dbuf_free(&e->c_v), dbuf_free(&e->c_t), dbuf_free(&e->c_counter);
	if (e->c_host) cudaFreeHost(e->c_host);
	e->c_host = 0, e->c_host_cap = 0;
}

/* the engine's pinned host buffer, grown to at least `need` bytes */
static void *pl_chain_pinned(pl_engine_t *e, size_t need)
{
	if (need == 0) need = 16;
	if (e->c_host_cap >= need) return e->c_host;
	if (e->c_host) cudaFreeHost(e->c_host);
	e->c_host = 0, e->c_host_cap = 0;
	if (cudaHostAlloc(&e->c_host, need, cudaHostAllocDefault) != cudaSuccess) {
		cudaGetLastError();
		e->c_host = 0;
		pl_set_error("cudaHostAlloc of %zu bytes failed", need);
		return 0;
	}
	e->c_host_cap = need;
	return e->c_host;
}

/* the options as mp_chain applies them before its fill (chain.c:173-175) */
static void pl_chain_norm(const pl_chain_opt_t *in, pl_chain_opt_t *o)
{
	*o = *in;
	if (o->max_dist_x < o->bw) o->max_dist_x = o->bw;
	if (o->max_dist_y < o->bw && !o->is_spliced) o->max_dist_y = o->bw;
}

static __thread const int32_t *pl_chain_sort_n;  /* the lengths pl_chain_cmp_len orders by */
static int pl_chain_cmp_len(const void *x, const void *y)
{
	const int32_t a = *(const int32_t*)x, b = *(const int32_t*)y;
	if (pl_chain_sort_n[a] != pl_chain_sort_n[b]) return pl_chain_sort_n[a] > pl_chain_sort_n[b] ? -1 : 1;
	return a < b ? -1 : a > b;
}

PL_EXPORT int pl_chain_fill_device(pl_engine_t *e, const pl_chain_opt_t *opt, int32_t n_q, const int64_t *off,
		const int32_t *n, const uint64_t *a_dev, int64_t n_a, int32_t *f_dev, int32_t *p_dev, int32_t *v_dev,
		void *stream)
{
	pl_chain_opt_t o;
	plk_chain_args_t A;
	int64_t *key = 0;
	int32_t *order = 0, q;
	int ok = 0;
	cudaStream_t st;
	if (!e || !opt) { pl_set_error("no engine or options"); return 0; }
	if (n_q <= 0) return 1;
	for (q = 0; q < n_q; ++q)
		if (n[q] < 0 || off[q] < 0 || off[q] + n[q] > n_a) { pl_set_error("query %d: anchors outside the buffer", q); return 0; }
	if (opt->bbit < 0 || opt->bbit > 31) { pl_set_error("bbit %d outside 0..31", opt->bbit); return 0; }
	pl_chain_norm(opt, &o);
	{ /* longest first, ties by query index: a counting sort on n while its table stays small next to
	   * the batch, else a comparison sort (one long query must not cost a table of its length) */
		int32_t max_n = 0, m;
		int64_t pos = 0;
		for (q = 0; q < n_q; ++q) if (n[q] > max_n) max_n = n[q];
		order = (int32_t*)malloc(sizeof(int32_t) * (size_t)n_q);
		if (!order) { pl_set_error("out of host memory"); goto fail; }
		if ((int64_t)max_n <= 4 * (int64_t)n_q + 65536) {
			key = (int64_t*)calloc((size_t)max_n + 1, sizeof(int64_t));
			if (!key) { pl_set_error("out of host memory"); goto fail; }
			for (q = 0; q < n_q; ++q) ++key[n[q]];
			for (m = max_n; m >= 0; --m) { const int64_t c = key[m]; key[m] = pos, pos += c; }
			for (q = 0; q < n_q; ++q) order[key[n[q]]++] = q;
		} else {
			pl_chain_sort_n = n;
			for (q = 0; q < n_q; ++q) order[q] = q;
			qsort(order, (size_t)n_q, sizeof(int32_t), pl_chain_cmp_len);
		}
	}
	CK(cudaSetDevice(e->device));
	st = stream ? (cudaStream_t)stream : e->stream;
	if (!dbuf_ensure(&e->c_off, sizeof(int64_t) * (size_t)n_q) || !dbuf_ensure(&e->c_n, sizeof(int32_t) * (size_t)n_q) ||
			!dbuf_ensure(&e->c_order, sizeof(int32_t) * (size_t)n_q) || !dbuf_ensure(&e->c_counter, 64) ||
			!dbuf_ensure(&e->c_t, sizeof(int32_t) * (size_t)(n_a > 0 ? n_a : 1)))
		goto fail;
	CK(cudaMemcpyAsync(e->c_off.p, off, sizeof(int64_t) * (size_t)n_q, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->c_n.p, n, sizeof(int32_t) * (size_t)n_q, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->c_order.p, order, sizeof(int32_t) * (size_t)n_q, cudaMemcpyHostToDevice, st));
	memset(&A, 0, sizeof(A));
	A.off = (const int64_t*)e->c_off.p, A.n = (const int32_t*)e->c_n.p, A.order = (const int32_t*)e->c_order.p;
	A.a = a_dev, A.f = f_dev, A.p = p_dev, A.v = v_dev, A.t = (int32_t*)e->c_t.p;
	A.err = (int32_t*)((char*)e->c_counter.p + 16), A.n_a = n_a;
	CK(cudaMemsetAsync(A.err, 0, 2 * sizeof(int32_t), st));
	A.n_q = n_q, A.max_dist_x = o.max_dist_x, A.max_dist_y = o.max_dist_y, A.bw = o.bw, A.max_skip = o.max_skip;
	A.max_iter = o.max_iter, A.is_spliced = o.is_spliced, A.kmer = o.kmer, A.bbit = o.bbit, A.coef = o.chn_coef_log;
	if (e->timing) { /* count the scored predecessors in the scratch block's second half */
		A.pairs = (unsigned long long*)((char*)e->c_counter.p + 32);
		CK(cudaMemsetAsync(A.pairs, 0, sizeof(unsigned long long), st));
	}
	{
		const int32_t ctas = (n_q + plk_chain_threads_per_cta() - 1) / plk_chain_threads_per_cta();
		e->n_ev = 0;
		PL_TIME(e, st, 1);
		CKK(plk_chain_fill(&A, ctas, st));
		PL_TIME(e, st, 1);
	}
	{ /* the kernel's own index checks: site and query of the last failure */
		int32_t err[2] = { 0, 0 };
		CK(cudaMemcpyAsync(err, A.err, sizeof(err), cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
		if (err[0]) { pl_set_error("chaining DP: index check %d failed on the device (query %d)", err[0], err[1]); goto fail; }
	}
	if (e->timing) { /* block until the fill's events are complete, then bank them */
		int k;
		float ms;
		unsigned long long pairs = 0;
		CK(cudaMemcpyAsync(&pairs, A.pairs, sizeof(pairs), cudaMemcpyDeviceToHost, st));
		CK(cudaStreamSynchronize(st));
		e->c_last_pairs = (int64_t)pairs;
		for (k = 0; k + 1 < e->n_ev; k += 2) {
			cudaEventElapsedTime(&ms, e->ev[k], e->ev[k + 1]);
			e->acc_ms[e->ev_kind[k]] += ms;
		}
		e->acc_dp_launches += 1, e->acc_cells += n_a;
	}
	ok = 1;
fail:
	free(key), free(order);
	return ok;
}

typedef struct {
	const pl_chain_opt_t *o;
	const int64_t *off;
	const int32_t *n;
	const uint64_t *a;
	const int32_t *f, *p;
	uint64_t *u, *a_out;
	int32_t *n_u;
	int32_t n_q, next, fail;
} pl_chain_work_t;

static void *pl_chain_worker(void *arg)
{
	pl_chain_work_t *W = (pl_chain_work_t*)arg;
	pl_chain_scr_t S;
	memset(&S, 0, sizeof(S));
	for (;;) {
		const int32_t q = __sync_fetch_and_add(&W->next, 1);
		if (q >= W->n_q) break;
		if (!pl_chain_scr_grow(&S, W->n[q] > 0 ? W->n[q] : 1)) { W->fail = 1; break; }
		W->n_u[q] = W->n[q] > 0 ? pl_chain_finish1(W->o, W->n[q], W->a + W->off[q], W->f + W->off[q],
				W->p + W->off[q], &S, W->u + W->off[q], W->a_out + W->off[q]) : 0;
		if (W->n_u[q] < 0) { W->n_u[q] = 0, W->fail = 2; break; }
	}
	pl_chain_scr_free(&S);
	return 0;
}

/* host threads for the backtrack: PLGPU_CHAIN_THREADS or every online core (at most 128) */
static int pl_chain_threads(void)
{
	const char *s = getenv("PLGPU_CHAIN_THREADS");
	long c = s && *s ? atol(s) : sysconf(_SC_NPROCESSORS_ONLN);
	if (c < 1) c = 1;
	if (c > 128) c = 128;
	return (int)c;
}

PL_EXPORT int pl_chain_host(pl_engine_t *e, const pl_chain_opt_t *opt, int32_t n_q, const int64_t *off, const int32_t *n,
		const uint64_t *a, int64_t n_a, uint64_t *u, int32_t *n_u, uint64_t *a_out)
{
	pl_chain_opt_t o;
	int32_t *hf = 0, *hp = 0;
	int ok = 0, nt, k;
	cudaStream_t st;
	pthread_t th[128];
	pl_chain_work_t W;
	if (!e || !opt) { pl_set_error("no engine or options"); return 0; }
	if (n_q <= 0) return 1;
	pl_chain_norm(opt, &o);
	CK(cudaSetDevice(e->device));
	st = e->stream;
	if (!dbuf_ensure(&e->c_a, sizeof(uint64_t) * (size_t)(n_a > 0 ? n_a : 1)) ||
			!dbuf_ensure(&e->c_f, sizeof(int32_t) * (size_t)(n_a > 0 ? n_a : 1)) ||
			!dbuf_ensure(&e->c_p, sizeof(int32_t) * (size_t)(n_a > 0 ? n_a : 1)) ||
			!dbuf_ensure(&e->c_v, sizeof(int32_t) * (size_t)(n_a > 0 ? n_a : 1)))
		return 0;
	hf = (int32_t*)pl_chain_pinned(e, 2 * sizeof(int32_t) * (size_t)(n_a > 0 ? n_a : 1));
	if (!hf) goto fail;
	hp = hf + (n_a > 0 ? n_a : 1);
	if (n_a > 0) CK(cudaMemcpyAsync(e->c_a.p, a, sizeof(uint64_t) * (size_t)n_a, cudaMemcpyHostToDevice, st));
	if (!pl_chain_fill_device(e, opt, n_q, off, n, (const uint64_t*)e->c_a.p, n_a, (int32_t*)e->c_f.p, (int32_t*)e->c_p.p,
			(int32_t*)e->c_v.p, st))
		goto fail;
	if (n_a > 0) {
		CK(cudaMemcpyAsync(hf, e->c_f.p, sizeof(int32_t) * (size_t)n_a, cudaMemcpyDeviceToHost, st));
		CK(cudaMemcpyAsync(hp, e->c_p.p, sizeof(int32_t) * (size_t)n_a, cudaMemcpyDeviceToHost, st));
	}
	CK(cudaStreamSynchronize(st));
	memset(&W, 0, sizeof(W));
	W.o = &o, W.off = off, W.n = n, W.a = a, W.f = hf, W.p = hp, W.u = u, W.a_out = a_out, W.n_u = n_u, W.n_q = n_q;
	nt = pl_chain_threads();
	if (nt > n_q) nt = n_q;
	for (k = 1; k < nt; ++k)
		if (pthread_create(&th[k], 0, pl_chain_worker, &W) != 0) { nt = k; break; }
	pl_chain_worker(&W);
	for (k = 1; k < nt; ++k) pthread_join(th[k], 0);
	if (W.fail) {
		pl_set_error(W.fail == 2 ? "chaining: predecessor array is not a forest of backward links" : "out of host memory");
		goto fail;
	}
	ok = 1;
fail:
	return ok;
}

PL_EXPORT int64_t pl_chain_last_pairs(const pl_engine_t *e) { return e ? e->c_last_pairs : 0; }
