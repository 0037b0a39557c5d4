/*
 * plext.c -- host layer of the batched extension DP: the bulk entry points
 * (pl_ext_batch_host / pl_ext_batch_device) and the reference's batch object
 * (ns_ext_batch_*, nasw.h:195-212), replacing nasw-ext-gpu.c.
 *
 * A flush hands its requests to one process-wide executor thread and returns.
 * The executor takes every flush that is waiting (from any mapping thread),
 * groups the requests by option set, packs them into staging buffers and runs
 * each group as one device batch (preparation, DP, results) on its own engine.
 * Results are fetched per request; get() blocks on the flush's completion.
 * There is no CPU fallback and nothing aborts: a failed device batch (or a host
 * allocation that fails) marks its requests as failed, ns_ext_batch_get()
 * returns NULL for them and the error text is in ns_gpu_error() and
 * pl_last_error().
 */
#define _POSIX_C_SOURCE 200809L
#include <limits.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "plhost.h"

/* ------------------------------------------------------------------ stripe width */

static int pl_host_avx2(void)
{
#if defined(__x86_64__) || defined(__i386__)
	static int v = -1;
	if (v < 0) {
		__builtin_cpu_init();
		v = __builtin_cpu_supports("avx2") ? 1 : 0;
	}
	return v;
#else
	return 0;
#endif
}

static pthread_once_t pl_lanes_once = PTHREAD_ONCE_INIT;
static int pl_wide_lanes;  /* 1: the CPU kernel this library matches dispatches ext DPs to AVX2 */

static void pl_lanes_init(void)
{
	const char *env = getenv("PLGPU_EXT_STRIPE");
	pl_wide_lanes = pl_host_avx2();
	if (env && (atoi(env) == 8 || atoi(env) == 16)) pl_wide_lanes = atoi(env) == 16;
}

PL_EXPORT int32_t pl_ext_stripe_width(const ns_opt_t *opt, int32_t al)
{ /* nasw-sse.c:744-750 */
	pthread_once(&pl_lanes_once, pl_lanes_init);
	return (opt->flag & (NS_F_EXT_LEFT | NS_F_EXT_RIGHT)) && al >= 16 && pl_wide_lanes ? 16 : 8;
}

/* ------------------------------------------------------------------ bulk engine */

void pl_ext_engine_free(pl_engine_t *e)
{
	dbuf_free(&e->x_jobs), dbuf_free(&e->x_order), dbuf_free(&e->x_counter), dbuf_free(&e->x_prep);
	dbuf_free(&e->x_ring), dbuf_free(&e->x_nt), dbuf_free(&e->x_aa), dbuf_free(&e->x_ss);
	dbuf_free(&e->x_pssm), dbuf_free(&e->x_res);
	free(e->x_hj), free(e->x_horder);
	e->x_hj = 0, e->x_horder = 0, e->x_m = 0;
}

/* Queue order: by (mode, variant) group, and inside a group by decreasing DP size
 * (longest first for load balance).  Sizes are bucketed on a quarter-octave log
 * scale, which is all the balancing needs, so one counting sort does it. */
#define PL_XBUCKETS (8 * 4 * 64)
static int pl_xbucket(const plk_ext_job_t *J)
{
	const int64_t cells = (int64_t)(J->nl - 2) * J->ncol;
	int lg = 0, frac;
	while (lg < 62 && (cells >> (lg + 1)) > 0) ++lg;
	frac = lg >= 2 ? (int)((cells >> (lg - 2)) & 3) : 0;
	return (J->mode / 2 * 4 + J->variant) * 256 + (255 - (lg * 4 + frac > 255 ? 255 : lg * 4 + frac));
}

/* the reference's answer when the DP has no row (nl < 3): the row loop of
 * nasw-sse.c:361 does not run and the column pick of :448-458 reads the
 * initial -32768 row, end_bonus added at al-1 */
static void pl_ext_norow(int32_t al, int32_t end_bonus, plk_ext_job_t *J)
{
	/* columns 0..al-2 score -32768, column al-1 scores -32768 + end_bonus; first maximum wins */
	if (al == 1 || end_bonus > 0) J->aa_len = al, J->score = -32768 + end_bonus;
	else J->aa_len = 1, J->score = -32768;
	J->nt_len = 0, J->status = 0;
}

static int pl_ext_run(pl_engine_t *e, const ns_opt_t *opt, const pl_ext_job_t *jobs, int32_t n,
		const uint8_t *nt, const uint8_t *aa, const uint8_t *ss, const int8_t *pssm, pl_ext_result_t *res_dev,
		cudaStream_t st)
{
	plk_params_t P;
	int32_t *key = 0;   /* bucket counts, then bucket starts */
	int32_t q, n_dp = 0, max_sub;
	int64_t prep_total = 0, cells_nominal = 0;
	unsigned long long cells_run = 0;
	int ok = 0;

	e->x_last_launches = 0;
	if (n <= 0) return 1;
	if (!pl_params(opt, &P, 1)) return 0;
	if (opt->end_bonus > (1 << 30) || opt->end_bonus < -(1 << 30)) { pl_set_error("end_bonus %d out of range", opt->end_bonus); return 0; }
	if (n > e->x_m) {
		free(e->x_hj), free(e->x_horder);
		e->x_hj = (plk_ext_job_t*)calloc((size_t)n, sizeof(plk_ext_job_t));
		e->x_horder = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
		e->x_m = e->x_hj && e->x_horder ? n : 0;
		if (!e->x_m) { pl_set_error("out of host memory"); return 0; }
	}
	key = (int32_t*)calloc(PL_XBUCKETS + 1, sizeof(int32_t));
	if (!key) { pl_set_error("out of host memory"); return 0; }
	max_sub = pl_max_sub(opt);
	for (q = 0; q < n; ++q) {
		const pl_ext_job_t *x = &jobs[q];
		plk_ext_job_t *J = &e->x_hj[q];
		const int kind = (x->flag & NS_F_EXT_LEFT) ? 1 : (x->flag & NS_F_EXT_RIGHT) ? 0 : 2;
		ns_opt_t o = *opt;
		int32_t width;
		int64_t bound;
		memset(J, 0, sizeof(*J));
		if (x->al < 1) { pl_set_error("job %d: al=%d (the reference needs al >= 1)", q, x->al); goto fail; }
		if (x->pssm_off >= 0 && !pssm) { pl_set_error("job %d: pssm_off set but no pssm buffer", q); goto fail; }
		o.flag = x->flag;
		width = x->width ? x->width : pl_ext_stripe_width(&o, x->al);
		if (width != 8 && width != 16) { pl_set_error("job %d: stripe width %d (8 or 16)", q, width); goto fail; }
		if (kind == 2) width = 8;
		J->nt_off = x->nt_off, J->aa_off = x->aa_off, J->ss_off = ss ? x->ss_off : -1;
		J->pssm_off = x->pssm_off, J->nl = x->nl, J->al = x->al, J->left = kind;
		J->slen = (x->al + width - 1) / width;
		J->ncol = kind == 2 ? x->al : J->slen * width;
		/* upper clamp needed when a value can come within 256 of +32767 (position-specific
		 * scores are bounded by the int8 range) */
		bound = (int64_t)x->al * (x->pssm_off >= 0 ? 127 : max_sub) + opt->end_bonus;
		J->mode = bound + 256 >= 32767 ? 2 : 0;
		J->variant = (x->pssm_off >= 0 ? 1 : 0) |
			(x->al > 16384 || opt->end_bonus < -32768 || opt->end_bonus > 65535 ? 2 : 0);
		J->score = INT32_MIN, J->status = 0;
		if (x->nl < 3) { /* no DP row */
			if (kind == 2) J->nt_len = x->nl, J->aa_len = x->al, J->score = INT32_MIN;
			else pl_ext_norow(x->al, opt->end_bonus, J);
			continue;
		}
		J->prep_off = prep_total, prep_total += plk_prep_bytes(x->nl, x->al);
		cells_nominal += (int64_t)(x->nl - 2) * x->al;
		++key[pl_xbucket(J) + 1];
		++n_dp;
	}
	for (q = 0; q < PL_XBUCKETS; ++q) key[q + 1] += key[q];
	for (q = 0; q < n; ++q)
		if (jobs[q].nl >= 3) e->x_horder[key[pl_xbucket(&e->x_hj[q])]++] = q;
	if (!dbuf_ensure(&e->x_jobs, sizeof(plk_ext_job_t) * (size_t)n) ||
			!dbuf_ensure(&e->x_order, sizeof(int32_t) * (size_t)(n_dp > 0 ? n_dp : 1)) ||
			!dbuf_ensure(&e->x_counter, 64) || !dbuf_ensure(&e->x_prep, (size_t)(prep_total > 0 ? prep_total : 16)))
		goto fail;
	CK(cudaMemcpyAsync(e->x_jobs.p, e->x_hj, sizeof(plk_ext_job_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	CK(cudaMemsetAsync(e->x_counter.p, 0, 64, st));
	if (n_dp > 0) {
		int32_t g0 = 0;
		CK(cudaMemcpyAsync(e->x_order.p, e->x_horder, sizeof(int32_t) * (size_t)n_dp, cudaMemcpyHostToDevice, st));
		e->n_ev = 0;
		PL_TIME(e, st, 0);
		CKK(plk_ext_prep((const plk_ext_job_t*)e->x_jobs.p, n, nt, aa, ss, (uint8_t*)e->x_prep.p, &P, st));
		PL_TIME(e, st, 0);
		++e->x_last_launches;
		while (g0 < n_dp) { /* one launch per (mode, variant) group */
			const plk_ext_job_t *J0 = &e->x_hj[e->x_horder[g0]];
			const int mode = J0->mode, variant = J0->variant;
			int32_t g1 = g0, max_ncol = 1, ctas;
			int64_t stride;
			while (g1 < n_dp && e->x_hj[e->x_horder[g1]].mode == mode && e->x_hj[e->x_horder[g1]].variant == variant) {
				if (e->x_hj[e->x_horder[g1]].ncol > max_ncol) max_ncol = e->x_hj[e->x_horder[g1]].ncol;
				++g1;
			}
			ctas = plk_ext_ctas_per_sm(mode, variant);
			if (ctas < 1) { pl_set_error("extension DP kernel does not fit on an SM"); goto fail; }
			ctas *= e->n_sm;
			if ((int64_t)ctas * plk_ext_warps_per_cta() > g1 - g0) /* at most one warp per request */
				ctas = (g1 - g0 + plk_ext_warps_per_cta() - 1) / plk_ext_warps_per_cta();
			stride = ((int64_t)max_ncol + 1) * PLK_RING_INTS;
			if (!dbuf_ensure(&e->x_ring, sizeof(int32_t) * (size_t)(stride * ctas * plk_ext_warps_per_cta()))) goto fail;
			PL_TIME(e, st, 1);
			CKK(plk_ext_dp((plk_ext_job_t*)e->x_jobs.p, (const int32_t*)e->x_order.p + g0, g1 - g0,
					(int32_t*)e->x_counter.p, (const uint8_t*)e->x_prep.p, pssm, (int32_t*)e->x_ring.p, stride,
					ctas, mode, variant, &P, st));
			PL_TIME(e, st, 1);
			++e->x_last_launches;
			g0 = g1;
		}
	}
	CKK(plk_ext_results((const plk_ext_job_t*)e->x_jobs.p, n, res_dev, st));
	++e->x_last_launches;
	CK(cudaMemcpyAsync(&cells_run, (char*)e->x_counter.p + 8, sizeof(cells_run), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	e->x_cells_run = (int64_t)cells_run, e->x_cells_nominal = cells_nominal;
	if (e->timing && n_dp > 0) { /* event pairs: prep, then one per DP launch */
		int k;
		float ms;
		for (k = 0; k + 1 < e->n_ev; k += 2) {
			cudaEventElapsedTime(&ms, e->ev[k], e->ev[k + 1]);
			e->acc_ms[e->ev_kind[k]] += ms;
		}
		e->acc_dp_launches += e->x_last_launches - 2;
		e->acc_cells += (int64_t)cells_run;
	}
	ok = 1;
fail:
	free(key);
	return ok;
}

PL_EXPORT void pl_ext_last_cells(const pl_engine_t *e, int64_t *cells_run, int64_t *cells_nominal)
{
	if (cells_run) *cells_run = e ? e->x_cells_run : 0;
	if (cells_nominal) *cells_nominal = e ? e->x_cells_nominal : 0;
}

PL_EXPORT int pl_ext_batch_device(pl_engine_t *e, const ns_opt_t *opt, const pl_ext_job_t *jobs, int32_t n,
		const uint8_t *nt, const uint8_t *aa, const uint8_t *ss, const int8_t *pssm, pl_ext_result_t *results_dev,
		void *stream)
{
	if (!e) { pl_set_error("no engine"); return 0; }
	if (cudaSetDevice(e->device) != cudaSuccess) { pl_set_error("cudaSetDevice failed"); return 0; }
	return pl_ext_run(e, opt, jobs, n, nt, aa, ss, pssm, results_dev, stream ? (cudaStream_t)stream : e->stream);
}

PL_EXPORT int pl_ext_batch_host(pl_engine_t *e, const ns_opt_t *opt, const pl_ext_job_t *jobs, int32_t n,
		const uint8_t *nt, int64_t nt_len, const uint8_t *aa, int64_t aa_len, const uint8_t *ss, int64_t ss_len,
		const int8_t *pssm, int64_t pssm_len, pl_ext_result_t *results)
{
	cudaStream_t st;
	int32_t q;
	if (!e) { pl_set_error("no engine"); return 0; }
	if (n <= 0) return 1;
	if (!jobs || !nt || !aa || !results) { pl_set_error("invalid batch arguments"); return 0; }
	for (q = 0; q < n; ++q) { /* every span inside its host buffer: the kernels read exactly these bytes */
		const pl_ext_job_t *x = &jobs[q];
		if (!pl_span_ok("request", q, "nt", x->nt_off, x->nl, nt_len) || !pl_span_ok("request", q, "aa", x->aa_off, x->al, aa_len) ||
				(ss && x->ss_off >= 0 && !pl_span_ok("request", q, "ss", x->ss_off, x->nl, ss_len)) ||
				(x->pssm_off >= 0 && (!pssm || !pl_span_ok("request", q, "pssm", x->pssm_off, (int64_t)x->al * 22, pssm_len))))
			return 0;
	}
	st = e->stream;
	CK(cudaSetDevice(e->device));
	if (!dbuf_ensure(&e->x_nt, (size_t)nt_len) || !dbuf_ensure(&e->x_aa, (size_t)aa_len) ||
			(ss && !dbuf_ensure(&e->x_ss, (size_t)ss_len)) || (pssm && !dbuf_ensure(&e->x_pssm, (size_t)pssm_len)) ||
			!dbuf_ensure(&e->x_res, sizeof(pl_ext_result_t) * (size_t)n))
		return 0;
	if (nt_len > 0) CK(cudaMemcpyAsync(e->x_nt.p, nt, (size_t)nt_len, cudaMemcpyHostToDevice, st));
	if (aa_len > 0) CK(cudaMemcpyAsync(e->x_aa.p, aa, (size_t)aa_len, cudaMemcpyHostToDevice, st));
	if (ss && ss_len > 0) CK(cudaMemcpyAsync(e->x_ss.p, ss, (size_t)ss_len, cudaMemcpyHostToDevice, st));
	if (pssm && pssm_len > 0) CK(cudaMemcpyAsync(e->x_pssm.p, pssm, (size_t)pssm_len, cudaMemcpyHostToDevice, st));
	if (!pl_ext_run(e, opt, jobs, n, (const uint8_t*)e->x_nt.p, (const uint8_t*)e->x_aa.p,
			ss ? (const uint8_t*)e->x_ss.p : 0, pssm ? (const int8_t*)e->x_pssm.p : 0, (pl_ext_result_t*)e->x_res.p, st))
		return 0;
	CK(cudaMemcpyAsync(results, e->x_res.p, sizeof(pl_ext_result_t) * (size_t)n, cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	return 1;
fail:
	return 0;
}

/* ------------------------------------------------------------------ batch object (nasw.h:195-212) */

typedef struct {            /* one option set, tables copied */
	ns_opt_t opt;
	int8_t sc[22 * 22];
	uint8_t nt4[256], aa20[256], codon[64];
} xr_opt_t;

typedef struct {
	const char *ns, *as;
	const uint8_t *ss;
	const int8_t *pssm;
	int32_t nl, al, flag, grp;
	int32_t failed;         /* set by the executor when the device batch of the request failed */
	ns_rst_t rst;
} xr_req_t;

typedef struct xr_gen_s {   /* one flush ("generation") */
	int32_t base, n, n_got, n_grp;
	xr_req_t *req;
	xr_opt_t *grp;          /* distinct option sets of the flush */
	int done;               /* set by the executor under xr_mu */
	struct xr_gen_s *qnext; /* executor queue */
	struct xr_gen_s *gnext; /* the batch object's flushes, oldest first */
} xr_gen_t;

#define XR_MAX_LOST 8
struct ns_ext_batch_s {
	void *km;
	int32_t n, m, next_id;
	int32_t pend_base;      /* id of the first queued request */
	int32_t dropped;        /* a request could not be queued (host memory): the pending set fails at flush */
	int32_t n_lost, lost[XR_MAX_LOST][2];  /* id ranges of flushes that failed before reaching the executor */
	xr_req_t *req;
	ns_opt_t *opts;         /* options of each queued request */
	xr_gen_t *gens;
};

static pthread_mutex_t xr_mu = PTHREAD_MUTEX_INITIALIZER;
static pthread_cond_t xr_cv_work = PTHREAD_COND_INITIALIZER, xr_cv_done = PTHREAD_COND_INITIALIZER;
static xr_gen_t *xr_head, *xr_tail;
static int xr_ready = -1;
static pl_engine_t *xr_engine;
static uint64_t xr_launches, xr_requests, xr_failed;

static void *xr_executor(void *arg);

static int xr_init_device(void)
{
	pthread_t th;
	int dev = 0, count = 0;
	const char *env = getenv("PLGPU_DEVICE");
	pthread_mutex_lock(&xr_mu);
	if (xr_ready >= 0) { const int r = xr_ready; pthread_mutex_unlock(&xr_mu); return r; }
	xr_ready = 0;
	if (env) dev = atoi(env);
	if (cudaGetDeviceCount(&count) != cudaSuccess || dev < 0 || count <= dev) {
		cudaGetLastError();
		pl_set_error("no CUDA device for the extension DP");
		goto out;
	}
	xr_engine = pl_engine_create(dev, 0);
	if (!xr_engine) goto out;
	if (pthread_create(&th, 0, xr_executor, 0) != 0) { pl_set_error("failed to start the extension executor"); goto out; }
	pthread_detach(th);
	xr_ready = 1;
out:
	pthread_mutex_unlock(&xr_mu);
	return xr_ready;
}

PL_EXPORT uint64_t ns_ext_gpu_launch_count(void) { return __sync_fetch_and_add(&xr_launches, 0ull); }
PL_EXPORT uint64_t ns_ext_gpu_request_count(void) { return __sync_fetch_and_add(&xr_requests, 0ull); }
PL_EXPORT uint64_t pl_ext_failed_count(void) { return __sync_fetch_and_add(&xr_failed, 0ull); }

PL_EXPORT ns_ext_batch_t *ns_ext_batch_init(void *km)
{
	ns_ext_batch_t *b;
	if (xr_init_device() != 1) return 0;
	b = (ns_ext_batch_t*)calloc(1, sizeof(*b));
	if (b) b->km = km;
	return b;
}

static void xr_fail(const char *what)
{
	pl_set_error("extension batch: %s", what);
	pl_ns_set_error(pl_last_error());
}

static void *xr_malloc(size_t n) { return pl_fault_hit(PL_FAULT_HOST_ALLOC) ? 0 : malloc(n); }
static void *xr_realloc(void *p, size_t n) { return pl_fault_hit(PL_FAULT_HOST_ALLOC) ? 0 : realloc(p, n); }

PL_EXPORT int32_t ns_ext_batch_add(ns_ext_batch_t *b, const char *ns, int32_t nl, const char *as, int32_t al,
		const ns_opt_t *opt, const uint8_t *ss)
{
	xr_req_t *q;
	if (b->n == 0 && !b->dropped) b->pend_base = b->next_id;
	if (b->dropped) return b->next_id++;  /* the pending set already lost a request: it fails as a whole */
	if (b->n == b->m) {
		const int32_t m = b->m ? b->m << 1 : 16;
		xr_req_t *r = (xr_req_t*)xr_realloc(b->req, sizeof(xr_req_t) * (size_t)m);
		ns_opt_t *o = r ? (ns_opt_t*)xr_realloc(b->opts, sizeof(ns_opt_t) * (size_t)m) : 0;
		if (r) b->req = r;
		if (o) b->opts = o;
		if (!r || !o) {
			xr_fail("out of host memory queueing a request");
			b->dropped = 1;
			return b->next_id++;
		}
		b->m = m;
	}
	q = &b->req[b->n];
	memset(q, 0, sizeof(*q));
	q->ns = ns, q->nl = nl, q->as = as, q->al = al, q->ss = ss, q->pssm = opt->pssm;
	q->flag = opt->flag & (NS_F_EXT_LEFT | NS_F_EXT_RIGHT);
	q->rst.nt_len = nl, q->rst.aa_len = al, q->rst.score = INT32_MIN; /* nasw-sse.c:244 */
	b->opts[b->n] = *opt;
	++b->n;
	return b->next_id++;
}

static int xr_same_opt(const ns_opt_t *a, const ns_opt_t *b)
{ /* every option the DP reads; tables by content */
	return a->go == b->go && a->ge == b->ge && a->io == b->io && a->fs == b->fs && a->xdrop == b->xdrop &&
		a->end_bonus == b->end_bonus && a->asize == b->asize && a->ie_coef == b->ie_coef &&
		a->sp_null_bonus == b->sp_null_bonus && memcmp(a->sp, b->sp, sizeof(a->sp)) == 0 &&
		(a->sc == b->sc || memcmp(a->sc, b->sc, 22 * 22) == 0) &&
		(a->nt4 == b->nt4 || memcmp(a->nt4, b->nt4, 256) == 0) &&
		(a->aa20 == b->aa20 || memcmp(a->aa20, b->aa20, 256) == 0) &&
		(a->codon == b->codon || memcmp(a->codon, b->codon, 64) == 0);
}

static void xr_opt_copy(xr_opt_t *d, const ns_opt_t *o)
{
	d->opt = *o;
	memcpy(d->sc, o->sc, 22 * 22), memcpy(d->nt4, o->nt4, 256), memcpy(d->aa20, o->aa20, 256), memcpy(d->codon, o->codon, 64);
	d->opt.sc = d->sc, d->opt.nt4 = d->nt4, d->opt.aa20 = d->aa20, d->opt.codon = d->codon;
	d->opt.pssm = 0, d->opt.flag = 0;
}

static int xr_released(xr_gen_t *g)
{
	int d;
	pthread_mutex_lock(&xr_mu);
	d = g->done;
	pthread_mutex_unlock(&xr_mu);
	return d;
}

/* drop flushes whose results have all been read */
static void xr_reap(ns_ext_batch_t *b)
{
	xr_gen_t **p = &b->gens;
	while (*p) {
		xr_gen_t *g = *p;
		if (g->n_got >= g->n && xr_released(g)) *p = g->gnext, free(g->req), free(g->grp), free(g);
		else p = &g->gnext;
	}
}

/* the pending requests can not reach the device: their ids are recorded as failed */
static int32_t xr_lose_pending(ns_ext_batch_t *b)
{
	if (b->n_lost < XR_MAX_LOST) {
		b->lost[b->n_lost][0] = b->pend_base, b->lost[b->n_lost][1] = b->next_id, ++b->n_lost;
	} else { /* fold into the last range: ids between belong to flushes found first by xr_find */
		b->lost[XR_MAX_LOST - 1][1] = b->next_id;
	}
	free(b->req), free(b->opts);
	b->req = 0, b->opts = 0, b->n = b->m = 0, b->dropped = 0;
	return 0;
}

static int xr_is_lost(const ns_ext_batch_t *b, int32_t id)
{
	int32_t k;
	for (k = 0; k < b->n_lost; ++k)
		if (id >= b->lost[k][0] && id < b->lost[k][1]) return 1;
	return 0;
}

PL_EXPORT int32_t ns_ext_batch_flush(ns_ext_batch_t *b)
{
	xr_gen_t *g;
	int32_t k, n;
	if (!b) return 0;
	xr_reap(b);
	if (b->dropped) return xr_lose_pending(b);
	if (b->n == 0) return 0;
	g = (xr_gen_t*)xr_malloc(sizeof(*g));
	if (g) memset(g, 0, sizeof(*g));
	if (g) g->grp = (xr_opt_t*)xr_malloc(sizeof(xr_opt_t) * (size_t)b->n);
	if (!g || !g->grp) {
		free(g);
		xr_fail("out of host memory at flush");
		return xr_lose_pending(b);
	}
	g->base = b->next_id - b->n, g->n = n = b->n;
	g->req = b->req, b->req = 0;
	for (k = 0; k < n; ++k) { /* distinct option sets */
		int32_t t;
		for (t = 0; t < g->n_grp; ++t) if (xr_same_opt(&g->grp[t].opt, &b->opts[k])) break;
		if (t == g->n_grp) xr_opt_copy(&g->grp[g->n_grp++], &b->opts[k]);
		g->req[k].grp = t;
	}
	b->n = b->m = 0;
	free(b->opts), b->opts = 0;
	{ /* counted when handed to the device, as nasw-ext-gpu.c:994 does; nl < 3 has no DP row */
		uint64_t nd = 0;
		for (k = 0; k < n; ++k) nd += g->req[k].nl >= 3;
		__sync_fetch_and_add(&xr_requests, nd);
	}
	if (b->gens) { xr_gen_t *t = b->gens; while (t->gnext) t = t->gnext; t->gnext = g; }
	else b->gens = g;
	pthread_mutex_lock(&xr_mu);
	if (xr_tail) xr_tail->qnext = g; else xr_head = g;
	xr_tail = g;
	pthread_cond_broadcast(&xr_cv_work);
	pthread_mutex_unlock(&xr_mu);
	return n;
}

static xr_gen_t *xr_find(const ns_ext_batch_t *b, int32_t id)
{
	xr_gen_t *g;
	for (g = b->gens; g; g = g->gnext)
		if (id >= g->base && id < g->base + g->n) return g;
	return 0;
}

PL_EXPORT int ns_ext_batch_ready(ns_ext_batch_t *b, int32_t id)
{
	xr_gen_t *g = b ? xr_find(b, id) : 0;
	if (!g) return b && xr_is_lost(b, id);
	return xr_released(g);
}

PL_EXPORT void ns_ext_batch_wait(ns_ext_batch_t *b)
{
	if (!b) return;
	pthread_mutex_lock(&xr_mu);
	for (;;) {
		int in_flight = 0, fresh = 0;
		xr_gen_t *g;
		for (g = b->gens; g; g = g->gnext) {
			if (g->n_got >= g->n) continue;
			if (g->done) fresh = 1;
			else in_flight = 1;
		}
		if (fresh || !in_flight) break;
		pthread_cond_wait(&xr_cv_done, &xr_mu);
	}
	pthread_mutex_unlock(&xr_mu);
}

PL_EXPORT const ns_rst_t *ns_ext_batch_get(ns_ext_batch_t *b, int32_t id)
{
	xr_gen_t *g = b ? xr_find(b, id) : 0;
	if (!g) return 0;  /* unknown id, or a flush that failed before reaching the device */
	pthread_mutex_lock(&xr_mu);
	while (!g->done) pthread_cond_wait(&xr_cv_done, &xr_mu);
	pthread_mutex_unlock(&xr_mu);
	++g->n_got;
	return g->req[id - g->base].failed ? 0 : &g->req[id - g->base].rst;
}

PL_EXPORT void ns_ext_batch_destroy(ns_ext_batch_t *b)
{
	xr_gen_t *g;
	if (!b) return;
	pthread_mutex_lock(&xr_mu); /* the executor may still hold submitted flushes */
	for (g = b->gens; g; g = g->gnext)
		while (!g->done) pthread_cond_wait(&xr_cv_done, &xr_mu);
	pthread_mutex_unlock(&xr_mu);
	while (b->gens) {
		g = b->gens, b->gens = g->gnext;
		free(g->req), free(g->grp), free(g);
	}
	free(b->req), free(b->opts), free(b);
}

/* ------------------------------------------------------------------ executor */

typedef struct { xr_gen_t *g; int32_t k; } xr_ref_t;

/* one device batch: every request of `refs` shares the options `o` */
static int xr_run(const ns_opt_t *o, const xr_ref_t *refs, int32_t n)
{
	pl_ext_job_t *jobs = (pl_ext_job_t*)malloc(sizeof(pl_ext_job_t) * (size_t)n);
	pl_ext_result_t *res = (pl_ext_result_t*)malloc(sizeof(pl_ext_result_t) * (size_t)n);
	int64_t l_nt = 0, l_aa = 0, l_ss = 0, l_ps = 0, p_nt = 0, p_aa = 0, p_ss = 0, p_ps = 0;
	uint8_t *nt = 0, *aa = 0, *ss = 0;
	int8_t *ps = 0;
	int32_t q;
	int ok = 0;
	if (!jobs || !res) goto out;
	for (q = 0; q < n; ++q) {
		const xr_req_t *r = &refs[q].g->req[refs[q].k];
		l_nt += r->nl, l_aa += r->al;
		if (r->ss) l_ss += r->nl;
		if (r->pssm) l_ps += (int64_t)r->al * 22;
	}
	nt = (uint8_t*)malloc((size_t)l_nt + 1), aa = (uint8_t*)malloc((size_t)l_aa + 1);
	ss = l_ss ? (uint8_t*)malloc((size_t)l_ss) : 0, ps = l_ps ? (int8_t*)malloc((size_t)l_ps) : 0;
	if (!nt || !aa || (l_ss && !ss) || (l_ps && !ps)) goto out;
	for (q = 0; q < n; ++q) {
		const xr_req_t *r = &refs[q].g->req[refs[q].k];
		pl_ext_job_t *x = &jobs[q];
		memcpy(nt + p_nt, r->ns, (size_t)r->nl), memcpy(aa + p_aa, r->as, (size_t)r->al);
		x->nt_off = p_nt, x->aa_off = p_aa, x->ss_off = -1, x->pssm_off = -1;
		x->nl = r->nl, x->al = r->al, x->flag = r->flag, x->width = 0;
		p_nt += r->nl, p_aa += r->al;
		if (r->ss) memcpy(ss + p_ss, r->ss, (size_t)r->nl), x->ss_off = p_ss, p_ss += r->nl;
		if (r->pssm) memcpy(ps + p_ps, r->pssm, (size_t)r->al * 22), x->pssm_off = p_ps, p_ps += (int64_t)r->al * 22;
	}
	ok = !pl_fault_hit(PL_FAULT_EXT_BATCH);
	if (!ok) pl_set_error("extension DP batch failed (injected)");
	else ok = pl_ext_batch_host(xr_engine, o, jobs, n, nt, l_nt, aa, l_aa, ss, l_ss, ps, l_ps, res);
	if (ok) {
		for (q = 0; q < n; ++q) {
			xr_req_t *r = &refs[q].g->req[refs[q].k];
			if (res[q].status != 0) { ok = 0; pl_set_error("extension request failed on the device"); break; }
			r->rst.n_cigar = 0, r->rst.nt_len = res[q].nt_len, r->rst.aa_len = res[q].aa_len, r->rst.score = res[q].score;
		}
		__sync_fetch_and_add(&xr_launches, (uint64_t)xr_engine->x_last_launches);
	}
out:
	if (!ok) { /* no CPU path to fall back on: every request of the batch reports failure */
		char msg[1100];
		snprintf(msg, sizeof(msg), "extension DP batch of %d requests failed: %s", n, pl_last_error());
		pl_set_error("%s", msg);
		pl_ns_set_error(msg);
		for (q = 0; q < n; ++q) refs[q].g->req[refs[q].k].failed = 1;
		__sync_fetch_and_add(&xr_failed, (uint64_t)n);
	}
	free(jobs), free(res), free(nt), free(aa), free(ss), free(ps);
	return ok;
}

static void *xr_executor(void *arg)
{
	(void)arg;
	cudaSetDevice(xr_engine->device);
	for (;;) {
		xr_gen_t *list, *g;
		xr_ref_t *refs;
		int32_t total = 0, n, k;
		pthread_mutex_lock(&xr_mu);
		while (!xr_head) pthread_cond_wait(&xr_cv_work, &xr_mu);
		list = xr_head, xr_head = xr_tail = 0;
		pthread_mutex_unlock(&xr_mu);
		for (g = list; g; g = g->qnext) total += g->n;
		refs = (xr_ref_t*)xr_malloc(sizeof(xr_ref_t) * (size_t)(total > 0 ? total : 1));
		if (!refs) { /* every request of these flushes fails */
			xr_fail("out of host memory in the executor");
			for (g = list; g; g = g->qnext)
				for (k = 0; k < g->n; ++k) g->req[k].failed = 1;
			__sync_fetch_and_add(&xr_failed, (uint64_t)total);
		}
		/* every waiting flush, grouped by option set across flushes: one device batch per set */
		for (g = refs ? list : 0; g; g = g->qnext) {
			int32_t t;
			for (t = 0; t < g->n_grp; ++t) {
				const ns_opt_t *o = &g->grp[t].opt;
				xr_gen_t *h;
				int32_t u, dup = 0;
				/* skip sets already run from an earlier flush of this list */
				for (h = list; h != g && !dup; h = h->qnext)
					for (u = 0; u < h->n_grp && !dup; ++u) dup = xr_same_opt(&h->grp[u].opt, o);
				for (u = 0; u < t && !dup; ++u) dup = xr_same_opt(&g->grp[u].opt, o);
				if (dup) continue;
				n = 0;
				for (h = g; h; h = h->qnext)
					for (k = 0; k < h->n; ++k)
						if (xr_same_opt(&h->grp[h->req[k].grp].opt, o)) refs[n].g = h, refs[n].k = k, ++n;
				xr_run(o, refs, n);
			}
		}
		free(refs);
		pthread_mutex_lock(&xr_mu);
		for (g = list; g; g = g->qnext) g->done = 1;
		pthread_cond_broadcast(&xr_cv_done);
		pthread_mutex_unlock(&xr_mu);
	}
	return 0;
}
