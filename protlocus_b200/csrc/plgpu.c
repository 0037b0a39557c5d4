/*
 * plgpu.c -- host layer of libplgpu (C99 + the CUDA runtime C API).
 *
 * Two ways in:
 *   - the bulk engine (pl_engine_*, pl_splice_batch_*): plans a whole batch of
 *     global spliced DPs, runs prep -> DP -> traceback -> compaction on one
 *     stream and returns scores and CIGARs;
 *   - the reference's request queue API (ns_gpu_init/submit/wait/global and
 *     counters, nasw.h:140-152, replacing nasw-cuda.cu:407-1145): submitted
 *     requests are collected by one executor thread into batches of at most
 *     128 (NS_GPU_MAX_BATCH of the reference) and run through an engine.
 *
 * Planning of a batch:
 *   1. width per job with ns_global_gs_auto's rule (nasw-sse.c:987-996):
 *      al*max(sc)+end_bonus > 30000 -> the 32-bit kernel semantics;
 *   2. jobs are distributed over "waves" whose traceback arenas fit the trace
 *      budget, by longest-processing-time bin packing so every wave gets a mix
 *      of large and small jobs;
 *   3. in each wave, jobs whose cell count is large compared with the per-warp
 *      share are run by a whole CTA (a 256-lane wavefront), the rest by one
 *      warp each; both queues are sorted by decreasing size.
 * There is no CPU fallback: failures are reported as errors.
 */
#define _POSIX_C_SOURCE 200809L
#include <errno.h>
#include <limits.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <cuda_runtime_api.h>
#include "plk.h"
#include "../../include/plgpu.h"
#include "plhost.h"


/* ------------------------------------------------------------------ km allocator hooks
 * The CIGAR of a request is appended into the caller's kalloc arena, as
 * nasw.h:219-229 does.  kalloc belongs to the host program (kalloc.c of the
 * reference); the library only holds a weak reference to krealloc, so the
 * linker exports the program's definition to it.  Callers that link no kalloc
 * (Python, tests) must pass km == NULL and get plain realloc. */
extern void *krealloc(void *km, void *ptr, size_t size) __attribute__((weak));

/* NULL (with the error text set) when the allocation fails or a km arena is passed by a
 * program that links no kalloc; the old block then stays valid */
static void *pl_krealloc(void *km, void *ptr, size_t size)
{
	void *q;
	if (pl_fault_hit(PL_FAULT_HOST_ALLOC)) q = 0;
	else if (krealloc) q = krealloc(km, ptr, size);
	else if (km) {
		pl_set_error("a km arena was passed but the program links no kalloc");
		return 0;
	} else q = realloc(ptr, size);
	if (!q) pl_set_error("out of host memory for a CIGAR of %zu bytes", size);
	return q;
}

/* ------------------------------------------------------------------ host-side fault injection (tests) */

static int32_t pl_fault_after[PL_FAULT_N];
static pthread_mutex_t pl_fault_mu = PTHREAD_MUTEX_INITIALIZER;

int pl_fault_hit(int site)
{
	int hit = 0;
	if (site < 0 || site >= PL_FAULT_N || __atomic_load_n(&pl_fault_after[site], __ATOMIC_RELAXED) <= 0) return 0;
	pthread_mutex_lock(&pl_fault_mu);
	if (pl_fault_after[site] > 0 && --pl_fault_after[site] == 0) hit = 1, pl_fault_after[site] = 0;
	pthread_mutex_unlock(&pl_fault_mu);
	return hit;
}

int pl_span_ok(const char *rec, int32_t q, const char *buf, int64_t off, int64_t len, int64_t cap)
{
	if (off < 0 || len < 0 || off > cap || len > cap - off) {
		pl_set_error("%s %d: %s span [%lld, +%lld) outside the %lld-byte buffer", rec, q, buf, (long long)off,
				(long long)len, (long long)cap);
		return 0;
	}
	return 1;
}

PL_EXPORT int pl_debug_fault(int32_t site, int32_t after)
{
	if (site < 0 || site >= PL_FAULT_N) return 0;
	pthread_mutex_lock(&pl_fault_mu);
	pl_fault_after[site] = after < 0 ? 0 : after + 1;
	pthread_mutex_unlock(&pl_fault_mu);
	return 1;
}

/* ------------------------------------------------------------------ errors */

static pthread_mutex_t pl_err_mu = PTHREAD_MUTEX_INITIALIZER;
static char pl_err[1024] = "none";

void pl_set_error(const char *fmt, ...)
{
	va_list ap;
	pthread_mutex_lock(&pl_err_mu);
	va_start(ap, fmt);
	vsnprintf(pl_err, sizeof(pl_err), fmt, ap);
	va_end(ap);
	pthread_mutex_unlock(&pl_err_mu);
}

PL_EXPORT const char *pl_last_error(void) { return pl_err; }

/* ------------------------------------------------------------------ buffers */

int dbuf_ensure(dbuf_t *b, size_t need)
{
	if (need == 0) need = 16;
	if (b->cap >= need) return 1;
	if (b->p) cudaFree(b->p);
	b->p = 0, b->cap = 0;
	if (pl_fault_hit(PL_FAULT_DEV_ALLOC)) {
		pl_set_error("cudaMalloc of %zu bytes failed (injected)", need);
		return 0;
	}
	if (cudaMalloc(&b->p, need) != cudaSuccess) {
		cudaGetLastError();
		pl_set_error("cudaMalloc of %zu bytes failed", need);
		return 0;
	}
	b->cap = need;
	return 1;
}

void dbuf_free(dbuf_t *b) { if (b->p) cudaFree(b->p); b->p = 0, b->cap = 0; }

PL_EXPORT uint64_t pl_kernel_launch_count(void) { return plk_launches(); }

PL_EXPORT pl_engine_t *pl_engine_create(int32_t device, int64_t trace_budget_bytes)
{
	pl_engine_t *e = (pl_engine_t*)calloc(1, sizeof(*e));
	size_t free_b = 0, total_b = 0;
	int m;
	if (!e) { pl_set_error("out of host memory"); return 0; }
	e->device = device;
	CK(cudaSetDevice(device));
	CK(cudaDeviceGetAttribute(&e->n_sm, cudaDevAttrMultiProcessorCount, device));
	for (m = 0; m < 4; ++m) {
		int r;
		for (r = 0; r < 2; ++r) {
			e->ctas_per_sm[m][r] = plk_dp_ctas_per_sm(m, r == 0 ? 8 : 4);
			if (e->ctas_per_sm[m][r] < 1) { pl_set_error("DP kernel does not fit on an SM (mode %d)", m); goto fail; }
		}
	}
	e->coop_ratio = pl_coop_ratio();
	e->r4_rows = pl_r4_rows();
	{
		const char *v = getenv("PLGPU_PAIR"), *g = getenv("PLGPU_GRAPHS");
		e->pairing = !(v && *v && atoi(v) == 0);
		e->graphs = !(g && *g && atoi(g) == 0);
	}
	CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
	CK(cudaStreamCreateWithFlags(&e->side, cudaStreamNonBlocking));
	CK(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
	CK(cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming));
	CK(cudaMemGetInfo(&free_b, &total_b));
	if (trace_budget_bytes <= 0) { /* default: 40% of free memory, at most 72 GB */
		trace_budget_bytes = (int64_t)(free_b * 0.4);
		if (trace_budget_bytes > (72LL << 30)) trace_budget_bytes = 72LL << 30;
	}
	e->trace_budget = trace_budget_bytes;
	return e;
fail:
	if (e->stream) cudaStreamDestroy(e->stream);
	if (e->side) cudaStreamDestroy(e->side);
	if (e->ev_fork) cudaEventDestroy(e->ev_fork);
	if (e->ev_join) cudaEventDestroy(e->ev_join);
	free(e);
	return 0;
}

PL_EXPORT void pl_engine_destroy(pl_engine_t *e)
{
	if (!e) return;
	cudaSetDevice(e->device);
	if (e->g_exec) cudaGraphExecDestroy(e->g_exec);
	dbuf_free(&e->jobs), dbuf_free(&e->order), dbuf_free(&e->counters), dbuf_free(&e->prep);
	dbuf_free(&e->trace), dbuf_free(&e->ring), dbuf_free(&e->tmp), dbuf_free(&e->total);
	dbuf_free(&e->nt), dbuf_free(&e->aa), dbuf_free(&e->ss), dbuf_free(&e->res), dbuf_free(&e->cig);
	pl_ext_engine_free(e);
	pl_hmm_engine_free(e);
	pl_gapless_engine_free(e);
	pl_rc_engine_free(e);
	pl_pf_engine_free(e);
	pl_feat_engine_free(e);
	pl_ps_engine_free(e);
	pl_chain_engine_free(e);
	pl_seed_engine_free(e);
	if (e->stream) cudaStreamDestroy(e->stream);
	if (e->side) cudaStreamDestroy(e->side);
	if (e->ev_fork) cudaEventDestroy(e->ev_fork);
	if (e->ev_join) cudaEventDestroy(e->ev_join);
	free(e->hj), free(e->horder), free(e->hwave);
	free(e);
}

PL_EXPORT int pl_engine_set_timing(pl_engine_t *e, int32_t enable)
{
	int k;
	if (!e) return 0;
	if (enable && !e->timing) {
		if (cudaSetDevice(e->device) != cudaSuccess) return 0;
		for (k = 0; k < (int)(sizeof(e->ev) / sizeof(e->ev[0])); ++k)
			if (cudaEventCreate(&e->ev[k]) != cudaSuccess) { pl_set_error("cudaEventCreate failed"); return 0; }
	}
	e->timing = enable ? 1 : e->timing;
	memset(e->acc_ms, 0, sizeof(e->acc_ms));
	e->acc_dp_launches = e->acc_cells = 0;
	return 1;
}

PL_EXPORT void pl_engine_times(const pl_engine_t *e, double *prep_ms, double *dp_ms, double *traceback_ms,
		double *compact_ms, int64_t *dp_launches, int64_t *cells)
{
	if (prep_ms) *prep_ms = e->acc_ms[0];
	if (dp_ms) *dp_ms = e->acc_ms[1];
	if (traceback_ms) *traceback_ms = e->acc_ms[2];
	if (compact_ms) *compact_ms = e->acc_ms[3];
	if (dp_launches) *dp_launches = e->acc_dp_launches;
	if (cells) *cells = e->acc_cells;
}

PL_EXPORT void *pl_engine_stream(const pl_engine_t *e) { return e ? (void*)e->stream : 0; }

PL_EXPORT void pl_engine_last_plan(const pl_engine_t *e, int32_t *n_waves, int32_t *n_coop, int32_t *n_dp_launches)
{
	if (n_waves) *n_waves = e->last_waves;
	if (n_coop) *n_coop = e->last_coop;
	if (n_dp_launches) *n_dp_launches = e->last_dp_launches;
}

/* ------------------------------------------------------------------ planning */

int pl_params(const ns_opt_t *opt, plk_params_t *p, int for_ext)
{
	int i;
	if (!opt || !opt->sc || !opt->nt4 || !opt->aa20 || !opt->codon) { pl_set_error("incomplete ns_opt_t"); return 0; }
	if (opt->asize != 22) { pl_set_error("asize %d unsupported (22 only)", opt->asize); return 0; }
	if (!for_ext && opt->pssm) { pl_set_error("position-specific scores are CPU-only in the reference's global path (nasw.h:73)"); return 0; }
	if (!for_ext && (opt->flag & (NS_F_EXT_LEFT | NS_F_EXT_RIGHT))) { pl_set_error("extension DPs go through the ext entry points, not the global path"); return 0; }
	memset(p, 0, sizeof(*p));
	p->go = opt->go, p->ge = opt->ge, p->io = opt->io, p->fs = opt->fs;
	p->end_bonus = opt->end_bonus, p->xdrop = opt->xdrop;
	for (i = 0; i < 6; ++i) p->sp[i] = opt->sp[i];
	p->sp_null_bonus = opt->sp_null_bonus, p->ie_coef = opt->ie_coef;
	memcpy(p->sc, opt->sc, 22 * 22);
	memcpy(p->nt4, opt->nt4, 256), memcpy(p->aa20, opt->aa20, 256), memcpy(p->codon, opt->codon, 64);
	p->aa_x = opt->aa20['X'];
	plk_fill_scaled(p);
	return 1;
}

int pl_max_sub(const ns_opt_t *opt)
{
	int i, m = 0;
	for (i = 0; i < opt->asize * opt->asize; ++i) if (m < opt->sc[i]) m = opt->sc[i];
	return m;
}

/* A job runs on a whole CTA (a 2048-row cooperative wavefront) when it holds more
 * than this multiple of a warp's share of its wave's cells: fewer, longer jobs then
 * finish with the rest instead of trailing them.  PLGPU_COOP_RATIO overrides it
 * (the tuning sweep of the batched workload). */
static double g_coop_ratio = 0.7;
static pthread_once_t g_coop_once = PTHREAD_ONCE_INIT;
static void pl_coop_ratio_init(void)
{
	const char *v = getenv("PLGPU_COOP_RATIO");
	if (v && *v) {
		const double x = atof(v);
		if (x > 0.0) g_coop_ratio = x;
	}
}
double pl_coop_ratio(void)
{
	pthread_once(&g_coop_once, pl_coop_ratio_init);
	return g_coop_ratio;
}

/* Jobs with at most this many DP rows (nl - 2) run with 4 rows per lane (80 registers,
 * three CTAs per SM), the rest with 8 (128 registers, two CTAs per SM): 4 pays on
 * short windows, 8 on long ones.  PLGPU_R4_ROWS overrides the default; the engine's
 * autotuner (pl_engine_autotune) picks it for a workload. */
static int32_t g_r4_rows = 0;
static pthread_once_t g_r4_once = PTHREAD_ONCE_INIT;
static void pl_r4_rows_init(void)
{
	const char *v = getenv("PLGPU_R4_ROWS");
	if (v && *v) g_r4_rows = atoi(v);
}
int32_t pl_r4_rows(void)
{
	pthread_once(&g_r4_once, pl_r4_rows_init);
	return g_r4_rows;
}

typedef struct { int64_t cells; int32_t idx; } pl_key_t;
static int pl_cmp_cells_desc(const void *a, const void *b)
{
	const pl_key_t *x = (const pl_key_t*)a, *y = (const pl_key_t*)b;
	if (x->cells != y->cells) return x->cells > y->cells ? -1 : 1;
	return x->idx - y->idx;
}

static int pl_max_ctas(const pl_engine_t *e)
{
	int m, r, c = 0;
	for (m = 0; m < 4; ++m)
		for (r = 0; r < 2; ++r) if (e->ctas_per_sm[m][r] > c) c = e->ctas_per_sm[m][r];
	return c;
}

static int pl_grow_host(pl_engine_t *e, int32_t n)
{
	if (n <= e->m_jobs) return 1;
	free(e->hj), free(e->horder), free(e->hwave);
	e->hj = (plk_job_t*)calloc((size_t)n, sizeof(plk_job_t));
	e->horder = (int32_t*)malloc(sizeof(int32_t) * (size_t)n * 2);
	e->hwave = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
	if (!e->hj || !e->horder || !e->hwave) { pl_set_error("out of host memory"); e->m_jobs = 0; return 0; }
	e->m_jobs = n;
	return 1;
}

/* length of the union of intervals [a[i], b[i]) (sorted in place by start) */
static double pl_union_ms(double *a, double *b, int n)
{
	int i, j;
	double tot = 0, lo, hi;
	for (i = 1; i < n; ++i) /* insertion sort by start */
		for (j = i; j > 0 && a[j - 1] > a[j]; --j) {
			double t = a[j]; a[j] = a[j - 1], a[j - 1] = t;
			t = b[j], b[j] = b[j - 1], b[j - 1] = t;
		}
	for (i = 0; i < n; i = j) {
		lo = a[i], hi = b[i];
		for (j = i + 1; j < n && a[j] <= hi; ++j) if (b[j] > hi) hi = b[j];
		tot += hi - lo;
	}
	return tot;
}

/* The paired int16x2 DP (mode 3) keeps values v + B in 15 bits per half with the
 * saturation floor at F.  Its admission bound, from the recurrences: a real H value
 * is at least the cost of one path to it (the diagonal out of column -1 at row 2,
 * insertions along row 2, one intron down the column: s_min - go - ge*al - io -
 * 256), every state derived from H values is at most two penalised steps below
 * (P1 = go + ge + io + fs + 256 each), and no value exceeds al*max(sc) + 256.  A
 * job of protein length al is admitted when [low bound, high bound] fits between
 * F + 512 and 0x7fff - 512 after biasing; every penalty stays below F so that the
 * floor never wraps under a subtraction. */
#define PL_PAIR_F 512
static int pl_pair_limits(const ns_opt_t *opt, int max_sub, int32_t *al_cap, int32_t *bias)
{
	int i, s_min = 0;
	int64_t c_low, per_al, cap;
	if (opt->go + opt->ge > 256 || opt->io > 256 || opt->fs > 256 || opt->go < 0 || opt->ge < 0 || opt->io < 0 ||
			opt->fs < 0 || opt->asize != 22)
		return 0;
	for (i = 0; i < 22 * 22; ++i) if (opt->sc[i] < s_min) s_min = opt->sc[i];
	c_low = -s_min + opt->go + opt->io + 256 + 2 * (opt->go + opt->ge + opt->io + opt->fs + 256);
	per_al = opt->ge + (max_sub > 0 ? max_sub : 0);
	cap = (32767 - PL_PAIR_F - 512 - 512 - 256 - c_low) / (per_al > 0 ? per_al : 1);
	if (cap < 1) return 0;
	*al_cap = cap > 65535 ? 65535 : (int32_t)cap;
	*bias = (int32_t)(PL_PAIR_F + 512 + c_low + (int64_t)opt->ge * *al_cap);
	return 1;
}

/* launch group of a job: its mode, with the second jobs of pairs in group 4 */
static int pl_group_of(const plk_job_t *J) { return J->mode == 3 && J->pair < 0 ? 4 : J->mode; }

typedef struct { int64_t aa_off; int32_t al, nl, idx; } pl_pkey_t;
static int pl_cmp_pair(const void *a, const void *b)
{
	const pl_pkey_t *x = (const pl_pkey_t*)a, *y = (const pl_pkey_t*)b;
	if (x->aa_off != y->aa_off) return x->aa_off < y->aa_off ? -1 : 1;
	if (x->al != y->al) return x->al - y->al;
	if (x->nl != y->nl) return x->nl - y->nl;
	return x->idx - y->idx;
}

/* A pair runs as one unit of work: one step of a pair costs about 1.7 steps of a single
 * job and does two jobs' cells.  While a batch's units fill the GPU that is a gain;
 * a batch with fewer units than the DP launch has warps would only make its units
 * longer.  So pairs are formed only when there are at least PLGPU_PAIR_MIN (default 1)
 * times as many of them as warps of a launch -- for every eligible job or none, since a
 * single job and a pair run in different launches, one after the other.  pairing = 2
 * pairs every eligible job. */
static double g_pair_min = 1.0;
static pthread_once_t g_pair_min_once = PTHREAD_ONCE_INIT;
static void pl_pair_min_init(void)
{
	const char *v = getenv("PLGPU_PAIR_MIN");
	if (v && *v) {
		const double x = atof(v);
		if (x >= 0.0) g_pair_min = x;
	}
}

/* Pairs of 16-bit jobs with one protein (the same aa_off) and one window length run as
 * mode 3; returns the number of pairs formed (0 on a host allocation failure too). */
static int32_t pl_form_pairs(pl_engine_t *e, const ns_opt_t *opt, int32_t n, int max_sub, plk_params_t *P)
{
	pl_pkey_t *key;
	int32_t q, m = 0, n_pairs = 0, al_cap = 0, bias = 0;
	if (!e->pairing || n < 2 || !pl_pair_limits(opt, max_sub, &al_cap, &bias)) return 0;
	key = (pl_pkey_t*)malloc(sizeof(*key) * (size_t)n);
	if (!key) return 0;
	for (q = 0; q < n; ++q) {
		const plk_job_t *J = &e->hj[q];
		if (J->mode != 0 || J->al > al_cap) continue;
		key[m].aa_off = J->aa_off, key[m].al = J->al, key[m].nl = J->nl, key[m].idx = q, ++m;
	}
	qsort(key, (size_t)m, sizeof(*key), pl_cmp_pair);
	for (q = 0; q + 1 < m; ++q) {
		if (key[q].aa_off != key[q + 1].aa_off || key[q].al != key[q + 1].al || key[q].nl != key[q + 1].nl) continue;
		/* a pair shares one wave: both traces must fit the budget together */
		if (2 * plk_trace_words(key[q].nl, key[q].al, PLK_WARPS_PER_CTA, e->hj[key[q].idx].rows) * 2 > e->trace_budget)
			continue;
		{
			plk_job_t *A = &e->hj[key[q].idx], *B = &e->hj[key[q + 1].idx];
			A->mode = B->mode = 3;
			A->pair = key[q + 1].idx, B->pair = -1;
			++n_pairs, ++q;
		}
	}
	free(key);
	pthread_once(&g_pair_min_once, pl_pair_min_init);
	if (e->pairing == 1 && n_pairs > 0 &&
			(double)n_pairs < g_pair_min * e->n_sm * e->ctas_per_sm[3][0] * PLK_WARPS_PER_CTA) {
		for (q = 0; q < n; ++q)  /* too few to fill the GPU: every job single */
			if (e->hj[q].mode == 3) e->hj[q].mode = 0, e->hj[q].pair = 0;
		return 0;
	}
	P->pair_b = bias, P->pair_f = PL_PAIR_F;
	return n_pairs;
}

/* FNV-1a of the launch sequence's shape: sizes, buffers, parameters and, per position of
 * the order array, the wave / launch group / rows / cooperative flag of its job */
static uint64_t pl_fnv(uint64_t h, const void *p, size_t n)
{
	const unsigned char *b = (const unsigned char*)p;
	size_t i;
	for (i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
	return h;
}

static int pl_group_of(const plk_job_t *J);

static uint64_t pl_plan_key(const pl_engine_t *e, int32_t n, int32_t n_waves, int32_t two, int64_t arena_words,
		int64_t ring_ints, int32_t max_al, const void *nt, const void *aa, const void *ss, const void *res,
		const void *cig, int64_t cig_cap, cudaStream_t st, const plk_params_t *P)
{
	uint64_t h = 1469598103934665603ull;
	const void *ptr[14];
	int64_t v[7];
	int32_t i;
	v[0] = n, v[1] = n_waves, v[2] = two, v[3] = arena_words, v[4] = ring_ints, v[5] = max_al, v[6] = cig_cap;
	ptr[0] = nt, ptr[1] = aa, ptr[2] = ss, ptr[3] = res, ptr[4] = cig, ptr[5] = (const void*)st, ptr[6] = e->jobs.p;
	ptr[7] = e->order.p, ptr[8] = e->counters.p, ptr[9] = e->prep.p, ptr[10] = e->trace.p, ptr[11] = e->ring.p;
	ptr[12] = e->tmp.p, ptr[13] = e->total.p;
	h = pl_fnv(h, v, sizeof(v)), h = pl_fnv(h, ptr, sizeof(ptr)), h = pl_fnv(h, P, sizeof(*P));
	for (i = 0; i < n; ++i) {
		const plk_job_t *J = &e->hj[e->horder[i]];
		const int32_t t = e->hwave[e->horder[i]] << 8 | pl_group_of(J) << 4 | J->rows << 1 | (J->nw > 1);
		h = pl_fnv(h, &t, sizeof(t));
	}
	return h ? h : 1;
}

/* Runs the whole batch on `st`.  Inputs (nt/aa/ss) and outputs (res/cig) are device pointers. */
static int pl_run(pl_engine_t *e, const ns_opt_t *opt, const pl_splice_job_t *jobs, int32_t n,
		const uint8_t *nt, const uint8_t *aa, const uint8_t *ss, pl_splice_result_t *res_dev,
		uint32_t *cig_dev, int64_t cig_cap, int64_t *total_out, cudaStream_t st)
{
	plk_params_t P;
	int32_t q, max_al = 1, n_waves = 1, w, max_sub, *sorted, wave_n_coop = 0, two = 0;
	int64_t prep_total = 0, tmp_total = 0, trace_total = 0, max_trace = 0, slots, arena_budget, arena_words = 0;
	int64_t ring_ints = 0;
	int64_t *wave_bytes = 0, *wave_cells = 0, total_words = 0;
	int ok = 0, capturing = 0;
	uint64_t g_launch0 = 0, g_key = 0;

	e->last_waves = e->last_coop = e->last_dp_launches = e->last_pairs = 0;
	if (n <= 0) { if (total_out) *total_out = 0; return 1; }
	if (!pl_params(opt, &P, 0)) return 0;
	if (!pl_grow_host(e, n)) return 0;
	max_sub = pl_max_sub(opt);
	slots = (int64_t)e->n_sm * e->ctas_per_sm[0][0] * PLK_WARPS_PER_CTA;

	/* 1. per-job metadata with nw = 1 sizes */
	for (q = 0; q < n; ++q) {
		plk_job_t *J = &e->hj[q];
		const pl_splice_job_t *x = &jobs[q];
		int64_t bound = (int64_t)x->al * max_sub;
		memset(J, 0, sizeof(*J));
		if (x->nl < 3 || x->al < 1) {
			pl_set_error("job %d: nl=%d al=%d outside the DP's domain (nl >= 3, al >= 1)", q, x->nl, x->al);
			return 0;
		}
		J->nt_off = x->nt_off, J->aa_off = x->aa_off, J->ss_off = ss ? x->ss_off : -1;
		J->nl = x->nl, J->al = x->al;
		J->mode = bound + opt->end_bonus > 30000 ? 1 : (bound + 256 >= 32767 ? 2 : 0);
		J->slen = J->mode == 1 ? (x->al + 3) / 4 : (x->al + 7) / 8;
		J->nw = 1;
		J->rows = x->nl - 2 <= e->r4_rows ? 4 : PLK_DP_ROWS;
		J->prep_off = prep_total, prep_total += plk_prep_bytes(x->nl, x->al);
		J->tmp_off = tmp_total, tmp_total += (int64_t)x->nl + x->al + 8;
		J->score = INT32_MIN;
		if (x->al > max_al) max_al = x->al;
		trace_total += plk_trace_words(x->nl, x->al, PLK_WARPS_PER_CTA, J->rows) * 2;
		if (plk_trace_words(x->nl, x->al, PLK_WARPS_PER_CTA, J->rows) * 2 > max_trace)
			max_trace = plk_trace_words(x->nl, x->al, PLK_WARPS_PER_CTA, J->rows) * 2;
	}
	if (max_trace > e->trace_budget) {
		pl_set_error("one job needs %lld trace bytes, over the budget of %lld", (long long)max_trace, (long long)e->trace_budget);
		return 0;
	}
	e->last_pairs = pl_form_pairs(e, opt, n, max_sub, &P);
	if (e->last_pairs > 0) /* the unit the waves are packed by is a pair: twice a job's trace */
		for (q = 0; q < n; ++q)
			if (e->hj[q].mode == 3 && e->hj[q].pair >= 0 &&
					2 * plk_trace_words(e->hj[q].nl, e->hj[q].al, PLK_WARPS_PER_CTA, e->hj[q].rows) * 2 > max_trace)
				max_trace = 2 * plk_trace_words(e->hj[q].nl, e->hj[q].al, PLK_WARPS_PER_CTA, e->hj[q].rows) * 2;
	/* 2. waves by LPT bin packing on trace bytes.  A batch over the budget runs its
	 * waves alternately on two streams, each with its own arena of half the budget:
	 * a wave's DP then starts while the one before drains instead of after it. */
	arena_budget = e->trace_budget;
	if (trace_total > e->trace_budget && 4 * max_trace <= e->trace_budget) two = 1, arena_budget = e->trace_budget / 2;
	sorted = e->horder + n;
	{
		pl_key_t *key = (pl_key_t*)malloc(sizeof(pl_key_t) * (size_t)n);
		if (!key) { pl_set_error("out of host memory"); return 0; }
		for (q = 0; q < n; ++q) key[q].cells = (int64_t)(e->hj[q].nl - 2) * e->hj[q].al, key[q].idx = q;
		qsort(key, (size_t)n, sizeof(pl_key_t), pl_cmp_cells_desc);
		for (q = 0; q < n; ++q) sorted[q] = key[q].idx;
		free(key);
	}
	if (trace_total > arena_budget)
		n_waves = (int32_t)((trace_total + (arena_budget - max_trace) - 1) / (arena_budget - max_trace));
	if (n_waves > n) n_waves = n;
	if (n_waves < 2) two = 0;
	wave_bytes = (int64_t*)calloc((size_t)n_waves, sizeof(int64_t));
	wave_cells = (int64_t*)calloc((size_t)n_waves, sizeof(int64_t));
	if (!wave_bytes || !wave_cells) { pl_set_error("out of host memory"); goto fail; }
	for (q = 0; q < n; ++q) {
		const int32_t j = sorted[q];
		const plk_job_t *J = &e->hj[j];
		int32_t best = 0, t;
		if (J->mode == 3 && J->pair < 0) continue;  /* the second job of a pair goes with the first */
		for (w = 1; w < n_waves; ++w) if (wave_bytes[w] < wave_bytes[best]) best = w;
		for (t = 0; t < (J->mode == 3 ? 2 : 1); ++t) {
			const int32_t jj = t == 0 ? j : J->pair;
			e->hwave[jj] = best;
			wave_bytes[best] += plk_trace_words(e->hj[jj].nl, e->hj[jj].al, PLK_WARPS_PER_CTA, e->hj[jj].rows) * 2;
			wave_cells[best] += (int64_t)(e->hj[jj].nl - 2) * e->hj[jj].al;
		}
	}
	/* 3. cooperative or solo, trace offsets inside each wave's arena */
	memset(wave_bytes, 0, sizeof(int64_t) * (size_t)n_waves);
	for (q = 0; q < n; ++q) {
		const int32_t j = sorted[q];
		plk_job_t *J = &e->hj[j];
		const int64_t cells = (int64_t)(J->nl - 2) * J->al, share = wave_cells[e->hwave[j]] / slots;
		if (J->al >= 200 && J->nl - 2 >= 32 * PLK_WARPS_PER_CTA * J->rows && (double)cells > share * e->coop_ratio)
			J->nw = PLK_WARPS_PER_CTA;
		if (J->mode == 3 && J->pair >= 0) e->hj[J->pair].nw = J->nw;  /* a pair shares one wavefront */
		J->trace_off = wave_bytes[e->hwave[j]] / 2;
		wave_bytes[e->hwave[j]] += (plk_trace_words(J->nl, J->al, J->nw, J->rows) * 2 + 15) / 16 * 16;
	}
	{
		int64_t need_trace = 0;
		for (w = 0; w < n_waves; ++w) if (wave_bytes[w] > need_trace) need_trace = wave_bytes[w];
		need_trace = (need_trace + 255) / 256 * 256;
		arena_words = need_trace / 2;
		if (!dbuf_ensure(&e->trace, (size_t)need_trace * (two ? 2 : 1))) goto fail;
	}
	if (!dbuf_ensure(&e->jobs, sizeof(plk_job_t) * (size_t)n) || !dbuf_ensure(&e->order, sizeof(int32_t) * (size_t)n) ||
			!dbuf_ensure(&e->counters, 64) || !dbuf_ensure(&e->prep, (size_t)prep_total + PLK_PREP_SLACK) ||
			!dbuf_ensure(&e->tmp, sizeof(uint32_t) * (size_t)tmp_total) || !dbuf_ensure(&e->total, 64))
		goto fail;
	{
		const int64_t stride = ((int64_t)max_al + 1) * PLK_RING_INTS;
		const int64_t n_ctas = (int64_t)e->n_sm * pl_max_ctas(e);
		ring_ints = stride * n_ctas * PLK_WARPS_PER_CTA;
		if (!dbuf_ensure(&e->ring, sizeof(int32_t) * (size_t)(ring_ints * (two ? 2 : 1)))) goto fail;
	}
	/* order array: per wave, per mode: cooperative jobs then solo jobs, each by decreasing size */
	{
		int32_t pos = 0;
		for (w = 0; w < n_waves; ++w) {
			int m, r;
			for (m = 0; m < 5; ++m)
				for (r = 0; r < 2; ++r) {
					const int rows = r == 0 ? 8 : 4;
					int pass;
					for (pass = 0; pass < 2; ++pass)
						for (q = 0; q < n; ++q) {
							const int32_t j = sorted[q];
							const plk_job_t *J = &e->hj[j];
							if (e->hwave[j] == w && pl_group_of(J) == m && J->rows == rows && (J->nw > 1) == (pass == 0))
								e->horder[pos++] = j;
						}
				}
		}
	}
	CK(cudaMemcpyAsync(e->jobs.p, e->hj, sizeof(plk_job_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->order.p, e->horder, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	e->n_ev = 0;
	{ /* Graph replay: the launches below depend only on the plan's shape (the groups of the
	   * order array, the waves, the buffers and the parameters), not on the job table's
	   * contents, which the copies above refresh.  A shape seen on the previous call is
	   * captured into a CUDA graph on this one and replayed while it recurs (timed runs
	   * launch directly: their events sit between the launches). */
		const uint64_t key = pl_plan_key(e, n, n_waves, two, arena_words, ring_ints, max_al, nt, aa, ss, res_dev,
				cig_dev, cig_cap, st, &P);
		const int use = e->graphs && !e->timing;
		if (use && e->g_exec && key == e->g_key) {
			CK(cudaGraphLaunch(e->g_exec, st));
			plk_add_launches((uint64_t)e->g_nlaunch);
			e->last_dp_launches = e->g_dp_launches, wave_n_coop = e->g_coop;
			++e->g_replays;
			goto launched;
		}
		capturing = use && key == e->g_prev_key;
		e->g_prev_key = key;
		if (capturing) {
			g_launch0 = plk_launches();
			if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
				cudaGetLastError();  /* a stream that cannot be captured (the legacy stream): launch directly */
				capturing = 0;
			}
			g_key = key;
		}
	}
	PL_TIME(e, st, 0);
	CKK(plk_prep((const plk_job_t*)e->jobs.p, n, nt, aa, ss, (uint8_t*)e->prep.p, &P, st));
	PL_TIME(e, st, 0);
	if (two) { /* fork: the side stream starts after the preparation */
		CK(cudaEventRecord(e->ev_fork, st));
		CK(cudaStreamWaitEvent(e->side, e->ev_fork, 0));
	}
	{
		int32_t pos = 0;
		for (w = 0; w < n_waves; ++w) {
			const int32_t wave_start = pos, a = two ? (w & 1) : 0;
			cudaStream_t sw = a ? e->side : st;
			uint16_t *trace_w = (uint16_t*)e->trace.p + a * arena_words;
			int m, r;
			for (m = 0; m < 5; ++m)
				for (r = 0; r < 2; ++r) {
					const int rows = r == 0 ? 8 : 4;
					int32_t n_coop = 0, n_solo = 0;
#define PL_IN_GROUP(x) (e->hwave[e->horder[(x)]] == w && pl_group_of(&e->hj[e->horder[(x)]]) == m && e->hj[e->horder[(x)]].rows == rows)
					while (pos + n_coop < n && PL_IN_GROUP(pos + n_coop) && e->hj[e->horder[pos + n_coop]].nw > 1) ++n_coop;
					while (pos + n_coop + n_solo < n && PL_IN_GROUP(pos + n_coop + n_solo)) ++n_solo;
#undef PL_IN_GROUP
					if (n_coop + n_solo > 0 && m < 4) {  /* group 4: second jobs of pairs, run with their first */
						const int32_t *ord = (const int32_t*)e->order.p + pos;
						const int64_t stride = ((int64_t)max_al + 1) * PLK_RING_INTS;
						const int32_t ctas = e->n_sm * e->ctas_per_sm[m][r];
						PL_TIME(e, sw, 1);
						CKK(plk_splice_dp((plk_job_t*)e->jobs.p, ord, n_coop, ord + n_coop, n_solo,
								(int32_t*)e->counters.p + 8 * a, (const uint8_t*)e->prep.p, trace_w,
								(int32_t*)e->ring.p + a * ring_ints, stride, ctas, m, rows, &P, sw));
						PL_TIME(e, sw, 1);
						++e->last_dp_launches;
						wave_n_coop += n_coop;
					}
					pos += n_coop + n_solo;
				}
			PL_TIME(e, sw, 2);
			CKK(plk_traceback((plk_job_t*)e->jobs.p, (const int32_t*)e->order.p + wave_start, pos - wave_start,
					trace_w, (uint32_t*)e->tmp.p, sw));
			PL_TIME(e, sw, 2);
		}
	}
	if (two) { /* join */
		CK(cudaEventRecord(e->ev_join, e->side));
		CK(cudaStreamWaitEvent(st, e->ev_join, 0));
	}
	PL_TIME(e, st, 3);
	CKK(plk_scan_compact((plk_job_t*)e->jobs.p, n, (const uint32_t*)e->tmp.p, cig_dev, cig_cap,
			(int64_t*)e->total.p, res_dev, st));
	PL_TIME(e, st, 3);
	if (capturing) {
		cudaGraph_t g = 0;
		capturing = 0;
		CK(cudaStreamEndCapture(st, &g));
		if (e->g_exec) cudaGraphExecDestroy(e->g_exec), e->g_exec = 0;
		{
			const cudaError_t ie = cudaGraphInstantiate(&e->g_exec, g, 0);
			cudaGraphDestroy(g);
			CK(ie);
		}
		e->g_key = g_key, e->g_nlaunch = (int64_t)(plk_launches() - g_launch0);
		e->g_dp_launches = e->last_dp_launches, e->g_coop = wave_n_coop;
		CK(cudaGraphLaunch(e->g_exec, st));
	}
launched:
	CK(cudaMemcpyAsync(&total_words, e->total.p, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	if (total_out) *total_out = total_words;
	e->last_waves = n_waves, e->last_coop = wave_n_coop;
	if (e->timing) {
		/* event pairs: prep, every DP launch and every traceback (on the stream of their
		 * wave), compaction.  DP time is the union of the DP launches' intervals, traceback
		 * time the part of the tracebacks' intervals outside that union. */
		int k, nd = 0, nb = 0;
		float ms;
		double dp0[sizeof(e->ev) / sizeof(e->ev[0]) / 2], dp1[sizeof(e->ev) / sizeof(e->ev[0]) / 2];
		double all0[sizeof(e->ev) / sizeof(e->ev[0]) / 2], all1[sizeof(e->ev) / sizeof(e->ev[0]) / 2], u_dp, u_all;
		e->acc_dp_launches += e->last_dp_launches;
		for (q = 0; q < n; ++q) e->acc_cells += (int64_t)(e->hj[q].nl - 2) * e->hj[q].al;
		for (k = 0; k + 1 < e->n_ev; k += 2) {
			if (e->ev_kind[k] == 1 || e->ev_kind[k] == 2) {
				float a0, a1;
				cudaEventElapsedTime(&a0, e->ev[0], e->ev[k]);
				cudaEventElapsedTime(&a1, e->ev[0], e->ev[k + 1]);
				if (e->ev_kind[k] == 1) dp0[nd] = a0, dp1[nd++] = a1;
				all0[nb] = a0, all1[nb++] = a1;
			} else {
				cudaEventElapsedTime(&ms, e->ev[k], e->ev[k + 1]);
				e->acc_ms[e->ev_kind[k]] += ms;
			}
		}
		u_dp = pl_union_ms(dp0, dp1, nd), u_all = pl_union_ms(all0, all1, nb);
		e->acc_ms[1] += u_dp, e->acc_ms[2] += u_all - u_dp;
	}
	ok = 1;
fail:
	if (capturing) { /* a launch failed during the capture: end it, keep the stream usable */
		cudaGraph_t g = 0;
		cudaStreamEndCapture(st, &g);
		if (g) cudaGraphDestroy(g);
		cudaGetLastError();
		e->g_prev_key = 0;
	}
	free(wave_bytes), free(wave_cells);
	return ok;
}

PL_EXPORT int32_t pl_engine_last_pairs(const pl_engine_t *e) { return e ? e->last_pairs : 0; }

PL_EXPORT void pl_engine_set_graphs(pl_engine_t *e, int32_t enable) { if (e) e->graphs = enable != 0; }

PL_EXPORT int64_t pl_engine_graph_replays(const pl_engine_t *e) { return e ? e->g_replays : 0; }

PL_EXPORT void pl_engine_set_pairing(pl_engine_t *e, int32_t enable) { if (e) e->pairing = enable == 2 ? 2 : enable != 0; }

PL_EXPORT void pl_engine_set_tuning(pl_engine_t *e, int32_t r4_rows, double coop_ratio)
{
	if (!e) return;
	if (r4_rows >= 0) e->r4_rows = r4_rows;
	if (coop_ratio > 0.0) e->coop_ratio = coop_ratio;
}

PL_EXPORT void pl_engine_get_tuning(const pl_engine_t *e, int32_t *r4_rows, double *coop_ratio)
{
	if (!e) return;
	if (r4_rows) *r4_rows = e->r4_rows;
	if (coop_ratio) *coop_ratio = e->coop_ratio;
}

static double pl_now(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* Autotuner of the batched global DP: runs the batch under every pair of (rows-per-lane
 * bin boundary, cooperative-job ratio) of a small grid, keeps the fastest for this
 * engine and reports it.  The batch should look like the workload (the same length
 * distributions); its results are discarded. */
PL_EXPORT int pl_engine_autotune(pl_engine_t *e, const ns_opt_t *opt, const pl_splice_job_t *jobs, int32_t n,
		const uint8_t *nt, const uint8_t *aa, const uint8_t *ss, int32_t *r4_rows_out, double *coop_ratio_out)
{
	static const int32_t r4s[] = { 0, 1536, 3072, 6144, 12288 };
	static const double ratios[] = { 0.5, 0.7, 1.0 };
	pl_splice_result_t *res = 0;
	uint32_t *cig = 0;
	int64_t cap = 0, total = 0;
	int32_t q, best_r4 = e ? e->r4_rows : 0;
	double best_ratio = e ? e->coop_ratio : 0.7, best_t = 1e30;
	int a, b, ok = 0, timing;
	if (!e || n <= 0) { pl_set_error("autotune: no engine or empty batch"); return 0; }
	CK(cudaSetDevice(e->device));
	for (q = 0; q < n; ++q) cap += (int64_t)jobs[q].al + 64;
	CK(cudaMalloc((void**)&res, sizeof(pl_splice_result_t) * (size_t)n));
	CK(cudaMalloc((void**)&cig, sizeof(uint32_t) * (size_t)cap));
	timing = e->timing, e->timing = 0;
	if (!pl_run(e, opt, jobs, n, nt, aa, ss, res, cig, cap, &total, e->stream)) goto done;  /* warm-up */
	for (a = 0; a < (int)(sizeof(r4s) / sizeof(r4s[0])); ++a)
		for (b = 0; b < (int)(sizeof(ratios) / sizeof(ratios[0])); ++b) {
			double t0, t;
			e->r4_rows = r4s[a], e->coop_ratio = ratios[b];
			t0 = pl_now();
			if (!pl_run(e, opt, jobs, n, nt, aa, ss, res, cig, cap, &total, e->stream)) goto done;
			t = pl_now() - t0;
			if (t < best_t) best_t = t, best_r4 = r4s[a], best_ratio = ratios[b];
		}
	ok = 1;
done:
	e->timing = timing;
	e->r4_rows = best_r4, e->coop_ratio = best_ratio;
	if (r4_rows_out) *r4_rows_out = best_r4;
	if (coop_ratio_out) *coop_ratio_out = best_ratio;
fail:
	if (res) cudaFree(res);
	if (cig) cudaFree(cig);
	return ok;
}

PL_EXPORT int pl_splice_batch_device(pl_engine_t *e, const ns_opt_t *opt, const pl_splice_job_t *jobs, int32_t n,
		const uint8_t *nt, const uint8_t *aa, const uint8_t *ss, pl_splice_result_t *results_dev,
		uint32_t *cigar_dev, int64_t cigar_cap, int64_t *total_cigar, void *stream)
{
	if (!e) { pl_set_error("no engine"); return 0; }
	if (cudaSetDevice(e->device) != cudaSuccess) { pl_set_error("cudaSetDevice failed"); return 0; }
	return pl_run(e, opt, jobs, n, nt, aa, ss, results_dev, cigar_dev, cigar_cap, total_cigar,
			stream ? (cudaStream_t)stream : e->stream);
}

PL_EXPORT int pl_splice_batch_host(pl_engine_t *e, const ns_opt_t *opt, const pl_splice_job_t *jobs, int32_t n,
		const uint8_t *nt, int64_t nt_len, const uint8_t *aa, int64_t aa_len, const uint8_t *ss, int64_t ss_len,
		pl_splice_result_t *results, uint32_t *cigar, int64_t cigar_cap)
{
	cudaStream_t st;
	int64_t total = 0;
	int32_t q;
	if (!e) { pl_set_error("no engine"); return 0; }
	if (n < 0 || (n > 0 && (!jobs || !nt || !aa || !results))) { pl_set_error("invalid batch arguments"); return 0; }
	for (q = 0; q < n; ++q) /* every span inside its host buffer: the kernels read exactly these bytes */
		if (!pl_span_ok("job", q, "nt", jobs[q].nt_off, jobs[q].nl, nt_len) ||
				!pl_span_ok("job", q, "aa", jobs[q].aa_off, jobs[q].al, aa_len) ||
				(ss && jobs[q].ss_off >= 0 && !pl_span_ok("job", q, "ss", jobs[q].ss_off, jobs[q].nl, ss_len)))
			return 0;
	st = e->stream;
	CK(cudaSetDevice(e->device));
	if (!dbuf_ensure(&e->nt, (size_t)nt_len) || !dbuf_ensure(&e->aa, (size_t)aa_len) ||
			(ss && !dbuf_ensure(&e->ss, (size_t)ss_len)) || !dbuf_ensure(&e->res, sizeof(pl_splice_result_t) * (size_t)n) ||
			!dbuf_ensure(&e->cig, sizeof(uint32_t) * (size_t)(cigar_cap > 0 ? cigar_cap : 1)))
		return 0;
	CK(cudaMemcpyAsync(e->nt.p, nt, (size_t)nt_len, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->aa.p, aa, (size_t)aa_len, cudaMemcpyHostToDevice, st));
	if (ss) CK(cudaMemcpyAsync(e->ss.p, ss, (size_t)ss_len, cudaMemcpyHostToDevice, st));
	if (!pl_run(e, opt, jobs, n, (const uint8_t*)e->nt.p, (const uint8_t*)e->aa.p, ss ? (const uint8_t*)e->ss.p : 0,
			(pl_splice_result_t*)e->res.p, (uint32_t*)e->cig.p, cigar_cap, &total, st))
		return 0;
	CK(cudaMemcpyAsync(results, e->res.p, sizeof(pl_splice_result_t) * (size_t)n, cudaMemcpyDeviceToHost, st));
	if (total > cigar_cap) total = cigar_cap;
	if (total > 0) CK(cudaMemcpyAsync(cigar, e->cig.p, sizeof(uint32_t) * (size_t)total, cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	return 1;
fail:
	return 0;
}

/* ------------------------------------------------------------------ request queue API */

#define NS_REQ_MAX_BATCH 128       /* NS_GPU_MAX_BATCH of nasw-cuda.cu:420 */
#define NS_REQ_WAIT_NS 2000000L    /* collect for up to 2 ms, nasw-cuda.cu:423 */

struct ns_gpu_request_s {
	void *km;
	char *buf;                  /* ns[nl] | as[al] | ss[nl] */
	int32_t nl, al, has_ss;
	ns_opt_t opt;               /* scalars; tables copied below */
	int8_t sc[22 * 22];
	uint8_t nt4[256], aa20[256], codon[64];
	int32_t score, n_cigar, done, success;
	uint32_t *cigar;
	struct ns_gpu_request_s *next;
};

static pthread_mutex_t ns_mu = PTHREAD_MUTEX_INITIALIZER;
static pthread_cond_t ns_cv_work = PTHREAD_COND_INITIALIZER, ns_cv_done = PTHREAD_COND_INITIALIZER;
static ns_gpu_request_t *ns_q_head, *ns_q_tail;
static int32_t ns_q_n;
static int ns_ready;
static pl_engine_t *ns_engine;
static pthread_t ns_thread;
static uint64_t ns_dispatches, ns_launches, ns_h2d_ns, ns_kernel_ns, ns_d2h_ns;
static char ns_msg[1024] = "GPU backend has not been initialized";
static char ns_dev_name[256] = "none";

static uint64_t ns_now_ns(void)
{
	struct timespec t;
	clock_gettime(CLOCK_MONOTONIC, &t);
	return (uint64_t)t.tv_sec * 1000000000ull + (uint64_t)t.tv_nsec;
}

static int ns_same_opt(const ns_gpu_request_t *a, const ns_gpu_request_t *b)
{
	return a->opt.go == b->opt.go && a->opt.ge == b->opt.ge && a->opt.io == b->opt.io && a->opt.fs == b->opt.fs &&
		memcmp(a->opt.sp, b->opt.sp, sizeof(a->opt.sp)) == 0 && a->opt.sp_null_bonus == b->opt.sp_null_bonus &&
		a->opt.end_bonus == b->opt.end_bonus && memcmp(a->sc, b->sc, sizeof(a->sc)) == 0 &&
		memcmp(a->nt4, b->nt4, 256) == 0 && memcmp(a->aa20, b->aa20, 256) == 0 && memcmp(a->codon, b->codon, 64) == 0;
}

/* run one batch of requests sharing options; fills each request and marks it done */
static void ns_run_batch(ns_gpu_request_t **rq, int32_t n)
{
	pl_splice_job_t *jobs = (pl_splice_job_t*)malloc(sizeof(*jobs) * (size_t)n);
	pl_splice_result_t *res = (pl_splice_result_t*)malloc(sizeof(*res) * (size_t)n);
	int64_t nt_len = 0, aa_len = 0, cap = 0, pos_nt = 0, pos_aa = 0;
	uint8_t *nt = 0, *aa = 0, *ss = 0;
	uint32_t *cig = 0;
	int32_t q, any_ss = 0, ok = 0;
	ns_opt_t opt;
	uint64_t t0, t1;
	for (q = 0; q < n; ++q) nt_len += rq[q]->nl, aa_len += rq[q]->al, cap += (int64_t)rq[q]->nl + rq[q]->al + 8, any_ss |= rq[q]->has_ss;
	nt = (uint8_t*)malloc((size_t)nt_len), aa = (uint8_t*)malloc((size_t)aa_len);
	ss = any_ss ? (uint8_t*)malloc((size_t)nt_len) : 0;
	cig = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)cap);
	if (!jobs || !res || !nt || !aa || (any_ss && !ss) || !cig) { snprintf(ns_msg, sizeof(ns_msg), "out of host memory"); goto done; }
	for (q = 0; q < n; ++q) {
		ns_gpu_request_t *r = rq[q];
		memcpy(nt + pos_nt, r->buf, (size_t)r->nl);
		memcpy(aa + pos_aa, r->buf + r->nl, (size_t)r->al);
		if (ss) {
			if (r->has_ss) memcpy(ss + pos_nt, r->buf + r->nl + r->al, (size_t)r->nl);
			else memset(ss + pos_nt, 0, (size_t)r->nl);
		}
		jobs[q].nt_off = pos_nt, jobs[q].aa_off = pos_aa, jobs[q].ss_off = r->has_ss ? pos_nt : -1;
		jobs[q].nl = r->nl, jobs[q].al = r->al;
		pos_nt += r->nl, pos_aa += r->al;
	}
	opt = rq[0]->opt;
	opt.sc = rq[0]->sc, opt.nt4 = rq[0]->nt4, opt.aa20 = rq[0]->aa20, opt.codon = rq[0]->codon, opt.pssm = 0;
	t0 = ns_now_ns();
	ok = pl_splice_batch_host(ns_engine, &opt, jobs, n, nt, nt_len, aa, aa_len, ss, ss ? nt_len : 0, res, cig, cap);
	t1 = ns_now_ns();
	__sync_fetch_and_add(&ns_kernel_ns, t1 - t0);
	if (!ok) snprintf(ns_msg, sizeof(ns_msg), "GPU alignment failed: %s", pl_last_error());
done:
	for (q = 0; q < n; ++q) {
		ns_gpu_request_t *r = rq[q];
		r->success = 0;
		if (ok && res[q].status == 0) {
			r->score = res[q].score, r->n_cigar = res[q].n_cigar;
			r->cigar = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(r->n_cigar > 0 ? r->n_cigar : 1));
			if (r->cigar) {
				memcpy(r->cigar, cig + res[q].cigar_off, sizeof(uint32_t) * (size_t)r->n_cigar);
				r->success = 1;
			}
		}
	}
	if (ok) __sync_fetch_and_add(&ns_dispatches, (uint64_t)n), __sync_fetch_and_add(&ns_launches, 1ull);
	pthread_mutex_lock(&ns_mu);
	for (q = 0; q < n; ++q) rq[q]->done = 1;
	pthread_cond_broadcast(&ns_cv_done);
	pthread_mutex_unlock(&ns_mu);
	free(jobs), free(res), free(nt), free(aa), free(ss), free(cig);
}

static void *ns_executor(void *arg)
{
	ns_gpu_request_t *batch[NS_REQ_MAX_BATCH];
	(void)arg;
	cudaSetDevice(ns_engine->device);
	for (;;) {
		int32_t n = 0;
		ns_gpu_request_t **pp;
		pthread_mutex_lock(&ns_mu);
		while (ns_q_n == 0) pthread_cond_wait(&ns_cv_work, &ns_mu);
		if (ns_q_n < NS_REQ_MAX_BATCH) { /* let concurrent submitters join the batch */
			struct timespec until;
			clock_gettime(CLOCK_REALTIME, &until);
			until.tv_nsec += NS_REQ_WAIT_NS;
			if (until.tv_nsec >= 1000000000L) until.tv_sec += 1, until.tv_nsec -= 1000000000L;
			while (ns_q_n < NS_REQ_MAX_BATCH)
				if (pthread_cond_timedwait(&ns_cv_work, &ns_mu, &until) == ETIMEDOUT) break;
		}
		/* take up to 128 requests sharing the first one's options */
		pp = &ns_q_head;
		while (*pp && n < NS_REQ_MAX_BATCH) {
			ns_gpu_request_t *r = *pp;
			if (n == 0 || ns_same_opt(batch[0], r)) {
				*pp = r->next, batch[n++] = r, --ns_q_n;
				r->next = 0;
			} else pp = &r->next;
		}
		ns_q_tail = 0;
		for (pp = &ns_q_head; *pp; pp = &(*pp)->next) ns_q_tail = *pp;
		pthread_mutex_unlock(&ns_mu);
		ns_run_batch(batch, n);
	}
	return 0;
}

PL_EXPORT int ns_gpu_init(int32_t device)
{
	int count = 0;
	struct cudaDeviceProp prop;
	pthread_mutex_lock(&ns_mu);
	if (ns_ready) { pthread_mutex_unlock(&ns_mu); return 1; }
	if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) {
		cudaGetLastError();
		snprintf(ns_msg, sizeof(ns_msg), "no CUDA device available");
		goto fail;
	}
	if (device < 0 || device >= count) {
		snprintf(ns_msg, sizeof(ns_msg), "CUDA GPU %d does not exist (%d available)", device, count);
		goto fail;
	}
	if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { snprintf(ns_msg, sizeof(ns_msg), "cudaGetDeviceProperties failed"); goto fail; }
	if (prop.major < 10) {
		snprintf(ns_msg, sizeof(ns_msg), "%s is sm_%d%d; this library is built for sm_100a", prop.name, prop.major, prop.minor);
		goto fail;
	}
	ns_engine = pl_engine_create(device, 0);
	if (!ns_engine) { snprintf(ns_msg, sizeof(ns_msg), "engine: %s", pl_last_error()); goto fail; }
	strncpy(ns_dev_name, prop.name, sizeof(ns_dev_name) - 1);
	if (pthread_create(&ns_thread, 0, ns_executor, 0) != 0) {
		snprintf(ns_msg, sizeof(ns_msg), "failed to start the GPU executor thread");
		pl_engine_destroy(ns_engine), ns_engine = 0;
		goto fail;
	}
	pthread_detach(ns_thread);
	strcpy(ns_msg, "none");
	ns_ready = 1;
	pthread_mutex_unlock(&ns_mu);
	return 1;
fail:
	pthread_mutex_unlock(&ns_mu);
	return 0;
}

/* device of the request queue once ns_gpu_init() succeeded, else -1 (other translation units
 * that require ns_gpu_init first, as the reference's gapless entry does, ask here) */
int pl_ns_device(void)
{
	int d;
	pthread_mutex_lock(&ns_mu);
	d = ns_ready && ns_engine ? ns_engine->device : -1;
	pthread_mutex_unlock(&ns_mu);
	return d;
}

void pl_ns_set_error(const char *msg)
{
	pthread_mutex_lock(&ns_mu);
	snprintf(ns_msg, sizeof(ns_msg), "%s", msg);
	pthread_mutex_unlock(&ns_mu);
}

PL_EXPORT const char *ns_gpu_error(void) { return ns_msg; }
PL_EXPORT const char *ns_gpu_name(void) { return ns_dev_name; }
PL_EXPORT uint64_t ns_gpu_dispatch_count(void) { return __sync_fetch_and_add(&ns_dispatches, 0ull); }
PL_EXPORT uint64_t ns_gpu_launch_count(void) { return __sync_fetch_and_add(&ns_launches, 0ull); }
PL_EXPORT double ns_gpu_h2d_seconds(void) { return (double)__sync_fetch_and_add(&ns_h2d_ns, 0ull) * 1e-9; }
PL_EXPORT double ns_gpu_kernel_seconds(void) { return (double)__sync_fetch_and_add(&ns_kernel_ns, 0ull) * 1e-9; }
PL_EXPORT double ns_gpu_d2h_seconds(void) { return (double)__sync_fetch_and_add(&ns_d2h_ns, 0ull) * 1e-9; }

PL_EXPORT ns_gpu_request_t *ns_gpu_submit(void *km, const char *ns, int32_t nl, const char *as, int32_t al,
		const ns_opt_t *opt, const uint8_t *ss)
{
	ns_gpu_request_t *r;
	int i, max_sub = 0;
	if (!ns_ready || !opt || !ns || !as) return 0;
	if (nl < 3 || al < 1 || opt->asize != 22 || opt->pssm || !opt->sc || !opt->nt4 || !opt->aa20 || !opt->codon) return 0;
	for (i = 0; i < 22 * 22; ++i) if (max_sub < opt->sc[i]) max_sub = opt->sc[i];
	if ((int64_t)al * max_sub + opt->end_bonus > 30000) return 0; /* 16-bit contract, nasw-cuda.cu:1084-1086 */
	r = (ns_gpu_request_t*)calloc(1, sizeof(*r));
	if (!r) return 0;
	r->buf = (char*)malloc((size_t)nl * (ss ? 2 : 1) + (size_t)al);
	if (!r->buf) { free(r); return 0; }
	memcpy(r->buf, ns, (size_t)nl), memcpy(r->buf + nl, as, (size_t)al);
	if (ss) memcpy(r->buf + nl + al, ss, (size_t)nl);
	r->km = km, r->nl = nl, r->al = al, r->has_ss = ss != 0;
	r->opt = *opt;
	memcpy(r->sc, opt->sc, sizeof(r->sc));
	memcpy(r->nt4, opt->nt4, 256), memcpy(r->aa20, opt->aa20, 256), memcpy(r->codon, opt->codon, 64);
	pthread_mutex_lock(&ns_mu);
	if (ns_q_tail) ns_q_tail->next = r; else ns_q_head = r;
	ns_q_tail = r, ++ns_q_n;
	pthread_cond_broadcast(&ns_cv_work);
	pthread_mutex_unlock(&ns_mu);
	return r;
}

PL_EXPORT int ns_gpu_wait(ns_gpu_request_t *r, ns_rst_t *rst)
{
	int success, k;
	if (!r) return 0;
	pthread_mutex_lock(&ns_mu);
	while (!r->done) pthread_cond_wait(&ns_cv_done, &ns_mu);
	pthread_mutex_unlock(&ns_mu);
	success = r->success;
	if (success) {
		rst->nt_len = r->nl, rst->aa_len = r->al, rst->score = r->score;
		for (k = 0; k < r->n_cigar; ++k) { /* append as ns_push_cigar (nasw.h:219-229) does */
			const uint32_t op = r->cigar[k] & 0xf, len = r->cigar[k] >> 4;
			if (rst->n_cigar == 0 || op != (rst->cigar[rst->n_cigar - 1] & 0xf) || op == NS_CIGAR_F || op == NS_CIGAR_G) {
				if (rst->n_cigar == rst->m_cigar) {
					const int32_t m = rst->m_cigar + (rst->m_cigar >> 1) + 8;
					uint32_t *c = (uint32_t*)pl_krealloc(r->km, rst->cigar, sizeof(uint32_t) * (size_t)m);
					if (!c) { /* the CIGAR so far stays in rst; the request reports failure */
						pl_ns_set_error(pl_last_error());
						success = 0;
						break;
					}
					rst->cigar = c, rst->m_cigar = m;
				}
				rst->cigar[rst->n_cigar++] = len << 4 | op;
			} else rst->cigar[rst->n_cigar - 1] += len << 4;
		}
	}
	free(r->cigar), free(r->buf), free(r);
	return success;
}

PL_EXPORT int ns_gpu_global(void *km, const char *ns, int32_t nl, const char *as, int32_t al, const ns_opt_t *opt,
		const uint8_t *ss, ns_rst_t *r)
{
	ns_gpu_request_t *q = ns_gpu_submit(km, ns, nl, as, al, opt, ss);
	return q ? ns_gpu_wait(q, r) : 0;
}
