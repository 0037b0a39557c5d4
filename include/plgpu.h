/*
 * plgpu.h -- C ABI of libplgpu, the B200 (sm_100a) implementation of ProtLocus's
 * alignment hot path.
 *
 * The library is a drop-in for the reference's GPU translation units
 * (nasw-cuda.o, nasw-ext-gpu.o, hmm-gpu.o): it exports the same symbols with the
 * same signatures and semantics, so the reference's map.c / align.c / hmm.c link
 * against it unchanged (swap the objects in the reference Makefile's OBJS).
 *
 * Plain C, no CUDA or torch types.  Every declaration cites the reference
 * interface it replaces as file:line within the reference project.
 *
 * Types ns_opt_t / ns_rst_t are layout-identical to nasw.h:62-82; when nasw.h
 * has already been included its definitions are used instead.
 */
#ifndef PLGPU_H
#define PLGPU_H

#include <stdint.h>
#include <string.h>

#ifndef NASW_H
/* CIGAR operators (nasw.h:33-44) */
#define NS_CIGAR_M	0
#define NS_CIGAR_I	1
#define NS_CIGAR_D	2
#define NS_CIGAR_N	3
#define NS_CIGAR_F	10
#define NS_CIGAR_G	11
#define NS_CIGAR_U	12
#define NS_CIGAR_V	13
#define NS_CIGAR_E	14
#define NS_CIGAR_STR   "MIDNSHP=XBFGUVE"

/* option flags (nasw.h:46-49) */
#define NS_F_CIGAR      0x1
#define NS_F_EXT_LEFT   0x2
#define NS_F_EXT_RIGHT  0x4
#define NS_F_GPU        0x8

#define NS_SPSC_OFFSET 64  /* nasw.h:55 */

/* alignment options; must stay layout-identical to nasw.h:62-75 */
typedef struct {
	int32_t flag;
	int32_t go, ge, io, fs;
	int32_t xdrop, end_bonus;
	int32_t asize;
	int32_t gpu_device;
	int64_t gpu_min_cells;
	int32_t sp[6];
	int32_t sp_null_bonus;
	float ie_coef;
	const int8_t *sc;
	const int8_t *pssm;
	uint8_t *nt4, *aa20, *codon;
} ns_opt_t;

/* alignment result; layout-identical to nasw.h:77-82 */
typedef struct {
	int32_t n_cigar, m_cigar;
	int32_t nt_len, aa_len;
	int32_t score;
	uint32_t *cigar;
} ns_rst_t;

typedef struct ns_gpu_request_s ns_gpu_request_t;

/* gapless prefilter records (nasw.h:157-171) */
typedef struct {
	int64_t target_offset, target_length;
	int64_t query_offset;
	int32_t query_length;
	int32_t anchor_offset, anchor_count;
	int32_t reverse;
} ns_gpu_gapless_candidate_t;
typedef struct {
	int64_t target_block;
	int32_t query_end;
	int32_t reserved;
} ns_gpu_gapless_anchor_t;
typedef struct {
	uint64_t batches, candidates, anchors, seed_positions;
} ns_gpu_gapless_profile_t;

typedef struct ns_ext_batch_s ns_ext_batch_t;
#endif /* NASW_H */

#ifndef PROTLOCUS_H
typedef struct mp_hmm_s mp_hmm_t;  /* protlocus.h:67, opaque (hmm.c:14-22) */
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------
 * Spliced global DP with CIGAR (replaces nasw-cuda.cu:516-1145)
 * ------------------------------------------------------------------------- */

/* nasw.h:141 -- 1 when the device is ready; idempotent and thread-safe. */
int ns_gpu_init(int32_t device);
/* nasw.h:142 -- text of the last error ("none" when healthy). */
const char *ns_gpu_error(void);
/* nasw.h:143 -- device name, "none" before ns_gpu_init(). */
const char *ns_gpu_name(void);
/* nasw.h:144 -- requests completed on the device (monotonic). */
uint64_t ns_gpu_dispatch_count(void);
/* nasw.h:145 -- kernel launches of the request path (monotonic). */
uint64_t ns_gpu_launch_count(void);
/* nasw.h:146-148 -- accumulated host-observed phase times. */
double ns_gpu_h2d_seconds(void);
double ns_gpu_kernel_seconds(void);
double ns_gpu_d2h_seconds(void);
/* nasw.h:150 -- queue one global spliced DP.  NULL when not taken: nl < 3,
 * al < 1, al*max(sc)+end_bonus > 30000 (the 16-bit contract), or device not
 * ready.  A non-NULL request must be consumed exactly once by ns_gpu_wait();
 * km must stay valid until then.  Thread-safe. */
ns_gpu_request_t *ns_gpu_submit(void *km, const char *ns, int32_t nl, const char *as, int32_t al,
		const ns_opt_t *opt, const uint8_t *ss);
/* nasw.h:151 -- block until done; 1 = r filled (nt_len, aa_len, score and the
 * CIGAR appended into r->cigar from the request's km), 0 = failed (device
 * failure, or the CIGAR could not be grown: host memory, or a km arena passed
 * by a program that links no kalloc; ns_gpu_error() says which).  Frees the
 * request either way. */
int ns_gpu_wait(ns_gpu_request_t *request, ns_rst_t *r);
/* nasw.h:152 -- submit + wait. */
int ns_gpu_global(void *km, const char *ns, int32_t nl, const char *as, int32_t al,
		const ns_opt_t *opt, const uint8_t *ss, ns_rst_t *r);

/* ---------------------------------------------------------------------------
 * Bulk entry points (no counterpart in the reference: the reference only has
 * the per-request queue above).  They take many DP jobs at once, with the
 * length binning, the persistent wavefront kernel and the device traceback
 * exposed directly.  Used by the benchmark and by callers that already hold
 * a whole batch.
 * ------------------------------------------------------------------------- */

/* One global spliced DP job inside packed buffers. */
typedef struct {
	int64_t nt_off;   /* first nucleotide in the packed nt buffer (ASCII or 0-4 codes) */
	int64_t aa_off;   /* first residue in the packed protein buffer (ASCII) */
	int64_t ss_off;   /* splice-score track offset in the ss buffer, -1 = none */
	int32_t nl, al;
} pl_splice_job_t;

/* Result of one job.  cigar_off indexes the caller's CIGAR buffer; the CIGAR
 * has exactly the words ns_global_gs_auto() (nasw-sse.c:980) would produce. */
typedef struct {
	int32_t score;
	int32_t n_cigar;
	int64_t cigar_off;
	int32_t mode;      /* 16 or 32: the DP width the job ran at (ns_global_gs_auto's rule) */
	int32_t status;    /* 0 = ok; <0 = error (see pl_last_error()) */
} pl_splice_result_t;

typedef struct pl_engine_s pl_engine_t;

/* Create an engine on the current CUDA device.  trace_budget_bytes bounds the
 * device traceback arena (jobs run in waves that fit); 0 = default. */
pl_engine_t *pl_engine_create(int32_t device, int64_t trace_budget_bytes);
void pl_engine_destroy(pl_engine_t *e);
const char *pl_last_error(void);

/* Host buffers in, host results out (H2D, kernels and D2H inside).
 * cigar_cap is the capacity of `cigar` in words; each job may need up to
 * nl + al + 4 words.  Returns 1 on success. */
int pl_splice_batch_host(pl_engine_t *e, const ns_opt_t *opt,
		const pl_splice_job_t *jobs, int32_t n_jobs,
		const uint8_t *nt, int64_t nt_len, const uint8_t *aa, int64_t aa_len,
		const uint8_t *ss, int64_t ss_len,
		pl_splice_result_t *results, uint32_t *cigar, int64_t cigar_cap);

/* Device-resident inputs and outputs: nt/aa/ss/results/cigar are device
 * pointers; the job table is read on the host (it drives the planning).
 * Work is issued on `stream` (a cudaStream_t passed as void*, NULL = the
 * engine's own stream; a multi-wave batch forks half its waves onto the
 * engine's second stream after the preparation and joins it back before the
 * compaction) and the call returns once it has completed.
 * *total_cigar (optional) receives the number of CIGAR words produced; jobs
 * beyond cigar_cap get status -2.  Returns 1 on success. */
int pl_splice_batch_device(pl_engine_t *e, const ns_opt_t *opt,
		const pl_splice_job_t *jobs, int32_t n_jobs,
		const uint8_t *nt, const uint8_t *aa, const uint8_t *ss,
		pl_splice_result_t *results_dev, uint32_t *cigar_dev, int64_t cigar_cap,
		int64_t *total_cigar, void *stream);

/* Optional CUDA-event timing of every batch phase (prep, DP kernel, traceback,
 * compaction), accumulated until the next pl_engine_set_timing() call.  A batch
 * over the trace budget runs its waves alternately on the engine's stream and a
 * second one; dp_ms is then the union of the DP launches' intervals and
 * traceback_ms the part of the tracebacks outside it. */
int pl_engine_set_timing(pl_engine_t *e, int32_t enable);
void pl_engine_times(const pl_engine_t *e, double *prep_ms, double *dp_ms, double *traceback_ms,
		double *compact_ms, int64_t *dp_launches, int64_t *cells);

/* The engine's own CUDA stream (a cudaStream_t as void*). */
void *pl_engine_stream(const pl_engine_t *e);

/* Measured integer-pipe throughput of a device, in lane-operations per second:
 * int32 add+max chains and int16x2 (__vadd2 + __vmaxs2) chains at full
 * occupancy.  The DP kernels are bound by this pipe.  Returns 1 on success. */
int pl_measure_int_peak(int32_t device, double *int32_lane_ops, double *int16x2_lane_ops);
/* Tuning of the batched global DP: jobs with at most r4_rows DP rows (nl - 2) run 4
 * rows per lane, the rest 8; a job takes a whole CTA when it holds more than
 * coop_ratio times a warp's share of its wave's cells.  set: negative / non-positive
 * arguments keep the current value.  autotune: times the given batch (results
 * discarded) under a grid of both, keeps the fastest on the engine and reports it. */
void pl_engine_set_tuning(pl_engine_t *e, int32_t r4_rows, double coop_ratio);
void pl_engine_get_tuning(const pl_engine_t *e, int32_t *r4_rows, double *coop_ratio);
int pl_engine_autotune(pl_engine_t *e, const ns_opt_t *opt, const pl_splice_job_t *jobs, int32_t n,
		const uint8_t *nt, const uint8_t *aa, const uint8_t *ss, int32_t *r4_rows, double *coop_ratio);

/* Host-side fault injection for failure tests (no counterpart in the
 * reference): site 0 = a host allocation of the request queue or the
 * extension batch object, 1 = a device buffer allocation of an engine, 2 = the
 * next device batch of the extension executor; the site fails once, on its
 * (after+1)-th pass from now (after < 0 disarms).  No device work is involved:
 * the failure is the error path the real failure takes.  Returns 1 when armed. */
int pl_debug_fault(int32_t site, int32_t after);

/* Number of trace waves, cooperative jobs and DP launches of the last batch. */
void pl_engine_last_plan(const pl_engine_t *e, int32_t *n_waves, int32_t *n_coop, int32_t *n_dp_launches);
/* Two 16-bit jobs that share one protein (the same aa_off in the job table) and one
 * window length -- the two strands of a locus -- run as a pair in the two halves of
 * the int16x2 DP kernel when their score range fits its 15-bit domain (on by
 * default; PLGPU_PAIR=0 or pl_engine_set_pairing(e, 0) turns it off).  With
 * enable = 1 the eligible jobs pair when they make at least PLGPU_PAIR_MIN (default 1)
 * times as many pairs as the DP launch has warps (a batch too small to fill the GPU
 * keeps its jobs single: a pair's unit of work is longer than a job's); enable = 2
 * pairs every eligible job.  Results are the same either way.
 * pl_engine_last_pairs: pairs formed in the last batch. */
void pl_engine_set_pairing(pl_engine_t *e, int32_t enable);
int32_t pl_engine_last_pairs(const pl_engine_t *e);
/* A batch whose launch plan has the same shape as the previous batch's (the same
 * job count, waves, launch groups, buffers and options: a repeated batch, or one
 * batch size fed again and again) is captured into a CUDA graph and, while the
 * shape recurs, replayed from it; untimed calls only (on by default;
 * PLGPU_GRAPHS=0 or pl_engine_set_graphs(e, 0) turns it off).
 * pl_engine_graph_replays: batches launched from a captured graph so far. */
void pl_engine_set_graphs(pl_engine_t *e, int32_t enable);
int64_t pl_engine_graph_replays(const pl_engine_t *e);

/* ---------------------------------------------------------------------------
 * Several GPUs for one batch (no counterpart in the reference, whose queue
 * drives one device, nasw-cuda.cu:516-576).  Jobs are independent, so a batch
 * shards with no exchange inside a DP: pl_group_plan assigns each job to a
 * device slot (by decreasing DP cells, each to the slot with the fewest cells
 * so far), one host thread per device runs its share on that device's engine,
 * and pl_group_gather writes results and CIGARs back in the caller's job order,
 * CIGARs dense from cigar[0] as pl_splice_batch_host writes them (a job whose
 * words pass cigar_cap gets status -2).  The planner and the gather are plain
 * host functions.
 * ------------------------------------------------------------------------- */
typedef struct pl_group_s pl_group_t;
pl_group_t *pl_group_create(const int32_t *devices, int32_t n_devices, int64_t trace_budget_bytes);
void pl_group_destroy(pl_group_t *g);
/* The engine of device slot `slot` (for tuning or timing), NULL outside the group. */
pl_engine_t *pl_group_engine(pl_group_t *g, int32_t slot);
/* pl_splice_batch_host over the group; *total_cigar (optional) = words written. */
int pl_group_splice_host(pl_group_t *g, const ns_opt_t *opt, const pl_splice_job_t *jobs, int32_t n_jobs,
		const uint8_t *nt, int64_t nt_len, const uint8_t *aa, int64_t aa_len, const uint8_t *ss, int64_t ss_len,
		pl_splice_result_t *results, uint32_t *cigar, int64_t cigar_cap, int64_t *total_cigar);
/* dev_of_job[q] = device slot of job q; cells_of_dev (optional, n_devices) = DP cells per slot. */
int pl_group_plan(const pl_splice_job_t *jobs, int32_t n_jobs, int32_t n_devices, int32_t *dev_of_job,
		int64_t *cells_of_dev);
/* Reassembly: dev_results[d] holds slot d's results in the order of its jobs
 * (cigar_off into dev_cigar[d]); writes results/cigar in job order. */
int pl_group_gather(int32_t n_jobs, const int32_t *dev_of_job, int32_t n_devices,
		const pl_splice_result_t *const *dev_results, const uint32_t *const *dev_cigar,
		pl_splice_result_t *results, uint32_t *cigar, int64_t cigar_cap, int64_t *total_cigar);

/* Allocation-free variant of pl_splice_batch_device() -- no counterpart in the
 * reference.  For callers that cannot allocate device memory on this path: a
 * program that gives all free device memory to its own pool and runs under that
 * fixed budget, or a latency-sensitive loop that cannot take the device-wide
 * synchronisation of cudaMalloc/cudaFree.  Inputs and outputs are the caller's
 * device pointers; all scratch comes from one fixed 96 MiB device array that the
 * library reserves at load time on every GPU it is used on.  Limits per call:
 * at most 4096 jobs, proteins of at most 2048 residues, and scratch (about 2
 * bytes per DP cell) within the array -- larger batches are rejected with a
 * message (pl_noalloc_error) before any GPU work.  Calls share the array: the
 * function returns only after its stream has finished and holds a library lock
 * for its whole duration, so calls never overlap on the GPU.  The first call on
 * a device looks up the array's address and caches it; make it before any
 * stream capture begins.  The cached address dies with the device's context:
 * after cudaDeviceReset() the entry point must not be called again.  Returns 1
 * on success. */
int pl_splice_batch_noalloc(const ns_opt_t *opt, const pl_splice_job_t *jobs, int32_t n_jobs,
		const uint8_t *nt, const uint8_t *aa, const uint8_t *ss,
		pl_splice_result_t *results_dev, uint32_t *cigar_dev, int64_t cigar_cap,
		int64_t *total_cigar, void *stream);
const char *pl_noalloc_error(void);

/* Kernel launches issued by this library since load (all entry points). */
uint64_t pl_kernel_launch_count(void);

/* ---------------------------------------------------------------------------
 * Batched extension DP (replaces nasw-ext-gpu.c and nasw-ext-kernel.h).
 * Results equal ns_global_gs16b() (nasw-sse.c:763-772) with the request's
 * NS_F_EXT_LEFT / NS_F_EXT_RIGHT flag exactly: nt_len, aa_len and score of the
 * x-drop extension, no CIGAR.  A request without an extension flag gets the
 * plain global score H(nl-1, al-1) with nt_len = nl, aa_len = al, as
 * ns_global_gs16b returns it without NS_F_CIGAR.  Every request runs on the
 * device: position-specific scores (ns_opt_t.pssm), any protein length and
 * mixed left/right requests included; requests with nl < 3 get the
 * reference's no-row answer (nt_len 0) without a DP.
 * ------------------------------------------------------------------------- */
/* nasw.h:203 -- NULL when no device is usable (the caller then runs the CPU). */
ns_ext_batch_t *ns_ext_batch_init(void *km);
/* nasw.h:204 -- queue one request; returns its id.  Pointers must stay valid
 * until the result has been fetched. */
int32_t ns_ext_batch_add(ns_ext_batch_t *b, const char *ns, int32_t nl, const char *as, int32_t al,
		const ns_opt_t *opt, const uint8_t *ss);
/* nasw.h:205 -- hand the queued requests to the device; does not wait.
 * Returns the number submitted. */
int32_t ns_ext_batch_flush(ns_ext_batch_t *b);
/* nasw.h:206 -- 1 when request `id` has completed (non-blocking). */
int ns_ext_batch_ready(ns_ext_batch_t *b, int32_t id);
/* nasw.h:207 -- sleep until some outstanding flush of b completes. */
void ns_ext_batch_wait(ns_ext_batch_t *b);
/* nasw.h:208 -- block until request `id` is done; the result stays valid until
 * a later flush after every result of its flush was fetched.  NULL when the
 * request failed: its device batch failed, or host memory ran out while it was
 * queued or flushed (ns_ext_batch_ready() is then 1 for it).  There is no CPU
 * fallback, so the caller must check: the error text is in ns_gpu_error() and
 * pl_last_error(), and pl_ext_failed_count() counts the failed requests.  The
 * executor keeps serving later flushes after a failure. */
const ns_rst_t *ns_ext_batch_get(ns_ext_batch_t *b, int32_t id);
/* Requests of the batch objects that failed on the device (monotonic). */
uint64_t pl_ext_failed_count(void);
/* nasw.h:209 -- waits for b's outstanding flushes, then frees b. */
void ns_ext_batch_destroy(ns_ext_batch_t *b);
/* nasw.h:210-211 -- kernel launches of the extension path / requests run on the device. */
uint64_t ns_ext_gpu_launch_count(void);
uint64_t ns_ext_gpu_request_count(void);

/* Bulk extension entry points (no counterpart in the reference, which only has
 * the batch object above).  One job per request inside packed buffers. */
typedef struct {
	int64_t nt_off;    /* nucleotides in the packed nt buffer (ASCII or 0-4 codes) */
	int64_t aa_off;    /* residues in the packed protein buffer (ASCII) */
	int64_t ss_off;    /* splice-score track in the ss buffer, -1 = none */
	int64_t pssm_off;  /* al x 22 int8 position-specific scores in the pssm buffer (query order), -1 = none */
	int32_t nl, al;
	int32_t flag;      /* NS_F_EXT_LEFT, NS_F_EXT_RIGHT, or 0 for the plain global score */
	int32_t width;     /* stripe width of the CPU kernel being matched: 8, 16, or 0 = pl_ext_stripe_width() */
} pl_ext_job_t;
typedef struct {
	int32_t nt_len, aa_len, score;
	int32_t status;    /* 0 = ok; <0 = error (see pl_last_error()) */
} pl_ext_result_t;
/* Stripe width the reference CPU kernel uses on this host (nasw-sse.c:744-750):
 * 16 for extension requests with al >= 16 when the CPU has AVX2, else 8.  The
 * environment variable PLGPU_EXT_STRIPE=8 or 16 overrides the CPU probe (to
 * match a reference built with no_avx2=1, or results from another machine). */
int32_t pl_ext_stripe_width(const ns_opt_t *opt, int32_t al);
/* Host buffers in, host results out.  opt->flag's extension bits and opt->pssm
 * are ignored: every job carries its own.  Returns 1 on success. */
int pl_ext_batch_host(pl_engine_t *e, const ns_opt_t *opt, const pl_ext_job_t *jobs, int32_t n_jobs,
		const uint8_t *nt, int64_t nt_len, const uint8_t *aa, int64_t aa_len, const uint8_t *ss, int64_t ss_len,
		const int8_t *pssm, int64_t pssm_len, pl_ext_result_t *results);
/* Device-resident inputs and results (job table on the host); work is issued
 * on `stream` (NULL = the engine's stream) and the call returns when it has
 * completed.  Returns 1 on success. */
int pl_ext_batch_device(pl_engine_t *e, const ns_opt_t *opt, const pl_ext_job_t *jobs, int32_t n_jobs,
		const uint8_t *nt, const uint8_t *aa, const uint8_t *ss, const int8_t *pssm,
		pl_ext_result_t *results_dev, void *stream);
/* ---------------------------------------------------------------------------
 * Integer profile-HMM DP (replaces hmm-gpu.c; semantics of mp_hmm_dp_score,
 * hmm.c:252-291): one profile, many regions of nt4 codes, one frame-0 codon
 * per DP row, score = the maximum M or I value (int32, exact).
 * ------------------------------------------------------------------------- */
/* mppriv.h:132 -- score n regions (nt + off[k], len[k] nucleotides) against h;
 * 1 = every score[k] filled with exactly mp_hmm_dp_score(h, nt + off[k],
 * len[k]), 0 = not taken (no device, or the host program lacks hmm.c's
 * accessors).  h's device tables are built on first use and cached in its GPU
 * slot (mp_hmm_gpu_slot(h, 0), hmm.c:215) until mp_hmm_gpu_release().
 * Thread-safe (calls are serialised on one device queue). */
int mp_hmm_dp_score_gpu_batch(const mp_hmm_t *h, int32_t n, const uint8_t *nt, int64_t l_nt,
		const int32_t *off, const int32_t *len, int32_t *score);
/* mppriv.h:129 -- one region; INT32_MIN when not taken or nlen < 3. */
int32_t mp_hmm_dp_score_gpu(const mp_hmm_t *h, const uint8_t *nt, int32_t nlen);
/* mppriv.h:134 -- free h's cached device tables (mp_hmm_destroy calls it, hmm.c:207-212). */
void mp_hmm_gpu_release(mp_hmm_t *h);

/* Bulk profile-HMM entry points (no counterpart in the reference).  A profile
 * is given as the reference parser's tables (hmm.c:112-195): emit m x 20 int16
 * in HMMER column order ACDEFGHIKLMNPQRSTVWY, trans m x 7 int16 (m->m, m->i,
 * m->d, i->m, i->i, d->m, d->d), and codon_alpha[64]: for codon b0<<4|b1<<2|b2
 * the HMMER column of its amino acid, 20 for a stop codon (ns_tab_codon through
 * mp_hmm_aa20_to_alpha, hmm.c:229-250). */
typedef struct pl_hmm_profile_s pl_hmm_profile_t;
pl_hmm_profile_t *pl_hmm_profile_create(int32_t device, int32_t m, const int16_t *emit, const int16_t *trans,
		const uint8_t *codon_alpha);
void pl_hmm_profile_destroy(pl_hmm_profile_t *p);
/* Host buffers: nt (l_nt nucleotide codes 0-4), off/len/score arrays of n regions.  Returns 1 on success. */
int pl_hmm_score_host(pl_engine_t *e, const pl_hmm_profile_t *p, int32_t n, const uint8_t *nt, int64_t l_nt,
		const int32_t *off, const int32_t *len, int32_t *score);
/* Device nt and scores; off/len on the host (they drive the planning).  Work on
 * `stream` (NULL = the engine's); returns when done.  Returns 1 on success. */
int pl_hmm_score_device(pl_engine_t *e, const pl_hmm_profile_t *p, int32_t n, const uint8_t *nt,
		const int32_t *off, const int32_t *len, int32_t *score_dev, void *stream);
/* n_prof profiles against one set of n regions (device nt; off/len on the host):
 * score_dev[k * n + q] = profile k on region q.  The region tables are planned, uploaded
 * and translated once, and the profiles' launches run side by side on the engine's HMM
 * streams (a region set that fills only part of the GPU per profile then keeps it busy).
 * Returns when done; 1 on success. */
int pl_hmm_score_many_device(pl_engine_t *e, const pl_hmm_profile_t *const *ps, int32_t n_prof, int32_t n,
		const uint8_t *nt, const int32_t *off, const int32_t *len, int32_t *score_dev, void *stream);
/* The same from host buffers (nt of l_nt bytes uploaded once; score: n_prof x n). */
int pl_hmm_score_many_host(pl_engine_t *e, const pl_hmm_profile_t *const *ps, int32_t n_prof, int32_t n,
		const uint8_t *nt, int64_t l_nt, const int32_t *off, const int32_t *len, int32_t *score);
/* DP cells (codon rows x m) of the last HMM batch of this engine. */
int64_t pl_hmm_last_cells(const pl_engine_t *e);

/* ---------------------------------------------------------------------------
 * Gapless X-drop candidate prefilter (replaces ns_gapless_xdrop_batch and its
 * entry points, nasw-cuda.cu:1151-1395; scores bit-exact).
 * ------------------------------------------------------------------------- */
/* nasw.h:171 -- 1: this library always has the kernel. */
int ns_gpu_gapless_supported(void);
/* nasw.h:172 -- forget the resident genome; the next batch re-uploads it. */
void ns_gpu_gapless_reset_target(void);
/* nasw.h:170 -- batches, candidates, anchors and seed positions (anchors x block_width) so far. */
void ns_gpu_gapless_profile(ns_gpu_gapless_profile_t *profile);
/* nasw.h:176-181 -- scores[i] = candidate i's gapless score, INT32_MIN when no anchor
 * gave a usable seed.  packed_nt: 4-bit codes, 2 bases per byte, low nibble first;
 * queries: aa20 codes; score_matrix: asize x asize; codon: 64 aa20 codes.  Needs
 * ns_gpu_init() first; returns 0 on failure (ns_gpu_error() says why).  The genome
 * stays resident while the caller passes the same pointer and length.  Thread-safe
 * (calls are serialised). */
int ns_gpu_gapless_score_batch(const uint8_t *packed_nt, int64_t packed_nt_bases,
		const uint8_t *queries, int64_t query_aa,
		const ns_gpu_gapless_candidate_t *candidates, int32_t n_candidates,
		const ns_gpu_gapless_anchor_t *anchors, int64_t n_anchors,
		int32_t block_width, int32_t kmer, int32_t xdrop,
		const int8_t *score_matrix, int32_t asize, const uint8_t *codon,
		int32_t *scores);
/* Bulk gapless entry points (no counterpart in the reference): the same scoring on
 * an engine, without the genome cache.  _host takes host buffers; _device takes
 * device pointers for the genome, queries, candidates, anchors and scores (matrix
 * and codon table on the host) and runs on `stream` (NULL = the engine's).  Limits:
 * block_width <= 8192, kmer <= 64, 21 <= asize <= 32.  Return 1 on success. */
int pl_gapless_score_host(pl_engine_t *e, const uint8_t *packed_nt, int64_t packed_nt_bases,
		const uint8_t *queries, int64_t query_aa, const ns_gpu_gapless_candidate_t *candidates, int32_t n_candidates,
		const ns_gpu_gapless_anchor_t *anchors, int64_t n_anchors, int32_t block_width, int32_t kmer, int32_t xdrop,
		const int8_t *score_matrix, int32_t asize, const uint8_t *codon, int32_t *scores);
int pl_gapless_score_device(pl_engine_t *e, const uint8_t *packed_nt, int64_t packed_nt_bases,
		const uint8_t *queries, int64_t query_aa, const ns_gpu_gapless_candidate_t *candidates, int32_t n_candidates,
		const ns_gpu_gapless_anchor_t *anchors, int64_t n_anchors, int32_t block_width, int32_t kmer, int32_t xdrop,
		const int8_t *score_matrix, int32_t asize, const uint8_t *codon, int32_t *scores_dev, void *stream);
/* Extension steps (both sides, all anchors) walked by the last gapless batch of this engine. */
int64_t pl_gapless_last_steps(const pl_engine_t *e);

/* ---------------------------------------------------------------------------
 * Recheck Forward score (no C ABI in the reference: rc_score is static in
 * recheck.c:283-440 and runs from its kt_for worker, recheck.c:546-568).
 * Multihit-local Forward in log space, float, with the optional null2
 * (ByExpectation) bias correction: bits = (fwd - null1 - bias) / ln 2 and the
 * bias in bits, the two numbers rc_score returns.  Every float step follows
 * rc_score's order, and rc_logsum's expf / log1pf are the host glibc's
 * algorithms restated, so the results equal the reference's bit for bit
 * whenever the reference runs on an x86-64 glibc 2.39 host with FMA (the only
 * steps left to the device are the double-precision exp/log of the bias,
 * whose results are rounded to float).
 * ------------------------------------------------------------------------- */
/* ---- Seeding (the sketch and anchor stages of mp_map_coarse, map.c:565-572) ----
 * The mapper's k-mer index (mp_idx_t's ki: the first kb entry of every bucket, n_bucket
 * = 1 << (4 kmer - mod_bit) of them; kb: the block ids, index.c:74-98) copied to a
 * device; kmer 1-7 (at 8 the reference's 32-bit k-mer mask is an undefined shift).  NULL
 * on bad sizes or a device failure (pl_last_error). */
typedef struct pl_seed_index_s pl_seed_index_t;
pl_seed_index_t *pl_seed_index_create(int32_t device, const int64_t *ki, int64_t n_bucket, const uint32_t *kb,
		int64_t n_kb, int32_t kmer, int32_t mod_bit);
void pl_seed_index_destroy(pl_seed_index_t *x);
/* The anchors of n proteins (seq: letters or residue codes 0-21, protein q at seq[off[q]],
 * len[q] bytes) in the mapper's default mode: mp_sketch_prot's seeds (sketch.c:18-37), the
 * occurrence cap of mp_cal_max_occ limited by max_occ (map.c:304-320, :566-569), every
 * block of every seed whose bucket holds at most the cap (mp_collect_anchors without the
 * accuracy mode's repeat rescue, map.c:346-397), sorted ascending (map.c:571).  Fills
 * a_off[0..n] (protein q's anchors at a[a_off[q] .. a_off[q+1]), block << 32 | position)
 * and returns the total; a is written only when the total fits a_cap (call again with a
 * larger array otherwise).  -1 on a bad argument or a device failure (pl_last_error); a batch
 * is limited to 2^31 - 1 residues and as many anchors. */
int64_t pl_seed_anchors_host(pl_engine_t *e, const pl_seed_index_t *x, int32_t n, const uint8_t *seq, int64_t seq_len,
		const int64_t *off, const int32_t *len, int32_t max_occ, int64_t *a_off, uint64_t *a, int64_t a_cap);
/* The same with the options of mp_collect_anchors (map.c:346-397): max_occ (opt->max_occ);
 * repeat_cap > 0 turns on the accuracy mode's repeat rescue (MP_F_ACCURACY with
 * MP_ACC_REPEAT_RESCUE: opt->acc_repeat_cap, opt->acc_anchor_budget), which needs every
 * protein's query-name hash (pl_seed_qname_hash of its name, as mp_hash_qname). */
typedef struct {
	int32_t max_occ, repeat_cap;
	int64_t anchor_budget;
	const uint32_t *qname_hash;
} pl_seed_opt_t;
int64_t pl_seed_anchors_opt_host(pl_engine_t *e, const pl_seed_index_t *x, int32_t n, const uint8_t *seq,
		int64_t seq_len, const int64_t *off, const int32_t *len, const pl_seed_opt_t *opt, int64_t *a_off, uint64_t *a,
		int64_t a_cap);
/* The same with the anchors left on the device: *a_dev points at them (engine memory,
 * valid until the engine's next seeding call; NULL when there are none), a_off is filled
 * on the host.  They can go to pl_chain_fill_device as they are (its off = a_off, n =
 * a_off[q+1] - a_off[q]). */
int64_t pl_seed_anchors_opt_device(pl_engine_t *e, const pl_seed_index_t *x, int32_t n, const uint8_t *seq,
		int64_t seq_len, const int64_t *off, const int32_t *len, const pl_seed_opt_t *opt, int64_t *a_off,
		const uint64_t **a_dev);
/* HMM-profile queries, as mp_map_hmm_file maps one (map.c:1184-1196): the protein is the
 * profile's consensus (hmm.c:181-189, the first column of the largest emission per match
 * state), and per protein its profile's match emissions give the profile-derived seeds of
 * mp_sketch_hmm (sketch.c:40-118), merged with the protein's own, sorted and deduplicated
 * (mp_sketch_query with a profile, map.c:332-343) before the cap and the anchors.
 * seed_max <= 0: the protein's own seeds only (as the reference, which then has nothing to
 * merge).  The rescue of opt applies as in pl_seed_anchors_opt_host. */
typedef struct {
	const int16_t *emit;    /* 20 int16 per match state, HMMER column order ACDEFGHIKLMNPQRSTVWY
	                           (mp_hmm_emissions) */
	int64_t n_state;        /* match states in emit */
	const int64_t *e_off;   /* protein q's profile: states e_off[q] .. e_off[q] + e_len[q] - 1 */
	const int32_t *e_len;
	int32_t pos_loss;       /* hmm_seed_pos_loss (options.c:112: 6) */
	int32_t win_loss;       /* hmm_seed_win_loss (options.c:113: 8) */
	int32_t seed_max;       /* hmm_seed_max for the coarse stage (options.c:114: 16) */
	int32_t pad;
} pl_seed_hmm_t;
/* as pl_seed_anchors_opt_host / _device; a batch's seed slots (each protein's length plus
 * min(seed_max, 4^kmer) per window of its profile) must stay within INT32_MAX */
int64_t pl_seed_anchors_hmm_host(pl_engine_t *e, const pl_seed_index_t *x, int32_t n, const uint8_t *seq,
		int64_t seq_len, const int64_t *off, const int32_t *len, const pl_seed_opt_t *opt, const pl_seed_hmm_t *h,
		int64_t *a_off, uint64_t *a, int64_t a_cap);
int64_t pl_seed_anchors_hmm_device(pl_engine_t *e, const pl_seed_index_t *x, int32_t n, const uint8_t *seq,
		int64_t seq_len, const int64_t *off, const int32_t *len, const pl_seed_opt_t *opt, const pl_seed_hmm_t *h,
		int64_t *a_off, const uint64_t **a_dev);
/* mp_hash_qname (map.c:322-329) of a query name */
uint32_t pl_seed_qname_hash(const char *qname);

typedef struct pl_rc_profile_s pl_rc_profile_t;
/* A search profile as recheck.c builds it (rc_prof_t, recheck.c:66-72): msc
 * M x 21 match log-odds in nats (column 20 = degenerate residue), tsc M x 8
 * transitions in the order MM, IM, DM, BM, MI, II, MD, DD (recheck.c:74).
 * M <= 2048. */
pl_rc_profile_t *pl_rc_profile_create(int32_t device, int32_t M, const float *msc, const float *tsc);
void pl_rc_profile_destroy(pl_rc_profile_t *p);
/* Score n peptides: peptide q is dsq[off[q] .. off[q]+len[q]) (residue codes
 * 0-19 in HMMER order ACDEFGHIKLMNPQRSTVWY, 20 = other, as recheck.c:52-62
 * encodes them; len >= 1) against profiles[prof_id[q]].  do_null2 as recheck's
 * default (its -n option turns it off); pairs above 2^25 cells skip it, as
 * recheck.c:273 does.  Host buffers; returns 1 on success. */
int pl_rc_score_host(pl_engine_t *e, const pl_rc_profile_t *const *profiles, int32_t n_prof, int32_t n,
		const int32_t *prof_id, const uint8_t *dsq, int64_t dsq_len, const int64_t *off, const int32_t *len,
		int32_t do_null2, float *bits, float *bias);
/* DP cells (sum of L*M) of the last recheck batch of this engine. */
int64_t pl_rc_last_cells(const pl_engine_t *e);
/* Self-check of the Forward's transcendental steps: evaluates on the device
 * fn 0 = expf, 1 = log1pf (the restated glibc algorithms), 2 / 3 = their
 * branch-free forms for rc_logsum's ranges (|x| < 88, 0 <= x <= 1) and 4 / 5 =
 * the four-wide forms of those, which the Forward runs, at the n floats whose bit
 * patterns are lo, lo + stride, lo + 2*stride, ... and copies the results to the
 * host array out.  Allocates device memory per call; returns 1 on success. */
int pl_rc_mathf_eval(int32_t device, int32_t fn, uint32_t lo, uint32_t stride, int64_t n, float *out);
/* Test hook (no counterpart in the reference): the clock-cycle limit of the waits
 * between the warps of a recheck Forward group, for every later call of the process;
 * 0 restores the default (some seconds).  A wait that runs out makes the call fail
 * (pl_rc_score_host returns 0, pl_last_error says so) without faulting the device:
 * the group's warps leave their loops and the kernel ends.  Returns 1. */
int pl_rc_debug_wait_limit(int64_t cycles);

/* DP cells of the last extension batch: the rows the reference's row loop
 * visits (up to the x-drop row, nasw-sse.c:361-447) times al, and the nominal
 * (nl-2)*al. */
void pl_ext_last_cells(const pl_engine_t *e, int64_t *cells_run, int64_t *cells_nominal);

/* ---------------------------------------------------------------------------
 * Learned candidate prefilter (augments the candidate selection of
 * map.c:1014-1089 / hit.c:217-263; no reference counterpart).  A 4-layer BF16
 * MLP (in_dim -> hidden x 3 -> 16, ReLU) on the tensor cores predicts from a
 * candidate's features whether the exact spliced DP over its window will pass
 * (output column 0, a logit) and where the alignment lies in the window
 * (columns 1-2, start and end as fractions of the window).  Kept candidates
 * still get every reported alignment from the exact DP.
 * ------------------------------------------------------------------------- */
#define PL_PF_FDIM 576
typedef struct pl_pf_model_s pl_pf_model_t;
/* in_dim: a multiple of 64 (PL_PF_FDIM for pl_pf_features_device rows); hidden 128 or 256. */
pl_pf_model_t *pl_pf_model_create(int32_t device, int32_t in_dim, int32_t hidden, uint64_t seed);
void pl_pf_model_destroy(pl_pf_model_t *m);
/* parameters as fp32, layer by layer: W [out x in] row-major then bias [out] */
int64_t pl_pf_model_size(const pl_pf_model_t *m);
int pl_pf_model_get(const pl_pf_model_t *m, float *params, int64_t n);
int pl_pf_model_set(pl_pf_model_t *m, const float *params, int64_t n);
/* Features of n candidates (nt_off, aa_off, nl, al of each job; ss_off ignored) over
 * device buffers nt (the window on the strand the DP reads) and aa (ASCII).
 * feats: bf16 [ceil(n/128)*128 x PL_PF_FDIM] device (pad rows are zeroed);
 * chain: int32 [n x 4] device, the best anchor chain's first/last window position
 * and first/last residue (-1 without a chain). */
int pl_pf_features_device(pl_engine_t *e, const ns_opt_t *opt, const pl_splice_job_t *jobs, int32_t n,
		const uint8_t *nt, const uint8_t *aa, void *feats, int32_t *chain, void *stream);
/* Scores of n candidates: out f32 [ceil(n/128)*128 x 16] device, from feats as above. */
int pl_pf_predict(pl_pf_model_t *m, const void *feats, int64_t n, float *out, void *stream);
/* The learned selector in one call (the hook it serves is the candidate selection
 * of mp_gpu_prefilter_select, map.c:511-532, run from mp_gpu_prefilter_batch,
 * map.c:1014-1089): features and the MLP over n candidates (host job table, nt/aa
 * device buffers), then pl_pf_decide.  prob (optional, host): sigmoid of column 0.
 * Host outputs: keep, fallback, out_jobs.  Returns 1 on success. */
int pl_pf_select_device(pl_pf_model_t *m, pl_engine_t *e, const ns_opt_t *opt, const pl_splice_job_t *jobs,
		int32_t n, const uint8_t *nt, const uint8_t *aa, double tau, int32_t margin, double tau_fb,
		uint8_t *keep, uint8_t *fallback, pl_splice_job_t *out_jobs, float *prob, void *stream);
/* The decision (host only): keep[q] = logit >= logit(tau); a kept candidate's window
 * becomes the union of the predicted span (columns 1-2 of out, clipped to [0, 1],
 * times nl) and the span its best anchor chain implies (chain[4q] minus 3x the
 * residues before chain[4q+2], chain[4q+1] plus 3x those after chain[4q+3]),
 * widened by margin + rel x its length on each side, cut to the window; a span
 * under 3 nt keeps the full window (out_jobs[q]: nt_off / nl moved, the rest
 * copied).  fallback[q] = logit >= logit(tau_fb): a kept candidate whose DP on
 * the cut window does not pass reruns on the full window. */
int pl_pf_decide(int32_t n, const pl_splice_job_t *jobs, const float *out, int64_t out_stride, const int32_t *chain,
		double tau, int32_t margin, double rel, double tau_fb, uint8_t *keep, uint8_t *fallback,
		pl_splice_job_t *out_jobs);
/* `steps` Adam steps on minibatches perm[s*batch .. (s+1)*batch) (s counts steps
 * modulo n_perm / batch) of feats (bf16 rows) and targets (f32 [label, start,
 * end, box weight] rows), device buffers; batch a multiple of 128.  Loss per step
 * into loss_log (host, `steps` floats) when not null. */
int pl_pf_train(pl_pf_model_t *m, const void *feats, const float *targets, const int32_t *perm, int64_t n_perm,
		int32_t batch, int32_t steps, float lr, float pos_weight, float box_weight, float *loss_log, void *stream);
/* One tensor-core GEMM C = A . B^T (+ bias, ReLU, mask), bf16 operands with K
 * contiguous; M % 128 == 0, K % 64 == 0, N and n_tile multiples of 16, n_tile <= 256. */
int pl_pf_gemm(int32_t device, const void *A, int64_t lda, const void *B, int64_t ldb, int32_t M, int32_t N, int32_t K,
		int32_t n_tile, const float *bias, int32_t relu, const void *mask, int64_t ldm, void *C, int64_t ldc, void *CT,
		int64_t ldct, float *Cf, int64_t ldcf, int32_t *err, void *stream);

/* ---------------------------------------------------------------------------
 * Alignment statistics and exon features from the CIGAR (the work of
 * align.c:148-269, mp_extra_cal), batched on the device.
 * ------------------------------------------------------------------------- */
typedef struct {
	int64_t cigar_off;   /* CIGAR words (nasw.h ops) of the alignment in the cigar buffer */
	int64_t nt_off;      /* target bases (0-3 A/C/G/T, 4 N) from the region start r->vs */
	int64_t aa_off;      /* protein (ASCII) from r->qs */
	int64_t pssm_off;    /* position-specific rows (asize wide) from r->qs, or -1: the matrix */
	int64_t l_nt;        /* target bases available from r->vs */
	int64_t vs, ve;      /* r->vs, r->ve */
	int64_t feat_off;    /* first feature slot of this alignment in the feature buffer */
	int32_t qs, qe;      /* r->qs, r->qe */
	int32_t n_cigar;
	int32_t has_stop;    /* r->qe == qlen && r->p->dist_stop == 0 (mp_extra_stop before the call) */
	int32_t feat_cap;    /* feature slots reserved (introns + 2 always suffice) */
	int32_t pad;
} pl_extra_job_t;
/* mp_feat_t (protlocus.h:230-237), layout-identical */
typedef struct {
	int64_t vs, ve;
	int32_t qs, qe;
	int16_t type, phase;      /* type 0: CDS, 1: stop codon */
	int32_t n_fs, n_stop;
	int32_t score, n_iden, blen;
	char donor[2], acceptor[2];
} pl_feat_t;
typedef struct {
	int32_t blen, n_iden, n_plus, n_fs, n_stop, dp_max;  /* the mp_extra_t fields mp_extra_cal sets */
	int32_t n_exon, n_feat;   /* r->n_exon, r->n_feat */
	int32_t ok;               /* 0: the CIGAR's span does not match the region (the reference drops r->p, r->feat) */
	int32_t pad;
} pl_extra_result_t;
/* Host buffers.  go/ge/fs/asize/mat: the mapping options (mp_mapopt_t); codon / aa20:
 * the genetic code and residue tables (ns_tab_codon, ns_tab_aa20). */
int pl_extra_cal_host(pl_engine_t *e, int32_t go, int32_t ge, int32_t fs, int32_t asize, const int8_t *mat,
		const uint8_t *codon, const uint8_t *aa20, const pl_extra_job_t *jobs, int32_t n,
		const uint32_t *cigar, int64_t n_cigar_words, const uint8_t *nt, int64_t l_nt, const uint8_t *aa, int64_t l_aa,
		const int8_t *pssm, int64_t l_pssm, pl_extra_result_t *results, pl_feat_t *feats, int64_t n_feat_slots);
/* Device-resident variant: cigar, nt, aa, pssm, results and feats are device
 * pointers (the offsets of jobs index them as in the host call; the caller
 * guarantees that every job's spans lie inside its buffers); the job table and the
 * tables are host memory.  Work is issued on `stream` (NULL = the engine's) and the
 * call returns when it has completed. */
int pl_extra_cal_device(pl_engine_t *e, int32_t go, int32_t ge, int32_t fs, int32_t asize, const int8_t *mat,
		const uint8_t *codon, const uint8_t *aa20, const pl_extra_job_t *jobs, int32_t n, const uint32_t *cigar,
		const uint8_t *nt, const uint8_t *aa, const int8_t *pssm, pl_extra_result_t *results, pl_feat_t *feats,
		void *stream);

/* ---------------------------------------------------------------------------
 * Prescreen banded gapped alignment (prescreen.c:346-382, ps_gapped) of many
 * (profile, ORF, diagonal) candidates: local affine-gap alignment of the profile's
 * PSSM (L rows x 22 int8) against the ORF's residue codes (0-21) within
 * |t - i - diag| <= band (band <= 0: full), score only.
 * ------------------------------------------------------------------------- */
typedef struct {
	int64_t pssm_off;    /* first byte of the L x 22 rows in the pssm buffer */
	int64_t orf_off;     /* first residue code of the ORF in the orf buffer */
	int32_t L, n;        /* profile length, ORF length */
	int32_t diag, band;  /* ps_cand_t.diag, mp_psopt_t.band */
} pl_ps_job_t;
/* Cells of one candidate's banded DP (rows [0, L), ORF positions within band of
 * row + diag, clipped to [0, n); the whole L x n matrix when band <= 0): the count
 * the timing counters report. */
int64_t pl_ps_band_cells(int32_t L, int32_t n, int32_t diag, int32_t band);
int pl_ps_gapped_host(pl_engine_t *e, const pl_ps_job_t *jobs, int32_t n, const int8_t *pssm, int64_t l_pssm,
		const uint8_t *orf, int64_t l_orf, int32_t go, int32_t ge, int32_t *scores);
/* Device-resident variant: pssm, orf and scores are device pointers; the caller
 * guarantees the spans and that every residue code is 0..21 (the host call checks
 * both).  The job table is host memory; returns when the work has completed. */
int pl_ps_gapped_device(pl_engine_t *e, const pl_ps_job_t *jobs, int32_t n, const int8_t *pssm, const uint8_t *orf,
		int32_t go, int32_t ge, int32_t *scores, void *stream);

/* ---------------------------------------------------------------------------
 * Anchor chaining (chain.c:160-219, mp_chain) of many queries at once.  A
 * query's anchors are blockId << 32 | queryPos, sorted ascending, as mp_chain
 * takes them; the arguments of mp_chain are the fields of pl_chain_opt_t.  The
 * chaining DP (the score f, predecessor p and peak v of every anchor,
 * chain.c:183-208) runs on the device, one warp per query; the backtrack and
 * compaction (chain.c:8-110) run on the host's cores.
 * ------------------------------------------------------------------------- */
typedef struct {
	int32_t max_dist_x, max_dist_y, bw, max_skip, max_iter, min_cnt, min_sc;
	float chn_coef_log;
	int32_t is_spliced, kmer, bbit, pad;
} pl_chain_opt_t;

/* Host buffers.  Query q's anchors are a[off[q] .. off[q] + n[q]) of the n_a in
 * `a`.  Out, per query: n_u[q] chains (score << 32 | #anchors, mp_chain's u[])
 * at u + off[q] and the chained anchors in mp_chain's output order at
 * a_out + off[q]; each region holds up to n[q] words.  Returns 1 on success. */
int pl_chain_host(pl_engine_t *e, const pl_chain_opt_t *opt, int32_t n_q, const int64_t *off, const int32_t *n,
		const uint64_t *a, int64_t n_a, uint64_t *u, int32_t *n_u, uint64_t *a_out);

/* The chaining DP alone on device buffers (a_dev, f/p/v out, one int32 each per
 * anchor; p = -1 where no predecessor), issued on `stream` (NULL = the engine's
 * own); off and n are host arrays.  Returns once the DP has completed: the kernel
 * checks every index it uses and the call fails when one was out of range. */
int pl_chain_fill_device(pl_engine_t *e, const pl_chain_opt_t *opt, int32_t n_q, const int64_t *off,
		const int32_t *n, const uint64_t *a_dev, int64_t n_a, int32_t *f_dev, int32_t *p_dev, int32_t *v_dev,
		void *stream);

/* Predecessor pairs scored by the last fill run with engine timing on. */
int64_t pl_chain_last_pairs(const pl_engine_t *e);

/* The host half for one query: chains from a fill's f and p (no device). */
int pl_chain_finish(const pl_chain_opt_t *opt, int64_t n, const uint64_t *a, const int32_t *f, const int32_t *p,
		uint64_t *u, int32_t *n_u, uint64_t *a_out);

#ifdef __cplusplus
}
#endif

#endif /* PLGPU_H */
