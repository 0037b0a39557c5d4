/*
 * plhost.h -- internals shared by the host translation units of libplgpu
 * (plgpu.c: engine, global DP, request queue; plext.c: extension DP).
 */
#ifndef PLHOST_H
#define PLHOST_H
#include <cuda_runtime_api.h>
#include "plk.h"
#include "../../include/plgpu.h"

#define PL_EXPORT __attribute__((visibility("default")))

#define CK(call) do { cudaError_t _e = (call); if (_e != cudaSuccess) { \
	pl_set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, __LINE__); goto fail; } } while (0)
#define CKK(call) do { int _e = (call); if (_e != 0) { \
	pl_set_error("%s failed: %s", #call, cudaGetErrorString((cudaError_t)_e)); goto fail; } } while (0)

/* grow-only device buffer */
/* host-side fault injection for the failure tests (pl_debug_fault): a site fails once, after
 * a set number of passes; no device work is involved */
enum { PL_FAULT_HOST_ALLOC = 0, PL_FAULT_DEV_ALLOC = 1, PL_FAULT_EXT_BATCH = 2, PL_FAULT_N = 3 };
int pl_fault_hit(int site);
/* 1 when [off, off+len) lies inside a buffer of cap bytes, else 0 with the error text set */
int pl_span_ok(const char *rec, int32_t q, const char *buf, int64_t off, int64_t len, int64_t cap);

typedef struct { void *p; size_t cap; } dbuf_t;
int dbuf_ensure(dbuf_t *b, size_t need);
void dbuf_free(dbuf_t *b);

struct pl_engine_s {
	int device, n_sm, ctas_per_sm[4][2];   /* per DP mode (3: paired int16x2), per rows per lane (8, 4) */
	int pairing;                            /* form int16x2 pairs (PLGPU_PAIR=0 turns it off) */
	int graphs;                             /* capture and replay recurring launch plans (PLGPU_GRAPHS=0: off) */
	uint64_t g_key, g_prev_key;             /* shape of the captured plan, of the previous call's plan */
	cudaGraphExec_t g_exec;
	int64_t g_nlaunch, g_replays;           /* kernel launches in the graph; replays so far */
	int32_t g_dp_launches, g_coop;
	int32_t r4_rows;                        /* jobs with at most this many DP rows take 4 rows per lane */
	double coop_ratio;                      /* cooperative-job threshold (pl_coop_ratio by default) */
	cudaStream_t stream;
	/* second stream of the global DP: when a batch needs several waves, odd waves run
	 * on it with their own trace arena, so a wave's DP fills the tail of the one before */
	cudaStream_t side;
	cudaEvent_t ev_fork, ev_join;
	int64_t trace_budget;
	dbuf_t jobs, order, counters, prep, trace, ring, tmp, total, nt, aa, ss, res, cig;
	/* extension DP */
	dbuf_t x_jobs, x_order, x_counter, x_prep, x_ring, x_nt, x_aa, x_ss, x_pssm, x_res;
	plk_ext_job_t *x_hj;
	int32_t *x_horder, x_m;
	int32_t x_last_launches;
	int64_t x_cells_run, x_cells_nominal;
	/* integer HMM DP */
	dbuf_t h_off, h_len, h_rowoff, h_rows, h_order, h_counter, h_edge, h_nt, h_score;
	/* several profiles at once: concurrent launches on PL_HMM_STREAMS streams, each with its
	 * own queue counter and edge buffer */
#define PL_HMM_STREAMS 4
	cudaStream_t h_st[PL_HMM_STREAMS];
	cudaEvent_t h_ev[PL_HMM_STREAMS + 1];
	dbuf_t h_edge_s[PL_HMM_STREAMS];
	void *h_hbuf;
	size_t h_hcap;
	int64_t h_last_cells;
	/* gapless prefilter */
	dbuf_t g_packed, g_queries, g_cand, g_anchors, g_mat, g_codon, g_scores, g_steps;
	const uint8_t *g_cached_src;   /* host genome currently resident (ns_gpu_gapless_* cache) */
	int64_t g_cached_bases;
	int64_t g_last_steps;
	/* recheck Forward */
	dbuf_t r_prof, r_pep, r_dsq, r_order, r_grp, r_err, r_scratch, r_bits, r_bias;
	/* seeding (plseed.c) */
	dbuf_t s_seq, s_off, s_len, s_seed, s_cnt, s_nseed, s_cap, s_nanc, s_aoff, s_anc, s_anc2, s_tmp;
	dbuf_t s_take, s_send, s_seed2, s_qh;
	dbuf_t s_soff, s_emit, s_eoff, s_elen, s_alts;  /* HMM-profile queries' seed slots and profiles */
	int64_t r_last_cells;
	/* learned-prefilter features */
	dbuf_t pf_cand, pf_feats, pf_chain, pf_out;
	void *pf_host;          /* the selector's chain and score rows read back (grow-only) */
	size_t pf_host_cap;
	/* alignment statistics / exon features */
	dbuf_t f_jobs, f_cig, f_nt, f_aa, f_pssm, f_mat, f_res, f_feat;
	/* prescreen banded alignment */
	dbuf_t s_jobs, s_pssm, s_orf, s_scr, s_score, s_order;
	/* anchor chaining */
	dbuf_t c_off, c_n, c_order, c_a, c_f, c_p, c_v, c_t, c_counter;
	void *c_host;           /* pinned host buffer for the fill's f and p (grow-only) */
	size_t c_host_cap;
	int64_t c_last_pairs;   /* predecessors scored by the last timed fill */
	/* host planning scratch */
	plk_job_t *hj;
	int32_t *horder, *hwave, m_jobs;
	int32_t last_waves, last_coop, last_dp_launches, last_pairs;
	/* optional CUDA-event timing of the phases: prep, DP, traceback, compaction */
	int timing;
	cudaEvent_t ev[2 + 4 * 64];
	int n_ev;
	unsigned char ev_kind[2 + 4 * 64];
	double acc_ms[4];
	int64_t acc_dp_launches, acc_cells;
};

/* records a timing event of phase k (0 prep, 1 DP, 2 traceback, 3 compaction) when timing is on */
#define PL_TIME(e, st, k) do { if ((e)->timing && (e)->n_ev < (int)(sizeof((e)->ev) / sizeof((e)->ev[0]))) { \
	(e)->ev_kind[(e)->n_ev] = (k); cudaEventRecord((e)->ev[(e)->n_ev++], (st)); } } while (0)

void pl_set_error(const char *fmt, ...);
double pl_coop_ratio(void);
int32_t pl_r4_rows(void);
int pl_params(const ns_opt_t *opt, plk_params_t *p, int for_ext);
int pl_max_sub(const ns_opt_t *opt);
void pl_ext_engine_free(pl_engine_t *e);
void pl_hmm_engine_free(pl_engine_t *e);
void pl_gapless_engine_free(pl_engine_t *e);
void pl_rc_engine_free(pl_engine_t *e);
void pl_seed_engine_free(pl_engine_t *e);
void pl_pf_engine_free(pl_engine_t *e);
void pl_feat_engine_free(pl_engine_t *e);
void pl_ps_engine_free(pl_engine_t *e);
void pl_chain_engine_free(pl_engine_t *e);
int pl_ns_device(void);
void pl_ns_set_error(const char *msg);

#endif
