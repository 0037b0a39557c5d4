/*
 * plk.h -- plain-C interface between the host layer (plgpu.c) and the sm_100a
 * kernels (splice.cu).  Only POD structs and C function prototypes; no CUDA
 * types other than the opaque stream handle passed as void*.
 */
#ifndef PLK_H
#define PLK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PLK_WARPS_PER_CTA 8     /* a CTA is one 256-lane wavefront (large jobs) or 8 independent warps */
#define PLK_ROWS 8              /* DP rows owned by one lane of a strip (extension DP) */
/* the global DP gives every lane of a strip PLK_DP_ROWS (8) or 4 rows, chosen per job
 * (plk_job_t.rows): the trace layout, the kernel instance and the traceback follow */
#define PLK_DP_ROWS 8
#define PLK_RING_INTS 12        /* column state handed from one strip to the next (9 used, 48-byte entries) */

/* scoring parameters and lookup tables, passed to kernels by value */
typedef struct {
	int32_t go, ge, io, fs, end_bonus, xdrop;
	int32_t sp[6];
	int32_t sp_null_bonus;
	float ie_coef;
	int8_t sc[22 * 22];
	uint8_t nt4[256], aa20[256], codon[64];
	uint8_t aa_x;               /* aa20['X'] */
	uint8_t pad[3];
	/* the global DP's penalties in its x16 tagged domain (filled by the host so the
	 * kernel reads them as constants): go, ge, io, -fs + 9/8/7/6 (frameshift
	 * candidates 6-9 with their tags), -fs, go + ge */
	int32_t s16[9];
	/* the paired int16x2 DP (mode 3): bias B of its 15-bit domain and the floor F that
	 * stands for the reference's -32768 (set by the host when it forms pairs) */
	int32_t pair_b, pair_f;
	/* the paired DP's trace-bit gather runs as multiply-adds on the FMA pipe, its
	 * multipliers read as kernel constants: 2^0 .. 2^15, and -(2^10 - 1), -2^10 .. -2^15 */
	int32_t pair_pw[16], pair_nw[7];
} plk_params_t;

/* fills plk_params_t.s16 from go/ge/io/fs (every host path that builds parameters calls it) */
static inline void plk_fill_scaled(plk_params_t *p)
{
	int i;
	p->s16[0] = 16 * p->go, p->s16[1] = 16 * p->ge, p->s16[2] = 16 * p->io;
	for (i = 0; i < 4; ++i) p->s16[3 + i] = -16 * p->fs + 9 - i;
	p->s16[7] = -16 * p->fs, p->s16[8] = 16 * (p->go + p->ge);
	for (i = 0; i < 16; ++i) p->pair_pw[i] = 1 << i;
	p->pair_nw[0] = -((1 << 10) - 1);
	for (i = 0; i < 6; ++i) p->pair_nw[1 + i] = -(1 << (10 + i));
}

/* per-job metadata, device resident */
typedef struct {
	int64_t nt_off, aa_off, ss_off;  /* inputs (ss_off < 0: no splice-score track) */
	int64_t prep_off;                /* nas[nl] | aas[al] | donor[nl+1] | acceptor[nl+1], 8-aligned */
	int64_t trace_off;               /* first trace word (uint16) of this job in the wave arena */
	int64_t tmp_off;                 /* reversed CIGAR scratch (uint32 words), capacity nl+al+8 */
	int64_t out_off;                 /* final CIGAR offset in the output buffer (filled by the scan) */
	int32_t nl, al;
	int32_t mode;                    /* 0: int16 (lower clamp suffices), 1: int32 (gs32b), 2: int16 both clamps,
	                                  * 3: int16 paired with a job of the same protein and window length */
	int32_t slen;                    /* segment length of the striping being reproduced */
	int32_t nw;                      /* warps cooperating on the job: 1 or PLK_WARPS_PER_CTA */
	int32_t rows;                    /* DP rows per lane of a strip: 8 or 4 */
	int32_t score, n_tmp;            /* outputs of the DP / traceback */
	int32_t status;
	int32_t pair;                    /* mode 3: the partner job's index in the first job of a pair, -1 in the second */
} plk_job_t;

/* per-request metadata of the extension DP, device resident */
typedef struct {
	int64_t nt_off, aa_off, ss_off;  /* inputs (ss_off < 0: no splice-score track) */
	int64_t pssm_off;                /* al x 22 position-specific scores in query order (< 0: none) */
	int64_t prep_off;                /* nas[nl] | aas[al] | donor[nl+1] | acceptor[nl+1] */
	int32_t nl, al;
	int32_t left;                    /* 0: right extension, 1: left (reversed inputs), 2: plain global score */
	int32_t slen, ncol;              /* stripe segment length and padded column count slen*width */
	int32_t mode;                    /* 0: int16 lower clamp only, 2: both clamps */
	int32_t variant;                 /* bit 0: position-specific scores, bit 1: wide row keys */
	int32_t nt_len, aa_len, score;   /* outputs */
	int32_t status;                  /* 0 = ok */
	int32_t pad;
} plk_ext_job_t;

/* a profile of the integer HMM DP on the device (hmm.c:14-22 tables, re-laid out) */
typedef struct {
	const int16_t *emit_t;   /* [21][mpad]: emissions by HMMER column (row 20: zeros, no emission), column j-1 */
	const int32_t *trans_t;  /* [7][mpad]: m->m, m->i, m->d, i->m, i->i, d->m, d->d of column j-1; -2^28 beyond m */
	int32_t m, mpad;         /* profile length, padded to the 256-column tile */
} plk_hmm_prof_t;
#define PLK_HMM_TILE 256
#define PLK_HMM_SMEM_MAX (96 * 1024)  /* emissions staged in shared memory up to mpad = 2048 */

/* bytes after the last job's preparation scratch that the DP may read (its row
 * inputs are copied in whole 16-byte chunks) */
#define PLK_PREP_SLACK 64

/* bytes of preparation scratch for a job (8-aligned) */
static inline int64_t plk_prep_bytes(int32_t nl, int32_t al)
{
	return ((int64_t)nl + al + 2 * ((int64_t)nl + 1) + 7) / 8 * 8;
}

/* trace words of a job in the strip layout (strips of 32*nw*rows rows) */
static inline int64_t plk_trace_words(int32_t nl, int32_t al, int32_t nw, int32_t rows)
{
	int64_t h = 32LL * nw * rows, nr = (int64_t)nl - 2, strips = (nr + h - 1) / h;
	return strips * h * (int64_t)al;
}

/* launchers; all return a cudaError_t value as int */
int plk_prep(const plk_job_t *jobs, int32_t n_jobs, const uint8_t *nt, const uint8_t *aa, const uint8_t *ss,
		uint8_t *prep, const plk_params_t *p, void *stream);
/* order_coop: jobs run by a whole CTA (nw = PLK_WARPS_PER_CTA); order_solo: one warp each.
 * counters: 2 ints of device scratch.  ring: PLK_WARPS_PER_CTA * n_ctas * ring_stride_ints ints. */
int plk_splice_dp(plk_job_t *jobs, const int32_t *order_coop, int32_t n_coop, const int32_t *order_solo,
		int32_t n_solo, int32_t *counters, const uint8_t *prep, uint16_t *trace, int32_t *ring,
		int64_t ring_stride_ints, int32_t n_ctas, int32_t mode, int32_t rows, const plk_params_t *p, void *stream);
int plk_traceback(plk_job_t *jobs, const int32_t *order, int32_t n_order, const uint16_t *trace,
		uint32_t *tmp, void *stream);
int plk_scan_compact(plk_job_t *jobs, int32_t n_jobs, const uint32_t *tmp, uint32_t *out, int64_t out_cap,
		int64_t *total_words, void *result_recs, void *stream);
/* extension DP: preparation in either orientation, then the score-only DP over
 * `order` (one warp per request).  counter: 16 bytes of device scratch -- int32 [0]
 * is the queue position (reset per launch), uint64 at byte 8 accumulates the DP
 * cells run (rows processed x al; reset by the caller); ring:
 * plk_ext_warps_per_cta() * n_ctas * ring_stride_ints ints; pssm: base of the
 * position-specific score buffer (variant bit 0). */
int plk_ext_prep(const plk_ext_job_t *jobs, int32_t n_jobs, const uint8_t *nt, const uint8_t *aa, const uint8_t *ss,
		uint8_t *prep, const plk_params_t *p, void *stream);
int plk_ext_dp(plk_ext_job_t *jobs, const int32_t *order, int32_t n_jobs, int32_t *counter, const uint8_t *prep,
		const int8_t *pssm, int32_t *ring, int64_t ring_stride_ints, int32_t n_ctas, int32_t mode, int32_t variant,
		const plk_params_t *p, void *stream);
int plk_ext_ctas_per_sm(int32_t mode, int32_t variant);
int plk_ext_warps_per_cta(void);
/* results[q] (pl_ext_result_t) from the job table */
int plk_ext_results(const plk_ext_job_t *jobs, int32_t n_jobs, void *results, void *stream);
void plk_add_launches(uint64_t n);
/* integer HMM DP: codon rows of every region, then one warp per region (order) */
int plk_hmm_codons(const uint8_t *nt, const int32_t *off, const int32_t *len, const int64_t *row_off, int32_t n,
		const uint8_t *codon_alpha, uint8_t *rows, void *stream);
int plk_hmm_dp(const plk_hmm_prof_t *p, const uint8_t *rows, const int64_t *row_off, const int32_t *len,
		const int32_t *order, int32_t n, int32_t *counter, void *edge, int64_t edge_stride_rows, int32_t n_ctas,
		int32_t *score, void *stream);
int plk_hmm_ctas_per_sm(int32_t mpad);
int plk_hmm_warps_per_cta(void);
int plk_hmm_smem_bytes(int32_t mpad);
/* gapless prefilter: one warp per candidate; steps accumulates the extension steps walked */
int plk_gapless(const uint8_t *packed, int64_t bases, const uint8_t *queries, int64_t query_aa, const void *cand,
		int32_t n_cand, const void *anchors, int64_t n_anchors, int32_t block_width, int32_t kmer, int32_t xdrop,
		const int8_t *mat_dev, int32_t asize, const uint8_t *codon_dev, int32_t *scores, unsigned long long *steps,
		int32_t n_sm, void *stream);
int plk_gapless_smem_bytes(int32_t block_width, int32_t kmer);

/* profile of the recheck Forward (recheck.c:66-72 search profile): device pointers */
typedef struct {
	const float *msc;   /* [M][21] match log-odds in nats, column 20 = degenerate residue */
	const float *tsc;   /* [M][8] transitions (recheck.c:74 order) */
	int32_t M, pad;
} plk_rc_prof_t;
/* one peptide */
typedef struct {
	int64_t dsq_off;      /* residue codes 0-20 */
	int32_t len, prof, null2, pad;
	/* the per-peptide logarithms of the length model, computed with the host's logf
	 * (recheck.c:289-290, :321, :433-434) so that they carry the host libm's bits */
	float lmove, lloop, logL, null1;
} plk_rc_pep_t;
/* a group: up to 32 peptides of one profile, one per lane of a warp, their DP
 * matrices interleaved by lane in a scratch region of plk_rc_group_floats floats */
typedef struct {
	int64_t scratch_off;  /* float offset of the region, a multiple of 4 */
	int32_t first, count; /* its peptides: order[first .. first + count) */
	int32_t prof, lmax;   /* the profile and the longest peptide */
	int32_t full, pad;    /* full: some peptide takes null2, so every M/I row is kept */
} plk_rc_grp_t;
/* seeding of a batch of proteins (seed.cu) */
typedef struct {
	const uint8_t *seq;          /* the proteins, concatenated (letters or codes 0-21) */
	const int64_t *off;          /* protein q at seq[off[q]], len[q] bytes */
	const int32_t *len;
	int32_t n;
	const int64_t *soff;         /* protein q's seed slots from soff[q] (n + 1 entries; off when
	                                the slots are the residues') */
	const int64_t *ki;           /* the index: bucket starts (n_bucket) and block ids (n_kb) */
	int64_t n_bucket;
	const uint32_t *kb;
	int64_t n_kb;
	int32_t kmer, mod_bit, max_occ;
	int32_t repeat_cap;          /* > 0: the accuracy mode's repeat rescue (map.c:360-384) */
	int64_t budget;              /* its anchor budget */
	const uint32_t *qhash;       /* per protein: the query name's hash (the rescue's start) */
	uint64_t *seeds;             /* per seed slot: the seeds (position order; sorted for the rescue
	                                and for profiles) */
	uint32_t *cnt;               /* per seed slot: the seeds' bucket sizes */
	int32_t *take;               /* per seed slot: the anchors each seed gives */
	int32_t *n_seed, *cap;       /* per protein: seeds, occurrence cap */
	int64_t *seed_end;           /* per protein: soff + n_seed (the seeds' segment for a sort) */
	/* HMM-profile queries (mp_sketch_hmm, sketch.c:40-118): per protein its profile's match
	 * states e_off[q] .. e_off[q] + e_len[q] - 1 of emit (20 int16 each), their offered
	 * groups in alts (sh_alts_t of seed_hmm.cuh, n_state of them) */
	const int16_t *emit;
	int64_t n_state;
	const int64_t *e_off;
	const int32_t *e_len;
	void *alts;
	int32_t pos_loss, win_loss, seed_max, pad1;
	int64_t *n_anchor;           /* per protein: anchors */
	const int64_t *a_off;        /* per protein: first anchor (n + 1 entries) */
	uint64_t *anchors;
} plk_seed_args_t;
int plk_seed_sketch(const plk_seed_args_t *a, void *stream);
int plk_seed_take(const plk_seed_args_t *a, void *stream);
int plk_seed_emit(const plk_seed_args_t *a, void *stream);
/* profiles: every state's offered groups; the windows' seeds appended to each protein's own */
int plk_seed_hmm_alts(const plk_seed_args_t *a, void *stream);
int plk_seed_hmm_enum(const plk_seed_args_t *a, void *stream);
/* the seeds sorted (sorted, soff..seed_end) without duplicates into seeds, their bucket
 * sizes, counts and the occurrence cap (the rest of mp_sketch_query with a profile and
 * mp_cal_max_occ) */
int plk_seed_unique(const plk_seed_args_t *a, const uint64_t *sorted, void *stream);
int plk_seed_sort(const uint64_t *keys_in, uint64_t *keys_out, int64_t n_items, int32_t n_seg, const int64_t *seg_off,
		const int64_t *seg_end, void *tmp, size_t *tmp_bytes, void *stream);
#define PLK_RC_MAX_M 2048
int64_t plk_rc_group_floats(int32_t lmax, int32_t M, int32_t full);
/* err: a device int, set to 1 when a wait between the warps of a group ran out (the
 * launch's results are then invalid); spin_limit: clock cycles a wait may take, 0 the
 * default */
int plk_rc_forward(const plk_rc_prof_t *prof, const plk_rc_pep_t *pep, const uint8_t *dsq, const int32_t *order,
		const plk_rc_grp_t *grp, int32_t n_grp, float *scratch, float *bits, float *bias, int *err,
		int64_t spin_limit, void *stream);
/* CTAs of the DP kernel that fit on one SM at once (occupancy) */
int plk_dp_ctas_per_sm(int32_t mode, int32_t rows);
uint64_t plk_launches(void);

/* BF16 GEMM on the tensor cores (mlp.cu): C = A . B^T + bias, optional ReLU / mask,
 * outputs bf16 row-major, bf16 transposed and/or f32.  Pointers are device memory. */
typedef struct {
	const void *A; int64_t lda;      /* bf16 [M x K] */
	const void *B; int64_t ldb;      /* bf16 [N x K] */
	int32_t M, N, K, n_tile;
	const float *bias;
	int32_t relu, pad0;
	const void *mask; int64_t ldm;   /* bf16 [M x N]: output zeroed where mask <= 0 */
	void *C; int64_t ldc;            /* bf16 [M x N] */
	void *CT; int64_t ldct;          /* bf16 [N x M] */
	float *Cf; int64_t ldcf;         /* f32 [M x N] */
	int32_t *err;
} plk_gemm_t;
int plk_gemm_smem(int32_t n_tile);
int plk_gemm_bf16(const plk_gemm_t *a, void *stream);
int plk_mlp_gather(const void *F, int32_t fdim, const int32_t *perm, int64_t n_perm, const int32_t *step,
		int32_t B, const float *tgt, int32_t tdim, void *X, void *XT, float *T, void *stream);
int plk_mlp_loss(const float *out, int32_t ldo, const float *T, int32_t B, float pos_w, float box_w,
		void *dout, int32_t ldd, void *doutT, float *loss_sum, void *stream);
int plk_mlp_colsum(const void *dZT, int32_t B, int32_t N, float *db, void *stream);
int plk_mlp_adam(float *p, float *m, float *v, const float *grad, int64_t ldg, int32_t rows, int32_t cols,
		const int32_t *step, float lr, float b1, float b2, float eps, float wd, void *W, int64_t ldw, void *WT,
		int64_t ldwt, void *stream);
int plk_mlp_step_inc(int32_t *step, float *loss_sum, float *loss_log, int32_t log_cap, void *stream);

/* learned-prefilter features (pffeat.cu) */
#define PLK_PF_FDIM 576
typedef struct { uint8_t nt4[256], aa20[256], codon[64]; } plk_pf_tabs_t;
typedef struct { int64_t nt_off, aa_off; int32_t nl, al; } plk_pf_cand_t;
typedef struct {
	const plk_pf_cand_t *cand;
	int64_t n;
	const uint8_t *nt, *aa;
	plk_pf_tabs_t tabs;
	void *feats;       /* bf16 [n x PLK_PF_FDIM] */
	int32_t *chain;    /* [n x 4]: first/last chained window position, first/last chained residue (-1: none) */
} plk_pf_feat_args_t;
int plk_pf_features(const plk_pf_feat_args_t *a, void *stream);

/* per-alignment statistics and exon features from the CIGAR (extra.cu) */
typedef struct {
	int64_t cigar_off, nt_off, aa_off, pssm_off;  /* pssm_off < 0: score with the matrix */
	int64_t l_nt;                                 /* window bases available from the region start */
	int64_t vs, ve;                               /* the region on the target (oriented, half-open) */
	int64_t feat_off;
	int32_t qs, qe, n_cigar, has_stop, feat_cap, pad;
} plk_extra_job_t;
typedef struct {
	int64_t vs, ve;
	int32_t qs, qe;
	int16_t type, phase;
	int32_t n_fs, n_stop;
	int32_t score, n_iden, blen;
	char donor[2], acceptor[2];
} plk_feat_t;
typedef struct {
	int32_t blen, n_iden, n_plus, n_fs, n_stop, dp_max, n_exon, n_feat, ok, pad;
} plk_extra_res_t;
typedef struct {
	const plk_extra_job_t *jobs;
	int64_t n;
	const uint32_t *cigar;
	const uint8_t *nt, *aa;
	const int8_t *pssm;
	const int8_t *mat;           /* asize x asize, device */
	int32_t go, ge, fs, asize;
	uint8_t codon[64], aa20[256];
	plk_extra_res_t *res;
	plk_feat_t *feat;
} plk_extra_args_t;
int plk_extra(const plk_extra_args_t *a, void *stream);

/* prescreen banded gapped alignment (pscreen.cu) */
typedef struct {
	int64_t pssm_off, orf_off, scratch_off;  /* scratch_off: in units of (n+1) ints x 2 per job, precomputed */
	int32_t L, n, diag, band;
} plk_ps_job_t;
typedef struct {
	const plk_ps_job_t *jobs;
	int64_t n;
	const int8_t *pssm;
	const uint8_t *orf;
	int32_t go, ge;
	int *scratch;
	int32_t *score;
	/* the candidates the band kernel takes (plk_ps_band_ok), longest profile first; the
	 * wavefront kernel skips them.  n_band = 0: the wavefront kernel takes every one. */
	const int32_t *band_order;
	int64_t n_band;
} plk_ps_args_t;
int plk_ps_gapped(const plk_ps_args_t *a, void *stream);
/* the band kernel's candidates: a band of at most PLK_PS_BAND_W cells per row (16 lanes x 5),
 * a profile and an ORF, and gap penalties with go >= ge >= 0 (its horizontal-gap scan relies
 * on an open costing at least an extension) */
#define PLK_PS_BAND_W 80
#ifdef __CUDACC__
#define PLK_HD __host__ __device__
#else
#define PLK_HD
#endif
static inline PLK_HD int plk_ps_band_ok(int32_t L, int32_t n, int32_t band, int32_t go, int32_t ge)
{
	return L > 0 && n > 0 && band > 0 && 2 * band + 1 <= PLK_PS_BAND_W && go >= ge && ge >= 0;
}

/* anchor chaining DP (chain.c:160-208): thread g takes query order[g], anchors a[off[q] ..
 * off[q] + n[q]); f, p, v per anchor out, t per anchor scratch (mark stamps) */
typedef struct {
	const int64_t *off;
	const int32_t *n, *order;
	const uint64_t *a;
	int32_t *f, *p, *v, *t;
	unsigned long long *pairs;   /* optional: predecessors scored, summed over queries */
	int32_t *err;                /* set non-zero by a query whose indices leave their ranges (then skipped) */
	int64_t n_a;                 /* anchors in a / f / p / v / t */
	int32_t n_q;
	int32_t max_dist_x, max_dist_y, bw, max_skip, max_iter, is_spliced, kmer, bbit;
	float coef;
} plk_chain_args_t;
int plk_chain_fill(const plk_chain_args_t *a, int32_t n_ctas, void *stream);
int plk_chain_threads_per_cta(void);

#ifdef __cplusplus
}
#endif

#endif
