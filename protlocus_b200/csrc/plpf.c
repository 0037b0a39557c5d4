/*
 * plpf.c -- host layer of the learned candidate prefilter: a 4-layer BF16 MLP
 * (in_dim -> hidden -> hidden -> hidden -> 16, ReLU) whose GEMMs run on the tensor
 * cores (mlp.cu), trained with Adam on candidate/outcome pairs that the exact spliced
 * DP produces, and used to decide which chained candidates reach the DP and how far
 * their windows can be tightened.  Output columns: 0 pass logit, 1 window-start
 * fraction, 2 window-end fraction (3..15 unused).
 *
 * Parameters live on the device as fp32 masters with bf16 copies W [out x in] (the
 * forward operand) and W^T [in x out_pad] (the backward operand, out padded to 64).
 * One optimizer step (gather, 4 forward GEMMs, loss, 7 backward GEMMs, 4 bias
 * reductions, 8 Adam updates, step counter) is captured once as a CUDA graph and
 * replayed; the batch position comes from a device step counter, so the graph is the
 * same for every step.
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "plhost.h"

#define PF_LAYERS 4
#define PF_OUT 16
#define PF_OUT_PAD 64    /* K of the first backward GEMM (dout . W3), padded to the GEMM's K step */
#define PF_OUT_ROWS 128  /* M of the output layer's weight-gradient GEMM, padded to the M tile */
#define PF_LOG_CAP 1048576

typedef struct {
	int32_t in, out, out_pad;
	float *p, *m, *v;        /* fp32 master W [out x in] */
	float *pb, *mb, *vb;     /* fp32 bias [out] */
	void *W, *WT;            /* bf16 [out x in], [in x out_pad] */
	float *gW, *gb;          /* gradients: [max(out, 128) x in], [out] */
} pf_layer_t;

struct pl_pf_model_s {
	int device;
	int32_t in_dim, hidden;
	pf_layer_t L[PF_LAYERS];
	int32_t *err, *step;
	float *loss_sum, *loss_log;
	/* training buffers for batch size tb */
	int32_t tb;
	void *X, *XT, *H[3], *HT[3], *dout, *doutT, *dZ[3], *dZT[3];
	float *out, *T;
	/* inference buffers */
	int64_t ib;
	void *IH[3];
	float *iout;
	/* captured optimizer step */
	cudaGraphExec_t gexec;
	const void *g_feats;
	const float *g_tgt;
	const int32_t *g_perm;
	int64_t g_nperm;
	float g_lr, g_pos_w, g_box_w;
};

static void pf_free_train(pl_pf_model_t *m)
{
	int i;
	cudaFree(m->X), cudaFree(m->XT), cudaFree(m->dout), cudaFree(m->doutT), cudaFree(m->out), cudaFree(m->T);
	for (i = 0; i < 3; ++i) cudaFree(m->H[i]), cudaFree(m->HT[i]), cudaFree(m->dZ[i]), cudaFree(m->dZT[i]);
	m->X = m->XT = m->dout = m->doutT = 0, m->out = m->T = 0;
	for (i = 0; i < 3; ++i) m->H[i] = m->HT[i] = m->dZ[i] = m->dZT[i] = 0;
	m->tb = 0;
	if (m->gexec) cudaGraphExecDestroy(m->gexec), m->gexec = 0;
}

static void pf_free_infer(pl_pf_model_t *m)
{
	int i;
	for (i = 0; i < 3; ++i) cudaFree(m->IH[i]), m->IH[i] = 0;
	cudaFree(m->iout), m->iout = 0;
	m->ib = 0;
}

PL_EXPORT void pl_pf_model_destroy(pl_pf_model_t *m)
{
	int l;
	if (!m) return;
	cudaSetDevice(m->device);
	pf_free_train(m), pf_free_infer(m);
	for (l = 0; l < PF_LAYERS; ++l) {
		pf_layer_t *y = &m->L[l];
		cudaFree(y->p), cudaFree(y->m), cudaFree(y->v), cudaFree(y->pb), cudaFree(y->mb), cudaFree(y->vb);
		cudaFree(y->W), cudaFree(y->WT), cudaFree(y->gW), cudaFree(y->gb);
	}
	cudaFree(m->err), cudaFree(m->step), cudaFree(m->loss_sum), cudaFree(m->loss_log);
	free(m);
}

PL_EXPORT int64_t pl_pf_model_size(const pl_pf_model_t *m)
{
	int64_t n = 0;
	int l;
	if (!m) return 0;
	for (l = 0; l < PF_LAYERS; ++l) n += (int64_t)m->L[l].out * m->L[l].in + m->L[l].out;
	return n;
}

/* bf16 copies of the masters (round to nearest even) */
static uint16_t f2bf(float f)
{
	uint32_t u;
	memcpy(&u, &f, 4);
	if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);
	u += 0x7fffu + ((u >> 16) & 1u);
	return (uint16_t)(u >> 16);
}

static int pf_upload(pl_pf_model_t *m, const float *params)
{
	int l;
	int64_t off = 0;
	uint16_t *wb = 0, *wt = 0;
	int ok = 0;
	for (l = 0; l < PF_LAYERS; ++l) {
		pf_layer_t *y = &m->L[l];
		const int64_t nw = (int64_t)y->out * y->in;
		int64_t r, c;
		wb = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)nw);
		wt = (uint16_t*)calloc((size_t)y->in * y->out_pad, sizeof(uint16_t));
		if (!wb || !wt) { pl_set_error("out of host memory"); goto fail; }
		for (r = 0; r < y->out; ++r)
			for (c = 0; c < y->in; ++c) {
				const uint16_t b = f2bf(params[off + r * y->in + c]);
				wb[r * y->in + c] = b, wt[c * y->out_pad + r] = b;
			}
		CK(cudaMemcpy(y->p, params + off, sizeof(float) * (size_t)nw, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(y->pb, params + off + nw, sizeof(float) * (size_t)y->out, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(y->W, wb, sizeof(uint16_t) * (size_t)nw, cudaMemcpyHostToDevice));
		CK(cudaMemcpy(y->WT, wt, sizeof(uint16_t) * (size_t)y->in * y->out_pad, cudaMemcpyHostToDevice));
		CK(cudaMemset(y->m, 0, sizeof(float) * (size_t)nw));
		CK(cudaMemset(y->v, 0, sizeof(float) * (size_t)nw));
		CK(cudaMemset(y->mb, 0, sizeof(float) * (size_t)y->out));
		CK(cudaMemset(y->vb, 0, sizeof(float) * (size_t)y->out));
		free(wb), free(wt), wb = wt = 0;
		off += nw + y->out;
	}
	CK(cudaMemset(m->step, 0, sizeof(int32_t)));
	ok = 1;
fail:
	free(wb), free(wt);
	return ok;
}

PL_EXPORT int pl_pf_model_set(pl_pf_model_t *m, const float *params, int64_t n)
{
	if (!m || !params || n != pl_pf_model_size(m)) { pl_set_error("parameter count %lld (model has %lld)", (long long)n,
		(long long)pl_pf_model_size(m)); return 0; }
	if (cudaSetDevice(m->device) != cudaSuccess) { pl_set_error("cudaSetDevice failed"); return 0; }
	return pf_upload(m, params);
}

PL_EXPORT int pl_pf_model_get(const pl_pf_model_t *m, float *params, int64_t n)
{
	int l;
	int64_t off = 0;
	if (!m || !params || n != pl_pf_model_size(m)) { pl_set_error("parameter count mismatch"); return 0; }
	CK(cudaSetDevice(m->device));
	CK(cudaDeviceSynchronize());
	for (l = 0; l < PF_LAYERS; ++l) {
		const pf_layer_t *y = &m->L[l];
		const int64_t nw = (int64_t)y->out * y->in;
		CK(cudaMemcpy(params + off, y->p, sizeof(float) * (size_t)nw, cudaMemcpyDeviceToHost));
		CK(cudaMemcpy(params + off + nw, y->pb, sizeof(float) * (size_t)y->out, cudaMemcpyDeviceToHost));
		off += nw + y->out;
	}
	return 1;
fail:
	return 0;
}

PL_EXPORT pl_pf_model_t *pl_pf_model_create(int32_t device, int32_t in_dim, int32_t hidden, uint64_t seed)
{
	pl_pf_model_t *m;
	float *init = 0;
	int l;
	int64_t n, off = 0;
	uint64_t s = seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
	if (in_dim < 64 || in_dim % 64 || hidden < 128 || hidden > 256 || hidden % 128) {
		pl_set_error("prefilter model %d -> %d: in_dim a multiple of 64, hidden 128 or 256", in_dim, hidden);
		return 0;
	}
	m = (pl_pf_model_t*)calloc(1, sizeof(*m));
	if (!m) { pl_set_error("out of host memory"); return 0; }
	m->device = device, m->in_dim = in_dim, m->hidden = hidden;
	CK(cudaSetDevice(device));
	for (l = 0; l < PF_LAYERS; ++l) {
		pf_layer_t *y = &m->L[l];
		y->in = l == 0 ? in_dim : hidden;
		y->out = l == PF_LAYERS - 1 ? PF_OUT : hidden;
		y->out_pad = y->out < PF_OUT_PAD ? PF_OUT_PAD : y->out;
		const int64_t nw = (int64_t)y->out * y->in, grow = y->out < PF_OUT_ROWS ? PF_OUT_ROWS : y->out;
		CK(cudaMalloc((void**)&y->p, sizeof(float) * (size_t)nw));
		CK(cudaMalloc((void**)&y->m, sizeof(float) * (size_t)nw));
		CK(cudaMalloc((void**)&y->v, sizeof(float) * (size_t)nw));
		CK(cudaMalloc((void**)&y->pb, sizeof(float) * (size_t)y->out));
		CK(cudaMalloc((void**)&y->mb, sizeof(float) * (size_t)y->out));
		CK(cudaMalloc((void**)&y->vb, sizeof(float) * (size_t)y->out));
		CK(cudaMalloc(&y->W, 2 * (size_t)nw));
		CK(cudaMalloc(&y->WT, 2 * (size_t)y->in * y->out_pad));
		CK(cudaMalloc((void**)&y->gW, sizeof(float) * (size_t)grow * y->in));
		CK(cudaMalloc((void**)&y->gb, sizeof(float) * (size_t)y->out));
	}
	CK(cudaMalloc((void**)&m->err, sizeof(int32_t)));
	CK(cudaMalloc((void**)&m->step, sizeof(int32_t)));
	CK(cudaMalloc((void**)&m->loss_sum, sizeof(float)));
	CK(cudaMalloc((void**)&m->loss_log, sizeof(float) * PF_LOG_CAP));
	CK(cudaMemset(m->err, 0, sizeof(int32_t)));
	CK(cudaMemset(m->loss_sum, 0, sizeof(float)));
	/* He-uniform weights from a seeded xorshift stream, zero biases */
	n = pl_pf_model_size(m);
	init = (float*)calloc((size_t)n, sizeof(float));
	if (!init) { pl_set_error("out of host memory"); goto fail; }
	for (l = 0; l < PF_LAYERS; ++l) {
		const pf_layer_t *y = &m->L[l];
		const int64_t nw = (int64_t)y->out * y->in;
		const double a = sqrt(6.0 / y->in) * (l == PF_LAYERS - 1 ? 0.25 : 1.0);
		int64_t i;
		for (i = 0; i < nw; ++i) {
			s ^= s << 13, s ^= s >> 7, s ^= s << 17;
			init[off + i] = (float)(a * (2.0 * (double)(s >> 11) / 9007199254740992.0 - 1.0));
		}
		off += nw + y->out;
	}
	if (!pf_upload(m, init)) goto fail;
	free(init);
	return m;
fail:
	free(init);
	pl_pf_model_destroy(m);
	return 0;
}

static int pf_gemm(pl_pf_model_t *m, const void *A, int64_t lda, const void *B, int64_t ldb, int32_t M, int32_t N, int32_t K,
		int32_t n_tile, const float *bias, int32_t relu, const void *mask, int64_t ldm, void *C, int64_t ldc, void *CT,
		int64_t ldct, float *Cf, int64_t ldcf, cudaStream_t st)
{
	plk_gemm_t g;
	memset(&g, 0, sizeof(g));
	g.A = A, g.lda = lda, g.B = B, g.ldb = ldb, g.M = M, g.N = N, g.K = K, g.n_tile = n_tile;
	g.bias = bias, g.relu = relu, g.mask = mask, g.ldm = ldm, g.C = C, g.ldc = ldc, g.CT = CT, g.ldct = ldct;
	g.Cf = Cf, g.ldcf = ldcf, g.err = m->err;
	return plk_gemm_bf16(&g, st);
}

/* n_tile for N columns: one tile up to 256, else the largest multiple of 16 <= 256 dividing N */
static int32_t pf_tile(int32_t N)
{
	int32_t t;
	if (N <= 256) return N;
	for (t = 256; t >= 16; t -= 16) if (N % t == 0) return t;
	return 16;
}

/* forward of rows [0, M) of X (bf16 [M x in]) into H[0..2] (and their transposes when HT) and out f32 [M x 16] */
static int pf_forward(pl_pf_model_t *m, const void *X, int32_t M, void *const *H, void *const *HT, float *out, cudaStream_t st)
{
	const int32_t h = m->hidden;
	int l;
	for (l = 0; l < 3; ++l) {
		const void *in = l == 0 ? X : H[l - 1];
		const int64_t ld_in = l == 0 ? m->in_dim : h;
		int e = pf_gemm(m, in, ld_in, m->L[l].W, m->L[l].in, M, h, m->L[l].in, pf_tile(h), m->L[l].pb, 1, 0, 0,
				H[l], h, HT ? HT[l] : 0, M, 0, 0, st);
		if (e) return e;
	}
	return pf_gemm(m, H[2], h, m->L[3].W, h, M, PF_OUT, h, PF_OUT, m->L[3].pb, 0, 0, 0, 0, 0, 0, 0, out, PF_OUT, st);
}

PL_EXPORT int pl_pf_predict(pl_pf_model_t *m, const void *feats, int64_t n, float *out, void *stream)
{
	cudaStream_t st = (cudaStream_t)stream;
	const int64_t chunk = 65536;
	int64_t r0;
	int l, ok = 0;
	if (!m || n < 0) { pl_set_error("no model"); return 0; }
	if (n == 0) return 1;
	CK(cudaSetDevice(m->device));
	if (m->ib == 0) {
		for (l = 0; l < 3; ++l) CK(cudaMalloc(&m->IH[l], 2 * (size_t)chunk * m->hidden));
		m->ib = chunk;
	}
	/* feats and out hold ceil(n / 128) * 128 rows */
	for (r0 = 0; r0 < n; r0 += chunk) {
		int64_t rows = n - r0 < chunk ? n - r0 : chunk;
		rows = (rows + 127) / 128 * 128;
		CKK(pf_forward(m, (const uint16_t*)feats + r0 * m->in_dim, (int32_t)rows, m->IH, 0, out + r0 * PF_OUT, st));
	}
	ok = 1;
fail:
	return ok;
}

static int pf_ensure_train(pl_pf_model_t *m, int32_t B)
{
	const int32_t h = m->hidden, in = m->in_dim;
	int i;
	if (m->tb == B) return 1;
	pf_free_train(m);
	CK(cudaMalloc(&m->X, 2 * (size_t)B * in));
	CK(cudaMalloc(&m->XT, 2 * (size_t)B * in));
	for (i = 0; i < 3; ++i) {
		CK(cudaMalloc(&m->H[i], 2 * (size_t)B * h));
		CK(cudaMalloc(&m->HT[i], 2 * (size_t)B * h));
		CK(cudaMalloc(&m->dZ[i], 2 * (size_t)B * h));
		CK(cudaMalloc(&m->dZT[i], 2 * (size_t)B * h));
	}
	CK(cudaMalloc(&m->dout, 2 * (size_t)B * PF_OUT_PAD));
	CK(cudaMalloc(&m->doutT, 2 * (size_t)B * PF_OUT_ROWS));
	CK(cudaMemset(m->dout, 0, 2 * (size_t)B * PF_OUT_PAD));
	CK(cudaMemset(m->doutT, 0, 2 * (size_t)B * PF_OUT_ROWS));
	CK(cudaMalloc((void**)&m->out, sizeof(float) * (size_t)B * PF_OUT));
	CK(cudaMalloc((void**)&m->T, sizeof(float) * (size_t)B * 4));
	m->tb = B;
	return 1;
fail:
	pf_free_train(m);
	return 0;
}

/* one optimizer step, enqueued on st (captured into the graph) */
static int pf_step(pl_pf_model_t *m, const void *feats, const float *tgt, const int32_t *perm, int64_t n_perm,
		float lr, float pos_w, float box_w, cudaStream_t st)
{
	const int32_t B = m->tb, h = m->hidden, in = m->in_dim;
	const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f, wd = 1e-5f;
	int l, e;
#define T_(x) do { if ((e = (x)) != 0) return e; } while (0)
	T_(plk_mlp_gather(feats, in, perm, n_perm, m->step, B, tgt, 4, m->X, m->XT, m->T, st));
	T_(pf_forward(m, m->X, B, m->H, m->HT, m->out, st));
	T_(plk_mlp_loss(m->out, PF_OUT, m->T, B, pos_w, box_w, m->dout, PF_OUT_PAD, m->doutT, m->loss_sum, st));
	/* output layer: gW3 = dout^T . H3 (rows >= 16 of dout^T are zero), db3; dZ2 = (dout . W3) masked by H3 */
	T_(pf_gemm(m, m->doutT, B, m->HT[2], B, PF_OUT_ROWS, h, B, pf_tile(h), 0, 0, 0, 0, 0, 0, 0, 0, m->L[3].gW, h, st));
	T_(plk_mlp_colsum(m->doutT, B, PF_OUT, m->L[3].gb, st));
	T_(pf_gemm(m, m->dout, PF_OUT_PAD, m->L[3].WT, PF_OUT_PAD, B, h, PF_OUT_PAD, pf_tile(h), 0, 0, m->H[2], h,
			m->dZ[2], h, m->dZT[2], B, 0, 0, st));
	for (l = 2; l >= 0; --l) {
		/* gW_l = dZ_l^T . (input of layer l); db_l; dZ_{l-1} = (dZ_l . W_l) masked by H_{l-1} */
		const void *inT = l == 0 ? m->XT : m->HT[l - 1];
		const int32_t K_in = l == 0 ? in : h;
		T_(pf_gemm(m, m->dZT[l], B, inT, B, h, K_in, B, pf_tile(K_in), 0, 0, 0, 0, 0, 0, 0, 0, m->L[l].gW, K_in, st));
		T_(plk_mlp_colsum(m->dZT[l], B, h, m->L[l].gb, st));
		if (l > 0)
			T_(pf_gemm(m, m->dZ[l], h, m->L[l].WT, m->L[l].out_pad, B, h, h, pf_tile(h), 0, 0, m->H[l - 1], h,
					m->dZ[l - 1], h, m->dZT[l - 1], B, 0, 0, st));
	}
	for (l = 0; l < PF_LAYERS; ++l) {
		pf_layer_t *y = &m->L[l];
		T_(plk_mlp_adam(y->p, y->m, y->v, y->gW, y->in, y->out, y->in, m->step, lr, b1, b2, eps, wd, y->W, y->in, y->WT,
				y->out_pad, st));
		T_(plk_mlp_adam(y->pb, y->mb, y->vb, y->gb, 1, y->out, 1, m->step, lr, b1, b2, eps, 0.0f, 0, 0, 0, 0, st));
	}
	T_(plk_mlp_step_inc(m->step, m->loss_sum, m->loss_log, PF_LOG_CAP, st));
#undef T_
	return 0;
}

PL_EXPORT int pl_pf_train(pl_pf_model_t *m, const void *feats, const float *targets, const int32_t *perm, int64_t n_perm,
		int32_t batch, int32_t steps, float lr, float pos_weight, float box_weight, float *loss_log, void *stream)
{
	cudaStream_t st = 0, user = (cudaStream_t)stream;
	cudaGraph_t graph = 0;
	int32_t step0 = 0, err = 0, i;
	int ok = 0;
	if (!m || !feats || !targets || !perm || batch < 128 || batch % 128 || n_perm < batch || steps < 0) {
		pl_set_error("prefilter training: batch %d (multiple of 128) and %lld permuted rows", batch, (long long)n_perm);
		return 0;
	}
	CK(cudaSetDevice(m->device));
	if (!pf_ensure_train(m, batch)) goto fail;
	CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
	if (user) CK(cudaStreamSynchronize(user));
	if (!m->gexec || m->g_feats != feats || m->g_tgt != targets || m->g_perm != perm || m->g_nperm != n_perm ||
			m->g_lr != lr || m->g_pos_w != pos_weight || m->g_box_w != box_weight) {
		if (m->gexec) cudaGraphExecDestroy(m->gexec), m->gexec = 0;
		CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
		if (pf_step(m, feats, targets, perm, n_perm, lr, pos_weight, box_weight, st) != 0) {
			cudaStreamEndCapture(st, &graph);
			if (graph) cudaGraphDestroy(graph);
			pl_set_error("prefilter training step could not be captured");
			goto fail;
		}
		CK(cudaStreamEndCapture(st, &graph));
		CK(cudaGraphInstantiate(&m->gexec, graph, 0));
		cudaGraphDestroy(graph), graph = 0;
		m->g_feats = feats, m->g_tgt = targets, m->g_perm = perm, m->g_nperm = n_perm;
		m->g_lr = lr, m->g_pos_w = pos_weight, m->g_box_w = box_weight;
	}
	CK(cudaMemcpyAsync(&step0, m->step, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	for (i = 0; i < steps; ++i) CK(cudaGraphLaunch(m->gexec, st));
	plk_add_launches((uint64_t)steps * 26);
	CK(cudaStreamSynchronize(st));
	CK(cudaMemcpy(&err, m->err, sizeof(int32_t), cudaMemcpyDeviceToHost));
	if (err) { pl_set_error("tensor-core GEMM reported a wait timeout"); goto fail; }
	if (loss_log && steps > 0) {
		int32_t lo = step0, cnt = steps;
		if (lo >= PF_LOG_CAP) cnt = 0;
		else if (lo + cnt > PF_LOG_CAP) cnt = PF_LOG_CAP - lo;
		if (cnt > 0) CK(cudaMemcpy(loss_log, m->loss_log + lo, sizeof(float) * (size_t)cnt, cudaMemcpyDeviceToHost));
	}
	ok = 1;
fail:
	if (st) cudaStreamDestroy(st);
	return ok;
}

/* single GEMM through the model's kernel, for tests of the tensor-core path */
PL_EXPORT int pl_pf_gemm(int32_t device, const void *A, int64_t lda, const void *B, int64_t ldb, int32_t M, int32_t N, int32_t K,
		int32_t n_tile, const float *bias, int32_t relu, const void *mask, int64_t ldm, void *C, int64_t ldc, void *CT,
		int64_t ldct, float *Cf, int64_t ldcf, int32_t *err, void *stream)
{
	plk_gemm_t g;
	int e;
	if (cudaSetDevice(device) != cudaSuccess) { pl_set_error("cudaSetDevice failed"); return 0; }
	memset(&g, 0, sizeof(g));
	g.A = A, g.lda = lda, g.B = B, g.ldb = ldb, g.M = M, g.N = N, g.K = K, g.n_tile = n_tile;
	g.bias = bias, g.relu = relu, g.mask = mask, g.ldm = ldm, g.C = C, g.ldc = ldc, g.CT = CT, g.ldct = ldct;
	g.Cf = Cf, g.ldcf = ldcf, g.err = err;
	e = plk_gemm_bf16(&g, stream);
	if (e) { pl_set_error("GEMM launch: %s", cudaGetErrorString((cudaError_t)e)); return 0; }
	return 1;
}

void pl_pf_engine_free(pl_engine_t *e)
{
	dbuf_free(&e->pf_cand), dbuf_free(&e->pf_feats), dbuf_free(&e->pf_chain), dbuf_free(&e->pf_out);
	free(e->pf_host);
	e->pf_host = 0, e->pf_host_cap = 0;
}

PL_EXPORT int pl_pf_features_device(pl_engine_t *e, const ns_opt_t *opt, const pl_splice_job_t *jobs, int32_t n,
		const uint8_t *nt, const uint8_t *aa, void *feats, int32_t *chain, void *stream)
{
	plk_pf_feat_args_t a;
	plk_pf_cand_t *hc = 0;
	cudaStream_t st = stream ? (cudaStream_t)stream : (e ? e->stream : 0);
	const int64_t npad = ((int64_t)n + 127) / 128 * 128;
	int32_t q;
	int ok = 0;
	if (!e || !opt || !opt->nt4 || !opt->aa20 || !opt->codon || n < 0) { pl_set_error("features: missing engine or tables"); return 0; }
	if (n == 0) return 1;
	CK(cudaSetDevice(e->device));
	hc = (plk_pf_cand_t*)malloc(sizeof(*hc) * (size_t)n);
	if (!hc) { pl_set_error("out of host memory"); goto fail; }
	for (q = 0; q < n; ++q) {
		if (jobs[q].nl < 1 || jobs[q].al < 1 || jobs[q].al >= (1 << 20) || jobs[q].nt_off < 0 || jobs[q].aa_off < 0) {
			pl_set_error("candidate %d: nl=%d al=%d", q, jobs[q].nl, jobs[q].al);
			goto fail;
		}
		hc[q].nt_off = jobs[q].nt_off, hc[q].aa_off = jobs[q].aa_off, hc[q].nl = jobs[q].nl, hc[q].al = jobs[q].al;
	}
	if (!dbuf_ensure(&e->pf_cand, sizeof(*hc) * (size_t)n)) goto fail;
	CK(cudaMemcpyAsync(e->pf_cand.p, hc, sizeof(*hc) * (size_t)n, cudaMemcpyHostToDevice, st));
	memset(&a, 0, sizeof(a));
	a.cand = (const plk_pf_cand_t*)e->pf_cand.p, a.n = n, a.nt = nt, a.aa = aa, a.feats = feats, a.chain = chain;
	memcpy(a.tabs.nt4, opt->nt4, 256), memcpy(a.tabs.aa20, opt->aa20, 256), memcpy(a.tabs.codon, opt->codon, 64);
	if (npad > n) CK(cudaMemsetAsync((uint16_t*)feats + (int64_t)n * PLK_PF_FDIM, 0, 2 * (size_t)(npad - n) * PLK_PF_FDIM, st));
	CKK(plk_pf_features(&a, st));
	CK(cudaStreamSynchronize(st));  /* the candidate table is reused by the next call */
	ok = 1;
fail:
	free(hc);
	return ok;
}

/* ------------------------------------------------------------------ the selector's decision */

PL_EXPORT int pl_pf_decide(int32_t n, const pl_splice_job_t *jobs, const float *out, int64_t out_stride,
		const int32_t *chain, double tau, int32_t margin, double rel, double tau_fb, uint8_t *keep, uint8_t *fallback,
		pl_splice_job_t *out_jobs)
{
	const double z_keep = tau <= 0.0 ? -INFINITY : tau >= 1.0 ? INFINITY : log(tau / (1.0 - tau));
	const double z_fb = tau_fb <= 0.0 ? -INFINITY : tau_fb >= 1.0 ? INFINITY : log(tau_fb / (1.0 - tau_fb));
	int32_t q;
	if (n < 0 || (n > 0 && (!jobs || !out || !keep || !out_jobs))) { pl_set_error("pf decide: bad arguments"); return 0; }
	for (q = 0; q < n; ++q) {
		const float *o = out + (int64_t)q * out_stride;
		const pl_splice_job_t *x = &jobs[q];
		const double nl = (double)x->nl, al = (double)x->al, z = (double)o[0];
		double ps, pe, lo, hi, pad, s, e;
		out_jobs[q] = *x;
		keep[q] = z >= z_keep;
		if (fallback) fallback[q] = z >= z_fb;
		if (!keep[q]) continue;
		/* the predicted span, window fractions clipped to [0, 1] */
		ps = (double)fminf(fmaxf(o[1], 0.0f), 1.0f) * nl, pe = (double)fminf(fmaxf(o[2], 0.0f), 1.0f) * nl;
		lo = ps < pe ? ps : pe, hi = ps < pe ? pe : ps;
		if (chain && chain[4 * q] >= 0) { /* united with the span the best anchor chain implies */
			const double c_lo = (double)chain[4 * q] - 3.0 * chain[4 * q + 2] - 2.0;
			const double c_hi = (double)chain[4 * q + 1] + 3.0 * (al - 1.0 - chain[4 * q + 3]) + 1.0;
			if (c_lo < lo) lo = c_lo;
			if (c_hi > hi) hi = c_hi;
		}
		pad = (double)margin + rel * (hi - lo);
		s = floor(lo - pad), e = ceil(hi + pad);
		s = s < 0.0 ? 0.0 : s > nl ? nl : s;
		e = e < 0.0 ? 0.0 : e > nl ? nl : e;
		if (e - s < 3.0) s = 0.0, e = nl;
		out_jobs[q].nt_off = x->nt_off + (int64_t)s;
		out_jobs[q].nl = (int32_t)(e - s);
	}
	return 1;
}

PL_EXPORT int pl_pf_select_device(pl_pf_model_t *m, pl_engine_t *e, const ns_opt_t *opt, const pl_splice_job_t *jobs,
		int32_t n, const uint8_t *nt, const uint8_t *aa, double tau, int32_t margin, double tau_fb, uint8_t *keep,
		uint8_t *fallback, pl_splice_job_t *out_jobs, float *prob, void *stream)
{
	cudaStream_t st = stream ? (cudaStream_t)stream : (e ? e->stream : 0);
	const int64_t npad = ((int64_t)n + 127) / 128 * 128;
	float *ho;
	int32_t *hc, q;
	if (!m || !e || n < 0) { pl_set_error("pf select: missing model or engine"); return 0; }
	if (n == 0) return 1;
	if (m->device != e->device || m->in_dim != PLK_PF_FDIM) { pl_set_error("pf select: model on another device or of another width"); return 0; }
	CK(cudaSetDevice(e->device));
	if (!dbuf_ensure(&e->pf_feats, 2 * (size_t)npad * PLK_PF_FDIM) || !dbuf_ensure(&e->pf_chain, 16 * (size_t)n) ||
			!dbuf_ensure(&e->pf_out, 4 * 16 * (size_t)npad))
		return 0;
	if (e->pf_host_cap < (size_t)n) {
		void *h = realloc(e->pf_host, (size_t)n * (16 + 16 * 4));
		if (!h) { pl_set_error("out of host memory"); return 0; }
		e->pf_host = h, e->pf_host_cap = (size_t)n;
	}
	hc = (int32_t*)e->pf_host, ho = (float*)((char*)e->pf_host + 16 * (size_t)n);
	if (!pl_pf_features_device(e, opt, jobs, n, nt, aa, e->pf_feats.p, (int32_t*)e->pf_chain.p, st)) return 0;
	if (!pl_pf_predict(m, e->pf_feats.p, n, (float*)e->pf_out.p, st)) return 0;
	CK(cudaMemcpyAsync(hc, e->pf_chain.p, 16 * (size_t)n, cudaMemcpyDeviceToHost, st));
	CK(cudaMemcpyAsync(ho, e->pf_out.p, 4 * 16 * (size_t)n, cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	if (prob) for (q = 0; q < n; ++q) prob[q] = 1.0f / (1.0f + expf(-ho[16 * q]));
	return pl_pf_decide(n, jobs, ho, 16, hc, tau, margin, 0.0, tau_fb, keep, fallback, out_jobs);
fail:
	return 0;
}
