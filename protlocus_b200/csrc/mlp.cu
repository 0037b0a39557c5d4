/*
 * mlp.cu -- the learned candidate prefilter's network on sm_100a: a BF16 GEMM on the
 * 5th-generation tensor cores (tcgen05.mma, FP32 accumulators in tensor memory) with
 * fused epilogues, and the small kernels of training (batch gather, loss, bias
 * gradients, Adam).
 *
 * GEMM: C[M x N] = A[M x K] . B[N x K]^T, A and B bf16 row-major with K contiguous
 * (the nn.Linear layout: B is the weight [out x in]).  One CTA computes a 128-row tile
 * of C over n_tile (<= 256) columns: the K loop stages 128 x 64 of A and n_tile x 64 of
 * B in shared memory (two stages, cp.async 16-byte copies into the canonical K-major
 * no-swizzle layout of 8-row x 16-byte core matrices), one thread issues four
 * 128 x n_tile x 16 tcgen05.mma per stage and commits them to the stage's mbarrier, and
 * the accumulator (128 lanes x n_tile fp32 columns of tensor memory) is read back with
 * tcgen05.ld by the four warps for the epilogue: + bias, ReLU, a ReLU-backward mask,
 * stored as bf16 (row-major and/or transposed) or fp32.  The transposed store gives the
 * next GEMM of the backward pass its K-contiguous operand without a transpose kernel.
 *
 * Every mbarrier wait is bounded: on expiry the kernel sets *err, waits once more
 * (bounded) for its own tensor-core work, frees its tensor memory and returns.
 *
 * Shapes the host guarantees: M % 128 == 0, K % 64 == 0, N % 16 == 0, n_tile % 16 == 0,
 * lda/ldb % 8 == 0 and 16-byte aligned bases (cp.async alignment).
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "plk.h"

extern "C" void plk_add_launches(uint64_t n);

namespace {

constexpr int BM = 128, BK = 64, THREADS = 128;
constexpr uint64_t WAIT_NS = 1000000000ull;  /* an mbarrier wait gives up after one second */

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

/* shared-memory matrix descriptor: K-major, no swizzle (tcgen05 smem descriptor, version 1) */
__device__ __forceinline__ uint64_t make_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
	uint64_t d = 0;
	d |= (uint64_t)((addr >> 4) & 0x3FFF);
	d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
	d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
	d |= (uint64_t)1 << 46;  /* descriptor version for sm_100 */
	/* base offset 0, absolute LBO mode 0, layout type 0 = no swizzle */
	return d;
}

/* instruction descriptor of kind::f16: bf16 x bf16 -> f32, both K-major, M = 128 */
__device__ __forceinline__ uint32_t make_idesc(int n)
{
	return (1u << 4)                     /* D format f32 */
	     | (1u << 7)                     /* A format bf16 */
	     | (1u << 10)                    /* B format bf16 */
	     | ((uint32_t)(n >> 3) << 17)    /* N / 8 */
	     | ((uint32_t)(BM >> 4) << 24);  /* M / 16 */
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ uint64_t now_ns()
{
	uint64_t t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

/* bounded wait for the phase with the given parity; returns 1 when it completed */
__device__ __forceinline__ int mbar_wait(uint64_t *bar, uint32_t parity)
{
	const uint32_t a = smem_u32(bar);
	const uint64_t t0 = now_ns();
	for (;;) {
		uint32_t done;
		asm volatile("{\n\t.reg .pred p;\n\t"
		             "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		             "selp.u32 %0, 1, 0, p;\n\t}"
		             : "=r"(done) : "r"(a), "r"(parity) : "memory");
		if (done) return 1;
		if (now_ns() - t0 > WAIT_NS) return 0;
	}
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(smem_u32(smem)), "l"(gmem) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
	asm volatile("{\n\t.reg .pred p;\n\t"
	             "setp.ne.b32 p, %4, 0;\n\t"
	             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
	             :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate) : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
	asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
	             :: "r"(smem_u32(bar)) : "memory");
}

/* 32 lanes x 32 bit, 16 consecutive columns: thread (lane l of warp w) gets row 32w+l */
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16])
{
	uint32_t r[16];
	asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
	             "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
	             : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
	               "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
	             : "r"(taddr));
	asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
	for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

struct GemmArgs {
	const __nv_bfloat16 *A; int64_t lda;
	const __nv_bfloat16 *B; int64_t ldb;
	int32_t M, N, K, n_tile;
	const float *bias;                   /* [N] or null */
	int32_t relu;
	const __nv_bfloat16 *mask; int64_t ldm;  /* zero where mask <= 0, or null */
	__nv_bfloat16 *C; int64_t ldc;           /* [M x N] bf16 or null */
	__nv_bfloat16 *CT; int64_t ldct;         /* [N x M] bf16 or null */
	float *Cf; int64_t ldcf;                 /* [M x N] f32 or null */
	int32_t *err;
};

/* stage kt of A (128 x 64) and B (nt x 64) into the canonical layout:
 * element (row, k) -> chunk kc = k / 8 at byte kc * rows * 16 + row * 16 + (k % 8) * 2 */
__device__ __forceinline__ void load_stage(const GemmArgs &g, int m0, int n0, int nt, int kt, uint8_t *sa, uint8_t *sb)
{
	const int tid = threadIdx.x;
	const int k0 = kt * BK;
#pragma unroll
	for (int j = 0; j < (BM * 8) / THREADS; ++j) {
		const int idx = tid + j * THREADS, row = idx % BM, kc = idx / BM;
		cp_async16(sa + kc * (BM * 16) + row * 16, g.A + (int64_t)(m0 + row) * g.lda + k0 + kc * 8);
	}
	for (int idx = tid; idx < nt * 8; idx += THREADS) {
		const int row = idx % nt, kc = idx / nt;
		cp_async16(sb + kc * (nt * 16) + row * 16, g.B + (int64_t)(n0 + row) * g.ldb + k0 + kc * 8);
	}
	asm volatile("cp.async.commit_group;" ::: "memory");
}

__global__ void __launch_bounds__(THREADS) k_gemm_bf16(GemmArgs g)
{
	extern __shared__ __align__(1024) uint8_t smem[];
	__shared__ uint64_t bars[2];
	__shared__ uint32_t tmem_holder;
	const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
	const int m0 = blockIdx.x * BM, n0 = blockIdx.y * g.n_tile;
	const int nt = min(g.n_tile, g.N - n0);
	if (nt <= 0 || m0 >= g.M) return;
	const int stage_bytes = BM * BK * 2 + g.n_tile * BK * 2;
	uint8_t *sa[2] = {smem, smem + stage_bytes};
	uint8_t *sb[2] = {smem + BM * BK * 2, smem + stage_bytes + BM * BK * 2};
	uint32_t ncols = 32;
	while ((int)ncols < nt) ncols <<= 1;

	if (warp == 0) {
		asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
		             :: "r"(smem_u32(&tmem_holder)), "r"(ncols) : "memory");
		asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
	}
	if (tid == 0) {
		mbar_init(&bars[0], 1);
		mbar_init(&bars[1], 1);
		asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	}
	tc_fence_before();
	__syncthreads();
	tc_fence_after();
	const uint32_t tmem = tmem_holder;
	const uint32_t idesc = make_idesc(nt);
	const int KT = g.K / BK;
	int ok = 1, last = -1;  /* last: the stage whose commit was issued last */

	load_stage(g, m0, n0, nt, 0, sa[0], sb[0]);
	asm volatile("cp.async.wait_all;" ::: "memory");
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
	__syncthreads();
	for (int kt = 0; kt < KT; ++kt) {
		const int buf = kt & 1;
		last = kt;
		if (tid == 0) {
			tc_fence_after();
			const uint32_t a0 = smem_u32(sa[buf]), b0 = smem_u32(sb[buf]);
#pragma unroll
			for (int s = 0; s < BK / 16; ++s) {
				/* K = 16 per instruction: core-matrix chunks 2s and 2s+1 */
				const uint64_t ad = make_desc(a0 + 2 * s * (BM * 16), BM * 16, 128);
				const uint64_t bd = make_desc(b0 + 2 * s * (nt * 16), nt * 16, 128);
				mma_bf16(tmem, ad, bd, idesc, (kt > 0 || s > 0) ? 1u : 0u);
			}
			mma_commit(&bars[buf]);
		}
		if (kt + 1 < KT) {
			const int nb = buf ^ 1;
			if (kt >= 1 && !mbar_wait(&bars[nb], (uint32_t)(((kt - 1) >> 1) & 1))) ok = 0;
			if (__syncthreads_and(ok) == 0) { ok = 0; break; }
			load_stage(g, m0, n0, nt, kt + 1, sa[nb], sb[nb]);
			asm volatile("cp.async.wait_all;" ::: "memory");
			asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
			__syncthreads();
		}
	}
	/* the last commit completes when every issued MMA has */
	if (ok && last >= 0 && !mbar_wait(&bars[last & 1], (uint32_t)((last >> 1) & 1))) ok = 0;
	ok = __syncthreads_and(ok);
	tc_fence_after();
	if (ok) {
		const int r = warp * 32 + lane, m = m0 + r;
		for (int c0 = 0; c0 < nt; c0 += 16) {
			float v[16];
			tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
			const int n = n0 + c0;
			if (g.bias) {
#pragma unroll
				for (int j = 0; j < 16; ++j) v[j] += g.bias[n + j];
			}
			if (g.relu) {
#pragma unroll
				for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j], 0.0f);
			}
			if (g.mask) {
				const uint4 *mp = reinterpret_cast<const uint4 *>(g.mask + (int64_t)m * g.ldm + n);
				uint4 q[2] = {mp[0], mp[1]};
				const __nv_bfloat16 *mb = reinterpret_cast<const __nv_bfloat16 *>(q);
#pragma unroll
				for (int j = 0; j < 16; ++j) if (!(__bfloat162float(mb[j]) > 0.0f)) v[j] = 0.0f;
			}
			if (g.C) {
				__align__(16) __nv_bfloat16 o[16];
#pragma unroll
				for (int j = 0; j < 16; ++j) o[j] = __float2bfloat16_rn(v[j]);
				uint4 *cp = reinterpret_cast<uint4 *>(g.C + (int64_t)m * g.ldc + n);
				cp[0] = reinterpret_cast<uint4 *>(o)[0];
				cp[1] = reinterpret_cast<uint4 *>(o)[1];
			}
			if (g.CT) {
#pragma unroll
				for (int j = 0; j < 16; ++j) g.CT[(int64_t)(n + j) * g.ldct + m] = __float2bfloat16_rn(v[j]);
			}
			if (g.Cf) {
				float4 *fp = reinterpret_cast<float4 *>(g.Cf + (int64_t)m * g.ldcf + n);
#pragma unroll
				for (int j = 0; j < 4; ++j) fp[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
			}
		}
	} else {
		if (tid == 0) atomicExch(g.err, 1);
		/* let in-flight tensor-core work drain (bounded) before the memory is released */
		if (last >= 0) mbar_wait(&bars[last & 1], (uint32_t)((last >> 1) & 1));
	}
	tc_fence_before();
	__syncthreads();
	if (warp == 0)
		asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(ncols) : "memory");
}

/* ---------------------------------------------------------------- training kernels */

/* X[b, :] = F[perm[base + b], :] and X^T; targets gathered alongside.  base = (*step % steps) * B */
__global__ void k_gather(const __nv_bfloat16 *F, int32_t fdim, const int32_t *perm, int64_t n_perm, const int32_t *step,
		int32_t B, const float *tgt, int32_t tdim, __nv_bfloat16 *X, __nv_bfloat16 *XT, float *T)
{
	const int64_t steps = n_perm / B;
	const int64_t base = ((int64_t)(*step) % steps) * B;
	const int b = blockIdx.x;
	const int32_t src = perm[base + b];
	for (int k = threadIdx.x; k < fdim; k += blockDim.x) {
		const __nv_bfloat16 v = F[(int64_t)src * fdim + k];
		X[(int64_t)b * fdim + k] = v;
		XT[(int64_t)k * B + b] = v;
	}
	for (int k = threadIdx.x; k < tdim; k += blockDim.x) T[(int64_t)b * tdim + k] = tgt[(int64_t)src * tdim + k];
}

/* Outputs: column 0 pass logit, 1 window-start fraction, 2 window-end fraction.
 * Targets: [label, start, end, box weight].  Loss = BCE(logit, label) * (label ? pos_w : 1)
 *   + box_w * box * (smoothL1(start) + smoothL1(end)), averaged over the batch.
 * dOut (bf16 [B x ldd]) and dOut^T (bf16 [>= 3 rows x B]) receive d loss / d out. */
__global__ void k_loss(const float *out, int32_t ldo, const float *T, int32_t B, float pos_w, float box_w,
		__nv_bfloat16 *dout, int32_t ldd, __nv_bfloat16 *doutT, float *loss_sum)
{
	const int b = blockIdx.x * blockDim.x + threadIdx.x;
	float l = 0.0f;
	if (b < B) {
		const float z = out[(int64_t)b * ldo], s = out[(int64_t)b * ldo + 1], e = out[(int64_t)b * ldo + 2];
		const float y = T[4 * b], ts = T[4 * b + 1], te = T[4 * b + 2], wb = T[4 * b + 3];
		const float cw = y > 0.5f ? pos_w : 1.0f;
		const float p = 1.0f / (1.0f + expf(-z));
		l = cw * (fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z))));
		const float ds = s - ts, de = e - te;
		const float hs = fabsf(ds) < 0.05f ? ds * ds / 0.1f : fabsf(ds) - 0.025f;
		const float he = fabsf(de) < 0.05f ? de * de / 0.1f : fabsf(de) - 0.025f;
		l += box_w * wb * (hs + he);
		const float inv = 1.0f / (float)B;
		const float gz = cw * (p - y) * inv;
		const float gs = box_w * wb * fminf(fmaxf(ds / 0.05f, -1.0f), 1.0f) * inv;
		const float ge = box_w * wb * fminf(fmaxf(de / 0.05f, -1.0f), 1.0f) * inv;
		dout[(int64_t)b * ldd] = __float2bfloat16_rn(gz);
		dout[(int64_t)b * ldd + 1] = __float2bfloat16_rn(gs);
		dout[(int64_t)b * ldd + 2] = __float2bfloat16_rn(ge);
		doutT[b] = __float2bfloat16_rn(gz);
		doutT[B + b] = __float2bfloat16_rn(gs);
		doutT[2 * (int64_t)B + b] = __float2bfloat16_rn(ge);
	}
	for (int o = 16; o >= 1; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
	if ((threadIdx.x & 31) == 0) atomicAdd(loss_sum, l / (float)B);
}

/* db[n] = sum_b dZT[n, b] for n < N (one warp per n) */
__global__ void k_colsum(const __nv_bfloat16 *dZT, int32_t B, int32_t N, float *db)
{
	const int n = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
	if (n >= N) return;
	float s = 0.0f;
	for (int b = lane; b < B; b += 32) s += __bfloat162float(dZT[(int64_t)n * B + b]);
	for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
	if (lane == 0) db[n] = s;
}

/* Adam over one parameter tensor of rows x cols (rows = out, cols = in) with fp32 master
 * weights; writes the bf16 copy W [rows x ldw] and its transpose WT [cols x ldwt].
 * grad is [>= rows x ldg] fp32.  Bias tensors pass cols = 1 and W = WT = null. */
__global__ void k_adam(float *p, float *m, float *v, const float *grad, int64_t ldg, int32_t rows, int32_t cols,
		const int32_t *step, float lr, float b1, float b2, float eps, float wd,
		__nv_bfloat16 *W, int64_t ldw, __nv_bfloat16 *WT, int64_t ldwt)
{
	const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= (int64_t)rows * cols) return;
	const int r = (int)(i / cols), c = (int)(i % cols);
	const float t = (float)(*step + 1);
	const float c1 = 1.0f - powf(b1, t), c2 = 1.0f - powf(b2, t);
	const float gr = grad[(int64_t)r * ldg + c];
	const float mi = b1 * m[i] + (1.0f - b1) * gr;
	const float vi = b2 * v[i] + (1.0f - b2) * gr * gr;
	m[i] = mi, v[i] = vi;
	float w = p[i];
	w -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * w);
	p[i] = w;
	if (W) W[(int64_t)r * ldw + c] = __float2bfloat16_rn(w);
	if (WT) WT[(int64_t)c * ldwt + r] = __float2bfloat16_rn(w);
}

__global__ void k_step_inc(int32_t *step, float *loss_sum, float *loss_log, int32_t log_cap)
{
	const int32_t s = *step;
	if (s < log_cap) loss_log[s] = *loss_sum;
	*loss_sum = 0.0f;
	*step = s + 1;
}

}  // namespace

extern "C" int plk_gemm_smem(int32_t n_tile) { return 2 * (BM * BK * 2 + n_tile * BK * 2); }

extern "C" int plk_gemm_bf16(const plk_gemm_t *a, void *stream)
{
	if (a->M % BM || a->K % BK || a->N % 16 || a->n_tile % 16 || a->n_tile < 16 || a->n_tile > 256 ||
			a->lda % 8 || a->ldb % 8 || a->M <= 0 || a->N <= 0 || a->K <= 0)
		return (int)cudaErrorInvalidValue;
	if (a->C && a->ldc % 8) return (int)cudaErrorInvalidValue;
	if (a->mask && a->ldm % 8) return (int)cudaErrorInvalidValue;
	if (a->Cf && a->ldcf % 4) return (int)cudaErrorInvalidValue;
	GemmArgs g;
	g.A = (const __nv_bfloat16 *)a->A, g.lda = a->lda, g.B = (const __nv_bfloat16 *)a->B, g.ldb = a->ldb;
	g.M = a->M, g.N = a->N, g.K = a->K, g.n_tile = a->n_tile, g.bias = a->bias, g.relu = a->relu;
	g.mask = (const __nv_bfloat16 *)a->mask, g.ldm = a->ldm;
	g.C = (__nv_bfloat16 *)a->C, g.ldc = a->ldc, g.CT = (__nv_bfloat16 *)a->CT, g.ldct = a->ldct;
	g.Cf = a->Cf, g.ldcf = a->ldcf, g.err = a->err;
	const int smem = plk_gemm_smem(a->n_tile);
	cudaError_t e = cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
	if (e != cudaSuccess) return (int)e;
	dim3 grid((unsigned)(a->M / BM), (unsigned)((a->N + a->n_tile - 1) / a->n_tile));
	k_gemm_bf16<<<grid, THREADS, smem, (cudaStream_t)stream>>>(g);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_mlp_gather(const void *F, int32_t fdim, const int32_t *perm, int64_t n_perm, const int32_t *step,
		int32_t B, const float *tgt, int32_t tdim, void *X, void *XT, float *T, void *stream)
{
	k_gather<<<B, 128, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)F, fdim, perm, n_perm, step, B, tgt, tdim,
	                                               (__nv_bfloat16 *)X, (__nv_bfloat16 *)XT, T);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_mlp_loss(const float *out, int32_t ldo, const float *T, int32_t B, float pos_w, float box_w,
		void *dout, int32_t ldd, void *doutT, float *loss_sum, void *stream)
{
	k_loss<<<(B + 255) / 256, 256, 0, (cudaStream_t)stream>>>(out, ldo, T, B, pos_w, box_w, (__nv_bfloat16 *)dout, ldd,
	                                                           (__nv_bfloat16 *)doutT, loss_sum);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_mlp_colsum(const void *dZT, int32_t B, int32_t N, float *db, void *stream)
{
	k_colsum<<<(N + 7) / 8, 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)dZT, B, N, db);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_mlp_adam(float *p, float *m, float *v, const float *grad, int64_t ldg, int32_t rows, int32_t cols,
		const int32_t *step, float lr, float b1, float b2, float eps, float wd, void *W, int64_t ldw, void *WT,
		int64_t ldwt, void *stream)
{
	const int64_t n = (int64_t)rows * cols;
	k_adam<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(p, m, v, grad, ldg, rows, cols, step, lr, b1, b2,
	                                                                        eps, wd, (__nv_bfloat16 *)W, ldw,
	                                                                        (__nv_bfloat16 *)WT, ldwt);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_mlp_step_inc(int32_t *step, float *loss_sum, float *loss_log, int32_t log_cap, void *stream)
{
	k_step_inc<<<1, 1, 0, (cudaStream_t)stream>>>(step, loss_sum, loss_log, log_cap);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}
