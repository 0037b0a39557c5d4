/*
 * forward.cu -- sm_100a kernel of the profile-HMM recheck score, rc_score
 * (recheck.c:283-440): multihit-local Forward in log space (float), and with
 * null2 the Backward pass, posterior usage and the biased-composition
 * correction (the ByExpectation null2), giving the bit score and the bias.
 *
 * One warp per peptide.  Row i of every DP matrix depends on row i-1 through
 * the whole row (the B state sums the previous row's specials), so rows are
 * sequential and the profile is spread over the lanes: lane t owns the
 * columns [1 + t*C, 1 + (t+1)*C).  Per row, the M and I states (which read
 * only the previous row) are computed by all lanes in parallel, in place from
 * the last column down; the chains that run along the row -- D and the exit
 * sum E in the Forward, the B sum and D in the Backward -- are evaluated by one
 * lane in the reference's column order.  The null2 posterior usage is summed
 * over the rows in the reference's order too, from the Forward and Backward
 * M/I rows kept in global scratch.  Keeping every float operation in the
 * reference's order matters here: the bias is exp of a sum over all residues
 * of log-odds that are normalised by the Forward total, so a reordering that
 * moves the total by 1e-4 nats moves the bias by L x 1e-4 of itself.
 * The transcendental steps carry the host's bits too: rc_logsum's expf and
 * log1pf are glibc's algorithms restated (glibc_mathf.cuh, equal to the host
 * libm on every float), the length model's logf values come from the host with
 * the peptide record, every float step is written in its rounded form (no
 * contraction into FMA), and the null2 residue sum runs in the reference's
 * order.  Only the final double-precision exp/log/log1p of the bias are the
 * device's own; their results are rounded to float.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include "plk.h"
#include "glibc_mathf.cuh"

#define FULL 0xffffffffu
#define RC_NEG (-1e30f)
#define RC_NCODE 21
#define RC_LN2 0.69314718055994531

extern "C" void plk_add_launches(uint64_t n);

enum { T_MM, T_IM, T_DM, T_BM, T_MI, T_II, T_MD, T_DD }; /* recheck.c:74 */

__device__ __forceinline__ float ls(float a, float b)
{ /* rc_logsum, recheck.c:260-265 */
	const float mx = a > b ? a : b, mn = a > b ? b : a;
	if (mn <= RC_NEG || __fsub_rn(mx, mn) > 50.0f) return mx;
	return __fadd_rn(mx, gl_log1pf(gl_expf(__fsub_rn(mn, mx))));
}

struct FwdArgs {
	const plk_rc_prof_t *prof;
	const plk_rc_pep_t *pep;
	const uint8_t *dsq;
	const int32_t *order;
	int32_t n;
	int32_t *counter;
	float *scratch;        /* Forward M/I rows of null2 peptides + specials, at pep.scratch_off */
	float *bits, *bias;
	int32_t warps_per_cta, max_m;
};

__global__ void __launch_bounds__(256) k_rc_forward(FwdArgs A)
{
	extern __shared__ __align__(16) float rc_smem[];
	const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
	for (;;) {
		int idx = 0;
		if (lane == 0) idx = atomicAdd(A.counter, 1);
		idx = __shfl_sync(FULL, idx, 0);
		if (idx >= A.n) break;
		const plk_rc_pep_t P = A.pep[A.order[idx]];
		const plk_rc_prof_t R = A.prof[P.prof];
		const int M = R.M, W = M + 1, L = P.len;
		const int wstride = (A.max_m + 1 + 3) / 4 * 4;  /* per-warp region sized for the launch's longest profile */
		float *Mrow = rc_smem + (size_t)wib * 3 * wstride, *Irow = Mrow + wstride, *Drow = Irow + wstride;
		float *lum = Mrow, *lui = Irow;  /* the usage sums reuse the row arrays once the Backward is done */
		const float *msc = R.msc, *tsc = R.tsc;
		const uint8_t *dsq = A.dsq + P.dsq_off;
		const int C = (M + 31) / 32, lo = 1 + lane * C, hi = min(M + 1, lo + C);
		const float lmove = P.lmove, lloop = P.lloop;
		const float lE = -(float)RC_LN2;
		const int do_null2 = P.null2;
		float *FM = do_null2 ? A.scratch + P.scratch_off : 0, *FI = FM ? FM + (size_t)(L + 1) * W : 0;
		float *xNf = FI ? FI + (size_t)(L + 1) * W : 0, *xJf = xNf ? xNf + (L + 1) : 0, *xCf = xJf ? xJf + (L + 1) : 0;
		for (int k = lane; k < W; k += 32) Mrow[k] = Irow[k] = Drow[k] = RC_NEG;
		float xN = 0.0f, xB = lmove, xJ = RC_NEG, xC = RC_NEG;
		if (FM) {
			for (int k = lane; k < W; k += 32) FM[k] = FI[k] = RC_NEG;
			if (lane == 0) xNf[0] = 0.0f, xJf[0] = RC_NEG, xCf[0] = RC_NEG;
		}
		__syncwarp();
		/* ---- Forward (recheck.c:298-318) ---- */
		for (int i = 1; i <= L; ++i) {
			const int xr = dsq[i - 1];
			const int lc = lo <= M ? lo - 1 : 0;  /* lanes past the profile read (and use) nothing */
			const float pm = Mrow[lc], pi = Irow[lc], pd = Drow[lc];
			__syncwarp();
			for (int k = hi - 1; k >= lo; --k) {
				const float *tp = tsc + (size_t)(k - 1) * 8;
				const float am = k == lo ? pm : Mrow[k - 1], ai = k == lo ? pi : Irow[k - 1], ad = k == lo ? pd : Drow[k - 1];
				const float m = ls(ls(am + __ldg(tp + T_MM), ai + __ldg(tp + T_IM)),
						ls(xB + __ldg(tp + T_BM), ad + __ldg(tp + T_DM)));
				const float inew = k < M ? ls(Mrow[k] + __ldg(tp + T_MI), Irow[k] + __ldg(tp + T_II)) : RC_NEG;
				Mrow[k] = m + __ldg(msc + (size_t)(k - 1) * RC_NCODE + xr);
				Irow[k] = inew;
			}
			__syncwarp();
			/* D(k) = ls(M(k-1) + t[k-2].MD, D(k-1) + t[k-2].DD) and E, along the row in column order */
			float e = RC_NEG;
			if (lane == 0) {
				float d = RC_NEG;
				for (int k = 1; k <= M; ++k) {
					if (k >= 2) { const float *tq = tsc + (size_t)(k - 2) * 8; d = ls(Mrow[k - 1] + __ldg(tq + T_MD), d + __ldg(tq + T_DD)); }
					Drow[k] = d;
					e = ls(e, ls(Mrow[k], d));
				}
			}
			e = __shfl_sync(FULL, e, 0);
			xJ = ls(xJ + lloop, e + lE);
			xC = ls(xC + lloop, e + lE);
			xN = xN + lloop;
			xB = ls(xN + lmove, xJ + lmove);
			if (FM) {
				for (int k = lane; k < W; k += 32) FM[(size_t)i * W + k] = Mrow[k], FI[(size_t)i * W + k] = Irow[k];
				if (lane == 0) xNf[i] = xN, xJf[i] = xJ, xCf[i] = xC;
			}
			__syncwarp();
		}
		const float tot = xC + lmove;
		float bias = 0.0f;
		/* ---- Backward + posterior null2 (recheck.c:321-431) ---- */
		if (FM) {
			const float logL = P.logL;
			float *BMg = xCf + (L + 1), *BIg = BMg + (size_t)(L + 1) * W;       /* Backward M / I rows */
			float *bNg = BIg + (size_t)(L + 1) * W, *bJg = bNg + (L + 1), *bCg = bJg + (L + 1);
			float bC = lmove, bE = bC + lE, bJ = RC_NEG, bN = RC_NEG;
			/* row L: M(M) = D(M) = bE; D(k) = ls(bE, D(k+1) + t[k-1].DD), M(k) = ls(bE, D(k+1) + t[k-1].MD) */
			if (lane == 0) {
				float dn = bE;
				Mrow[M] = bE, Drow[M] = bE, Irow[M] = RC_NEG;
				for (int k = M - 1; k >= 1; --k) {
					const float *tq = tsc + (size_t)(k - 1) * 8;
					Mrow[k] = ls(bE, dn + __ldg(tq + T_MD));
					dn = ls(bE, dn + __ldg(tq + T_DD));
					Drow[k] = dn, Irow[k] = RC_NEG;
				}
				Mrow[0] = Irow[0] = Drow[0] = RC_NEG;
				bNg[L] = bN, bJg[L] = bJ, bCg[L] = bC;
			}
			__syncwarp();
			for (int k = lane; k < W; k += 32) BMg[(size_t)L * W + k] = Mrow[k], BIg[(size_t)L * W + k] = Irow[k];
			for (int i = L - 1; i >= 1; --i) {
				const int xn = dsq[i];  /* residue i+1; Mrow / Irow hold row i+1 */
				if (lane == 0) {
					float bB = RC_NEG;
					for (int k = 1; k <= M; ++k)
						bB = ls(bB, Mrow[k] + __ldg(tsc + (size_t)(k - 1) * 8 + T_BM) + __ldg(msc + (size_t)(k - 1) * RC_NCODE + xn));
					const float bJn = bJ, bCn = bC, bNn = bN;
					bJ = ls(bJn + lloop, bB + lmove);
					bC = bCn + lloop;
					bE = ls(bJ + lE, bC + lE);
					bN = ls(bNn + lloop, bB + lmove);
					bNg[i] = bN, bJg[i] = bJ, bCg[i] = bC;
					/* D along the row, last column first (Drow now holds row i) */
					float dn = bE;
					Drow[M] = bE;
					for (int k = M - 1; k >= 1; --k) {
						const float mn1 = Mrow[k + 1] + __ldg(msc + (size_t)k * RC_NCODE + xn);
						dn = ls(mn1 + __ldg(tsc + (size_t)k * 8 + T_DM), ls(dn + __ldg(tsc + (size_t)(k - 1) * 8 + T_DD), bE));
						Drow[k] = dn;
					}
				}
				bE = __shfl_sync(FULL, bE, 0), bJ = __shfl_sync(FULL, bJ, 0), bC = __shfl_sync(FULL, bC, 0), bN = __shfl_sync(FULL, bN, 0);
				__syncwarp();
				float mk_new[PLK_RC_MAX_C], ik_new[PLK_RC_MAX_C];  /* row i of this block */
				int nk = 0;
				for (int k = lo; k < hi; ++k, ++nk) {
					if (k == M) { mk_new[nk] = bE, ik_new[nk] = RC_NEG; continue; }
					const float *tk = tsc + (size_t)k * 8, *tk1 = tsc + (size_t)(k - 1) * 8;
					const float mn1 = Mrow[k + 1] + __ldg(msc + (size_t)k * RC_NCODE + xn);
					mk_new[nk] = ls(ls(mn1 + __ldg(tk + T_MM), Irow[k] + __ldg(tk1 + T_MI)), ls(bE, Drow[k + 1] + __ldg(tk1 + T_MD)));
					ik_new[nk] = ls(mn1 + __ldg(tk + T_IM), Irow[k] + __ldg(tk1 + T_II));
				}
				__syncwarp();  /* every lane has read row i+1 */
				nk = 0;
				for (int k = lo; k < hi; ++k, ++nk) {
					Mrow[k] = mk_new[nk], Irow[k] = ik_new[nk];
					BMg[(size_t)i * W + k] = mk_new[nk], BIg[(size_t)i * W + k] = ik_new[nk];
				}
				if (lane == 0) BMg[(size_t)i * W] = RC_NEG, BIg[(size_t)i * W] = RC_NEG;
				__syncwarp();
			}
			/* usage, rows in ascending order (recheck.c:382-395) */
			__syncwarp();
			for (int k = lo; k < hi; ++k) {
				float um = RC_NEG, ui = RC_NEG;
				for (int i = 1; i <= L; ++i) {
					um = ls(um, FM[(size_t)i * W + k] + BMg[(size_t)i * W + k]);
					if (k < M) ui = ls(ui, FI[(size_t)i * W + k] + BIg[(size_t)i * W + k]);
				}
				lum[k] = um, lui[k] = ui;
			}
			float uN = RC_NEG, uJ = RC_NEG, uC = RC_NEG;
			if (lane == 0)
				for (int i = 1; i <= L; ++i) {
					uN = ls(uN, xNf[i - 1] + bNg[i] + lloop);
					uJ = ls(uJ, xJf[i - 1] + bJg[i] + lloop);
					uC = ls(uC, xCf[i - 1] + bCg[i] + lloop);
				}
			uN = __shfl_sync(FULL, uN, 0), uJ = __shfl_sync(FULL, uJ, 0), uC = __shfl_sync(FULL, uC, 0);
			/* null2 from the usage (recheck.c:404-426) */
			const float xfac = ls(ls(uN, uJ), uC) - tot - logL;
			__syncwarp();
			/* li and lnodds[x] in the reference's order (recheck.c:405-412): lane x < 20 runs
			 * residue x's sum over k = 1..M sequentially, lane 20 the insert sum */
			float v = RC_NEG;
			if (lane == 20) {
				for (int k = 1; k < M; ++k) v = ls(v, lui[k] - tot - logL);
			}
			const float li = __shfl_sync(FULL, v, 20);
			if (lane < 20) {
				v = ls(xfac, li);
				for (int k = 1; k <= M; ++k) v = ls(v, (lum[k] - tot - logL) + __ldg(msc + (size_t)(k - 1) * RC_NCODE + lane));
			}
			float lnodds_x[20];
			double s_odds = 0.0;
#pragma unroll
			for (int x = 0; x < 20; ++x) {
				lnodds_x[x] = __shfl_sync(FULL, v, x);
				s_odds += exp((double)lnodds_x[x]);
			}
			const float lnodds_X = (float)log(s_odds / 20.0);
			/* the residue sum in the reference's order (recheck.c:427), on lane 0 */
			double n2 = 0.0;
			if (lane == 0)
				for (int i = 0; i < L; ++i) {
					const int x = dsq[i];
					float v = lnodds_X;
#pragma unroll
					for (int q = 0; q < 20; ++q) if (x == q) v = lnodds_x[q];
					n2 = __dadd_rn(n2, (double)v);
				}
			n2 = __shfl_sync(FULL, n2, 0);
			const double a = __dadd_rn(log(1.0 / 256.0), n2);
			bias = (float)(a > 0.0 ? __dadd_rn(a, log1p(exp(-a))) : log1p(exp(a)));
		}
		if (lane == 0) {  /* recheck.c:432-437; null1 = L*logf(p1) + logf(1-p1) comes from the host */
			A.bits[A.order[idx]] = __fdiv_rn(__fsub_rn(__fsub_rn(tot, P.null1), bias), (float)RC_LN2);
			A.bias[A.order[idx]] = __fdiv_rn(bias, (float)RC_LN2);
		}
		__syncwarp();
	}
}

extern "C" int plk_rc_smem_per_warp(int32_t max_m) { return 3 * ((max_m + 1 + 3) / 4 * 4) * (int)sizeof(float); }

extern "C" int plk_rc_forward(const plk_rc_prof_t *prof, const plk_rc_pep_t *pep, const uint8_t *dsq,
		const int32_t *order, int32_t n, int32_t *counter, float *scratch, float *bits, float *bias, int32_t max_m,
		int32_t n_sm, void *stream)
{
	if (n <= 0) return 0;
	cudaStream_t st = (cudaStream_t)stream;
	const int per_warp = plk_rc_smem_per_warp(max_m);
	int warps = (100 * 1024) / per_warp;  /* two CTAs per SM when the rows fit */
	if (warps > 8) warps = 8;
	if (warps < 1 && per_warp <= 200 * 1024) warps = 1;
	if (warps < 1) return (int)cudaErrorInvalidValue;
	const int smem = warps * per_warp;
	cudaError_t e = cudaFuncSetAttribute(k_rc_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
	if (e != cudaSuccess) return (int)e;
	e = cudaMemsetAsync(counter, 0, sizeof(int32_t), st);
	if (e != cudaSuccess) return (int)e;
	int per_sm = 0;
	e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rc_forward, 32 * warps, smem);
	if (e != cudaSuccess) return (int)e;
	int64_t grid = (int64_t)(per_sm > 0 ? per_sm : 1) * n_sm;
	const int64_t need = (n + warps - 1) / warps;
	if (grid > need) grid = need;
	FwdArgs A;
	A.prof = prof, A.pep = pep, A.dsq = dsq, A.order = order, A.n = n, A.counter = counter, A.scratch = scratch;
	A.bits = bits, A.bias = bias, A.warps_per_cta = warps, A.max_m = max_m;
	k_rc_forward<<<(unsigned)grid, 32 * warps, smem, st>>>(A);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

__global__ void k_mathf_eval(int fn, uint32_t lo, uint32_t stride, int64_t n, float *out)
{
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const float x = __uint_as_float(lo + (uint32_t)((uint64_t)i * stride));
		out[i] = fn == 0 ? gl_expf(x) : gl_log1pf(x);
	}
}

extern "C" __attribute__((visibility("default"))) int pl_rc_mathf_eval(int32_t device, int32_t fn, uint32_t lo,
		uint32_t stride, int64_t n, float *out)
{
	float *d = 0;
	if ((fn != 0 && fn != 1) || n < 0 || !out) return 0;
	if (n == 0) return 1;
	if (cudaSetDevice(device) != cudaSuccess || cudaMalloc((void**)&d, sizeof(float) * (size_t)n) != cudaSuccess) return 0;
	int64_t grid = (n + 255) / 256;
	if (grid > 148 * 16) grid = 148 * 16;
	k_mathf_eval<<<(unsigned)grid, 256>>>(fn, lo, stride, n, d);
	plk_add_launches(1);
	cudaError_t e = cudaGetLastError();
	if (e == cudaSuccess) e = cudaMemcpy(out, d, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost);
	cudaFree(d);
	return e == cudaSuccess;
}
