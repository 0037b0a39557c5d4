/*
 * forward.cu -- sm_100a kernel of the profile-HMM recheck score, rc_score
 * (recheck.c:283-440): multihit-local Forward in log space (float), and with
 * null2 the Backward pass, posterior usage and the biased-composition
 * correction (the ByExpectation null2), giving the bit score and the bias.
 *
 * One lane per peptide.  Every DP of rc_score is a chain along the row (D and
 * the exit sum E in the Forward, the B sum and D in the Backward) on top of
 * work that only reads the row before, so a peptide is one thread running the
 * reference's loops in the reference's order, and the parallelism is across
 * peptides: a warp takes up to 32 peptides of one profile (the transition and
 * emission rows it reads are the same for every lane), sorted by length so the
 * lanes run about as many rows.  The loop over a row's columns is
 * software-pipelined so that the seven logsums of a step depend only on earlier
 * steps (the one level of M(k)'s sum that needs another is taken one step
 * ahead), which keeps several transcendental evaluations in flight per thread.
 *
 * The DP matrices live in a per-group scratch region, interleaved by lane
 * (element e of lane l at e*32 + l), so every access of a warp is one coalesced
 * run: the Forward M/I rows (all rows when some peptide of the group takes
 * null2, else two), the Backward M/I rows, two Forward D rows, and the special
 * states of every row.
 *
 * Keeping every float operation in the reference's order matters: the bias is
 * exp of a sum over all residues of log-odds normalised by the Forward total,
 * so a reordering that moves the total by 1e-4 nats moves the bias by L x 1e-4
 * of itself.  The transcendental steps carry the host's bits too: rc_logsum's
 * expf and log1pf are glibc's algorithms restated (glibc_mathf.cuh, equal to
 * the host libm on every float), the length model's logf values come from the
 * host with the peptide record, every float step is written in its rounded form
 * (no contraction into FMA), and the null2 residue sum runs in the reference's
 * order.  Only the final double-precision exp/log/log1p of the bias are the
 * device's own; their results are rounded to float.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include "plk.h"
#include "glibc_mathf.cuh"

#define RC_NEG (-1e30f)
#define RC_NCODE 21
#define RC_LN2 0.69314718055994531

extern "C" void plk_add_launches(uint64_t n);

enum { T_MM, T_IM, T_DM, T_BM, T_MI, T_II, T_MD, T_DD }; /* recheck.c:74; a row is two float4 */

/* the 2^(j/32) table of expf, copied to shared memory by every CTA of the kernel */
__shared__ uint64_t s_exp2[32];

__device__ __forceinline__ float ls(float a, float b)
{ /* rc_logsum, recheck.c:260-265, without branches: mn - mx is -(mx - mn) exactly, the
   * logarithm is taken at max(mn - mx, -50) (the same argument wherever it is kept)
   * and the result selected */
	const float mx = a > b ? a : b, mn = a > b ? b : a;
	const float d = __fsub_rn(mn, mx);
	const float r = __fadd_rn(mx, gl_log1pf_unit(gl_expf_rng_t(fmaxf(d, -50.0f), s_exp2)));
	return glm_self(mn <= RC_NEG || d < -50.0f, mx, r);
}

/* a group's region, every array interleaved by lane:
 *   FMI float2 {M, I} [rows][M+1]: rows = lmax+1 when full, else rows i-1 and i at (i & 1)
 *   BMI float2 {M, I} [lmax+1][M+1]: the Backward rows (full groups only)
 *   D   float [2][M+1]: the Forward's two D rows (recheck.c:296), then lum / lui
 *   SP  float [6][lmax+1]: xN, xJ, xC of the Forward, bN, bJ, bC of the Backward (full) */
extern "C" int64_t plk_rc_group_floats(int32_t lmax, int32_t M, int32_t full)
{
	const int64_t W = (int64_t)M + 1, rows = full ? (int64_t)lmax + 1 : 2, sp = full ? (int64_t)lmax + 1 : 0;
	return (2 * rows * W + 2 * sp * W + 2 * W + 6 * sp) * 32;
}

struct RcLane {
	float2 *fmi, *bmi;  /* the lane's element 0 of each array */
	float *d, *sp;
	int full, lmax;
};

/* element (row, column k) of a lane's matrix with rows of W columns */
__device__ __forceinline__ size_t rc_ix(int row, int k, int W) { return ((size_t)row * W + k) << 5; }

/* the DP rows stream through L2 only, which keeps L1 for the profile's rows */
__device__ __forceinline__ float2 ldr2(const float2 *p) { return __ldcg(p); }
__device__ __forceinline__ float ldr(const float *p) { return __ldcg(p); }
__device__ __forceinline__ void str2(float2 *p, float2 v) { __stcg(p, v); }
__device__ __forceinline__ void str(float *p, float v) { __stcg(p, v); }

/* Forward (recheck.c:298-318) of one lane's peptide; returns the total tot (nats).
 * Step k of a row's loop forms M(k) from the first-level sums taken in step k-1,
 * the first-level sums of M(k+1), I(k), D(k), the exit term ls(M(k-1), D(k-1)),
 * and adds column k-2's term to E: the same operations on the same operands as the
 * reference's column loop, with E's terms added in column order. */
__device__ float rc_forward_lane(const RcLane &S, const plk_rc_pep_t &P, const plk_rc_prof_t &R,
		const uint8_t *__restrict__ dsq)
{
	const int M = R.M, W = M + 1, L = P.len;
	const float4 *T4 = (const float4*)R.tsc;
	const float *msc = R.msc;
	const float lmove = P.lmove, lloop = P.lloop, lE = -(float)RC_LN2;
	const size_t sps = (size_t)(S.lmax + 1) << 5;
	float *xNf = S.sp, *xJf = xNf + sps, *xCf = xJf + sps;
	for (int k = 0; k <= M; ++k) str2(S.fmi + rc_ix(0, k, W), make_float2(RC_NEG, RC_NEG)), str(S.d + ((size_t)k << 5), RC_NEG);
	float xN = 0.0f, xB = lmove, xJ = RC_NEG, xC = RC_NEG;
	if (P.null2) str(xNf, 0.0f), str(xJf, RC_NEG), str(xCf, RC_NEG);
	for (int i = 1; i <= L; ++i) {
		const int rp = S.full ? i - 1 : (i - 1) & 1, rc = S.full ? i : i & 1;
		const float2 *pr = S.fmi + rc_ix(rp, 0, W);
		float2 *cr = S.fmi + rc_ix(rc, 0, W);
		const float *dp = S.d + ((i & 1) ? 0 : ((size_t)W << 5));   /* recheck.c:303 */
		float *dr = S.d + ((i & 1) ? ((size_t)W << 5) : 0);
		const int xr = dsq[i - 1];
		const float *mcol = msc + xr;  /* M(k)'s emission at mcol[(k-1)*21] */
		str2(cr, make_float2(RC_NEG, RC_NEG)), str(dr, RC_NEG);
		/* step 1's first-level sums read column 0 of the previous row (-inf) and tsc row 0 */
		float4 t0 = __ldg(T4), t1 = __ldg(T4 + 1);   /* tsc row k-1 in step k */
		float a = ls(RC_NEG + t0.x, RC_NEG + t0.y), b = ls(xB + t0.w, RC_NEG + t0.z);
		float2 cur = ldr2(pr + ((size_t)1 << 5));      /* M, I of the previous row at column k */
		float cd = ldr(dp + ((size_t)1 << 5));          /* its D at column k */
		float4 n0 = t0, n1 = t1;                        /* tsc row k */
		if (M > 1) n0 = __ldg(T4 + 2), n1 = __ldg(T4 + 3);
		float ms = __ldg(mcol);                         /* emission of column k */
		/* D(1) = ls(M(0) + 0, D(0) + 0) = -inf exactly, as the reference's D(1) */
		float mr1 = RC_NEG, dr1 = RC_NEG, tq = RC_NEG, e = RC_NEG, mdq = 0.0f, ddq = 0.0f;
#pragma unroll 1
		for (int k = 1; k < M; ++k) {
			/* loads for step k+1, used after this step's logsums */
			const float2 nxt = ldr2(pr + ((size_t)(k + 1) << 5));
			const float nd = ldr(dp + ((size_t)(k + 1) << 5));
			const int kn = k + 1 < M ? k + 1 : k;
			const float4 p0 = __ldg(T4 + 2 * kn), p1 = __ldg(T4 + 2 * kn + 1);  /* tsc row k+1 */
			const float msn = __ldg(mcol + (size_t)k * RC_NCODE);
			const float mrk = ls(a, b) + ms;                            /* M(k) */
			const float irk = ls(cur.x + t1.x, cur.y + t1.y);           /* I(k): tsc row k-1 */
			const float drk = ls(mr1 + mdq, dr1 + ddq);                 /* D(k): tsc row k-2 */
			const float tk1 = ls(mr1, dr1);                             /* E's term of column k-1 */
			e = ls(e, tq);                                             /* E += column k-2's */
			a = ls(cur.x + n0.x, cur.y + n0.y), b = ls(xB + n0.w, cd + n0.z);  /* M(k+1)'s first level */
			str2(cr + ((size_t)k << 5), make_float2(mrk, irk)), str(dr + ((size_t)k << 5), drk);
			tq = tk1, mr1 = mrk, dr1 = drk, mdq = t1.z, ddq = t1.w;
			t0 = n0, t1 = n1, n0 = p0, n1 = p1, cur = nxt, cd = nd, ms = msn;
		}
		{ /* column M: I(M) = -inf */
			const float mrk = ls(a, b) + ms;
			const float drk = M >= 2 ? ls(mr1 + mdq, dr1 + ddq) : RC_NEG;
			const float tk1 = ls(mr1, dr1);
			e = ls(e, tq);
			str2(cr + ((size_t)M << 5), make_float2(mrk, RC_NEG)), str(dr + ((size_t)M << 5), drk);
			tq = tk1, mr1 = mrk, dr1 = drk;
		}
		e = ls(e, tq);            /* column M-1 */
		e = ls(e, ls(mr1, dr1));  /* column M */
		xJ = ls(xJ + lloop, e + lE);
		xC = ls(xC + lloop, e + lE);
		xN = xN + lloop;
		xB = ls(xN + lmove, xJ + lmove);
		if (P.null2) str(xNf + ((size_t)i << 5), xN), str(xJf + ((size_t)i << 5), xJ), str(xCf + ((size_t)i << 5), xC);
	}
	return xC + lmove;  /* C->T */
}

/* Backward (recheck.c:321-375) of one lane's peptide: its M/I rows and special states.
 * It reads neither the Forward's rows nor its total, so it runs beside the Forward. */
__device__ void rc_backward_lane(const RcLane &S, const plk_rc_pep_t &P, const plk_rc_prof_t &R,
		const uint8_t *__restrict__ dsq)
{
	const int M = R.M, W = M + 1, L = P.len;
	const float4 *T4 = (const float4*)R.tsc;
	const float *msc = R.msc;
	const float lmove = P.lmove, lloop = P.lloop, lE = -(float)RC_LN2;
	const size_t sps = (size_t)(S.lmax + 1) << 5;
	float *bNg = S.sp + 3 * sps, *bJg = bNg + sps, *bCg = bJg + sps;
	float bC = lmove, bE = bC + lE, bJ = RC_NEG, bN = RC_NEG;
	{ /* row L: M(M) = D(M) = bE; M(k) = ls(bE, D(k+1) + t[k-1].MD), D(k) = ls(bE, D(k+1) + t[k-1].DD) */
		float2 *rw = S.bmi + rc_ix(L, 0, W);
		float dn = bE;
		str2(rw + ((size_t)M << 5), make_float2(bE, RC_NEG));
		float4 t1 = __ldg(T4 + 2 * (M >= 2 ? M - 2 : 0) + 1);  /* tsc row k-1 for k = M-1 */
		for (int k = M - 1; k >= 1; --k) {
			const float4 tn = __ldg(T4 + 2 * (k >= 2 ? k - 2 : 0) + 1);
			const float m = ls(bE, dn + t1.z);
			dn = ls(bE, dn + t1.w);
			str2(rw + ((size_t)k << 5), make_float2(m, RC_NEG));
			t1 = tn;
		}
		str2(rw, make_float2(RC_NEG, RC_NEG));
		str(bNg + ((size_t)L << 5), bN), str(bJg + ((size_t)L << 5), bJ), str(bCg + ((size_t)L << 5), bC);
	}
	for (int i = L - 1; i >= 1; --i) {
		const float2 *nx = S.bmi + rc_ix(i + 1, 0, W);  /* row i+1 */
		float2 *rw = S.bmi + rc_ix(i, 0, W);
		const int xn = dsq[i];                           /* residue i+1 */
		const float *mcol = msc + xn;
		/* B = sum over the columns of M(i+1, k) + t[k-1].BM + e(k, x(i+1)), in column order;
		 * the next column's operands are loaded a step ahead */
		float bB = RC_NEG;
		float um = ldr2(nx + ((size_t)1 << 5)).x, ut = __ldg(R.tsc + T_BM), ue = __ldg(mcol);
#pragma unroll 1
		for (int k = 1; k <= M; ++k) {
			const int kn = k < M ? k + 1 : k;
			const float vm = ldr2(nx + ((size_t)kn << 5)).x, vt = __ldg(R.tsc + (size_t)(kn - 1) * 8 + T_BM),
			            ve = __ldg(mcol + (size_t)(kn - 1) * RC_NCODE);
			bB = ls(bB, um + ut + ue);
			um = vm, ut = vt, ue = ve;
		}
		const float bJn = bJ, bCn = bC, bNn = bN;
		bJ = ls(bJn + lloop, bB + lmove);
		bC = bCn + lloop;
		bE = ls(bJ + lE, bC + lE);
		bN = ls(bNn + lloop, bB + lmove);
		str(bNg + ((size_t)i << 5), bN), str(bJg + ((size_t)i << 5), bJ), str(bCg + ((size_t)i << 5), bC);
		/* M, I and D of row i, last column first (recheck.c:359-370); D(k+1) is the previous
		 * step's; the next step's operands are loaded a step ahead */
		str2(rw + ((size_t)M << 5), make_float2(bE, RC_NEG));
		float dn = bE;
		float mup = ldr2(nx + ((size_t)M << 5)).x;           /* M(i+1, k+1) */
		const int k1 = M - 1 > 0 ? M - 1 : 0;
		float4 tk = __ldg(T4 + 2 * k1);                       /* tsc row k: MM, IM, DM */
		float4 r0 = __ldg(T4 + 2 * (k1 > 0 ? k1 - 1 : 0)), r1 = __ldg(T4 + 2 * (k1 > 0 ? k1 - 1 : 0) + 1);  /* row k-1 */
		float2 here = ldr2(nx + ((size_t)k1 << 5));          /* M, I of row i+1 at column k */
		float me = __ldg(mcol + (size_t)k1 * RC_NCODE);       /* e(k+1, x(i+1)) */
#pragma unroll 1
		for (int k = M - 1; k >= 1; --k) {
			const int kp = k >= 2 ? k - 2 : 0;
			const float4 q0 = __ldg(T4 + 2 * kp), q1 = __ldg(T4 + 2 * kp + 1);  /* tsc row k-2 */
			const float2 nh = ldr2(nx + ((size_t)(k - 1) << 5));                /* column k-1 */
			const float mne = __ldg(mcol + (size_t)(k - 1) * RC_NCODE);
			const float mn1 = mup + me;
			const float m = ls(ls(mn1 + tk.x, here.y + r1.x), ls(bE, dn + r1.z));
			const float ii = ls(mn1 + tk.y, here.y + r1.y);
			dn = ls(mn1 + tk.z, ls(dn + r1.w, bE));
			str2(rw + ((size_t)k << 5), make_float2(m, ii));
			mup = here.x, tk = r0, r0 = q0, r1 = q1, here = nh, me = mne;
		}
		str2(rw, make_float2(RC_NEG, RC_NEG));
	}
}

/* posterior usage of columns [k_lo, k_hi] in log space, rows in ascending order
 * (recheck.c:382-390), eight columns at a time with the next row's values loaded one
 * row ahead (a block past k_hi repeats column k_hi and is not stored; lui(M) stays
 * -inf); lum / lui go to the D rows */
#define RC_UB 8
__device__ void rc_usage_lane(const RcLane &S, const plk_rc_pep_t &P, const int M, const int k_lo, const int k_hi)
{
	const int W = M + 1, L = P.len;
	float *lum = S.d, *lui = S.d + ((size_t)W << 5);
	for (int k0 = k_lo; k0 <= k_hi; k0 += RC_UB) {
		int kk[RC_UB];
		float um[RC_UB], ui[RC_UB];
		float2 f[RC_UB], g[RC_UB];
#pragma unroll
		for (int j = 0; j < RC_UB; ++j) {
			kk[j] = min(k0 + j, k_hi);
			um[j] = ui[j] = RC_NEG;
			f[j] = ldr2(S.fmi + rc_ix(1, kk[j], W)), g[j] = ldr2(S.bmi + rc_ix(1, kk[j], W));
		}
		for (int i = 1; i <= L; ++i) {
			const int in = min(i + 1, L);  /* row L's values again on the last row: not used */
			float2 fn[RC_UB], gn[RC_UB];
#pragma unroll
			for (int j = 0; j < RC_UB; ++j) fn[j] = ldr2(S.fmi + rc_ix(in, kk[j], W)), gn[j] = ldr2(S.bmi + rc_ix(in, kk[j], W));
#pragma unroll
			for (int j = 0; j < RC_UB; ++j) {
				um[j] = ls(um[j], f[j].x + g[j].x);
				ui[j] = ls(ui[j], f[j].y + g[j].y);
				f[j] = fn[j], g[j] = gn[j];
			}
		}
#pragma unroll
		for (int j = 0; j < RC_UB; ++j)
			if (k0 + j <= k_hi) str(lum + ((size_t)(k0 + j) << 5), um[j]), str(lui + ((size_t)(k0 + j) << 5), k0 + j < M ? ui[j] : RC_NEG);
	}
}

/* usage of the special states N, J, C (recheck.c:391-395) */
__device__ void rc_special_usage(const RcLane &S, const plk_rc_pep_t &P, float &uN, float &uJ, float &uC)
{
	const size_t sps = (size_t)(S.lmax + 1) << 5;
	const float *xNf = S.sp, *xJf = xNf + sps, *xCf = xJf + sps, *bNg = xCf + sps, *bJg = bNg + sps, *bCg = bJg + sps;
	const float lloop = P.lloop;
	uN = uJ = uC = RC_NEG;
	for (int i = 1; i <= P.len; ++i) {
		uN = ls(uN, ldr(xNf + ((size_t)(i - 1) << 5)) + ldr(bNg + ((size_t)i << 5)) + lloop);
		uJ = ls(uJ, ldr(xJf + ((size_t)(i - 1) << 5)) + ldr(bJg + ((size_t)i << 5)) + lloop);
		uC = ls(uC, ldr(xCf + ((size_t)(i - 1) << 5)) + ldr(bCg + ((size_t)i << 5)) + lloop);
	}
}

/* the null2 bias (recheck.c:404-431) from the usage; returns it in nats */
__device__ float rc_null2_bias(const RcLane &S, const plk_rc_pep_t &P, const plk_rc_prof_t &R,
		const uint8_t *__restrict__ dsq, const float tot, const float uN, const float uJ, const float uC)
{
	const int M = R.M, W = M + 1, L = P.len;
	const float *msc = R.msc, logL = P.logL;
	const float *lum = S.d, *lui = S.d + ((size_t)W << 5);
	/* li, then the 20 residues' sums over the columns, each in column order */
	const float xfac = ls(ls(uN, uJ), uC) - tot - logL;
	float li = RC_NEG;
	for (int k = 1; k < M; ++k) li = ls(li, ldr(lui + ((size_t)k << 5)) - tot - logL);
	float v[20];
#pragma unroll
	for (int x = 0; x < 20; ++x) v[x] = ls(xfac, li);
	for (int k = 1; k <= M; ++k) {
		const float u = ldr(lum + ((size_t)k << 5)) - tot - logL;
		const float *mr = msc + (size_t)(k - 1) * RC_NCODE;
#pragma unroll
		for (int x = 0; x < 20; ++x) v[x] = ls(v[x], u + __ldg(mr + x));
	}
	double s_odds = 0.0;
#pragma unroll
	for (int x = 0; x < 20; ++x) s_odds += exp((double)v[x]);
	const float lnodds_X = (float)log(s_odds / 20.0);
	/* the residue sum in the reference's order (recheck.c:427) */
	double n2 = 0.0;
	for (int i = 0; i < L; ++i) {
		const int x = dsq[i];
		float w = lnodds_X;
#pragma unroll
		for (int c = 0; c < 20; ++c) if (x == c) w = v[c];
		n2 = __dadd_rn(n2, (double)w);
	}
	const double a = __dadd_rn(log(1.0 / 256.0), n2);
	return (float)(a > 0.0 ? __dadd_rn(a, log1p(exp(-a))) : log1p(exp(a)));
}

struct RcArgs {
	const plk_rc_prof_t *prof;
	const plk_rc_pep_t *pep;
	const uint8_t *dsq;
	const int32_t *order;
	const plk_rc_grp_t *grp;
	int32_t n_grp;
	float *scratch, *bits, *bias;
};

/* one CTA per group, two warps (the hardware hands the groups, longest first, to the
 * SMs as they free up); lane l of both warps takes the group's l-th peptide.  Warp 0
 * runs the Forward, warp 1 the Backward (null2 peptides), side by side; then each
 * takes half of the columns' usage sums, warp 1 the special states' too, and warp 0
 * the bias and the score. */
__global__ void __launch_bounds__(64, 1) k_rc_lanes(RcArgs A)
{
	__shared__ float s_u[3][32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	if (threadIdx.x < 32) s_exp2[threadIdx.x] = glm_exp2_tab_dev[threadIdx.x];
	__syncthreads();
	const plk_rc_grp_t G = A.grp[blockIdx.x];
	const bool on = lane < G.count;  /* every thread stays for the barriers */
	const int q = on ? A.order[G.first + lane] : 0;
	const plk_rc_pep_t P = A.pep[q];
	const plk_rc_prof_t R = A.prof[G.prof];
	const int M = R.M;
	const size_t W = (size_t)M + 1, rows = G.full ? (size_t)G.lmax + 1 : 2, brows = G.full ? (size_t)G.lmax + 1 : 0;
	float *base = A.scratch + G.scratch_off;
	RcLane S;
	S.fmi = (float2*)base + lane;
	S.bmi = (float2*)base + ((rows * W) << 5) + lane;
	S.d = base + (((rows + brows) * W) << 6) + lane;
	S.sp = S.d + ((2 * W) << 5);
	S.full = G.full, S.lmax = G.lmax;
	const uint8_t *dsq = A.dsq + P.dsq_off;
	const bool n2 = on && P.null2;
	float tot = 0.0f;
	if (w == 0 && on) tot = rc_forward_lane(S, P, R, dsq);
	if (w == 1 && n2) rc_backward_lane(S, P, R, dsq);
	float bias = 0.0f;
	if (G.full) {  /* the same for the whole CTA */
		__syncthreads();
		const int half = (M + 1) / 2;
		if (n2) rc_usage_lane(S, P, M, w == 0 ? 1 : half + 1, w == 0 ? half : M);
		if (w == 1 && n2) {
			float uN, uJ, uC;
			rc_special_usage(S, P, uN, uJ, uC);
			s_u[0][lane] = uN, s_u[1][lane] = uJ, s_u[2][lane] = uC;
		}
		__syncthreads();
		if (w == 0 && n2) bias = rc_null2_bias(S, P, R, dsq, tot, s_u[0][lane], s_u[1][lane], s_u[2][lane]);
	}
	if (w == 0 && on) {  /* recheck.c:432-437; null1 = L*logf(p1) + logf(1-p1) comes from the host */
		A.bits[q] = __fdiv_rn(__fsub_rn(__fsub_rn(tot, P.null1), bias), (float)RC_LN2);
		A.bias[q] = __fdiv_rn(bias, (float)RC_LN2);
	}
}

extern "C" int plk_rc_forward(const plk_rc_prof_t *prof, const plk_rc_pep_t *pep, const uint8_t *dsq,
		const int32_t *order, const plk_rc_grp_t *grp, int32_t n_grp, float *scratch, float *bits, float *bias,
		void *stream)
{
	if (n_grp <= 0) return 0;
	RcArgs A;
	A.prof = prof, A.pep = pep, A.dsq = dsq, A.order = order, A.grp = grp, A.n_grp = n_grp;
	A.scratch = scratch, A.bits = bits, A.bias = bias;
	k_rc_lanes<<<(unsigned)n_grp, 64, 0, (cudaStream_t)stream>>>(A);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

__global__ void k_mathf_eval(int fn, uint32_t lo, uint32_t stride, int64_t n, float *out)
{
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const float x = __uint_as_float(lo + (uint32_t)((uint64_t)i * stride));
		out[i] = fn == 0 ? gl_expf(x) : fn == 1 ? gl_log1pf(x) : fn == 2 ? gl_expf_rng(x) : gl_log1pf_unit(x);
	}
}

extern "C" __attribute__((visibility("default"))) int pl_rc_mathf_eval(int32_t device, int32_t fn, uint32_t lo,
		uint32_t stride, int64_t n, float *out)
{
	float *d = 0;
	if (fn < 0 || fn > 3 || n < 0 || !out) return 0;
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
