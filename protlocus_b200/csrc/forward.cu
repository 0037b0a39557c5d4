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

/* N independent logsums, each exactly ls(a[j], b[j]), written across the N arguments
 * statement by statement so that their dependence chains interleave */
template <int N>
__device__ __forceinline__ void lsn(const float (&a)[N], const float (&b)[N], float (&r)[N])
{
	float mx[N], x[N], ex[N], lg[N];
	int keep[N];
#pragma unroll
	for (int j = 0; j < N; ++j) {
		mx[j] = a[j] > b[j] ? a[j] : b[j];
		const float mn = a[j] > b[j] ? b[j] : a[j], d = __fsub_rn(mn, mx[j]);
		keep[j] = mn <= RC_NEG || d < -50.0f;
		x[j] = fmaxf(d, -50.0f);
	}
	gl_expf_rng_n<N>(x, ex, s_exp2);
	gl_log1pf_unit_n<N>(ex, lg);
#pragma unroll
	for (int j = 0; j < N; ++j) r[j] = glm_self(keep[j], mx[j], __fadd_rn(mx[j], lg[j]));
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

/*
 * The passes run on four warps of a group's CTA, each pass split in two along its
 * dependences: the Forward's M/I warp (M(k), I(k): they read only the row above) and
 * its chain warp (D and the exit sum E along the row, one column behind, then the
 * row's special states, whose xB the M/I warp needs for the next row); the
 * Backward's chain warp (the B sum over the row below, then D along the row from the
 * last column) and its M/I warp (M(k), I(k), one column behind the D it needs).
 * Per column, a value crosses between the two warps of a pass through a ring in
 * shared memory whose slots are 64-bit words holding the value and a tag (the pass
 * step t and column count c as t * (M + 2) + c), written and read whole, so the
 * consumer lane waits for its slot to carry the tag and needs no fence; the consumer
 * hands its progress back the same way, and the producer does not overwrite a slot
 * the consumer has not taken.  Once per row, where a warp reads rows the other wrote
 * to global memory, a counter is advanced after a block fence.  Every wait is bounded
 * by a clock limit: on expiry the CTA's abort flag and the launch's error word are
 * set and every warp leaves its loops (the barriers that follow are still met).
 */
#define RC_Q 32                        /* ring depth, columns */
#define RC_SPIN_LIMIT 10000000000LL    /* clock cycles, some seconds: the default limit of a wait */
#define FULL 0xffffffffu

struct RcSync {
	volatile int fc, bc, bp, abort;             /* row hand-offs: Forward chain row done, Backward M/I row done, row L */
	long long lim;                              /* clock cycles a wait may take */
	volatile unsigned long long m[RC_Q][32];    /* M(i, k) of the Forward's M/I warp, tagged */
	volatile unsigned long long dn[RC_Q][32];   /* D(i, k+1) of the Backward's chain warp, tagged */
	volatile unsigned long long fcons[32], bcons[32], bE[32];  /* consumer progress; bE of a Backward row */
	float xB[32], tot[32], u[3][32];
};

__device__ __forceinline__ unsigned long long rc_pack(const int tag, const float v)
{
	return ((unsigned long long)(unsigned)tag << 32) | __float_as_uint(v);
}

/* the value of a slot once it carries tag (exactly, or at least tag when ge); false in
 * ok when the wait ran out or the CTA aborted */
__device__ __forceinline__ float rc_take(RcSync &Y, volatile unsigned long long &slot, const int tag, const bool ge,
		int *err, bool &ok)
{
	unsigned long long v = slot;
	if (ge ? (int)(v >> 32) < tag : (int)(v >> 32) != tag) {
		const long long t0 = clock64();
		for (;;) {
			v = slot;
			if (ge ? (int)(v >> 32) >= tag : (int)(v >> 32) == tag) break;
			if (Y.abort) { ok = false; break; }
			if (clock64() - t0 > Y.lim) { Y.abort = 1; atomicExch(err, 1); ok = false; break; }
		}
	}
	return __uint_as_float((unsigned)v);
}

/* warp-wide wait until ctr >= target, then a block fence (the rows the other warp wrote
 * before its matching rc_publish are visible); false when it ran out or the CTA aborted */
__device__ __forceinline__ bool rc_wait(RcSync &Y, volatile int &ctr, const int target, int *err)
{
	int ok = 1;
	if ((threadIdx.x & 31) == 0 && ctr < target) {
		const long long t0 = clock64();
		while (ctr < target) {
			if (Y.abort) { ok = 0; break; }
			if (clock64() - t0 > Y.lim) { Y.abort = 1; atomicExch(err, 1); ok = 0; break; }
			__nanosleep(32);
		}
	}
	ok = __shfl_sync(FULL, ok, 0);
	__threadfence_block();
	return ok != 0;
}

/* make the warp's writes so far visible to the CTA, then set ctr = v */
__device__ __forceinline__ void rc_publish(volatile int &ctr, const int v)
{
	__syncwarp();
	__threadfence_block();
	if ((threadIdx.x & 31) == 0) ctr = v;
}

#define NEG2 make_float2(RC_NEG, RC_NEG)

/* Forward M/I warp (recheck.c:305-311): for row i, M(k) = ls(ls(M'(k-1) + MM, I'(k-1) +
 * IM), ls(xB' + BM, D'(k-1) + DM)) + e(k) and I(k) = ls(M'(k) + MI, I'(k) + II) from the
 * row above ('); the first level of M(k+1) is taken in step k. */
__device__ bool rc_fwd_mi(const RcLane &S, const plk_rc_pep_t &P, const plk_rc_prof_t &R,
		const uint8_t *__restrict__ dsq, const bool on, RcSync &Y, int *err)
{
	const int M = R.M, W = M + 1, W2 = M + 2, lane = threadIdx.x & 31, L = on ? P.len : 0;
	const float4 *T4 = (const float4*)R.tsc;
	if (on)
		for (int k = 0; k <= M; ++k) str2(S.fmi + rc_ix(0, k, W), NEG2), str(S.d + ((size_t)k << 5), RC_NEG);
	float xB = P.lmove;
	for (int i = 1; i <= S.lmax; ++i) {
		if (i >= 2) {  /* the chain warp's row i-1: its D row and xB */
			if (!rc_wait(Y, Y.fc, (i - 1) * W2 + M + 1, err)) return false;
			xB = Y.xB[lane];
		}
		const bool act = i <= L;
		const int rp = S.full ? i - 1 : (i - 1) & 1, rc = S.full ? i : i & 1;
		const float2 *pr = S.fmi + rc_ix(rp, 0, W);
		float2 *cr = S.fmi + rc_ix(rc, 0, W);
		const float *dp = S.d + ((i & 1) ? 0 : ((size_t)W << 5));   /* recheck.c:303 */
		const float *mcol = R.msc + (act ? dsq[i - 1] : 0);
		if (act) str2(cr, NEG2);
		const float4 t0 = __ldg(T4);
		float4 t1 = __ldg(T4 + 1);                      /* tsc row k-1 in step k */
		float a = ls(RC_NEG + t0.x, RC_NEG + t0.y), b = ls(xB + t0.w, RC_NEG + t0.z);
		float2 cur = act ? ldr2(pr + ((size_t)1 << 5)) : NEG2;  /* M, I of the row above at column k */
		float cd = act ? ldr(dp + ((size_t)1 << 5)) : RC_NEG;   /* its D */
		float4 n0 = __ldg(T4 + 2 * (M > 1 ? 1 : 0)), n1 = __ldg(T4 + 2 * (M > 1 ? 1 : 0) + 1);  /* tsc row k */
		float ms = __ldg(mcol);
#pragma unroll 1
		for (int k = 1; k <= M; ++k) {
			if (k > RC_Q) {  /* the chain warp has taken column k - Q from this slot */
				bool ok = true;
				rc_take(Y, Y.fcons[lane], i * W2 + k - RC_Q, true, err, ok);
				if (!__all_sync(FULL, ok)) return false;
			}
			const int kn = k + 1 <= M ? k + 1 : M, kt = k + 1 < M ? k + 1 : (M > 1 ? M - 1 : 0);
			const float2 nxt = act ? ldr2(pr + ((size_t)kn << 5)) : NEG2;
			const float nd = act ? ldr(dp + ((size_t)kn << 5)) : RC_NEG;
			const float4 p0 = __ldg(T4 + 2 * kt), p1 = __ldg(T4 + 2 * kt + 1);  /* tsc row k+1 */
			const float msn = __ldg(mcol + (size_t)(kn - 1) * RC_NCODE);
			/* M(k)'s second level, I(k), M(k+1)'s first level */
			const float la[4] = {a, cur.x + t1.x, cur.x + n0.x, xB + n0.w}, lb[4] = {b, cur.y + t1.y, cur.y + n0.y, cd + n0.z};
			float lr[4];
			lsn<4>(la, lb, lr);
			const float mrk = lr[0] + ms;                    /* M(k) */
			const float irk = glm_self(k < M, lr[1], RC_NEG); /* I(k) */
			a = lr[2], b = lr[3];
			if (act) str2(cr + ((size_t)k << 5), make_float2(mrk, irk));
			Y.m[k % RC_Q][lane] = rc_pack(i * W2 + k, mrk);
			t1 = n1, n0 = p0, n1 = p1, cur = nxt, cd = nd, ms = msn;
		}
	}
	return true;
}

/* Forward chain warp (recheck.c:312-317): D(k) = ls(M(k-1) + MD, D(k-1) + DD) and
 * E = ls(E, ls(M(k), D(k))) in column order from the M/I warp's M, then xJ, xC, xN and
 * xB of the row; tot = xC(L) + lmove. */
__device__ bool rc_fwd_chain(const RcLane &S, const plk_rc_pep_t &P, const plk_rc_prof_t &R, const bool on,
		RcSync &Y, int *err)
{
	const int M = R.M, W = M + 1, W2 = M + 2, lane = threadIdx.x & 31, L = on ? P.len : 0;
	const float4 *T4 = (const float4*)R.tsc;
	const float lmove = P.lmove, lloop = P.lloop, lE = -(float)RC_LN2;
	const size_t sps = (size_t)(S.lmax + 1) << 5;
	float *xNf = S.sp, *xJf = xNf + sps, *xCf = xJf + sps;
	const bool keep = on && P.null2;
	float xN = 0.0f, xB = lmove, xJ = RC_NEG, xC = RC_NEG;
	if (keep) str(xNf, 0.0f), str(xJf, RC_NEG), str(xCf, RC_NEG);
	for (int i = 1; i <= S.lmax; ++i) {
		const bool act = i <= L;
		float *dr = S.d + ((i & 1) ? ((size_t)W << 5) : 0);
		if (act) str(dr, RC_NEG);
		/* D(1) = ls(M(0) + 0, D(0) + 0) = -inf exactly, as the reference's D(1) */
		float mr1 = RC_NEG, dr1 = RC_NEG, tq = RC_NEG, e = RC_NEG, mdq = 0.0f, ddq = 0.0f;
		float4 tr = __ldg(T4 + 1);  /* tsc row k-1 in step k: MD, DD */
#pragma unroll 1
		for (int k = 1; k <= M; ++k) {
			const float4 tn = __ldg(T4 + 2 * (k < M ? k : k - 1) + 1);
			bool ok = true;
			const float mrk = rc_take(Y, Y.m[k % RC_Q][lane], i * W2 + k, false, err, ok);
			if (!__all_sync(FULL, ok)) return false;
			Y.fcons[lane] = rc_pack(i * W2 + k, 0.0f);
			/* D(k) (tsc row k-2), E's term of column k-1, E += column k-2's term */
			const float la[3] = {mr1 + mdq, mr1, e}, lb[3] = {dr1 + ddq, dr1, tq};
			float lr[3];
			lsn<3>(la, lb, lr);
			const float drk = lr[0], tk1 = lr[1];
			e = lr[2];
			if (act) str(dr + ((size_t)k << 5), drk);
			tq = tk1, mr1 = mrk, dr1 = drk, mdq = tr.z, ddq = tr.w, tr = tn;
		}
		e = ls(e, tq);            /* column M-1 */
		e = ls(e, ls(mr1, dr1));  /* column M */
		xJ = ls(xJ + lloop, e + lE);
		xC = ls(xC + lloop, e + lE);
		xN = xN + lloop;
		xB = ls(xN + lmove, xJ + lmove);
		if (keep && act) str(xNf + ((size_t)i << 5), xN), str(xJf + ((size_t)i << 5), xJ), str(xCf + ((size_t)i << 5), xC);
		if (act) Y.tot[lane] = xC + lmove;  /* C->T after the peptide's last row */
		Y.xB[lane] = xB;
		rc_publish(Y.fc, i * W2 + M + 1);
	}
	return true;
}

/* Backward chain warp (recheck.c:323-375 without M and I): row L, then for each row i
 * (step t = L-1-i of the lane's rows) B = the sum over the columns of M(i+1, k) +
 * t[k-1].BM + e(k, x(i+1)) in column order, the special states, and D along the row
 * from the last column, D(k) = ls(M(i+1, k+1) + e(k+1) + DM, ls(D(k+1) + DD, bE)), handing
 * D(k+1) and bE to the M/I warp. */
__device__ bool rc_bwd_chain(const RcLane &S, const plk_rc_pep_t &P, const plk_rc_prof_t &R,
		const uint8_t *__restrict__ dsq, const bool n2, RcSync &Y, int *err)
{
	const int M = R.M, W = M + 1, W2 = M + 2, lane = threadIdx.x & 31, L = n2 ? P.len : 1;
	const float4 *T4 = (const float4*)R.tsc;
	const float lmove = P.lmove, lloop = P.lloop, lE = -(float)RC_LN2;
	const size_t sps = (size_t)(S.lmax + 1) << 5;
	float *bNg = S.sp + 3 * sps, *bJg = bNg + sps, *bCg = bJg + sps;
	float bC = lmove, bE = bC + lE, bJ = RC_NEG, bN = RC_NEG;
	if (n2) { /* row L: M(M) = D(M) = bE; M(k) = ls(bE, D(k+1) + t[k-1].MD), D(k) = ls(bE, D(k+1) + t[k-1].DD) */
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
		str2(rw, NEG2);
		str(bNg + ((size_t)L << 5), bN), str(bJg + ((size_t)L << 5), bJ), str(bCg + ((size_t)L << 5), bC);
	}
	rc_publish(Y.bp, 0);  /* row L */
	for (int t = 0; t + 2 <= S.lmax; ++t) {
		const int i = L - 1 - t;
		const bool act = n2 && i >= 1;
		if (t >= 1 && !rc_wait(Y, Y.bc, (t - 1) * W2 + M + 1, err)) return false;  /* row i+1's M */
		const float2 *nx = S.bmi + rc_ix(act ? i + 1 : 0, 0, W);
		const float *mcol = R.msc + (act ? dsq[i] : 0);  /* residue i+1 */
		float bB = RC_NEG;
		{ /* the next column's operands a step ahead */
			float um = act ? ldr2(nx + ((size_t)1 << 5)).x : RC_NEG, ut = __ldg(R.tsc + T_BM), ue = __ldg(mcol);
#pragma unroll 1
			for (int k = 1; k <= M; ++k) {
				const int kn = k < M ? k + 1 : k;
				const float vm = act ? ldr2(nx + ((size_t)kn << 5)).x : RC_NEG,
				            vt = __ldg(R.tsc + (size_t)(kn - 1) * 8 + T_BM), ve = __ldg(mcol + (size_t)(kn - 1) * RC_NCODE);
				bB = ls(bB, um + ut + ue);
				um = vm, ut = vt, ue = ve;
			}
		}
		if (act) {
			const float bJn = bJ, bCn = bC, bNn = bN;
			bJ = ls(bJn + lloop, bB + lmove);
			bC = bCn + lloop;
			bE = ls(bJ + lE, bC + lE);
			bN = ls(bNn + lloop, bB + lmove);
			str(bNg + ((size_t)i << 5), bN), str(bJg + ((size_t)i << 5), bJ), str(bCg + ((size_t)i << 5), bC);
		}
		Y.bE[lane] = rc_pack(t * W2, bE);
		/* D along the row, last column first; D(k+1) goes to the ring before D(k) is formed */
		float dn = bE;
		float mup = act ? ldr2(nx + ((size_t)M << 5)).x : RC_NEG;   /* M(i+1, k+1) */
		float me = __ldg(mcol + (size_t)(M >= 2 ? M - 1 : 0) * RC_NCODE);  /* e(k+1, x(i+1)) */
		float dm = __ldg(R.tsc + (size_t)(M >= 2 ? M - 1 : 0) * 8 + T_DM);  /* tsc row k: DM */
		float dd = __ldg(R.tsc + (size_t)(M >= 2 ? M - 2 : 0) * 8 + T_DD);  /* tsc row k-1: DD */
#pragma unroll 1
		for (int k = M - 1; k >= 1; --k) {
			const int c = M - k;  /* columns handed over so far, this one included */
			if (c > RC_Q) {  /* the M/I warp has taken column count c - Q from this slot */
				bool ok = true;
				rc_take(Y, Y.bcons[lane], t * W2 + c - RC_Q, true, err, ok);
				if (!__all_sync(FULL, ok)) return false;
			}
			const int kp = k >= 2 ? k - 1 : 0;
			const float nmup = act ? ldr2(nx + ((size_t)k << 5)).x : RC_NEG;
			const float nme = __ldg(mcol + (size_t)kp * RC_NCODE), ndm = __ldg(R.tsc + (size_t)kp * 8 + T_DM),
			            ndd = __ldg(R.tsc + (size_t)(kp >= 1 ? kp - 1 : 0) * 8 + T_DD);
			Y.dn[k % RC_Q][lane] = rc_pack(t * W2 + c, dn);
			const float mn1 = mup + me;
			dn = ls(mn1 + dm, ls(dn + dd, bE));
			mup = nmup, me = nme, dm = ndm, dd = ndd;
		}
	}
	return true;
}

/* Backward M/I warp (recheck.c:362-366): for row i, M(k) = ls(ls(mn1 + MM, I(i+1, k) + MI),
 * ls(bE, D(k+1) + MD)) and I(k) = ls(mn1 + IM, I(i+1, k) + II), mn1 = M(i+1, k+1) + e(k+1),
 * from the chain warp's bE and D(k+1). */
__device__ bool rc_bwd_mi(const RcLane &S, const plk_rc_pep_t &P, const plk_rc_prof_t &R,
		const uint8_t *__restrict__ dsq, const bool n2, RcSync &Y, int *err)
{
	const int M = R.M, W = M + 1, W2 = M + 2, lane = threadIdx.x & 31, L = n2 ? P.len : 1;
	const float4 *T4 = (const float4*)R.tsc;
	for (int t = 0; t + 2 <= S.lmax; ++t) {
		const int i = L - 1 - t;
		const bool act = n2 && i >= 1;
		if (t == 0 && !rc_wait(Y, Y.bp, 0, err)) return false;  /* row L, written by the chain warp */
		bool ok = true;
		const float bE = rc_take(Y, Y.bE[lane], t * W2, false, err, ok);
		if (!__all_sync(FULL, ok)) return false;
		const float2 *nx = S.bmi + rc_ix(act ? i + 1 : 0, 0, W);
		float2 *rw = S.bmi + rc_ix(act ? i : 0, 0, W);
		const float *mcol = R.msc + (act ? dsq[i] : 0);
		if (act) str2(rw + ((size_t)M << 5), make_float2(bE, RC_NEG));
		const int k1 = M - 1 > 0 ? M - 1 : 0;
		float mup = act ? ldr2(nx + ((size_t)M << 5)).x : RC_NEG;    /* M(i+1, k+1) */
		float4 tk = __ldg(T4 + 2 * k1);                               /* tsc row k: MM, IM */
		float4 r1 = __ldg(T4 + 2 * (k1 > 0 ? k1 - 1 : 0) + 1);         /* tsc row k-1: MI, II, MD */
		float4 r0 = __ldg(T4 + 2 * (k1 > 0 ? k1 - 1 : 0));
		float2 here = act ? ldr2(nx + ((size_t)k1 << 5)) : NEG2;      /* M, I of row i+1 at column k */
		float me = __ldg(mcol + (size_t)k1 * RC_NCODE);
#pragma unroll 1
		for (int k = M - 1; k >= 1; --k) {
			const int c = M - k;

			const int kp = k >= 2 ? k - 2 : 0;
			const float4 q0 = __ldg(T4 + 2 * kp), q1 = __ldg(T4 + 2 * kp + 1);  /* tsc row k-2 */
			const float2 nh = act ? ldr2(nx + ((size_t)(k - 1) << 5)) : NEG2;
			const float mne = __ldg(mcol + (size_t)(k - 1) * RC_NCODE);
			const float dk1 = rc_take(Y, Y.dn[k % RC_Q][lane], t * W2 + c, false, err, ok);
			if (!__all_sync(FULL, ok)) return false;
			Y.bcons[lane] = rc_pack(t * W2 + c, 0.0f);
			const float mn1 = mup + me;
			const float la[3] = {mn1 + tk.x, bE, mn1 + tk.y}, lb[3] = {here.y + r1.x, dk1 + r1.z, here.y + r1.y};
			float lr[3];
			lsn<3>(la, lb, lr);
			const float m = ls(lr[0], lr[1]), ii = lr[2];
			if (act) str2(rw + ((size_t)k << 5), make_float2(m, ii));
			mup = here.x, tk = r0, r0 = q0, r1 = q1, here = nh, me = mne;
		}
		if (act) str2(rw, NEG2);
		rc_publish(Y.bc, t * W2 + M + 1);
	}
	return true;
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
			float sa[RC_UB], sb[RC_UB];
#pragma unroll
			for (int j = 0; j < RC_UB; ++j) sa[j] = f[j].x + g[j].x, sb[j] = f[j].y + g[j].y;
			lsn<RC_UB>(um, sa, um);
			lsn<RC_UB>(ui, sb, ui);
#pragma unroll
			for (int j = 0; j < RC_UB; ++j) f[j] = fn[j], g[j] = gn[j];
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
		const float ua[3] = {uN, uJ, uC};
		const float ub[3] = {ldr(xNf + ((size_t)(i - 1) << 5)) + ldr(bNg + ((size_t)i << 5)) + lloop,
		                     ldr(xJf + ((size_t)(i - 1) << 5)) + ldr(bJg + ((size_t)i << 5)) + lloop,
		                     ldr(xCf + ((size_t)(i - 1) << 5)) + ldr(bCg + ((size_t)i << 5)) + lloop};
		float ur[3];
		lsn<3>(ua, ub, ur);
		uN = ur[0], uJ = ur[1], uC = ur[2];
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
		for (int x0 = 0; x0 < 20; x0 += 4) {
			const float va[4] = {v[x0], v[x0 + 1], v[x0 + 2], v[x0 + 3]};
			const float vb[4] = {u + __ldg(mr + x0), u + __ldg(mr + x0 + 1), u + __ldg(mr + x0 + 2), u + __ldg(mr + x0 + 3)};
			float vr[4];
			lsn<4>(va, vb, vr);
			v[x0] = vr[0], v[x0 + 1] = vr[1], v[x0 + 2] = vr[2], v[x0 + 3] = vr[3];
		}
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
	int *err;  /* set when a wait between warps ran out */
	long long spin_limit;
};

/* one CTA per group, four warps (the hardware hands the groups, longest first, to the
 * SMs as they free up); lane l of every warp takes the group's l-th peptide.  Warps 0/1
 * run the Forward, warps 2/3 the Backward (null2 peptides); then each warp takes a
 * quarter of the columns' usage sums, warp 3 the special states' too, and warp 0 the
 * bias and the score. */
__global__ void __launch_bounds__(128, 1) k_rc_lanes(RcArgs A)
{
	__shared__ RcSync Y;
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	if (threadIdx.x < 32) s_exp2[threadIdx.x] = glm_exp2_tab_dev[threadIdx.x];
	if (threadIdx.x == 0) Y.fc = Y.bp = Y.bc = -1, Y.abort = 0, Y.lim = A.spin_limit;
	for (int x = threadIdx.x; x < RC_Q * 32; x += blockDim.x)  /* no slot carries a tag yet */
		Y.m[x >> 5][x & 31] = Y.dn[x >> 5][x & 31] = rc_pack(-1, 0.0f);
	if (threadIdx.x < 32) Y.fcons[threadIdx.x] = Y.bcons[threadIdx.x] = Y.bE[threadIdx.x] = rc_pack(-1, 0.0f);
	__syncthreads();
	const plk_rc_grp_t G = A.grp[blockIdx.x];
	const bool on = lane < G.count;  /* every thread stays for the barriers and the warp-wide steps */
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
	if (w == 0) rc_fwd_mi(S, P, R, dsq, on, Y, A.err);
	else if (w == 1) rc_fwd_chain(S, P, R, on, Y, A.err);
	else if (G.full && w == 2) rc_bwd_chain(S, P, R, dsq, n2, Y, A.err);
	else if (G.full && w == 3) rc_bwd_mi(S, P, R, dsq, n2, Y, A.err);
	__syncthreads();
	const bool ok = !Y.abort;
	if (G.full && ok) {  /* the same for the whole CTA */
		const int k0 = 1 + (M * w) / 4, k1 = (M * (w + 1)) / 4;
		if (n2 && k0 <= k1) rc_usage_lane(S, P, M, k0, k1);
		if (w == 3 && n2) {
			float uN, uJ, uC;
			rc_special_usage(S, P, uN, uJ, uC);
			Y.u[0][lane] = uN, Y.u[1][lane] = uJ, Y.u[2][lane] = uC;
		}
	}
	__syncthreads();
	if (w == 0 && on && ok) {
		const float tot = Y.tot[lane];
		const float bias = n2 ? rc_null2_bias(S, P, R, dsq, tot, Y.u[0][lane], Y.u[1][lane], Y.u[2][lane]) : 0.0f;
		/* recheck.c:432-437; null1 = L*logf(p1) + logf(1-p1) comes from the host */
		A.bits[q] = __fdiv_rn(__fsub_rn(__fsub_rn(tot, P.null1), bias), (float)RC_LN2);
		A.bias[q] = __fdiv_rn(bias, (float)RC_LN2);
	}
}

extern "C" int plk_rc_forward(const plk_rc_prof_t *prof, const plk_rc_pep_t *pep, const uint8_t *dsq,
		const int32_t *order, const plk_rc_grp_t *grp, int32_t n_grp, float *scratch, float *bits, float *bias,
		int *err, int64_t spin_limit, void *stream)
{
	if (n_grp <= 0) return 0;
	RcArgs A;
	A.spin_limit = spin_limit > 0 ? spin_limit : RC_SPIN_LIMIT;
	A.prof = prof, A.pep = pep, A.dsq = dsq, A.order = order, A.grp = grp, A.n_grp = n_grp;
	A.scratch = scratch, A.bits = bits, A.bias = bias, A.err = err;
	k_rc_lanes<<<(unsigned)n_grp, 128, 0, (cudaStream_t)stream>>>(A);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

__global__ void k_mathf_eval(int fn, uint32_t lo, uint32_t stride, int64_t n, float *out)
{
	if (fn >= 4) {  /* the N-wide forms, four consecutive arguments per thread */
		for (int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4; i0 < n; i0 += (int64_t)gridDim.x * blockDim.x * 4) {
			float x[4], y[4];
#pragma unroll
			for (int j = 0; j < 4; ++j) x[j] = __uint_as_float(lo + (uint32_t)((uint64_t)(i0 + j < n ? i0 + j : i0) * stride));
			if (fn == 4) gl_expf_rng_n<4>(x, y, glm_exp2_tab_dev);
			else gl_log1pf_unit_n<4>(x, y);
#pragma unroll
			for (int j = 0; j < 4; ++j) if (i0 + j < n) out[i0 + j] = y[j];
		}
		return;
	}
	for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const float x = __uint_as_float(lo + (uint32_t)((uint64_t)i * stride));
		out[i] = fn == 0 ? gl_expf(x) : fn == 1 ? gl_log1pf(x) : fn == 2 ? gl_expf_rng(x) : gl_log1pf_unit(x);
	}
}

extern "C" __attribute__((visibility("default"))) int pl_rc_mathf_eval(int32_t device, int32_t fn, uint32_t lo,
		uint32_t stride, int64_t n, float *out)
{
	float *d = 0;
	if (fn < 0 || fn > 5 || n < 0 || !out) return 0;
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
