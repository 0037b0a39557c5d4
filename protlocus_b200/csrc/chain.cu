/*
 * chain.cu -- the anchor-chaining DP on the device (chain.c:160-208, the fill loop
 * of mp_chain): for every anchor i of a query, the best chain score f[i] ending
 * there, its predecessor p[i] and the peak score v[i] along that chain.
 *
 * One thread per query (the host orders queries longest first, so the longest
 * start in the first warps).  The loop over predecessors is the reference's,
 * statement for statement: a running best (strictly greater wins, so the nearest j
 * keeps a tie), a skip counter that rises on a non-improving predecessor already
 * marked by this anchor (t[j] == i), falls on an improving one (floored at 0) and
 * ends the loop when it passes max_skip, and a mark t[p[j]] = i after every scored
 * j.  Queries are independent, so thousands of them fill the GPU; within a query
 * the order of comparisons is the reference's and the results are bit-exact.
 * Scores (comput_sc, chain.c:112-152) use the reference's float operations one at
 * a time, rounded to nearest as the CPU build rounds them (no fused multiply-add).
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <limits.h>
#include "plk.h"

extern "C" void plk_add_launches(uint64_t n);

namespace {

constexpr int CHAIN_THREADS = 64;
constexpr int BLOCK_BONUS = 2;  /* MP_BLOCK_BONUS (protlocus.h:47) */

/* log2 approximation of the reference (mppriv.h:143-151), valid for x >= 2: the
 * exponent field minus 128 plus a quadratic in the mantissa scaled to [1, 2); the
 * coefficients are the reference's, so the penalties match it bit for bit */
__device__ __forceinline__ float chain_log2(float x)
{
	uint32_t i = __float_as_uint(x);
	const float e = (float)(int)(((i >> 23) & 255u) - 128u);
	i = (i & ~(255u << 23)) + (127u << 23);
	const float m = __uint_as_float(i);
	float q = __fadd_rn(__fmul_rn(-0.34484843f, m), 2.02466578f);
	q = __fsub_rn(__fmul_rn(q, m), 0.67487759f);
	return __fadd_rn(e, q);
}

/* the score of chaining anchor aj before ai, INT_MIN when they cannot chain */
__device__ __forceinline__ int chain_score(uint64_t ai, uint64_t aj, const plk_chain_args_t &A)
{
	const int32_t dq = (int32_t)ai - (int32_t)aj, dq3 = dq * 3;
	int32_t dr3, dd, sc, dd_signed = 0;
	if (dq <= 0 || dq3 > A.max_dist_x) return INT_MIN;
	if (dq > A.max_dist_y) return INT_MIN;
	if (A.bbit > 0) { /* block resolution: gaps inside one block width count as zero */
		const int32_t bs = 1 << A.bbit;
		dr3 = (int32_t)(((ai >> 32) - (aj >> 32)) << A.bbit);
		if (dq3 >= dr3 - bs && dq3 <= dr3 + bs) dd = dd_signed = 0;
		else if (dq3 < dr3 - bs) dd = dr3 - bs - dq3, dd_signed = -dd;
		else dd = dq3 - (dr3 + bs), dd_signed = dd;
	} else {
		dr3 = (int32_t)((ai >> 32) - (aj >> 32));
		if (dr3 == 0) return INT_MIN;
		dd = dr3 > dq3 ? dr3 - dq3 : dq3 - dr3;
		dd_signed = dq3 - dr3;
	}
	if (dd > A.bw) return INT_MIN;
	if (A.bbit > 0) {
		sc = A.kmer < dq ? A.kmer : dq;
	} else if (A.kmer <= dq && A.kmer * 3 <= dr3) {
		sc = A.kmer;
	} else {
		const int32_t dr = dr3 / 3, rem = dr3 - dr * 3, dg = dr < dq ? dr : dq;
		sc = dg < A.kmer ? dg : A.kmer;
		if (rem != 0) --sc; /* frameshift */
	}
	if (dd > 0) {
		const float lin = __fmul_rn((float)dd, 0.33334f);
		const float lg = dd >= 2 ? __fadd_rn(__fmul_rn(A.coef, __fsub_rn(chain_log2((float)(dd + 1)), 1.0f)), 1.0f)
				: (float)dd;
		if (A.is_spliced && dd_signed < 0) sc -= __float2int_rz(lin < lg ? lin : lg);
		else sc -= __float2int_rz(__fadd_rn(lin, lg));
	}
	if (A.bbit > 0 && (ai >> 32) == (aj >> 32) && dd == 0) sc += BLOCK_BONUS;
	return sc;
}

/* One thread per query: the reference's sequential loop over predecessors, with its
 * early exit, skip counter and marks, so the order of every comparison is the
 * reference's.  Every per-query index is checked against the query's length; a bad
 * one records the site and the query (err[0], err[1]) and the access is skipped. */
__global__ void __launch_bounds__(CHAIN_THREADS) k_chain_fill(plk_chain_args_t A)
{
	const int qi = blockIdx.x * CHAIN_THREADS + threadIdx.x;
	if (qi >= A.n_q) return;
	const int q = A.order[qi];
	if (q < 0 || q >= A.n_q) { atomicExch(A.err, 1); return; }
	const int64_t base = A.off[q];
	const int n = A.n[q];
	if (base < 0 || n < 0 || base + n > A.n_a) { atomicExch(A.err, 2), atomicExch(A.err + 1, q); return; }
	const uint64_t *__restrict__ a = A.a + base;
	int32_t *f = A.f + base, *p = A.p + base, *v = A.v + base, *t = A.t + base;
#define CHK(x, site) ((unsigned)(x) < (unsigned)n ? true : (atomicExch(A.err, (site)), atomicExch(A.err + 1, q), false))
	for (int k = 0; k < n; ++k) t[k] = 0;
	int st = 0, hi = -1, hf = 0;
	unsigned long long pairs = 0;
	for (int i = 0; i < n; ++i) {
		const uint64_t ai = a[i];
		int max_f = A.kmer, max_j = -1, n_skip = 0;
		while (st < i && (((ai >> 32) - (a[st] >> 32)) << A.bbit) > (uint64_t)(int64_t)A.max_dist_x) ++st;
		if (hi >= 0 && hi >= st && CHK(hi, 12)) { /* the best anchor so far, even beyond the skip limit */
			const int s = hf + chain_score(ai, a[hi], A);
			if (s > max_f) max_f = s, max_j = hi;
		} else hf = 0, hi = -1;
		if (i - st > A.max_iter) st = i - A.max_iter;
		for (int j = i - 1; j >= st; --j) {
			int s = chain_score(ai, a[j], A);
			++pairs;
			if (s == INT_MIN) continue;
			s += f[j];
			if (s > max_f) {
				max_f = s, max_j = j;
				if (n_skip > 0) --n_skip;
			} else if (t[j] == i) {
				if (++n_skip > A.max_skip) break;
			}
			const int pj = p[j];
			if (pj >= 0 && CHK(pj, 14)) t[pj] = i;
		}
		f[i] = max_f, p[i] = max_j;
		v[i] = max_j >= 0 && CHK(max_j, 16) && v[max_j] > max_f ? v[max_j] : max_f;
		if (hf < max_f) hf = max_f, hi = i;
	}
#undef CHK
	if (A.pairs) atomicAdd(A.pairs, pairs);
}

} /* namespace */

extern "C" int plk_chain_fill(const plk_chain_args_t *a, int32_t n_ctas, void *stream)
{
	if (a->n_q <= 0) return 0;
	cudaStream_t st = (cudaStream_t)stream;
	k_chain_fill<<<n_ctas, CHAIN_THREADS, 0, st>>>(*a);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_chain_threads_per_cta(void) { return CHAIN_THREADS; }
