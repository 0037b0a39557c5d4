/*
 * pscreen.cu -- the prescreen's banded gapped alignment on the device
 * (prescreen.c:346-382, ps_gapped): local affine-gap Smith-Waterman of a profile
 * (L rows of 22 int8 scores, the HMM's PSSM) against an ORF (n residue codes),
 * restricted to |t - i - diag| <= band (band <= 0: the full matrix), score only.
 *
 * One warp per candidate.  Rows go in strips of 32, one row per lane; lane L works
 * on absolute column t = tmin + s - L in step s, one column behind lane L-1, so the
 * row above arrives by __shfl_up_sync: its H and F at t (lane L-1's previous step)
 * and its H at t-1 (the step before).  A lane outside its row's band passes H = 0,
 * F = -inf, which is what the reference's row arrays hold for a column the row above
 * did not touch (the band only moves right).  Lane 0 takes the previous strip's last
 * row from a per-warp scratch row in global memory, valid inside that row's band.
 * The horizontal gap restarts at each row's first column, as in the reference.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include "plk.h"

extern "C" void plk_add_launches(uint64_t n);

namespace {

constexpr unsigned FULL_MASK = 0xffffffffu;
constexpr int NEG = -0x3fffffff;
constexpr int WARPS = 4;

struct Band { int lo, hi; };

/* the columns of row i (empty when lo > hi) */
__device__ __forceinline__ Band band_of(int i, int diag, int band, int n)
{
	Band b;
	b.lo = band > 0 ? i + diag - band : 0;
	b.hi = band > 0 ? i + diag + band : n - 1;
	if (b.lo < 0) b.lo = 0;
	if (b.hi > n - 1) b.hi = n - 1;
	return b;
}

__global__ void __launch_bounds__(32 * WARPS) k_ps_gapped(plk_ps_args_t A)
{
	__shared__ int8_t s_row[WARPS][32][24];
	const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
	const int64_t q = (int64_t)blockIdx.x * WARPS + wib;
	if (q >= A.n) return;
	const plk_ps_job_t J = A.jobs[q];
	const int8_t *pssm = A.pssm + J.pssm_off;
	const uint8_t *orf = A.orf + J.orf_off;
	const int L = J.L, n = J.n, diag = J.diag, band = J.band, go = A.go, ge = A.ge;
	int *rowH = A.scratch + 2 * J.scratch_off, *rowF = rowH + (n + 1);
	int best = 0;
	if (n <= 0 || L <= 0) { if (lane == 0) A.score[q] = 0; return; }
	for (int r0 = 0; r0 < L; r0 += 32) {
		const int i = r0 + lane;
		const Band b = i < L ? band_of(i, diag, band, n) : Band{1, 0};
		const Band bp = r0 > 0 ? band_of(r0 - 1, diag, band, n) : Band{1, 0};  /* the row above lane 0 */
		/* lane L works on column tmin + s - L in step s: it must be at or before its first
		 * column in step 0 (tmin <= lo_L + L) and reach its last (steps > hi_L + L - tmin) */
		int tmin, tend;
		{
			int lo = b.lo <= b.hi ? b.lo + lane : 0x7fffffff, hi = b.lo <= b.hi ? b.hi + lane : -1;
#pragma unroll
			for (int o = 16; o >= 1; o >>= 1) {
				lo = min(lo, __shfl_xor_sync(FULL_MASK, lo, o));
				hi = max(hi, __shfl_xor_sync(FULL_MASK, hi, o));
			}
			tmin = lo, tend = hi;
		}
		if (tend < tmin) continue;  /* no row of the strip touches the ORF */
		if (i < L) {
#pragma unroll
			for (int x = 0; x < 22; ++x) s_row[wib][lane][x] = pssm[(int64_t)i * 22 + x];
		}
		__syncwarp();
		const int steps = tend - tmin + 1;
		int hp = 0, fp = NEG, hp2 = 0;  /* this lane's outputs one and two steps back */
		int e = NEG;
		for (int s = 0; s < steps; ++s) {
			const int t = tmin + s - lane;
			int h_up = __shfl_up_sync(FULL_MASK, hp, 1);
			int f_up = __shfl_up_sync(FULL_MASK, fp, 1);
			int h_dg = __shfl_up_sync(FULL_MASK, hp2, 1);
			if (lane == 0) { /* the previous strip's last row, inside its band; initial values elsewhere */
				const bool in_t = t >= bp.lo && t <= bp.hi, in_t1 = t - 1 >= bp.lo && t - 1 <= bp.hi;
				h_up = in_t ? rowH[t] : 0, f_up = in_t ? rowF[t] : NEG;
				h_dg = in_t1 ? rowH[t - 1] : 0;
			}
			int hout = 0, fout = NEG;
			if (t >= b.lo && t <= b.hi) {
				if (t == b.lo) e = NEG;
				if (t == 0) h_dg = 0;
				int h = h_dg + s_row[wib][lane][orf[t]];
				const int f = max(f_up - ge, h_up - go);
				h = max(max(h, f), max(e, 0));
				best = max(best, h);
				e = max(e - ge, h - go);
				hout = h, fout = f;
			}
			hp2 = hp, hp = hout, fp = fout;
			if (lane == 31 && t >= b.lo && t <= b.hi) rowH[t] = hout, rowF[t] = fout;
			__syncwarp();
		}
	}
#pragma unroll
	for (int o = 16; o >= 1; o >>= 1) best = max(best, __shfl_xor_sync(FULL_MASK, best, o));
	if (lane == 0) A.score[q] = best;
}

}  // namespace

extern "C" int plk_ps_gapped(const plk_ps_args_t *a, void *stream)
{
	if (a->n <= 0) return 0;
	k_ps_gapped<<<(unsigned)((a->n + WARPS - 1) / WARPS), 32 * WARPS, 0, (cudaStream_t)stream>>>(*a);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}
