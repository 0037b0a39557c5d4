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
	if (A.n_band > 0 && plk_ps_band_ok(J.L, J.n, J.band, A.go, A.ge)) return;  /* the band kernel's */
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

/*
 * Band kernel: 16 lanes per candidate (two per warp, consecutive in the longest-first
 * order, so the halves of a warp run about as many rows), the band of a row across the
 * lanes, rows in turn.  In band coordinates (u = t - (i + diag - band), 0 <= u < 2*band+1)
 * the cell (i, u) needs row i-1's H at u (the diagonal) and its H and F at u+1 (above),
 * so lane l keeps, for its five slots u = 5l..5l+4, the H/F the reference's row arrays
 * hold at column i + diag - band - 1 + u before row i: one shuffle brings slot u+1 of the
 * lane's last cell, and slots past the band hold the arrays' untouched 0 / -inf.  A cell
 * outside the ORF is not computed and takes the value from u+1 (the arrays keep it).  The
 * horizontal gap of a row is a prefix maximum across the band: with go >= ge a gap opened
 * from a cell whose H came from a horizontal gap never beats extending that gap, so
 *   e(u) = max over computed v < u of (max(H'(v), 0) + v*ge) - go - (u-1)*ge,
 * H' being the cell's value before the horizontal gap, exactly the reference's e of
 * prescreen.c:373; the row's first cell gets -inf as there.
 */
constexpr int BC = 5;                  /* band cells per lane */
constexpr int BL = 16;                 /* lanes per candidate */
static_assert(BC * BL == PLK_PS_BAND_W, "band width");

__global__ void __launch_bounds__(32 * WARPS) k_ps_band(plk_ps_args_t A)
{
	const int lane = threadIdx.x & 31, half = lane >> 4, l = lane & 15;
	const unsigned hm = 0xffffu << (16 * half);
	const int64_t slot = ((int64_t)blockIdx.x * WARPS + (threadIdx.x >> 5)) * 2 + half;
	if (slot >= A.n_band) return;  /* the whole half-warp leaves together */
	const int q = A.band_order[slot];
	const plk_ps_job_t J = A.jobs[q];
	const int8_t *pssm = A.pssm + J.pssm_off;
	const uint8_t *orf = A.orf + J.orf_off;
	const int L = J.L, n = J.n, diag = J.diag, band = J.band, go = A.go, ge = A.ge, W = 2 * band + 1;
	int SH[BC], SF[BC], ug[BC];  /* ug: u * ge of the lane's slots */
#pragma unroll
	for (int c = 0; c < BC; ++c) SH[c] = 0, SF[c] = NEG, ug[c] = (BC * l + c) * ge;
	const int goe = go - ge;
	int best = 0;
	for (int i = 0; i < L; ++i) {
		const int base = i + diag - band;
		if (base > n - 1) break;          /* this band and every later one lie right of the ORF */
		if (base + W - 1 < 0) continue;   /* left of the ORF: nothing computed yet, the slots hold 0 / -inf */
		int nh = __shfl_down_sync(hm, SH[0], 1, BL), nf = __shfl_down_sync(hm, SF[0], 1, BL);
		if (l == BL - 1) nh = 0, nf = NEG;
		const int8_t *prow = pssm + (int64_t)i * 22;
		const int t0 = base + BC * l;                    /* the lane's first column */
		const int c_lo = -t0, c_hi = min(W - 1 - BC * l, n - 1 - t0);  /* its valid slots: c_lo <= c <= c_hi */
		const uint8_t *orow = orf + t0;
		int hh[BC], fc[BC], P[BC];
		bool v[BC];
#pragma unroll
		for (int c = 0; c < BC; ++c) {
			const int hup = c + 1 < BC ? SH[c + 1] : nh, fup = c + 1 < BC ? SF[c + 1] : nf;
			v[c] = c >= c_lo && c <= c_hi;
			int g = NEG;
			hh[c] = 0, fc[c] = NEG;
			if (v[c]) {
				const int h0 = SH[c] + __ldg(prow + __ldg(orow + c));
				fc[c] = max(fup - ge, hup - go);
				hh[c] = max(h0, fc[c]);
				g = max(hh[c], 0) + ug[c];
			}
			P[c] = c == 0 ? g : max(P[c - 1], g);  /* inclusive prefix inside the lane */
		}
		/* exclusive prefix maximum of the lanes' totals across the half-warp */
		int x = P[BC - 1];
#pragma unroll
		for (int off = 1; off < BL; off <<= 1) {
			const int y = __shfl_up_sync(hm, x, off, BL);
			if (l >= off) x = max(x, y);
		}
		int ex = __shfl_up_sync(hm, x, 1, BL);
		if (l == 0) ex = NEG;
		int nSH[BC], nSF[BC];
#pragma unroll
		for (int c = 0; c < BC; ++c) {
			const int pre = c == 0 ? ex : max(ex, P[c - 1]);
			const int e = pre - goe - ug[c];  /* pre - go - (u - 1) * ge */
			const int h = max(max(hh[c], e), 0);
			if (v[c]) best = max(best, h);
			nSH[c] = v[c] ? h : (c + 1 < BC ? SH[c + 1] : nh);
			nSF[c] = v[c] ? fc[c] : (c + 1 < BC ? SF[c + 1] : nf);
		}
#pragma unroll
		for (int c = 0; c < BC; ++c) SH[c] = nSH[c], SF[c] = nSF[c];
	}
#pragma unroll
	for (int o = 8; o >= 1; o >>= 1) best = max(best, __shfl_xor_sync(hm, best, o, BL));
	if (l == 0) A.score[q] = best;
}

}  // namespace

extern "C" int plk_ps_gapped(const plk_ps_args_t *a, void *stream)
{
	if (a->n <= 0) return 0;
	k_ps_gapped<<<(unsigned)((a->n + WARPS - 1) / WARPS), 32 * WARPS, 0, (cudaStream_t)stream>>>(*a);
	plk_add_launches(1);
	if (a->n_band > 0) {
		const int64_t warps = (a->n_band + 1) / 2;
		k_ps_band<<<(unsigned)((warps + WARPS - 1) / WARPS), 32 * WARPS, 0, (cudaStream_t)stream>>>(*a);
		plk_add_launches(1);
	}
	return (int)cudaGetLastError();
}
