/*
 * ext.cu -- sm_100a kernels of the batched extension DP: ns_global_gs16b with
 * NS_F_EXT_LEFT / NS_F_EXT_RIGHT (nasw-sse.c:360-459 and the 16-lane variant
 * :596-741), the device replacement of nasw-ext-gpu.c and its OpenCL kernels.
 *
 * Kernels
 *   k_ext_prep  per-position preparation in either orientation
 *               (ns_prep_seq / ns_prep_seq_left, nasw-sse.c:95-214).
 *   k_ext_dp    the score-only DP, one warp per request, persistent over a
 *               size-sorted queue.  Same transposed wavefront as the global DP
 *               (lane t owns 8 rows of a 256-row strip and walks the columns one
 *               step behind lane t-1), with the striped schedule of the CPU
 *               kernel reproduced for its stripe width (8 lanes, or 16 when the
 *               CPU would dispatch to AVX2), including the padded columns
 *               [al, slen*width) that feed the row maximum.
 *
 * Per row the lane keeps two running values:
 *   rmax  the maximum of H over all (padded) columns -- the row maximum of
 *         nasw-sse.c:414-431;
 *   key   (H + end_bonus*[j == al-1]) * KW + (KW-1-j) over the real columns,
 *         whose maximum gives the best real column and, on ties, the first one.
 * The row score is tmp = max(rmax, key / KW), the end-bonus rule of
 * nasw-sse.c:434-435.  The reference then keeps the row with the largest
 * penalised score tmp - ie_penalty(i - 3*al) (first such row), stops when that
 * maximum exceeds the current row's penalised score by more than xdrop, and
 * reports the first real column of the kept row whose value equals the row
 * score, else the best real column (nasw-sse.c:448-458).  Both cases reduce to
 * the key maximum of the kept row: score = key / KW, aa_len = KW - key % KW.
 *
 * The row scan runs once per strip, when lane 31 has finished it: every lane
 * reads its 8 rows' (tmp, key) from shared memory, and a warp prefix-max finds
 * the first x-drop row and the kept row.  A request ends at the first strip
 * whose scan finds the x-drop row; work already issued on the next strip is
 * discarded.
 */
#include <limits.h>
#include "dp_common.cuh"

extern "C" void plk_add_launches(uint64_t n);

#define EXT_STRIP (32 * PLK_ROWS)
#define EXT_WARPS 4          /* warps (independent requests) per CTA; 3 CTAs per SM at <= 168 registers */

struct ExtShared {
	int32_t sct[23 * 22];                                   /* sct[b*22 + a]; b = 22: padding column (neg_inf) */
	int32_t rts[EXT_WARPS][EXT_STRIP];                      /* row score tmp of the strip being scanned */
	long long rkey[EXT_WARPS][EXT_STRIP];                   /* row key */
	int32_t pre[EXT_WARPS][PLK_RING_INTS] __attribute__((aligned(16)));
};

/* ie_coef * ns_log2(d) + .5f truncated, d >= 2 (nasw-sse.c:341-349, :437):
 * the reference's float steps, each rounded on its own (no contraction). */
__device__ __forceinline__ int ext_penalty(int d, float ie_coef)
{
	if (d < 2) return 0;
	unsigned u = __float_as_uint(__int2float_rn(d));
	float l2 = __int2float_rn((int)((u >> 23) & 255) - 128);
	u &= ~(255u << 23);
	u += 127u << 23;
	const float z = __uint_as_float(u);
	float t = __fmul_rn(-0.34484843f, z);
	t = __fadd_rn(t, 2.02466578f);
	t = __fmul_rn(t, z);
	t = __fsub_rn(t, 0.67487759f);
	l2 = __fadd_rn(l2, t);
	return __float2int_rz(__fadd_rn(__fmul_rn(ie_coef, l2), 0.5f));
}

__global__ void k_ext_prep(const plk_ext_job_t *__restrict__ jobs, int n_jobs, const uint8_t *__restrict__ nt,
		const uint8_t *__restrict__ aa, const uint8_t *__restrict__ ss, uint8_t *__restrict__ prep, plk_params_t P)
{
	__shared__ uint8_t s_nt4[256], s_aa20[256], s_codon[64];
	for (int x = threadIdx.x; x < 256; x += blockDim.x) s_nt4[x] = P.nt4[x], s_aa20[x] = P.aa20[x];
	for (int x = threadIdx.x; x < 64; x += blockDim.x) s_codon[x] = P.codon[x];
	__syncthreads();
	for (int jb = blockIdx.x; jb < n_jobs; jb += gridDim.x) {
		const plk_ext_job_t J = jobs[jb];
		const int nl = J.nl, al = J.al;
		if (nl < 3) continue; /* answered on the host, no scratch reserved */
		const uint8_t *ns = nt + J.nt_off, *as = aa + J.aa_off, *sst = J.ss_off >= 0 ? ss + J.ss_off : 0;
		uint8_t *nas = prep + J.prep_off, *aas = nas + nl;
		int8_t *donor = (int8_t*)(aas + al), *acceptor = donor + nl + 1;
		if (J.left == 1) {
			for (int j = threadIdx.x; j < al; j += blockDim.x) aas[j] = s_aa20[as[al - 1 - j]];
			for (int p = threadIdx.x; p <= nl; p += blockDim.x)
				prep_left_pos(p, ns, nl, sst, s_nt4, s_codon, P, nas, donor, acceptor);
		} else {
			for (int j = threadIdx.x; j < al; j += blockDim.x) aas[j] = s_aa20[as[j]];
			for (int p = threadIdx.x; p <= nl; p += blockDim.x)
				prep_fwd_pos(p, ns, nl, sst, s_nt4, s_codon, P, nas, donor, acceptor);
		}
	}
}

/* One column step of the 8 rows of a lane (first pass + carried insertion).
 * MODE 0 drops the clamps that cannot bind: a value entering a maximum with an
 * operand already >= -32768 needs no clamp of its own. */
template <int MODE>
__device__ __forceinline__ void cells_ext(const int (&in)[9], const int (&hm)[PLK_ROWS], const int ah1, const int ah2,
		const int ah3, const bool row2, const int (&sv)[PLK_ROWS], const int (&gim)[PLK_ROWS],
		const int (&dnn)[PLK_ROWS + 2], const int (&acn)[PLK_ROWS + 2], int (&ip)[PLK_ROWS], int (&lh)[PLK_ROWS],
		const int (&ic)[PLK_ROWS], const int GOI, const int NGO, const int NGE, const int NIO, const int NFS,
		int (&o)[9], int (&hn)[PLK_ROWS])
{
	constexpr int R = PLK_ROWS, NEG = -32768;
	typedef Ar<MODE> A;
	int h1 = in[0], h2 = in[1], h3 = in[2], d1 = in[3], d2 = in[4], d3 = in[5], va = in[6], vb = in[7], vc = in[8];
#pragma unroll
	for (int r = 0; r < R; ++r) {
		int h1m1 = r >= 1 ? hm[r - 1] : ah1;
		int h2m1 = r >= 2 ? hm[r - 2] : (r == 1 ? ah1 : ah2);
		int h3m1 = r >= 3 ? hm[r - 3] : (r == 2 ? ah1 : (r == 1 ? ah2 : ah3));
		if (r == 0 && row2) h1m1 = NFS, h2m1 = NFS, h3m1 = 0; /* column -1 while row 2 is computed: {0, -fs, -fs} */
		int he, dnew, anew, bnew, cnew;
		if (MODE == 0) {
			/* one fused add+max (or three-way max) per step; the four frameshift
			 * candidates share their penalty, so their maximum is taken first */
			const int c0 = __viaddmax_s32(h3m1, sv[r], NEG);
			ip[r] = __viaddmax_s32(__viaddmax_s32(lh[r], GOI, ip[r]), NGE, NEG);  /* GOI: -go, or -inf at a segment start */
			dnew = __viaddmax_s32(__viaddmax_s32(h3, NGO, d3), gim[r], NEG);
			he = __vimax3_s32(c0, ip[r], dnew);
			const int u = __viaddmax_s32(h1, NIO, NEG);
			anew = __viaddmax_s32(u, dnn[r], va);
			const int u2 = __viaddmax_s32(h1m1, NIO, NEG);
			bnew = __viaddmax_s32(u2, dnn[r + 1], vb);
			cnew = __viaddmax_s32(u2, dnn[r + 2], vc);
			he = __viaddmax_s32(anew, acn[r + 2], he);
			he = __viaddmax_s32(bnew, acn[r], he);
			he = __viaddmax_s32(cnew, acn[r + 1], he);
			he = __viaddmax_s32(max(__vimax3_s32(h1, h2, h1m1), h2m1), NFS, he);
		} else {
			he = A::add(h3m1, sv[r]);
			ip[r] = A::add(max(A::add(lh[r], GOI), ip[r]), NGE);
			he = max(he, ip[r]);
			dnew = A::add(max(A::add(h3, NGO), d3), gim[r]);
			he = max(he, dnew);
			const int u = A::add(h1, NIO);
			anew = max(A::add(u, dnn[r]), va);
			he = max(he, A::add(anew, acn[r + 2]));
			const int u2 = A::add(h1m1, NIO);
			bnew = max(A::add(u2, dnn[r + 1]), vb);
			he = max(he, A::add(bnew, acn[r]));
			cnew = max(A::add(u2, dnn[r + 2]), vc);
			he = max(he, A::add(cnew, acn[r + 1]));
			he = max(he, A::add(h1, NFS));
			he = max(he, A::add(h2, NFS));
			he = max(he, A::add(h1m1, NFS));
			he = max(he, A::add(h2m1, NFS));
		}
		lh[r] = he;
		const int h = max(ic[r], he);
		hn[r] = h;
		h3 = h2, h2 = h1, h1 = h;
		d3 = d2, d2 = d1, d1 = dnew;
		va = anew, vb = bnew, vc = cnew;
	}
	o[0] = h1, o[1] = h2, o[2] = h3, o[3] = d1, o[4] = d2, o[5] = d3, o[6] = va, o[7] = vb, o[8] = vc;
}

/* Row keys.  A real column j contributes (v << S) + (2^S - 1 - j), v = H (+ end_bonus
 * at j = al-1); a padding column contributes (H << S) + PAD, below every real key.
 * Narrow: S = 14, for al <= 16384 and -32768 <= end_bonus <= 65535 (every key fits
 * in int32 and PAD keeps padding keys below the smallest real key).  Wide: S = 31
 * in int64, for any al and |end_bonus| <= 2^30. */
template <bool WIDE> struct KeyOf;
template <> struct KeyOf<false> {
	typedef int T;
	static constexpr int KW = 16384;
	static constexpr int MIN = INT_MIN, PAD = INT_MIN + (1 << 29);
	static __device__ __forceinline__ int hi(int k) { return k >> 14; }
	static __device__ __forceinline__ int col(int k) { return KW - 1 - (k & (KW - 1)); }
};
template <> struct KeyOf<true> {
	typedef long long T;
	static constexpr long long KW = 1ll << 31;
	static constexpr long long MIN = LLONG_MIN, PAD = -(1ll << 62);
	static __device__ __forceinline__ int hi(long long k) { return (int)(k >> 31); }
	static __device__ __forceinline__ int col(long long k) { return (int)(KW - 1 - (k & (KW - 1))); }
};

template <int MODE, bool PSSM, bool WIDE>
__device__ __forceinline__ void ext_job(plk_ext_job_t *__restrict__ J, const uint8_t *__restrict__ prep,
		const int8_t *__restrict__ pssm, int32_t *__restrict__ ring, ExtShared &sh, const plk_params_t &P,
		unsigned long long *cells_acc, const int lane, const int wib)
{
	typedef KeyOf<WIDE> K;
	typedef typename K::T KeyT;
	constexpr int R = PLK_ROWS, NEG = -32768;
	const int nl = J->nl, al = J->al, ncol = J->ncol, slen = J->slen;
	const uint8_t *nas = prep + J->prep_off, *aas = nas + nl;
	const int8_t *donor = (const int8_t*)(aas + al), *acceptor = donor + nl + 1;
	const int8_t *pq = PSSM ? pssm + J->pssm_off : 0;
	const bool left = J->left == 1, glob = J->left == 2; /* glob: plain global score, no x-drop scan */
	const int nr = nl - 2, nstrip = (nr + EXT_STRIP - 1) / EXT_STRIP;
	const int Pc = ncol > 32 ? ncol : 33;  /* >= 33 keeps lane 0's ring prefetch behind lane 31's writes */
	const int total = nstrip * Pc + 31;
	const int NGO = -P.go, NGE = -P.ge, NIO = -P.io, NFS = -P.fs, NGOE = -(P.go + P.ge);
	const int pen_len = 3 * al, xdrop = P.xdrop;
	int32_t *pre = sh.pre[wib];

	int c = -lane, k = 0, cs = 0, i0 = 0;
	int ip[R], lh[R], ic[R], hm[R], code[R], gim[R], dnn[R + 2], acn[R + 2], rmax[R];
	KeyT key[R];
	int ah1 = NEG, ah2 = NEG, ah3 = NEG, o[9];
#pragma unroll
	for (int q = 0; q < 9; ++q) o[q] = NEG;
#pragma unroll
	for (int r = 0; r < R; ++r) ip[r] = lh[r] = ic[r] = hm[r] = rmax[r] = NEG, code[r] = 0, gim[r] = 0, key[r] = K::MIN;
#pragma unroll
	for (int r = 0; r < R + 2; ++r) dnn[r] = acn[r] = 0;

	/* row-scan state (warp-uniform) */
	int best_sc = NEG, best_row = -1, best_col = 0, M = INT_MIN, ks = 0, next_scan = glob ? INT_MAX : 31 + ncol - 1;
	int last_row = nl - 1;  /* last row the reference processes: the x-drop row, else nl-1 */

	for (int s = 0; s < total; ++s) {
		int in[9];
#pragma unroll
		for (int q = 0; q < 9; ++q) in[q] = __shfl_up_sync(FULL, o[q], 1);
		const bool started = c >= 0 && k < nstrip;
		if (lane == 0 && started) {
			if (k > 0) cp_async_wait_all();
#pragma unroll
			for (int q = 0; q < 9; ++q) in[q] = k == 0 ? NEG : pre[q];
		}
		if (started && c == 0) { /* strip start: per-row constants, column -1 */
			i0 = 2 + k * EXT_STRIP + lane * R;
#pragma unroll
			for (int r = 0; r < R; ++r) {
				const int i = i0 + r;
				code[r] = i < nl ? nas[i] : 0;
				gim[r] = code[r] == 20 ? -P.fs : -P.ge;
				ip[r] = lh[r] = ic[r] = hm[r] = rmax[r] = NEG;
				key[r] = K::MIN;
			}
#pragma unroll
			for (int r = 0; r < R + 2; ++r) {
				const int pd = i0 - 1 + r, pa = i0 - 2 + r;
				dnn[r] = pd <= nl ? -donor[pd] : 0;
				acn[r] = pa <= nl ? -acceptor[pa] : 0;
			}
			ah1 = ah2 = ah3 = NEG;
			cs = 0;
		}
		const bool live = started && c < ncol && i0 < nl;
		const bool any_seg = __any_sync(FULL, live && cs == 0);  /* some lane starts a segment this step */
		/* the row maximum over the padding columns: with end_bonus >= 0 the real columns'
		 * maximum is already in the key, so it is kept only on steps where some lane pads */
		const bool track_rmax = __any_sync(FULL, live && c >= al) || P.end_bonus < 0;
		if (live) {
			/* segment hand-over of the striped schedule (nasw-sse.c:432-433 and the lazy-F loop):
			 * the carried insertion takes the hand-over candidates, and the first-pass H' and I
			 * restart at -inf -- H' through the cell's open penalty go_e, I by an addend that
			 * sends it below every candidate -- with one warp-uniform branch per step (a strip's
			 * first column needs no case of its own: its H', I and carried insertion are -inf) */
			const bool seg = cs == 0;
			const int go_e = seg ? -(1 << 28) : NGO;
			if (any_seg) {
				const int goe_e = seg ? NGOE : -(1 << 28), ge_e = seg ? NGE : -(1 << 28), seg_i = seg ? -(1 << 28) : 0;
#pragma unroll
				for (int r = 0; r < R; ++r) {
					ic[r] = max(Ar<MODE>::add(ic[r], NGE), max(Ar<MODE>::add(lh[r], goe_e), Ar<MODE>::add(ip[r], ge_e)));
					ip[r] += seg_i;
				}
			} else {
#pragma unroll
				for (int r = 0; r < R; ++r) ic[r] = Ar<MODE>::add(ic[r], NGE);
			}
			int sv[R];
			if (c < al) {
				if (PSSM) {
					const int8_t *pc = pq + (int64_t)(left ? al - 1 - c : c) * 22;
#pragma unroll
					for (int r = 0; r < R; ++r) sv[r] = __ldg(pc + code[r]);
				} else {
					const int *sct_b = sh.sct + 22 * aas[c];
#pragma unroll
					for (int r = 0; r < R; ++r) sv[r] = sct_b[code[r]];
				}
			} else {
#pragma unroll
				for (int r = 0; r < R; ++r) sv[r] = NEG;
			}
			int hn[R];
			cells_ext<MODE>(in, hm, ah1, ah2, ah3, c == 0 && i0 == 2, sv, gim, dnn, acn, ip, lh, ic,
					go_e, NGO, NGE, NIO, NFS, o, hn);
			const KeyT kc = c < al - 1 ? (KeyT)(K::KW - 1 - c)
				: c == al - 1 ? (KeyT)P.end_bonus * K::KW + (KeyT)(K::KW - 1 - c) : (KeyT)K::PAD;
			if (track_rmax) {
#pragma unroll
				for (int r = 0; r < R; ++r) rmax[r] = max(rmax[r], hn[r]);
			}
#pragma unroll
			for (int r = 0; r < R; ++r) key[r] = max(key[r], (KeyT)hn[r] * K::KW + kc);
			if (glob && c == al - 1) { /* the global score H(nl-1, al-1) (nasw-sse.c:559) */
				const int rl = nl - 1 - i0;
#pragma unroll
				for (int r = 0; r < R; ++r)
					if (r == rl) J->score = hn[r];
			}
			if (lane == 31 && k + 1 < nstrip) {
				int32_t *e = ring + (int64_t)c * PLK_RING_INTS;
#pragma unroll
				for (int q = 0; q < 9; ++q) __stcg(e + q, o[q]);
			}
			if (c == ncol - 1) { /* this lane's rows are complete: hand them to the strip scan */
#pragma unroll
				for (int r = 0; r < R; ++r) {
					sh.rts[wib][lane * R + r] = max(rmax[r], K::hi(key[r]));
					sh.rkey[wib][lane * R + r] = (long long)key[r];
				}
			}
#pragma unroll
			for (int r = 0; r < R; ++r) hm[r] = hn[r];
			ah1 = in[0], ah2 = in[1], ah3 = in[2];
		}
		__syncwarp();
		if (s == next_scan) { /* lane 31 finished strip ks: scan its rows in order */
			const int rb = 2 + ks * EXT_STRIP + lane * R;
			int tl[R], lp[R], lmax = INT_MIN;
#pragma unroll
			for (int r = 0; r < R; ++r) {
				const int i = rb + r;
				tl[r] = i < nl ? sh.rts[wib][lane * R + r] - ext_penalty(i - pen_len, P.ie_coef) : INT_MIN;
				lmax = max(lmax, tl[r]);
				lp[r] = lmax;
			}
			int incl = lmax;
#pragma unroll
			for (int off = 1; off < 32; off <<= 1) {
				const int v = __shfl_up_sync(FULL, incl, off);
				if (lane >= off) incl = max(incl, v);
			}
			int excl = __shfl_up_sync(FULL, incl, 1);
			if (lane == 0) excl = INT_MIN;
			const int base = max(M, excl);
			int br = R;  /* first row of this lane at which the x-drop test fires */
#pragma unroll
			for (int r = R - 1; r >= 0; --r)
				if (tl[r] != INT_MIN && max(base, lp[r]) - tl[r] > xdrop) br = r;
			const unsigned bm = __ballot_sync(FULL, br < R);
			const int brk_lane = bm ? __ffs(bm) - 1 : 32;
			const int brk_r = __shfl_sync(FULL, br, brk_lane & 31);
			int cmax = INT_MIN;
#pragma unroll
			for (int r = 0; r < R; ++r) {
				const bool consider = tl[r] != INT_MIN && (lane < brk_lane || (lane == brk_lane && r <= brk_r));
				if (consider) cmax = max(cmax, tl[r]);
			}
			int mx = cmax;
#pragma unroll
			for (int off = 16; off >= 1; off >>= 1) mx = max(mx, __shfl_xor_sync(FULL, mx, off));
			if (mx > M) { /* a later row improved the kept maximum: the first row reaching mx */
				int fr = R;
				long long fk = 0;
#pragma unroll
				for (int r = R - 1; r >= 0; --r) {
					const bool consider = tl[r] != INT_MIN && (lane < brk_lane || (lane == brk_lane && r <= brk_r));
					if (consider && tl[r] == mx) fr = r, fk = sh.rkey[wib][lane * R + r];
				}
				const unsigned fm = __ballot_sync(FULL, fr < R);
				const int fl = __ffs(fm) - 1;
				fr = __shfl_sync(FULL, fr, fl);
				fk = __shfl_sync(FULL, fk, fl);
				best_row = 2 + ks * EXT_STRIP + fl * R + fr;
				best_sc = K::hi((KeyT)fk);
				best_col = K::col((KeyT)fk);
				M = mx;
			}
			if (bm != 0) last_row = 2 + ks * EXT_STRIP + brk_lane * R + brk_r;
			const bool done = bm != 0 || ks == nstrip - 1;
			++ks, next_scan += Pc;
			__syncwarp();
			if (done) break;
		}
		/* advance; lane 0 prefetches the ring entry of its next position */
		++c;
		if (c > 0 && ++cs == slen) cs = 0;
		if (c == Pc) c = 0, ++k;
		if (lane == 0 && k >= 1 && k < nstrip && c < ncol) {
			const int32_t *e = ring + (int64_t)c * PLK_RING_INTS;
			cp_async16(pre, e), cp_async16(pre + 4, e + 4), cp_async16(pre + 8, e + 8);
		}
	}
	if (lane == 0) cp_async_wait_all();
	__syncwarp();
	if (lane == 0) {
		if (glob) J->nt_len = nl, J->aa_len = al, J->status = 0;
		else J->nt_len = best_row + 1, J->aa_len = best_col + 1, J->score = best_sc, J->status = best_row >= 2 ? 0 : -1;
		/* algorithmic cells: rows 2..last_row (the rows the reference's loop visits) x al */
		atomicAdd(cells_acc, (unsigned long long)((int64_t)(last_row - 1) * al));
	}
	__syncwarp();
}

template <int MODE, bool PSSM, bool WIDE>
__global__ void __launch_bounds__(32 * EXT_WARPS, 3)
k_ext_dp(plk_ext_job_t *__restrict__ jobs, const int32_t *__restrict__ order, int n_jobs, int32_t *counter,
		unsigned long long *cells_acc,
		const uint8_t *__restrict__ prep, const int8_t *__restrict__ pssm, int32_t *__restrict__ ring,
		int64_t ring_stride, plk_params_t P)
{
	__shared__ ExtShared sh;
	for (int x = threadIdx.x; x < 23 * 22; x += blockDim.x) { /* sct[b*22 + a] = s(a, b); b = 22 pads */
		const int b = x / 22, a = x % 22;
		sh.sct[x] = b < 22 ? P.sc[a * 22 + b] : -32768;
	}
	__syncthreads();
	const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
	int32_t *myring = ring + ((int64_t)blockIdx.x * EXT_WARPS + wib) * ring_stride;
	for (;;) {
		int idx = 0;
		if (lane == 0) idx = atomicAdd(counter, 1);
		idx = __shfl_sync(FULL, idx, 0);
		if (idx >= n_jobs) break;
		ext_job<MODE, PSSM, WIDE>(jobs + order[idx], prep, pssm, myring, sh, P, cells_acc, lane, wib);
	}
}

__global__ void k_ext_results(const plk_ext_job_t *__restrict__ jobs, int n_jobs, pl_ext_result_t *__restrict__ res)
{
	const int q = blockIdx.x * blockDim.x + threadIdx.x;
	if (q >= n_jobs) return;
	pl_ext_result_t r;
	r.nt_len = jobs[q].nt_len, r.aa_len = jobs[q].aa_len, r.score = jobs[q].score, r.status = jobs[q].status;
	res[q] = r;
}

/* ------------------------------------------------------------------ launchers */

extern "C" int plk_ext_results(const plk_ext_job_t *jobs, int32_t n_jobs, void *results, void *stream)
{
	if (n_jobs <= 0) return 0;
	k_ext_results<<<(n_jobs + 255) / 256, 256, 0, (cudaStream_t)stream>>>(jobs, n_jobs, (pl_ext_result_t*)results);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_ext_prep(const plk_ext_job_t *jobs, int32_t n_jobs, const uint8_t *nt, const uint8_t *aa,
		const uint8_t *ss, uint8_t *prep, const plk_params_t *p, void *stream)
{
	if (n_jobs <= 0) return 0;
	const int grid = n_jobs < 65535 ? n_jobs : 65535;
	k_ext_prep<<<grid, 128, 0, (cudaStream_t)stream>>>(jobs, n_jobs, nt, aa, ss, prep, *p);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

#define EXT_VARIANTS(X) X(0, false, false) X(0, true, false) X(0, false, true) X(0, true, true) \
	X(2, false, false) X(2, true, false) X(2, false, true) X(2, true, true)

static const void *ext_kernel(int mode, int variant)
{
	const bool pssm = variant & 1, wide = variant & 2;
#define PICK(M, PS, WI) if (mode == M && pssm == PS && wide == WI) return (const void*)k_ext_dp<M, PS, WI>;
	EXT_VARIANTS(PICK)
#undef PICK
	return 0;
}

extern "C" int plk_ext_warps_per_cta(void) { return EXT_WARPS; }

extern "C" int plk_ext_ctas_per_sm(int32_t mode, int32_t variant)
{
	int n = 0;
	const void *f = ext_kernel(mode, variant);
	if (!f) return -1;
	return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, 32 * EXT_WARPS, 0) == cudaSuccess ? n : -1;
}

extern "C" int plk_ext_dp(plk_ext_job_t *jobs, const int32_t *order, int32_t n_jobs, int32_t *counter,
		const uint8_t *prep, const int8_t *pssm, int32_t *ring, int64_t ring_stride_ints, int32_t n_ctas,
		int32_t mode, int32_t variant, const plk_params_t *p, void *stream)
{
	if (n_jobs <= 0) return 0;
	cudaStream_t st = (cudaStream_t)stream;
	cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int32_t), st);
	if (e != cudaSuccess) return (int)e;
	const dim3 grid(n_ctas), block(32 * EXT_WARPS);
	const bool ps = variant & 1, wi = variant & 2;
#define LAUNCH(M, PS, WI) if (mode == M && ps == PS && wi == WI) \
	k_ext_dp<M, PS, WI><<<grid, block, 0, st>>>(jobs, order, n_jobs, counter, (unsigned long long*)(counter + 2), \
			prep, pssm, ring, ring_stride_ints, *p);
	EXT_VARIANTS(LAUNCH)
#undef LAUNCH
	plk_add_launches(1);
	return (int)cudaGetLastError();
}
