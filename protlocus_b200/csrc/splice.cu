/*
 * splice.cu -- sm_100a kernels of the global spliced protein-to-DNA DP
 * (the GPU replacement of nasw-cuda.cu:151-401 and of the host backtrack
 * nasw-cuda.cu:676-707; semantics of nasw-sse.c:351-567 and :779-973).
 *
 * Kernels
 *   k_prep       per-position input preparation (nasw-sse.c:95-159): codon
 *                translation, donor/acceptor penalties with the int8 wrap of the
 *                reference, optional splice-score track.
 *   k_splice_dp  the DP.  One warp per job (persistent, jobs pulled from a
 *                length-sorted queue).  A job's rows are cut into strips of
 *                32*R rows; lane t owns rows [tR, tR+R) of the strip and walks
 *                the protein columns one per step, one step behind lane t-1
 *                (anti-diagonal wavefront).  The column state of the three rows
 *                above a lane (H and D of rows i-1..i-3, A/B/C of row i-1) comes
 *                from lane t-1 by __shfl_up_sync; lane 0 gets it from lane 31 of
 *                the previous strip through a per-warp ring in L2.  The
 *                reference's striped schedule (vsize lanes of slen columns, a
 *                first pass with the insertion chain restarted at every segment
 *                start, then the lazy-F correction) is reproduced exactly with
 *                three running values per row: ip (first-pass insertion), ic
 *                (carried insertion) and lh (first-pass H of the previous
 *                column).  Saturating int16 arithmetic is emulated in int32.
 *                Trace words (state in bits 0-3, extension and lazy-F flags) are written
 *                with one 16-byte store per lane per step into a diagonal-major
 *                layout, so every warp store is a contiguous 512-byte run.
 *   k_traceback  one thread per job walks the trace (nasw-sse.c:44-93) and
 *                writes the run-length merged CIGAR in reverse.
 *   k_scan / k_compact  exclusive scan of CIGAR lengths and the reversed copy
 *                into the dense output with ns_fix_tiny_UV (nasw-sse.c:34-42).
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include "plk.h"
#include "../../include/plgpu.h"

static unsigned long long g_launches = 0;

#include "dp_common.cuh"

/* ------------------------------------------------------------------ preparation */

__global__ void k_prep(const plk_job_t *__restrict__ jobs, int n_jobs, const uint8_t *__restrict__ nt,
		const uint8_t *__restrict__ aa, const uint8_t *__restrict__ ss, uint8_t *__restrict__ prep, plk_params_t P)
{
	__shared__ uint8_t s_nt4[256], s_aa20[256], s_codon[64];
	for (int x = threadIdx.x; x < 256; x += blockDim.x) s_nt4[x] = P.nt4[x], s_aa20[x] = P.aa20[x];
	for (int x = threadIdx.x; x < 64; x += blockDim.x) s_codon[x] = P.codon[x];
	__syncthreads();
	for (int jb = blockIdx.x; jb < n_jobs; jb += gridDim.x) {
		const plk_job_t J = jobs[jb];
		const int nl = J.nl, al = J.al;
		const uint8_t *ns = nt + J.nt_off, *as = aa + J.aa_off, *sst = J.ss_off >= 0 ? ss + J.ss_off : 0;
		uint8_t *nas = prep + J.prep_off, *aas = nas + nl;
		int8_t *donor = (int8_t*)(aas + al), *acceptor = donor + nl + 1;
		for (int j = threadIdx.x; j < al; j += blockDim.x) aas[j] = s_aa20[as[j]];
		for (int p = threadIdx.x; p <= nl; p += blockDim.x)
			prep_fwd_pos(p, ns, nl, sst, s_nt4, s_codon, P, nas, donor, acceptor);
	}
}

/* ------------------------------------------------------------------ the DP */

/* the R trace words of a lane and step, stored and loaded as one vector */
template <int R> struct TraceVec;
template <> struct TraceVec<8> { typedef uint4 T; };
template <> struct TraceVec<4> { typedef uint2 T; };

template <int R>
__device__ __forceinline__ void store_trace(uint16_t *p, const unsigned (&z)[R])
{
	uint32_t w[R / 2];
#pragma unroll
	for (int q = 0; q < R / 2; ++q) w[q] = (z[2 * q] & 0xffffu) | (z[2 * q + 1] << 16);
	*(typename TraceVec<R>::T*)p = *(const typename TraceVec<R>::T*)w;
}

/* Bytes of one staged row-input block: 32*R + 2 bytes starting anywhere inside a
 * 16-byte chunk, copied as whole chunks (R = 8 at most). */
#define ROWBLK 288

struct DpShared {
	int32_t sct[22 * 22];                               /* score table, transposed: sct[b*22 + a] */
	int32_t slot[2][PLK_WARPS_PER_CTA][PLK_RING_INTS];  /* warp-to-warp hand-off of a cooperative wavefront */
	int32_t job;
	int32_t pre[PLK_WARPS_PER_CTA][PLK_RING_INTS] __attribute__((aligned(16)));
	/* per warp, double-buffered by strip parity: the codons, donor and acceptor
	 * penalties of the warp's 32*R rows of a strip, staged ahead of the strip */
	uint8_t rows[PLK_WARPS_PER_CTA][2][3][ROWBLK] __attribute__((aligned(16)));
};

/* Stage the row inputs of the warp's block of a strip, rows [b, b + 32R): codons
 * nas[b..], donor[b-1..] and acceptor[b-2..], 32R+2 bytes each.  Each block is
 * copied as 16-byte cp.async chunks from the 16-byte boundary at or below its
 * start; chunks that start past the end of their array are skipped (their bytes
 * are never read: the readers apply the row bounds).  Lanes 1-31 issue the
 * copies; lane 0 keeps its own cp.async queue for the strip hand-off ring.  The
 * preparation arrays sit inside a 16-byte aligned allocation with at least 16
 * bytes after the last one. */
template <int R>
__device__ __forceinline__ void stage_rows(uint8_t (*buf)[ROWBLK], const uint8_t *nas, const int8_t *donor,
		const int8_t *acceptor, const int nl, const int b, const int lane)
{
	constexpr int CH = (32 * R + 2 + 15 + 15) / 16;  /* chunks per block */
	static_assert(CH * 16 <= ROWBLK, "row block");
	if (lane == 0) return;
#pragma unroll
	for (int g = lane - 1; g < 3 * CH; g += 31) {
		const int a = g / CH, j = g - a * CH;
		const uint8_t *s = a == 0 ? nas + b : (const uint8_t*)(a == 1 ? donor + b - 1 : acceptor + b - 2);
		const uint8_t *end = a == 0 ? nas + nl : (const uint8_t*)(a == 1 ? donor : acceptor) + nl + 1;
		const uint8_t *src = (const uint8_t*)((uintptr_t)s & ~(uintptr_t)15) + 16 * j;
		if (src < end) cp_async16(buf[a] + 16 * j, src);
	}
}


/*
 * Trace word of a cell (all modes): bits 0-3 = 15 - state (state 0..9 in the
 * candidate order of nasw-sse.c:464-536); extension bits of I (bit 4), D (bit 5),
 * C (bit 6), A (bit 12), B (bit 13); bit 14 = raised by the carried insertion (the
 * reference's lazy-F bit; state 1 when read without a pending extension).  Bits
 * 7-11 and 15 are undefined.  The positions let MODE 0 gather the six flags from
 * the signs of six differences with three byte permutes (a sign-replicated byte
 * per flag, two flags per permute) and three bit-selects.
 *
 * MODE 0 works in a scaled domain: every DP value is kept times 16, so the low
 * four bits of a running maximum can carry the index of the candidate that
 * set it.  A candidate k enters as value*16 + (15-k); the maximum of the
 * encoded candidates is the maximum value, ties going to the smallest k --
 * exactly the strictly-greater, first-wins order of the reference -- and no
 * compare/select per candidate is needed.  Values entering only the maximum
 * need no clamp at -32768: the running maximum starts clamped, so a value
 * below the floor can neither win nor tie.  Stored states (I, D, A, B, C) are
 * clamped exactly; sat(sat(x-a)-b) is max(max(x-a, NEG)-b, NEG).
 */
/* byte 0 = 0xFF if a < 0 else 0, byte 1 = the same for b (prmt selector nibbles with
 * the sign-replicate bit set: 0xB = byte 3 of a, 0xF = byte 3 of b) */
__device__ __forceinline__ unsigned sign_bytes(int a, int b)
{
	unsigned d;
	asm("prmt.b32 %0, %1, %2, 0x00FB;" : "=r"(d) : "r"(a), "r"(b));
	return d;
}

template <int NW, int R>
__device__ __forceinline__ void cells_scaled(const int (&in)[9], int (&hm)[R], const int ah1, const int ah2,
		const int ah3, const bool row2, const int *__restrict__ sct_b, const int (&code)[R],
		const int (&gi)[R], const int (&dn)[R + 2], const int (&ac)[R + 2],
		int (&ip)[R], int (&lh)[R], const int (&ic)[R], const int *__restrict__ c16, const int go_e, const int seg_i,
		int (&o)[9], unsigned (&z)[R], int (&hn)[R])
{
	/* The integer pipe is the bound, so the update is written in the DPX forms that
	 * issue one instruction each: __viaddmax_s32 (max(a + b, c)) for every clamped
	 * state, __vibmax_s32 (max with the a >= b predicate) where a trace bit is the
	 * comparison of the two operands of a max, and __vimax3_s32 to fold two
	 * candidates into the running maximum at once (their tag adds can issue on the
	 * FMA pipe).  The maximum of the encoded candidates does not depend on the
	 * order in which they are folded. */
	constexpr int N16 = -32768 * 16;
	const int GO = c16[0], GE = c16[1], IO = c16[2], F6 = c16[3], F7 = c16[4], F8 = c16[5], F9 = c16[6], FS = c16[7];
	int h1 = in[0], h2 = in[1], h3 = in[2], d1 = in[3], d2 = in[4], d3 = in[5], va = in[6], vb = in[7], vc = in[8];
#pragma unroll
	for (int r = 0; r < R; ++r) {
		int h1m1 = r >= 1 ? hm[r - 1] : ah1;
		int h2m1 = r >= 2 ? hm[r - 2] : (r == 1 ? ah1 : ah2);
		int h3m1 = r >= 3 ? hm[r - 3] : (r == 2 ? ah1 : (r == 1 ? ah2 : ah3));
		if (r == 0 && row2) h1m1 = FS, h2m1 = FS, h3m1 = 0; /* column -1 while row 2 is computed: {0, -fs, -fs} */
		/* each extension flag is the sign of a difference: x > y exactly when y - x < 0
		 * (|values| < 2^21, no overflow) */
		/* 1: I -- p4 = I(c-1) > H'(c-1) - go */
		const int t4 = __viaddmax_s32(lh[r], go_e, N16);     /* go_e: -go, or below the floor at a segment start */
		const int d4 = t4 - ip[r] - seg_i;
		ip[r] = __vimax3_s32(t4 - GE, ip[r] + seg_i - GE, N16);  /* max(max(t4, ip) - ge, floor) */
		/* 2: D -- p5 = D(i-3) > H(i-3) - go */
		const int u5 = __viaddmax_s32(h3, -GO, N16);
		const int d5 = u5 - d3;
		const int dnew = __vimax3_s32(u5 + gi[r], d3 + gi[r], N16);  /* max(max(u, D) + gi, floor) */
		/* 3-5: phase-0/1/2 introns */
		const int ua = __viaddmax_s32(h1, -IO, N16);
		const int t6 = __viaddmax_s32(ua, dn[r], N16);
		const int d6 = t6 - va;
		const int anew = max(t6, va);
		const int ub = __viaddmax_s32(h1m1, -IO, N16);
		const int t7 = __viaddmax_s32(ub, dn[r + 1], N16);
		const int d7 = t7 - vb;
		const int bnew = max(t7, vb);
		const int t8 = __viaddmax_s32(ub, dn[r + 2], N16);
		const int d8 = t8 - vc;
		const int cnew = max(t8, vc);
		/* candidates 0..9, each value*16 + (15 - k) */
		int he = __viaddmax_s32(h3m1, sct_b[code[r]], N16 + 15);   /* 0: H(i-3,j-1) + s(i,j) */
		he = __vimax3_s32(he, ip[r] + 14, dnew + 13);               /* 1: I, 2: D */
		he = __vimax3_s32(he, anew + ac[r + 2] + 12, bnew + ac[r] + 11); /* 3: A - a(i), 4: B - a(i-2) */
		he = __vimax3_s32(he, cnew + ac[r + 1] + 10, h1 + F6);      /* 5: C - a(i-1), 6: H(i-1,j) - f */
		he = __vimax3_s32(he, h2 + F7, h1m1 + F8);                  /* 7: H(i-2,j) - f, 8: H(i-1,j-1) - f */
		he = __viaddmax_s32(h2m1, F9, he);                          /* 9: H(i-2,j-1) - f */
		const int hfp = he & ~15;
		lh[r] = hfp;
		/* the carried insertion is a multiple of 16: ic > he exactly when ic > hfp */
		const int d9 = hfp - ic[r];
		const int h = max(hfp, ic[r]);
		const unsigned pa = sign_bytes(d4, d6);  /* p4 -> bit 4, p6 -> bit 12 */
		const unsigned pb = sign_bytes(d5, d7);  /* p5 -> bit 5, p7 -> bit 13 */
		const unsigned pc = sign_bytes(d8, d9);  /* p8 -> bit 6, p9 -> bit 14 */
		unsigned zz = (pa & 0x1010u) | (pb & ~0x1010u);
		zz = (zz & 0x3030u) | (pc & ~0x3030u);
		z[r] = ((unsigned)he & 0xFu) | (zz & ~0xFu);
		hn[r] = h;
		h3 = h2, h2 = h1, h1 = h;
		d3 = d2, d2 = d1, d1 = dnew;
		va = anew, vb = bnew, vc = cnew;
	}
	o[0] = h1, o[1] = h2, o[2] = h3, o[3] = d1, o[4] = d2, o[5] = d3, o[6] = va, o[7] = vb, o[8] = vc;
}

/* Straightforward formulation for the 32-bit width (MODE 1) and the doubly
 * clamped int16 case (MODE 2). */
template <int MODE, int R>
__device__ __forceinline__ void cells_plain(const int (&in)[9], int (&hm)[R], const int ah1, const int ah2,
		const int ah3, const bool row2, const bool seg, const bool first, const int *__restrict__ sct_b,
		const int (&code)[R], const int (&gi)[R], const int (&dn)[R + 2],
		const int (&ac)[R + 2], int (&ip)[R], int (&lh)[R], int (&ic)[R],
		const plk_params_t &P, int (&o)[9], unsigned (&z)[R], int (&hn)[R])
{
	typedef Ar<MODE> A;
	const int NEG = A::NEG, go = P.go, ge = P.ge, goe = P.go + P.ge, io = P.io, fs = P.fs;
	int h1 = in[0], h2 = in[1], h3 = in[2], d1 = in[3], d2 = in[4], d3 = in[5], va = in[6], vb = in[7], vc = in[8];
#pragma unroll
	for (int r = 0; r < R; ++r) {
		int h1m1 = r >= 1 ? hm[r - 1] : ah1;
		int h2m1 = r >= 2 ? hm[r - 2] : (r == 1 ? ah1 : ah2);
		int h3m1 = r >= 3 ? hm[r - 3] : (r == 2 ? ah1 : (r == 1 ? ah2 : ah3));
		if (r == 0 && row2) h1m1 = -fs, h2m1 = -fs, h3m1 = 0;
		const int S = sct_b[code[r]];
		const int dim1 = dn[r], di = dn[r + 1], dip1 = dn[r + 2], aim2 = ac[r], aim1 = ac[r + 1], ai = ac[r + 2];
		int it = 16, icr;
		if (seg) {
			const int hop = A::sub(lh[r], goe), iext = A::sub(ip[r], ge), c0 = max(hop, iext);
			const int older = A::sub(ic[r], ge);
			it = first ? 0 : (c0 >= older ? (iext > hop ? 16 : 0) : 16);
			icr = first ? NEG : max(c0, older);
			ip[r] = NEG, lh[r] = NEG;
		} else icr = A::sub(ic[r], ge);
		ic[r] = icr;
		int h, t, u, y = 0;
		unsigned zz = 0;
		h = A::add(h3m1, S);
		t = A::sub(lh[r], go);
		zz |= ip[r] > t ? 1u << 4 : 0u;
		t = max(t, ip[r]);
		ip[r] = A::sub(t, ge);
		y = ip[r] > h ? 1 : y;
		h = max(h, ip[r]);
		u = A::sub(h3, go);
		zz |= d3 > u ? 1u << 5 : 0u;
		t = A::sub(max(u, d3), gi[r]);
		const int dnew = t;
		y = t > h ? 2 : y;
		h = max(h, t);
		u = A::sub(h1, io);
		t = A::sub(u, dim1);
		zz |= va > t ? 1u << 12 : 0u;
		t = max(t, va);
		const int anew = t;
		t = A::sub(t, ai);
		y = t > h ? 3 : y;
		h = max(h, t);
		u = A::sub(h1m1, io);
		t = A::sub(u, di);
		zz |= vb > t ? 1u << 13 : 0u;
		t = max(t, vb);
		const int bnew = t;
		t = A::sub(t, aim2);
		y = t > h ? 4 : y;
		h = max(h, t);
		t = A::sub(u, dip1);
		zz |= vc > t ? 1u << 6 : 0u;
		t = max(t, vc);
		const int cnew = t;
		t = A::sub(t, aim1);
		y = t > h ? 5 : y;
		h = max(h, t);
		t = A::sub(h1, fs);
		y = t > h ? 6 : y;
		h = max(h, t);
		t = A::sub(h2, fs);
		y = t > h ? 7 : y;
		h = max(h, t);
		t = A::sub(h1m1, fs);
		y = t > h ? 8 : y;
		h = max(h, t);
		t = A::sub(h2m1, fs);
		y = t > h ? 9 : y;
		h = max(h, t);
		lh[r] = h;
		if (icr > h) { /* raised by the carried insertion */
			h = icr;
			zz = MODE == 1 ? ((unsigned)it | 14u | 1u << 14) /* 32-bit: the word is replaced by 1|i_trace, nasw-sse.c:949 */
				: (zz | (unsigned)(15 - y) | 1u << 14);
		} else zz |= (unsigned)(15 - y);
		z[r] = zz;
		hn[r] = h;
		h3 = h2, h2 = h1, h1 = h;
		d3 = d2, d2 = d1, d1 = dnew;
		va = anew, vb = bnew, vc = cnew;
	}
	o[0] = h1, o[1] = h2, o[2] = h3, o[3] = d1, o[4] = d2, o[5] = d3, o[6] = va, o[7] = vb, o[8] = vc;
}

/* One DP job on a wavefront of NW warps (32*NW lanes).  All threads of the
 * group call this with the same job; `L` is the lane index in the wavefront. */
template <int MODE, int NW, int R>
__device__ __forceinline__ void dp_job(plk_job_t *__restrict__ J, const uint8_t *__restrict__ prep,
		uint16_t *__restrict__ trace, int32_t *__restrict__ myring, DpShared &sh, const plk_params_t &P,
		const int L, const int wib)
{
	constexpr int NL = 32 * NW, HS = NL * R;
	constexpr int SC = MODE == 0 ? 16 : 1;                  /* value scale of the mode */
	const int NEG = Ar<MODE>::NEG * SC;
	const int lane = L & 31, w = L >> 5;
	const int nl = J->nl, al = J->al, slen = J->slen;
	const uint8_t *nas = prep + J->prep_off, *aas = nas + nl;
	const int8_t *donor = (const int8_t*)(aas + al), *acceptor = donor + nl + 1;
	uint16_t *tr = trace + J->trace_off;
	const int nr = nl - 2, nstrip = (nr + HS - 1) / HS;
	const int Pc = al > NL ? al : NL + 1;  /* period >= NL+1 keeps lane 0's one-step ring prefetch behind the writer */
	const int total = nstrip * Pc + NL - 1;
	int32_t *pre = sh.pre[wib];          /* lane 0's prefetched ring entry (cp.async target) */
	uint8_t (*rowbuf)[3][ROWBLK] = sh.rows[wib];
	const int *c16 = P.s16;             /* x16 penalties, read as kernel constants */
	const int GOE = P.s16[8], GE16 = P.s16[1];

	int c = -L, k = 0, cs = 0, dcol = 0, i0 = 0;
	int ip[R], lh[R], ic[R], hm[R], code[R], gi[R], dn[R + 2], ac[R + 2];
	int ah1 = NEG, ah2 = NEG, ah3 = NEG; /* H(i0-1..i0-3, c-1) */
	int o[9];
#pragma unroll
	for (int q = 0; q < 9; ++q) o[q] = NEG;
#pragma unroll
	for (int r = 0; r < R; ++r) ip[r] = lh[r] = ic[r] = hm[r] = NEG, code[r] = 0, gi[r] = 0;
#pragma unroll
	for (int r = 0; r < R + 2; ++r) dn[r] = ac[r] = 0;
	/* the first strip's row inputs, and the ring entry of the first strip (the -inf row) */
	stage_rows<R>(rowbuf[0], nas, donor, acceptor, nl, 2 + w * 32 * R, lane);
	if (L == 0) {
#pragma unroll
		for (int q = 0; q < 9; ++q) pre[q] = NEG;
	}
	cp_async_wait_all();
	__syncwarp();

	for (int s = 0; s < total; ++s) {
		if (__shfl_sync(FULL, c, 0) == 0) {
			/* lane 0 of the warp starts a strip: the strip's row inputs (staged one
			 * period ago) are visible after the wait; stage those of the next strip */
			cp_async_wait_all();
			__syncwarp();
			const int kn = (s - 32 * w) / Pc + 1;
			if (kn < nstrip) stage_rows<R>(rowbuf[kn & 1], nas, donor, acceptor, nl, 2 + kn * HS + w * 32 * R, lane);
		}
		/* column state of the rows above: lane-1's output of the previous step */
		int in[9];
#pragma unroll
		for (int q = 0; q < 9; ++q) in[q] = __shfl_up_sync(FULL, o[q], 1);
		const bool started = c >= 0 && k < nstrip;
		if (lane == 0 && started) {
			/* the ring entry (prefetched, -inf before the second strip) or the slot of the warp above */
			if (w == 0) cp_async_wait_all();
			const int32_t *p = w == 0 ? pre : sh.slot[(s - 1) & 1][wib - 1];
			const int4 v0 = *(const int4*)p, v1 = *(const int4*)(p + 4);
			in[0] = v0.x, in[1] = v0.y, in[2] = v0.z, in[3] = v0.w;
			in[4] = v1.x, in[5] = v1.y, in[6] = v1.z, in[7] = v1.w, in[8] = p[8];
		}
		if (started && c == 0) { /* strip start: per-row constants from the staged block, column -1 */
			i0 = 2 + k * HS + L * R;
			const int b = i0 - lane * R;
			const uint8_t *rb = &rowbuf[k & 1][0][0] + lane * R;
			const int on = (int)((uintptr_t)(nas + b) & 15), od = (int)((uintptr_t)(donor + b - 1) & 15),
				oa = (int)((uintptr_t)(acceptor + b - 2) & 15);
#pragma unroll
			for (int r = 0; r < R; ++r) {
				const int i = i0 + r;
				code[r] = i < nl ? rb[on + r] : 0;
				gi[r] = MODE == 0 ? -16 * (code[r] == 20 ? P.fs : P.ge) : (code[r] == 20 ? P.fs : P.ge);
				ip[r] = lh[r] = ic[r] = hm[r] = NEG;
			}
#pragma unroll
			for (int r = 0; r < R + 2; ++r) {
				const int pd = i0 - 1 + r, pa = i0 - 2 + r;
				const int dv = pd <= nl ? (int8_t)rb[ROWBLK + od + r] : 0, av = pa <= nl ? (int8_t)rb[2 * ROWBLK + oa + r] : 0;
				dn[r] = MODE == 0 ? -16 * dv : dv;
				ac[r] = MODE == 0 ? -16 * av : av;
			}
			ah1 = ah2 = ah3 = NEG;
			cs = 0, dcol = L % al;
		}
		const bool live = started && c < al && i0 < nl;
		const bool any_seg = __any_sync(FULL, live && cs == 0);  /* some lane starts a segment this step */
		if (live) {
			const bool seg = cs == 0, first = c == 0, row2 = first && i0 == 2;
			const int *sct_b = sh.sct + 22 * aas[c];
			int hn[R];
			unsigned z[R];
			if (MODE == 0) {
				/* the striped schedule's segment hand-over (nasw-sse.c:537-553): at a segment start
				 * the carried insertion takes the hand-over candidates, and the first-pass H' and I
				 * restart at -inf -- the cell reads them through go_e / seg_i, which push them below
				 * the floor, so no lane branches on its own segment start */
				const int go_e = seg ? -(1 << 28) : -c16[0], seg_i = seg ? -(1 << 28) : 0;
				if (any_seg) {
					const int goe_e = seg ? -GOE : -(1 << 28), ge_e = seg ? -GE16 : -(1 << 28);
#pragma unroll
					for (int r = 0; r < R; ++r)
						ic[r] = __viaddmax_s32(ic[r], -GE16, __viaddmax_s32(ip[r], ge_e, __viaddmax_s32(lh[r], goe_e, NEG)));
				} else {
#pragma unroll
					for (int r = 0; r < R; ++r) ic[r] = max(ic[r] - GE16, NEG);
				}
				cells_scaled<NW, R>(in, hm, ah1, ah2, ah3, row2, sct_b, code, gi, dn, ac, ip, lh, ic, c16, go_e, seg_i,
						o, z, hn);
			} else {
				cells_plain<MODE, R>(in, hm, ah1, ah2, ah3, row2, seg, first, sct_b, code, gi, dn, ac, ip, lh, ic, P,
						o, z, hn);
			}
			/* trace: one store of R 16-bit words per lane, contiguous across the lanes of a strip */
			store_trace<R>(tr + (((int64_t)k * al + dcol) * NL + L) * R, z);
			if (L == NL - 1) {
				int32_t *e = myring + (int64_t)c * PLK_RING_INTS;
#pragma unroll
				for (int q = 0; q < 9; ++q) __stcg(e + q, o[q]);
			}
#pragma unroll
			for (int r = 0; r < R; ++r) hm[r] = hn[r];
			ah1 = in[0], ah2 = in[1], ah3 = in[2];
		}
		if (NW > 1) {
			if (lane == 31) {
				int32_t *sl = sh.slot[s & 1][wib];
#pragma unroll
				for (int q = 0; q < 9; ++q) sl[q] = o[q];
			}
			__syncthreads();
		} else __syncwarp();
		/* advance; lane 0 of the wavefront prefetches the ring entry of its next position */
		++c;
		if (c > 0) {
			if (++cs == slen) cs = 0;
			if (++dcol >= al) dcol = 0;
		}
		if (c == Pc) c = 0, ++k;
		if (L == 0 && k >= 1 && k < nstrip && c < al) {
			const int32_t *e = myring + (int64_t)c * PLK_RING_INTS;
			cp_async16(pre, e), cp_async16(pre + 4, e + 4), cp_async16(pre + 8, e + 8);
		}
	}
	cp_async_wait_all();
	/* the final score H(nl-1, al-1): the lane holding row nl-1 in the last strip keeps
	 * that strip's last column in hm */
	{
		const int rl = nl - 1 - i0;
		if (rl >= 0 && rl < R) {
#pragma unroll
			for (int r = 0; r < R; ++r)
				if (r == rl) J->score = MODE == 0 ? hm[r] >> 4 : hm[r];
		}
	}
}

/* Persistent DP kernel: first every CTA takes cooperative jobs (a whole CTA per
 * job) until that queue is empty, then every warp takes solo jobs.  Both queues
 * are sorted by decreasing size on the host (longest-processing-time first). */
template <int MODE, int R>
__global__ void __launch_bounds__(32 * PLK_WARPS_PER_CTA, R == 8 ? 2 : 3)
k_splice_dp(plk_job_t *__restrict__ jobs, const int32_t *__restrict__ order_coop, int n_coop,
		const int32_t *__restrict__ order_solo, int n_solo, int32_t *counters,
		const uint8_t *__restrict__ prep, uint16_t *__restrict__ trace, int32_t *__restrict__ ring,
		int64_t ring_stride, plk_params_t P)
{
	__shared__ DpShared sh;
	for (int x = threadIdx.x; x < 22 * 22; x += blockDim.x) { /* sct[b*22 + a] = s(a, b), scaled and tagged in mode 0 */
		const int b = x / 22, a = x % 22, v = P.sc[a * 22 + b];
		sh.sct[x] = MODE == 0 ? v * 16 + 15 : v;
	}
	__syncthreads();
	const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
	for (;;) {
		if (threadIdx.x == 0) sh.job = atomicAdd(&counters[0], 1);
		__syncthreads();
		const int idx = sh.job;
		__syncthreads();
		if (idx >= n_coop) break;
		dp_job<MODE, PLK_WARPS_PER_CTA, R>(jobs + order_coop[idx], prep, trace,
				ring + (int64_t)blockIdx.x * PLK_WARPS_PER_CTA * ring_stride, sh, P, threadIdx.x, wib);
		__syncthreads();
	}
	int32_t *myring = ring + ((int64_t)blockIdx.x * PLK_WARPS_PER_CTA + wib) * ring_stride;
	for (;;) {
		int idx = 0;
		if (lane == 0) idx = atomicAdd(&counters[1], 1);
		idx = __shfl_sync(FULL, idx, 0);
		if (idx >= n_solo) break;
		dp_job<MODE, 1, R>(jobs + order_solo[idx], prep, trace, myring, sh, P, lane, wib);
		__syncwarp();
	}
}

/* ------------------------------------------------------------------ paired int16x2 DP (mode 3) */

/*
 * Two jobs with one protein and windows of one length -- the two strands of a
 * locus -- run in the two 16-bit halves of every 32-bit register, so one DPX
 * instruction (__viaddmax_s16x2: max(a + b, c); __vimax3_s16x2) updates the same
 * cell of both.  Values live in a biased 15-bit domain per half: v -> v + B, with
 * the reference's saturation floor (-32768) mapped to F.  The host admits a pair
 * only when every value the DP can reach provably stays within [F + 512,
 * 0x7fff - 512] after biasing: the 16-bit adds then never wrap, values at the
 * floor never meet real ones, and every clamp at F is exactly the reference's
 * _mm_subs_epi16 saturation.  Every value, and every sum formed on the way, lies in
 * [0, 0x7fff] per half, so the signed 16-bit forms order them as unsigned numbers.
 *
 * The first-winning candidate cannot ride in the low bits of the value as in the
 * 32-bit kernel.  Each cell stores ten bits "candidate k equals the maximum" (the
 * traceback takes the first set one: first wins, nasw-sse.c:517-530) and the six
 * extension / lazy-F comparisons.  Each bit comes out clean from one DPX step: for
 * c <= m per half, max(c + 1, m) - m is 1 exactly when c == m and 0 otherwise, in
 * both halves at once with no borrow between them; the candidates use the form
 * max(c, m - 1) - (m - 1), which takes a candidate that is a sum c = a + b in the
 * same step.  The subtraction and the placement of the bit are linear, so the whole
 * word is one sum of multiply-adds,
 *   z = sum_k max(c_k + 1, m_k) * 2^p_k  -  sum_k m_k * 2^p_k   (mod 2^32),
 * which runs on the FMA pipe (the multipliers are kernel constants) while the DPX
 * steps keep the ALU pipe.  Bit p of each half: p = k for candidates 0-9 (m = the
 * cell's maximum) and p = 10-15 for g4-g9 with m = the maximum the compared value
 * entered:
 *   g4: I opened from H' (not I-extended)   g5: D opened (not D-extended)
 *   g6/g7/g8: A/B/C opened (not extended)   g9: H' >= the carried insertion;
 * the traceback converts such a word to the layout of the other modes.
 */
struct DpSharedPair {
	int32_t slot[2][PLK_WARPS_PER_CTA][PLK_RING_INTS];
	int32_t job;
	int32_t pre[PLK_WARPS_PER_CTA][PLK_RING_INTS] __attribute__((aligned(16)));
	uint8_t rows[PLK_WARPS_PER_CTA][2][2][3][ROWBLK] __attribute__((aligned(16)));  /* [warp][job][parity][array] */
};
#define PAIR_SCT_WORDS (22 * 22 * 22)   /* [protein residue][codon residue of job 1][of job 2] */

__device__ __forceinline__ unsigned pk16(int a, int b) { return ((unsigned)a & 0xffffu) | ((unsigned)b << 16); }
/* per-half signed maximum of two */
__device__ __forceinline__ unsigned vmax2u(unsigned a, unsigned b)
{
	unsigned d;
	asm("max.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
	return d;
}

struct PairK { unsigned F2, GOn, GEn, IOn, FSn, GOEn, ONE; };

template <int R>
__device__ __forceinline__ void cells_pair(const unsigned (&in)[9], unsigned (&hm)[R], const unsigned ah1,
		const unsigned ah2, const unsigned ah3, const bool row2, const unsigned r2h, const unsigned r2f,
		const uint32_t *__restrict__ srow, const int (&cp)[R], const unsigned (&gi)[R], const unsigned (&dn)[R + 2],
		const unsigned (&ac)[R + 2], unsigned (&ip)[R], unsigned (&lh)[R], const unsigned (&ic)[R], const PairK &K,
		const plk_params_t &P, const unsigned go_e, const unsigned seg_i, unsigned (&o)[9], unsigned (&z)[R],
		unsigned (&hn)[R])
{
	unsigned h1 = in[0], h2 = in[1], h3 = in[2], d1 = in[3], d2 = in[4], d3 = in[5], va = in[6], vb = in[7], vc = in[8];
#pragma unroll
	for (int r = 0; r < R; ++r) {
		unsigned h1m1 = r >= 1 ? hm[r - 1] : ah1;
		unsigned h2m1 = r >= 2 ? hm[r - 2] : (r == 1 ? ah1 : ah2);
		unsigned h3m1 = r >= 3 ? hm[r - 3] : (r == 2 ? ah1 : (r == 1 ? ah2 : ah3));
		if (r == 0 && row2) h1m1 = r2f, h2m1 = r2f, h3m1 = r2h; /* column -1 while row 2 is computed: {0, -fs, -fs} */
		/* 1: I -- g4 = H'(c-1) - go >= I(c-1) */
		const unsigned t4 = __viaddmax_s16x2(lh[r], go_e, K.F2);  /* go_e: -go, or below the floor at a segment start */
		const unsigned m4 = __viaddmax_s16x2(ip[r], seg_i, t4);
		const unsigned ipn = __viaddmax_s16x2(m4, K.GEn, K.F2);
		ip[r] = ipn;
		/* 2: D -- g5 = H(i-3) - go >= D(i-3) */
		const unsigned u5 = __viaddmax_s16x2(h3, K.GOn, K.F2);
		const unsigned m5 = vmax2u(u5, d3);
		const unsigned dnew = __viaddmax_s16x2(m5, gi[r], K.F2);
		/* 3-5: phase-0/1/2 introns */
		const unsigned ua = __viaddmax_s16x2(h1, K.IOn, K.F2);
		const unsigned t6 = __viaddmax_s16x2(ua, dn[r], K.F2);
		const unsigned anew = vmax2u(t6, va);
		const unsigned ub = __viaddmax_s16x2(h1m1, K.IOn, K.F2);
		const unsigned t7 = __viaddmax_s16x2(ub, dn[r + 1], K.F2);
		const unsigned bnew = vmax2u(t7, vb);
		const unsigned t8 = __viaddmax_s16x2(ub, dn[r + 2], K.F2);
		const unsigned cnew = vmax2u(t8, vc);
		/* candidates 0-5 and the frameshifts 6-9 into the maximum he.  c0 keeps its floor F;
		 * c3-c5 (A - a(i), B - a(i-2), C - a(i-1)) are folded in as sums: he >= c0 >= F, so
		 * their floors cannot change he (every sum stays in [0, 0x7fff]) */
		const unsigned c0 = __viaddmax_s16x2(h3m1, srow[cp[r]], K.F2);  /* H(i-3,j-1) + s(i,j) */
		unsigned x = __vimax3_s16x2(c0, ipn, dnew);
		x = __viaddmax_s16x2(anew, ac[r + 2], x);
		x = __viaddmax_s16x2(bnew, ac[r], x);
		x = __viaddmax_s16x2(cnew, ac[r + 1], x);
		const unsigned fsm = vmax2u(__vimax3_s16x2(h1, h2, h1m1), h2m1);
		const unsigned he = __viaddmax_s16x2(fsm, K.FSn, x);     /* 6-9: H(i-1|i-2, j|j-1) - fs */
		lh[r] = he;
		const unsigned h = vmax2u(he, ic[r]);                  /* the carried insertion */
		/* the sixteen bits of both cells.  Candidate k's bit is max(c_k, he - 1) - (he - 1),
		 * 1 exactly when c_k == he (c_k <= he; he - 1 per half has no borrow, he >= F); a
		 * floor cell (he == F) sets bit 0, c0 == F, so its first set bit, the state the
		 * traceback reads, is the reference's 0 whatever the unfloored sums give.  The g
		 * bits are max(c + 1, m) - m with m the maximum the value entered.  The maxima run
		 * on the ALU pipe, the sum on the FMA pipe. */
		const unsigned hm1 = he * (unsigned)P.pair_pw[0] - 0x00010001u;
		unsigned zz = vmax2u(c0, hm1);
		zz += vmax2u(ipn, hm1) * (unsigned)P.pair_pw[1];
		zz += vmax2u(dnew, hm1) * (unsigned)P.pair_pw[2];
		zz += __viaddmax_s16x2(anew, ac[r + 2], hm1) * (unsigned)P.pair_pw[3];
		zz += __viaddmax_s16x2(bnew, ac[r], hm1) * (unsigned)P.pair_pw[4];
		zz += __viaddmax_s16x2(cnew, ac[r + 1], hm1) * (unsigned)P.pair_pw[5];
		zz += __viaddmax_s16x2(h1, K.FSn, hm1) * (unsigned)P.pair_pw[6];
		zz += __viaddmax_s16x2(h2, K.FSn, hm1) * (unsigned)P.pair_pw[7];
		zz += __viaddmax_s16x2(h1m1, K.FSn, hm1) * (unsigned)P.pair_pw[8];
		zz += __viaddmax_s16x2(h2m1, K.FSn, hm1) * (unsigned)P.pair_pw[9];
		zz += hm1 * (unsigned)P.pair_nw[0];
		zz += __viaddmax_s16x2(t4, K.ONE, m4) * (unsigned)P.pair_pw[10] + m4 * (unsigned)P.pair_nw[1];
		zz += __viaddmax_s16x2(u5, K.ONE, m5) * (unsigned)P.pair_pw[11] + m5 * (unsigned)P.pair_nw[2];
		zz += __viaddmax_s16x2(t6, K.ONE, anew) * (unsigned)P.pair_pw[12] + anew * (unsigned)P.pair_nw[3];
		zz += __viaddmax_s16x2(t7, K.ONE, bnew) * (unsigned)P.pair_pw[13] + bnew * (unsigned)P.pair_nw[4];
		zz += __viaddmax_s16x2(t8, K.ONE, cnew) * (unsigned)P.pair_pw[14] + cnew * (unsigned)P.pair_nw[5];
		zz += __viaddmax_s16x2(he, K.ONE, h) * (unsigned)P.pair_pw[15] + h * (unsigned)P.pair_nw[6];
		z[r] = zz;
		hn[r] = h;
		h3 = h2, h2 = h1, h1 = h;
		d3 = d2, d2 = d1, d1 = dnew;
		va = anew, vb = bnew, vc = cnew;
	}
	o[0] = h1, o[1] = h2, o[2] = h3, o[3] = d1, o[4] = d2, o[5] = d3, o[6] = va, o[7] = vb, o[8] = vc;
}

template <int R>
__device__ __forceinline__ void store_trace_pair(uint16_t *pa, uint16_t *pb, const unsigned (&z)[R])
{ /* low halves to the first job's trace, high halves to the second's */
	uint32_t wa[R / 2], wb[R / 2];
#pragma unroll
	for (int q = 0; q < R / 2; ++q) wa[q] = __byte_perm(z[2 * q], z[2 * q + 1], 0x5410), wb[q] = __byte_perm(z[2 * q], z[2 * q + 1], 0x7632);
	*(typename TraceVec<R>::T*)pa = *(const typename TraceVec<R>::T*)wa;
	*(typename TraceVec<R>::T*)pb = *(const typename TraceVec<R>::T*)wb;
}

/* One pair of jobs on a wavefront of NW warps; the structure of dp_job with packed values. */
template <int NW, int R>
__device__ __forceinline__ void dp_pair(plk_job_t *__restrict__ JA, plk_job_t *__restrict__ JB,
		const uint8_t *__restrict__ prep, uint16_t *__restrict__ trace, int32_t *__restrict__ myring,
		DpSharedPair &sh, const uint32_t *__restrict__ sct2, const PairK &K, const plk_params_t &P,
		const int L, const int wib)
{
	constexpr int NL = 32 * NW, HS = NL * R;
	const unsigned NEG = K.F2;
	const int lane = L & 31, w = L >> 5;
	const int nl = JA->nl, al = JA->al, slen = JA->slen;
	const uint8_t *nasA = prep + JA->prep_off, *aas = nasA + nl;
	const int8_t *donA = (const int8_t*)(aas + al), *accA = donA + nl + 1;
	const uint8_t *nasB = prep + JB->prep_off;
	const int8_t *donB = (const int8_t*)(nasB + nl + al), *accB = donB + nl + 1;
	uint16_t *trA = trace + JA->trace_off, *trB = trace + JB->trace_off;
	const int nr = nl - 2, nstrip = (nr + HS - 1) / HS;
	const int Pc = al > NL ? al : NL + 1;
	const int total = nstrip * Pc + NL - 1;
	int32_t *pre = sh.pre[wib];
	uint8_t (*rowA)[3][ROWBLK] = sh.rows[wib][0], (*rowB)[3][ROWBLK] = sh.rows[wib][1];
	const unsigned r2h = P.pair_b * 0x10001u, r2f = (unsigned)(P.pair_b - P.fs) * 0x10001u;

	int c = -L, k = 0, cs = 0, dcol = 0, i0 = 0;
	unsigned ip[R], lh[R], ic[R], hm[R], gi[R], dn[R + 2], ac[R + 2];
	int cp[R];
	unsigned ah1 = NEG, ah2 = NEG, ah3 = NEG;
	unsigned o[9];
#pragma unroll
	for (int q = 0; q < 9; ++q) o[q] = NEG;
#pragma unroll
	for (int r = 0; r < R; ++r) ip[r] = lh[r] = ic[r] = hm[r] = NEG, cp[r] = 0, gi[r] = 0;
#pragma unroll
	for (int r = 0; r < R + 2; ++r) dn[r] = ac[r] = 0;
	stage_rows<R>(rowA[0], nasA, donA, accA, nl, 2 + w * 32 * R, lane);
	stage_rows<R>(rowB[0], nasB, donB, accB, nl, 2 + w * 32 * R, lane);
	if (L == 0) {
#pragma unroll
		for (int q = 0; q < 9; ++q) pre[q] = (int32_t)NEG;
	}
	cp_async_wait_all();
	__syncwarp();

	for (int s = 0; s < total; ++s) {
		if (__shfl_sync(FULL, c, 0) == 0) {
			cp_async_wait_all();
			__syncwarp();
			const int kn = (s - 32 * w) / Pc + 1;
			if (kn < nstrip) {
				stage_rows<R>(rowA[kn & 1], nasA, donA, accA, nl, 2 + kn * HS + w * 32 * R, lane);
				stage_rows<R>(rowB[kn & 1], nasB, donB, accB, nl, 2 + kn * HS + w * 32 * R, lane);
			}
		}
		unsigned in[9];
#pragma unroll
		for (int q = 0; q < 9; ++q) in[q] = __shfl_up_sync(FULL, o[q], 1);
		const bool started = c >= 0 && k < nstrip;
		if (lane == 0 && started) {
			if (w == 0) cp_async_wait_all();
			const int32_t *p = w == 0 ? pre : sh.slot[(s - 1) & 1][wib - 1];
			const int4 v0 = *(const int4*)p, v1 = *(const int4*)(p + 4);
			in[0] = v0.x, in[1] = v0.y, in[2] = v0.z, in[3] = v0.w;
			in[4] = v1.x, in[5] = v1.y, in[6] = v1.z, in[7] = v1.w, in[8] = p[8];
		}
		if (started && c == 0) { /* strip start: per-row constants of both jobs, column -1 */
			i0 = 2 + k * HS + L * R;
			const int b = i0 - lane * R;
			const uint8_t *ra = &rowA[k & 1][0][0] + lane * R, *rb = &rowB[k & 1][0][0] + lane * R;
			const int onA = (int)((uintptr_t)(nasA + b) & 15), odA = (int)((uintptr_t)(donA + b - 1) & 15),
				oaA = (int)((uintptr_t)(accA + b - 2) & 15);
			const int onB = (int)((uintptr_t)(nasB + b) & 15), odB = (int)((uintptr_t)(donB + b - 1) & 15),
				oaB = (int)((uintptr_t)(accB + b - 2) & 15);
#pragma unroll
			for (int r = 0; r < R; ++r) {
				const int i = i0 + r;
				const int ca = i < nl ? ra[onA + r] : 0, cb = i < nl ? rb[onB + r] : 0;
				cp[r] = ca * 22 + cb;
				gi[r] = pk16(-(ca == 20 ? P.fs : P.ge), -(cb == 20 ? P.fs : P.ge));
				ip[r] = lh[r] = ic[r] = hm[r] = NEG;
			}
#pragma unroll
			for (int r = 0; r < R + 2; ++r) {
				const int pd = i0 - 1 + r, pa = i0 - 2 + r;
				const int dva = pd <= nl ? (int8_t)ra[ROWBLK + odA + r] : 0, dvb = pd <= nl ? (int8_t)rb[ROWBLK + odB + r] : 0;
				const int ava = pa <= nl ? (int8_t)ra[2 * ROWBLK + oaA + r] : 0, avb = pa <= nl ? (int8_t)rb[2 * ROWBLK + oaB + r] : 0;
				dn[r] = pk16(-dva, -dvb);
				ac[r] = pk16(-ava, -avb);
			}
			ah1 = ah2 = ah3 = NEG;
			cs = 0, dcol = L % al;
		}
		const bool live = started && c < al && i0 < nl;
		const bool any_seg = __any_sync(FULL, live && cs == 0);  /* some lane starts a segment this step */
		if (live) {
			const bool seg = cs == 0, first = c == 0, row2 = first && i0 == 2;
			const uint32_t *srow = sct2 + 484 * aas[c];
			unsigned hn[R], z[R];
			/* the striped schedule's segment hand-over (nasw-sse.c:537-553), as in the 32-bit
			 * kernel: an addend of 0x8000 per half sends a value below the floor (every value
			 * is in [0, 0x7fff], so the sum is negative as a signed half) */
			const unsigned go_e = seg ? 0x80008000u : K.GOn, seg_i = seg ? 0x80008000u : 0u;
			if (any_seg) {
				const unsigned goe_e = seg ? K.GOEn : 0x80008000u, ge_e = seg ? K.GEn : 0x80008000u;
#pragma unroll
				for (int r = 0; r < R; ++r)
					ic[r] = __viaddmax_s16x2(ic[r], K.GEn, __viaddmax_s16x2(ip[r], ge_e, __viaddmax_s16x2(lh[r], goe_e, NEG)));
			} else {
#pragma unroll
				for (int r = 0; r < R; ++r) ic[r] = __viaddmax_s16x2(ic[r], K.GEn, NEG);
			}
			cells_pair<R>(in, hm, ah1, ah2, ah3, row2, r2h, r2f, srow, cp, gi, dn, ac, ip, lh, ic, K, P, go_e, seg_i,
					o, z, hn);
			const int64_t toff = (((int64_t)k * al + dcol) * NL + L) * R;
			store_trace_pair<R>(trA + toff, trB + toff, z);
			if (L == NL - 1) {
				int32_t *e = myring + (int64_t)c * PLK_RING_INTS;
#pragma unroll
				for (int q = 0; q < 9; ++q) __stcg(e + q, (int32_t)o[q]);
			}
#pragma unroll
			for (int r = 0; r < R; ++r) hm[r] = hn[r];
			ah1 = in[0], ah2 = in[1], ah3 = in[2];
		}
		if (NW > 1) {
			if (lane == 31) {
				int32_t *sl = sh.slot[s & 1][wib];
#pragma unroll
				for (int q = 0; q < 9; ++q) sl[q] = (int32_t)o[q];
			}
			__syncthreads();
		} else __syncwarp();
		++c;
		if (c > 0) {
			if (++cs == slen) cs = 0;
			if (++dcol >= al) dcol = 0;
		}
		if (c == Pc) c = 0, ++k;
		if (L == 0 && k >= 1 && k < nstrip && c < al) {
			const int32_t *e = myring + (int64_t)c * PLK_RING_INTS;
			cp_async16(pre, e), cp_async16(pre + 4, e + 4), cp_async16(pre + 8, e + 8);
		}
	}
	cp_async_wait_all();
	{ /* H(nl-1, al-1) of both jobs, unbiased */
		const int rl = nl - 1 - i0;
		if (rl >= 0 && rl < R) {
#pragma unroll
			for (int r = 0; r < R; ++r)
				if (r == rl) JA->score = (int)(hm[r] & 0xffffu) - P.pair_b, JB->score = (int)(hm[r] >> 16) - P.pair_b;
		}
	}
}

template <int R>
__global__ void __launch_bounds__(32 * PLK_WARPS_PER_CTA, R == 8 ? 2 : 3)
k_splice_pair(plk_job_t *__restrict__ jobs, const int32_t *__restrict__ order_coop, int n_coop,
		const int32_t *__restrict__ order_solo, int n_solo, int32_t *counters,
		const uint8_t *__restrict__ prep, uint16_t *__restrict__ trace, int32_t *__restrict__ ring,
		int64_t ring_stride, plk_params_t P)
{
	__shared__ DpSharedPair sh;
	extern __shared__ __align__(16) uint32_t pair_sct[];  /* [a][ca][cb] = s(ca, a) | s(cb, a) << 16 */
	for (int x = threadIdx.x; x < PAIR_SCT_WORDS; x += blockDim.x) {
		const int a = x / 484, ca = (x / 22) % 22, cb = x % 22;
		pair_sct[x] = pk16(P.sc[ca * 22 + a], P.sc[cb * 22 + a]);
	}
	PairK K;
	K.F2 = (unsigned)P.pair_f * 0x10001u;
	K.GOn = pk16(-P.go, -P.go), K.GEn = pk16(-P.ge, -P.ge), K.IOn = pk16(-P.io, -P.io);
	K.FSn = pk16(-P.fs, -P.fs), K.GOEn = pk16(-(P.go + P.ge), -(P.go + P.ge));
	K.ONE = 0x00010001u;
	__syncthreads();
	const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
	for (;;) {
		if (threadIdx.x == 0) sh.job = atomicAdd(&counters[0], 1);
		__syncthreads();
		const int idx = sh.job;
		__syncthreads();
		if (idx >= n_coop) break;
		plk_job_t *J = jobs + order_coop[idx];
		dp_pair<PLK_WARPS_PER_CTA, R>(J, jobs + J->pair, prep, trace,
				ring + (int64_t)blockIdx.x * PLK_WARPS_PER_CTA * ring_stride, sh, pair_sct, K, P, threadIdx.x, wib);
		__syncthreads();
	}
	int32_t *myring = ring + ((int64_t)blockIdx.x * PLK_WARPS_PER_CTA + wib) * ring_stride;
	for (;;) {
		int idx = 0;
		if (lane == 0) idx = atomicAdd(&counters[1], 1);
		idx = __shfl_sync(FULL, idx, 0);
		if (idx >= n_solo) break;
		plk_job_t *J = jobs + order_solo[idx];
		dp_pair<1, R>(J, jobs + J->pair, prep, trace, myring, sh, pair_sct, K, P, lane, wib);
		__syncwarp();
	}
}

/* ------------------------------------------------------------------ traceback */

/* trace-word bit of the extension flag of state 1..5 (I, D, A, B, C) */
__device__ __forceinline__ int tb_ext_bit(int state) { return (0x6DC540 >> (4 * state)) & 15; }

__device__ __forceinline__ void tb_push(uint32_t *out, int &n, uint32_t op, int len)
{ /* ns_push_cigar merge rule (nasw.h:219-229) */
	if (n == 0 || op != (out[n - 1] & 0xf) || op == NS_CIGAR_F || op == NS_CIGAR_G) out[n++] = (uint32_t)len << 4 | op;
	else out[n - 1] += (uint32_t)len << 4;
}

/* Traceback: one warp per job.  The walk is inherently sequential, so the warp
 * stages the trace words around the current cell in shared memory -- a tile of
 * 8 row-chunks (64 rows) x 32 columns, one coalesced round of 16-byte loads --
 * and lane 0 walks inside the tile until the path leaves it. */
#define TB_GROUPS 8   /* 8-row groups per tile: 64 rows */
#define TB_COLS 32
#define TB_WARPS 8

/* the R trace words of chunk ch (R rows of one lane of a strip) in column col, into w[0..R) */
__device__ __forceinline__ void tb_load_chunk(const uint16_t *__restrict__ tr, int R, int nlanes, int al, int ch, int col,
		uint16_t (&w)[8])
{
	const int ra = ch * R, hs = nlanes * R, k = ra / hs, t = ch % nlanes;
	int d = col + t;
	if (d >= al) d %= al;
	const uint16_t *src = tr + (((int64_t)k * al + d) * nlanes + t) * R;
	if (R == 8) {
		const uint4 v = *(const uint4*)src;
		*(uint4*)w = v;
	} else {
		const uint2 v = *(const uint2*)src;
		*(uint2*)w = v;
	}
}

/* a trace word of the paired kernel in the layout of the other modes (15 - state in
 * bits 0-3, extension bits I 4, D 5, C 6, A 12, B 13, carried-insertion bit 14) */
__device__ __forceinline__ uint16_t tb_pair_norm(unsigned x)
{
	const unsigned state = __ffs(x & 0x3ffu) - 1;  /* the first candidate equal to the maximum */
	const unsigned n = ~x;                         /* the g bits are negated flags */
	return (uint16_t)((15u - state) | (n >> 6 & 0x30u) | (n >> 8 & 0x40u) | (n & 0x3000u) | (n >> 1 & 0x4000u));
}

__device__ __forceinline__ void tb_norm8(uint16_t (&w)[8], const bool pair)
{
	if (!pair) return;
#pragma unroll
	for (int r = 0; r < 8; ++r) w[r] = tb_pair_norm(w[r]);
}

__global__ void __launch_bounds__(32 * TB_WARPS) k_traceback(plk_job_t *__restrict__ jobs,
		const int32_t *__restrict__ order, int n_order, const uint16_t *__restrict__ trace, uint32_t *__restrict__ tmp)
{
	__shared__ uint4 s_tile[TB_WARPS][TB_GROUPS][TB_COLS]; /* the trace words of 8 rows per entry */
	const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
	const int q = blockIdx.x * TB_WARPS + wib;
	if (q >= n_order) return;
	plk_job_t *J = jobs + order[q];
	const int nl = J->nl, al = J->al, R = J->rows;
	const uint16_t *tr = trace + J->trace_off;
	uint32_t *out = tmp + J->tmp_off;
	const int nlanes = 32 * J->nw;
	const bool pair = J->mode == 3;
	int i = nl - 1, j = al - 1, last = 0, n = 0;
	while (i >= 2 && j >= 0) {
		/* stage the tile whose top-right corner holds (i, j): 8-row groups, one or two chunks each */
		const int qc = (i - 2) / 8, jc = j;
#pragma unroll
		for (int m = 0; m < TB_GROUPS * TB_COLS / 32; ++m) {
			const int idx = lane + 32 * m, dq = idx / TB_COLS, dc = idx % TB_COLS;
			const int g = qc - dq, col = jc - dc;
			if (g >= 0 && col >= 0) {
				__align__(16) uint16_t w[8];
				if (R == 8) tb_load_chunk(tr, 8, nlanes, al, g, col, w);
				else {
					/* chunks 2g and 2g+1 sit in the same strip (nlanes is even) */
					__align__(8) uint16_t w2[8];
					tb_load_chunk(tr, 4, nlanes, al, 2 * g, col, w);
					tb_load_chunk(tr, 4, nlanes, al, 2 * g + 1, col, w2);
					*(uint2*)(w + 4) = *(const uint2*)w2;
				}
				tb_norm8(w, pair);
				s_tile[wib][dq][dc] = *(const uint4*)w;
			}
		}
		__syncwarp();
		if (lane == 0) {
			while (i >= 2 && j >= 0) {
				const int dq = qc - (i - 2) / 8, dc = jc - j;
				if (dq >= TB_GROUPS || dc >= TB_COLS) break;
				const uint16_t *cell = (const uint16_t*)&s_tile[wib][dq][dc];
				const int x = cell[(i - 2) % 8];
				const int state = last != 0 ? last : (x >> 14 & 1) ? 1 : 15 - (x & 0xf);
				const int ext = state >= 1 && state <= 5 ? (x >> tb_ext_bit(state)) & 1 : 0;
				switch (state) {
				case 0: tb_push(out, n, NS_CIGAR_M, 1), i -= 3, --j; break;
				case 1: tb_push(out, n, NS_CIGAR_I, 1), --j; break;
				case 2: tb_push(out, n, NS_CIGAR_D, 1), i -= 3; break;
				case 3: tb_push(out, n, NS_CIGAR_N, 1), --i; break;
				case 4: tb_push(out, n, NS_CIGAR_U, 1), --i; if (!ext) --j; break;
				case 5: tb_push(out, n, NS_CIGAR_V, 1), --i; if (!ext) --j; break;
				case 6: tb_push(out, n, NS_CIGAR_F, 1), --i; break;
				case 7: tb_push(out, n, NS_CIGAR_F, 2), i -= 2; break;
				case 8: tb_push(out, n, NS_CIGAR_G, 1), --i, --j; break;
				default: tb_push(out, n, NS_CIGAR_G, 2), i -= 2, --j; break;
				}
				last = state >= 1 && state <= 5 && ext ? state : 0;
			}
		}
		i = __shfl_sync(FULL, i, 0), j = __shfl_sync(FULL, j, 0);
		last = __shfl_sync(FULL, last, 0), n = __shfl_sync(FULL, n, 0);
		__syncwarp();
		/* Inside an intron run (A/B/C extended: the path climbs column j one row per
		 * step while the state's extension bit stays set) the warp scans 32*R rows of
		 * the column at once: each lane reads one R-row chunk, and the run ends at the
		 * highest row <= i whose bit is clear.  The rows of the run become one merged
		 * N/U/V op, exactly what the row-by-row walk pushes. */
		while (last >= 3 && last <= 5 && i >= 2 && j >= 0) {
			const int ch_top = (i - 2) / R, ch = ch_top - lane;
			const int bit = tb_ext_bit(last);
			int end_row = -1;
			if (ch >= 0) {
				__align__(16) uint16_t w[8];
				tb_load_chunk(tr, R, nlanes, al, ch, j, w);
				tb_norm8(w, pair);
				const int ra = ch * R;
#pragma unroll
				for (int r = 7; r >= 0; --r) {
					const int row = ra + 2 + r;
					if (r < R && end_row < 0 && row <= i && !((w[r] >> bit) & 1u)) end_row = row;
				}
			}
#pragma unroll
			for (int o = 16; o >= 1; o >>= 1) end_row = max(end_row, __shfl_xor_sync(FULL, end_row, o));
			const int low = max(2, (ch_top - 31) * R + 2);
			const int op = last == 3 ? NS_CIGAR_N : (last == 4 ? NS_CIGAR_U : NS_CIGAR_V);
			if (end_row >= low) { /* the run ends at end_row: its step clears the state (and moves j for U/V) */
				if (lane == 0) tb_push(out, n, op, i - end_row + 1);
				i = end_row - 1;
				if (last != 3) --j;
				last = 0;
			} else {              /* every row down to `low` extends the run */
				if (lane == 0) tb_push(out, n, op, i - low + 1);
				i = low - 1;
			}
			n = __shfl_sync(FULL, n, 0);
		}
	}
	if (lane == 0) {
		if (j > 0) tb_push(out, n, NS_CIGAR_I, j);
		if (i >= 0) {
			const int l = (i + 1) / 3, t = (i + 1) % 3;
			if (l > 0) tb_push(out, n, NS_CIGAR_D, l);
			if (t != 0) tb_push(out, n, NS_CIGAR_F, t);
		}
		J->n_tmp = n;
	}
}

/* exclusive scan of the CIGAR lengths in job order (single CTA) */
__global__ void k_scan(plk_job_t *jobs, int n_jobs, int64_t *total)
{
	__shared__ int64_t s_part[1024];
	const int tid = threadIdx.x, nt = blockDim.x;
	const int per = (n_jobs + nt - 1) / nt, b = tid * per, e = min(n_jobs, b + per);
	int64_t acc = 0;
	for (int q = b; q < e; ++q) acc += jobs[q].n_tmp;
	s_part[tid] = acc;
	__syncthreads();
	for (int off = 1; off < nt; off <<= 1) {
		int64_t v = tid >= off ? s_part[tid - off] : 0;
		__syncthreads();
		s_part[tid] += v;
		__syncthreads();
	}
	int64_t run = s_part[tid] - acc;
	for (int q = b; q < e; ++q) jobs[q].out_off = run, run += jobs[q].n_tmp;
	if (tid == nt - 1) *total = s_part[tid];
}

__global__ void k_compact(const plk_job_t *__restrict__ jobs, int n_jobs, const uint32_t *__restrict__ tmp,
		uint32_t *__restrict__ out, int64_t out_cap, pl_splice_result_t *__restrict__ res)
{
	const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
	if (w >= n_jobs) return;
	const plk_job_t J = jobs[w];
	const int n = J.n_tmp;
	const bool fits = J.out_off + n <= out_cap;
	for (int q = lane; q < n && fits; q += 32) {
		uint32_t x = tmp[J.tmp_off + n - 1 - q];
		const uint32_t op = x & 0xf;
		if ((op == NS_CIGAR_U || op == NS_CIGAR_V) && (x >> 4) < 3) x = x >> 4 << 4 | NS_CIGAR_G;
		out[J.out_off + q] = x;
	}
	if (lane == 0) {
		pl_splice_result_t r;
		r.score = J.score, r.n_cigar = n, r.cigar_off = J.out_off, r.mode = J.mode == 1 ? 32 : 16;
		r.status = fits ? J.status : -2;
		res[w] = r;
	}
}

/* ------------------------------------------------------------------ launchers */

extern "C" int plk_prep(const plk_job_t *jobs, int32_t n_jobs, const uint8_t *nt, const uint8_t *aa,
		const uint8_t *ss, uint8_t *prep, const plk_params_t *p, void *stream)
{
	if (n_jobs <= 0) return 0;
	const int grid = n_jobs < 65535 ? n_jobs : 65535;
	k_prep<<<grid, 256, 0, (cudaStream_t)stream>>>(jobs, n_jobs, nt, aa, ss, prep, *p);
	__sync_fetch_and_add(&g_launches, 1ull);
	return (int)cudaGetLastError();
}

template <int MODE, int R>
static int dp_occupancy()
{
	int n = 0;
	const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_splice_dp<MODE, R>, 32 * PLK_WARPS_PER_CTA, 0);
	return e == cudaSuccess ? n : -1;
}

#define PAIR_SMEM (PAIR_SCT_WORDS * 4)

template <int R>
static int pair_occupancy()
{
	int n = 0;
	if (cudaFuncSetAttribute(k_splice_pair<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, PAIR_SMEM) != cudaSuccess) return -1;
	const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_splice_pair<R>, 32 * PLK_WARPS_PER_CTA, PAIR_SMEM);
	return e == cudaSuccess ? n : -1;
}

extern "C" int plk_dp_ctas_per_sm(int32_t mode, int32_t rows)
{
	if (mode == 3) return rows == 4 ? pair_occupancy<4>() : pair_occupancy<8>();
	if (rows == 4) return mode == 1 ? dp_occupancy<1, 4>() : mode == 2 ? dp_occupancy<2, 4>() : dp_occupancy<0, 4>();
	return mode == 1 ? dp_occupancy<1, 8>() : mode == 2 ? dp_occupancy<2, 8>() : dp_occupancy<0, 8>();
}

extern "C" int plk_splice_dp(plk_job_t *jobs, const int32_t *order_coop, int32_t n_coop, const int32_t *order_solo,
		int32_t n_solo, int32_t *counters, const uint8_t *prep, uint16_t *trace, int32_t *ring,
		int64_t ring_stride_ints, int32_t n_ctas, int32_t mode, int32_t rows, const plk_params_t *p, void *stream)
{
	if (n_coop + n_solo <= 0) return 0;
	if (rows != 4 && rows != 8) return (int)cudaErrorInvalidValue;
	cudaStream_t st = (cudaStream_t)stream;
	cudaError_t e = cudaMemsetAsync(counters, 0, 2 * sizeof(int32_t), st);
	if (e != cudaSuccess) return (int)e;
	const dim3 grid(n_ctas), block(32 * PLK_WARPS_PER_CTA);
#define DP_LAUNCH(M, RR) k_splice_dp<M, RR><<<grid, block, 0, st>>>(jobs, order_coop, n_coop, order_solo, n_solo, \
		counters, prep, trace, ring, ring_stride_ints, *p)
	if (mode == 3) { /* pairs: order_* hold the first job of each pair (jobs[q].pair: the second) */
		if (rows == 4) k_splice_pair<4><<<grid, block, PAIR_SMEM, st>>>(jobs, order_coop, n_coop, order_solo, n_solo,
				counters, prep, trace, ring, ring_stride_ints, *p);
		else k_splice_pair<8><<<grid, block, PAIR_SMEM, st>>>(jobs, order_coop, n_coop, order_solo, n_solo,
				counters, prep, trace, ring, ring_stride_ints, *p);
	} else if (rows == 4) {
		if (mode == 1) DP_LAUNCH(1, 4); else if (mode == 2) DP_LAUNCH(2, 4); else DP_LAUNCH(0, 4);
	} else {
		if (mode == 1) DP_LAUNCH(1, 8); else if (mode == 2) DP_LAUNCH(2, 8); else DP_LAUNCH(0, 8);
	}
#undef DP_LAUNCH
	__sync_fetch_and_add(&g_launches, 1ull);
	return (int)cudaGetLastError();
}

extern "C" int plk_traceback(plk_job_t *jobs, const int32_t *order, int32_t n_order, const uint16_t *trace,
		uint32_t *tmp, void *stream)
{
	if (n_order <= 0) return 0;
	k_traceback<<<(n_order + TB_WARPS - 1) / TB_WARPS, 32 * TB_WARPS, 0, (cudaStream_t)stream>>>(jobs, order, n_order, trace, tmp);
	__sync_fetch_and_add(&g_launches, 1ull);
	return (int)cudaGetLastError();
}

extern "C" int plk_scan_compact(plk_job_t *jobs, int32_t n_jobs, const uint32_t *tmp, uint32_t *out, int64_t out_cap,
		int64_t *total_words, void *result_recs, void *stream)
{
	if (n_jobs <= 0) return 0;
	cudaStream_t st = (cudaStream_t)stream;
	k_scan<<<1, 1024, 0, st>>>(jobs, n_jobs, total_words);
	k_compact<<<(n_jobs * 32 + 255) / 256, 256, 0, st>>>(jobs, n_jobs, tmp, out, out_cap, (pl_splice_result_t*)result_recs);
	__sync_fetch_and_add(&g_launches, 2ull);
	return (int)cudaGetLastError();
}

extern "C" uint64_t plk_launches(void) { return __sync_fetch_and_add(&g_launches, 0ull); }
extern "C" void plk_add_launches(uint64_t n) { __sync_fetch_and_add(&g_launches, (unsigned long long)n); }
