/*
 * gapless.cu -- sm_100a kernel of the gapless X-drop candidate prefilter (the
 * device replacement of ns_gapless_xdrop_batch, nasw-cuda.cu:1151-1295; same
 * scores, bit for bit).
 *
 * One warp per candidate.  For each anchor (at most 32, nasw-cuda.cu:1174):
 *   seed    the warp loads the oriented bases of the anchor's block (plus the
 *           k-mer's reach) into shared memory once, translates every codon end
 *           of the window once, and each lane scores its deltas from the staged
 *           residues: kmer shared-memory lookups per delta instead of 3*kmer
 *           scattered genome reads.  The best seed is a warp max over the key
 *           (score << 32 | ~delta), so ties go to the smaller target end as in
 *           the reference's reduction;
 *   extend  left, then right: 32 steps at a time, one per lane, with warp
 *           prefix sums of the step scores and prefix maxima of the running
 *           score; the first step that leaves the sequence or breaks the X-drop
 *           ends the walk, and the best prefix (first step reaching it) is the
 *           reference's left_best / left_len (nasw-cuda.cu:1229-1252).
 * Lane 0 then sorts the segments and sums them greedily with the overlap rule
 * of nasw-cuda.cu:1259-1293.
 * Every index is bounds-checked against the buffer sizes, so malformed
 * candidates read as missing bases / residues instead of faulting.
 */
#include <cuda_runtime.h>
#include <limits.h>
#include <stdint.h>
#include "plk.h"
#include "../../include/plgpu.h"

#define FULL 0xffffffffu
#define GL_WARPS 8
#define GL_MAX_ANCHORS 32

extern "C" void plk_add_launches(uint64_t n);

struct GlArgs {
	const uint8_t *packed;
	int64_t bases;
	const uint8_t *queries;
	int64_t query_aa;
	const ns_gpu_gapless_candidate_t *cand;
	int32_t n_cand;
	const ns_gpu_gapless_anchor_t *anchors;
	int64_t n_anchors;
	int32_t block_width, kmer, xdrop, asize;
	int32_t *scores;
	unsigned long long *steps;  /* extension steps walked (for throughput accounting) */
};

__device__ __forceinline__ int gl_base(const GlArgs &A, const ns_gpu_gapless_candidate_t &C, int64_t pos)
{ /* nasw-cuda.cu:1151-1160 */
	if (pos < 0 || pos >= C.target_length) return 4;
	const int64_t a = C.target_offset + (C.reverse ? C.target_length - 1 - pos : pos);
	if (a < 0 || a >= A.bases) return 4;
	const int b = (__ldg(A.packed + (a >> 1)) >> ((a & 1) * 4)) & 0xf;
	return C.reverse && b < 4 ? 3 - b : b;
}

__device__ __forceinline__ int gl_aa(const GlArgs &A, const ns_gpu_gapless_candidate_t &C, const uint8_t *codon,
		int64_t end)
{ /* nasw-cuda.cu:1162-1170 */
	const int b0 = gl_base(A, C, end - 2), b1 = gl_base(A, C, end - 1), b2 = gl_base(A, C, end);
	return b0 < 4 && b1 < 4 && b2 < 4 ? codon[b0 << 4 | b1 << 2 | b2] : 20;
}

__device__ __forceinline__ int gl_query(const GlArgs &A, const ns_gpu_gapless_candidate_t &C, int64_t pos)
{
	const int64_t a = C.query_offset + pos;
	return a >= 0 && a < A.query_aa ? __ldg(A.queries + a) : 0;
}

/* One side of the X-drop extension, 32 steps per round.  dir = -1: left, +1: right.
 * Returns best (>= 0) and sets len (steps up to the first step reaching it). */
__device__ int gl_extend(const GlArgs &A, const ns_gpu_gapless_candidate_t &C, const uint8_t *codon,
		const int *sm, const int lane, const int dir, const int qend, const int64_t te0, int &len, int &walked)
{
	int carry = 0, best = 0, blen = 0, st = 0;
	const int kmer = A.kmer;
	walked = 0;
	for (;;) {
		const int step = st + lane + 1;
		int pos;
		int64_t te;
		bool valid;
		if (dir < 0) {
			pos = qend - kmer - (step - 1);
			te = te0 - (int64_t)(kmer - 1 + step) * 3;
			valid = pos >= 0 && te - 2 >= 0;
		} else {
			pos = qend + step;
			te = te0 + (int64_t)step * 3;
			valid = pos < C.query_length && te < C.target_length;
		}
		int v = 0;
		if (valid) {
			const int a = gl_aa(A, C, codon, te), q = gl_query(A, C, pos);
			v = sm[a * A.asize + (q < A.asize ? q : A.asize - 1)];
		}
		int incl = v;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int x = __shfl_up_sync(FULL, incl, o);
			if (lane >= o) incl += x;
		}
		const int running = carry + incl;
		const unsigned inval = __ballot_sync(FULL, !valid);
		const int first_invalid = inval ? __ffs(inval) - 1 : 32;
		int rmax = lane < first_invalid ? running : INT_MIN;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int x = __shfl_up_sync(FULL, rmax, o);
			if (lane >= o) rmax = max(rmax, x);
		}
		const int bestv = max(best, rmax);
		const unsigned brk = __ballot_sync(FULL, lane < first_invalid && bestv - running > A.xdrop);
		const int first_brk = brk ? __ffs(brk) - 1 : 32;
		const int stop = min(first_invalid, first_brk + 1);  /* steps processed in this round */
		int m = lane < stop ? running : INT_MIN;
#pragma unroll
		for (int o = 16; o >= 1; o >>= 1) m = max(m, __shfl_xor_sync(FULL, m, o));
		if (m > best) { /* strict improvement: the first step reaching it */
			const unsigned at = __ballot_sync(FULL, lane < stop && running == m);
			blen = st + __ffs(at);
			best = m;
		}
		walked += stop;
		if (stop < 32) break;
		carry = __shfl_sync(FULL, running, 31);
		st += 32;
	}
	len = blen;
	return best;
}

__global__ void __launch_bounds__(32 * GL_WARPS) k_gapless(GlArgs A, const int8_t *__restrict__ mat,
		const uint8_t *__restrict__ codon_g)
{
	extern __shared__ __align__(16) uint8_t gl_smem[];
	__shared__ int sm[32 * 32];
	__shared__ uint8_t codon[64];
	__shared__ int seg[GL_WARPS][3][GL_MAX_ANCHORS];
	const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
	for (int x = threadIdx.x; x < A.asize * A.asize; x += blockDim.x) sm[x] = mat[x];
	for (int x = threadIdx.x; x < 64; x += blockDim.x) codon[x] = codon_g[x];
	__syncthreads();
	const int win = A.block_width + 3 * (A.kmer - 1);       /* codon ends of one anchor's seed scan */
	const int stride = (win + 2 + 15) / 16 * 16;               /* bytes of one staging array */
	uint8_t *sb = gl_smem + (size_t)wib * 2 * stride;          /* bases of the window */
	uint8_t *saa = sb + stride;                                /* residue of each codon end */
	unsigned long long walked_sum = 0;
	for (int ci = blockIdx.x * GL_WARPS + wib; ci < A.n_cand; ci += gridDim.x * GL_WARPS) {
		const ns_gpu_gapless_candidate_t C = A.cand[ci];
		const int na = C.anchor_count < GL_MAX_ANCHORS ? C.anchor_count : GL_MAX_ANCHORS;
		int n_seg = 0;
		for (int ai = 0; ai < na; ++ai) {
			const int64_t aidx = (int64_t)C.anchor_offset + ai;
			if (aidx < 0 || aidx >= A.n_anchors) break;
			const ns_gpu_gapless_anchor_t an = A.anchors[aidx];
			const int qe = an.query_end;
			if (!(qe >= A.kmer - 1 && qe < C.query_length)) continue;
			/* seed: stage bases [base-2, base+win) and translate every codon end once */
			const int64_t base = an.target_block - (int64_t)3 * (A.kmer - 1);
			for (int x = lane; x < win + 2; x += 32) sb[x] = (uint8_t)gl_base(A, C, base - 2 + x);
			__syncwarp();
			for (int x = lane; x < win; x += 32) {
				const int b0 = sb[x], b1 = sb[x + 1], b2 = sb[x + 2];
				saa[x] = b0 < 4 && b1 < 4 && b2 < 4 ? codon[b0 << 4 | b1 << 2 | b2] : 20;
			}
			__syncwarp();
			long long key = LLONG_MIN;
			for (int d = lane; d < A.block_width; d += 32) {
				const int64_t te = an.target_block + d;
				if (te - (int64_t)(A.kmer - 1) * 3 - 2 < 0 || te >= C.target_length) continue;
				int s = 0;
				for (int k = 0; k < A.kmer; ++k) {
					const int q = gl_query(A, C, qe - A.kmer + 1 + k);
					s += sm[saa[d + 3 * k] * A.asize + (q < A.asize ? q : A.asize - 1)];
				}
				const long long kk = (long long)s * 4294967296ll + (long long)(0xFFFFFFFFu - (unsigned)d);
				key = max(key, kk);
			}
#pragma unroll
			for (int o = 16; o >= 1; o >>= 1) key = max(key, __shfl_xor_sync(FULL, key, o));
			__syncwarp();
			if (key == LLONG_MIN) continue;  /* no valid target end in the block */
			const int seed = (int)(key >> 32);
			const int64_t te = an.target_block + (int64_t)(0xFFFFFFFFu - (unsigned)(key & 0xFFFFFFFFll));
			int ll, rl, wl, wr;
			const int lb = gl_extend(A, C, codon, sm, lane, -1, qe, te, ll, wl);
			const int rb = gl_extend(A, C, codon, sm, lane, +1, qe, te, rl, wr);
			walked_sum += (unsigned long long)(wl + wr);
			if (lane == 0) {
				seg[wib][0][n_seg] = seed + lb + rb;
				seg[wib][1][n_seg] = qe - (A.kmer - 1) - ll;
				seg[wib][2][n_seg] = qe + rl;
			}
			++n_seg;
		}
		__syncwarp();
		if (lane == 0) { /* nasw-cuda.cu:1259-1293: stable sort by score, greedy overlap-scaled sum */
			int ss[GL_MAX_ANCHORS], qs[GL_MAX_ANCHORS], qq[GL_MAX_ANCHORS], n = 0, total = 0;
			for (int i = 0; i < n_seg; ++i) {
				const int sc = seg[wib][0][i];
				int j;
				for (j = n; j > 0 && ss[j - 1] < sc; --j) ss[j] = ss[j - 1], qs[j] = qs[j - 1], qq[j] = qq[j - 1];
				ss[j] = sc, qs[j] = seg[wib][1][i], qq[j] = seg[wib][2][i], ++n;
			}
			for (int i = 0; i < n; ++i) {
				const int len = qq[i] - qs[i] + 1;
				int overlap = 0;
				if (i > 0 && ss[i] < A.xdrop) break;
				for (int j = 0; j < i; ++j) {
					const int s = max(qs[i], qs[j]), e = min(qq[i], qq[j]);
					if (ss[j] != INT_MIN && e >= s) overlap += e - s + 1;
				}
				if (overlap >= len) { ss[i] = INT_MIN; continue; }
				if (overlap > 0) total += (int)((long long)ss[i] * (len - overlap) / len);
				else total += ss[i];
			}
			A.scores[ci] = n_seg ? total : INT_MIN;
		}
		__syncwarp();
	}
	if (lane == 0 && walked_sum) atomicAdd(A.steps, walked_sum);
}

extern "C" int plk_gapless_smem_bytes(int32_t block_width, int32_t kmer)
{
	const int win = block_width + 3 * (kmer - 1);
	return GL_WARPS * 2 * ((win + 2 + 15) / 16 * 16);
}

extern "C" int plk_gapless(const uint8_t *packed, int64_t bases, const uint8_t *queries, int64_t query_aa,
		const void *cand, int32_t n_cand, const void *anchors, int64_t n_anchors, int32_t block_width, int32_t kmer,
		int32_t xdrop, const int8_t *mat_dev, int32_t asize, const uint8_t *codon_dev, int32_t *scores,
		unsigned long long *steps, int32_t n_sm, void *stream)
{
	if (n_cand <= 0) return 0;
	GlArgs A;
	A.packed = packed, A.bases = bases, A.queries = queries, A.query_aa = query_aa;
	A.cand = (const ns_gpu_gapless_candidate_t*)cand, A.n_cand = n_cand;
	A.anchors = (const ns_gpu_gapless_anchor_t*)anchors, A.n_anchors = n_anchors;
	A.block_width = block_width, A.kmer = kmer, A.xdrop = xdrop, A.asize = asize, A.scores = scores, A.steps = steps;
	const int smem = plk_gapless_smem_bytes(block_width, kmer);
	cudaError_t e = cudaFuncSetAttribute(k_gapless, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
	if (e != cudaSuccess) return (int)e;
	int per_sm = 0;
	e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gapless, 32 * GL_WARPS, smem);
	if (e != cudaSuccess) return (int)e;
	int64_t grid = (int64_t)(per_sm > 0 ? per_sm : 1) * n_sm;
	const int64_t need = (n_cand + GL_WARPS - 1) / GL_WARPS;
	if (grid > need) grid = need;
	k_gapless<<<(unsigned)grid, 32 * GL_WARPS, smem, (cudaStream_t)stream>>>(A, mat_dev, codon_dev);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}
