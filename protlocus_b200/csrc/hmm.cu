/*
 * hmm.cu -- sm_100a kernels of the integer profile DP, mp_hmm_dp_score
 * (hmm.c:252-291): one profile, many regions, one frame-0 codon per row.
 *
 * Every cell of row i depends only on row i-1 (columns j-1 and j), so a row is
 * computed in parallel across the profile: one warp per region, lane t owns
 * HMM_C consecutive columns of a 32*HMM_C-column tile and keeps their M/I/D
 * values of the previous row in registers, updated in place from the last
 * column down.  The value of column j-1 at a lane's first column comes from lane
 * t-1 by __shfl_up_sync, and across tiles from a per-row edge buffer that lane
 * 31 of the previous tile wrote (two buffers by tile parity, so a tile never
 * writes the rows it reads).  The 7 transition scores of a lane's columns
 * are row-invariant and sit in registers for the whole tile; the emissions are
 * staged in shared memory transposed ([residue][column], a zero row for stop
 * and ambiguous codons) so that one 16-byte load gives a lane its 8 columns.
 * Padding columns beyond m carry transitions of -2^28: every state there stays
 * 0 and cannot change the maximum.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include "plk.h"

#define FULL 0xffffffffu
#define HMM_C 8                    /* columns per lane */
#define HMM_TILE (32 * HMM_C)      /* columns per tile */
#define HMM_WARPS 8

extern "C" void plk_add_launches(uint64_t n);

/* codon index per row of every region: HMMER column, 20 = no emission (stop or a code > 3) */
__global__ void k_hmm_codons(const uint8_t *__restrict__ nt, const int32_t *__restrict__ off,
		const int32_t *__restrict__ len, const int64_t *__restrict__ row_off, int n,
		const uint8_t *__restrict__ codon_alpha, uint8_t *__restrict__ rows)
{
	for (int q = blockIdx.x; q < n; q += gridDim.x) {
		const int tlen = len[q] / 3;
		const uint8_t *s = nt + off[q];
		uint8_t *o = rows + row_off[q];
		for (int i = threadIdx.x; i < tlen; i += blockDim.x) {
			const int b0 = s[3 * i], b1 = s[3 * i + 1], b2 = s[3 * i + 2];
			o[i] = b0 > 3 || b1 > 3 || b2 > 3 ? 20 : codon_alpha[b0 << 4 | b1 << 2 | b2];
		}
	}
}

template <bool SMEM_EMIT>
__global__ void __launch_bounds__(32 * HMM_WARPS)
k_hmm_dp(const plk_hmm_prof_t P, const uint8_t *__restrict__ rows, const int64_t *__restrict__ row_off,
		const int32_t *__restrict__ len, const int32_t *__restrict__ order, int n, int32_t *counter,
		int4 *__restrict__ edge, int64_t edge_stride, int32_t *__restrict__ score)
{
	extern __shared__ __align__(16) int16_t s_emit[];  /* [21][mpad] when SMEM_EMIT */
	const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
	const int ntile = P.mpad / HMM_TILE;
	if (SMEM_EMIT) {
		const int4 *src = (const int4*)P.emit_t;
		int4 *dst = (int4*)s_emit;
		for (int x = threadIdx.x; x < 21 * P.mpad / 8; x += blockDim.x) dst[x] = src[x];
		__syncthreads();
	}
	const int16_t *emit = SMEM_EMIT ? s_emit : P.emit_t;
	int4 *my_edge = edge + (int64_t)(blockIdx.x * HMM_WARPS + wib) * 2 * edge_stride;
	for (;;) {
		int idx = 0;
		if (lane == 0) idx = atomicAdd(counter, 1);
		idx = __shfl_sync(FULL, idx, 0);
		if (idx >= n) break;
		const int q = order[idx];
		const int tlen = len[q] / 3;
		const uint8_t *aa = rows + row_off[q];
		int best = 0;
		for (int t = 0; t < ntile; ++t) {
			const int c0 = t * HMM_TILE + lane * HMM_C;     /* column j-1 of the lane's first cell */
			int tr[7][HMM_C];
#pragma unroll
			for (int k = 0; k < 7; ++k) {
				const int4 *p = (const int4*)(P.trans_t + (int64_t)k * P.mpad + c0);
				const int4 a = __ldg(p), b = __ldg(p + 1);
				tr[k][0] = a.x, tr[k][1] = a.y, tr[k][2] = a.z, tr[k][3] = a.w;
				tr[k][4] = b.x, tr[k][5] = b.y, tr[k][6] = b.z, tr[k][7] = b.w;
			}
			int pm[HMM_C], pi[HMM_C], pd[HMM_C];
#pragma unroll
			for (int c = 0; c < HMM_C; ++c) pm[c] = pi[c] = pd[c] = 0;
			int4 nxt = make_int4(0, 0, 0, 0);                 /* edge of row i-1 for lane 0 */
			const int4 *rd = my_edge + (int64_t)((t + 1) & 1) * edge_stride;  /* written by tile t-1 */
			int4 *wr = my_edge + (int64_t)(t & 1) * edge_stride;              /* read by tile t+1 */
			for (int i = 0; i < tlen; ++i) {
				const int a = aa[i];
				const int4 ev = *(const int4*)(emit + (int64_t)a * P.mpad + c0);
				int e[HMM_C];
				e[0] = (int)(int16_t)(ev.x & 0xffff), e[1] = ev.x >> 16;
				e[2] = (int)(int16_t)(ev.y & 0xffff), e[3] = ev.y >> 16;
				e[4] = (int)(int16_t)(ev.z & 0xffff), e[5] = ev.z >> 16;
				e[6] = (int)(int16_t)(ev.w & 0xffff), e[7] = ev.w >> 16;
				/* previous-row values of column j-1 for the lane's first cell */
				int nm = __shfl_up_sync(FULL, pm[HMM_C - 1], 1);
				int ni = __shfl_up_sync(FULL, pi[HMM_C - 1], 1);
				int nd = __shfl_up_sync(FULL, pd[HMM_C - 1], 1);
				if (lane == 0) nm = nxt.x, ni = nxt.y, nd = nxt.z;
				if (lane == 0 && t > 0) nxt = rd[i];  /* row i of the previous tile, used by row i+1 */
#pragma unroll
				for (int c = HMM_C - 1; c >= 0; --c) {
					const int am = c ? pm[c - 1] : nm, ai = c ? pi[c - 1] : ni, ad = c ? pd[c - 1] : nd;
					int from = max(am + tr[0][c], ai + tr[3][c]);
					from = max(from, ad + tr[5][c]);
					const int cm = max(from + e[c], 0);
					const int ci = max(max(pm[c] + tr[1][c], pi[c] + tr[4][c]), 0);
					const int cd = max(max(am + tr[2][c], ad + tr[6][c]), 0);
					best = max(best, max(cm, ci));
					pm[c] = cm, pi[c] = ci, pd[c] = cd;
				}
				if (lane == 31 && t + 1 < ntile) wr[i] = make_int4(pm[HMM_C - 1], pi[HMM_C - 1], pd[HMM_C - 1], 0);
			}
			__syncwarp();  /* the next tile reads this tile's edge */
		}
#pragma unroll
		for (int o = 16; o >= 1; o >>= 1) best = max(best, __shfl_xor_sync(FULL, best, o));
		if (lane == 0) score[q] = best;
	}
}

extern "C" int plk_hmm_smem_bytes(int32_t mpad) { return 21 * mpad * 2; }

extern "C" int plk_hmm_ctas_per_sm(int32_t mpad)
{
	int n = 0;
	const int smem = plk_hmm_smem_bytes(mpad);
	cudaError_t e;
	if (smem <= PLK_HMM_SMEM_MAX) {
		e = cudaFuncSetAttribute(k_hmm_dp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, PLK_HMM_SMEM_MAX);
		if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_hmm_dp<true>, 32 * HMM_WARPS, smem);
	} else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_hmm_dp<false>, 32 * HMM_WARPS, 0);
	return e == cudaSuccess ? n : -1;
}

extern "C" int plk_hmm_warps_per_cta(void) { return HMM_WARPS; }

extern "C" int plk_hmm_codons(const uint8_t *nt, const int32_t *off, const int32_t *len, const int64_t *row_off,
		int32_t n, const uint8_t *codon_alpha, uint8_t *rows, void *stream)
{
	if (n <= 0) return 0;
	k_hmm_codons<<<n < 4096 ? n : 4096, 128, 0, (cudaStream_t)stream>>>(nt, off, len, row_off, n, codon_alpha, rows);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_hmm_dp(const plk_hmm_prof_t *p, const uint8_t *rows, const int64_t *row_off, const int32_t *len,
		const int32_t *order, int32_t n, int32_t *counter, void *edge, int64_t edge_stride_rows, int32_t n_ctas,
		int32_t *score, void *stream)
{
	if (n <= 0) return 0;
	cudaStream_t st = (cudaStream_t)stream;
	cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int32_t), st);
	if (e != cudaSuccess) return (int)e;
	const int smem = plk_hmm_smem_bytes(p->mpad);
	if (smem <= PLK_HMM_SMEM_MAX) {
		e = cudaFuncSetAttribute(k_hmm_dp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, PLK_HMM_SMEM_MAX);
		if (e != cudaSuccess) return (int)e;
	}
	if (smem <= PLK_HMM_SMEM_MAX)
		k_hmm_dp<true><<<n_ctas, 32 * HMM_WARPS, smem, st>>>(*p, rows, row_off, len, order, n, counter, (int4*)edge,
				edge_stride_rows, score);
	else
		k_hmm_dp<false><<<n_ctas, 32 * HMM_WARPS, 0, st>>>(*p, rows, row_off, len, order, n, counter, (int4*)edge,
				edge_stride_rows, score);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}
