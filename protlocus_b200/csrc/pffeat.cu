/*
 * pffeat.cu -- per-candidate features of the learned prefilter, one CTA per
 * candidate (a protein and the genomic window a chained candidate spans, on the
 * strand the DP would read).
 *
 *  1. the protein's aa 5-mers go into a shared-memory hash table (4096 slots, first
 *     occurrence kept) and its aa 3-mers into 256 composition bins;
 *  2. the window is translated in chunks of 4096 codon ends (all three frames: every
 *     position is the end of a codon) into shared memory; each codon end adds its
 *     window 3-mer to 256 more bins and looks its 5-mer up in the table: a hit is an
 *     anchor (window position, protein position);
 *  3. the anchors are sorted by position (bitonic, shared memory) and one warp chains
 *     them: the longest chain increasing in both coordinates whose nucleotide gap is
 *     not shorter than 3x the residue gap minus 60 (frameshift slack);
 *  4. features: the 512 composition bins (scaled so a uniform composition is 1) and 20
 *     scalars of the anchors and the best chain (counts, coverage, span, frame
 *     changes, the window positions where the protein would start and end); the chain
 *     ends are also returned as integers for window tightening.
 *
 * Feature row layout (bf16, F_DIM = 576 columns): [0,256) protein 3-mer bins,
 * [256,512) window 3-mer bins, [512,532) scalars, [532,576) zero.
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "plk.h"

extern "C" void plk_add_launches(uint64_t n);

namespace {

constexpr int THREADS = 256;
constexpr int HSLOTS = 4096;
constexpr int CH = 4096;
constexpr int MAXA = 1024;
constexpr int F_DIM = PLK_PF_FDIM;
constexpr uint8_t BAD = 255;

struct FeatSmem {
	int32_t hkey[HSLOTS];
	int32_t hpos[HSLOTS];
	int32_t bins[512];
	int64_t akey[MAXA];
	int32_t f[MAXA], prev[MAXA];
	uint8_t aab[CH + 16];
	int32_t n_anchor, tot_p, tot_w;
	int32_t chain[8];
};

__device__ __forceinline__ uint32_t h5(uint32_t code) { return (code * 2654435761u) >> 20; }          /* 12 bits */
__device__ __forceinline__ uint32_t h3(uint32_t code) { return ((code * 40503u) >> 8) & 255u; }

__device__ __forceinline__ uint8_t codon_aa(const uint8_t *nt, int64_t p, const plk_pf_tabs_t &T)
{
	const uint8_t a = T.nt4[nt[p - 2]], b = T.nt4[nt[p - 1]], c = T.nt4[nt[p]];
	if ((a | b | c) > 3) return BAD;
	const uint8_t x = T.codon[a * 16 + b * 4 + c];
	return x < 20 ? x : BAD;
}

__global__ void __launch_bounds__(THREADS) k_pf_features(plk_pf_feat_args_t A)
{
	extern __shared__ __align__(16) uint8_t smem_raw[];
	FeatSmem &S = *reinterpret_cast<FeatSmem *>(smem_raw);
	const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
	const int64_t q = blockIdx.x;
	if (q >= A.n) return;
	const plk_pf_cand_t C = A.cand[q];
	const int32_t nl = C.nl, al = C.al;
	const uint8_t *nt = A.nt + C.nt_off;
	const uint8_t *aa = A.aa + C.aa_off;
	const plk_pf_tabs_t &T = A.tabs;

	for (int i = tid; i < HSLOTS; i += THREADS) S.hkey[i] = 0, S.hpos[i] = 0x7fffffff;
	for (int i = tid; i < 512; i += THREADS) S.bins[i] = 0;
	if (tid == 0) S.n_anchor = 0, S.tot_p = 0, S.tot_w = 0;
	__syncthreads();

	/* 1. protein k-mers */
	int cnt3 = 0;
	for (int p = tid; p < al; p += THREADS) {
		uint8_t r[5];
		bool ok = true;
		const int w = p >= 4 ? 5 : p + 1;
		for (int k = 0; k < w; ++k) {
			const uint8_t x = T.aa20[aa[p - k]];
			r[k] = x < 20 ? x : BAD;
			if (r[k] == BAD) ok = false;
		}
		if (p >= 2 && r[0] != BAD && r[1] != BAD && r[2] != BAD) {
			atomicAdd(&S.bins[h3((uint32_t)r[2] * 400u + r[1] * 20u + r[0])], 1);
			++cnt3;
		}
		if (p >= 4 && ok) {
			const uint32_t code = (((r[4] * 20u + r[3]) * 20u + r[2]) * 20u + r[1]) * 20u + r[0];
			uint32_t s = h5(code);
			for (int t = 0; t < HSLOTS; ++t, s = (s + 1) & (HSLOTS - 1)) {
				const int32_t old = atomicCAS(&S.hkey[s], 0, (int32_t)code + 1);
				if (old == 0 || old == (int32_t)code + 1) { atomicMin(&S.hpos[s], p); break; }
			}
		}
	}
	atomicAdd(&S.tot_p, cnt3);
	__syncthreads();

	/* 2. window scan */
	int cntw = 0;
	for (int64_t cs = 0; cs < nl; cs += CH) {
		/* aab[j] = residue of the codon ending at cs - 12 + j */
		for (int j = tid; j < CH + 12; j += THREADS) {
			const int64_t p = cs - 12 + j;
			S.aab[j] = (p >= 2 && p < nl) ? codon_aa(nt, p, T) : BAD;
		}
		__syncthreads();
		for (int j = 12 + tid; j < CH + 12; j += THREADS) {
			const int64_t p = cs - 12 + j;
			if (p >= nl) break;
			const uint8_t a0 = S.aab[j], a1 = S.aab[j - 3], a2 = S.aab[j - 6];
			if (a0 == BAD || a1 == BAD || a2 == BAD) continue;
			atomicAdd(&S.bins[256 + h3((uint32_t)a2 * 400u + a1 * 20u + a0)], 1);
			++cntw;
			const uint8_t a3 = S.aab[j - 9], a4 = S.aab[j - 12];
			if (a3 == BAD || a4 == BAD) continue;
			const uint32_t code = (((a4 * 20u + a3) * 20u + a2) * 20u + a1) * 20u + a0;
			uint32_t s = h5(code);
			for (int t = 0; t < HSLOTS; ++t, s = (s + 1) & (HSLOTS - 1)) {
				const int32_t key = S.hkey[s];
				if (key == 0) break;
				if (key == (int32_t)code + 1) {
					const int idx = atomicAdd(&S.n_anchor, 1);
					if (idx < MAXA) S.akey[idx] = (p << 20) | (int64_t)S.hpos[s];  /* both coordinates are k-mer ends */
					break;
				}
			}
		}
		__syncthreads();
	}
	atomicAdd(&S.tot_w, cntw);
	__syncthreads();

	/* 3. sort the kept anchors by (position, protein position) and chain them */
	const int na_all = S.n_anchor, na = na_all < MAXA ? na_all : MAXA;
	int np2 = 1;
	while (np2 < na) np2 <<= 1;
	for (int i = na + tid; i < np2; i += THREADS) S.akey[i] = INT64_MAX;
	__syncthreads();
	for (int k = 2; k <= np2; k <<= 1)
		for (int j = k >> 1; j > 0; j >>= 1) {
			for (int i = tid; i < np2; i += THREADS) {
				const int l = i ^ j;
				if (l > i) {
					const int64_t a = S.akey[i], b = S.akey[l];
					const bool up = (i & k) == 0;
					if ((a > b) == up) S.akey[i] = b, S.akey[l] = a;
				}
			}
			__syncthreads();
		}
	if (warp == 0) {
		for (int j = 0; j < na; ++j) {
			const int64_t kj = S.akey[j];
			const int64_t pj = kj >> 20;
			const int32_t rj = (int32_t)(kj & 0xFFFFF);
			int32_t best = 0;  /* f * 2048 + k + 1 of the best predecessor */
			for (int k = lane; k < j; k += 32) {
				const int64_t kk = S.akey[k];
				const int64_t pk = kk >> 20;
				const int32_t rk = (int32_t)(kk & 0xFFFFF);
				if (pk < pj && rk < rj && (pj - pk) >= 3LL * (rj - rk) - 60) {
					const int32_t v = S.f[k] * 2048 + k + 1;
					best = v > best ? v : best;
				}
			}
#pragma unroll
			for (int o = 16; o >= 1; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
			if (lane == 0) {
				S.f[j] = best ? (best >> 11) + 1 : 1;
				S.prev[j] = best ? (best & 2047) - 1 : -1;
			}
			__syncwarp();
		}
		if (lane == 0) {
			int jb = -1, fb = 0;
			for (int j = 0; j < na; ++j) if (S.f[j] > fb) fb = S.f[j], jb = j;
			int32_t len = 0, fc = 0, cov = 0, first_p = -1, last_p = -1, first_r = -1, last_r = -1, nxt_r = -1, nxt_p = -1;
			for (int j = jb; j >= 0; j = S.prev[j]) {
				const int32_t pj = (int32_t)(S.akey[j] >> 20), rj = (int32_t)(S.akey[j] & 0xFFFFF);
				if (len == 0) last_p = pj, last_r = rj;
				else {
					if ((nxt_p % 3) != (pj % 3)) ++fc;
					cov += min(5, nxt_r - rj);
				}
				first_p = pj, first_r = rj, nxt_p = pj, nxt_r = rj;
				++len;
			}
			if (len > 0) cov += 5;
			S.chain[0] = len, S.chain[1] = fc, S.chain[2] = cov;
			S.chain[3] = first_p, S.chain[4] = last_p, S.chain[5] = first_r, S.chain[6] = last_r;
		}
	}
	__syncthreads();

	/* 4. features */
	__nv_bfloat16 *F = reinterpret_cast<__nv_bfloat16 *>(A.feats) + q * F_DIM;
	const float sp = 256.0f / (float)max(1, S.tot_p), sw = 256.0f / (float)max(1, S.tot_w);
	for (int i = tid; i < 512; i += THREADS) F[i] = __float2bfloat16_rn((float)S.bins[i] * (i < 256 ? sp : sw));
	for (int i = 532 + tid; i < F_DIM; i += THREADS) F[i] = __float2bfloat16_rn(0.0f);
	if (tid == 0) {
		const int32_t len = S.chain[0], fc = S.chain[1], cov = S.chain[2];
		const int32_t fp = S.chain[3], lp = S.chain[4], fr = S.chain[5], lr = S.chain[6];
		const float fnl = (float)max(nl, 1), fal = (float)max(al, 1);
		float v[20];
		v[0] = log2f(1.0f + al) / 12.0f;
		v[1] = log2f(1.0f + nl) / 16.0f;
		v[2] = log2f(1.0f + na_all) / 10.0f;
		v[3] = (float)len / (float)max(1, al - 4);
		v[4] = log2f(1.0f + len) / 10.0f;
		v[5] = (float)cov / fal;
		v[6] = len > 0 ? (float)(lp - fp) / fnl : 0.0f;
		v[7] = len > 0 ? (float)fp / fnl : 0.0f;
		v[8] = len > 0 ? (float)lp / fnl : 0.0f;
		v[9] = len > 0 ? (float)fr / fal : 0.0f;
		v[10] = len > 0 ? (float)lr / fal : 0.0f;
		v[11] = (float)fc / 8.0f;
		v[12] = len > 0 ? log2f(1.0f + (lp - fp)) / 16.0f : 0.0f;
		v[13] = len > 0 ? fminf(fmaxf((float)(fp - 3 * fr - 2) / fnl, -1.0f), 2.0f) : 0.0f;
		v[14] = len > 0 ? fminf(fmaxf((float)(lp + 3 * (al - 1 - lr)) / fnl, -1.0f), 2.0f) : 0.0f;
		v[15] = (float)min(na_all, 65535) * 1000.0f / fnl / 8.0f;
		v[16] = (float)len / (float)max(1, na);
		v[17] = 1.0f;
		v[18] = len >= 2 ? 1.0f : 0.0f;
		v[19] = na_all > MAXA ? 1.0f : 0.0f;
#pragma unroll
		for (int i = 0; i < 20; ++i) F[512 + i] = __float2bfloat16_rn(v[i]);
		int32_t *ci = A.chain + 4 * q;
		ci[0] = len > 0 ? fp : -1, ci[1] = len > 0 ? lp : -1, ci[2] = len > 0 ? fr : -1, ci[3] = len > 0 ? lr : -1;
	}
}

}  // namespace

extern "C" int plk_pf_features(const plk_pf_feat_args_t *a, void *stream)
{
	if (a->n <= 0) return 0;
	const int smem = (int)sizeof(FeatSmem);
	cudaError_t e = cudaFuncSetAttribute(k_pf_features, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
	if (e != cudaSuccess) return (int)e;
	k_pf_features<<<(unsigned)a->n, THREADS, smem, (cudaStream_t)stream>>>(*a);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}
