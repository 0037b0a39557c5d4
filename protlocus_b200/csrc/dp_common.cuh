/*
 * dp_common.cuh -- device helpers shared by the spliced-DP kernels (splice.cu,
 * ext.cu): the saturating arithmetic modes, cp.async helpers and the
 * per-position input preparation of nasw-sse.c:95-214.
 */
#ifndef DP_COMMON_CUH
#define DP_COMMON_CUH
#include <cuda_runtime.h>
#include <stdint.h>
#include "plk.h"
#include "../../include/plgpu.h"

#define FULL 0xffffffffu

/* ------------------------------------------------------------------ arithmetic modes
 * MODE 0: int16 semantics where no value can reach +32767 (al*max(sc)+256 < 32767):
 *         _mm_subs/_mm_adds_epi16 reduce to a clamp at -32768.
 * MODE 1: int32 semantics of ns_global_gs32b (no saturation, neg_inf -2^30).
 * MODE 2: int16 semantics with both clamps (long proteins). */
template <int MODE> struct Ar;
template <> struct Ar<0> {
	static constexpr int NEG = -32768;
	static __device__ __forceinline__ int sub(int x, int k) { return max(x - k, NEG); }
	static __device__ __forceinline__ int add(int x, int k) { return max(x + k, NEG); }
};
template <> struct Ar<1> {
	static constexpr int NEG = -0x40000000;
	static __device__ __forceinline__ int sub(int x, int k) { return x - k; }
	static __device__ __forceinline__ int add(int x, int k) { return x + k; }
};
template <> struct Ar<2> {
	static constexpr int NEG = -32768;
	static __device__ __forceinline__ int sub(int x, int k) { return min(max(x - k, NEG), 32767); }
	static __device__ __forceinline__ int add(int x, int k) { return min(max(x + k, NEG), 32767); }
};


__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
	const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" :: "r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

/* ------------------------------------------------------------------ preparation
 * One position p in [0, nl] of a job: donor[p], acceptor[p] and (p < nl)
 * the translated codon nas[p].  s_nt4 / s_codon are the option tables staged
 * in shared memory.  Values are int8 with the reference's wrap-around. */

/* forward orientation: ns_prep_seq (nasw-sse.c:95-159) */
__device__ __forceinline__ void prep_fwd_pos(const int p, const uint8_t *__restrict__ ns, const int nl,
		const uint8_t *__restrict__ sst, const uint8_t *s_nt4, const uint8_t *s_codon, const plk_params_t &P,
		uint8_t *__restrict__ nas, int8_t *__restrict__ donor, int8_t *__restrict__ acceptor)
{
	const int max_spsc = (P.io + 1) / 2 - 1;
#define B4(q) ((q) >= 0 && (q) < nl ? s_nt4[ns[(q)]] : 4)
	int dv = P.sp[3], av = P.sp[3];
	if (p < nl - 3) { /* nasw-sse.c:124-131 */
		const int b0 = B4(p), b1 = B4(p + 1), b2 = B4(p + 2), b3 = B4(p + 3);
		int t = 3;
		if (b1 == 2 && b2 == 3) t = (b3 == 0 || b3 == 2) ? (b0 == 2 ? -1 : 4) : 0;
		else if (b1 == 2 && b2 == 1 && b0 == 2) t = 1;
		else if (b1 == 0 && b2 == 3) t = 2;
		dv = t < 0 ? 0 : P.sp[t];
	}
	int8_t d8 = (int8_t)dv, a8 = (int8_t)av;
	if (p >= 1 && p < nl) { /* nasw-sse.c:132-141 */
		const int bm1 = B4(p - 1), b0 = B4(p);
		int t = 3, pen = 0;
		if (bm1 == 0 && b0 == 2) {
			const int bm2 = B4(p - 2);
			t = (p >= 2 && (bm2 == 1 || bm2 == 3)) ? -1 : 0;
			for (int q = p - 4; q >= 0 && q > p - 7; --q) {
				const int bq = B4(q);
				if (bq != 1 && bq != 3) pen += P.sp[5];
			}
		} else if (bm1 == 0 && b0 == 1) t = 2;
		a8 = (int8_t)(t < 0 ? 0 : P.sp[t]);
		if (t == -1 || t == 0) a8 = (int8_t)(a8 + pen);
	}
	if (sst && p + 1 >= 1 && p + 1 < nl) { /* nasw-sse.c:142-156 */
		const uint8_t x = sst[p + 1];
		int spsc = (int8_t)(x >> 1) - (int8_t)NS_SPSC_OFFSET;
		if (spsc > max_spsc) spsc = max_spsc;
		if (x == 0xff) d8 = (int8_t)(d8 - P.sp_null_bonus), a8 = (int8_t)(a8 - P.sp_null_bonus);
		else if (x & 1) a8 = (int8_t)(a8 - spsc);
		else d8 = (int8_t)(d8 - spsc);
	}
	donor[p] = d8, acceptor[p] = a8;
	if (p < nl) { /* nasw-sse.c:95-108 */
		const int b2 = B4(p), b1 = B4(p - 1), b0 = B4(p - 2);
		nas[p] = (p >= 2 && b0 < 4 && b1 < 4 && b2 < 4) ? s_codon[(b0 << 4 | b1 << 2 | b2) & 0x3f] : P.aa_x;
	}
#undef B4
}

/* left-extension orientation: ns_prep_seq_left (nasw-sse.c:161-214).  The
 * nucleotides are read backwards (R(q) = base nl-1-q); the splice signals are
 * the mirrored rules on that reversed sequence; the splice-score track is
 * applied mirrored; nas[p] (p >= 2) is the forward codon ending at nl+1-p and
 * nas[0] = nas[1] = X. */
__device__ __forceinline__ void prep_left_pos(const int p, const uint8_t *__restrict__ ns, const int nl,
		const uint8_t *__restrict__ sst, const uint8_t *s_nt4, const uint8_t *s_codon, const plk_params_t &P,
		uint8_t *__restrict__ nas, int8_t *__restrict__ donor, int8_t *__restrict__ acceptor)
{
	const int max_spsc = (P.io + 1) / 2 - 1;
#define R4(q) ((q) >= 0 && (q) < nl ? s_nt4[ns[nl - 1 - (q)]] : 4)
#define F4(q) ((q) >= 0 && (q) < nl ? s_nt4[ns[(q)]] : 4)
	int8_t d8 = (int8_t)P.sp[3], a8 = (int8_t)P.sp[3];
	if (p < nl - 3) { /* nasw-sse.c:176-186 */
		int t = 3, pen = 0;
		if (R4(p + 1) == 2 && R4(p + 2) == 0) {
			const int r3 = R4(p + 3);
			t = (p + 3 < nl && (r3 == 1 || r3 == 3)) ? -1 : 0;
			for (int q = p + 5; q < nl && q < p + 8; ++q) {
				const int bq = R4(q);
				if (bq != 1 && bq != 3) pen += P.sp[5];
			}
		} else if (R4(p + 1) == 1 && R4(p + 2) == 0) t = 2;
		d8 = (int8_t)(t < 0 ? 0 : P.sp[t]);
		if (t == -1 || t == 0) d8 = (int8_t)(d8 + pen);
	}
	if (p >= 1 && p < nl) { /* nasw-sse.c:187-195 */
		const int rm1 = R4(p - 1), r0 = R4(p);
		int t = 3;
		if (rm1 == 3 && r0 == 2) {
			const int rm2 = R4(p - 2);
			t = (p >= 2 && (rm2 == 0 || rm2 == 2)) ? ((p + 1 < nl && R4(p + 1) == 2) ? -1 : 4) : 0;
		} else if (rm1 == 1 && r0 == 2 && p + 1 < nl && R4(p + 1) == 1) t = 1;
		else if (rm1 == 3 && r0 == 0) t = 2;
		a8 = (int8_t)(t < 0 ? 0 : P.sp[t]);
	}
	if (sst && p < nl) { /* nasw-sse.c:196-207, position p holds ss[nl-1-p] */
		const uint8_t x = sst[nl - 1 - p];
		int spsc = (int8_t)(x >> 1) - (int8_t)NS_SPSC_OFFSET;
		if (spsc > max_spsc) spsc = max_spsc;
		if (x == 0xff) d8 = (int8_t)(d8 - P.sp_null_bonus), a8 = (int8_t)(a8 - P.sp_null_bonus);
		else if (x & 1) d8 = (int8_t)(d8 - spsc);
		else a8 = (int8_t)(a8 - spsc);
	}
	donor[p] = d8, acceptor[p] = a8;
	if (p < nl) { /* nasw-sse.c:208-213: forward codons, reversed, shifted by two */
		uint8_t v = P.aa_x;
		if (p >= 2) {
			const int q = nl + 1 - p, b2 = F4(q), b1 = F4(q - 1), b0 = F4(q - 2);
			if (q >= 2 && b0 < 4 && b1 < 4 && b2 < 4) v = s_codon[(b0 << 4 | b1 << 2 | b2) & 0x3f];
		}
		nas[p] = v;
	}
#undef R4
#undef F4
}

#endif
