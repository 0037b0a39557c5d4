/*
 * seed_hmm.cuh -- the profile-derived seeds of an HMM-profile query (mp_sketch_hmm,
 * sketch.c:40-118), as functions of one match state and of one window, shared by the
 * device kernel (seed.cu, k_seed_hmm_alts / k_seed_hmm_enum) and a host build of the same
 * code that tests compare with the reference (plain C99 when not compiled by nvcc).
 *
 * A match state's emissions are 20 int16 in HMMER column order ACDEFGHIKLMNPQRSTVWY
 * (mp_hmm_emissions).  Each of the 13-letter groups (nasw-tab.c:12) takes the best
 * emission of its residues; the state offers the groups whose loss (best group's emission
 * minus the group's) is at most pos_loss, four at most (MP_HMM_MAX_ALT), placed in group
 * order into a list kept in ascending loss order by insertion (a new group goes after
 * every kept entry not above it; when the list is full it enters only below the last
 * entry, which then drops out).  A group none of the 20 residues maps to (9), or whose
 * best emission is INT16_MIN, offers nothing.  The list keeps its losses in 16 bits, as
 * the reference does (a loss over 32767, reachable only with pos_loss over 32767, wraps,
 * and the later comparisons and the window sums see the wrapped value).
 *
 * A window of kmer states ending at state `end` yields the k-mers of the states' offered
 * groups in lexicographic order of their ranks, walked depth first: a state's next rank is
 * tried while the losses so far plus its loss stay within win_loss, the first that does not
 * ends that state's choices; the first max_per_win whole k-mers count, and each whose masked
 * hash (sketch.c:7-16) has mod_bit zero low bits gives the seed
 * (hash >> mod_bit) << 32 | end.
 */
#ifndef PL_SEED_HMM_CUH
#define PL_SEED_HMM_CUH

#include <stdint.h>

#ifdef __CUDACC__
#define SH_FN __host__ __device__ __forceinline__
#else
#define SH_FN static inline
#endif

#define SH_ALT 4       /* MP_HMM_MAX_ALT */
#define SH_MAX_KMER 7  /* the index's largest k-mer (4 bits per residue in 32) */

/* a state's offered groups: n in bits 0-3, group r in bits 4 + 4r .. 7 + 4r; loss[r] the
 * loss as a 16-bit value (sign-extended) */
typedef struct { uint32_t code_n; int32_t loss[SH_ALT]; } sh_alts_t;

/* the 13-letter group of HMMER column j (A C D E F G H I K L M N P Q R S T V W Y) */
SH_FN int32_t sh_col_group(int32_t j)
{
	/* 4 bits per column, columns 0-7 in the first word's nibbles from the bottom, 8-15 in
	 * the second, 16-19 in the third: groups 0 6 4 5 12 8 3 10 | 2 11 11 4 7 5 2 1 | 1 10 13 12 */
	const uint32_t lo = 0xA38C5460u, mid = 0x12574BB2u, hi = 0x0000CDA1u;
	const uint32_t w = j < 8 ? lo : j < 16 ? mid : hi;
	return (int32_t)((w >> ((j & 7) * 4)) & 15u);
}

SH_FN uint32_t sh_hash(uint32_t key, uint32_t mask)
{ /* sketch.c:7-16 */
	key = (key + ~(key << 15)) & mask;
	key ^= key >> 10;
	key = (key + (key << 3)) & mask;
	key ^= key >> 6;
	key = (key + ~(key << 11)) & mask;
	key ^= key >> 16;
	return key;
}

/* one match state's offered groups */
SH_FN sh_alts_t sh_state_alts(const int16_t *e20, int32_t pos_loss)
{
	int32_t gs[14], best = INT16_MIN, code[SH_ALT], g, j, n = 0;
	sh_alts_t a;
	for (g = 0; g < 14; ++g) gs[g] = INT16_MIN;
	for (j = 0; j < 20; ++j) {
		const int32_t c = sh_col_group(j), v = e20[j];
		gs[c] = v > gs[c] ? v : gs[c];
	}
	for (g = 0; g < 14; ++g) best = gs[g] > best ? gs[g] : best;
	for (j = 0; j < SH_ALT; ++j) a.loss[j] = 0, code[j] = 0;
	for (g = 0; g < 14; ++g) {
		const int32_t l = best - gs[g];
		int32_t keep, p;
		if (gs[g] == INT16_MIN || l > pos_loss) continue;
		if (n == SH_ALT && l >= a.loss[SH_ALT - 1]) continue;  /* full, and not below the last */
		keep = n < SH_ALT ? n : SH_ALT - 1;                   /* the entries that stay */
		for (p = keep; p > 0 && a.loss[p - 1] > l; --p) {}    /* after the last one not above l */
		for (j = keep; j > p; --j) a.loss[j] = a.loss[j - 1], code[j] = code[j - 1];
		a.loss[p] = (int16_t)l, code[p] = g;
		n = keep + 1;
	}
	a.code_n = (uint32_t)n;
	for (j = 0; j < n; ++j) a.code_n |= (uint32_t)code[j] << (4 + 4 * j);
	return a;
}

/* the seeds of the window of states al[0 .. kmer-1] ending at state `end`, into out
 * (room for max_per_win; NULL: only counted); returns their number */
SH_FN int32_t sh_window_seeds(const sh_alts_t *al, int32_t kmer, int32_t mod_bit, int32_t win_loss,
		int32_t max_per_win, int32_t end, uint64_t *out)
{
	const uint32_t mask_k = (1U << kmer * 4) - 1, mask_mod = (1U << mod_bit) - 1;
	/* acc: the states' summed 16-bit losses, within 7 x 32768 of 0, so no sum overflows */
	int32_t rank[SH_MAX_KMER], acc[SH_MAX_KMER + 1], d = 0, n_kmer = 0, n_out = 0;
	uint32_t pre[SH_MAX_KMER + 1];
	if (kmer < 1 || kmer > SH_MAX_KMER || max_per_win <= 0) return 0;
	rank[0] = 0, acc[0] = 0, pre[0] = 0;
	/* depth-first over the ranks: at depth d, state d's choice rank[d] with the losses of
	 * the states before it in acc[d]; a whole k-mer at depth kmer - 1 */
	while (d >= 0) {
		const uint32_t cn = al[d].code_n;
		const int32_t r = rank[d];
		if (r >= (int32_t)(cn & 15u) || acc[d] + al[d].loss[r] > win_loss) {  /* state d has no more choices */
			if (--d >= 0) ++rank[d];
			continue;
		}
		{
			const uint32_t x = (pre[d] << 4 | ((cn >> (4 + 4 * r)) & 15u)) & mask_k;
			if (d + 1 == kmer) {
				const uint32_t y = sh_hash(x, mask_k);
				if ((y & mask_mod) == 0) {
					if (out) out[n_out] = (uint64_t)(y >> mod_bit) << 32 | (uint32_t)end;
					++n_out;
				}
				if (++n_kmer >= max_per_win) break;
				++rank[d];
			} else {
				pre[d + 1] = x, acc[d + 1] = acc[d] + al[d].loss[r];
				rank[++d] = 0;
			}
		}
	}
	return n_out;
}

#endif
