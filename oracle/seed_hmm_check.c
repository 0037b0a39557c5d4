/*
 * seed_hmm_check.c -- test infrastructure: a host build of the device's profile-derived
 * seeding functions (protlocus_b200/csrc/seed_hmm.cuh: sh_state_alts, sh_window_seeds),
 * run window by window as the device kernel runs them, so that tests compare the very
 * code the device executes with the reference's mp_sketch_hmm (sketch.c:40-118) and with
 * oracle/seed_port.c on the CPU.
 *
 *   shc_sketch_hmm: the seeds of an emission table (len x 20 int16) in the reference's
 *                   order, into out (room for (len - kmer + 1) * max_per_win); returns
 *                   their number, -1 on a host allocation failure.
 */
#include <stdlib.h>
#include "../protlocus_b200/csrc/seed_hmm.cuh"

#define SHC_EXPORT __attribute__((visibility("default")))

SHC_EXPORT int64_t shc_sketch_hmm(const int16_t *emit, int32_t len, int32_t kmer, int32_t mod_bit, int32_t pos_loss,
		int32_t win_loss, int32_t max_per_win, uint64_t *out)
{
	sh_alts_t *al;
	int64_t n = 0;
	int32_t i;
	if (!emit || len < kmer || max_per_win <= 0) return 0;
	al = (sh_alts_t*)malloc(sizeof(sh_alts_t) * (size_t)len);
	if (!al) return -1;
	for (i = 0; i < len; ++i) al[i] = sh_state_alts(emit + (size_t)i * 20, pos_loss);
	for (i = kmer - 1; i < len; ++i)
		n += sh_window_seeds(al + (i - kmer + 1), kmer, mod_bit, win_loss, max_per_win, i, out + n);
	free(al);
	return n;
}
