/*
 * ref_prescreen.c -- test infrastructure: the reference's own ps_gapped
 * (prescreen.c:346-382, static there) behind a plain-array wrapper, so that the
 * device version (pscreen.cu) is checked against the reference itself.
 */
#include "prescreen.c"

int32_t ref_ps_gapped(const int8_t *pssm, int32_t L, const uint8_t *orf, int32_t n, int32_t diag, int32_t band,
		int32_t go, int32_t ge)
{
	ps_scratch_t s;
	int32_t sc;
	memset(&s, 0, sizeof(s));
	sc = ps_gapped(&s, pssm, L, orf, n, diag, band, go, ge);
	ps_scratch_free(&s);
	return sc;
}
