/*
 * hmm_port.c -- ORACLE (test infrastructure only): C restatement of the
 * reference's integer profile DP, mp_hmm_dp_score (hmm.c:252-291).
 *
 * Inputs are the tables the reference parser builds (hmm.c:112-195): emit
 * [m][20] int16 in HMMER column order, trans [m][7] int16 (m->m, m->i, m->d,
 * i->m, i->i, d->m, d->d), and codon_alpha[64]: the HMMER column of the amino
 * acid a codon encodes, or 20 for a stop codon (no emission), the reference's
 * ns_tab_codon remapped by mp_hmm_aa20_to_alpha (hmm.c:229-250).  nt holds
 * 0-4 nucleotide codes; a codon with a code > 3 emits nothing.
 *
 * Pinned against the reference build (oracle/_ref) and the golden fixture
 * tests/golden/hmm_golden.json.
 */
#include <stdint.h>
#include <stdlib.h>

#define PORT_EXPORT __attribute__((visibility("default")))

PORT_EXPORT int32_t port_hmm_dp_score(int32_t m, const int16_t *emit, const int16_t *trans, const uint8_t *codon_alpha,
		const uint8_t *nt, int32_t nlen)
{
	int32_t *buf, *pm, *pi, *pd, *cm, *ci, *cd, *x;
	int32_t i, j, tlen, best = 0;
	if (!nt || nlen < 3 || m <= 0) return 0;
	tlen = nlen / 3;
	buf = (int32_t*)calloc((size_t)(m + 1) * 6, sizeof(int32_t));
	if (!buf) return 0;
	pm = buf, pi = pm + m + 1, pd = pi + m + 1, cm = pd + m + 1, ci = cm + m + 1, cd = ci + m + 1;
	for (i = 0; i < tlen; ++i) { /* one row per frame-0 codon; column 0 stays 0 */
		const uint8_t *c = nt + 3 * i;
		const int aa = c[0] > 3 || c[1] > 3 || c[2] > 3 ? 20 : codon_alpha[c[0] << 4 | c[1] << 2 | c[2]];
		for (j = 1; j <= m; ++j) {
			const int16_t *t = trans + (size_t)(j - 1) * 7;
			int32_t from = pm[j - 1] + t[0], v;
			if (pi[j - 1] + t[3] > from) from = pi[j - 1] + t[3];
			if (pd[j - 1] + t[5] > from) from = pd[j - 1] + t[5];
			v = from + (aa < 20 ? emit[(size_t)(j - 1) * 20 + aa] : 0);
			cm[j] = v < 0 ? 0 : v;
			v = pm[j] + t[1] > pi[j] + t[4] ? pm[j] + t[1] : pi[j] + t[4];
			ci[j] = v < 0 ? 0 : v;
			v = pm[j - 1] + t[2] > pd[j - 1] + t[6] ? pm[j - 1] + t[2] : pd[j - 1] + t[6];
			cd[j] = v < 0 ? 0 : v;
			if (cm[j] > best) best = cm[j];
			if (ci[j] > best) best = ci[j];
		}
		x = pm, pm = cm, cm = x;
		x = pi, pi = ci, ci = x;
		x = pd, pd = cd, cd = x;
	}
	free(buf);
	return best;
}
