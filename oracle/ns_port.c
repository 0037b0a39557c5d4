/*
 * ns_port.c -- ORACLE (test infrastructure only; never part of the product path).
 *
 * A plain-C restatement of the reference CPU alignment path, used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.
 * It is pinned against the reference library compiled from the reference's own
 * sources (oracle/Makefile -> oracle/_ref/libnsref.so) and against the golden
 * fixtures under tests/golden/.
 *
 * What it restates (file:line in the reference project):
 *   - input preparation          nasw-sse.c:95-214 (ns_prep_nas/ns_prep_seq/ns_prep_seq_left)
 *   - 16-bit striped spliced DP   nasw-sse.c:351-567 (ns_global_gs16b_128)
 *   - 16-lane AVX2 ext DP         nasw-sse.c:596-741 (ns_global_gs16b_avx2)
 *   - 32-bit striped spliced DP   nasw-sse.c:779-973 (ns_global_gs32b)
 *   - width dispatch              nasw-sse.c:744-772, 980-999
 *   - backtrack                   nasw-sse.c:34-93, nasw.h:219-229
 *
 * The reference computes each DP row with Farrar striping: vsize lanes of
 * slen = ceil(al/vsize) consecutive columns, a first pass in which the
 * insertion (I) chain restarts at every segment start (column c with
 * c % slen == 0), then a "lazy-F" loop that carries the insertion across
 * segments.  The trace words depend on that schedule.  This file walks the
 * columns of a row in natural order and reproduces the schedule exactly with
 * three running values per row:
 *   ip  -- the first-pass insertion, reset at segment starts;
 *   ic  -- the carried insertion: at a segment start it is the max of the
 *          carry the first pass hands over (max(hfp(c-1)-(go+ge), ip(c-1)-ge))
 *          and the previous segment's carry decayed by ge; inside a segment it
 *          decays by ge per column;
 *   hfp -- the first-pass H (all candidates, using ip).
 * The final H is max(hfp, ic); a cell whose H was raised by ic gets trace
 * bit 9 (16-bit) or has its trace word replaced by 1|i_trace (32-bit).
 * All 16-bit arithmetic saturates exactly like _mm_adds/_mm_subs_epi16.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>
#include "../include/plgpu.h"

#define PORT_EXPORT __attribute__((visibility("default")))

static inline int32_t sat16(int32_t x) { return x < -32768 ? -32768 : x > 32767 ? 32767 : x; }
static inline int32_t max32(int32_t a, int32_t b) { return a > b ? a : b; }

/* ---------------------------------------------------------------- prep */

/* translation of the nucleotide string: nas[i] = codon ending at i, X after N
 * (nasw-sse.c:95-108) */
static void port_prep_nas(const char *ns, int32_t nl, const ns_opt_t *opt, uint8_t *nas)
{
	int32_t i, run = 0;
	uint8_t codon = 0;
	memset(nas, opt->aa20['X'], nl);
	for (i = 0; i < nl; ++i) {
		uint8_t c = opt->nt4[(uint8_t)ns[i]];
		if (c < 4) {
			codon = (uint8_t)((codon << 2 | c) & 0x3f);
			if (++run >= 3) nas[i] = opt->codon[codon];
		} else codon = 0, run = 0;
	}
}

/* forward preparation (nasw-sse.c:110-159); buffers are caller-allocated:
 * nas[nl], aas[al], donor[nl+1], acceptor[nl+1] */
static void port_prep_fwd(const char *ns, int32_t nl, const char *as, int32_t al, const ns_opt_t *opt,
		const uint8_t *ss, uint8_t *nas, uint8_t *aas, int8_t *donor, int8_t *acceptor)
{
	int32_t i, j;
	for (j = 0; j < al; ++j) aas[j] = opt->aa20[(uint8_t)as[j]];
	for (i = 0; i < nl; ++i) nas[i] = opt->nt4[(uint8_t)ns[i]];
	for (i = 0; i < nl + 1; ++i) donor[i] = acceptor[i] = (int8_t)opt->sp[3];
	for (i = 0; i < nl - 3; ++i) {
		int32_t t = 3;
		if (nas[i+1] == 2 && nas[i+2] == 3)
			t = i + 3 < nl && (nas[i+3] == 0 || nas[i+3] == 2) ? (nas[i] == 2 ? -1 : 4) : 0;
		else if (nas[i+1] == 2 && nas[i+2] == 1 && nas[i] == 2) t = 1;
		else if (nas[i+1] == 0 && nas[i+2] == 3) t = 2;
		donor[i] = (int8_t)(t < 0 ? 0 : opt->sp[t]);
	}
	for (i = 1; i < nl; ++i) {
		int32_t t = 3, pen = 0;
		if (nas[i-1] == 0 && nas[i] == 2) {
			t = i >= 2 && (nas[i-2] == 1 || nas[i-2] == 3) ? -1 : 0;
			for (j = i - 4; j >= 0 && j > i - 7; --j)
				if (nas[j] != 1 && nas[j] != 3) pen += opt->sp[5];
		} else if (nas[i-1] == 0 && nas[i] == 1) t = 2;
		acceptor[i] = (int8_t)(t < 0 ? 0 : opt->sp[t]);
		if (t == -1 || t == 0) acceptor[i] = (int8_t)(acceptor[i] + pen);
	}
	if (ss) {
		int32_t max_spsc = (opt->io + 1) / 2 - 1;
		for (i = 1; i < nl; ++i) {
			int32_t spsc = (int8_t)(ss[i] >> 1) - (int8_t)NS_SPSC_OFFSET;
			if (spsc > max_spsc) spsc = max_spsc;
			if (ss[i] == 0xff) {
				donor[i-1] = (int8_t)(donor[i-1] - opt->sp_null_bonus);
				acceptor[i-1] = (int8_t)(acceptor[i-1] - opt->sp_null_bonus);
			} else if (ss[i] & 1) acceptor[i-1] = (int8_t)(acceptor[i-1] - spsc);
			else donor[i-1] = (int8_t)(donor[i-1] - spsc);
		}
	}
	port_prep_nas(ns, nl, opt, nas);
}

/* left-extension preparation: everything reversed (nasw-sse.c:161-214) */
static void port_prep_left(const char *ns, int32_t nl, const char *as, int32_t al, const ns_opt_t *opt,
		const uint8_t *ss, uint8_t *nas, uint8_t *aas, int8_t *donor, int8_t *acceptor)
{
	int32_t i, j;
	uint8_t tmp;
	for (j = 0; j < al; ++j) aas[al - 1 - j] = opt->aa20[(uint8_t)as[j]];
	for (i = 0; i < nl; ++i) nas[nl - 1 - i] = opt->nt4[(uint8_t)ns[i]];
	for (i = 0; i < nl + 1; ++i) donor[i] = acceptor[i] = (int8_t)opt->sp[3];
	for (i = 0; i < nl - 3; ++i) {
		int32_t t = 3, pen = 0;
		if (nas[i+1] == 2 && nas[i+2] == 0) {
			t = i + 3 < nl && (nas[i+3] == 1 || nas[i+3] == 3) ? -1 : 0;
			for (j = i + 5; j < nl && j < i + 8; ++j)
				if (nas[j] != 1 && nas[j] != 3) pen += opt->sp[5];
		} else if (nas[i+1] == 1 && nas[i+2] == 0) t = 2;
		donor[i] = (int8_t)(t < 0 ? 0 : opt->sp[t]);
		if (t == -1 || t == 0) donor[i] = (int8_t)(donor[i] + pen);
	}
	for (i = 1; i < nl; ++i) {
		int32_t t = 3;
		if (nas[i-1] == 3 && nas[i] == 2)
			t = i >= 2 && (nas[i-2] == 0 || nas[i-2] == 2) ? (i + 1 < nl && nas[i+1] == 2 ? -1 : 4) : 0;
		else if (nas[i-1] == 1 && nas[i] == 2 && i + 1 < nl && nas[i+1] == 1) t = 1;
		else if (nas[i-1] == 3 && nas[i] == 0) t = 2;
		acceptor[i] = (int8_t)(t < 0 ? 0 : opt->sp[t]);
	}
	if (ss) {
		int32_t max_spsc = (opt->io + 1) / 2 - 1;
		for (i = 0; i < nl; ++i) {
			int32_t spsc = (int8_t)(ss[i] >> 1) - (int8_t)NS_SPSC_OFFSET;
			if (spsc > max_spsc) spsc = max_spsc;
			if (ss[i] == 0xff) {
				donor[nl - i - 1] = (int8_t)(donor[nl - i - 1] - opt->sp_null_bonus);
				acceptor[nl - i - 1] = (int8_t)(acceptor[nl - i - 1] - opt->sp_null_bonus);
			} else if (ss[i] & 1) donor[nl - i - 1] = (int8_t)(donor[nl - i - 1] - spsc);
			else acceptor[nl - i - 1] = (int8_t)(acceptor[nl - i - 1] - spsc);
		}
	}
	port_prep_nas(ns, nl, opt, nas);
	for (i = 0; i < nl >> 1; ++i)
		tmp = nas[i], nas[i] = nas[nl - 1 - i], nas[nl - 1 - i] = tmp;
	if (nl > 2) memmove(nas + 2, nas, nl - 2);
	if (nl > 0) nas[0] = opt->aa20['X'];
	if (nl > 1) nas[1] = opt->aa20['X'];
}

/* ------------------------------------------------------------- CIGAR */

static uint32_t *port_push(int32_t *n, int32_t *m, uint32_t *cigar, uint32_t op, int32_t len)
{ /* nasw.h:219-229 with km == NULL */
	if (*n == 0 || op != (cigar[*n - 1] & 0xf) || op == NS_CIGAR_F || op == NS_CIGAR_G) {
		if (*n == *m) {
			*m += (*m >> 1) + 8;
			cigar = (uint32_t*)realloc(cigar, (size_t)*m * sizeof(uint32_t));
		}
		cigar[(*n)++] = (uint32_t)len << 4 | op;
	} else cigar[*n - 1] += (uint32_t)len << 4;
	return cigar;
}

/* trace words here are "effective": bits 0-3 hold the state (already 1 where
 * the reference's lazy-F bit 9 is set), bits 4-8 the extension bits.
 * Walk follows nasw-sse.c:44-93. */
static void port_backtrack(const uint16_t *tb, int32_t nl, int32_t al, ns_rst_t *r)
{
	int32_t i = nl - 1, j = al - 1, last = 0, k;
	uint32_t tmp;
	while (i >= 2 && j >= 0) {
		int32_t x = tb[(int64_t)(i - 2) * al + j];
		int32_t state = last == 0 ? (x & 0xf) : last;
		int32_t ext = state >= 1 && state <= 5 ? (x >> (state + 3)) & 1 : 0;
		switch (state) {
		case 0: r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_M, 1), i -= 3, --j; break;
		case 1: r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_I, 1), --j; break;
		case 2: r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_D, 1), i -= 3; break;
		case 3: r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_N, 1), --i; break;
		case 4: r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_U, 1), --i; if (!ext) --j; break;
		case 5: r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_V, 1), --i; if (!ext) --j; break;
		case 6: r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_F, 1), --i; break;
		case 7: r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_F, 2), i -= 2; break;
		case 8: r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_G, 1), --i, --j; break;
		default: r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_G, 2), i -= 2, --j; break;
		}
		last = state >= 1 && state <= 5 && ext ? state : 0;
	}
	if (j > 0) r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_I, j);
	if (i >= 0) {
		int32_t l = (i + 1) / 3, t = (i + 1) % 3;
		if (l > 0) r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_D, l);
		if (t != 0) r->cigar = port_push(&r->n_cigar, &r->m_cigar, r->cigar, NS_CIGAR_F, t);
	}
	for (k = 0; k < r->n_cigar >> 1; ++k)
		tmp = r->cigar[k], r->cigar[k] = r->cigar[r->n_cigar - 1 - k], r->cigar[r->n_cigar - 1 - k] = tmp;
	for (k = 0; k < r->n_cigar; ++k) { /* nasw-sse.c:34-42 */
		int32_t op = r->cigar[k] & 0xf;
		if ((op == NS_CIGAR_U || op == NS_CIGAR_V) && r->cigar[k] >> 4 < 3)
			r->cigar[k] = r->cigar[k] >> 4 << 4 | NS_CIGAR_G;
	}
}

/* ---------------------------------------------------------- the DP core */

typedef struct {
	int32_t wide;     /* 0: int16 saturating, vsize 8 (or 16); 1: int32, vsize 4 */
	int32_t vsize;
	int32_t ext;      /* NS_F_EXT_LEFT|RIGHT set */
} port_mode_t;

/* one sub/add with the width's arithmetic */
#define OPS(x) (m.wide ? (x) : sat16(x))

static void port_dp(const ns_opt_t *opt, port_mode_t m, int32_t nl, int32_t al,
		const uint8_t *nas, const uint8_t *aas, const int8_t *donor, const int8_t *acceptor,
		uint16_t *tb, ns_rst_t *r)
{
	const int32_t NEG = m.wide ? -0x40000000 : -32768;
	const int32_t slen = (al + m.vsize - 1) / m.vsize;
	const int32_t ncol = m.ext ? slen * m.vsize : al; /* ext mode feeds padded columns to the row max */
	const int32_t go = opt->go, ge = opt->ge, goe = opt->go + opt->ge, io = opt->io, fs = opt->fs;
	int32_t *buf, *Hr[4], *Dr[4], *A, *B, *C, *Hmax, *prof;
	int32_t i, c, a;
	int32_t max_sc = INT32_MIN, max_sc_log = INT32_MIN, max_i = -1, pen_len = al * 3;

	buf = (int32_t*)malloc(sizeof(int32_t) * (size_t)ncol * 12 + sizeof(int32_t) * (size_t)opt->asize * ncol);
	for (i = 0; i < 4; ++i) Hr[i] = buf + (size_t)i * ncol, Dr[i] = buf + (size_t)(4 + i) * ncol;
	A = buf + (size_t)8 * ncol, B = A + ncol, C = B + ncol, Hmax = C + ncol;
	prof = Hmax + ncol;
	for (i = 0; i < ncol * 12; ++i) buf[i] = NEG;
	for (a = 0; a < opt->asize; ++a) /* query profile, nasw-sse.c:223-235 (padding = neg_inf) */
		for (c = 0; c < ncol; ++c) {
			/* position-specific scores (nasw-sse.c:217-221): rows in query order, reversed for a left extension */
			const int32_t q = (opt->flag & NS_F_EXT_LEFT) ? al - 1 - c : c;
			prof[a * ncol + c] = c >= al ? NEG : opt->pssm ? opt->pssm[q * opt->asize + a] : opt->sc[a * opt->asize + aas[c]];
		}

	for (i = 2; i < nl; ++i) {
		int32_t *H = Hr[i & 3], *H1 = Hr[(i - 1) & 3], *H2 = Hr[(i - 2) & 3], *H3 = Hr[(i - 3) & 3];
		int32_t *D = Dr[i & 3], *D3 = Dr[(i - 3) & 3];
		const int32_t *S = prof + nas[i] * ncol;
		const int32_t gei = nas[i] == 20 ? fs : ge;
		const int32_t dim1 = donor[i-1], di = donor[i], dip1 = donor[i+1];
		const int32_t ai = acceptor[i], aim1 = acceptor[i-1], aim2 = acceptor[i-2];
		int32_t ip = NEG, last_h = NEG, ic = NEG, h3m1, h2m1, h1m1, row_max = NEG;
		/* column -1 (nasw-sse.c:264-282): {0,-fs,-fs} for rows -1,0,1 while computing row 2, else neg_inf */
		h3m1 = i == 2 ? 0 : NEG, h2m1 = i == 2 ? -fs : NEG, h1m1 = i == 2 ? -fs : NEG;
		for (c = 0; c < ncol; ++c) {
			int32_t h, t, u, v, y = 0, z = 0, it = 16, hfp;
			/* segment start: hand over the carry, restart the first-pass chain */
			if (c % slen == 0) {
				if (c == 0) ic = NEG, it = 0;
				else {
					int32_t hop = OPS(last_h - goe), iext = OPS(ip - ge), c0 = max32(hop, iext);
					int32_t older = OPS(ic - ge);
					it = c0 >= older ? (iext > hop ? 16 : 0) : 16;
					ic = max32(c0, older);
				}
				ip = NEG, last_h = NEG;
			} else ic = OPS(ic - ge);
			/* first pass, candidate order of nasw-sse.c:464-536 */
			h = OPS(h3m1 + S[c]);
			t = OPS(last_h - go);
			z |= ip > t ? 1 << 4 : 0;
			t = max32(t, ip);
			ip = OPS(t - ge);
			if (ip > h) y = 1;
			h = max32(h, ip);
			u = OPS(H3[c] - go);
			v = D3[c];
			z |= v > u ? 1 << 5 : 0;
			t = OPS(max32(u, v) - gei);
			D[c] = t;
			if (t > h) y = 2;
			h = max32(h, t);
			u = OPS(H1[c] - io);
			v = A[c];
			t = OPS(u - dim1);
			z |= v > t ? 1 << 6 : 0;
			t = max32(t, v);
			A[c] = t;
			t = OPS(t - ai);
			if (t > h) y = 3;
			h = max32(h, t);
			u = OPS(h1m1 - io);
			v = B[c];
			t = OPS(u - di);
			z |= v > t ? 1 << 7 : 0;
			t = max32(t, v);
			B[c] = t;
			t = OPS(t - aim2);
			if (t > h) y = 4;
			h = max32(h, t);
			v = C[c];
			t = OPS(u - dip1);
			z |= v > t ? 1 << 8 : 0;
			t = max32(t, v);
			C[c] = t;
			t = OPS(t - aim1);
			if (t > h) y = 5;
			h = max32(h, t);
			t = OPS(H1[c] - fs);
			if (t > h) y = 6;
			h = max32(h, t);
			t = OPS(H2[c] - fs);
			if (t > h) y = 7;
			h = max32(h, t);
			t = OPS(h1m1 - fs);
			if (t > h) y = 8;
			h = max32(h, t);
			t = OPS(h2m1 - fs);
			if (t > h) y = 9;
			h = max32(h, t);
			hfp = h;
			/* lazy-F: raise by the carried insertion */
			if (ic > hfp) {
				h = ic;
				if (m.wide) z = 1 | it; /* nasw-sse.c:949: the whole word is replaced */
				else z |= 1;            /* bit 9 -> state 1, extension bits kept (nasw-sse.c:54) */
				y = 0;
			}
			z |= y;
			if (tb && c < al) tb[(int64_t)(i - 2) * al + c] = (uint16_t)z;
			/* column c-1 values of the rows above for the next column */
			h3m1 = H3[c], h2m1 = H2[c], h1m1 = H1[c];
			H[c] = h;
			if (h > row_max) row_max = h;
			last_h = hfp;
		}
		if (m.ext) { /* nasw-sse.c:436-446 */
			int32_t tmp_sc = row_max, end_sc = H[al - 1] + opt->end_bonus, tmp_sc_log, d = i - pen_len, pen = 0;
			if (end_sc > tmp_sc) tmp_sc = end_sc;
			if (d >= 2) { /* (int32_t)(ie_coef * ns_log2(d) + .5f), nasw-sse.c:341-349 */
				union { float f; uint32_t u; } z = { (float)d };
				float l2 = (float)(((z.u >> 23) & 255) - 128);
				float p1, p2, p3, p4;
				z.u &= ~(255u << 23);
				z.u += 127u << 23;
				p1 = -0.34484843f * z.f;
				p2 = p1 + 2.02466578f;
				p3 = p2 * z.f;
				p4 = p3 - 0.67487759f;
				l2 = l2 + p4;
				pen = (int32_t)(opt->ie_coef * l2 + .5f);
			}
			tmp_sc_log = tmp_sc - pen;
			if (tmp_sc_log > max_sc_log) {
				max_sc = tmp_sc, max_sc_log = tmp_sc_log, max_i = i;
				memcpy(Hmax, H, sizeof(int32_t) * (size_t)ncol);
			}
			if (max_sc_log - tmp_sc_log > opt->xdrop) break;
		}
	}
	if (m.ext) { /* nasw-sse.c:448-458 */
		int32_t best_j = -1, best_sc = INT32_MIN, j;
		for (j = 0; j < al; ++j) {
			int32_t sc = Hmax[j];
			if (j == al - 1) sc += opt->end_bonus;
			if (sc > best_sc) best_sc = sc, best_j = j;
			if (sc == max_sc) break;
		}
		if (j >= al) j = best_j, max_sc = best_sc;
		r->nt_len = max_i + 1, r->aa_len = j + 1, r->score = max_sc;
	} else r->score = nl > 2 ? Hr[(nl - 1) & 3][al - 1] : Hr[1][al - 1];
	free(buf);
}

static int32_t port_stripe_width(const ns_opt_t *opt, int32_t al, int32_t avx2)
{ /* nasw-sse.c:744-750; avx2 = whether the CPU kernel would dispatch to AVX2 */
	if ((opt->flag & (NS_F_EXT_LEFT | NS_F_EXT_RIGHT)) && al >= 16 && avx2) return 16;
	return 8;
}

static void port_run(const char *ns, int32_t nl, const char *as, int32_t al, const ns_opt_t *opt,
		const uint8_t *ss, ns_rst_t *r, port_mode_t m)
{
	uint8_t *nas = (uint8_t*)malloc((size_t)nl + al + 2 * ((size_t)nl + 1) + 8), *aas = nas + nl;
	int8_t *donor = (int8_t*)aas + al, *acceptor = donor + nl + 1;
	uint16_t *tb = 0;
	int32_t want_tb = (opt->flag & NS_F_CIGAR) && !m.ext;
	r->n_cigar = 0, r->nt_len = nl, r->aa_len = al, r->score = INT32_MIN;
	if (opt->flag & NS_F_EXT_LEFT) port_prep_left(ns, nl, as, al, opt, ss, nas, aas, donor, acceptor);
	else port_prep_fwd(ns, nl, as, al, opt, ss, nas, aas, donor, acceptor);
	if (want_tb && nl > 2) tb = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)(nl - 2) * al);
	port_dp(opt, m, nl, al, nas, aas, donor, acceptor, tb, r);
	if (want_tb) port_backtrack(tb, nl, al, r);
	free(tb);
	free(nas);
}

/* ns_global_gs16b (nasw-sse.c:763-772); avx2 selects the 16-lane ext kernel as the CPU would */
PORT_EXPORT void port_global_gs16b(const char *ns, int32_t nl, const char *as, int32_t al, const ns_opt_t *opt,
		const uint8_t *ss, ns_rst_t *r, int32_t avx2)
{
	port_mode_t m;
	m.wide = 0, m.ext = !!(opt->flag & (NS_F_EXT_LEFT | NS_F_EXT_RIGHT));
	m.vsize = port_stripe_width(opt, al, avx2);
	port_run(ns, nl, as, al, opt, ss, r, m);
}

/* ns_global_gs32b (nasw-sse.c:779-973) */
PORT_EXPORT void port_global_gs32b(const char *ns, int32_t nl, const char *as, int32_t al, const ns_opt_t *opt,
		const uint8_t *ss, ns_rst_t *r)
{
	port_mode_t m;
	m.wide = 1, m.ext = 0, m.vsize = 4;
	port_run(ns, nl, as, al, opt, ss, r, m);
}

/* 1 when ns_global_gs_auto() would pick the 32-bit kernel (nasw-sse.c:987-996) */
PORT_EXPORT int32_t port_needs_wide(const ns_opt_t *opt, int32_t al)
{
	int32_t i, max_sub = 0;
	int64_t max_score;
	if (opt->pssm) {
		for (i = 0; i < al * opt->asize; ++i) if (max_sub < opt->pssm[i]) max_sub = opt->pssm[i];
	} else {
		for (i = 0; i < opt->asize * opt->asize; ++i) if (max_sub < opt->sc[i]) max_sub = opt->sc[i];
	}
	max_score = (int64_t)al * max_sub + opt->end_bonus;
	return !(opt->flag & (NS_F_EXT_LEFT | NS_F_EXT_RIGHT)) && max_score > 30000;
}

/* ns_global_gs_auto without the GPU branch (nasw-sse.c:980-999) */
PORT_EXPORT void port_global_gs_auto(const char *ns, int32_t nl, const char *as, int32_t al, const ns_opt_t *opt,
		const uint8_t *ss, ns_rst_t *r, int32_t avx2)
{
	if (port_needs_wide(opt, al)) port_global_gs32b(ns, nl, as, al, opt, ss, r);
	else port_global_gs16b(ns, nl, as, al, opt, ss, r, avx2);
}

/* the preparation step alone (nasw-sse.c:752-756): fills caller buffers */
PORT_EXPORT void port_prep(const char *ns, int32_t nl, const char *as, int32_t al, const ns_opt_t *opt,
		const uint8_t *ss, uint8_t *nas, uint8_t *aas, int8_t *donor, int8_t *acceptor)
{
	if (opt->flag & NS_F_EXT_LEFT) port_prep_left(ns, nl, as, al, opt, ss, nas, aas, donor, acceptor);
	else port_prep_fwd(ns, nl, as, al, opt, ss, nas, aas, donor, acceptor);
}

PORT_EXPORT void port_free(void *p) { free(p); }
