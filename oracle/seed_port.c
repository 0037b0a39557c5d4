/*
 * seed_port.c -- test infrastructure: a plain C restatement of the coarse mapper's
 * seeding (the checker of protlocus_b200/csrc/seed.cu), for protein queries and for
 * HMM-profile queries (sp_sketch_hmm, sp_seeds_hmm_query, sp_anchors_hmm below):
 *
 *   sketch    mp_sketch_prot (sketch.c:18-37): residues in the 13-letter alphabet of
 *             nasw-tab.c:12 (codes 14 and 15, '*', 'X' and other bytes, restart the
 *             k-mer), 4 bits per residue, the masked integer hash of sketch.c:7-16,
 *             a seed (hash >> mod_bit) << 32 | position where the hash's low mod_bit
 *             bits are 0;
 *   max_occ   mp_cal_max_occ (map.c:304-320): from 8 seeds on, the box-plot bound
 *             q75 + 1.5 (q75 - q25) + 10 over the seeds' bucket sizes, capped by the
 *             option (map.c:566-569);
 *   anchors   mp_collect_anchors (map.c:346-397): every block of every seed whose bucket
 *             holds at most max_occ, as block << 32 | position; with the accuracy mode's
 *             repeat rescue (sp_anchors_acc), up to repeat_cap evenly spaced blocks of the
 *             other buckets, within anchor_budget: the seeds' shares scaled down, then the
 *             rest handed out one at a time from the query name's hash onwards, over the
 *             seeds in their sorted order (map.c:360-384);
 *   order     radix_sort_mp64 of the anchors (map.c:571): ascending.
 * The index is the reference's (index.c:74-98): ki[b] the first entry of bucket b in
 * kb, the bucket's end ki[b+1] (n_kb for the last bucket).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SP_EXPORT __attribute__((visibility("default")))

/* nasw-tab.c:9-12: the residue letters and their 13-letter groups */
static const char *sp_aa = "ARNDCQEGHILKMFPSTWYV*X";
static const uint8_t sp_a2r[22] = { 0, 2, 4, 4, 6, 5, 5, 8, 3, 10, 11, 2, 11, 12, 7, 1, 1, 13, 12, 10, 14, 15 };

SP_EXPORT void sp_aa13_table(uint8_t *tab)
{
	int i;
	memset(tab, 15, 256);
	for (i = 0; sp_aa[i]; ++i) {
		const uint8_t c = (uint8_t)sp_aa[i];
		tab[i] = tab[c] = sp_a2r[i];
		if (c >= 'A' && c <= 'Z') tab[c + 32] = sp_a2r[i];
	}
}

static uint32_t sp_hash(uint32_t key, uint32_t mask)
{ /* sketch.c:7-16 */
	key = (key + ~(key << 15)) & mask;
	key ^= key >> 10;
	key = (key + (key << 3)) & mask;
	key ^= key >> 6;
	key = (key + ~(key << 11)) & mask;
	key ^= key >> 16;
	return key;
}

static int sp_cmp64(const void *a, const void *b)
{
	const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
	return x < y ? -1 : x > y;
}

/* the seeds of one protein; returns their number (at most len) */
SP_EXPORT int32_t sp_sketch(const uint8_t *seq, int32_t len, int32_t kmer, int32_t mod_bit, uint64_t *seeds)
{
	uint8_t tab[256];
	int32_t i, l = 0, n = 0;
	const uint32_t mask_k = (1U << kmer * 4) - 1, mask_mod = (1U << mod_bit) - 1;
	uint32_t x = 0;
	sp_aa13_table(tab);
	for (i = 0; i < len; ++i) {
		const uint32_t c = tab[seq[i]];
		if (c < 14) {
			x = (x << 4 | c) & mask_k;
			if (++l >= kmer) {
				const uint32_t y = sp_hash(x, mask_k);
				if ((y & mask_mod) == 0) seeds[n++] = (uint64_t)(y >> mod_bit) << 32 | (uint32_t)i;
			}
		} else x = 0, l = 0;
	}
	return n;
}

/* mp_hash_qname (map.c:322-329): FNV-1a over the name's bytes */
SP_EXPORT uint32_t sp_qname_hash(const char *qname)
{
	uint32_t h = 2166136261U;
	if (!qname) return h;
	for (; *qname; ++qname) h = (h ^ (uint8_t)*qname) * 16777619U;
	return h;
}

/* the anchors of n seeds sd (sorted; freed here) into *out (malloc'd, sorted); returns
 * their number, -1 on a host allocation failure.  repeat_cap > 0: the accuracy mode's
 * repeat rescue with anchor_budget and the query name's hash qhash */
static int64_t sp_anchors_of(const int64_t *ki, int64_t n_bucket, const uint32_t *kb, int64_t n_kb, int32_t max_occ_opt,
		int32_t repeat_cap, int64_t anchor_budget, uint32_t qhash, uint64_t *sd, int32_t n, uint64_t **out)
{
	uint64_t *cnt, *a;
	int64_t *take;
	int32_t i, max_occ = max_occ_opt;
	int64_t n_a = 0, n_res = 0, k = 0, j;
	*out = 0;
	if (n >= 8) {
		uint64_t q25, q75;
		cnt = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
		if (!cnt) { free(sd); return -1; }
		for (i = 0; i < n; ++i) {
			const int64_t b = (int64_t)(sd[i] >> 32), en = b + 1 < n_bucket ? ki[b + 1] : n_kb;
			cnt[i] = (uint64_t)(en - ki[b]);
		}
		qsort(cnt, (size_t)n, sizeof(uint64_t), sp_cmp64);
		q25 = cnt[(int64_t)(n * .25 + .499)], q75 = cnt[(int64_t)(n * .75 + .499)];
		max_occ = (int32_t)(q75 + (q75 - q25) * 1.5 + 10.);
		free(cnt);
		if (max_occ > max_occ_opt) max_occ = max_occ_opt;
	}
	take = (int64_t*)calloc((size_t)(n > 0 ? n : 1), sizeof(int64_t));
	if (!take) { free(sd); return -1; }
	for (i = 0; i < n; ++i) {
		const int64_t b = (int64_t)(sd[i] >> 32), sz = (b + 1 < n_bucket ? ki[b + 1] : n_kb) - ki[b];
		if (sz <= max_occ) take[i] = sz, n_a += sz;
		else if (repeat_cap > 0) take[i] = sz < repeat_cap ? sz : repeat_cap, n_res += take[i];
	}
	if (n_res > anchor_budget) {
		int64_t used = 0;
		const uint32_t start = n > 0 ? qhash % (uint32_t)n : 0;
		for (i = 0; i < n; ++i) {
			const int64_t b = (int64_t)(sd[i] >> 32), sz = (b + 1 < n_bucket ? ki[b + 1] : n_kb) - ki[b];
			if (sz > max_occ && take[i] > 0) take[i] = take[i] * anchor_budget / n_res, used += take[i];
		}
		for (i = 0; i < n && used < anchor_budget; ++i) {
			const int32_t jj = (int32_t)((start + (uint32_t)i) % (uint32_t)n);
			const int64_t b = (int64_t)(sd[jj] >> 32), sz = (b + 1 < n_bucket ? ki[b + 1] : n_kb) - ki[b];
			const int64_t cap = sz < repeat_cap ? sz : repeat_cap;
			if (sz > max_occ && take[jj] < cap) ++take[jj], ++used;
		}
		n_res = used;
	}
	n_a += n_res;
	a = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n_a > 0 ? n_a : 1));
	if (!a) { free(sd), free(take); return -1; }
	for (i = 0; i < n; ++i) {
		const int64_t b = (int64_t)(sd[i] >> 32), st = ki[b], sz = (b + 1 < n_bucket ? ki[b + 1] : n_kb) - st;
		if (take[i] == sz) {
			for (j = 0; j < sz; ++j) a[k++] = (uint64_t)kb[st + j] << 32 | (uint32_t)sd[i];
		} else if (take[i] > 0) {
			const int64_t mid = sz / (2 * take[i]);
			for (j = 0; j < take[i]; ++j) a[k++] = (uint64_t)kb[st + j * sz / take[i] + mid] << 32 | (uint32_t)sd[i];
		}
	}
	qsort(a, (size_t)n_a, sizeof(uint64_t), sp_cmp64);
	free(sd), free(take);
	*out = a;
	return n_a;
}

SP_EXPORT int64_t sp_anchors_acc(const int64_t *ki, int64_t n_bucket, const uint32_t *kb, int64_t n_kb, int32_t kmer,
		int32_t mod_bit, int32_t max_occ_opt, int32_t repeat_cap, int64_t anchor_budget, uint32_t qhash,
		const uint8_t *seq, int32_t len, uint64_t **out)
{
	uint64_t *sd = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(len > 0 ? len : 1));
	int32_t n;
	*out = 0;
	if (!sd) return -1;
	n = sp_sketch(seq, len, kmer, mod_bit, sd);
	qsort(sd, (size_t)n, sizeof(uint64_t), sp_cmp64);  /* mp_sketch_query's order */
	return sp_anchors_of(ki, n_bucket, kb, n_kb, max_occ_opt, repeat_cap, anchor_budget, qhash, sd, n, out);
}

/* ---- HMM-profile queries: mp_sketch_hmm (sketch.c:40-118) and mp_sketch_query's merge
 * (map.c:332-343) ---- */

#define SP_HMM_ALT 4  /* MP_HMM_MAX_ALT (sketch.c:40) */

typedef struct { int32_t n; int16_t loss[SP_HMM_ALT]; uint8_t code[SP_HMM_ALT]; } sp_alt_t;

/* one match state's alternatives (sketch.c:57-76): every 13-letter group takes the best
 * emission of its residues (20 columns in HMMER order ACDEFGHIKLMNPQRSTVWY; a group none of
 * them maps to, or whose best is INT16_MIN, offers nothing); the groups within pos_loss of
 * the state's best are offered in group order to a list of four kept in ascending order by
 * insertion: a full list takes a group only below its last entry, which drops out, and a
 * group goes after the kept entries not above it.  Losses are stored in 16 bits as the
 * reference's alt_loss (a loss over 32767 wraps; the comparisons then see the wrapped
 * entries against the new group's full loss) */
static void sp_hmm_alts(const int16_t *e20, int32_t pos_loss, const uint8_t *tab, sp_alt_t *al)
{
	static const char col[] = "ACDEFGHIKLMNPQRSTVWY";
	int32_t gs[14], best = INT16_MIN, g, j;
	for (g = 0; g < 14; ++g) gs[g] = INT16_MIN;
	for (j = 0; j < 20; ++j) {
		g = tab[(uint8_t)col[j]];
		if (e20[j] > gs[g]) gs[g] = e20[j];
	}
	for (g = 0; g < 14; ++g) if (gs[g] > best) best = gs[g];
	memset(al, 0, sizeof(*al));
	for (g = 0; g < 14; ++g) {
		const int32_t loss = best - gs[g];
		int32_t stay, at;
		if (gs[g] == INT16_MIN || loss > pos_loss) continue;
		if (al->n == SP_HMM_ALT && loss >= al->loss[SP_HMM_ALT - 1]) continue;
		stay = al->n < SP_HMM_ALT ? al->n : SP_HMM_ALT - 1;
		at = stay;
		while (at > 0 && al->loss[at - 1] > loss) --at;
		memmove(&al->loss[at + 1], &al->loss[at], sizeof(int16_t) * (size_t)(stay - at));
		memmove(&al->code[at + 1], &al->code[at], (size_t)(stay - at));
		al->loss[at] = (int16_t)loss, al->code[at] = (uint8_t)g;
		al->n = stay + 1;
	}
}

typedef struct {
	const sp_alt_t *al;
	int32_t kmer, mod_bit, win_loss, n_emit, max_per_win, end;
	uint32_t mask_k, mask_mod;
	uint64_t *out;
	int64_t n_out;
} sp_walk_t;

/* the k-mers of one window in lexicographic order of their alternatives' ranks (sketch.c:
 * 78-110): a position's next alternative is taken while the losses so far (acc) plus its
 * own stay within win_loss, the first that does not ends the position; every whole k-mer
 * counts towards max_per_win, a seed is kept where its hash passes the sampling */
static void sp_hmm_walk(sp_walk_t *w, int32_t d, int32_t acc, uint32_t x)
{
	int32_t r;
	if (d == w->kmer) {
		const uint32_t y = sp_hash(x, w->mask_k);
		if ((y & w->mask_mod) == 0) w->out[w->n_out++] = (uint64_t)(y >> w->mod_bit) << 32 | (uint32_t)w->end;
		++w->n_emit;
		return;
	}
	for (r = 0; r < w->al[d].n && w->n_emit < w->max_per_win && acc + w->al[d].loss[r] <= w->win_loss; ++r)
		sp_hmm_walk(w, d + 1, acc + w->al[d].loss[r], (x << 4 | w->al[d].code[r]) & w->mask_k);
}

/* mp_sketch_hmm: the profile-derived seeds of every window of kmer match states (emit:
 * len x 20), appended to out (room for (len - kmer + 1) * max_per_win); returns their
 * number, -1 on a host allocation failure */
SP_EXPORT int64_t sp_sketch_hmm(const int16_t *emit, int32_t len, int32_t kmer, int32_t mod_bit, int32_t pos_loss,
		int32_t win_loss, int32_t max_per_win, uint64_t *out)
{
	uint8_t tab[256];
	sp_alt_t *al;
	sp_walk_t w;
	int32_t i;
	if (!emit || len < kmer || max_per_win <= 0) return 0;
	al = (sp_alt_t*)malloc(sizeof(sp_alt_t) * (size_t)len);
	if (!al) return -1;
	sp_aa13_table(tab);
	for (i = 0; i < len; ++i) sp_hmm_alts(emit + (size_t)i * 20, pos_loss, tab, &al[i]);
	memset(&w, 0, sizeof(w));
	w.kmer = kmer, w.mod_bit = mod_bit, w.win_loss = win_loss, w.max_per_win = max_per_win, w.out = out;
	w.mask_k = (1U << kmer * 4) - 1, w.mask_mod = (1U << mod_bit) - 1;
	for (i = kmer - 1; i < len; ++i) {
		w.al = al + (i - kmer + 1), w.end = i, w.n_emit = 0;
		sp_hmm_walk(&w, 0, 0, 0);
	}
	free(al);
	return w.n_out;
}

/* an HMM-profile query's seeds (mp_sketch_query with a profile): the sequence's own (the
 * parser's consensus, in the mapper) and, when seed_max > 0, the profile-derived ones,
 * sorted with the duplicates removed; *out malloc'd, returns the number, -1 on a host
 * allocation failure */
SP_EXPORT int64_t sp_seeds_hmm_query(const uint8_t *seq, int32_t len, const int16_t *emit, int32_t hmm_len, int32_t kmer,
		int32_t mod_bit, int32_t pos_loss, int32_t win_loss, int32_t seed_max, uint64_t **out)
{
	const int64_t n_win = seed_max > 0 && hmm_len >= kmer ? (int64_t)(hmm_len - kmer + 1) * seed_max : 0;
	uint64_t *sd = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(len + n_win > 0 ? len + n_win : 1));
	int64_t n, m, i, k;
	*out = 0;
	if (!sd) return -1;
	n = sp_sketch(seq, len, kmer, mod_bit, sd);
	if (seed_max > 0) {
		m = sp_sketch_hmm(emit, hmm_len, kmer, mod_bit, pos_loss, win_loss, seed_max, sd + n);
		if (m < 0) { free(sd); return -1; }
		n += m;
	}
	qsort(sd, (size_t)n, sizeof(uint64_t), sp_cmp64);
	for (i = k = 0; i < n; ++i)
		if (k == 0 || sd[i] != sd[k - 1]) sd[k++] = sd[i];
	*out = sd;
	return k;
}

/* the anchors of an HMM-profile query: its seeds (sp_seeds_hmm_query), then the cap and
 * the collection (map.c:565-572), with the repeat rescue when repeat_cap > 0 */
SP_EXPORT int64_t sp_anchors_hmm(const int64_t *ki, int64_t n_bucket, const uint32_t *kb, int64_t n_kb, int32_t kmer,
		int32_t mod_bit, int32_t max_occ_opt, int32_t repeat_cap, int64_t anchor_budget, uint32_t qhash,
		const uint8_t *seq, int32_t len, const int16_t *emit, int32_t hmm_len, int32_t pos_loss, int32_t win_loss,
		int32_t seed_max, uint64_t **out)
{
	uint64_t *sd;
	const int64_t n = sp_seeds_hmm_query(seq, len, emit, hmm_len, kmer, mod_bit, pos_loss, win_loss, seed_max, &sd);
	*out = 0;
	if (n < 0) return -1;
	return sp_anchors_of(ki, n_bucket, kb, n_kb, max_occ_opt, repeat_cap, anchor_budget, qhash, sd, (int32_t)n, out);
}

SP_EXPORT int64_t sp_anchors(const int64_t *ki, int64_t n_bucket, const uint32_t *kb, int64_t n_kb, int32_t kmer,
		int32_t mod_bit, int32_t max_occ_opt, const uint8_t *seq, int32_t len, uint64_t **out)
{
	return sp_anchors_acc(ki, n_bucket, kb, n_kb, kmer, mod_bit, max_occ_opt, 0, 0, 0, seq, len, out);
}

SP_EXPORT void sp_free(void *p) { free(p); }
