/*
 * gapless_port.c -- ORACLE (test infrastructure only): sequential C restatement
 * of the reference's gapless X-drop candidate prefilter, ns_gapless_xdrop_batch
 * (nasw-cuda.cu:1151-1295, entry point nasw-cuda.cu:1330-1395).  The reference
 * has no CPU twin of this kernel; this restatement is pinned against the
 * reference kernel's own outputs (tests/golden/gapless_golden.json, made by
 * running the reference CUDA code, see tests/golden/make_gapless_golden.py).
 *
 * Per candidate (at most 32 anchors, nasw-cuda.cu:1174):
 *   seed    for each anchor, the best k-mer seed over the block_width target
 *           ends target_block + delta: the sum of kmer codon-vs-query scores;
 *           ties go to the smaller target end (nasw-cuda.cu:1198-1221);
 *   extend  from the seed, left then right, one codon per query residue, with
 *           the X-drop rule; the best prefix of each side counts
 *           (nasw-cuda.cu:1227-1256);
 *   combine segments sorted by score (stable), then greedily summed: a segment
 *           after the first that scores below xdrop stops the sum, one fully
 *           covered by better segments is dropped, a partly covered one adds
 *           score*(len-overlap)/len (nasw-cuda.cu:1259-1293).
 * The genome is 4-bit packed, low nibble first; reverse candidates read the
 * mirrored, complemented strand (nasw-cuda.cu:1151-1160).
 */
#include <limits.h>
#include <stdint.h>
#include <string.h>
#include "../include/plgpu.h"

#define PORT_EXPORT __attribute__((visibility("default")))
#define MAX_ANCHORS 32

static uint8_t base_at(const uint8_t *packed, const ns_gpu_gapless_candidate_t *c, int64_t pos)
{
	int64_t a;
	uint8_t b;
	if (pos < 0 || pos >= c->target_length) return 4;
	a = c->target_offset + (c->reverse ? c->target_length - 1 - pos : pos);
	b = packed[a >> 1] >> ((a & 1) * 4) & 0xf;
	return c->reverse && b < 4 ? 3 - b : b;
}

static uint8_t aa_at(const uint8_t *packed, const uint8_t *codon, const ns_gpu_gapless_candidate_t *c, int64_t end)
{
	const uint8_t b0 = base_at(packed, c, end - 2), b1 = base_at(packed, c, end - 1), b2 = base_at(packed, c, end);
	return b0 < 4 && b1 < 4 && b2 < 4 ? codon[b0 << 4 | b1 << 2 | b2] : 20;
}

PORT_EXPORT int32_t port_gapless_score_batch(const uint8_t *packed, const uint8_t *queries,
		const ns_gpu_gapless_candidate_t *cands, int32_t n_cand, const ns_gpu_gapless_anchor_t *anchors,
		int32_t block_width, int32_t kmer, int32_t xdrop, const int8_t *mat, int32_t asize, const uint8_t *codon,
		int32_t *scores)
{
	int32_t ci;
	for (ci = 0; ci < n_cand; ++ci) {
		const ns_gpu_gapless_candidate_t *c = &cands[ci];
		const uint8_t *q = queries + c->query_offset;
		const int32_t na = c->anchor_count < MAX_ANCHORS ? c->anchor_count : MAX_ANCHORS;
		int32_t seg_qs[MAX_ANCHORS], seg_qe[MAX_ANCHORS], seg_sc[MAX_ANCHORS];
		int32_t n_seg = 0, total = 0, any = 0, a, i, j;
		for (a = 0; a < na; ++a) {
			const ns_gpu_gapless_anchor_t *an = &anchors[c->anchor_offset + a];
			int32_t best_seed = INT32_MIN, qend = -1, delta, sc, qs, qe;
			int64_t best_te = INT64_MAX;
			if (an->query_end >= kmer - 1 && an->query_end < c->query_length) {
				for (delta = 0; delta < block_width; ++delta) {
					const int64_t te = an->target_block + delta;
					int32_t s = 0, k;
					if (te - (int64_t)(kmer - 1) * 3 - 2 < 0 || te >= c->target_length) continue;
					for (k = 0; k < kmer; ++k)
						s += mat[aa_at(packed, codon, c, te - (int64_t)(kmer - 1 - k) * 3) * asize + q[an->query_end - kmer + 1 + k]];
					if (s > best_seed) best_seed = s, best_te = te, qend = an->query_end; /* deltas ascend: ties keep the smaller end */
				}
			}
			if (qend < 0) continue;
			{
				int32_t lr = 0, lb = 0, ll = 0, rr = 0, rb = 0, rl = 0, pos, step;
				for (pos = qend - kmer, step = 1; pos >= 0; --pos, ++step) {
					const int64_t te = best_te - (int64_t)(kmer - 1 + step) * 3;
					if (te - 2 < 0) break;
					lr += mat[aa_at(packed, codon, c, te) * asize + q[pos]];
					if (lr > lb) lb = lr, ll = step;
					if (lb - lr > xdrop) break;
				}
				for (pos = qend + 1, step = 1; pos < c->query_length; ++pos, ++step) {
					const int64_t te = best_te + (int64_t)step * 3;
					if (te >= c->target_length) break;
					rr += mat[aa_at(packed, codon, c, te) * asize + q[pos]];
					if (rr > rb) rb = rr, rl = step;
					if (rb - rr > xdrop) break;
				}
				sc = best_seed + lb + rb, qs = qend - (kmer - 1) - ll, qe = qend + rl;
			}
			any = 1;
			for (j = n_seg; j > 0 && seg_sc[j - 1] < sc; --j)
				seg_qs[j] = seg_qs[j - 1], seg_qe[j] = seg_qe[j - 1], seg_sc[j] = seg_sc[j - 1];
			seg_qs[j] = qs, seg_qe[j] = qe, seg_sc[j] = sc, ++n_seg;
		}
		for (i = 0; i < n_seg; ++i) {
			const int32_t len = seg_qe[i] - seg_qs[i] + 1;
			int32_t overlap = 0;
			if (i > 0 && seg_sc[i] < xdrop) break;
			for (j = 0; j < i; ++j) {
				const int32_t s = seg_qs[i] > seg_qs[j] ? seg_qs[i] : seg_qs[j];
				const int32_t e = seg_qe[i] < seg_qe[j] ? seg_qe[i] : seg_qe[j];
				if (seg_sc[j] != INT32_MIN && e >= s) overlap += e - s + 1;
			}
			if (overlap >= len) { seg_sc[i] = INT32_MIN; continue; }
			if (overlap > 0) total += (int32_t)((int64_t)seg_sc[i] * (len - overlap) / len);
			else total += seg_sc[i];
		}
		scores[ci] = any ? total : INT32_MIN;
	}
	return 1;
}
