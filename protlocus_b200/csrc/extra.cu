/*
 * extra.cu -- per-alignment statistics and exon features from the CIGAR on the
 * device (the work of align.c:148-269, mp_extra_cal): CDS length, identities,
 * positive-scoring pairs, frameshifts, in-frame stops, the alignment's own score
 * (dp_max), and one feature per exon (plus the stop codon) with its coordinates,
 * phase, per-exon counts and donor/acceptor dinucleotides -- what format.c needs
 * for the PAF tags and the GFF3 records.
 *
 * One warp per alignment.  The CIGAR is walked in order by the whole warp; inside a
 * codon-match or deletion run the lanes take the codons in turn and the counts are
 * summed with warp shuffles, so every lane holds the running totals; exon features
 * are written by lane 0 at each intron and at the end.  Every nucleotide and
 * residue read is bounds-checked against the window and the region (a CIGAR whose
 * span does not match its region is reported as such, as the reference drops its
 * features; only then can a clamped read change a count).
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include "plk.h"

extern "C" void plk_add_launches(uint64_t n);

namespace {

constexpr unsigned FULL_MASK = 0xffffffffu;
enum { OP_M = 0, OP_I = 1, OP_D = 2, OP_N = 3, OP_F = 10, OP_G = 11, OP_U = 12, OP_V = 13 };

__device__ __forceinline__ int warp_sum(int v)
{
#pragma unroll
	for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
	return v;
}

__device__ __forceinline__ int nt_at(const uint8_t *nt, int64_t l_nt, int64_t x)
{
	return x >= 0 && x < l_nt ? nt[x] : 4;
}

__device__ __forceinline__ char nt_char(int c) { return "ACGTN"[c < 4 ? c : 4]; }

__global__ void __launch_bounds__(256) k_extra(plk_extra_args_t A)
{
	const int lane = threadIdx.x & 31;
	const int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (q >= A.n) return;
	const plk_extra_job_t J = A.jobs[q];
	const uint32_t *cig = A.cigar + J.cigar_off;
	const uint8_t *nt = A.nt + J.nt_off;
	const uint8_t *aa = A.aa + J.aa_off;
	const int8_t *pssm = J.pssm_off >= 0 ? A.pssm + J.pssm_off : 0;
	const int64_t l_nt = J.l_nt;
	const int asize = A.asize;
	const int aa_lim = J.qe - J.qs;  /* residues (and pssm rows) readable from the region start */
	const uint8_t aa_ambi = A.aa20['X'], aa_stop = A.aa20['*'];
	plk_feat_t *F = A.feat + J.feat_off;

	int n_intron = 0;
	for (int k = lane; k < J.n_cigar; k += 32) {
		const int op = cig[k] & 0xf;
		n_intron += op == OP_N || op == OP_U || op == OP_V;
	}
	n_intron = warp_sum(n_intron);

	int64_t nl = 0, vs0 = J.vs;
	int al = 0, blen = 0, n_iden = 0, n_plus = 0, n_fs = 0, n_stop = 0, dp_max = 0;
	int blen0 = 0, n_iden0 = 0, score0 = 0, n_fs0 = 0, n_stop0 = 0, phase0 = 0, qs0 = J.qs, ft = 0;
	char acc0 = 0, acc1 = 0;
	for (int k = 0; k < J.n_cigar; ++k) {
		const uint32_t w = cig[k];
		const int op = w & 0xf, len = (int)(w >> 4);
		if (op == OP_M) {
			int st = 0, id = 0, pl = 0, sc = 0;
			for (int l = lane; l < len; l += 32) {
				const int64_t i = nl + 3LL * l;
				const int j = al + l;
				const int c0 = nt_at(nt, l_nt, i), c1 = nt_at(nt, l_nt, i + 1), c2 = nt_at(nt, l_nt, i + 2);
				const int nt_aa = c0 > 3 || c1 > 3 || c2 > 3 ? aa_ambi : A.codon[c0 << 4 | c1 << 2 | c2];
				const int aa_aa = j < aa_lim ? A.aa20[aa[j]] : aa_ambi;
				const int s = pssm ? (j < aa_lim ? pssm[(int64_t)j * asize + nt_aa] : 0) : A.mat[nt_aa * asize + aa_aa];
				st += nt_aa == aa_stop, id += nt_aa == aa_aa, pl += s > 0, sc += s;
			}
			n_stop += warp_sum(st), n_iden += warp_sum(id), n_plus += warp_sum(pl), dp_max += warp_sum(sc);
			nl += 3LL * len, al += len, blen += 3 * len;
		} else if (op == OP_I) {
			dp_max -= A.go + A.ge * len;
			al += len, blen += 3 * len;
		} else if (op == OP_D) { /* in-frame stop codons inside deletions count too */
			int st = 0;
			for (int l = lane; l < len; l += 32) {
				const int64_t i = nl + 3LL * l;
				const int c0 = nt_at(nt, l_nt, i), c1 = nt_at(nt, l_nt, i + 1), c2 = nt_at(nt, l_nt, i + 2);
				const int nt_aa = c0 > 3 || c1 > 3 || c2 > 3 ? aa_ambi : A.codon[c0 << 4 | c1 << 2 | c2];
				st += nt_aa == aa_stop;
			}
			n_stop += warp_sum(st);
			dp_max -= A.go + A.ge * len;
			nl += 3LL * len, blen += 3 * len;
		} else if (op == OP_F) {
			dp_max -= A.fs;
			nl += len, blen += len, ++n_fs;
		} else if (op == OP_G) {
			dp_max -= A.fs;
			nl += len, ++al, blen += 3, ++n_fs;
		} else if (op == OP_N || op == OP_U || op == OP_V) {
			if (op != OP_N) { /* the codon split by a phase-1 or phase-2 intron */
				int n1, n2, n3;
				if (op == OP_U) n1 = nt_at(nt, l_nt, nl), n2 = nt_at(nt, l_nt, nl + len - 2), n3 = nt_at(nt, l_nt, nl + len - 1);
				else n1 = nt_at(nt, l_nt, nl), n2 = nt_at(nt, l_nt, nl + 1), n3 = nt_at(nt, l_nt, nl + len - 1);
				const int nt_aa = n1 > 3 || n2 > 3 || n3 > 3 ? aa_ambi : A.codon[n1 << 4 | n2 << 2 | n3];
				const int aa_aa = al < aa_lim ? A.aa20[aa[al]] : aa_ambi;
				const int s = pssm ? (al < aa_lim ? pssm[(int64_t)al * asize + nt_aa] : 0) : A.mat[nt_aa * asize + aa_aa];
				n_stop += nt_aa == aa_stop, n_iden += nt_aa == aa_aa, n_plus += s > 0, dp_max += s;
				blen += 3;
			}
			int64_t ve;
			int64_t nvs0;
			int nphase0;
			if (op == OP_N) ve = J.vs + nl, nvs0 = J.vs + nl + len, nphase0 = 0;
			else if (op == OP_U) ve = J.vs + nl + 1, nvs0 = J.vs + nl + len - 2, nphase0 = 2;
			else ve = J.vs + nl + 2, nvs0 = J.vs + nl + len - 1, nphase0 = 1;
			if (lane == 0 && ft < J.feat_cap) {
				plk_feat_t f;
				f.vs = vs0, f.ve = ve, f.qs = qs0, f.qe = J.qs + al, f.type = 0, f.phase = (int16_t)phase0;
				f.n_fs = n_fs - n_fs0, f.n_stop = n_stop - n_stop0, f.score = dp_max - score0;
				f.n_iden = n_iden - n_iden0, f.blen = blen - blen0;
				f.donor[0] = ve - J.vs < l_nt ? nt_char(nt_at(nt, l_nt, ve - J.vs)) : '.';
				f.donor[1] = ve - J.vs + 1 < l_nt ? nt_char(nt_at(nt, l_nt, ve - J.vs + 1)) : '.';
				f.acceptor[0] = ft > 0 ? acc0 : 0, f.acceptor[1] = ft > 0 ? acc1 : 0;
				F[ft] = f;
			}
			++ft;
			vs0 = nvs0, phase0 = nphase0;
			qs0 = J.qs + al, n_fs0 = n_fs, n_stop0 = n_stop, score0 = dp_max, blen0 = blen, n_iden0 = n_iden;
			acc0 = vs0 - J.vs >= 2 ? nt_char(nt_at(nt, l_nt, vs0 - J.vs - 2)) : '.';
			acc1 = vs0 - J.vs >= 1 ? nt_char(nt_at(nt, l_nt, vs0 - J.vs - 1)) : '.';
			nl += len, al += op != OP_N;
		}
	}
	if (lane == 0) {
		if (ft < J.feat_cap) { /* the last exon */
			plk_feat_t f;
			f.vs = vs0, f.ve = J.vs + nl, f.qs = qs0, f.qe = J.qs + al, f.type = 0, f.phase = (int16_t)phase0;
			f.n_fs = n_fs - n_fs0, f.n_stop = n_stop - n_stop0, f.score = dp_max - score0;
			f.n_iden = n_iden - n_iden0, f.blen = blen - blen0;
			f.donor[0] = f.donor[1] = 0;
			f.acceptor[0] = ft > 0 ? acc0 : 0, f.acceptor[1] = ft > 0 ? acc1 : 0;
			F[ft] = f;
		}
		++ft;
		if (J.has_stop) {
			if (ft < J.feat_cap) {
				plk_feat_t f;
				const int64_t ve_mrna = J.ve + 3;
				f.vs = ve_mrna - 3, f.ve = ve_mrna, f.qs = f.qe = J.qe + al, f.type = 1, f.phase = 0;
				f.n_fs = 0, f.n_stop = 0, f.score = 0, f.n_iden = 0, f.blen = 3;
				f.donor[0] = f.donor[1] = f.acceptor[0] = f.acceptor[1] = 0;
				F[ft] = f;
			}
			++ft;
		}
		plk_extra_res_t r;
		r.blen = blen, r.n_iden = n_iden, r.n_plus = n_plus, r.n_fs = n_fs, r.n_stop = n_stop, r.dp_max = dp_max;
		r.n_exon = n_intron + 1, r.n_feat = ft;
		r.ok = nl == J.ve - J.vs && al == J.qe - J.qs && ft <= J.feat_cap;
		r.pad = 0;
		A.res[q] = r;
	}
}

}  // namespace

extern "C" int plk_extra(const plk_extra_args_t *a, void *stream)
{
	if (a->n <= 0) return 0;
	const int64_t threads = a->n * 32;
	k_extra<<<(unsigned)((threads + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*a);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}
