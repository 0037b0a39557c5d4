/*
 * plseed.c -- host layer of the coarse mapper's seeding on the device (the sketch and
 * anchor stages of mp_map_coarse, map.c:565-572, default mode; seed.cu).
 *
 * The index is the mapper's own (mp_idx_t's ki / kb, index.c:74-98), uploaded once with
 * pl_seed_index_create.  A batch takes proteins (letters or residue codes 0-21) and
 * returns, per protein, its anchors (block << 32 | position) sorted ascending, as
 * mp_collect_anchors and the following radix sort leave them, with the accuracy mode's
 * repeat rescue (map.c:360-384) when asked (pl_seed_anchors_opt_host), and for
 * HMM-profile queries (pl_seed_anchors_hmm_host: the profile-derived seeds of
 * mp_sketch_hmm merged with the query's own, map.c:332-343).
 */
#define _POSIX_C_SOURCE 200809L
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include "plhost.h"
#include "seed_hmm.cuh"

struct pl_seed_index_s {
	int device;
	int32_t kmer, mod_bit;
	int64_t n_bucket, n_kb;
	int64_t *ki;
	uint32_t *kb;
};

PL_EXPORT pl_seed_index_t *pl_seed_index_create(int32_t device, const int64_t *ki, int64_t n_bucket, const uint32_t *kb,
		int64_t n_kb, int32_t kmer, int32_t mod_bit)
{
	pl_seed_index_t *x;
	/* kmer 8 would need the 32-bit shift 1U << 32 for the k-mer mask, which C leaves undefined
	 * (sketch.c:21): the reference's mask then depends on its compiler, so it is refused */
	if (kmer < 1 || kmer > 7 || mod_bit < 0 || mod_bit >= kmer * 4 || n_bucket != (int64_t)1 << (kmer * 4 - mod_bit) ||
			n_kb < 0 || n_kb > (int64_t)UINT32_MAX || !ki || (n_kb > 0 && !kb)) {
		pl_set_error("seed index: kmer %d, mod_bit %d, %lld buckets, %lld entries (kmer 1-7, 1 << (4 kmer - mod_bit) buckets)",
				kmer, mod_bit, (long long)n_bucket, (long long)n_kb);
		return 0;
	}
	x = (pl_seed_index_t*)calloc(1, sizeof(*x));
	if (!x) { pl_set_error("out of host memory"); return 0; }
	x->device = device, x->kmer = kmer, x->mod_bit = mod_bit, x->n_bucket = n_bucket, x->n_kb = n_kb;
	CK(cudaSetDevice(device));
	CK(cudaMalloc((void**)&x->ki, sizeof(int64_t) * (size_t)n_bucket));
	CK(cudaMalloc((void**)&x->kb, sizeof(uint32_t) * (size_t)(n_kb > 0 ? n_kb : 1)));
	CK(cudaMemcpy(x->ki, ki, sizeof(int64_t) * (size_t)n_bucket, cudaMemcpyHostToDevice));
	if (n_kb > 0) CK(cudaMemcpy(x->kb, kb, sizeof(uint32_t) * (size_t)n_kb, cudaMemcpyHostToDevice));
	return x;
fail:
	if (x->ki) cudaFree(x->ki);
	if (x->kb) cudaFree(x->kb);
	free(x);
	return 0;
}

PL_EXPORT void pl_seed_index_destroy(pl_seed_index_t *x)
{
	if (!x) return;
	cudaSetDevice(x->device);
	cudaFree(x->ki), cudaFree(x->kb);
	free(x);
}

void pl_seed_engine_free(pl_engine_t *e)
{
	dbuf_free(&e->s_seq), dbuf_free(&e->s_off), dbuf_free(&e->s_len), dbuf_free(&e->s_seed), dbuf_free(&e->s_cnt);
	dbuf_free(&e->s_nseed), dbuf_free(&e->s_cap), dbuf_free(&e->s_nanc), dbuf_free(&e->s_aoff);
	dbuf_free(&e->s_anc), dbuf_free(&e->s_anc2), dbuf_free(&e->s_tmp);
	dbuf_free(&e->s_take), dbuf_free(&e->s_send), dbuf_free(&e->s_seed2), dbuf_free(&e->s_qh);
	dbuf_free(&e->s_soff), dbuf_free(&e->s_emit), dbuf_free(&e->s_eoff), dbuf_free(&e->s_elen), dbuf_free(&e->s_alts);
}

PL_EXPORT uint32_t pl_seed_qname_hash(const char *qname)
{ /* mp_hash_qname (map.c:322-329): FNV-1a over the name's bytes */
	uint32_t h = 2166136261U;
	if (!qname) return h;
	for (; *qname; ++qname) h = (h ^ (uint8_t)*qname) * 16777619U;
	return h;
}

/* the seed slots of an HMM-profile batch: protein q's from soff[q], its own seeds (at most
 * len[q]) and at most min(seed_max, 4^kmer) per window of its profile (a window has no
 * more distinct k-mers); soff[n] the total, or -1 with the error set */
static int64_t pl_seed_hmm_slots(int32_t n, const int32_t *len, const pl_seed_hmm_t *h, int32_t kmer, int64_t *soff)
{
	const int64_t per_win = h->seed_max < ((int64_t)1 << (2 * kmer)) ? h->seed_max : (int64_t)1 << (2 * kmer);
	int64_t t = 0;
	int32_t q;
	for (q = 0; q < n; ++q) {
		if (h->e_len[q] < 0 || h->e_off[q] < 0 || h->e_off[q] + h->e_len[q] > h->n_state) {
			pl_set_error("protein %d: profile of %d states at %lld of %lld", q, h->e_len[q], (long long)h->e_off[q],
					(long long)h->n_state);
			return -1;
		}
		soff[q] = t;
		t += len[q] + (h->e_len[q] >= kmer ? (int64_t)(h->e_len[q] - kmer + 1) * per_win : 0);
		if (t > INT32_MAX) {  /* the segmented sorts count items in an int */
			pl_set_error("seed batch with room for %lld seeds at protein %d: at most %d per call, split the batch",
					(long long)t, q, INT32_MAX);
			return -1;
		}
	}
	soff[n] = t;
	return t;
}

/* the batch's anchors: into the host array a (when they fit a_cap), or left on the device
 * (a_dev != 0: *a_dev at the engine's sorted array); h with seed_max > 0: HMM-profile queries */
static int64_t pl_seed_run(pl_engine_t *e, const pl_seed_index_t *x, int32_t n, const uint8_t *seq, int64_t seq_len,
		const int64_t *off, const int32_t *len, const pl_seed_opt_t *o, const pl_seed_hmm_t *h, int64_t *a_off,
		uint64_t *a, int64_t a_cap, const uint64_t **a_dev)
{
	const int rescue = o && o->repeat_cap > 0, hmm = h && h->seed_max > 0;
	const int32_t max_occ = o ? o->max_occ : 0;
	plk_seed_args_t A;
	int64_t *na = 0, *soff = 0, total = 0, ret = -1, n_slot;
	int32_t q;
	size_t tmp_bytes = 0;
	cudaStream_t st;
	if (!e || !x) { pl_set_error("no engine or index"); return -1; }
	if (x->device != e->device) { pl_set_error("seed index on device %d, engine on %d", x->device, e->device); return -1; }
	if (n < 0 || !o || !a_off || (n > 0 && (!seq || !off || !len)) || (rescue && (o->anchor_budget < 0 || !o->qname_hash)) ||
			(hmm && (h->n_state < 0 || (h->n_state > 0 && !h->emit) || (n > 0 && (!h->e_off || !h->e_len))))) {
		pl_set_error("seed batch: bad arguments");
		return -1;
	}
	a_off[0] = 0;
	if (n == 0) return 0;
	if (seq_len > INT32_MAX) {  /* the segmented sorts count items in an int */
		pl_set_error("seed batch of %lld residues: at most %d per call", (long long)seq_len, INT32_MAX);
		return -1;
	}
	for (q = 0; q < n; ++q)
		if (len[q] < 0 || off[q] < 0 || off[q] + len[q] > seq_len) {
			pl_set_error("protein %d: length %d at %lld of %lld", q, len[q], (long long)off[q], (long long)seq_len);
			return -1;
		}
	n_slot = seq_len;
	if (hmm) {
		soff = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
		if (!soff) { pl_set_error("out of host memory"); return -1; }
		if ((n_slot = pl_seed_hmm_slots(n, len, h, x->kmer, soff)) < 0) { free(soff); return -1; }
	}
	st = e->stream;
	CK(cudaSetDevice(e->device));
	na = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
	if (!na) { pl_set_error("out of host memory"); free(soff); return -1; }
	if (!dbuf_ensure(&e->s_seq, (size_t)(seq_len > 0 ? seq_len : 1)) || !dbuf_ensure(&e->s_off, sizeof(int64_t) * (size_t)n) ||
			!dbuf_ensure(&e->s_len, sizeof(int32_t) * (size_t)n) ||
			!dbuf_ensure(&e->s_seed, sizeof(uint64_t) * (size_t)(n_slot > 0 ? n_slot : 1)) ||
			!dbuf_ensure(&e->s_cnt, sizeof(uint32_t) * (size_t)(n_slot > 0 ? n_slot : 1)) ||
			!dbuf_ensure(&e->s_nseed, sizeof(int32_t) * (size_t)n) || !dbuf_ensure(&e->s_cap, sizeof(int32_t) * (size_t)n) ||
			!dbuf_ensure(&e->s_nanc, sizeof(int64_t) * (size_t)n) || !dbuf_ensure(&e->s_aoff, sizeof(int64_t) * (size_t)(n + 1)) ||
			!dbuf_ensure(&e->s_take, sizeof(int32_t) * (size_t)(n_slot > 0 ? n_slot : 1)) ||
			!dbuf_ensure(&e->s_send, sizeof(int64_t) * (size_t)n) ||
			((rescue || hmm) && !dbuf_ensure(&e->s_seed2, sizeof(uint64_t) * (size_t)(n_slot > 0 ? n_slot : 1))) ||
			(rescue && !dbuf_ensure(&e->s_qh, sizeof(uint32_t) * (size_t)n)) ||
			(hmm && (!dbuf_ensure(&e->s_soff, sizeof(int64_t) * (size_t)(n + 1)) ||
			         !dbuf_ensure(&e->s_emit, sizeof(int16_t) * 20 * (size_t)(h->n_state > 0 ? h->n_state : 1)) ||
			         !dbuf_ensure(&e->s_eoff, sizeof(int64_t) * (size_t)n) || !dbuf_ensure(&e->s_elen, sizeof(int32_t) * (size_t)n) ||
			         !dbuf_ensure(&e->s_alts, sizeof(sh_alts_t) * (size_t)(h->n_state > 0 ? h->n_state : 1)))))
		goto fail;
	if (seq_len > 0) CK(cudaMemcpyAsync(e->s_seq.p, seq, (size_t)seq_len, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->s_off.p, off, sizeof(int64_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	CK(cudaMemcpyAsync(e->s_len.p, len, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
	memset(&A, 0, sizeof(A));
	A.seq = (const uint8_t*)e->s_seq.p, A.off = (const int64_t*)e->s_off.p, A.len = (const int32_t*)e->s_len.p, A.n = n;
	A.soff = A.off;  /* the default slots: one per residue */
	if (hmm) {
		CK(cudaMemcpyAsync(e->s_soff.p, soff, sizeof(int64_t) * (size_t)(n + 1), cudaMemcpyHostToDevice, st));
		if (h->n_state > 0)
			CK(cudaMemcpyAsync(e->s_emit.p, h->emit, sizeof(int16_t) * 20 * (size_t)h->n_state, cudaMemcpyHostToDevice, st));
		CK(cudaMemcpyAsync(e->s_eoff.p, h->e_off, sizeof(int64_t) * (size_t)n, cudaMemcpyHostToDevice, st));
		CK(cudaMemcpyAsync(e->s_elen.p, h->e_len, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
		A.soff = (const int64_t*)e->s_soff.p;
		A.emit = (const int16_t*)e->s_emit.p, A.n_state = h->n_state;
		A.e_off = (const int64_t*)e->s_eoff.p, A.e_len = (const int32_t*)e->s_elen.p, A.alts = e->s_alts.p;
		A.pos_loss = h->pos_loss, A.win_loss = h->win_loss, A.seed_max = h->seed_max;
	}
	A.ki = x->ki, A.n_bucket = x->n_bucket, A.kb = x->kb, A.n_kb = x->n_kb;
	A.kmer = x->kmer, A.mod_bit = x->mod_bit, A.max_occ = max_occ;
	A.repeat_cap = rescue ? o->repeat_cap : 0, A.budget = rescue ? o->anchor_budget : 0;
	A.seeds = (uint64_t*)e->s_seed.p, A.cnt = (uint32_t*)e->s_cnt.p, A.take = (int32_t*)e->s_take.p;
	A.n_seed = (int32_t*)e->s_nseed.p, A.cap = (int32_t*)e->s_cap.p, A.n_anchor = (int64_t*)e->s_nanc.p;
	A.seed_end = (int64_t*)e->s_send.p;
	if (rescue) {
		CK(cudaMemcpyAsync(e->s_qh.p, o->qname_hash, sizeof(uint32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
		A.qhash = (const uint32_t*)e->s_qh.p;
	}
	e->n_ev = 0;
	PL_TIME(e, st, 1);
	if (hmm) CKK(plk_seed_hmm_alts(&A, st));
	CKK(plk_seed_sketch(&A, st));
	if (hmm) {  /* the profile's seeds after the query's own, then sorted without duplicates */
		size_t tb = 0;
		CKK(plk_seed_hmm_enum(&A, st));
		CKK(plk_seed_sort((const uint64_t*)e->s_seed.p, (uint64_t*)e->s_seed2.p, n_slot, n, A.soff,
				(const int64_t*)e->s_send.p, 0, &tb, st));
		if (!dbuf_ensure(&e->s_tmp, tb > 0 ? tb : 16)) goto fail;
		CKK(plk_seed_sort((const uint64_t*)e->s_seed.p, (uint64_t*)e->s_seed2.p, n_slot, n, A.soff,
				(const int64_t*)e->s_send.p, e->s_tmp.p, &tb, st));
		CKK(plk_seed_unique(&A, (const uint64_t*)e->s_seed2.p, st));
	} else if (rescue) { /* the rescue hands its budget out over the seeds in mp_sketch_query's sorted order */
		size_t tb = 0;
		CKK(plk_seed_sort((const uint64_t*)e->s_seed.p, (uint64_t*)e->s_seed2.p, seq_len, n, (const int64_t*)e->s_off.p,
				(const int64_t*)e->s_send.p, 0, &tb, st));
		if (!dbuf_ensure(&e->s_tmp, tb > 0 ? tb : 16)) goto fail;
		CKK(plk_seed_sort((const uint64_t*)e->s_seed.p, (uint64_t*)e->s_seed2.p, seq_len, n, (const int64_t*)e->s_off.p,
				(const int64_t*)e->s_send.p, e->s_tmp.p, &tb, st));
		A.seeds = (uint64_t*)e->s_seed2.p;
	}
	CKK(plk_seed_take(&A, st));
	PL_TIME(e, st, 1);
	CK(cudaMemcpyAsync(na, e->s_nanc.p, sizeof(int64_t) * (size_t)n, cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
	for (q = 0; q < n; ++q) total += na[q], a_off[q + 1] = total;
	if (total > INT32_MAX) {  /* the anchors' segmented sort counts items in an int */
		pl_set_error("seed batch with %lld anchors: at most %d per call, split the batch", (long long)total, INT32_MAX);
		goto fail;
	}
	ret = total;
	if (a_dev) *a_dev = 0;
	if (total == 0 || (!a_dev && total > a_cap)) goto done;  /* a_off only: the caller grows a to a_off[n] */
	if (!dbuf_ensure(&e->s_anc, sizeof(uint64_t) * (size_t)total) || !dbuf_ensure(&e->s_anc2, sizeof(uint64_t) * (size_t)total))
		goto fail;
	CK(cudaMemcpyAsync(e->s_aoff.p, a_off, sizeof(int64_t) * (size_t)(n + 1), cudaMemcpyHostToDevice, st));
	A.a_off = (const int64_t*)e->s_aoff.p, A.anchors = (uint64_t*)e->s_anc.p;
	PL_TIME(e, st, 1);
	CKK(plk_seed_emit(&A, st));
	CKK(plk_seed_sort((const uint64_t*)e->s_anc.p, (uint64_t*)e->s_anc2.p, total, n, (const int64_t*)e->s_aoff.p, 0, 0,
			&tmp_bytes, st));
	if (!dbuf_ensure(&e->s_tmp, tmp_bytes > 0 ? tmp_bytes : 16)) goto fail;
	CKK(plk_seed_sort((const uint64_t*)e->s_anc.p, (uint64_t*)e->s_anc2.p, total, n, (const int64_t*)e->s_aoff.p, 0,
			e->s_tmp.p, &tmp_bytes, st));
	PL_TIME(e, st, 1);
	if (a_dev) *a_dev = (const uint64_t*)e->s_anc2.p;
	else CK(cudaMemcpyAsync(a, e->s_anc2.p, sizeof(uint64_t) * (size_t)total, cudaMemcpyDeviceToHost, st));
	CK(cudaStreamSynchronize(st));
done:
	if (e->timing) {  /* the sketch, and the emission with the sort */
		int k;
		float ms;
		for (k = 0; k + 1 < e->n_ev; k += 2) {
			cudaEventElapsedTime(&ms, e->ev[k], e->ev[k + 1]);
			e->acc_ms[e->ev_kind[k]] += ms;
		}
		e->acc_dp_launches += e->n_ev / 2;
	}
	free(na), free(soff);
	return ret;
fail:
	free(na), free(soff);
	return -1;
}

PL_EXPORT int64_t pl_seed_anchors_opt_host(pl_engine_t *e, const pl_seed_index_t *x, int32_t n, const uint8_t *seq,
		int64_t seq_len, const int64_t *off, const int32_t *len, const pl_seed_opt_t *o, int64_t *a_off, uint64_t *a,
		int64_t a_cap)
{
	return pl_seed_run(e, x, n, seq, seq_len, off, len, o, 0, a_off, a, a_cap, 0);
}

PL_EXPORT int64_t pl_seed_anchors_opt_device(pl_engine_t *e, const pl_seed_index_t *x, int32_t n, const uint8_t *seq,
		int64_t seq_len, const int64_t *off, const int32_t *len, const pl_seed_opt_t *o, int64_t *a_off,
		const uint64_t **a_dev)
{
	if (!a_dev) { pl_set_error("seed batch: no output pointer"); return -1; }
	return pl_seed_run(e, x, n, seq, seq_len, off, len, o, 0, a_off, 0, 0, a_dev);
}

PL_EXPORT int64_t pl_seed_anchors_hmm_host(pl_engine_t *e, const pl_seed_index_t *x, int32_t n, const uint8_t *seq,
		int64_t seq_len, const int64_t *off, const int32_t *len, const pl_seed_opt_t *o, const pl_seed_hmm_t *h,
		int64_t *a_off, uint64_t *a, int64_t a_cap)
{
	if (!h) { pl_set_error("seed batch: no profiles"); return -1; }
	return pl_seed_run(e, x, n, seq, seq_len, off, len, o, h, a_off, a, a_cap, 0);
}

PL_EXPORT int64_t pl_seed_anchors_hmm_device(pl_engine_t *e, const pl_seed_index_t *x, int32_t n, const uint8_t *seq,
		int64_t seq_len, const int64_t *off, const int32_t *len, const pl_seed_opt_t *o, const pl_seed_hmm_t *h,
		int64_t *a_off, const uint64_t **a_dev)
{
	if (!h || !a_dev) { pl_set_error("seed batch: no profiles or no output pointer"); return -1; }
	return pl_seed_run(e, x, n, seq, seq_len, off, len, o, h, a_off, 0, 0, a_dev);
}

PL_EXPORT int64_t pl_seed_anchors_host(pl_engine_t *e, const pl_seed_index_t *x, int32_t n, const uint8_t *seq,
		int64_t seq_len, const int64_t *off, const int32_t *len, int32_t max_occ, int64_t *a_off, uint64_t *a,
		int64_t a_cap)
{
	pl_seed_opt_t o;
	memset(&o, 0, sizeof(o));
	o.max_occ = max_occ;
	return pl_seed_anchors_opt_host(e, x, n, seq, seq_len, off, len, &o, a_off, a, a_cap);
}
