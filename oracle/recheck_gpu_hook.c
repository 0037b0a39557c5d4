/*
 * recheck_gpu_hook.c -- the reference's recheck program (protlocus-recheck) scoring its
 * peptides through libplgpu's Forward (pl_rc_score_host) instead of its thread pool.
 *
 * rc_score is static in recheck.c, so the integration replaces the scoring loop: this
 * file is included into a copy of recheck.c right before main, and main's
 * `kt_for(n_threads, worker, &d, d.n_pep);` (recheck.c:727) becomes
 * `pl_recheck_gpu(&d);` (oracle/Makefile, target progs -> oracle/_ref/protlocus_recheck_gpu;
 * test infrastructure for tests/test_gpu_program.py: the product is libplgpu, this is its
 * caller).  Every peptide the worker would score (a profile bound, a non-empty sequence)
 * goes into one batch: its residue codes (recheck's own table, recheck.c:52-62), its
 * profile, the null2 switch.  The bits and the bias come back from the device; the
 * E-value and the done flag are set exactly as worker() sets them (recheck.c:546-567).
 * A device failure ends the program with an error: nothing is scored on the CPU.
 */
#include "plgpu.h"

static void pl_recheck_gpu(rc_data_t *d)
{
	pl_engine_t *e = pl_engine_create(0, 0);
	pl_rc_profile_t **gp = (pl_rc_profile_t**)calloc(d->n_prof > 0 ? d->n_prof : 1, sizeof(*gp));
	int32_t *pid = 0, *len = 0, n = 0, k;
	int64_t *off = 0, *which = 0, n_res = 0, i, j;
	uint8_t *dsq = 0;
	float *bits = 0, *bias = 0;
	int ok = e && gp;
	for (k = 0; ok && k < d->n_prof; ++k)
		ok = (gp[k] = pl_rc_profile_create(0, d->prof[k].M, d->prof[k].msc, d->prof[k].tsc)) != 0;
	for (i = 0; i < d->n_pep; ++i)
		if (d->pep[i].prof_id >= 0 && d->pep[i].len > 0) ++n, n_res += d->pep[i].len;
	if (ok && n > 0) {
		pid = (int32_t*)malloc(n * sizeof(int32_t)), len = (int32_t*)malloc(n * sizeof(int32_t));
		off = (int64_t*)malloc(n * sizeof(int64_t)), which = (int64_t*)malloc(n * sizeof(int64_t));
		dsq = (uint8_t*)malloc(n_res), bits = (float*)malloc(n * sizeof(float)), bias = (float*)malloc(n * sizeof(float));
		ok = pid && len && off && which && dsq && bits && bias;
	}
	if (ok && n > 0) {
		int64_t o = 0;
		for (i = 0, k = 0; i < d->n_pep; ++i) {
			const rc_pep_t *p = &d->pep[i];
			if (p->prof_id < 0 || p->len == 0) continue;
			for (j = 0; j < p->len; ++j) dsq[o + j] = rc_aa2idx[(uint8_t)p->seq[j]];
			pid[k] = p->prof_id, len[k] = p->len, off[k] = o, which[k] = i, o += p->len, ++k;
		}
		ok = pl_rc_score_host(e, (const pl_rc_profile_t *const*)gp, d->n_prof, n, pid, dsq, n_res, off, len,
				!d->no_null2, bits, bias);
	}
	if (!ok) {
		fprintf(stderr, "[recheck] ERROR: GPU scoring failed: %s\n", pl_last_error());
		exit(1);
	}
	for (i = 0; i < d->n_pep; ++i) d->pep[i].done = 0;
	for (k = 0; k < n; ++k) {
		rc_pep_t *p = &d->pep[which[k]];
		const rc_prof_t *pr = &d->prof[p->prof_id];
		p->bits = bits[k];
		p->bias_bits = bias[k];
		if (pr->has_stats) {
			double pv = bits[k] >= pr->ftau ? exp(-(double)pr->flambda * (bits[k] - pr->ftau)) : 1.0;
			double ev = pv * d->Z;
			p->evalue = (float)(ev < d->Z ? ev : d->Z);
		} else p->evalue = NAN;
		p->done = 1;
	}
	for (k = 0; k < d->n_prof; ++k) pl_rc_profile_destroy(gp[k]);
	pl_engine_destroy(e);
	free(gp), free(pid), free(len), free(off), free(which), free(dsq), free(bits), free(bias);
}
