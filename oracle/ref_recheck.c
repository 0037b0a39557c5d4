/*
 * ref_recheck.c -- ORACLE build helper (test infrastructure only).
 *
 * Compiles the reference's own recheck.c where it lies (included, never copied;
 * its main is renamed) into oracle/_ref/librecheck_ref.so and exports the
 * static pieces the checker needs: the profile reader (rc_read_prof,
 * recheck.c:120-258, which also builds the multihit-local search profile), the
 * Forward / null2 scorer rc_score (recheck.c:283-440) and a kt_for driver over
 * many peptides, the way recheck.c's worker runs it (recheck.c:546-568).
 */
#include <time.h>
#define main recheck_main
#include "recheck.c"
#undef main

/* all profiles of a HMMER3 file; returns the count (< 0 on a parse error) */
int ref_rc_load(const char *path, rc_prof_t **out)
{
	FILE *fp = fopen(path, "r");
	rc_prof_t *a = 0;
	int n = 0, m = 0, r, skipped;
	if (!fp) return -1;
	rc_init_tables();
	for (;;) {
		if (n == m) {
			m = m ? 2 * m : 16;
			a = (rc_prof_t*)realloc(a, sizeof(rc_prof_t) * (size_t)m);
		}
		r = rc_read_prof(fp, &a[n], 0, 0, &skipped);
		if (r == -1) break;
		if (r < 0) { fclose(fp); *out = a; return -2; }
		++n;
	}
	fclose(fp);
	*out = a;
	return n;
}

int32_t ref_rc_M(const rc_prof_t *p, int k) { return p[k].M; }
const float *ref_rc_msc(const rc_prof_t *p, int k) { return p[k].msc; }
const float *ref_rc_tsc(const rc_prof_t *p, int k) { return p[k].tsc; }

/* residue letters -> the codes rc_score reads (recheck.c:52-62) */
void ref_rc_encode(const char *s, int32_t n, uint8_t *dsq)
{
	int32_t j;
	rc_init_tables();
	for (j = 0; j < n; ++j) dsq[j] = rc_aa2idx[(uint8_t)s[j]];
}

void ref_rc_score(const rc_prof_t *p, int k, const uint8_t *dsq, int32_t L, int do_null2, float *bits, float *bias)
{
	rc_scratch_t sc = {0, 0};
	rc_score(&p[k], dsq, L, do_null2, &sc, bits, bias);
	free(sc.buf);
}

typedef struct {
	const rc_prof_t *prof;
	const int32_t *prof_id, *len;
	const int64_t *off;
	const uint8_t *dsq;
	int do_null2;
	rc_scratch_t *scr;
	float *bits, *bias;
} ref_rc_bench_t;

static void ref_rc_worker(void *data, long i, int tid)
{
	ref_rc_bench_t *b = (ref_rc_bench_t*)data;
	rc_score(&b->prof[b->prof_id[i]], b->dsq + b->off[i], b->len[i], b->do_null2, &b->scr[tid], &b->bits[i], &b->bias[i]);
}

/* rc_score of every peptide over kt_for; returns wall seconds */
double ref_rc_bench(int n_threads, const rc_prof_t *prof, int32_t n, const int32_t *prof_id, const uint8_t *dsq,
		const int64_t *off, const int32_t *len, int do_null2, float *bits, float *bias)
{
	ref_rc_bench_t b;
	struct timespec t0, t1;
	int t;
	b.prof = prof, b.prof_id = prof_id, b.off = off, b.len = len, b.dsq = dsq, b.do_null2 = do_null2;
	b.bits = bits, b.bias = bias;
	b.scr = (rc_scratch_t*)calloc((size_t)n_threads, sizeof(rc_scratch_t));
	clock_gettime(CLOCK_MONOTONIC, &t0);
	kt_for(n_threads, ref_rc_worker, &b, n);
	clock_gettime(CLOCK_MONOTONIC, &t1);
	for (t = 0; t < n_threads; ++t) free(b.scr[t].buf);
	free(b.scr);
	return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}
