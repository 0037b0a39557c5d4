/*
 * ref_shim.c -- ORACLE build helper (test infrastructure only).
 *
 * Linked into oracle/_ref/libnsref.so next to the reference's own hmm.c.  hmm.c's
 * batch wrapper (hmm.c:319-335) calls mp_set_rank_score() from hit.c, which drags in
 * the whole candidate-ranking layer; the oracle only needs mp_hmm_dp_score(), so a
 * no-op stand-in resolves the symbol.
 */
struct mp_mapopt_s_opaque;
struct mp_reg1_s_opaque;
void mp_set_rank_score(const struct mp_mapopt_s_opaque *opt, int qlen, struct mp_reg1_s_opaque *r)
{
	(void)opt, (void)qlen, (void)r;
}

/* ns_global_gs_auto() (nasw-sse.c:984-986) offers NS_F_GPU jobs to ns_gpu_global() first; in the
 * CPU oracle no device exists, so the offer is always declined and the CPU kernels run. */
int ns_gpu_global(void *km, const char *ns, int nl, const char *as, int al, const void *opt,
		const unsigned char *ss, void *r)
{
	(void)km, (void)ns, (void)nl, (void)as, (void)al, (void)opt, (void)ss, (void)r;
	return 0;
}
