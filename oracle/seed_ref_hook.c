/*
 * seed_ref_hook.c -- test infrastructure: appended to a copy of the reference's map.c
 * (oracle/Makefile, target seedref -> oracle/_ref/libseed_ref.so) so that its static
 * seeding steps can be called on a given index: mp_sketch_query (map.c:332-343),
 * mp_cal_max_occ (map.c:304-320), mp_collect_anchors (map.c:346-397) and the anchor
 * sort (map.c:571), as mp_map_coarse strings them together (map.c:565-572) in the
 * default mode (options from mp_mapopt_init), with the accuracy mode's repeat rescue,
 * and for HMM-profile queries (the profile read by hmm.c's parser, its consensus the
 * query, mp_sketch_hmm's profile-derived seeds merged in).  The checker of
 * oracle/seed_port.c and of the device seeding.
 */
__attribute__((visibility("default")))
int64_t ref_seed_anchors(const int64_t *ki, const uint32_t *kb, int64_t n_kb, int32_t kmer, int32_t mod_bit,
		int32_t max_occ_opt, const char *seq, int32_t len, uint64_t **out)
{
	mp_idx_t mi;
	mp_mapopt_t opt;
	mp64_v sd = {0, 0, 0};
	int32_t max_occ;
	int64_t n_a = 0, n_rescued = 0;
	memset(&mi, 0, sizeof(mi));
	mp_idxopt_init(&mi.opt);
	mi.opt.kmer = kmer, mi.opt.mod_bit = mod_bit;
	mi.ki = (int64_t*)ki, mi.kb = (uint32_t*)kb, mi.n_kb = n_kb;
	mp_mapopt_init(&opt);
	opt.max_occ = max_occ_opt;
	mp_sketch_query(0, &opt, seq, len, kmer, mod_bit, opt.hmm_seed_max, &sd);
	if (sd.n >= 8) {
		max_occ = mp_cal_max_occ(0, &mi, sd.n, sd.a);
		if (max_occ > opt.max_occ) max_occ = opt.max_occ;
	} else max_occ = opt.max_occ;
	*out = mp_collect_anchors(0, &mi, &opt, &sd, max_occ, "q", &n_a, &n_rescued);
	kfree(0, sd.a);
	radix_sort_mp64(*out, *out + n_a);
	return n_a;
}

__attribute__((visibility("default"))) void ref_seed_free(void *p) { kfree(0, p); }

/* the same with the accuracy mode's repeat rescue (map.c:360-384): repeat_cap blocks at
 * most per over-cap bucket, anchor_budget in all, qname for the round-robin start */
__attribute__((visibility("default")))
int64_t ref_seed_anchors_acc(const int64_t *ki, const uint32_t *kb, int64_t n_kb, int32_t kmer, int32_t mod_bit,
		int32_t max_occ_opt, int32_t repeat_cap, int64_t anchor_budget, const char *qname, const char *seq,
		int32_t len, uint64_t **out)
{
	mp_idx_t mi;
	mp_mapopt_t opt;
	mp64_v sd = {0, 0, 0};
	int32_t max_occ;
	int64_t n_a = 0, n_rescued = 0;
	memset(&mi, 0, sizeof(mi));
	mp_idxopt_init(&mi.opt);
	mi.opt.kmer = kmer, mi.opt.mod_bit = mod_bit;
	mi.ki = (int64_t*)ki, mi.kb = (uint32_t*)kb, mi.n_kb = n_kb;
	mp_mapopt_init(&opt);
	opt.max_occ = max_occ_opt;
	opt.flag |= MP_F_ACCURACY, opt.acc_flags |= MP_ACC_REPEAT_RESCUE;
	opt.acc_repeat_cap = repeat_cap, opt.acc_anchor_budget = anchor_budget;
	mp_sketch_query(0, &opt, seq, len, kmer, mod_bit, opt.hmm_seed_max, &sd);
	if (sd.n >= 8) {
		max_occ = mp_cal_max_occ(0, &mi, sd.n, sd.a);
		if (max_occ > opt.max_occ) max_occ = opt.max_occ;
	} else max_occ = opt.max_occ;
	*out = mp_collect_anchors(0, &mi, &opt, &sd, max_occ, qname, &n_a, &n_rescued);
	kfree(0, sd.a);
	radix_sort_mp64(*out, *out + n_a);
	return n_a;
}

__attribute__((visibility("default"))) uint32_t ref_seed_qname_hash(const char *qname) { return mp_hash_qname(qname); }

/* ---- HMM-profile queries: the profile-derived seeds (sketch.c:40-118) ---- */

/* mp_sketch_hmm on a given emission table (len x 20, HMMER column order), appended to an
 * empty seed array as the reference leaves it (unsorted); returns the number of seeds */
__attribute__((visibility("default")))
int64_t ref_sketch_hmm(const int16_t *emit, int32_t len, int32_t kmer, int32_t mod_bit, int32_t pos_loss,
		int32_t win_loss, int32_t max_per_win, uint64_t **out)
{
	mp64_v sd = {0, 0, 0};
	mp_sketch_hmm(0, emit, len, kmer, mod_bit, pos_loss, win_loss, max_per_win, &sd);
	*out = sd.a;
	return sd.n;
}

/* a profile read by the reference's parser (hmm.c:112-195), its consensus the query and
 * its name the query name, as mp_map_hmm_file runs it (map.c:1184-1196): the seeds of
 * mp_sketch_query (consensus and profile-derived, sorted and deduplicated, map.c:332-343)
 * when ki is NULL, else the anchors of mp_map_coarse's seeding steps (map.c:565-572), with
 * the accuracy mode's repeat rescue when repeat_cap > 0 */
static int64_t ref_hmm_seed_steps(mp_hmm_t *h, const int64_t *ki, const uint32_t *kb, int64_t n_kb, int32_t kmer,
		int32_t mod_bit, int32_t max_occ_opt, int32_t repeat_cap, int64_t anchor_budget, int32_t pos_loss,
		int32_t win_loss, int32_t seed_max, uint64_t **out)
{
	mp_idx_t mi;
	mp_mapopt_t opt;
	mp64_v sd = {0, 0, 0};
	const char *cons = mp_hmm_consensus(h);
	int32_t max_occ, qlen = mp_hmm_length(h);
	int64_t n_a = 0, n_rescued = 0;
	mp_mapopt_init(&opt);
	opt.hmm = h, opt.max_occ = max_occ_opt;
	opt.hmm_seed_pos_loss = pos_loss, opt.hmm_seed_win_loss = win_loss;
	if (repeat_cap > 0) {
		opt.flag |= MP_F_ACCURACY, opt.acc_flags |= MP_ACC_REPEAT_RESCUE;
		opt.acc_repeat_cap = repeat_cap, opt.acc_anchor_budget = anchor_budget;
	}
	mp_sketch_query(0, &opt, cons, qlen, kmer, mod_bit, seed_max, &sd);
	if (!ki) {
		*out = sd.a;
		return sd.n;
	}
	memset(&mi, 0, sizeof(mi));
	mp_idxopt_init(&mi.opt);
	mi.opt.kmer = kmer, mi.opt.mod_bit = mod_bit;
	mi.ki = (int64_t*)ki, mi.kb = (uint32_t*)kb, mi.n_kb = n_kb;
	if (sd.n >= 8) {
		max_occ = mp_cal_max_occ(0, &mi, sd.n, sd.a);
		if (max_occ > opt.max_occ) max_occ = opt.max_occ;
	} else max_occ = opt.max_occ;
	*out = mp_collect_anchors(0, &mi, &opt, &sd, max_occ, mp_hmm_name(h), &n_a, &n_rescued);
	kfree(0, sd.a);
	radix_sort_mp64(*out, *out + n_a);
	return n_a;
}

/* the same on an HMMER3 file, read for this call */
__attribute__((visibility("default")))
int64_t ref_seed_hmm_query(const char *hmm_path, const int64_t *ki, const uint32_t *kb, int64_t n_kb, int32_t kmer,
		int32_t mod_bit, int32_t max_occ_opt, int32_t repeat_cap, int64_t anchor_budget, int32_t pos_loss,
		int32_t win_loss, int32_t seed_max, uint64_t **out)
{
	mp_hmm_t *h = mp_hmm_read(hmm_path);
	int64_t n;
	*out = 0;
	if (!h) return -1;
	n = ref_hmm_seed_steps(h, ki, kb, n_kb, kmer, mod_bit, max_occ_opt, repeat_cap, anchor_budget, pos_loss, win_loss,
			seed_max, out);
	mp_hmm_destroy(h);
	return n;
}

/* a profile read once (ref_hmm_load) and seeded many times (ref_seed_hmm_run), for timing
 * the reference's seeding without its parser */
__attribute__((visibility("default"))) void *ref_hmm_load(const char *hmm_path) { return mp_hmm_read(hmm_path); }
__attribute__((visibility("default"))) void ref_hmm_free(void *h) { mp_hmm_destroy((mp_hmm_t*)h); }
__attribute__((visibility("default")))
int64_t ref_seed_hmm_run(void *h, const int64_t *ki, const uint32_t *kb, int64_t n_kb, int32_t kmer, int32_t mod_bit,
		int32_t max_occ_opt, int32_t pos_loss, int32_t win_loss, int32_t seed_max, uint64_t **out)
{
	*out = 0;
	if (!h) return -1;
	return ref_hmm_seed_steps((mp_hmm_t*)h, ki, kb, n_kb, kmer, mod_bit, max_occ_opt, 0, 0, pos_loss, win_loss,
			seed_max, out);
}

/* the consensus the reference's parser derives (hmm.c:181-189), len + 1 bytes with the 0 */
__attribute__((visibility("default")))
int32_t ref_hmm_consensus(const char *hmm_path, char *out, int32_t cap)
{
	mp_hmm_t *h = mp_hmm_read(hmm_path);
	int32_t len;
	if (!h) return -1;
	len = mp_hmm_length(h);
	if (len + 1 <= cap) memcpy(out, mp_hmm_consensus(h), (size_t)len + 1);
	mp_hmm_destroy(h);
	return len;
}

/* the emission table the parser stores (len x 20 int16, HMMER column order) */
__attribute__((visibility("default")))
int32_t ref_hmm_emissions(const char *hmm_path, int16_t *out, int32_t cap)
{
	mp_hmm_t *h = mp_hmm_read(hmm_path);
	int32_t len;
	if (!h) return -1;
	len = mp_hmm_length(h);
	if (len * 20 <= cap) memcpy(out, mp_hmm_emissions(h), sizeof(int16_t) * (size_t)len * 20);
	mp_hmm_destroy(h);
	return len;
}
