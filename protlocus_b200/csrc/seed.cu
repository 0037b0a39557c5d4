/*
 * seed.cu -- the coarse mapper's seeding on the device (mp_map_coarse's sketch and
 * anchor stages, map.c:565-572, default mode): per protein the k-mer sketch
 * (mp_sketch_prot, sketch.c:18-37), the occurrence cap (mp_cal_max_occ,
 * map.c:304-320, and map.c:566-569), the anchors of every seed whose bucket holds at
 * most the cap (mp_collect_anchors without the rescue, map.c:346-397) and their sort
 * (map.c:571).  The index is the reference's own (index.c:74-98), on the device:
 * ki[b] the first entry of bucket b in kb, the bucket's end ki[b+1] (n_kb for the last).
 *
 *   k_seed_sketch  one warp per protein: the 4-bit k-mers over the 13-letter alphabet of
 *                  32 positions at a time, the masked integer hash, the seeds compacted
 *                  in position order, their bucket sizes (32 lookups in flight), the cap
 *                  (the 25 % and 75 % order statistics of the sizes by a warp radix
 *                  select) and the anchor count.
 *   k_seed_emit    one warp per protein: 32 seeds at a time, their kept buckets laid out by
 *                  a warp scan, the lanes copy the blocks as block << 32 | position.
 * HMM-profile queries (the query the profile's consensus, mp_sketch_query with a profile,
 * map.c:332-343) add the profile-derived seeds of mp_sketch_hmm (sketch.c:40-118) before
 * the cap: k_seed_hmm_alts (a thread per match state: its offered groups), k_seed_hmm_enum
 * (a warp per protein, a lane per window: the seeds appended after the protein's own), a
 * segmented sort and k_seed_unique (duplicates removed, then the cap as in the sketch).
 * The anchors of each protein are then sorted (cub::DeviceSegmentedSort, ascending 64-bit
 * keys: equal keys are equal values, so any sort leaves the reference's array).
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <cub/cub.cuh>
#include "plk.h"
#include "seed_hmm.cuh"

extern "C" void plk_add_launches(uint64_t n);

namespace {

/* nasw-tab.c:9-12: residue letters, codes 0-21 and their 13-letter groups; other bytes 15 */
__constant__ uint8_t c_a2r[22] = { 0, 2, 4, 4, 6, 5, 5, 8, 3, 10, 11, 2, 11, 12, 7, 1, 1, 13, 12, 10, 14, 15 };
__constant__ char c_aa[23] = "ARNDCQEGHILKMFPSTWYV*X";

__device__ __forceinline__ uint32_t sd_hash(uint32_t key, const uint32_t mask)
{ /* sketch.c:7-16 */
	key = (key + ~(key << 15)) & mask;
	key ^= key >> 10;
	key = (key + (key << 3)) & mask;
	key ^= key >> 6;
	key = (key + ~(key << 11)) & mask;
	key ^= key >> 16;
	return key;
}

__device__ __forceinline__ int64_t sd_bucket_size(const int64_t *ki, const int64_t n_bucket, const int64_t n_kb, const int64_t b)
{
	return (b + 1 < n_bucket ? ki[b + 1] : n_kb) - ki[b];
}

__device__ __forceinline__ int64_t sd_warp_sum(int64_t v)
{
#pragma unroll
	for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

/* the k-th smallest (0-based) of v[0..n), the whole warp: bit by bit from the top, the
 * values that share the bits chosen so far and have a 0 next are counted */
__device__ uint32_t sd_select(const uint32_t *v, const int32_t n, int64_t k, const int lane)
{
	uint32_t prefix = 0, mask = 0;
	for (int bit = 31; bit >= 0; --bit) {
		const uint32_t m = mask | 1u << bit;
		int64_t c = 0;
		for (int32_t j = lane; j < n; j += 32) c += (v[j] & m) == prefix;
		c = sd_warp_sum(c);
		if (k >= c) k -= c, prefix |= 1u << bit;
		mask = m;
	}
	return prefix;
}

/* the end of a protein's sketch, the whole warp: its n seeds' bucket sizes cnt (written
 * by the warp's lanes) give the occurrence cap, from 8 seeds on the box-plot bound over
 * the sizes' order statistics at these indices (map.c:310-319) limited by the option
 * (map.c:566-569); lane 0 records the count, the cap and the seeds' segment end */
__device__ __forceinline__ void sd_finish(const plk_seed_args_t &A, const int64_t q, const uint32_t *cnt, const int32_t n,
		const int lane)
{
	__syncwarp();
	int32_t max_occ = A.max_occ;
	if (n >= 8) {
		const int64_t k25 = (int64_t)(n * .25 + .499), k75 = (int64_t)(n * .75 + .499);
		const uint64_t q75 = sd_select(cnt, n, k75, lane), q25 = sd_select(cnt, n, k25, lane);
		max_occ = (int32_t)__dadd_rn(__dadd_rn((double)q75, __dmul_rn((double)(q75 - q25), 1.5)), 10.);
		if (max_occ > A.max_occ) max_occ = A.max_occ;
	}
	if (lane == 0) A.n_seed[q] = n, A.cap[q] = max_occ, A.seed_end[q] = A.soff[q] + n;
}

/* one warp per protein: the seeds in position order (a position's k-mer is its last kmer
 * residues when none of them restarts the k-mer, which is what the reference's rolling
 * k-mer holds), their bucket sizes, the cap and the anchor count */
__global__ void __launch_bounds__(256) k_seed_sketch(plk_seed_args_t A)
{
	__shared__ uint8_t tab[256];
	for (int x = threadIdx.x; x < 256; x += blockDim.x) tab[x] = 15;
	__syncthreads();
	if (threadIdx.x < 22) {
		const uint8_t c = (uint8_t)c_aa[threadIdx.x], g = c_a2r[threadIdx.x];
		tab[threadIdx.x] = g, tab[c] = g;
		if (c >= 'A' && c <= 'Z') tab[c + 32] = g;
	}
	__syncthreads();
	const int lane = threadIdx.x & 31;
	const int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (q >= A.n) return;  /* whole warps */
	const uint8_t *seq = A.seq + A.off[q];
	const int32_t len = A.len[q], kmer = A.kmer;
	uint64_t *sd = A.seeds + A.soff[q];
	uint32_t *cnt = A.cnt + A.soff[q];
	const uint32_t mask_k = (1U << kmer * 4) - 1, mask_mod = (1U << A.mod_bit) - 1;
	int32_t n = 0;
	for (int32_t i0 = 0; i0 < len; i0 += 32) {
		const int32_t i = i0 + lane;
		bool is_seed = false;
		uint64_t key = 0;
		if (i < len && i >= kmer - 1) {
			uint32_t x = 0;
			bool ok = true;
			for (int32_t t = i - kmer + 1; t <= i; ++t) {
				const uint32_t c = tab[seq[t]];
				ok = ok && c < 14;
				x = (x << 4 | c) & mask_k;
			}
			if (ok) {
				const uint32_t y = sd_hash(x, mask_k);
				if ((y & mask_mod) == 0) is_seed = true, key = (uint64_t)(y >> A.mod_bit) << 32 | (uint32_t)i;
			}
		}
		const unsigned bal = __ballot_sync(0xffffffffu, is_seed);
		if (is_seed) {
			const int32_t j = n + __popc(bal & ((1u << lane) - 1));
			sd[j] = key;
			cnt[j] = (uint32_t)sd_bucket_size(A.ki, A.n_bucket, A.n_kb, (int64_t)(key >> 32));
		}
		n += __popc(bal);
	}
	sd_finish(A, q, cnt, n, lane);
}

/* one warp per protein: the anchors each seed gives (mp_collect_anchors, map.c:352-384):
 * a bucket within the cap whole; with the repeat rescue, up to repeat_cap blocks of a
 * bucket over it, and when those exceed the budget, every share scaled down, then the rest
 * of the budget handed out one block at a time over the seeds in their sorted order from
 * the query name's hash onwards (lane 0, as the reference's loop) */
__global__ void __launch_bounds__(256) k_seed_take(plk_seed_args_t A)
{
	const int lane = threadIdx.x & 31;
	const int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (q >= A.n) return;  /* whole warps */
	const uint64_t *sd = A.seeds + A.soff[q];
	int32_t *take = A.take + A.soff[q];
	const int32_t n = A.n_seed[q], max_occ = A.cap[q], rcap = A.repeat_cap;
	int64_t n_base = 0, n_res = 0;
	for (int32_t j = lane; j < n; j += 32) {
		const int64_t sz = sd_bucket_size(A.ki, A.n_bucket, A.n_kb, (int64_t)(sd[j] >> 32));
		int32_t t = 0;
		if (sz <= max_occ) t = (int32_t)sz, n_base += sz;
		else if (rcap > 0) t = (int32_t)(sz < rcap ? sz : rcap), n_res += t;
		take[j] = t;
	}
	n_base = sd_warp_sum(n_base), n_res = sd_warp_sum(n_res);
	if (n_res > A.budget) {
		int64_t used = 0;
		for (int32_t j = lane; j < n; j += 32) {
			const int64_t sz = sd_bucket_size(A.ki, A.n_bucket, A.n_kb, (int64_t)(sd[j] >> 32));
			if (sz > max_occ && take[j] > 0) take[j] = (int32_t)((int64_t)take[j] * A.budget / n_res), used += take[j];
		}
		used = sd_warp_sum(used);
		__syncwarp();
		if (lane == 0) {
			const uint32_t start = n > 0 ? A.qhash[q] % (uint32_t)n : 0;
			for (int32_t i = 0; i < n && used < A.budget; ++i) {
				const int32_t j = (int32_t)((start + (uint32_t)i) % (uint32_t)n);
				const int64_t sz = sd_bucket_size(A.ki, A.n_bucket, A.n_kb, (int64_t)(sd[j] >> 32));
				const int64_t cap = sz < rcap ? sz : rcap;
				if (sz > max_occ && take[j] < cap) ++take[j], ++used;
			}
		}
		n_res = __shfl_sync(0xffffffffu, used, 0);
		__syncwarp();
	}
	if (lane == 0) A.n_anchor[q] = n_base + n_res;
}

#define SD_EMIT_WARPS 8
__global__ void __launch_bounds__(32 * SD_EMIT_WARPS) k_seed_emit(plk_seed_args_t A)
{
	__shared__ int64_t s_pre[SD_EMIT_WARPS][33], s_st[SD_EMIT_WARPS][32];
	__shared__ uint32_t s_pos[SD_EMIT_WARPS][32];
	__shared__ int64_t s_sz[SD_EMIT_WARPS][32];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	const int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (q >= A.n) return;  /* whole warps */
	const uint64_t *sd = A.seeds + A.soff[q];
	const int32_t n = A.n_seed[q];
	const int32_t *take = A.take + A.soff[q];
	uint64_t *a = A.anchors + A.a_off[q];
	int64_t k = 0;
	/* 32 seeds at a time: their buckets' starts and sizes (0 past the cap) side by side, an
	 * exclusive scan of the sizes, then every lane copies blocks of any of the 32 seeds
	 * (the seed of output t: the last one whose offset is at most t) */
	for (int32_t j0 = 0; j0 < n; j0 += 32) {
		const int32_t j = j0 + lane;
		int64_t st = 0, sz = 0, tk = 0;
		uint32_t pos = 0;
		if (j < n) {
			const int64_t b = (int64_t)(sd[j] >> 32);
			st = A.ki[b];
			sz = (b + 1 < A.n_bucket ? A.ki[b + 1] : A.n_kb) - st;
			tk = take[j];
			pos = (uint32_t)sd[j];
		}
		int64_t inc = tk;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int64_t t = __shfl_up_sync(0xffffffffu, inc, o);
			if (lane >= o) inc += t;
		}
		const int64_t total = __shfl_sync(0xffffffffu, inc, 31);
		s_pre[w][lane] = inc - tk, s_st[w][lane] = st, s_pos[w][lane] = pos, s_sz[w][lane] = sz;
		if (lane == 31) s_pre[w][32] = total;  /* s_pre[lo + 1] - s_pre[lo]: seed lo's take */
		__syncwarp();
		for (int64_t t = lane; t < total; t += 32) {
			int lo = 0, hi = 31;
			while (lo < hi) {
				const int mid = (lo + hi + 1) >> 1;
				if (s_pre[w][mid] <= t) lo = mid;
				else hi = mid - 1;
			}
			const int64_t u = t - s_pre[w][lo], bsz = s_sz[w][lo], btk = s_pre[w][lo + 1] - s_pre[w][lo];
			/* a whole bucket, or take of its blocks evenly spaced (map.c:390-393) */
			const int64_t o = btk == bsz ? u : u * bsz / btk + bsz / (2 * btk);
			a[k + t] = (uint64_t)A.kb[s_st[w][lo] + o] << 32 | s_pos[w][lo];
		}
		k += total;
		__syncwarp();
	}
}

/* HMM-profile queries: one thread per match state, its offered groups (seed_hmm.cuh) */
__global__ void __launch_bounds__(256) k_seed_hmm_alts(plk_seed_args_t A)
{
	const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= A.n_state) return;
	((sh_alts_t*)A.alts)[s] = sh_state_alts(A.emit + s * 20, A.pos_loss);
}

/* one warp per protein, 32 windows of its profile at a time: each lane counts its window's
 * seeds, a warp scan places them after the protein's own seeds (the sketch's), and the lane
 * walks its window again to write them.  The protein's slots hold its own seeds (at most
 * len) and at most min(seed_max, 4^kmer) per window */
__global__ void __launch_bounds__(256) k_seed_hmm_enum(plk_seed_args_t A)
{
	const int lane = threadIdx.x & 31;
	const int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (q >= A.n) return;  /* whole warps */
	const int32_t kmer = A.kmer, el = A.e_len[q], mx = A.seed_max;
	const int32_t n_win = mx > 0 && el >= kmer ? el - kmer + 1 : 0;
	const sh_alts_t *al = (const sh_alts_t*)A.alts + A.e_off[q];
	const int32_t n0 = A.n_seed[q];
	uint64_t *out = A.seeds + A.soff[q] + n0;
	int64_t k = 0;
	for (int32_t w0 = 0; w0 < n_win; w0 += 32) {
		const int32_t w = w0 + lane;
		int64_t c = 0;
		if (w < n_win) c = sh_window_seeds(al + w, kmer, A.mod_bit, A.win_loss, mx, w + kmer - 1, 0);
		int64_t inc = c;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int64_t t = __shfl_up_sync(0xffffffffu, inc, o);
			if (lane >= o) inc += t;
		}
		if (c > 0) sh_window_seeds(al + w, kmer, A.mod_bit, A.win_loss, mx, w + kmer - 1, out + k + inc - c);
		k += __shfl_sync(0xffffffffu, inc, 31);
	}
	__syncwarp();
	if (lane == 0) A.n_seed[q] = n0 + (int32_t)k, A.seed_end[q] = A.soff[q] + n0 + k;
}

/* one warp per protein: its seeds, sorted (sorted + soff, n_seed of them), without
 * duplicates into its slots (mp_sketch_query with a profile, map.c:338-342), their bucket
 * sizes, and the cap over them (sd_finish) */
__global__ void __launch_bounds__(256) k_seed_unique(plk_seed_args_t A, const uint64_t *sorted)
{
	const int lane = threadIdx.x & 31;
	const int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (q >= A.n) return;  /* whole warps */
	const int64_t base = A.soff[q];
	const int32_t n_in = A.n_seed[q];
	const uint64_t *in = sorted + base;
	uint64_t *sd = A.seeds + base;
	uint32_t *cnt = A.cnt + base;
	int32_t n = 0;
	uint64_t last = 0;
	for (int32_t j0 = 0; j0 < n_in; j0 += 32) {
		const int32_t j = j0 + lane;
		const uint64_t v = j < n_in ? in[j] : 0;
		uint64_t prev = __shfl_up_sync(0xffffffffu, v, 1);
		if (lane == 0) prev = last;
		const bool keep = j < n_in && (j == 0 || v != prev);
		const unsigned bal = __ballot_sync(0xffffffffu, keep);
		if (keep) {
			const int32_t t = n + __popc(bal & ((1u << lane) - 1));
			sd[t] = v;
			cnt[t] = (uint32_t)sd_bucket_size(A.ki, A.n_bucket, A.n_kb, (int64_t)(v >> 32));
		}
		n += __popc(bal);
		last = __shfl_sync(0xffffffffu, v, 31);
	}
	sd_finish(A, q, cnt, n, lane);
}

}  // namespace

extern "C" int plk_seed_hmm_alts(const plk_seed_args_t *a, void *stream)
{
	if (a->n_state <= 0) return 0;
	k_seed_hmm_alts<<<(unsigned)((a->n_state + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*a);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_seed_hmm_enum(const plk_seed_args_t *a, void *stream)
{
	if (a->n <= 0) return 0;
	k_seed_hmm_enum<<<(unsigned)(((int64_t)a->n * 32 + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*a);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_seed_unique(const plk_seed_args_t *a, const uint64_t *sorted, void *stream)
{
	if (a->n <= 0) return 0;
	k_seed_unique<<<(unsigned)(((int64_t)a->n * 32 + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*a, sorted);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_seed_sketch(const plk_seed_args_t *a, void *stream)
{
	if (a->n <= 0) return 0;
	k_seed_sketch<<<(unsigned)(((int64_t)a->n * 32 + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*a);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_seed_take(const plk_seed_args_t *a, void *stream)
{
	if (a->n <= 0) return 0;
	k_seed_take<<<(unsigned)(((int64_t)a->n * 32 + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*a);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_seed_emit(const plk_seed_args_t *a, void *stream)
{
	if (a->n <= 0) return 0;
	k_seed_emit<<<(unsigned)(((int64_t)a->n * 32 + 32 * SD_EMIT_WARPS - 1) / (32 * SD_EMIT_WARPS)), 32 * SD_EMIT_WARPS, 0,
			(cudaStream_t)stream>>>(*a);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

/* per-segment ascending sort of keys_in into keys_out, segment i at [seg_off[i],
 * seg_end[i]) (seg_end 0: up to seg_off[i + 1]); tmp == 0 asks for the scratch size */
extern "C" int plk_seed_sort(const uint64_t *keys_in, uint64_t *keys_out, int64_t n_items, int32_t n_seg,
		const int64_t *seg_off, const int64_t *seg_end, void *tmp, size_t *tmp_bytes, void *stream)
{
	cudaError_t e = cub::DeviceSegmentedSort::SortKeys(tmp, *tmp_bytes, keys_in, keys_out, n_items, n_seg, seg_off,
			seg_end ? seg_end : seg_off + 1, (cudaStream_t)stream);
	if (tmp) plk_add_launches(1);
	return (int)e;
}
