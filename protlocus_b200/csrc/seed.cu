/*
 * seed.cu -- the coarse mapper's seeding on the device (mp_map_coarse's sketch and
 * anchor stages, map.c:565-572, default mode): per protein the k-mer sketch
 * (mp_sketch_prot, sketch.c:18-37), the occurrence cap (mp_cal_max_occ,
 * map.c:304-320, and map.c:566-569), the anchors of every seed whose bucket holds at
 * most the cap (mp_collect_anchors without the rescue, map.c:346-397) and their sort
 * (map.c:571).  The index is the reference's own (index.c:74-98), on the device:
 * ki[b] the first entry of bucket b in kb, the bucket's end ki[b+1] (n_kb for the last).
 *
 *   k_seed_sketch  one thread per protein: the rolling 4-bit k-mer over the 13-letter
 *                  alphabet, the masked integer hash, the seeds in position order, each
 *                  seed's bucket size, and the cap (the 25 % and 75 % order statistics
 *                  of the sizes by an in-place selection) and the anchor count.
 *   k_seed_emit    one warp per protein: for each seed in order whose bucket is within
 *                  the cap, the lanes copy the bucket's blocks as block << 32 | position.
 * The anchors of each protein are then sorted (cub::DeviceSegmentedSort, ascending 64-bit
 * keys: equal keys are equal values, so any sort leaves the reference's array).
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <cub/cub.cuh>
#include "plk.h"

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

/* the k-th smallest of v[0..n) (0-based), reordering v: Hoare partitions */
__device__ uint32_t sd_select(uint32_t *v, int64_t n, const int64_t k)
{
	int64_t lo = 0, hi = n - 1;
	while (lo < hi) {
		const uint32_t pivot = v[lo + (hi - lo) / 2];
		int64_t i = lo, j = hi;
		while (i <= j) {
			while (v[i] < pivot) ++i;
			while (v[j] > pivot) --j;
			if (i <= j) {
				const uint32_t t = v[i];
				v[i] = v[j], v[j] = t;
				++i, --j;
			}
		}
		if (k <= j) hi = j;
		else if (k >= i) lo = i;
		else return v[k];
	}
	return v[k];
}

__device__ __forceinline__ int64_t sd_bucket_size(const int64_t *ki, const int64_t n_bucket, const int64_t n_kb, const int64_t b)
{
	return (b + 1 < n_bucket ? ki[b + 1] : n_kb) - ki[b];
}

__global__ void __launch_bounds__(128) k_seed_sketch(plk_seed_args_t A)
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
	const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (q >= A.n) return;
	const uint8_t *seq = A.seq + A.off[q];
	const int32_t len = A.len[q];
	uint64_t *sd = A.seeds + A.off[q];
	uint32_t *cnt = A.cnt + A.off[q];
	const uint32_t mask_k = (1U << A.kmer * 4) - 1, mask_mod = (1U << A.mod_bit) - 1;
	uint32_t x = 0;
	int32_t l = 0, n = 0;
	for (int32_t i = 0; i < len; ++i) {
		const uint32_t c = tab[seq[i]];
		if (c < 14) {
			x = (x << 4 | c) & mask_k;
			if (++l >= A.kmer) {
				const uint32_t y = sd_hash(x, mask_k);
				if ((y & mask_mod) == 0) {
					sd[n] = (uint64_t)(y >> A.mod_bit) << 32 | (uint32_t)i;
					cnt[n] = (uint32_t)sd_bucket_size(A.ki, A.n_bucket, A.n_kb, (int64_t)(y >> A.mod_bit));
					++n;
				}
			}
		} else x = 0, l = 0;
	}
	int32_t max_occ = A.max_occ;
	if (n >= 8) {  /* map.c:310-319: sizes sorted, q25 and q75 picked by index */
		const int64_t k25 = (int64_t)(n * .25 + .499), k75 = (int64_t)(n * .75 + .499);
		const uint64_t q75 = sd_select(cnt, n, k75);
		const uint64_t q25 = sd_select(cnt, k75 + 1, k25);  /* the k75+1 smallest are in cnt[0..k75] now */
		max_occ = (int32_t)__dadd_rn(__dadd_rn((double)q75, __dmul_rn((double)(q75 - q25), 1.5)), 10.);
		if (max_occ > A.max_occ) max_occ = A.max_occ;
	}
	int64_t n_a = 0;
	for (int32_t j = 0; j < n; ++j) {
		const int64_t sz = sd_bucket_size(A.ki, A.n_bucket, A.n_kb, (int64_t)(sd[j] >> 32));
		if (sz <= max_occ) n_a += sz;
	}
	A.n_seed[q] = n, A.cap[q] = max_occ, A.n_anchor[q] = n_a;
}

__global__ void __launch_bounds__(256) k_seed_emit(plk_seed_args_t A)
{
	const int lane = threadIdx.x & 31;
	const int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (q >= A.n) return;
	const uint64_t *sd = A.seeds + A.off[q];
	const int32_t n = A.n_seed[q], max_occ = A.cap[q];
	uint64_t *a = A.anchors + A.a_off[q];
	int64_t k = 0;
	for (int32_t j = 0; j < n; ++j) {
		const int64_t b = (int64_t)(sd[j] >> 32), st = A.ki[b];
		const int64_t sz = (b + 1 < A.n_bucket ? A.ki[b + 1] : A.n_kb) - st;
		if (sz > max_occ) continue;
		const uint64_t pos = (uint32_t)sd[j];
		for (int64_t t = lane; t < sz; t += 32) a[k + t] = (uint64_t)A.kb[st + t] << 32 | pos;
		k += sz;
	}
}

}  // namespace

extern "C" int plk_seed_sketch(const plk_seed_args_t *a, void *stream)
{
	if (a->n <= 0) return 0;
	k_seed_sketch<<<(unsigned)((a->n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(*a);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

extern "C" int plk_seed_emit(const plk_seed_args_t *a, void *stream)
{
	if (a->n <= 0) return 0;
	k_seed_emit<<<(unsigned)((a->n * 32 + 255) / 256), 256, 0, (cudaStream_t)stream>>>(*a);
	plk_add_launches(1);
	return (int)cudaGetLastError();
}

/* per-protein ascending sort of the anchors from keys_in into keys_out; tmp == 0 asks for
 * the scratch size in *tmp_bytes */
extern "C" int plk_seed_sort(const uint64_t *keys_in, uint64_t *keys_out, int64_t n_items, int32_t n_seg,
		const int64_t *seg_off, void *tmp, size_t *tmp_bytes, void *stream)
{
	cudaError_t e = cub::DeviceSegmentedSort::SortKeys(tmp, *tmp_bytes, keys_in, keys_out, n_items, n_seg, seg_off,
			seg_off + 1, (cudaStream_t)stream);
	if (tmp) plk_add_launches(1);
	return (int)e;
}
