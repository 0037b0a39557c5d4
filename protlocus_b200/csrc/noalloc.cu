/*
 * noalloc.cu -- an allocation-free variant of the batched spliced-DP entry point.
 *
 * Who needs it: some host programs cannot call cudaMalloc/cudaFree from the
 * alignment path.  A program that hands all free device memory to its own pool
 * at start-up and runs under that fixed budget has nothing left for a library to
 * allocate; a latency-sensitive loop cannot afford the device-wide
 * synchronisation that cudaMalloc/cudaFree imply.  pl_splice_batch_noalloc()
 * serves them: it runs the same kernels as pl_splice_batch_device() (input
 * preparation, the wavefront DP, the traceback, the CIGAR compaction), but every
 * byte of scratch those kernels need -- job table, prepared sequences, the
 * strip-to-strip ring, the traceback arena, the reversed-CIGAR buffer -- is
 * carved out of one fixed array in device memory that the library reserves at
 * load time.  The caller passes inputs and outputs as device pointers, as with
 * the device entry point.
 *
 * Limits and rules:
 *   - the scratch array is PL_NOALLOC_SCRATCH_BYTES (96 MiB); every GPU that
 *     loads this library holds it until the process exits;
 *   - a batch may hold at most PL_NOALLOC_MAX_JOBS jobs with proteins of at most
 *     PL_NOALLOC_MAX_AL residues, and its scratch (about 2 bytes per DP cell plus
 *     small per-job buffers) must fit the array; larger batches are rejected with
 *     an error message (pl_noalloc_error) before any GPU work, so split them;
 *   - all calls share the one array and it keeps the previous call's contents:
 *     the launch counters are cleared on every call, everything else is
 *     rewritten before it is read.  Two calls whose GPU work overlapped would
 *     race on the array; the function therefore returns only after its stream
 *     has finished, and holds a library lock for the whole call, so calls from
 *     several host threads run one after another;
 *   - the first call on a device looks the array's device address up
 *     (cudaGetSymbolAddress, with that device current) and caches it; make that
 *     first call before any stream capture begins.  The cached address belongs
 *     to the device's context: a process that calls cudaDeviceReset() (or
 *     otherwise tears that context down) must not call this entry point again;
 *   - no cudaMalloc, cudaFree or other allocating routine is called; host-side
 *     planning uses fixed static tables.
 * Host code must not pass g_noalloc_scratch itself to a kernel: in host code
 * that name is only a stand-in for the symbol, not a device address.
 */
#include <cuda_runtime.h>
#include <pthread.h>
#include <stdio.h>
#include <stdint.h>
#include <string.h>
#include "plk.h"
#include "../../include/plgpu.h"

#define PL_NOALLOC_SCRATCH_BYTES (96u << 20)
#define PL_NOALLOC_MAX_JOBS 4096
#define PL_NOALLOC_MAX_AL 2048
#define PL_NOALLOC_CTAS 32          /* persistent grid of this variant: 32 CTAs x 8 warps */
#define PL_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[PL_NOALLOC_SCRATCH_BYTES];

static pthread_mutex_t g_na_mu = PTHREAD_MUTEX_INITIALIZER;
static void *g_na_addr[PL_NOALLOC_MAX_DEVICES];      /* device address of the array, per device */
static plk_job_t g_na_jobs[PL_NOALLOC_MAX_JOBS];      /* host planning tables (no heap) */
static int32_t g_na_order[PL_NOALLOC_MAX_JOBS];
static char g_na_err[512] = "none";

static int na_fail(const char *msg, long long a, long long b)
{
	snprintf(g_na_err, sizeof(g_na_err), "pl_splice_batch_noalloc: %s (%lld, %lld)", msg, a, b);
	return 0;
}

extern "C" __attribute__((visibility("default"))) const char *pl_noalloc_error(void) { return g_na_err; }

static inline int64_t na_align(int64_t x) { return (x + 255) / 256 * 256; }

static int na_run(const ns_opt_t *opt, const pl_splice_job_t *jobs, int32_t n_jobs,
		const uint8_t *nt, const uint8_t *aa, const uint8_t *ss, pl_splice_result_t *results_dev,
		uint32_t *cigar_dev, int64_t cigar_cap, int64_t *total_cigar, void *stream)
{
	cudaStream_t st = (cudaStream_t)stream;
	plk_params_t P;
	int dev = 0, max_sub = 0, i, m;
	int64_t prep_total = 0, tmp_total = 0, trace_total = 0, off = 0, total_words = 0;
	int32_t max_al = 1, pos = 0;
	unsigned char *base;
	cudaError_t e;

	/* per-device set-up: the array's device address, looked up with the device current */
	if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= PL_NOALLOC_MAX_DEVICES)
		return na_fail("no usable current device", dev, PL_NOALLOC_MAX_DEVICES);
	if (!g_na_addr[dev]) {
		void *p = 0;
		e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess || !p) {
			snprintf(g_na_err, sizeof(g_na_err), "pl_splice_batch_noalloc: cudaGetSymbolAddress of the scratch "
					"array failed: %s", cudaGetErrorString(e));
			return 0;
		}
		g_na_addr[dev] = p;
	}
	base = (unsigned char*)g_na_addr[dev];

	/* options (the same checks as the allocating entry points) */
	if (!opt || !opt->sc || !opt->nt4 || !opt->aa20 || !opt->codon || opt->asize != 22 || opt->pssm ||
			(opt->flag & (NS_F_EXT_LEFT | NS_F_EXT_RIGHT)))
		return na_fail("unsupported options: asize must be 22, no pssm, global DP only (asize, flag)",
				opt ? opt->asize : -1, opt ? opt->flag : -1);
	if (n_jobs < 0 || n_jobs > PL_NOALLOC_MAX_JOBS)
		return na_fail("too many jobs for one call (jobs, limit)", n_jobs, PL_NOALLOC_MAX_JOBS);
	if (n_jobs == 0) { if (total_cigar) *total_cigar = 0; return 1; }
	memset(&P, 0, sizeof(P));
	P.go = opt->go, P.ge = opt->ge, P.io = opt->io, P.fs = opt->fs, P.end_bonus = opt->end_bonus, P.xdrop = opt->xdrop;
	for (i = 0; i < 6; ++i) P.sp[i] = opt->sp[i];
	P.sp_null_bonus = opt->sp_null_bonus, P.ie_coef = opt->ie_coef;
	memcpy(P.sc, opt->sc, 22 * 22), memcpy(P.nt4, opt->nt4, 256), memcpy(P.aa20, opt->aa20, 256), memcpy(P.codon, opt->codon, 64);
	P.aa_x = opt->aa20['X'];
	plk_fill_scaled(&P);
	for (i = 0; i < 22 * 22; ++i) if (max_sub < opt->sc[i]) max_sub = opt->sc[i];

	/* plan: one wave, one warp per job, width by ns_global_gs_auto's rule (nasw-sse.c:987-996) */
	for (i = 0; i < n_jobs; ++i) {
		const pl_splice_job_t *x = &jobs[i];
		plk_job_t *J = &g_na_jobs[i];
		const int64_t bound = (int64_t)x->al * max_sub;
		if (x->nl < 3 || x->al < 1 || x->al > PL_NOALLOC_MAX_AL)
			return na_fail("job outside 3 <= nl and 1 <= al <= 2048 (nl, al)", x->nl, x->al);
		memset(J, 0, sizeof(*J));
		J->nt_off = x->nt_off, J->aa_off = x->aa_off, J->ss_off = ss ? x->ss_off : -1;
		J->nl = x->nl, J->al = x->al;
		J->mode = bound + opt->end_bonus > 30000 ? 1 : (bound + 256 >= 32767 ? 2 : 0);
		J->slen = J->mode == 1 ? (x->al + 3) / 4 : (x->al + 7) / 8;
		J->nw = 1, J->rows = PLK_DP_ROWS;
		J->score = INT32_MIN;
		J->prep_off = prep_total, prep_total += plk_prep_bytes(x->nl, x->al);
		J->tmp_off = tmp_total, tmp_total += (int64_t)x->nl + x->al + 8;
		J->trace_off = trace_total / 2, trace_total += (plk_trace_words(x->nl, x->al, 1, PLK_DP_ROWS) * 2 + 15) / 16 * 16;
		if (x->al > max_al) max_al = x->al;
	}
	/* carve the array: jobs | order | counters | total | prep | tmp | ring | trace */
	{
		const int64_t ring_stride = ((int64_t)max_al + 1) * PLK_RING_INTS;
		const int64_t o_jobs = 0, o_order = na_align(o_jobs + (int64_t)sizeof(plk_job_t) * n_jobs);
		const int64_t o_cnt = na_align(o_order + 4LL * n_jobs), o_tot = o_cnt + 256;
		const int64_t o_prep = o_tot + 256, o_tmp = na_align(o_prep + prep_total + PLK_PREP_SLACK);
		const int64_t o_ring = na_align(o_tmp + 4 * tmp_total);
		const int64_t o_trace = na_align(o_ring + 4 * ring_stride * PL_NOALLOC_CTAS * PLK_WARPS_PER_CTA);
		off = o_trace + trace_total;
		if (off > (int64_t)PL_NOALLOC_SCRATCH_BYTES)
			return na_fail("the batch needs more scratch than the fixed array holds; split it (bytes needed, bytes held)",
					off, (long long)PL_NOALLOC_SCRATCH_BYTES);
		/* job order: grouped by width, longest first inside a group (insertion sort on a static table) */
		for (m = 0; m < 3; ++m)
			for (i = 0; i < n_jobs; ++i)
				if (g_na_jobs[i].mode == m) {
					const int64_t ci = (int64_t)(g_na_jobs[i].nl - 2) * g_na_jobs[i].al;
					int32_t q = pos++;
					while (q > 0 && g_na_jobs[g_na_order[q - 1]].mode == m &&
							(int64_t)(g_na_jobs[g_na_order[q - 1]].nl - 2) * g_na_jobs[g_na_order[q - 1]].al < ci) {
						g_na_order[q] = g_na_order[q - 1];
						--q;
					}
					g_na_order[q] = i;
				}
		plk_job_t *d_jobs = (plk_job_t*)(base + o_jobs);
		int32_t *d_order = (int32_t*)(base + o_order), *d_cnt = (int32_t*)(base + o_cnt);
		int64_t *d_tot = (int64_t*)(base + o_tot);
		uint8_t *d_prep = base + o_prep;
		uint32_t *d_tmp = (uint32_t*)(base + o_tmp);
		int32_t *d_ring = (int32_t*)(base + o_ring);
		uint16_t *d_trace = (uint16_t*)(base + o_trace);
		if ((e = cudaMemcpyAsync(d_jobs, g_na_jobs, sizeof(plk_job_t) * (size_t)n_jobs, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
				(e = cudaMemcpyAsync(d_order, g_na_order, 4 * (size_t)n_jobs, cudaMemcpyHostToDevice, st)) != cudaSuccess)
			goto cuda_fail;
		if ((e = (cudaError_t)plk_prep(d_jobs, n_jobs, nt, aa, ss, d_prep, &P, st)) != cudaSuccess) goto cuda_fail;
		for (m = 0, pos = 0; m < 3; ++m) {
			int32_t n_m = 0;
			while (pos + n_m < n_jobs && g_na_jobs[g_na_order[pos + n_m]].mode == m) ++n_m;
			if (n_m > 0 && (e = (cudaError_t)plk_splice_dp(d_jobs, d_order + pos, 0, d_order + pos, n_m, d_cnt, d_prep,
					d_trace, d_ring, ring_stride, PL_NOALLOC_CTAS, m, PLK_DP_ROWS, &P, st)) != cudaSuccess)
				goto cuda_fail;
			pos += n_m;
		}
		if ((e = (cudaError_t)plk_traceback(d_jobs, d_order, n_jobs, d_trace, d_tmp, st)) != cudaSuccess ||
				(e = (cudaError_t)plk_scan_compact(d_jobs, n_jobs, d_tmp, cigar_dev, cigar_cap, d_tot, results_dev, st)) != cudaSuccess ||
				(e = cudaMemcpyAsync(&total_words, d_tot, sizeof(int64_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
				(e = cudaStreamSynchronize(st)) != cudaSuccess)
			goto cuda_fail;
	}
	if (total_cigar) *total_cigar = total_words;
	strcpy(g_na_err, "none");
	return 1;
cuda_fail:
	/* work queued before the failing step may still be running on the array: wait for it (ignoring
	 * the result) so that the array is idle once the lock is released */
	cudaStreamSynchronize(st);
	snprintf(g_na_err, sizeof(g_na_err), "pl_splice_batch_noalloc: %s", cudaGetErrorString(e));
	return 0;
}

extern "C" __attribute__((visibility("default")))
int pl_splice_batch_noalloc(const ns_opt_t *opt, const pl_splice_job_t *jobs, int32_t n_jobs,
		const uint8_t *nt, const uint8_t *aa, const uint8_t *ss, pl_splice_result_t *results_dev,
		uint32_t *cigar_dev, int64_t cigar_cap, int64_t *total_cigar, void *stream)
{
	int ok;
	pthread_mutex_lock(&g_na_mu);
	ok = na_run(opt, jobs, n_jobs, nt, aa, ss, results_dev, cigar_dev, cigar_cap, total_cigar, stream);
	pthread_mutex_unlock(&g_na_mu);
	return ok;
}
