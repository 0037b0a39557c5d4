/*
 * libm_check.c -- test infrastructure: the host C library's expf / log1pf as the
 * checker of the restated glibc algorithms in protlocus_b200/csrc/glibc_mathf.cuh
 * (which the device's recheck Forward uses in rc_logsum, recheck.c:260-265).
 *
 *   lm_mismatch: runs the header's host build (fn 0 expf, 1 log1pf, 2 and 3 their
 *                branch-free forms for rc_logsum's ranges) and the host libm over float bit
 *                patterns lo, lo+stride, ... < hi and counts the results that differ
 *                in any bit (NaN results compare equal to NaN);
 *   lm_host:     fills out[] with the host libm's values at n bit patterns, for the
 *                comparison with the device build.
 * Built with -ffp-contract=off so the header's host build keeps its written roundings.
 */
#include <stdint.h>
#include <string.h>
#include <math.h>
#include "../protlocus_b200/csrc/glibc_mathf.cuh"

#define LM_EXPORT __attribute__((visibility("default")))

/* fn 0 / 1: gl_expf / gl_log1pf; fn 2 / 3: their branch-free forms for rc_logsum's ranges,
 * gl_expf_rng (|x| < 88) and gl_log1pf_unit (0 <= x <= 1), checked on those ranges */
static float lm_host_fn(int fn, float x) { return (fn & 1) == 0 ? expf(x) : log1pf(x); }
static float lm_port_fn(int fn, float x)
{
	return fn == 0 ? gl_expf(x) : fn == 1 ? gl_log1pf(x) : fn == 2 ? gl_expf_rng(x) : gl_log1pf_unit(x);
}

LM_EXPORT int64_t lm_mismatch(int fn, uint32_t lo, uint32_t hi, uint32_t stride, uint32_t *first_bad)
{
	int64_t bad = 0;
	uint64_t u;
	if (stride == 0) stride = 1;
	for (u = lo; u < hi; u += stride) {
		const float x = glm_u2f((uint32_t)u), a = lm_host_fn(fn, x), b = lm_port_fn(fn, x);
		if (glm_f2u(a) != glm_f2u(b) && !(isnan(a) && isnan(b))) {
			if (bad == 0 && first_bad) *first_bad = (uint32_t)u;
			++bad;
		}
	}
	return bad;
}

LM_EXPORT void lm_host(int fn, uint32_t lo, uint32_t stride, int64_t n, float *out)
{
	int64_t i;
	for (i = 0; i < n; ++i) out[i] = lm_host_fn(fn, glm_u2f(lo + (uint32_t)((uint64_t)i * stride)));
}
