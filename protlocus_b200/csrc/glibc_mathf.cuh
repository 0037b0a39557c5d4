/*
 * glibc_mathf.cuh -- expf and log1pf that return, for every float argument, the
 * bits the x86-64 host's GNU C library (2.39) returns, so that a float DP whose
 * reference runs on the host's libm can be reproduced bit for bit on the device.
 *
 * The Forward of recheck.c (rc_logsum, recheck.c:260-265) evaluates
 * mx + log1pf(expf(mn - mx)) millions of times per peptide; the device's own
 * expf / log1pf are accurate to an ulp or two but not equal to glibc's, and a
 * one-ulp change of the Forward total moves the null2 bias by about L ulps.
 *
 * Both functions are restated from the published sources that glibc 2.39 builds:
 *
 *  - expf: the table-driven algorithm of Szabolcs Nagy (ARM optimized-routines,
 *    glibc sysdeps/ieee754/flt-32/e_expf.c and e_exp2f_data.c, since glibc 2.27):
 *    k = round(x*32/ln2), r = x*32/ln2 - k, exp(x) = 2^(k/32) * p(r) with a cubic
 *    p evaluated in double and 2^(j/32) from a 32-entry table of doubles.  The
 *    x86-64 build selects the variant compiled with FMA on CPUs that have it,
 *    which fuses r = x*32/ln2 - k and the polynomial's multiply-adds; the fused
 *    forms are written out below.  The table entries are bits(2^(j/32)) - (j << 47),
 *    2^(j/32) rounded to the nearest double.
 *  - log1pf: the Sun fdlibm algorithm (glibc sysdeps/ieee754/flt-32/s_log1pf.c):
 *    1+x = 2^k (1+f), log(1+f) = f - hfsq + s*(hfsq + R(s^2)) with s = f/(2+f),
 *    a degree-7 polynomial R in single precision, k*ln2 in two parts and a
 *    correction term c for the rounding of 1+x; no fused operations.
 *
 * Every operation is written with an explicitly rounded form on the device
 * (__fmul_rn, __fadd_rn, __fma_rn, ...), so the compiler's contraction of
 * a*b+c into an FMA cannot change a result.  In host C the header compiles with
 * plain operators (build it with -ffp-contract=off) and C99 fma().
 *
 * Checked: the host build of these functions against the host's libm on every
 * one of the 4.28e9 non-NaN floats (0 mismatches each), and the device build
 * against the host's libm over the whole argument range the Forward reaches.
 */
#ifndef PL_GLIBC_MATHF_CUH
#define PL_GLIBC_MATHF_CUH

#include <stdint.h>

#if defined(__CUDACC__)
#define GLM_FN static __host__ __device__ __forceinline__
#else
#include <math.h>
#include <string.h>
#define GLM_FN static inline
#endif

#if defined(__CUDA_ARCH__)
#define GLM_FMUL(a, b) __fmul_rn((a), (b))
#define GLM_FADD(a, b) __fadd_rn((a), (b))
#define GLM_FSUB(a, b) __fsub_rn((a), (b))
#define GLM_FDIV(a, b) __fdiv_rn((a), (b))
#define GLM_DMUL(a, b) __dmul_rn((a), (b))
#define GLM_DADD(a, b) __dadd_rn((a), (b))
#define GLM_DSUB(a, b) __dsub_rn((a), (b))
#define GLM_DFMA(a, b, c) __fma_rn((a), (b), (c))
#define GLM_D2F(a) __double2float_rn(a)
GLM_FN uint32_t glm_f2u(float f) { return __float_as_uint(f); }
GLM_FN float glm_u2f(uint32_t u) { return __uint_as_float(u); }
GLM_FN uint64_t glm_d2u(double d) { return (uint64_t)__double_as_longlong(d); }
GLM_FN double glm_u2d(uint64_t u) { return __longlong_as_double((long long)u); }
#else
#define GLM_FMUL(a, b) ((a) * (b))
#define GLM_FADD(a, b) ((a) + (b))
#define GLM_FSUB(a, b) ((a) - (b))
#define GLM_FDIV(a, b) ((a) / (b))
#define GLM_DMUL(a, b) ((a) * (b))
#define GLM_DADD(a, b) ((a) + (b))
#define GLM_DSUB(a, b) ((a) - (b))
#define GLM_DFMA(a, b, c) fma((a), (b), (c))
#define GLM_D2F(a) ((float)(a))
GLM_FN uint32_t glm_f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
GLM_FN float glm_u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
GLM_FN uint64_t glm_d2u(double d) { uint64_t u; memcpy(&u, &d, 8); return u; }
GLM_FN double glm_u2d(uint64_t u) { double d; memcpy(&d, &u, 8); return d; }
#endif

/* 2^(j/32) for j = 0..31 as bits(2^(j/32)) - (j << 47), the nearest doubles */
#define GLM_EXP2_TAB_INIT { \
	0x3ff0000000000000ull, 0x3fefd9b0d3158574ull, 0x3fefb5586cf9890full, 0x3fef9301d0125b51ull, \
	0x3fef72b83c7d517bull, 0x3fef54873168b9aaull, 0x3fef387a6e756238ull, 0x3fef1e9df51fdee1ull, \
	0x3fef06fe0a31b715ull, 0x3feef1a7373aa9cbull, 0x3feedea64c123422ull, 0x3feece086061892dull, \
	0x3feebfdad5362a27ull, 0x3feeb42b569d4f82ull, 0x3feeab07dd485429ull, 0x3feea47eb03a5585ull, \
	0x3feea09e667f3bcdull, 0x3fee9f75e8ec5f74ull, 0x3feea11473eb0187ull, 0x3feea589994cce13ull, \
	0x3feeace5422aa0dbull, 0x3feeb737b0cdc5e5ull, 0x3feec49182a3f090ull, 0x3feed503b23e255dull, \
	0x3feee89f995ad3adull, 0x3feeff76f2fb5e47ull, 0x3fef199bdd85529cull, 0x3fef3720dcef9069ull, \
	0x3fef5818dcfba487ull, 0x3fef7c97337b9b5full, 0x3fefa4afa2a490daull, 0x3fefd0765b6e4540ull }

#if defined(__CUDACC__)
static __device__ const uint64_t glm_exp2_tab_dev[32] = GLM_EXP2_TAB_INIT;
#endif
static const uint64_t glm_exp2_tab_host[32] = GLM_EXP2_TAB_INIT;

GLM_FN float gl_expf(float x)
{
#if defined(__CUDA_ARCH__)
	const uint64_t *tab = glm_exp2_tab_dev;
#else
	const uint64_t *tab = glm_exp2_tab_host;
#endif
	const double inv_ln2_32 = 0x1.71547652b82fep+0 * 32, shift = 0x1.8p+52;
	const double c0 = 0x1.c6af84b912394p-5 / 32 / 32 / 32, c1 = 0x1.ebfce50fac4f3p-3 / 32 / 32,
	             c2 = 0x1.62e42ff0c52d6p-1 / 32;
	const uint32_t ux = glm_f2u(x), abstop = (ux >> 20) & 0x7ff;
	if (abstop >= (0x42b00000u >> 20)) { /* |x| >= 88 or NaN */
		if (ux == 0xff800000u) return 0.0f;                 /* -inf */
		if (abstop >= (0x7f800000u >> 20)) return GLM_FADD(x, x);
		if (x > 0x1.62e42ep6f) return glm_u2f(0x7f800000u);  /* overflow: +inf */
		if (x < -0x1.9fe368p6f) return 0.0f;                 /* underflow */
	}
	const double xd = (double)x;
	double kd = GLM_DFMA(inv_ln2_32, xd, shift);  /* round(x*32/ln2) in the low mantissa bits */
	const uint64_t ki = glm_d2u(kd);
	kd = GLM_DSUB(kd, shift);
	const double r = GLM_DFMA(inv_ln2_32, xd, -kd);
	const uint64_t t = tab[ki % 32] + (ki << 47);
	const double s = glm_u2d(t);
	const double z = GLM_DFMA(c0, r, c1), r2 = GLM_DMUL(r, r);
	double y = GLM_DFMA(c2, r, 1.0);
	y = GLM_DFMA(z, r2, y);
	y = GLM_DMUL(y, s);
	return GLM_D2F(y);
}

GLM_FN float gl_log1pf(float x)
{
	const float ln2_hi = 6.9313812256e-01f, ln2_lo = 9.0580006145e-06f;
	const float lp1 = 6.6666668653e-01f, lp2 = 4.0000000596e-01f, lp3 = 2.8571429849e-01f,
	            lp4 = 2.2222198546e-01f, lp5 = 1.8183572590e-01f, lp6 = 1.5313838422e-01f,
	            lp7 = 1.4798198640e-01f;
	float hfsq, f = 0.0f, c = 0.0f, s, z, R, u;
	const int32_t hx = (int32_t)glm_f2u(x), ax = hx & 0x7fffffff;
	int32_t k = 1, hu = 0;
	if (hx < 0x3ed413d7) {            /* x < 0.41422 */
		if (ax >= 0x3f800000) {        /* x <= -1 */
			if (x == -1.0f) return glm_u2f(0xff800000u);
			return glm_u2f(0x7fc00000u);
		}
		if (ax < 0x31000000) {         /* |x| < 2^-29 */
			if (ax < 0x24800000) return x;
			return GLM_FSUB(x, GLM_FMUL(GLM_FMUL(x, x), 0.5f));
		}
		if (hx > 0 || hx <= (int32_t)0xbe95f61f) { k = 0; f = x; hu = 1; }  /* -0.2929 < x < 0.41422 */
	} else if (hx >= 0x7f800000) {
		return GLM_FADD(x, x);
	}
	if (k != 0) {
		if (hx < 0x5a000000) {
			u = GLM_FADD(1.0f, x);
			hu = (int32_t)glm_f2u(u);
			k = (hu >> 23) - 127;
			c = (k > 0) ? GLM_FSUB(1.0f, GLM_FSUB(u, x)) : GLM_FSUB(x, GLM_FSUB(u, 1.0f));
			c = GLM_FDIV(c, u);
		} else {
			u = x;
			hu = (int32_t)glm_f2u(u);
			k = (hu >> 23) - 127;
			c = 0.0f;
		}
		hu &= 0x007fffff;
		if (hu < 0x3504f7) {
			u = glm_u2f((uint32_t)hu | 0x3f800000u);
		} else {
			k += 1;
			u = glm_u2f((uint32_t)hu | 0x3f000000u);
			hu = (0x00800000 - hu) >> 2;
		}
		f = GLM_FSUB(u, 1.0f);
	}
	hfsq = GLM_FMUL(GLM_FMUL(0.5f, f), f);
	const float kf = (float)k;
	if (hu == 0) {                    /* |f| < 2^-20 */
		if (f == 0.0f) {
			if (k == 0) return 0.0f;
			c = GLM_FADD(c, GLM_FMUL(kf, ln2_lo));
			return GLM_FADD(GLM_FMUL(kf, ln2_hi), c);
		}
		R = GLM_FMUL(hfsq, GLM_FSUB(1.0f, GLM_FMUL(0.66666666666666666f, f)));
		if (k == 0) return GLM_FSUB(f, R);
		return GLM_FSUB(GLM_FMUL(kf, ln2_hi), GLM_FSUB(GLM_FSUB(R, GLM_FADD(GLM_FMUL(kf, ln2_lo), c)), f));
	}
	s = GLM_FDIV(f, GLM_FADD(2.0f, f));
	z = GLM_FMUL(s, s);
	R = GLM_FMUL(lp7, z);
	R = GLM_FMUL(z, GLM_FADD(lp6, R));
	R = GLM_FMUL(z, GLM_FADD(lp5, R));
	R = GLM_FMUL(z, GLM_FADD(lp4, R));
	R = GLM_FMUL(z, GLM_FADD(lp3, R));
	R = GLM_FMUL(z, GLM_FADD(lp2, R));
	R = GLM_FMUL(z, GLM_FADD(lp1, R));
	if (k == 0) return GLM_FSUB(f, GLM_FSUB(hfsq, GLM_FMUL(s, GLM_FADD(hfsq, R))));
	return GLM_FSUB(GLM_FMUL(kf, ln2_hi),
	                GLM_FSUB(GLM_FSUB(hfsq, GLM_FADD(GLM_FMUL(s, GLM_FADD(hfsq, R)), GLM_FADD(GLM_FMUL(kf, ln2_lo), c))), f));
}

/*
 * Branch-free forms for rc_logsum's arguments, which lie in narrow ranges: expf of
 * mn - mx in [-50, 0] and log1pf of its result in [0, 1].  Without branches, lanes
 * with different arguments do not diverge and a thread can keep several logsums in
 * flight.  Each returns the same bits as the function above on its range (every
 * path's value is formed by the same operations, then selected); the checks cover
 * every float of both ranges, on the host and on the device.
 */

/* a / b for 1 <= b <= 2.5 and |a| <= 1 (a zero or normal), correctly rounded, with no
 * branch and no conversion on the device: a reciprocal estimate refined by one Newton
 * step, the quotient, and Markstein's correction with a fused multiply-add (the
 * remainder a - q*b is exact for q this close to a/b; P. Markstein, IBM J. Res. Dev.
 * 34(1), 1990).  gl_log1pf_unit's two quotients (f / (2 + f) and c / (1 + x)) are
 * checked equal to the correctly rounded ones at every float x of [0, 1] through
 * the function's whole result, against the host libm. */
GLM_FN float glm_div(float a, float b)
{
#if defined(__CUDA_ARCH__)
	float r;
	asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
	r = __fmaf_rn(__fmaf_rn(-b, r, 1.0f), r, r);
	const float q = __fmul_rn(a, r);
	return __fmaf_rn(__fmaf_rn(-q, b, a), r, q);
#else
	return a / b;
#endif
}

/* c ? a : b for floats, as a select on the device (both operands are computed, so no
 * branch splits independent evaluations) */
GLM_FN float glm_self(int c, float a, float b)
{
#if defined(__CUDA_ARCH__)
	float r;
	asm("{\n\t.reg .pred p;\n\tsetp.ne.s32 p, %1, 0;\n\tselp.f32 %0, %2, %3, p;\n\t}" : "=f"(r) : "r"(c), "f"(a), "f"(b));
	return r;
#else
	return c ? a : b;
#endif
}

/* gl_expf for |x| < 88 (rc_logsum: [-50, 0]), where its special cases never apply;
 * tab is the 2^(j/32) table (a copy in shared memory on the device) */
GLM_FN float gl_expf_rng_t(float x, const uint64_t *tab)
{
	const double inv_ln2_32 = 0x1.71547652b82fep+0 * 32, shift = 0x1.8p+52;
	const double c0 = 0x1.c6af84b912394p-5 / 32 / 32 / 32, c1 = 0x1.ebfce50fac4f3p-3 / 32 / 32,
	             c2 = 0x1.62e42ff0c52d6p-1 / 32;
	const double xd = (double)x;
	double kd = GLM_DFMA(inv_ln2_32, xd, shift);
	const uint64_t ki = glm_d2u(kd);
	kd = GLM_DSUB(kd, shift);
	const double r = GLM_DFMA(inv_ln2_32, xd, -kd);
	const uint64_t t = tab[ki % 32] + (ki << 47);
	const double s = glm_u2d(t);
	const double z = GLM_DFMA(c0, r, c1), r2 = GLM_DMUL(r, r);
	double y = GLM_DFMA(c2, r, 1.0);
	y = GLM_DFMA(z, r2, y);
	y = GLM_DMUL(y, s);
	return GLM_D2F(y);
}

GLM_FN float gl_expf_rng(float x)
{
#if defined(__CUDA_ARCH__)
	return gl_expf_rng_t(x, glm_exp2_tab_dev);
#else
	return gl_expf_rng_t(x, glm_exp2_tab_host);
#endif
}

/* gl_log1pf for 0 <= x <= 1: the paths of gl_log1pf that this range reaches (x below
 * 2^-29; k = 0 below 0.41422; 1+x = 2^k (1+f) above, with the |f| < 2^-20 cases),
 * each evaluated with gl_log1pf's operations, the result selected */
GLM_FN float gl_log1pf_unit(float x)
{
	const float ln2_hi = 6.9313812256e-01f, ln2_lo = 9.0580006145e-06f;
	const float lp1 = 6.6666668653e-01f, lp2 = 4.0000000596e-01f, lp3 = 2.8571429849e-01f,
	            lp4 = 2.2222198546e-01f, lp5 = 1.8183572590e-01f, lp6 = 1.5313838422e-01f,
	            lp7 = 1.4798198640e-01f;
	const int32_t hx = (int32_t)glm_f2u(x);
	const int small = hx < 0x3ed413d7, tiny = hx < 0x31000000;
	const float r_tiny = glm_self(hx < 0x24800000, x, GLM_FSUB(x, GLM_FMUL(GLM_FMUL(x, x), 0.5f)));
	/* 1 + x = 2^k (1 + f) with the rounding correction c / u */
	const float u1 = GLM_FADD(1.0f, x);
	const int32_t hu1 = (int32_t)glm_f2u(u1), k1 = (hu1 >> 23) - 127, m = hu1 & 0x007fffff;
	const float c1 = glm_div(k1 > 0 ? GLM_FSUB(1.0f, GLM_FSUB(u1, x)) : GLM_FSUB(x, GLM_FSUB(u1, 1.0f)), u1);
	const int hi_m = m >= 0x3504f7;
	const float uL = glm_u2f((uint32_t)m | (hi_m ? 0x3f000000u : 0x3f800000u));
	const int32_t k = small ? 0 : (hi_m ? k1 + 1 : k1), hu = small ? 1 : (hi_m ? (0x00800000 - m) >> 2 : m);
	const float f = glm_self(small, x, GLM_FSUB(uL, 1.0f)), c = glm_self(small, 0.0f, c1);
	const float hfsq = GLM_FMUL(GLM_FMUL(0.5f, f), f), kf = k == 0 ? 0.0f : (k == 1 ? 1.0f : 2.0f);  /* k <= 2 */
	/* |f| < 2^-20 */
	const float r_f0 = glm_self(k == 0, 0.0f, GLM_FADD(GLM_FMUL(kf, ln2_hi), GLM_FADD(c, GLM_FMUL(kf, ln2_lo))));
	const float R0 = GLM_FMUL(hfsq, GLM_FSUB(1.0f, GLM_FMUL(0.66666666666666666f, f)));
	const float r_fs = glm_self(k == 0, GLM_FSUB(f, R0),
	                            GLM_FSUB(GLM_FMUL(kf, ln2_hi), GLM_FSUB(GLM_FSUB(R0, GLM_FADD(GLM_FMUL(kf, ln2_lo), c)), f)));
	/* the polynomial */
	const float s = glm_div(f, GLM_FADD(2.0f, f)), z = GLM_FMUL(s, s);
	float R = GLM_FMUL(lp7, z);
	R = GLM_FMUL(z, GLM_FADD(lp6, R));
	R = GLM_FMUL(z, GLM_FADD(lp5, R));
	R = GLM_FMUL(z, GLM_FADD(lp4, R));
	R = GLM_FMUL(z, GLM_FADD(lp3, R));
	R = GLM_FMUL(z, GLM_FADD(lp2, R));
	R = GLM_FMUL(z, GLM_FADD(lp1, R));
	const float sR = GLM_FMUL(s, GLM_FADD(hfsq, R));
	const float r_p = glm_self(k == 0, GLM_FSUB(f, GLM_FSUB(hfsq, sR)),
	                           GLM_FSUB(GLM_FMUL(kf, ln2_hi), GLM_FSUB(GLM_FSUB(hfsq, GLM_FADD(sR, GLM_FADD(GLM_FMUL(kf, ln2_lo), c))), f)));
	const float r = glm_self(hu == 0, glm_self(f == 0.0f, r_f0, r_fs), r_p);
	return glm_self(tiny, r_tiny, r);
}

#if defined(__CUDACC__)
/*
 * N independent evaluations of gl_expf_rng_t / gl_log1pf_unit, written statement by
 * statement across the N arguments so that the N dependence chains interleave in the
 * instruction stream (the compiler does not interleave N separate calls).  Every
 * element goes through exactly the operations of the scalar form.
 */
#define GLM_N for (int j = 0; j < N; ++j)
template <int N>
static __device__ __forceinline__ void gl_expf_rng_n(const float (&x)[N], float (&out)[N], const uint64_t *tab)
{
	const double inv_ln2_32 = 0x1.71547652b82fep+0 * 32, shift = 0x1.8p+52;
	const double c0 = 0x1.c6af84b912394p-5 / 32 / 32 / 32, c1 = 0x1.ebfce50fac4f3p-3 / 32 / 32,
	             c2 = 0x1.62e42ff0c52d6p-1 / 32;
	double xd[N], kd[N], r[N], s[N], z[N], r2[N], y[N];
	uint64_t ki[N];
#pragma unroll
	GLM_N xd[j] = (double)x[j];
#pragma unroll
	GLM_N kd[j] = GLM_DFMA(inv_ln2_32, xd[j], shift);
#pragma unroll
	GLM_N ki[j] = glm_d2u(kd[j]);
#pragma unroll
	GLM_N kd[j] = GLM_DSUB(kd[j], shift);
#pragma unroll
	GLM_N r[j] = GLM_DFMA(inv_ln2_32, xd[j], -kd[j]);
#pragma unroll
	GLM_N s[j] = glm_u2d(tab[ki[j] % 32] + (ki[j] << 47));
#pragma unroll
	GLM_N z[j] = GLM_DFMA(c0, r[j], c1), r2[j] = GLM_DMUL(r[j], r[j]);
#pragma unroll
	GLM_N y[j] = GLM_DFMA(c2, r[j], 1.0);
#pragma unroll
	GLM_N y[j] = GLM_DFMA(z[j], r2[j], y[j]);
#pragma unroll
	GLM_N y[j] = GLM_DMUL(y[j], s[j]);
#pragma unroll
	GLM_N out[j] = GLM_D2F(y[j]);
}

template <int N>
static __device__ __forceinline__ void gl_log1pf_unit_n(const float (&x)[N], float (&out)[N])
{
	const float ln2_hi = 6.9313812256e-01f, ln2_lo = 9.0580006145e-06f;
	const float lp1 = 6.6666668653e-01f, lp2 = 4.0000000596e-01f, lp3 = 2.8571429849e-01f,
	            lp4 = 2.2222198546e-01f, lp5 = 1.8183572590e-01f, lp6 = 1.5313838422e-01f,
	            lp7 = 1.4798198640e-01f;
	int32_t hx[N], k1[N], m[N], k[N], hu[N];
	int small[N], tiny[N], hi_m[N];
	float r_tiny[N], u1[N], c1[N], uL[N], f[N], c[N], hfsq[N], kf[N], r_f0[N], R0[N], r_fs[N], s[N], zz[N], R[N],
	      sR[N], r_p[N], t2[N];
#pragma unroll
	GLM_N hx[j] = (int32_t)glm_f2u(x[j]), small[j] = hx[j] < 0x3ed413d7, tiny[j] = hx[j] < 0x31000000;
#pragma unroll
	GLM_N r_tiny[j] = glm_self(hx[j] < 0x24800000, x[j], GLM_FSUB(x[j], GLM_FMUL(GLM_FMUL(x[j], x[j]), 0.5f)));
#pragma unroll
	GLM_N u1[j] = GLM_FADD(1.0f, x[j]);
#pragma unroll
	GLM_N {
		const int32_t hu1 = (int32_t)glm_f2u(u1[j]);
		k1[j] = (hu1 >> 23) - 127, m[j] = hu1 & 0x007fffff;
	}
#pragma unroll
	GLM_N t2[j] = k1[j] > 0 ? GLM_FSUB(1.0f, GLM_FSUB(u1[j], x[j])) : GLM_FSUB(x[j], GLM_FSUB(u1[j], 1.0f));
#pragma unroll
	GLM_N c1[j] = glm_div(t2[j], u1[j]);
#pragma unroll
	GLM_N {
		hi_m[j] = m[j] >= 0x3504f7;
		uL[j] = glm_u2f((uint32_t)m[j] | (hi_m[j] ? 0x3f000000u : 0x3f800000u));
		k[j] = small[j] ? 0 : (hi_m[j] ? k1[j] + 1 : k1[j]);
		hu[j] = small[j] ? 1 : (hi_m[j] ? (0x00800000 - m[j]) >> 2 : m[j]);
	}
#pragma unroll
	GLM_N f[j] = glm_self(small[j], x[j], GLM_FSUB(uL[j], 1.0f)), c[j] = glm_self(small[j], 0.0f, c1[j]);
#pragma unroll
	GLM_N hfsq[j] = GLM_FMUL(GLM_FMUL(0.5f, f[j]), f[j]), kf[j] = k[j] == 0 ? 0.0f : (k[j] == 1 ? 1.0f : 2.0f);
#pragma unroll
	GLM_N r_f0[j] = glm_self(k[j] == 0, 0.0f, GLM_FADD(GLM_FMUL(kf[j], ln2_hi), GLM_FADD(c[j], GLM_FMUL(kf[j], ln2_lo))));
#pragma unroll
	GLM_N R0[j] = GLM_FMUL(hfsq[j], GLM_FSUB(1.0f, GLM_FMUL(0.66666666666666666f, f[j])));
#pragma unroll
	GLM_N r_fs[j] = glm_self(k[j] == 0, GLM_FSUB(f[j], R0[j]),
	                         GLM_FSUB(GLM_FMUL(kf[j], ln2_hi), GLM_FSUB(GLM_FSUB(R0[j], GLM_FADD(GLM_FMUL(kf[j], ln2_lo), c[j])), f[j])));
#pragma unroll
	GLM_N s[j] = glm_div(f[j], GLM_FADD(2.0f, f[j]));
#pragma unroll
	GLM_N zz[j] = GLM_FMUL(s[j], s[j]);
#pragma unroll
	GLM_N R[j] = GLM_FMUL(lp7, zz[j]);
#pragma unroll
	GLM_N R[j] = GLM_FMUL(zz[j], GLM_FADD(lp6, R[j]));
#pragma unroll
	GLM_N R[j] = GLM_FMUL(zz[j], GLM_FADD(lp5, R[j]));
#pragma unroll
	GLM_N R[j] = GLM_FMUL(zz[j], GLM_FADD(lp4, R[j]));
#pragma unroll
	GLM_N R[j] = GLM_FMUL(zz[j], GLM_FADD(lp3, R[j]));
#pragma unroll
	GLM_N R[j] = GLM_FMUL(zz[j], GLM_FADD(lp2, R[j]));
#pragma unroll
	GLM_N R[j] = GLM_FMUL(zz[j], GLM_FADD(lp1, R[j]));
#pragma unroll
	GLM_N sR[j] = GLM_FMUL(s[j], GLM_FADD(hfsq[j], R[j]));
#pragma unroll
	GLM_N r_p[j] = glm_self(k[j] == 0, GLM_FSUB(f[j], GLM_FSUB(hfsq[j], sR[j])),
	                        GLM_FSUB(GLM_FMUL(kf[j], ln2_hi),
	                                 GLM_FSUB(GLM_FSUB(hfsq[j], GLM_FADD(sR[j], GLM_FADD(GLM_FMUL(kf[j], ln2_lo), c[j]))), f[j])));
#pragma unroll
	GLM_N out[j] = glm_self(tiny[j], r_tiny[j], glm_self(hu[j] == 0, glm_self(f[j] == 0.0f, r_f0[j], r_fs[j]), r_p[j]));
}
#undef GLM_N
#endif

#endif
