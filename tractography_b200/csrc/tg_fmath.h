/*
 * tg_fmath.h -- portable, bit-reproducible binary32 transcendentals.
 *
 * Every function here is a fixed sequence of IEEE-754 binary32 operations
 * (add, mul, fma, div, sqrt, rint, comparisons and exponent bit edits), so a
 * CPU build (gcc, -ffp-contract=off, no fast-math) and a CUDA build
 * (nvcc -fmad=false, IEEE div/sqrt, no flush-to-zero) return the same bits
 * for the same input.  The streamline integrator is sensitive to the last
 * bit (the Transport orientation update at a 0.1-voxel step amplifies a
 * 1e-7 perturbation to whole voxels), so the tracking kernels and the CPU
 * oracle share this layer the way OpenCL kernels share a platform libm.
 *
 * Methods (all coefficients derived from the mathematics, not from any
 * vendor library):
 *   - argument reduction: Cody & Waite (1980) with the constant split into
 *     three binary32 parts and fused multiply-adds;
 *   - sin/cos on |r| <= pi/4: truncated Taylor series (terms to r^9 / r^10,
 *     truncation error < 0.05 ulp), Horner form;
 *   - exp on |r| <= ln2/2: Taylor series to r^7, scaled by 2^k in two exact
 *     steps;
 *   - log: x = m * 2^e with m in [sqrt(1/2), sqrt(2)), log(m) = 2 atanh(s),
 *     s = (m-1)/(m+1), odd series to s^9.
 * Measured accuracy against double-precision libm is checked by the tests
 * (max error <= 2 ulp over dense sweeps).
 */
#ifndef TG_FMATH_H
#define TG_FMATH_H

#include <stdint.h>
#ifndef __CUDACC__
#include <math.h>
#include <string.h>
#endif

#if defined(__CUDACC__)
#define TGM_FN __host__ __device__ __forceinline__
#else
#define TGM_FN static inline
#endif

/* Constants (hexadecimal binary32 values). */
#define TGM_PI        0x1.921fb6p+1f     /* float(pi) */
#define TGM_TWO_PI    0x1.921fb6p+2f     /* 2 * float(pi), exact */
#define TGM_2_OVER_PI 0x1.45f306p-1f
#define TGM_PIO2_A    0x1.921fb6p+0f     /* pi/2 = A + B + C */
#define TGM_PIO2_B   -0x1.777a5cp-25f
#define TGM_PIO2_C   -0x1.ee59dap-50f
#define TGM_LOG2E     0x1.715476p+0f
#define TGM_LN2_HI    0x1.62e430p-1f     /* ln2 = HI + LO */
#define TGM_LN2_LO   -0x1.05c610p-29f
#define TGM_SQRT2     0x1.6a09e6p+0f

TGM_FN uint32_t tgm_f2u(float x)
{
#if defined(__CUDA_ARCH__)
    return __float_as_uint(x);
#else
    uint32_t u;
    memcpy(&u, &x, sizeof u);
    return u;
#endif
}

TGM_FN float tgm_u2f(uint32_t u)
{
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float x;
    memcpy(&x, &u, sizeof x);
    return x;
#endif
}

/* 2^k as a binary32 value for k in [-126, 127]. */
TGM_FN float tgm_pow2i(int k)
{
    return tgm_u2f((uint32_t)(k + 127) << 23);
}

/* Quadrant index from the rounded reduction multiple (NaN/huge -> 0). */
TGM_FN int tgm_quadrant(float q)
{
    const float finite_q = (q == q && fabsf(q) < 8388608.0f) ? q : 0.0f;
    return (int)finite_q;
}

/* The functions below compute their main path for every input and patch
 * special inputs (NaN, infinities, out-of-range) with selects at the end, so
 * GPU warps do not branch on data; the values are those of the obvious
 * early-return formulation. */

/*
 * sincos: s = sin(x), c = cos(x).  Reduction x = q*pi/2 + r, |r| <~ pi/4.
 */
TGM_FN void tgm_sincosf(float x, float* s_out, float* c_out)
{
    const float q = rintf(x * TGM_2_OVER_PI);
    float r = fmaf(-q, TGM_PIO2_A, x);
    r = fmaf(-q, TGM_PIO2_B, r);
    r = fmaf(-q, TGM_PIO2_C, r);
    const float r2 = r * r;

    /* sin r = r + r^3 (-1/3! + r^2 (1/5! + r^2 (-1/7! + r^2 / 9!))) */
    float ps = 0x1.71de3ap-19f;                  /*  1/9! */
    ps = fmaf(ps, r2, -0x1.a01a02p-13f);         /* -1/7! */
    ps = fmaf(ps, r2, 0x1.111112p-7f);           /*  1/5! */
    ps = fmaf(ps, r2, -0x1.555556p-3f);          /* -1/3! */
    const float sr = fmaf(r * r2, ps, r);

    /* cos r = 1 + r^2 (-1/2 + r^2 (1/4! + r^2 (-1/6! + r^2 (1/8! - r^2/10!)))) */
    float pc = -0x1.27e4fcp-22f;                 /* -1/10! */
    pc = fmaf(pc, r2, 0x1.a01a02p-16f);          /*  1/8!  */
    pc = fmaf(pc, r2, -0x1.6c16c2p-10f);         /* -1/6!  */
    pc = fmaf(pc, r2, 0x1.555556p-5f);           /*  1/4!  */
    pc = fmaf(pc, r2, -0.5f);
    const float cr = fmaf(r2, pc, 1.0f);

    /* quadrant 0: (sr, cr); 1: (cr, -sr); 2: (-sr, -cr); 3: (-cr, sr) */
    const int quadrant = tgm_quadrant(q) & 3;
    const float s = (quadrant & 1) ? cr : sr;
    const float c = (quadrant & 1) ? sr : cr;
    *s_out = (quadrant & 2) ? -s : s;
    *c_out = ((quadrant + 1) & 2) ? -c : c;
}

TGM_FN float tgm_cosf(float x)
{
    float s, c;
    tgm_sincosf(x, &s, &c);
    return c;
}

TGM_FN float tgm_sinf(float x)
{
    float s, c;
    tgm_sincosf(x, &s, &c);
    return s;
}

/*
 * exp: x = k ln2 + r, |r| <= ln2/2; e^r by Taylor to r^7; scale by 2^k.
 */
TGM_FN float tgm_expf(float x_in)
{
    /* main path on the input clamped to the finite-result range */
    const float x = fminf(fmaxf(x_in, -103.97208f), 88.72284f);
    const float k = rintf(x * TGM_LOG2E);
    float r = fmaf(-k, TGM_LN2_HI, x);
    r = fmaf(-k, TGM_LN2_LO, r);
    float p = 0x1.a01a02p-13f;                   /* 1/7! */
    p = fmaf(p, r, 0x1.6c16c2p-10f);             /* 1/6! */
    p = fmaf(p, r, 0x1.111112p-7f);              /* 1/5! */
    p = fmaf(p, r, 0x1.555556p-5f);              /* 1/4! */
    p = fmaf(p, r, 0x1.555556p-3f);              /* 1/3! */
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    const int ki = (int)k;                       /* -150 <= k <= 128 here */
    const int k1 = ki / 2;
    const int k2 = ki - k1;
    float result = (p * tgm_pow2i(k1)) * tgm_pow2i(k2);
    result = (x_in > 88.72284f) ? tgm_u2f(0x7f800000u) : result;   /* +inf */
    result = (x_in < -103.97208f) ? 0.0f : result;
    return (x_in != x_in) ? x_in : result;
}

/*
 * log: natural logarithm for binary32.
 */
TGM_FN float tgm_logf(float x_in)
{
    const int subnormal = x_in < 0x1p-126f;           /* scale subnormals up by 2^24 */
    const float x = subnormal ? x_in * 0x1p+24f : x_in;
    const int e_adjust = subnormal ? -24 : 0;
    const uint32_t bits = tgm_f2u(x);
    int e = (int)((bits >> 23) & 0xffu) - 127 + e_adjust;
    float m = tgm_u2f((bits & 0x007fffffu) | 0x3f800000u);   /* [1, 2) */
    if (m > TGM_SQRT2) {
        m = m * 0.5f;
        e = e + 1;
    }
    const float f = m - 1.0f;                         /* exact */
    const float s = f / (2.0f + f);
    const float z = s * s;
    /* log(m) = 2s (1 + z/3 + z^2/5 + z^3/7 + z^4/9) */
    float p = 0x1.c71c72p-4f;                         /* 1/9 */
    p = fmaf(p, z, 0x1.24924ap-3f);                   /* 1/7 */
    p = fmaf(p, z, 0x1.99999ap-3f);                   /* 1/5 */
    p = fmaf(p, z, 0x1.555556p-2f);                   /* 1/3 */
    const float two_s = s + s;
    const float logm = fmaf(two_s * z, p, two_s);
    const float ef = (float)e;
    float result = fmaf(ef, TGM_LN2_HI, fmaf(ef, TGM_LN2_LO, logm));
    result = (x_in == tgm_u2f(0x7f800000u)) ? x_in : result;          /* +inf */
    result = (x_in == 0.0f) ? tgm_u2f(0xff800000u) : result;          /* -inf */
    result = (x_in < 0.0f) ? tgm_u2f(0x7fc00000u) : result;           /* NaN */
    return (x_in != x_in) ? x_in : result;
}

/*
 * log for positive, finite, normal x -- the tracking step's arguments:
 * Box-Muller's uniform in [2^-24, 1) and 1 + e^{kx} in [1, 1 + e^30].
 * The reduction x = m 2^e, m in [sqrt(1/2), sqrt(2)), comes from one
 * integer subtraction: with B the bits of sqrt(1/2), d = bits(x) - B, m has
 * the bits B + (d mod 2^23) (a carry out of the mantissa field lifts m into
 * [1, sqrt(2))) and e = floor(d / 2^23).  Then log m = log(1 + f), f = m - 1
 * exact, as f - f^2/2 + f^3 Q(f) with Q of degree 7 fitted to the relative
 * error on [sqrt(1/2) - 1, sqrt(2) - 1] (gen_fmath_coefficients.py): no
 * division, unlike tgm_logf's series in f / (2 + f).  Within one ulp of the
 * correctly rounded logarithm on the floats tests/test_math.py checks.
 */
TGM_FN float tgm_log_pos(float x)
{
    const uint32_t d = tgm_f2u(x) - 0x3f3504f3u;
    const int e = (int)((d + 0x3f800000u) >> 23) - 127;
    const float m = tgm_u2f((d & 0x007fffffu) + 0x3f3504f3u);
    const float f = m - 1.0f;
    float q = -0x1.38b4ccp-4f;                        /* Q7 */
    q = fmaf(q, f, 0x1.055b46p-3f);                   /* Q6 */
    q = fmaf(q, f, -0x1.0d8552p-3f);                  /* Q5 */
    q = fmaf(q, f, 0x1.22da22p-3f);                   /* Q4 */
    q = fmaf(q, f, -0x1.547244p-3f);                  /* Q3 */
    q = fmaf(q, f, 0x1.99a008p-3f);                   /* Q2 */
    q = fmaf(q, f, -0x1.000228p-2f);                  /* Q1 */
    q = fmaf(q, f, 0x1.555554p-2f);                   /* Q0 */
    const float t = fmaf(f, q, -0.5f);
    const float logm = fmaf(f * f, t, f);
    const float ef = (float)e;
    return fmaf(ef, TGM_LN2_HI, fmaf(ef, TGM_LN2_LO, logm));
}

/*
 * 1/sqrt(x) for x >= 2^-100, finite: the initial estimate of Lomont ("Fast
 * Inverse Square Root", 2003; relative error below 3.5e-2) from one integer
 * subtraction, then three Newton steps y (3/2 - (x/2) y^2), which take the
 * error below 1e-10 before rounding (each step squares it, times 3/2).
 * Within two ulp (tested); for the orientation frame, where a square root
 * and a division did the same work.
 */
TGM_FN float tgm_rsqrt_pos(float x)
{
    const float hx = 0.5f * x;
    float y = tgm_u2f(0x5f375a86u - (tgm_f2u(x) >> 1));
    y = y * fmaf(-hx * y, y, 1.5f);
    y = y * fmaf(-hx * y, y, 1.5f);
    y = y * fmaf(-hx * y, y, 1.5f);
    return y;
}

/*
 * e^x for x <= 30, not NaN (softplus's argument, capped at 30 by its
 * caller): the series of tgm_expf, scaled by 2^k in one step; below
 * -87.3 (where the result would leave the normal range) the result is 0.
 */
TGM_FN float tgm_exp_upto30(float x_in)
{
    const float x = fmaxf(x_in, -87.33654f);
    const float k = rintf(x * TGM_LOG2E);             /* -126 <= k <= 44 */
    float r = fmaf(-k, TGM_LN2_HI, x);
    r = fmaf(-k, TGM_LN2_LO, r);
    float p = 0x1.a01a02p-13f;                   /* 1/7! */
    p = fmaf(p, r, 0x1.6c16c2p-10f);             /* 1/6! */
    p = fmaf(p, r, 0x1.111112p-7f);              /* 1/5! */
    p = fmaf(p, r, 0x1.555556p-5f);              /* 1/4! */
    p = fmaf(p, r, 0x1.555556p-3f);              /* 1/3! */
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    const float result = p * tgm_pow2i((int)k);
    return (x_in < -87.33654f) ? 0.0f : result;
}

/*
 * The exponential map's factors (core.cl:101-109) from n2 = |t|^2 > 0:
 * c = cos(n) and k = sin(n) / n with n = sqrt(n2).  For n2 < 1 both are
 * 1 + n2 times a cubic in n2 fitted to the relative error on [0, 1)
 * (gen_fmath_coefficients.py; fits within 2^-30), which needs neither the
 * square root, the range reduction nor the division; larger angles take
 * the general path.
 */
TGM_FN void tgm_exps2_factors(float n2, float* c_out, float* k_out)
{
    if (n2 < 1.0f) {
        float pc = 0x1.94a4c6p-16f;                 /* P3 */
        pc = fmaf(pc, n2, -0x1.6beef6p-10f);        /* P2 */
        pc = fmaf(pc, n2, 0x1.5554e6p-5f);          /* P1 */
        pc = fmaf(pc, n2, -0x1.fffffep-2f);         /* P0 */
        *c_out = fmaf(pc, n2, 1.0f);
        float pk = 0x1.69b0f6p-19f;                 /* K3 */
        pk = fmaf(pk, n2, -0x1.9ffe56p-13f);        /* K2 */
        pk = fmaf(pk, n2, 0x1.1110ecp-7f);          /* K1 */
        pk = fmaf(pk, n2, -0x1.555556p-3f);         /* K0 */
        *k_out = fmaf(pk, n2, 1.0f);
    } else {
        const float n = sqrtf(n2);
        float s, c;
        tgm_sincosf(n, &s, &c);
        *c_out = c;
        *k_out = s / n;
    }
}

/*
 * softplus(x) = log(1 + e^{kx}) / k for kx < 30 (else x) and its derivative
 * 1 / (1 + e^{-kx}) (core.cl:111-120), from one exponential: with
 * E = e^{kx} the derivative is E / (1 + E).  For kx >= 30 the derivative
 * rounds to 1 in binary32 (e^{-30} < 2^-24), and NaN propagates.  The
 * division by k is a multiplication by inv_k = 1/k rounded.
 *
 * The tracking step also divides by the model value, floored at 1e-6
 * (algorithm.py:98, :216); *inv_floor receives 1 / max(value, 1e-6).  Below
 * kx = 30 both reciprocals come from one division,
 * q = 1 / ((1 + E) max(value, 1e-6)).
 */
TGM_FN void tgm_softplus(float x, float k, float inv_k, float* value, float* derivative, float* inv_floor)
{
    /* branch-free: one exponential, one logarithm and one division whatever
     * kx is (the exponential's argument is capped at 30, where it is not
     * used, so that the logarithm stays in its domain) */
    const float kx = x * k;
    const int small = kx < 30.0f;
    const float e = tgm_exp_upto30(fminf(kx, 30.0f));
    const float one_e = 1.0f + e;
    const float lg = tgm_log_pos(one_e) * inv_k;
    const float v = small ? lg : x;
    const float m = (v < 1e-6f) ? 1e-6f : v;
    const float q = 1.0f / (small ? one_e * m : m);
    *value = v;
    *derivative = small ? (e * m) * q : ((kx == kx) ? 1.0f : kx);
    *inv_floor = small ? one_e * q : q;
}

/*
 * cos(2 pi k / 2^24) for a 24-bit k (the uniform k 2^-24 of core.cl:212-214
 * that Box-Muller turns into an angle, core.cl:240-245).  The quarter turns
 * q = round(k / 2^22) come out exactly in integer arithmetic; the remainder
 * |r| <= 2^21 becomes an angle |t| <= pi/4 by one multiplication, and
 * cos(t + q pi/2) is cos t, -sin t, -cos t or sin t, each a polynomial in
 * t^2 fitted to the relative error on |t| <= pi/4
 * (gen_fmath_coefficients.py).  No float argument reduction is needed.
 */
#define TGM_TWO_PI_2M24 0x1.921fb6p-22f   /* float(2 pi) / 2^24, exact scaling */
TGM_FN float tgm_cos2pi_u24(uint32_t k)
{
    const uint32_t q = (k + 0x200000u) >> 22;
    const int32_t r = (int32_t)k - (int32_t)(q << 22);
    const float t = (float)r * TGM_TWO_PI_2M24;
    const float t2 = t * t;
    float ps = -0x1.9943e0p-13f;                 /* S2 */
    ps = fmaf(ps, t2, 0x1.11073ap-7f);           /* S1 */
    ps = fmaf(ps, t2, -0x1.555546p-3f);          /* S0 */
    const float st = fmaf(t * t2, ps, t);
    float pc = 0x1.9916a0p-16f;                  /* C3 */
    pc = fmaf(pc, t2, -0x1.6c07f2p-10f);         /* C2 */
    pc = fmaf(pc, t2, 0x1.55553cp-5f);           /* C1 */
    pc = fmaf(pc, t2, -0.5f);                    /* C0 */
    const float ct = fmaf(t2, pc, 1.0f);
    const float c = (q & 1u) ? st : ct;
    return ((q + 1u) & 2u) ? -c : c;
}

#endif /* TG_FMATH_H */
