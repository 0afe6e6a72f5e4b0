/*
 * fpmath.h - the binary32 transcendental functions of the hdcx arithmetic
 * contract.
 *
 * The integrator's exp, log, pow, sin, cos, acos and atan2 are these
 * functions, on the GPU and in every CPU evaluation of the integrator, so that
 * both produce the same bits. Each is built from binary32 operations and
 * explicit fused multiply-adds in a fixed order:
 *   - sin/cos: Cody-Waite reduction by pi/2 (three-part constant), Taylor
 *     polynomials of sin and cos on [-pi/4, pi/4] to degree 11 / 12;
 *   - exp: reduction by ln 2 (two-part constant), Taylor polynomial of e^r on
 *     |r| <= ln2/2 to degree 7, exponent scaling by exact powers of two;
 *   - log: x = m 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s),
 *     s = (m-1)/(m+1), odd series to s^11;
 *   - atan2: octant reduction to t in [0, 1], t > 2 - sqrt(3) mapped by
 *     atan t = pi/6 + atan((sqrt3 t - 1)/(sqrt3 + t)), Taylor series of atan
 *     to t^15;
 *   - acos: through asin (Taylor series of asin on [0, 1/2], the half-angle
 *     identity above 1/2);
 *   - pow: y = 2 is x * x, y = 5 is x^5 in binary64 products rounded once;
 *     C99 special cases (pow(x, 0) = 1, pow(1, y) = 1, pow(0, y)); else
 *     e^(y log x) with log x and the product carried as hi + lo pairs of
 *     binary32 (two-sum and fused multiply-add residuals).
 * Accuracy against binary64 references is checked by tests/test_fpmath.py:
 * sin, cos, exp, acos within 1 ulp, log within 2 ulp, atan2 within 4 ulp,
 * pow within 8 ulp on the integrator's argument ranges.
 */
#ifndef HDCX_FPMATH_H
#define HDCX_FPMATH_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define HDCX_FP static __host__ __device__ __forceinline__
#else
#define HDCX_FP static inline
#endif

#ifdef __cplusplus
#include <cmath>
#define HDCX_FP_FMA(a, b, c) ::fmaf((a), (b), (c))
#else
#include <math.h>
#define HDCX_FP_FMA(a, b, c) fmaf((a), (b), (c))
#endif

#if defined(__CUDA_ARCH__)
#undef HDCX_FP_FMA
#define HDCX_FP_FMA(a, b, c) __fmaf_rn((a), (b), (c))
#endif

HDCX_FP float hdcx_fp_bits_to_float(uint32_t u)
{
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, sizeof f);
    return f;
#endif
}

HDCX_FP uint32_t hdcx_fp_float_to_bits(float f)
{
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, sizeof u);
    return u;
#endif
}

/* Nearest integer (ties to even) as float. */
HDCX_FP float hdcx_fp_round(float x)
{
#if defined(__CUDA_ARCH__)
    return rintf(x);
#else
    return nearbyintf(x);
#endif
}

/* 2^k for integer k in [-149, 127] (0 below, inf above). */
HDCX_FP float hdcx_fp_pow2i(int32_t k)
{
    if (k > 127) return hdcx_fp_bits_to_float(0x7f800000u);
    if (k >= -126) return hdcx_fp_bits_to_float((uint32_t)(k + 127) << 23);
    if (k >= -149) return hdcx_fp_bits_to_float(1u << (uint32_t)(k + 149));
    return 0.0f;
}

HDCX_FP float hdcx_fp_sin_poly(float r)
{
    /* sin r = r - r^3/3! + r^5/5! - r^7/7! + r^9/9! - r^11/11! */
    const float r2 = r * r;
    float p = -2.5052108385441718775e-8f;           /* -1/11! */
    p = HDCX_FP_FMA(p, r2, 2.7557319223985890653e-6f);  /* 1/9! */
    p = HDCX_FP_FMA(p, r2, -1.9841269841269841270e-4f); /* -1/7! */
    p = HDCX_FP_FMA(p, r2, 8.3333333333333333333e-3f);  /* 1/5! */
    p = HDCX_FP_FMA(p, r2, -1.6666666666666666667e-1f); /* -1/3! */
    return HDCX_FP_FMA(p * r2, r, r);
}

HDCX_FP float hdcx_fp_cos_poly(float r)
{
    /* cos r = 1 - r^2/2! + r^4/4! - ... + r^12/12! */
    const float r2 = r * r;
    float p = 2.0876756987868098979e-9f;            /* 1/12! */
    p = HDCX_FP_FMA(p, r2, -2.7557319223985890653e-7f); /* -1/10! */
    p = HDCX_FP_FMA(p, r2, 2.4801587301587301587e-5f);  /* 1/8! */
    p = HDCX_FP_FMA(p, r2, -1.3888888888888888889e-3f); /* -1/6! */
    p = HDCX_FP_FMA(p, r2, 4.1666666666666666667e-2f);  /* 1/4! */
    p = HDCX_FP_FMA(p, r2, -0.5f);
    return HDCX_FP_FMA(p, r2, 1.0f);
}

/* Reduction x = k pi/2 + r, |r| <= ~pi/4, accurate for |x| < 2^17 (larger
 * arguments still give the same bits on host and device). The quadrant is
 * k mod 4, computed exactly in binary32 so that no float-to-int conversion
 * can overflow. */
HDCX_FP float hdcx_fp_reduce_half_pi(float x, int32_t* quadrant)
{
    const float k = hdcx_fp_round(x * 0.63661977236758134308f);
    /* pi/2 = C1 + C2 + C3, C1 = fl(pi/2), C2 = fl(pi/2 - C1), C3 = fl(pi/2 - C1 - C2). */
    float r = HDCX_FP_FMA(k, -1.57079637050628662109375f, x);
    r = HDCX_FP_FMA(k, 4.371138828673792886547744274139404296875e-08f, r);
    r = HDCX_FP_FMA(k, 1.7763568394002504646778106689453125e-15f, r);
    *quadrant = (int32_t)(k - 4.0f * floorf(k * 0.25f));
    return r;
}

HDCX_FP float hdcx_fp_sin(float x)
{
    if (!(x == x) || x - x != 0.0f) return (x - x) / (x - x); /* NaN for NaN and inf */
    int32_t q;
    const float r = hdcx_fp_reduce_half_pi(x, &q);
    const float s = (q & 1) ? hdcx_fp_cos_poly(r) : hdcx_fp_sin_poly(r);
    return (q & 2) ? -s : s;
}

HDCX_FP float hdcx_fp_cos(float x)
{
    if (!(x == x) || x - x != 0.0f) return (x - x) / (x - x);
    int32_t q;
    const float r = hdcx_fp_reduce_half_pi(x, &q);
    const float c = (q & 1) ? hdcx_fp_sin_poly(r) : hdcx_fp_cos_poly(r);
    return ((q + 1) & 2) ? -c : c;
}

HDCX_FP float hdcx_fp_exp(float x)
{
    if (!(x == x)) return x;
    if (x > 88.72283935546875f) return hdcx_fp_bits_to_float(0x7f800000u);
    if (x < -103.97208404541015625f) return 0.0f;
    const float k = hdcx_fp_round(x * 1.4426950408889634074f);
    float r = HDCX_FP_FMA(k, -0.693145751953125f, x);       /* ln2 high part */
    r = HDCX_FP_FMA(k, -1.428606765330187045e-6f, r);         /* ln2 low part */
    /* e^r, Taylor to r^7 */
    float p = 1.9841269841269841270e-4f;                     /* 1/7! */
    p = HDCX_FP_FMA(p, r, 1.3888888888888888889e-3f);        /* 1/6! */
    p = HDCX_FP_FMA(p, r, 8.3333333333333333333e-3f);        /* 1/5! */
    p = HDCX_FP_FMA(p, r, 4.1666666666666666667e-2f);        /* 1/4! */
    p = HDCX_FP_FMA(p, r, 1.6666666666666666667e-1f);        /* 1/3! */
    p = HDCX_FP_FMA(p, r, 0.5f);
    p = HDCX_FP_FMA(p, r, 1.0f);
    p = HDCX_FP_FMA(p, r, 1.0f);
    const int32_t ki = (int32_t)k;
    /* Scale in two steps so that 2^k never overflows or flushes early. */
    const int32_t k1 = ki / 2;
    return (p * hdcx_fp_pow2i(k1)) * hdcx_fp_pow2i(ki - k1);
}

HDCX_FP float hdcx_fp_log(float x)
{
    if (!(x == x) || x < 0.0f) return (x - x) / (x - x);
    if (x == 0.0f) return -hdcx_fp_bits_to_float(0x7f800000u);
    if (x - x != 0.0f) return x; /* +inf */
    uint32_t u = hdcx_fp_float_to_bits(x);
    int32_t e = 0;
    if (u < 0x00800000u) { /* subnormal: scale up by 2^23 */
        x = x * 8388608.0f;
        u = hdcx_fp_float_to_bits(x);
        e = -23;
    }
    e += (int32_t)(u >> 23) - 127;
    float m = hdcx_fp_bits_to_float((u & 0x007fffffu) | 0x3f800000u); /* [1, 2) */
    if (m > 1.41421356237309504880f) {
        m = m * 0.5f;
        e += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float s2 = s * s;
    float p = 9.0909090909090909091e-2f;                     /* 1/11 */
    p = HDCX_FP_FMA(p, s2, 1.1111111111111111111e-1f);       /* 1/9 */
    p = HDCX_FP_FMA(p, s2, 1.4285714285714285714e-1f);       /* 1/7 */
    p = HDCX_FP_FMA(p, s2, 2.0e-1f);                         /* 1/5 */
    p = HDCX_FP_FMA(p, s2, 3.3333333333333333333e-1f);       /* 1/3 */
    const float lm = 2.0f * HDCX_FP_FMA(p * s2, s, s);       /* 2 atanh(s) */
    const float fe = (float)e;
    return HDCX_FP_FMA(fe, 0.693145751953125f, HDCX_FP_FMA(fe, 1.428606765330187045e-6f, lm));
}

/* x^5 as binary64 products (x^2 and x^4 exact), rounded once to binary32. */
HDCX_FP float hdcx_fp_pow5(float x)
{
#if defined(__CUDA_ARCH__)
    const double d = (double)x;
    const double d2 = __dmul_rn(d, d);
    return __double2float_rn(__dmul_rn(__dmul_rn(d2, d2), d));
#else
    const double d = (double)x;
    const double d2 = d * d;
    const double d4 = d2 * d2;
    return (float)(d4 * d);
#endif
}

/* log x as an unevaluated sum hi + lo carrying about 40 significant bits, for
 * finite x > 0. Same decomposition as hdcx_fp_log; the quotient s and the
 * final sum keep their rounding errors in lo (exact residuals by fused
 * multiply-add and two-sum). */
HDCX_FP float hdcx_fp_log_ext(float x, float* lo)
{
    uint32_t u = hdcx_fp_float_to_bits(x);
    int32_t e = 0;
    if (u < 0x00800000u) {
        x = x * 8388608.0f;
        u = hdcx_fp_float_to_bits(x);
        e = -23;
    }
    e += (int32_t)(u >> 23) - 127;
    float m = hdcx_fp_bits_to_float((u & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421356237309504880f) {
        m = m * 0.5f;
        e += 1;
    }
    const float f = m - 1.0f;                   /* exact */
    const float d = 2.0f + f;
    const float dLo = (2.0f - d) + f;           /* 2 + f = d + dLo exactly */
    const float sHi = f / d;
    const float sLo = (HDCX_FP_FMA(-sHi, d, f) - sHi * dLo) / d;
    const float s2 = sHi * sHi;
    float p = 9.0909090909090909091e-2f;                     /* 1/11 */
    p = HDCX_FP_FMA(p, s2, 1.1111111111111111111e-1f);       /* 1/9 */
    p = HDCX_FP_FMA(p, s2, 1.4285714285714285714e-1f);       /* 1/7 */
    p = HDCX_FP_FMA(p, s2, 2.0e-1f);                         /* 1/5 */
    p = HDCX_FP_FMA(p, s2, 3.3333333333333333333e-1f);       /* 1/3 */
    /* log m = 2 s + 2 s^3 p(s^2) */
    const float lmHi = 2.0f * sHi;
    const float lmLo = HDCX_FP_FMA(2.0f * sHi * s2, p, 2.0f * sLo);
    const float fe = (float)e;
    const float a = fe * 0.693145751953125f;                 /* exact */
    const float hi = a + lmHi;
    const float bb = hi - a;
    const float err = (a - (hi - bb)) + (lmHi - bb);        /* two-sum */
    const float tail = err + HDCX_FP_FMA(fe, 1.428606765330187045e-6f, lmLo);
    const float sum = hi + tail;                              /* fast two-sum */
    *lo = tail - (sum - hi);
    return sum;
}

/* e^(hi + lo) for |lo| <= ~2^-20 |hi|. */
HDCX_FP float hdcx_fp_exp_ext(float hi, float lo)
{
    if (!(hi == hi)) return hi;
    if (hi > 88.72283935546875f) return hdcx_fp_bits_to_float(0x7f800000u);
    if (hi < -103.97208404541015625f) return 0.0f;
    const float k = hdcx_fp_round(hi * 1.4426950408889634074f);
    float r = HDCX_FP_FMA(k, -0.693145751953125f, hi);
    r = HDCX_FP_FMA(k, -1.428606765330187045e-6f, r);
    r = r + lo;
    float p = 1.9841269841269841270e-4f;
    p = HDCX_FP_FMA(p, r, 1.3888888888888888889e-3f);
    p = HDCX_FP_FMA(p, r, 8.3333333333333333333e-3f);
    p = HDCX_FP_FMA(p, r, 4.1666666666666666667e-2f);
    p = HDCX_FP_FMA(p, r, 1.6666666666666666667e-1f);
    p = HDCX_FP_FMA(p, r, 0.5f);
    p = HDCX_FP_FMA(p, r, 1.0f);
    p = HDCX_FP_FMA(p, r, 1.0f);
    const int32_t ki = (int32_t)k;
    const int32_t k1 = ki / 2;
    return (p * hdcx_fp_pow2i(k1)) * hdcx_fp_pow2i(ki - k1);
}

HDCX_FP float hdcx_fp_pow(float x, float y)
{
    /* The integral exponents the integrator uses: x * x is the correctly
     * rounded square; x^5 goes through exact binary64 products. */
    if (y == 2.0f) return x * x;
    if (y == 5.0f) return hdcx_fp_pow5(x);
    if (y == 0.0f) return 1.0f;
    if (x == 1.0f) return 1.0f;
    if (!(x == x) || !(y == y)) return x + y;
    if (x == 0.0f) return y > 0.0f ? 0.0f : hdcx_fp_bits_to_float(0x7f800000u);
    if (x < 0.0f) return (x - x) / (x - x); /* non-integral use only: NaN */
    if (x - x != 0.0f) return y > 0.0f ? x : 0.0f; /* +inf */
    if (y - y != 0.0f) /* y = +-inf */
        return (x > 1.0f) == (y > 0.0f) ? hdcx_fp_bits_to_float(0x7f800000u) : 0.0f;
    /* y log x as hi + lo, then e^(hi + lo). */
    float logLo;
    const float logHi = hdcx_fp_log_ext(x, &logLo);
    const float prod = y * logHi;
    const float prodLo = HDCX_FP_FMA(y, logHi, -prod) + y * logLo;
    const float pHi = prod + prodLo;                          /* fast two-sum */
    const float pLo = prodLo - (pHi - prod);
    return hdcx_fp_exp_ext(pHi, pLo);
}

/* atan of t in [0, 1]. */
HDCX_FP float hdcx_fp_atan01(float t)
{
    float offset = 0.0f;
    if (t > 0.26794919243112270647f) { /* 2 - sqrt(3) */
        t = (t * 1.7320508075688772935f - 1.0f) / (t + 1.7320508075688772935f);
        offset = 0.52359877559829887308f; /* pi/6 */
    }
    const float t2 = t * t;
    float p = 6.6666666666666666667e-2f;                     /* 1/15 */
    p = HDCX_FP_FMA(p, t2, -7.6923076923076923077e-2f);      /* -1/13 */
    p = HDCX_FP_FMA(p, t2, 9.0909090909090909091e-2f);       /* 1/11 */
    p = HDCX_FP_FMA(p, t2, -1.1111111111111111111e-1f);      /* -1/9 */
    p = HDCX_FP_FMA(p, t2, 1.4285714285714285714e-1f);       /* 1/7 */
    p = HDCX_FP_FMA(p, t2, -2.0e-1f);                        /* -1/5 */
    p = HDCX_FP_FMA(p, t2, 3.3333333333333333333e-1f);       /* 1/3 */
    return offset + HDCX_FP_FMA(-(p * t2), t, t);
}

HDCX_FP float hdcx_fp_atan2(float y, float x)
{
    if (!(x == x) || !(y == y)) return x + y;
    const float ax = x < 0.0f ? -x : x;
    const float ay = y < 0.0f ? -y : y;
    const int negY = hdcx_fp_float_to_bits(y) >> 31;
    const int negX = hdcx_fp_float_to_bits(x) >> 31;
    if (ax == 0.0f && ay == 0.0f) {
        const float a = negX ? 3.14159265358979323846f : 0.0f;
        return negY ? -a : a;
    }
    float a;
    if (ax - ax != 0.0f || ay - ay != 0.0f) { /* infinities */
        if (ax - ax != 0.0f && ay - ay != 0.0f) a = 0.78539816339744830962f;
        else a = (ay - ay != 0.0f) ? 1.57079632679489661923f : 0.0f;
    } else if (ay <= ax) {
        a = hdcx_fp_atan01(ay / ax);
    } else {
        a = 1.57079632679489661923f - hdcx_fp_atan01(ax / ay);
    }
    if (negX) a = 3.14159265358979323846f - a;
    return negY ? -a : a;
}

/* asin of s in [0, 1/2]: Taylor series sum_n (2n)!/(4^n (n!)^2 (2n+1)) s^(2n+1), n <= 12. */
HDCX_FP float hdcx_fp_asin_half(float s)
{
    const float s2 = s * s;
    float p = 6.447210311889649e-3f;                            /* n = 12 */
    p = HDCX_FP_FMA(p, s2, 7.3125258735988454e-3f);             /* n = 11 */
    p = HDCX_FP_FMA(p, s2, 8.390335809616815e-3f);              /* n = 10 */
    p = HDCX_FP_FMA(p, s2, 9.761609529194078e-3f);              /* n = 9 */
    p = HDCX_FP_FMA(p, s2, 1.1551800896139705e-2f);             /* n = 8 */
    p = HDCX_FP_FMA(p, s2, 1.396484375e-2f);                    /* n = 7 */
    p = HDCX_FP_FMA(p, s2, 1.7352764423076924e-2f);             /* n = 6 */
    p = HDCX_FP_FMA(p, s2, 2.2372159090909092e-2f);             /* n = 5 */
    p = HDCX_FP_FMA(p, s2, 3.0381944444444444e-2f);             /* n = 4 */
    p = HDCX_FP_FMA(p, s2, 4.4642857142857144e-2f);             /* n = 3 */
    p = HDCX_FP_FMA(p, s2, 7.5e-2f);                            /* n = 2 */
    p = HDCX_FP_FMA(p, s2, 1.6666666666666666e-1f);             /* n = 1 */
    return HDCX_FP_FMA(p * s2, s, s);
}

HDCX_FP float hdcx_fp_acos(float x)
{
    if (!(x >= -1.0f && x <= 1.0f)) return hdcx_fp_bits_to_float(0x7fc00000u);
    const float ax = x < 0.0f ? -x : x;
    float r;
    if (ax <= 0.5f) {
        r = 1.57079632679489661923f - (x < 0.0f ? -hdcx_fp_asin_half(ax) : hdcx_fp_asin_half(ax));
    } else {
        /* acos|x| = 2 asin(sqrt((1 - |x|)/2)) */
#if defined(__CUDA_ARCH__)
        const float h = 2.0f * hdcx_fp_asin_half(__fsqrt_rn((1.0f - ax) * 0.5f));
#else
        const float h = 2.0f * hdcx_fp_asin_half(sqrtf((1.0f - ax) * 0.5f));
#endif
        r = x < 0.0f ? 3.14159265358979323846f - h : h;
    }
    return r;
}

#endif /* HDCX_FPMATH_H */
