/*
 * phx_math.h — bit-reproducible single-precision transcendental functions for host and device.
 *
 * The reference kernels call OpenCL builtins (sin, cos, exp, log, pow, acos, atan2, native_exp)
 * whose precision OpenCL leaves to the implementation (OpenCL C 3.0 s7.4: sin/cos <= 4 ulp,
 * exp/log <= 3 ulp, pow <= 16 ulp, native_* implementation-defined).  This library fixes one
 * implementation and uses it on both sides: the device kernels and any host code that wants to
 * reproduce a device result bit for bit.  Every function is built only from IEEE-754 binary32
 * +, -, *, / and sqrt (correctly rounded on x86-64 SSE and on sm_100a with -prec-div/-prec-sqrt),
 * evaluated in a fixed order with no fused multiply-add, so it returns identical bits on both.
 * Build host code with -ffp-contract=off and device code with -fmad=false.
 *
 * Methods (textbook, no vendor code): Cody-Waite additive range reduction by pi/2 and ln 2 with
 * the reduction constants split so that k*hi is exact (W. J. Cody and W. Waite, "Software Manual
 * for the Elementary Functions", 1980), followed by truncated Taylor series on the reduced
 * interval; log via m = 2^e * f with f in [sqrt(1/2), sqrt(2)) and the atanh series of
 * s = (f-1)/(f+1); atan via the pi/6 argument shift atan(t) = pi/6 + atan((sqrt3*t-1)/(t+sqrt3))
 * and the Taylor series on |u| <= tan(pi/12).  Accuracy on the ranges the renderer uses is a few
 * ulp; tests/test_math.py checks it against libm in double precision.
 */
#ifndef PHX_MATH_H
#define PHX_MATH_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define PHX_MATH_FN __host__ __device__ __forceinline__
#else
#define PHX_MATH_FN static inline
#endif

PHX_MATH_FN float pm_bits_to_f(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}

PHX_MATH_FN uint32_t pm_f_to_bits(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
#endif
}

/* 2^k for k in [-149, 127] as an exact float (0 below, +inf above). */
PHX_MATH_FN float pm_exp2i(int k) {
    if (k > 127)
        return pm_bits_to_f(0x7f800000u);
    if (k >= -126)
        return pm_bits_to_f((uint32_t)(k + 127) << 23);
    if (k >= -149)
        return pm_bits_to_f(1u << (uint32_t)(k + 149));
    return 0.0f;
}

/* round-half-away integer of a float of moderate magnitude, as an int */
PHX_MATH_FN int pm_round_int(float x) { return (int)(x >= 0.0f ? floorf(x + 0.5f) : -floorf(0.5f - x)); }

/* ---- sin / cos -------------------------------------------------------------------------- */
#define PM_TWO_OVER_PI 0.6366197466850281f
#define PM_PIO2_HI 1.5703125f                 /* 8 significant bits */
#define PM_PIO2_MID 0.0004837512969970703f    /* 12 significant bits */
#define PM_PIO2_LO 7.549533620476723e-08f     /* 12 significant bits */
#define PM_PIO2_LO2 2.5633440682570896e-12f

/* sin(r), cos(r) for |r| <= pi/4 (Taylor to r^9 / r^10) */
PHX_MATH_FN float pm_sin_kernel(float r) {
    float z = r * r;
    float p = 2.7557319223985893e-06f;  /* 1/9! */
    p = p * z + -1.984126984126984e-04f; /* -1/7! */
    p = p * z + 8.333333333333333e-03f;  /* 1/5! */
    p = p * z + -1.6666666666666666e-01f; /* -1/3! */
    return r + (r * z) * p;
}

PHX_MATH_FN float pm_cos_kernel(float r) {
    float z = r * r;
    float p = -2.755731922398589e-07f;  /* -1/10! */
    p = p * z + 2.48015873015873e-05f;  /* 1/8! */
    p = p * z + -1.388888888888889e-03f; /* -1/6! */
    p = p * z + 4.1666666666666664e-02f;  /* 1/4! */
    p = p * z + -0.5f;
    return 1.0f + z * p;
}

/* quadrant reduction: x = k*pi/2 + r, with pi/2 split in four parts so that k*part is exact for
 * the first three (|k| < 2^12) and only the last, tiny product rounds */
PHX_MATH_FN float pm_reduce_pio2(float x, int *quadrant) {
    float kf = floorf(x * PM_TWO_OVER_PI + 0.5f);
    float r = x - kf * PM_PIO2_HI;
    r = r - kf * PM_PIO2_MID;
    r = r - kf * PM_PIO2_LO;
    r = r - kf * PM_PIO2_LO2;
    int k = (int)kf;
    *quadrant = k & 3;
    return r;
}

/* sin and cos of x from one reduction: both polynomials, then the quadrant picks and signs them
 * (selects, not branches, so that lanes in different quadrants stay together) */
PHX_MATH_FN void pm_sincosf(float x, float *sn, float *cs) {
    if (!(fabsf(x) < 1.0e5f)) {
        if (x != x || fabsf(x) == pm_bits_to_f(0x7f800000u)) {
            *sn = x - x; /* NaN */
            *cs = x - x;
            return;
        }
    }
    int q;
    float r = pm_reduce_pio2(x, &q);
    float s = pm_sin_kernel(r);
    float c = pm_cos_kernel(r);
    float a = (q & 1) ? c : s; /* sin: s, c, -s, -c in quadrants 0..3 */
    float b = (q & 1) ? s : c; /* cos: c, -s, -c, s */
    *sn = (q & 2) ? -a : a;
    *cs = ((q + 1) & 2) ? -b : b;
}

PHX_MATH_FN float pm_sinf(float x) {
    float s, c;
    pm_sincosf(x, &s, &c);
    return s;
}

PHX_MATH_FN float pm_cosf(float x) {
    float s, c;
    pm_sincosf(x, &s, &c);
    return c;
}

/* ---- exp / log ---------------------------------------------------------------------------- */
#define PM_LOG2E 1.4426950216293335f
#define PM_LN2_HI 0.69140625f
#define PM_LN2_LO 0.0017409306019544601f

PHX_MATH_FN float pm_expf(float x) {
    if (x != x)
        return x;
    if (x > 88.72283935546875f)
        return pm_bits_to_f(0x7f800000u);
    if (x < -103.97208404541016f)
        return 0.0f;
    float kf = floorf(x * PM_LOG2E + 0.5f);
    float r = x - kf * PM_LN2_HI;
    r = r - kf * PM_LN2_LO;
    /* Taylor to r^7 on |r| <= ln2/2 */
    float p = 1.984126984126984e-04f;      /* 1/7! */
    p = p * r + 1.388888888888889e-03f;    /* 1/6! */
    p = p * r + 8.333333333333333e-03f;    /* 1/5! */
    p = p * r + 4.1666666666666664e-02f;   /* 1/4! */
    p = p * r + 1.6666666666666666e-01f;   /* 1/3! */
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    int k = (int)kf;
    if (k < -126) {
        /* two-step scale keeps the intermediate normal */
        return (p * pm_exp2i(k + 64)) * pm_exp2i(-64);
    }
    if (k > 127)
        return (p * pm_exp2i(k - 1)) * 2.0f;
    return p * pm_exp2i(k);
}

PHX_MATH_FN float pm_logf(float x) {
    if (x != x)
        return x;
    if (x < 0.0f)
        return pm_bits_to_f(0x7fc00000u);
    if (x == 0.0f)
        return -pm_bits_to_f(0x7f800000u);
    if (x == pm_bits_to_f(0x7f800000u))
        return x;
    uint32_t u = pm_f_to_bits(x);
    int e;
    if ((u >> 23) == 0) { /* subnormal: scale by 2^25 */
        x = x * 33554432.0f;
        u = pm_f_to_bits(x);
        e = (int)(u >> 23) - 127 - 25;
    } else {
        e = (int)(u >> 23) - 127;
    }
    float f = pm_bits_to_f((u & 0x007fffffu) | 0x3f800000u); /* [1, 2) */
    if (f > 1.41421353816986083984375f) {
        f = f * 0.5f;
        e = e + 1;
    }
    float s = (f - 1.0f) / (f + 1.0f);
    float z = s * s;
    float p = 0.09090909090909091f;   /* 1/11 */
    p = p * z + 0.1111111111111111f;  /* 1/9 */
    p = p * z + 0.14285714285714285f; /* 1/7 */
    p = p * z + 0.2f;
    p = p * z + 0.3333333333333333f;
    float ls = (s + s) + ((s + s) * z) * p; /* 2 atanh(s) */
    float ef = (float)e;
    return ef * PM_LN2_HI + (ls + ef * PM_LN2_LO);
}

/* pow with OpenCL's pow(gentype, gentype) meaning.  Small integral exponents use a fixed
 * square-and-multiply chain; other exponents exp(y log x). */
PHX_MATH_FN float pm_powf(float x, float y) {
    if (y == 0.0f)
        return 1.0f;
    if (x == 1.0f)
        return 1.0f;
    if (x != x || y != y)
        return x + y;
    float yi = floorf(y);
    int is_int = (yi == y);
    if (is_int && fabsf(y) <= 32.0f) {
        int n = (int)fabsf(y);
        float base = x;
        float acc = 1.0f;
        int first = 1;
        while (n > 0) {
            if (n & 1) {
                acc = first ? base : acc * base;
                first = 0;
            }
            n >>= 1;
            if (n > 0)
                base = base * base;
        }
        return (y < 0.0f) ? 1.0f / acc : acc;
    }
    if (x > 0.0f)
        return pm_expf(y * pm_logf(x));
    if (x == 0.0f)
        return (y > 0.0f) ? 0.0f : pm_bits_to_f(0x7f800000u);
    if (is_int) {
        float m = pm_expf(y * pm_logf(-x));
        int odd = ((int64_t)yi) & 1;
        return odd ? -m : m;
    }
    return pm_bits_to_f(0x7fc00000u);
}

/* ---- atan / atan2 / acos ------------------------------------------------------------------ */
#define PM_PI_F 3.1415927410125732f
#define PM_PIO2_F 1.5707963705062866f
#define PM_PIO6_F 0.5235987901687622f
#define PM_SQRT3_F 1.7320507764816284f
#define PM_TAN_PIO12_F 0.2679491937160492f

/* atan on [0, 1] */
PHX_MATH_FN float pm_atan01(float t) {
    float base = 0.0f;
    if (t > PM_TAN_PIO12_F) {
        t = (t * PM_SQRT3_F - 1.0f) / (t + PM_SQRT3_F);
        base = PM_PIO6_F;
    }
    float z = t * t;
    float p = 0.07692307692307693f;    /* 1/13 */
    p = p * z + -0.09090909090909091f; /* -1/11 */
    p = p * z + 0.1111111111111111f;   /* 1/9 */
    p = p * z + -0.14285714285714285f; /* -1/7 */
    p = p * z + 0.2f;
    p = p * z + -0.3333333333333333f;
    return base + (t + (t * z) * p);
}

PHX_MATH_FN float pm_atan2f(float y, float x) {
    if (x != x || y != y)
        return x + y;
    float ax = fabsf(x), ay = fabsf(y);
    float a;
    if (ax == 0.0f && ay == 0.0f) {
        a = 0.0f;
    } else if (ay <= ax) {
        a = pm_atan01(ay / ax);
    } else {
        a = PM_PIO2_F - pm_atan01(ax / ay);
    }
    if (x < 0.0f || (x == 0.0f && (pm_f_to_bits(x) >> 31)))
        a = PM_PI_F - a;
    return (y < 0.0f || (y == 0.0f && (pm_f_to_bits(y) >> 31))) ? -a : a;
}

PHX_MATH_FN float pm_acosf(float x) {
    if (x != x || x > 1.0f || x < -1.0f)
        return pm_bits_to_f(0x7fc00000u);
    float s = sqrtf((1.0f - x) * (1.0f + x));
    return pm_atan2f(s, x);
}

#endif /* PHX_MATH_H */
