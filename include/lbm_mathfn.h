/*
 * lbm_mathfn.h - lattice tables and scalar helpers shared by the CUDA
 * library and the CPU oracle.
 *
 * Why this exists: the reference evaluates sin/cos/log/exp in f32 inside
 * Taichi kernels (e.g. the bed harmonics, CODEX.py:1129-1135, the log-law
 * wall model, CODEX.py:3104).  For the GPU path to be bit-identical to the
 * CPU oracle, both sides must produce the same f32 result for these
 * functions.  Neither the CUDA math library nor glibc promise that, so
 * both sides call the functions below: each is evaluated in double with
 * plain IEEE +,-,*,/ (no contraction: the oracle is built with
 * -ffp-contract=off and the CUDA library with -fmad=false) and rounded to
 * f32 once.  The error in double is far below one f32 ulp, so the f32
 * result is the correctly rounded value except in vanishingly rare ties;
 * what matters for parity is that host and device round the identical
 * double.
 *
 * Methods (textbook, written out here):
 *   sin/cos: Cody-Waite reduction by pi/2 with a three-part split of pi/2
 *            (30 + 30 + 53 significant bits), then the Taylor series of
 *            sin and cos on |r| <= pi/4 through degree 21/20.
 *   log:     x = m * 2^e with m in [sqrt(1/2), sqrt(2)),
 *            log x = e*ln2 + 2*atanh(s), s = (m-1)/(m+1), atanh by its
 *            odd power series through s^25 (|s| <= 0.1716).
 *   exp:     x = n*ln2 + r (two-part ln2), |r| <= ln2/2, Taylor series of
 *            exp(r) through r^14, then scale by 2^n through the exponent
 *            bits.
 *   RNG:     SplitMix64 (Steele, Lea, Flood 2014) over (seed, step, cell),
 *            24 high bits -> uniform f32 in [0,1).
 */
#ifndef LBM_MATHFN_H
#define LBM_MATHFN_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define LBM_HD __host__ __device__ __forceinline__
#define LBM_CONST_TABLE __constant__
#else
#define LBM_HD static inline
#define LBM_CONST_TABLE static const
#endif

/* ---- D3Q19 lattice (lbm_lattice.py:3-43) ---- */
#define LBM_Q 19
#define LBM_W0 (1.0 / 3.0)
#define LBM_W1 (1.0 / 18.0)
#define LBM_W2 (1.0 / 36.0)

static const int lbm_cx_h[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0};
static const int lbm_cy_h[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, -1, 1};
static const int lbm_cz_h[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
static const int lbm_opp_h[19] = {0, 2, 1, 4, 3, 6, 5, 9, 10, 7, 8, 13, 14, 11, 12, 17, 18, 15, 16};

/* ---- bit casts ---- */
LBM_HD int64_t lbm_d2ll(double x) {
#if defined(__CUDA_ARCH__)
    return __double_as_longlong(x);
#else
    int64_t r;
    memcpy(&r, &x, sizeof r);
    return r;
#endif
}
LBM_HD double lbm_ll2d(int64_t x) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double(x);
#else
    double r;
    memcpy(&r, &x, sizeof r);
    return r;
#endif
}

/* floor for doubles that fit in int64 range, exact */
LBM_HD double lbm_floor_d(double x) {
    double t = (double)(int64_t)x; /* truncation toward zero */
    return (t > x) ? t - 1.0 : t;
}

/* pi/2 = PIO2_1 + PIO2_2 + PIO2_3 (PIO2_1, PIO2_2 carry 30 significant bits) */
#define LBM_PIO2_1 1.5707963276654482
#define LBM_PIO2_2 (-8.705515692000731e-10)
#define LBM_PIO2_3 (-3.50343439808993e-19)
#define LBM_TWO_OVER_PI 0.6366197723675814
#define LBM_LN2_HI 0.6931471806019545
#define LBM_LN2_LO (-4.2009150726810846e-11)
#define LBM_INV_LN2 1.4426950408889634
#define LBM_SQRT_HALF 0.7071067811865476

/* Taylor polynomial of sin on the reduced interval */
LBM_HD double lbm_sin_poly(double r) {
    double r2 = r * r;
    /* coefficients (-1)^k / (2k+1)!, k = 1..10 */
    double p = 1.9572941063391263e-20;         /*  1/21! */
    p = p * r2 - 8.220635246624329e-18;        /* -1/19! */
    p = p * r2 + 2.8114572543455206e-15;       /*  1/17! */
    p = p * r2 - 7.647163731819816e-13;        /* -1/15! */
    p = p * r2 + 1.6059043836821613e-10;       /*  1/13! */
    p = p * r2 - 2.505210838544172e-08;        /* -1/11! */
    p = p * r2 + 2.7557319223985893e-06;       /*  1/9!  */
    p = p * r2 - 0.0001984126984126984;        /* -1/7!  */
    p = p * r2 + 0.008333333333333333;         /*  1/5!  */
    p = p * r2 - 0.16666666666666666;          /* -1/3!  */
    return r + (r * r2) * p;
}
/* Taylor polynomial of cos on the reduced interval */
LBM_HD double lbm_cos_poly(double r) {
    double r2 = r * r;
    /* coefficients (-1)^k / (2k)!, k = 1..10 */
    double p = 4.110317623312165e-19;          /*  1/20! */
    p = p * r2 - 1.561920696858623e-16;        /* -1/18! */
    p = p * r2 + 4.779477332387385e-14;        /*  1/16! */
    p = p * r2 - 1.1470745597729725e-11;       /* -1/14! */
    p = p * r2 + 2.08767569878681e-09;         /*  1/12! */
    p = p * r2 - 2.755731922398589e-07;        /* -1/10! */
    p = p * r2 + 2.48015873015873e-05;         /*  1/8!  */
    p = p * r2 - 0.001388888888888889;         /* -1/6!  */
    p = p * r2 + 0.041666666666666664;         /*  1/4!  */
    p = p * r2 - 0.5;                          /* -1/2!  */
    return 1.0 + r2 * p;
}

/* reduce x to r in [-pi/4, pi/4], quadrant n mod 4 */
LBM_HD double lbm_reduce_pio2(double x, int *quadrant) {
    double n = lbm_floor_d(x * LBM_TWO_OVER_PI + 0.5);
    double r = ((x - n * LBM_PIO2_1) - n * LBM_PIO2_2) - n * LBM_PIO2_3;
    int64_t ni = (int64_t)n;
    *quadrant = (int)(ni & 3);
    return r;
}

LBM_HD double lbm_sin_d(double x) {
    int q;
    double r = lbm_reduce_pio2(x, &q);
    switch (q) {
        case 0: return lbm_sin_poly(r);
        case 1: return lbm_cos_poly(r);
        case 2: return -lbm_sin_poly(r);
        default: return -lbm_cos_poly(r);
    }
}
LBM_HD double lbm_cos_d(double x) {
    int q;
    double r = lbm_reduce_pio2(x, &q);
    switch (q) {
        case 0: return lbm_cos_poly(r);
        case 1: return -lbm_sin_poly(r);
        case 2: return -lbm_cos_poly(r);
        default: return lbm_sin_poly(r);
    }
}

/* natural log for finite x > 0 (callers guarantee the domain) */
LBM_HD double lbm_log_d(double x) {
    int64_t bits = lbm_d2ll(x);
    int e = (int)((bits >> 52) & 0x7ff);
    if (e == 0) { /* subnormal: scale up by 2^54 */
        x = x * 18014398509481984.0;
        bits = lbm_d2ll(x);
        e = (int)((bits >> 52) & 0x7ff) - 54;
    }
    e -= 1023;
    double m = lbm_ll2d((bits & 0x000fffffffffffffLL) | 0x3ff0000000000000LL); /* [1,2) */
    if (m > 1.0 / LBM_SQRT_HALF) { m = m * 0.5; e += 1; }
    double s = (m - 1.0) / (m + 1.0);
    double s2 = s * s;
    /* atanh(s)/s = sum s^(2k)/(2k+1), k = 0..12 */
    double p = 1.0 / 25.0;
    p = p * s2 + 1.0 / 23.0;
    p = p * s2 + 1.0 / 21.0;
    p = p * s2 + 1.0 / 19.0;
    p = p * s2 + 1.0 / 17.0;
    p = p * s2 + 1.0 / 15.0;
    p = p * s2 + 1.0 / 13.0;
    p = p * s2 + 1.0 / 11.0;
    p = p * s2 + 1.0 / 9.0;
    p = p * s2 + 1.0 / 7.0;
    p = p * s2 + 1.0 / 5.0;
    p = p * s2 + 1.0 / 3.0;
    double at2 = 2.0 * s + (2.0 * s) * (s2 * p);
    double de = (double)e;
    return (de * LBM_LN2_HI + at2) + de * LBM_LN2_LO;
}

/* exp for |x| < 700 */
LBM_HD double lbm_exp_d(double x) {
    double n = lbm_floor_d(x * LBM_INV_LN2 + 0.5);
    double r = (x - n * LBM_LN2_HI) - n * LBM_LN2_LO;
    /* Taylor through r^14 */
    double p = 1.0 / 87178291200.0;           /* 1/14! */
    p = p * r + 1.0 / 6227020800.0;           /* 1/13! */
    p = p * r + 1.0 / 479001600.0;            /* 1/12! */
    p = p * r + 1.0 / 39916800.0;             /* 1/11! */
    p = p * r + 1.0 / 3628800.0;              /* 1/10! */
    p = p * r + 1.0 / 362880.0;               /* 1/9!  */
    p = p * r + 1.0 / 40320.0;                /* 1/8!  */
    p = p * r + 1.0 / 5040.0;                 /* 1/7!  */
    p = p * r + 1.0 / 720.0;                  /* 1/6!  */
    p = p * r + 1.0 / 120.0;                  /* 1/5!  */
    p = p * r + 1.0 / 24.0;                   /* 1/4!  */
    p = p * r + 1.0 / 6.0;                    /* 1/3!  */
    p = p * r + 0.5;                          /* 1/2!  */
    p = p * r + 1.0;
    p = p * r + 1.0;
    int64_t ni = (int64_t)n;
    if (ni < -1000) return 0.0;
    if (ni > 1000) ni = 1000;
    /* multiply by 2^ni in two halves to stay in range */
    int64_t h1 = ni / 2, h2 = ni - h1;
    double s1 = lbm_ll2d((int64_t)(h1 + 1023) << 52);
    double s2 = lbm_ll2d((int64_t)(h2 + 1023) << 52);
    return (p * s1) * s2;
}

LBM_HD float lbm_sinf(float x) { return (float)lbm_sin_d((double)x); }
LBM_HD float lbm_cosf(float x) { return (float)lbm_cos_d((double)x); }
LBM_HD float lbm_logf(float x) { return (float)lbm_log_d((double)x); }
LBM_HD float lbm_expf(float x) { return (float)lbm_exp_d((double)x); }

/* ---- counter-based RNG: SplitMix64 finaliser ---- */
LBM_HD uint64_t lbm_splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
/* uniform f32 in [0,1) keyed by (seed, step, cell) */
LBM_HD float lbm_uniform01(uint64_t seed, uint64_t step, uint64_t cell) {
    uint64_t h = lbm_splitmix64(seed ^ lbm_splitmix64(step ^ lbm_splitmix64(cell + 0x632BE59BD9B4E019ULL)));
    return (float)(h >> 40) * (1.0f / 16777216.0f);
}

#endif /* LBM_MATHFN_H */
