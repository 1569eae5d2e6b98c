/* ORACLE TEST INFRASTRUCTURE — CPU restatement, never linked by the product.
 *
 * Bit-reproducible scalar math shared (by restatement) with the CUDA kernels:
 * every operation is an IEEE-754 binary32 add/mul/div/sqrt or an explicit
 * fused multiply-add, compiled with contraction off, so the same sequence of
 * operations gives the same bits on the host and on the device.
 *
 *   orc_log   : ln(m 2^e) = e ln2 + 2 atanh(s), s = (m-1)/(m+1), m in [sqrt(1/2), sqrt(2));
 *               atanh by its Maclaurin series to s^9 (|s| <= 0.1716; the next
 *               term is below 2e-9 relative).
 *   orc_exp   : Cody-Waite reduction x = k ln2 + r, |r| <= ln2/2, Taylor to r^7
 *               (the next term is below 8e-9 relative).
 *   orc_pow15 : x^1.5 = x sqrt(x).
 *   orc_sincos: reduction by multiples of pi/2 (three-part Cody-Waite split),
 *               Taylor series of sin to r^9 and cos to r^10 on |r| <= pi/4
 *               (next terms below 3e-9).
 *   orc_acos_ref: the reference's polynomial arccos (src/smmath.inl:414-420),
 *               reproduced because the reference's Mie lookup and sky use it.
 *   PCG32     : O'Neill's permuted congruential generator (XSH-RR output).
 */
#ifndef ORC_MATH_H
#define ORC_MATH_H

#include <stdint.h>
#include <math.h>
#include <string.h>

static inline uint32_t orc_f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float orc_u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

#define ORC_LN2_HI 0.693115234375f           /* ln2 rounded to 14 bits (exact) */
#define ORC_LN2_LO 3.19461833e-05f            /* ln2 - LN2_HI, rounded to binary32 */

static inline float orc_log(float x) {
    /* x in (0, inf); handles zero -> -inf, subnormals by pre-scaling. */
    if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
    if (x == INFINITY) return x;
    int e = 0;
    uint32_t u = orc_f2u(x);
    if (u < 0x00800000u) { x = x * 16777216.0f; u = orc_f2u(x); e = -24; }
    e += (int)(u >> 23) - 127;
    float m = orc_u2f((u & 0x007fffffu) | 0x3f800000u); /* [1,2) */
    if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
    float s = (m - 1.0f) / (m + 1.0f);
    float s2 = s * s;
    float p = 0.111111111f;                   /* 1/9  */
    p = fmaf(p, s2, 0.142857143f);            /* 1/7  */
    p = fmaf(p, s2, 0.2f);                    /* 1/5  */
    p = fmaf(p, s2, 0.333333333f);            /* 1/3  */
    float t = s * s2;
    float atanh2 = fmaf(t * p, 2.0f, s * 2.0f);   /* 2(s + s^3 P(s^2)) */
    float fe = (float)e;
    return fmaf(fe, ORC_LN2_HI, fmaf(fe, ORC_LN2_LO, atanh2));
}

static inline float orc_exp(float x) {
    if (x != x) return x;
    if (x > 88.7f) return INFINITY;
    if (x < -103.0f) return 0.0f;
    float k = floorf(fmaf(x, 1.44269504f, 0.5f));
    float r = fmaf(-k, ORC_LN2_HI, x);
    r = fmaf(-k, ORC_LN2_LO, r);
    float p = 1.98412698e-04f;                /* 1/7!  */
    p = fmaf(p, r, 1.38888889e-03f);          /* 1/6!  */
    p = fmaf(p, r, 8.33333333e-03f);          /* 1/5!  */
    p = fmaf(p, r, 4.16666667e-02f);          /* 1/4!  */
    p = fmaf(p, r, 1.66666667e-01f);          /* 1/3!  */
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    int ki = (int)k;
    /* scale by 2^k in two steps: k in [-149, 128] keeps both halves normal */
    int k1 = ki / 2, k2 = ki - k1;
    float s1 = orc_u2f((uint32_t)(k1 + 127) << 23);
    float s2 = orc_u2f((uint32_t)(k2 + 127) << 23);
    return (p * s1) * s2;
}

/* x^y for x >= 0 (the only case the renderer uses; negative x gives NaN). */
static inline float orc_pow(float x, float y) {
    if (x == 0.0f) return y > 0.0f ? 0.0f : (y == 0.0f ? 1.0f : INFINITY);
    if (x < 0.0f || x != x) return NAN;
    return orc_exp(y * orc_log(x));
}

/* x^1.5 for x >= 0 (the sky's and HG's exponent); negative x or NaN gives NaN. */
static inline float orc_pow15(float x) {
    if (x < 0.0f || x != x) return NAN;
    return x * sqrtf(x);
}

#define ORC_PIO2_1 1.5703125f                 /* pi/2 rounded to 12 bits (exact) */
#define ORC_PIO2_2 4.83751297e-04f            /* pi/2 - PIO2_1 rounded to 12 bits */
#define ORC_PIO2_3 7.54979013e-08f            /* pi/2 - PIO2_1 - PIO2_2, binary32 */

static inline void orc_sincos(float x, float *ps, float *pc) {
    float k = rintf(x * 0.636619772f);        /* nearest multiple of pi/2 */
    float r = fmaf(-k, ORC_PIO2_1, x);
    r = fmaf(-k, ORC_PIO2_2, r);
    r = fmaf(-k, ORC_PIO2_3, r);
    float r2 = r * r;
    float sp = 2.75573192e-06f;               /*  1/9!  */
    sp = fmaf(sp, r2, -1.98412698e-04f);      /* -1/7!  */
    sp = fmaf(sp, r2, 8.33333333e-03f);       /*  1/5!  */
    sp = fmaf(sp, r2, -1.66666667e-01f);      /* -1/3!  */
    float sn = fmaf(sp * r2, r, r);
    float cp = -2.75573192e-07f;              /* -1/10! */
    cp = fmaf(cp, r2, 2.48015873e-05f);       /*  1/8!  */
    cp = fmaf(cp, r2, -1.38888889e-03f);      /* -1/6!  */
    cp = fmaf(cp, r2, 4.16666667e-02f);       /*  1/4!  */
    cp = fmaf(cp, r2, -0.5f);
    float cs = fmaf(cp, r2, 1.0f);
    int q = ((int)k) & 3;
    float s, c;
    switch (q) {
    case 0: s = sn; c = cs; break;
    case 1: s = cs; c = -sn; break;
    case 2: s = -sn; c = -cs; break;
    default: s = -cs; c = sn; break;
    }
    *ps = s;
    *pc = c;
}

#define ORC_PI 3.14159265358979f              /* SM_PI, src/smmath.inl:16 */

/* src/smmath.inl:414-420: abs as _mm_max_ps(0-s, s); madd/msub without fusion. */
static inline float orc_acos_ref(float s) {
    float z = 0.0f - s;
    float x = z > s ? z : s;
    float r = -0.0187293f * x + 0.0742610f;
    r = r * x - 0.2121144f;
    r = r * x + 1.5707288f;
    r = r * sqrtf(1.0f - x);
    int n = s < 0.0f;
    r = r - (n ? 2.0f * r : 0.0f);
    return (n ? ORC_PI : 0.0f) + r;
}

/* ---- PCG32 ---------------------------------------------------------------- */
typedef struct { uint64_t state, inc; } orc_rng;

static inline uint32_t orc_rng_u32(orc_rng *g) {
    uint64_t old = g->state;
    g->state = old * 6364136223846793005ull + g->inc;
    uint32_t xs = (uint32_t)(((old >> 18) ^ old) >> 27);
    uint32_t rot = (uint32_t)(old >> 59);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

/* uniform on the open interval (0,1): (2k+1) 2^-24 for the top 23 bits k,
 * exactly representable, never 0 or 1 */
static inline float orc_rng_uniform(orc_rng *g) {
    return (float)(((orc_rng_u32(g) >> 9) << 1) | 1u) * 5.96046448e-08f;
}

static inline uint64_t orc_mix64(uint64_t z) {
    /* SplitMix64 finaliser (Steele, Lea, Flood 2014) */
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

/* One independent stream per (seed, pixel, sample): PCG32's documented
 * seeding (state 0, step, add initstate, step) with hashed state and stream. */
static inline void orc_rng_seed(orc_rng *g, uint64_t seed, uint64_t pixel, uint64_t sample) {
    uint64_t a = orc_mix64(seed ^ orc_mix64(pixel * 0x9e3779b97f4a7c15ull + sample));
    uint64_t b = orc_mix64(a + 0x632be59bd9b4e019ull);
    g->state = 0u;
    g->inc = (b << 1) | 1u;
    (void)orc_rng_u32(g);
    g->state += a;
    (void)orc_rng_u32(g);
}

#endif
