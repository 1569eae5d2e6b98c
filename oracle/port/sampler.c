/* ORACLE TEST INFRASTRUCTURE — restatement of the reference's per-vertex
 * samplers with the same binary32 operation order (no fused multiply-adds:
 * the reference's SSE4 build evaluates madd/msub as separate mul and add).
 *
 *   SampleVoxelSpace          src/kernel.cpp:96-126
 *   MiePhase::Evaluate/RGB    src/KernelSampler.cpp:214-255
 *   MiePhase::Sample          src/KernelSampler.cpp:257-285 (linear scan)
 *   SamplingBasis             src/KernelSampler.cpp:145-154
 *   SunLight Evaluate/Pdf/Sample src/KernelSampler.cpp:318-345
 *   Hosek sky radiance        src/kernel.cpp:329-360
 *   camera ray                src/kernel.cpp:461-474
 * Transcendentals (log, exp, pow, sin, cos) come from orc_math.h and differ
 * from the reference's SSE approximations by a few ulps.
 */
#include "oracle.h"
#include "orc_math.h"
#include <math.h>
#include <float.h>
#include <stdlib.h>

static inline float sse_max(float a, float b) { return a > b ? a : b; } /* _mm_max_ps(a,b) */
static inline float sse_min(float a, float b) { return a < b ? a : b; } /* _mm_min_ps(a,b) */
static inline float lerp_ref(float a, float b, float t) { return t * (b - a) + a; } /* t.madd(b-a, a) */

float orc_sample_voxel_space(const float p[3], const float *v, const float ce[4], uint32_t N) {
    const float nv = (float)N;
    const float nm1 = nv - 1.0f;
    const float top = (float)(N - 1);
    uint32_t ia[3], ib[3];
    float nl[3];
    for (int k = 0; k < 3; ++k) {
        float ni = ((-0.5f * ((ce[k] - ce[3]) - p[k])) * nm1) / ce[3];
        float nf = sse_max(floorf(ni), 0.0f);
        float nc = sse_min(ceilf(ni), nm1);
        nl[k] = ni - nf;
        nc = sse_max(sse_min(nc, top), 0.0f);
        nf = sse_max(sse_min(nf, top), 0.0f);
        ia[k] = (uint32_t)nf;
        ib[k] = (uint32_t)nc;
    }
    const uint32_t N2 = N * N;
#define V(z, y, x) v[(z) * N2 + (y) * N + (x)]
    float u0 = lerp_ref(V(ia[2], ia[1], ia[0]), V(ia[2], ia[1], ib[0]), nl[0]);
    float u1 = lerp_ref(V(ia[2], ib[1], ia[0]), V(ia[2], ib[1], ib[0]), nl[0]);
    float u2 = lerp_ref(V(ib[2], ia[1], ia[0]), V(ib[2], ia[1], ib[0]), nl[0]);
    float u3 = lerp_ref(V(ib[2], ib[1], ia[0]), V(ib[2], ib[1], ib[0]), nl[0]);
#undef V
    float v0 = lerp_ref(u0, u1, nl[1]);
    float v1 = lerp_ref(u2, u3, nl[1]);
    return lerp_ref(v0, v1, nl[2]);
}

static inline float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* index of the lower table entry and the lerp weight, src/KernelSampler.cpp:232-239 */
static void mie_index(const orc_params *P, float ct, uint32_t *X, float *t) {
    float ct1 = sse_max(sse_min(ct, 1.0f), -1.0f);       /* saturate2 */
    float a = orc_acos_ref(0.0f - ct1) / ORC_PI;
    float b = (float)P->mie_n * a;
    float c = floorf(b);
    c = sse_min(c, (float)(P->mie_n - 2));
    c = sse_max(c, 0.0f);
    *t = b - c;
    *X = (uint32_t)c;
}

void orc_mie_eval_rgb(const orc_params *P, float ct, float out[3]) {
    uint32_t X;
    float t;
    mie_index(P, ct, &X, &t);
    for (int k = 0; k < 3; ++k) out[k] = lerp_ref(P->mie_pdf[3 * X + k], P->mie_pdf[3 * (X + 1) + k], t);
}

float orc_mie_eval(const orc_params *P, float ct) {
    uint32_t X;
    float t;
    mie_index(P, ct, &X, &t);
    return lerp_ref(P->mie_pdf[3 * X], P->mie_pdf[3 * (X + 1)], t);
}

/* interpolated red CDF value at scan step i, src/KernelSampler.cpp:262-267 */
static inline float mie_scan_cdf(const orc_params *P, float ub, uint32_t i, float *t_out) {
    const uint32_t n = P->mie_n;
    float b = sse_max(ub, (float)i);
    float c = sse_min(floorf(b), (float)(n - 1));
    float t = b - c;
    *t_out = t;
    return lerp_ref(P->mie_cdf[3 * i], P->mie_cdf[3 * (i + 1)], t);
}

float orc_mie_sample_theta_scan(const orc_params *P, float u1) {
    const uint32_t n = P->mie_n;
    float th = 0.0f;
    float ub = (float)n * u1;
    for (uint32_t i = 0; i < n - 1; ++i) {
        float t;
        float cdf = mie_scan_cdf(P, ub, i, &t);
        int m = cdf < u1;
        float s = (float)i / (float)n + t / (float)n;
        if (m) th = s;
        else break;
    }
    return th;
}

/* The scan's predicate is non-decreasing in i, so the first failing step is
 * found by bisection; the result equals the scan's whenever that holds. */
float orc_mie_sample_theta_bisect(const orc_params *P, float u1) {
    const uint32_t n = P->mie_n;
    float ub = (float)n * u1;
    uint32_t lo = 0, hi = n - 1; /* first i in [0, n-1) with !(cdf < u1), or n-1 */
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        float t;
        if (mie_scan_cdf(P, ub, mid, &t) < u1) lo = mid + 1;
        else hi = mid;
    }
    if (lo == 0) return 0.0f;
    float t;
    (void)mie_scan_cdf(P, ub, lo - 1, &t);
    return (float)(lo - 1) / (float)n + t / (float)n;
}

/* SamplingBasis, src/KernelSampler.cpp:145-154 */
static void sampling_basis(const float iv[3], float b1[3], float b2[3]) {
    float len = sqrtf(iv[0] * iv[0] + 0.0f * 0.0f + iv[2] * iv[2]);
    b1[0] = (0.0f - iv[2]) / len;
    b1[1] = 0.0f / len;
    b1[2] = iv[0] / len;
    b2[0] = iv[1] * b1[2] - iv[2] * b1[1];
    b2[1] = iv[2] * b1[0] - iv[0] * b1[2];
    b2[2] = iv[0] * b1[1] - iv[1] * b1[0];
}

static void compose_dir(const float b1[3], const float b2[3], const float iv[3], float st, float ct, float ph,
                        float out[3]) {
    float sph, cph;
    orc_sincos(ph, &sph, &cph);
    for (int k = 0; k < 3; ++k) out[k] = ((b1[k] * st) * cph + (b2[k] * st) * sph) + iv[k] * ct;
}

void orc_mie_sample(const orc_params *P, const float iv[3], float u1, float u2, float out[3]) {
    float th = orc_mie_sample_theta_bisect(P, u1) * ORC_PI;
    float ph = (2.0f * ORC_PI) * u2;
    float b1[3], b2[3];
    sampling_basis(iv, b1, b2);
    float s_, c_;
    orc_sincos(th, &s_, &c_);
    float ct = -c_; /* -cos_ps(): sign flip of the __m128 */
    float st = sqrtf(sse_max(1.0f - ct * ct, 0.0f));
    compose_dir(b1, b2, iv, st, ct, ph, out);
}

/* ---- exact-mode Mie sampler (DR_PHASE_MIE_EXACT) ---------------------------
 * Target density over phi = acos(-ct) in [0, pi] (phi = 0 is backscatter):
 * f(phi) sin(phi), with f the red channel of the table interpolated linearly in
 * phi exactly as MiePhase::Evaluate interpolates it (src/KernelSampler.cpp:
 * 214-231: knots at phi_k = k pi / n, the last bin extrapolating the line
 * through the last two entries).  Bin k carries f = f0 + beta (phi - phi_k) and
 * mass M_k = H_k(pi/n), where H_k(x) = int_0^x (f0 + beta s) sin(phi_k + s) ds
 *   = S [(f0 + beta x) sin x - beta (1 - cos x)]
 *   + C [f0 (1 - cos x) + beta (sin x - x cos x)],   S, C = sin, cos(phi_k).
 * The sampler inverts the CDF exactly: the bin by bisection on the
 * cumulative masses, then x in [0, pi/n] by safeguarded Newton on H_k.
 * Table (float): per bin (cdf_k, f0, beta, M_k), (S, C, pi/n, 0); then (1, 0, 0, 0). */
void orc_mie_exact_table(const float *pdf_rgb, uint32_t n, float *out) {
    const double dphi = 3.14159265358979323846 / (double)n;
    double *mass = (double *)malloc(sizeof(double) * n);
    double total = 0.0;
    for (uint32_t k = 0; k < n; ++k) {
        double fa, fb;
        if (k + 1 < n) {
            fa = pdf_rgb[3 * k];
            fb = pdf_rgb[3 * (k + 1)];
        } else {
            fa = pdf_rgb[3 * (n - 1)];
            fb = 2.0 * pdf_rgb[3 * (n - 1)] - pdf_rgb[3 * (n - 2)];
        }
        if (fa < 0.0) fa = 0.0;
        if (fb < 0.0) fb = 0.0;
        const double beta = (fb - fa) / dphi, phi = dphi * (double)k, x = dphi;
        const double S = sin(phi), C = cos(phi);
        const double m = S * ((fa + beta * x) * sin(x) - beta * (1.0 - cos(x))) +
                         C * (fa * (1.0 - cos(x)) + beta * (sin(x) - x * cos(x)));
        mass[k] = m > 0.0 ? m : 0.0;
        float *o = out + 8 * (size_t)k;
        o[1] = (float)fa;
        o[2] = (float)beta;
        o[3] = (float)mass[k];
        o[4] = (float)S;
        o[5] = (float)C;
        o[6] = (float)dphi;
        o[7] = 0.0f;
        total += mass[k];
    }
    double acc = 0.0;
    for (uint32_t k = 0; k < n; ++k) {
        out[8 * (size_t)k] = (float)(acc / total);
        acc += mass[k];
    }
    float *e = out + 8 * (size_t)n;
    e[0] = 1.0f;
    e[1] = e[2] = e[3] = 0.0f;
    free(mass);
}

/* sin x, 1 - cos x and sin x - x cos x by their Taylor series (x <= pi/4) */
static inline void local_trig(float x, float *sx, float *omc, float *sxc) {
    const float x2 = x * x;
    *sx = x * (1.0f - (x2 / 6.0f) * (1.0f - (x2 / 20.0f) * (1.0f - (x2 / 42.0f) * (1.0f - x2 / 72.0f))));
    *omc = (x2 / 2.0f) * (1.0f - (x2 / 12.0f) * (1.0f - (x2 / 30.0f) * (1.0f - (x2 / 56.0f) * (1.0f - x2 / 90.0f))));
    *sxc = ((x2 * x) / 3.0f) * (1.0f - (x2 / 10.0f) * (1.0f - (x2 / 28.0f) * (1.0f - x2 / 54.0f)));
}

/* ct = -cos(phi) and st = sin(phi) of the exact-mode sample for u1. */
void orc_mie_exact_dir(const float *tab, uint32_t n, float u1, float *ct, float *st) {
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (tab[8 * (size_t)mid] <= u1) lo = mid;
        else hi = mid - 1;
    }
    const float *b = tab + 8 * (size_t)lo;
    const float c0 = b[0], c1 = tab[8 * (size_t)(lo + 1)];
    const float f0 = b[1], beta = b[2], mk = b[3], S = b[4], C = b[5], dx = b[6];
    const float d = c1 - c0;
    const float up = d > 0.0f ? (u1 - c0) / d : 0.5f;
    const float m = up * mk;
    float xl = 0.0f, xh = dx, x = up * dx;
    for (int it = 0; it < 8; ++it) {
        float sx, omc, sxc;
        local_trig(x, &sx, &omc, &sxc);
        const float fx = f0 + beta * x;
        const float h = (S * (fx * sx - beta * omc) + C * (f0 * omc + beta * sxc)) - m;
        const float hp = fx * (S * (1.0f - omc) + C * sx);
        if (h > 0.0f) xh = x;
        else xl = x;
        float xn = hp > 0.0f ? x - h / hp : 0.5f * (xl + xh);
        if (!(xn > xl && xn < xh)) xn = 0.5f * (xl + xh);
        x = xn;
    }
    float sx, omc, sxc;
    local_trig(x, &sx, &omc, &sxc);
    const float cx = 1.0f - omc;
    *ct = 0.0f - (C * cx - S * sx);
    *st = sse_max(S * cx + C * sx, 0.0f);
}

void orc_mie_exact_dirs(const float *tab, uint32_t n, const float *u1, uint32_t count, float *ct, float *st) {
    for (uint32_t i = 0; i < count; ++i) orc_mie_exact_dir(tab, n, u1[i], &ct[i], &st[i]);
}

void orc_mie_sample_exact(const orc_params *P, const float iv[3], float u1, float u2, float out[3]) {
    float ct, st;
    orc_mie_exact_dir(P->mie_exact, P->mie_n, u1, &ct, &st);
    const float ph = (2.0f * ORC_PI) * u2;
    float b1[3], b2[3];
    sampling_basis(iv, b1, b2);
    compose_dir(b1, b2, iv, st, ct, ph, out);
}

void orc_sun_eval(const orc_params *P, const float rd[3], float out[3]) {
    int lt = dot3(rd, P->sun_dir) > P->sun_cos_angle;
    for (int k = 0; k < 3; ++k) out[k] = lt ? P->sun_color[k] : 0.0f;
}

float orc_sun_pdf(const orc_params *P, const float v[3]) {
    float ctm = P->sun_cos_angle;
    int lt = dot3(v, P->sun_dir) > ctm;
    return lt ? 1.0f / ((2.0f * ORC_PI) * (1.0f - ctm * ctm)) : 0.0f;
}

void orc_sun_sample(const orc_params *P, float u1, float u2, float out[3]) {
    float ctm = P->sun_cos_angle;
    float ct = (1.0f - u1) + u1 * ctm;
    float st = sqrtf(1.0f - ct * ct);
    float ph = (2.0f * ORC_PI) * u2;
    float b1[3], b2[3];
    sampling_basis(P->sun_dir, b1, b2);
    compose_dir(b1, b2, P->sun_dir, st, ct, ph, out);
}

void orc_sky_eval(const orc_params *P, const float rd[3], float out[3]) {
    const float *sd = P->sun_dir;
    float rdz = rd[2];
    float sth = sqrtf(1.0f - rd[2] * rd[2]);
    float cth = rdz;
    float slth = sqrtf(1.0f - sd[2] * sd[2]);
    float clth = sd[2];
    float slph = sd[1];
    float clph = sd[0];
    float rdd = rd[0] / rd[1];
    float acr = 1.0f / sqrtf(rdd * rdd + 1.0f);
    float czp = acr * (rdd * slph + clph);
    float cph = (sth * slth) * czp + cth * clth;
    float gmma = orc_acos_ref(cph);
    float gacs = sse_max(sse_min(cph, 1.0f), 0.0f);
    float thcs = sse_max(rdz, 0.0f);
    float raym = gacs * gacs;
    float zenh = sqrtf(thcs);
    float izen = 1.0f / (thcs + 0.01f); /* c1 / (thcs + 0.01) taken as c1 * izen (within an ulp) */
    for (int i = 0; i < 3; ++i) {
        const float *c = P->sky_cfg[i];
        float expm = orc_exp(c[4] * gmma);
        float miem = (1.0f + raym) / orc_pow15((1.0f + c[8] * c[8]) - (2.0f * c[8]) * gacs);
        float ca = (1.0f + c[0] * orc_exp(c[1] * izen)) *
                   ((((c[2] + c[3] * expm) + c[5] * raym) + c[6] * miem) + c[7] * zenh);
        ca = ca * P->sky_rad[i];
        out[i] = 1e-3f * orc_pow(ca, 2.2f);
    }
}

/* ---- HGPhase, src/KernelSampler.cpp:164-204 ------------------------------------
 * Evaluate: (1 - g g) / (4 SM_PI pow(1 + g g - 2 g ct, 1.5)), 4 SM_PI rounded to
 * binary32; Sample: sq = (1 - g g) / (1 - g + 2 g u1), ct = (1 + g g - sq sq) /
 * (2 g), composed with SamplingBasis like the Mie sampler. */
float orc_hg_eval(float g, float ct) {
    float den = 12.566371f * orc_pow15((1.0f + g * g) - (2.0f * g) * ct);
    return (1.0f - g * g) / den;
}

void orc_hg_sample(float g, const float iv[3], float u1, float u2, float out[3]) {
    float sq = (1.0f - g * g) / ((1.0f - g) + (2.0f * g) * u1);
    float ct = ((1.0f + g * g) - sq * sq) / (2.0f * g);
    float st = sqrtf(sse_max(1.0f - ct * ct, 0.0f));
    float b1[3], b2[3];
    sampling_basis(iv, b1, b2);
    compose_dir(b1, b2, iv, st, ct, (2.0f * ORC_PI) * u2, out);
}

void orc_phase_eval_rgb(const orc_params *P, float ct, float out[3]) {
    if (P->phase_mode == 2) {
        out[0] = out[1] = out[2] = orc_hg_eval(P->hg_g, ct);
        return;
    }
    orc_mie_eval_rgb(P, ct, out);
}

void orc_phase_sample(const orc_params *P, const float iv[3], float u1, float u2, float out[3]) {
    if (P->phase_mode == 2) orc_hg_sample(P->hg_g, iv, u1, u2, out);
    else if (P->phase_mode == 1) orc_mie_sample_exact(P, iv, u1, u2, out);
    else orc_mie_sample(P, iv, u1, u2, out);
}

/* atan2 of smmath.inl: a = min/max of |x|, |y|, the odd polynomial, then the
 * octant corrections (0.5 SM_PI and SM_PI rounded to binary32). */
float orc_atan2_ref(float y, float x) {
    float X = sse_max(0.0f - x, x), Y = sse_max(0.0f - y, y);
    float a = sse_min(X, Y) / sse_max(X, Y);
    float b = a * a;
    float p = -0.013480470f * b + 0.057477314f;
    p = p * b - 0.121239071f;
    p = p * b + 0.195635925f;
    p = p * b - 0.332994597f;
    p = p * b + 0.999995630f;
    a = a * p;
    if (Y > X) a = 1.57079637f - a;
    if (x < 0.0f) a = ORC_PI - a;
    if (y < 0.0f) a = 0.0f - a;
    return a;
}

/* MapEnv::Evaluate: theta row from acos(-rd.z) / pi, phi column from
 * 0.5 + atan2(rd.y, -rd.x) / (2 pi); saturate = max(min(x, 1), 0) (NaN -> 1);
 * texel indices formed in binary32 (w * row + column). */
void orc_env_map_eval(const orc_params *P, const float rd[3], float out[3]) {
    const float fw = (float)P->env_w, fh = (float)P->env_h;
    float tha = orc_acos_ref(0.0f - rd[2]) / ORC_PI;
    float thb = fh * sse_max(sse_min(tha, 1.0f), 0.0f);
    float thc = floorf(thb);
    thc = sse_min(thc, (float)(P->env_h - 2));
    thc = sse_max(thc, 0.0f);
    float tht = thb - thc;
    float pha = 0.5f + orc_atan2_ref(rd[1], 0.0f - rd[0]) / 6.2831855f;
    float phb = fw * sse_max(sse_min(pha, 1.0f), 0.0f);
    float phc = floorf(phb);
    phc = sse_min(phc, (float)(P->env_w - 2));
    phc = sse_max(phc, 0.0f);
    float pht = phb - phc;
    const float *T = P->env_map;
    const float *ca = T + 4 * (size_t)(uint32_t)(fw * thc + phc), *cb = T + 4 * (size_t)(uint32_t)(fw * (thc + 1.0f) + phc);
    const float *da = T + 4 * (size_t)(uint32_t)(fw * thc + phc + 1.0f),
                *db = T + 4 * (size_t)(uint32_t)(fw * (thc + 1.0f) + phc + 1.0f);
    for (int i = 0; i < 3; ++i) out[i] = lerp_ref(lerp_ref(ca[i], cb[i], tht), lerp_ref(da[i], db[i], tht), pht);
}

void orc_sky_light(const orc_params *P, const float rd[3], float out[3]) {
    if (P->env_mode == 0) {
        orc_sky_eval(P, rd, out);
        return;
    }
    float e[3] = {0.0f, 0.0f, 0.0f};
    if (P->env_mode == 2) orc_env_map_eval(P, rd, e);
    for (int i = 0; i < 3; ++i) out[i] = orc_pow(e[i], 2.2f);
}

/* K_ParallelRender ray generation for pixel (px, py), src/kernel.cpp:461-474 */
void orc_camera_ray(const orc_params *P, uint32_t px, uint32_t py, float ro[3], float rd[3], int *in_frame) {
    float hx = 0.0f - (((2.0f * ((float)px + 0.5f)) / (float)P->w) - 1.0f);
    float hy = 0.0f - (((2.0f * ((float)py + 0.5f)) / (float)P->h) - 1.0f);
    const float *V = P->viewi, *Q = P->proji;
    float rv[4], d[3];
    for (int k = 0; k < 4; ++k) rv[k] = ((hx * Q[k] + hy * Q[4 + k]) + 0.0f * Q[8 + k]) + 1.0f * Q[12 + k];
    for (int k = 0; k < 3; ++k) d[k] = ((rv[0] * V[k] + rv[1] * V[4 + k]) + rv[2] * V[8 + k]) + 0.0f * V[12 + k];
    float len = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int k = 0; k < 3; ++k) {
        rd[k] = d[k] / len;
        ro[k] = V[12 + k];
    }
    *in_frame = (hx > -1.0f && hx < 1.0f) && (hy > -1.0f && hy < 1.0f);
}

/* The scalar math of orc_math.h over an array (accuracy tests): kind 0 log,
 * 1 exp, 2 sin, 3 cos, 4 x^1.5, 5 x^2.2. */
void orc_math_eval(int kind, const float *x, uint32_t n, float *out) {
    for (uint32_t i = 0; i < n; ++i) {
        float s, c;
        switch (kind) {
        case 0: out[i] = orc_log(x[i]); break;
        case 1: out[i] = orc_exp(x[i]); break;
        case 2: orc_sincos(x[i], &s, &c); out[i] = s; break;
        case 3: orc_sincos(x[i], &s, &c); out[i] = c; break;
        case 4: out[i] = orc_pow15(x[i]); break;
        default: out[i] = orc_pow(x[i], 2.2f); break;
        }
    }
}
