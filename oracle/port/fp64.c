/* ORACLE TEST INFRASTRUCTURE — FP64 references for the transmittance and
 * gradient gates.
 *
 * The medium seen by the tracker is, inside each leaf the ray visits, the
 * trilinear interpolant of that leaf's brick (src/kernel.cpp:96-126 with the
 * index clamps), and empty between leaves.  Along a ray the interpolant is a
 * polynomial of degree <= 3 between brick-cell planes, so 3-point
 * Gauss-Legendre on every cell segment integrates it exactly in FP64.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

static double dens64(const double p[3], const float *v, const float ce[4], uint32_t N, double *w8, uint32_t *i8) {
    const double e = ce[3];
    double nl[3];
    uint32_t a[3], b[3];
    for (int k = 0; k < 3; ++k) {
        double ni = (p[k] - ((double)ce[k] - e)) * (double)(N - 1) / (2.0 * e);
        double nf = floor(ni), nc = ceil(ni);
        if (nf < 0) nf = 0;
        if (nc > N - 1) nc = N - 1;
        nl[k] = ni - nf;
        if (nc < 0) nc = 0;
        if (nf > N - 1) nf = N - 1;
        a[k] = (uint32_t)nf;
        b[k] = (uint32_t)nc;
    }
    double acc = 0.0;
    for (int c = 0; c < 8; ++c) {
        uint32_t x = (c & 1) ? b[0] : a[0], y = (c & 2) ? b[1] : a[1], z = (c & 4) ? b[2] : a[2];
        double wx = (c & 1) ? nl[0] : 1.0 - nl[0];
        double wy = (c & 2) ? nl[1] : 1.0 - nl[1];
        double wz = (c & 4) ? nl[2] : 1.0 - nl[2];
        /* when a == b the two corners coincide and their weights sum to 1 */
        double w = wx * wy * wz;
        uint32_t idx = z * N * N + y * N + x;
        acc += w * (double)v[idx];
        if (w8) {
            w8[c] = w;
            i8[c] = idx;
        }
    }
    return acc;
}

static int cmpd(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* Splits [ta, tb] at brick-cell planes of leaf o and calls fn on each piece. */
typedef void (*seg_fn)(void *ctx, double t0, double t1, const orc_node *o, const float *brick, uint32_t N);

static void for_cell_segments(const orc_scene *S, const orc_node *o, const double ro[3], const double rd[3],
                              double ta, double tb, seg_fn fn, void *ctx) {
    const uint32_t N = S->lvoxc;
    const float *brick = S->bricks + (size_t)o->volx[ORC_FOG] * N * N * N;
    double cuts[3 * 64 + 2];
    int nc = 0;
    cuts[nc++] = ta;
    const double e = o->ce[3];
    for (int k = 0; k < 3; ++k) {
        if (rd[k] == 0.0) continue;
        for (uint32_t j = 1; j + 1 < N; ++j) {
            double plane = ((double)o->ce[k] - e) + 2.0 * e * (double)j / (double)(N - 1);
            double t = (plane - ro[k]) / rd[k];
            if (t > ta && t < tb && nc < 3 * 64) cuts[nc++] = t;
        }
    }
    cuts[nc++] = tb;
    qsort(cuts, (size_t)nc, sizeof(double), cmpd);
    for (int i = 0; i + 1 < nc; ++i)
        if (cuts[i + 1] > cuts[i]) fn(ctx, cuts[i], cuts[i + 1], o, brick, N);
}

static const double GL_X[3] = {-0.7745966692414834, 0.0, 0.7745966692414834};
static const double GL_W[3] = {0.5555555555555556, 0.8888888888888888, 0.5555555555555556};

typedef struct {
    const double *ro, *rd;
    double acc;
} od_ctx;

static void od_seg(void *vctx, double t0, double t1, const orc_node *o, const float *brick, uint32_t N) {
    od_ctx *c = (od_ctx *)vctx;
    double h = 0.5 * (t1 - t0), m = 0.5 * (t1 + t0);
    for (int g = 0; g < 3; ++g) {
        double t = m + h * GL_X[g];
        double p[3] = {c->ro[0] + c->rd[0] * t, c->ro[1] + c->rd[1] * t, c->ro[2] + c->rd[2] * t};
        c->acc += h * GL_W[g] * dens64(p, brick, o->ce, N, 0, 0);
    }
}

double orc_optical_depth(const orc_scene *S, const double ro[3], const double rd[3], double tmax) {
    float rof[3] = {(float)ro[0], (float)ro[1], (float)ro[2]}, rdf[3] = {(float)rd[0], (float)rd[1], (float)rd[2]};
    uint32_t nodes[4096];
    float tr0[4096], tr1[4096];
    uint32_t n = orc_leaf_sequence(S->nodes, rof, rdf, 4096, nodes, tr0, tr1);
    od_ctx c = {ro, rd, 0.0};
    for (uint32_t i = 0; i < n; ++i) {
        const orc_node *o = &S->nodes[nodes[i]];
        if (o->volx[ORC_FOG] == ORC_NONE || o->qval[ORC_FOG] == 0.0f) continue;
        if (!isfinite(tr0[i]) || !isfinite(tr1[i])) continue; /* axis-parallel rays: NaN intervals */
        double ta = tr0[i] > 0.0f ? (double)tr0[i] : 0.0, tb = (double)tr1[i] < tmax ? (double)tr1[i] : tmax;
        if (tb > ta) for_cell_segments(S, o, ro, rd, ta, tb, od_seg, &c);
    }
    return c.acc;
}

typedef struct {
    const double *ro, *rd;
    double *grad;     /* per brick value: d(optical depth)/d(value) */
    uint32_t lv3;
} gr_ctx;

static void gr_seg(void *vctx, double t0, double t1, const orc_node *o, const float *brick, uint32_t N) {
    gr_ctx *c = (gr_ctx *)vctx;
    double h = 0.5 * (t1 - t0), m = 0.5 * (t1 + t0);
    for (int g = 0; g < 3; ++g) {
        double t = m + h * GL_X[g];
        double p[3] = {c->ro[0] + c->rd[0] * t, c->ro[1] + c->rd[1] * t, c->ro[2] + c->rd[2] * t};
        double w8[8];
        uint32_t i8[8];
        dens64(p, brick, o->ce, N, w8, i8);
        for (int k = 0; k < 8; ++k) c->grad[(size_t)o->volx[ORC_FOG] * c->lv3 + i8[k]] += h * GL_W[g] * w8[k];
    }
}

/* d(optical depth)/d(brick value) for every brick value, accumulated into
 * grad (n_leaves * lvoxc^3 doubles, caller-zeroed).  The transmittance
 * gradient is -sigma_t * T * grad. */
void orc_optical_depth_grad(const orc_scene *S, const double ro[3], const double rd[3], double tmax, double *grad) {
    float rof[3] = {(float)ro[0], (float)ro[1], (float)ro[2]}, rdf[3] = {(float)rd[0], (float)rd[1], (float)rd[2]};
    uint32_t nodes[4096];
    float tr0[4096], tr1[4096];
    uint32_t n = orc_leaf_sequence(S->nodes, rof, rdf, 4096, nodes, tr0, tr1);
    gr_ctx c = {ro, rd, grad, S->lvoxc * S->lvoxc * S->lvoxc};
    for (uint32_t i = 0; i < n; ++i) {
        const orc_node *o = &S->nodes[nodes[i]];
        if (o->volx[ORC_FOG] == ORC_NONE || o->qval[ORC_FOG] == 0.0f) continue;
        if (!isfinite(tr0[i]) || !isfinite(tr1[i])) continue; /* axis-parallel rays: NaN intervals */
        double ta = tr0[i] > 0.0f ? (double)tr0[i] : 0.0, tb = (double)tr1[i] < tmax ? (double)tr1[i] : tmax;
        if (tb > ta) for_cell_segments(S, o, ro, rd, ta, tb, gr_seg, &c);
    }
}

/* ---- single-scatter sun image by quadrature (the adjoint's independent check) ----
 * With scattevs = 1 the estimator (src/kernel.cpp:128-445, restated in
 * render.c) adds sun light to a camera path only through the shadow ray of
 * its first real collision: per path, E[sun_c] = f sun_c p_hit
 *   int sigma_t rho(t) T0(t) E_lrd[ p3_c/(p3_c + p2) T_sh(x(t), lrd) ] dt,
 * with T0 the camera ray's transmittance to t, lrd uniform in the sun cone
 * (u1, u2 of orc_sun_sample), p3 = phase(lrd . rd), p2 = the sun Pdf, and
 * p_hit the probability that a sampled lrd passes the cone test (a rim
 * rounding effect, estimated by the caller).  The continuation reaches the
 * sun only through the cone's solid angle times its MIS weight (about 1e-6 of
 * the shadow-ray term for the check's geometry): left out.  Every factor that
 * depends on the brick samples is an FP64 quadrature: 3-point Gauss-Legendre
 * on each brick-cell segment (cubic density, smooth transmittance), and the
 * cone by nu x nphi Gauss-Legendre x midpoint nodes.  The gradient is the
 * exact derivative of the quadrature. */

typedef struct {
    const double *ro, *rd;
    double *grad;     /* accumulated: scale * d(optical depth)/d(value) */
    double scale;
    uint32_t lv3;
} sgr_ctx;

static void sgr_seg(void *vctx, double t0, double t1, const orc_node *o, const float *brick, uint32_t N) {
    sgr_ctx *c = (sgr_ctx *)vctx;
    double h = 0.5 * (t1 - t0), m = 0.5 * (t1 + t0);
    for (int g = 0; g < 3; ++g) {
        double t = m + h * GL_X[g];
        double p[3] = {c->ro[0] + c->rd[0] * t, c->ro[1] + c->rd[1] * t, c->ro[2] + c->rd[2] * t};
        double w8[8];
        uint32_t i8[8];
        dens64(p, brick, o->ce, N, w8, i8);
        for (int k = 0; k < 8; ++k)
            c->grad[(size_t)o->volx[ORC_FOG] * c->lv3 + i8[k]] += c->scale * h * GL_W[g] * w8[k];
    }
}

/* optical depth from ro along rd (to infinity); with grad, adds scale * d/dv */
static double od_scaled(const orc_scene *S, const double ro[3], const double rd[3], double *grad, double scale) {
    float rof[3] = {(float)ro[0], (float)ro[1], (float)ro[2]}, rdf[3] = {(float)rd[0], (float)rd[1], (float)rd[2]};
    uint32_t nodes[4096];
    float tr0[4096], tr1[4096];
    uint32_t n = orc_leaf_sequence(S->nodes, rof, rdf, 4096, nodes, tr0, tr1);
    od_ctx c = {ro, rd, 0.0};
    sgr_ctx g = {ro, rd, grad, scale, S->lvoxc * S->lvoxc * S->lvoxc};
    for (uint32_t i = 0; i < n; ++i) {
        const orc_node *o = &S->nodes[nodes[i]];
        if (o->volx[ORC_FOG] == ORC_NONE || o->qval[ORC_FOG] == 0.0f) continue;
        if (!isfinite(tr0[i]) || !isfinite(tr1[i])) continue;
        double ta = tr0[i] > 0.0f ? (double)tr0[i] : 0.0, tb = (double)tr1[i];
        if (!(tb > ta)) continue;
        if (grad) for_cell_segments(S, o, ro, rd, ta, tb, sgr_seg, &g);
        else for_cell_segments(S, o, ro, rd, ta, tb, od_seg, &c);
    }
    if (grad) { /* the value as well */
        for (uint32_t i = 0; i < n; ++i) {
            const orc_node *o = &S->nodes[nodes[i]];
            if (o->volx[ORC_FOG] == ORC_NONE || o->qval[ORC_FOG] == 0.0f) continue;
            if (!isfinite(tr0[i]) || !isfinite(tr1[i])) continue;
            double ta = tr0[i] > 0.0f ? (double)tr0[i] : 0.0, tb = (double)tr1[i];
            if (tb > ta) for_cell_segments(S, o, ro, rd, ta, tb, od_seg, &c);
        }
    }
    return c.acc;
}

/* one collision node of the camera ray: position, density, trilinear weights,
 * quadrature weight, and the optical depth from the camera to it */
typedef struct {
    double t, w, rho, tau;
    double w8[8];
    uint32_t i8[8];
    uint32_t brick;
} cnode;

typedef struct {
    const double *ro, *rd;
    cnode *nodes;
    uint32_t n, cap;
    double tau_start;   /* optical depth at the start of the current segment */
} cam_ctx;

static void cam_seg(void *vctx, double t0, double t1, const orc_node *o, const float *brick, uint32_t N) {
    cam_ctx *c = (cam_ctx *)vctx;
    double h = 0.5 * (t1 - t0), m = 0.5 * (t1 + t0);
    for (int g = 0; g < 3 && c->n < c->cap; ++g) {
        cnode *q = &c->nodes[c->n++];
        q->t = m + h * GL_X[g];
        q->w = h * GL_W[g];
        double p[3] = {c->ro[0] + c->rd[0] * q->t, c->ro[1] + c->rd[1] * q->t, c->ro[2] + c->rd[2] * q->t};
        q->rho = dens64(p, brick, o->ce, N, q->w8, q->i8);
        q->brick = o->volx[ORC_FOG];
        /* optical depth from the segment start to q->t: the density is a cubic
         * in t on the segment, so 3-point Gauss-Legendre on [t0, t] is exact */
        double hh = 0.5 * (q->t - t0), mm = 0.5 * (q->t + t0), acc = 0.0;
        for (int k = 0; k < 3; ++k) {
            double s = mm + hh * GL_X[k];
            double ps[3] = {c->ro[0] + c->rd[0] * s, c->ro[1] + c->rd[1] * s, c->ro[2] + c->rd[2] * s};
            acc += hh * GL_W[k] * dens64(ps, brick, o->ce, N, 0, 0);
        }
        q->tau = c->tau_start + acc;
    }
    double full = 0.0;
    for (int k = 0; k < 3; ++k) {
        double s = m + h * GL_X[k];
        double ps[3] = {c->ro[0] + c->rd[0] * s, c->ro[1] + c->rd[1] * s, c->ro[2] + c->rd[2] * s};
        full += h * GL_W[k] * dens64(ps, brick, o->ce, N, 0, 0);
    }
    c->tau_start += full;
}

/* adds scale * d(tau from the camera to node q)/dv into grad */
static void cam_tau_grad(const orc_scene *S, const double ro[3], const double rd[3], const cnode *nodes, uint32_t upto,
                         double tq, double *grad, double scale) {
    /* every node before q covers whole cell segments up to q's segment; the
     * segment holding q contributes [t0, tq]: recompute by walking the leaf list */
    float rof[3] = {(float)ro[0], (float)ro[1], (float)ro[2]}, rdf[3] = {(float)rd[0], (float)rd[1], (float)rd[2]};
    uint32_t ln[4096];
    float tr0[4096], tr1[4096];
    uint32_t n = orc_leaf_sequence(S->nodes, rof, rdf, 4096, ln, tr0, tr1);
    sgr_ctx g = {ro, rd, grad, scale, S->lvoxc * S->lvoxc * S->lvoxc};
    (void)nodes;
    (void)upto;
    for (uint32_t i = 0; i < n; ++i) {
        const orc_node *o = &S->nodes[ln[i]];
        if (o->volx[ORC_FOG] == ORC_NONE || o->qval[ORC_FOG] == 0.0f) continue;
        if (!isfinite(tr0[i]) || !isfinite(tr1[i])) continue;
        double ta = tr0[i] > 0.0f ? (double)tr0[i] : 0.0, tb = (double)tr1[i] < tq ? (double)tr1[i] : tq;
        if (tb > ta) for_cell_segments(S, o, ro, rd, ta, tb, sgr_seg, &g);
    }
}

/* For each camera ray r (ro, rd: float32, as the kernel generates them):
 * out[3 r + c] = E[sun_c] per path sample / (f sun_c p_hit) scaled back in,
 * i.e. the expected sun sum of one sample; with grad (n_leaves * lvoxc^3
 * doubles, caller-zeroed), adds d(sum_r sum_c wc[c] out[3 r + c])/dv. */
void orc_single_scatter_sun(const orc_scene *S, const orc_params *P, const float *ro, const float *rd, uint32_t n_rays,
                            double p_hit, uint32_t nu, uint32_t nphi, const double wc[3], double *out, double *grad) {
    const double st = (double)(P->sigma_s + P->sigma_a);
    const float f = P->sigma_s / (P->sigma_a + P->sigma_s);
    enum { CAP = 3 * 4096 };
    cnode *nodes = (cnode *)malloc(sizeof(cnode) * CAP);
    /* cone nodes: u1 by Gauss-Legendre on [0, 1], u2 by the midpoint rule */
    const uint32_t nd = nu * nphi;
    float (*ld)[3] = (float (*)[3])malloc(sizeof(float) * 3 * nd);
    double *lw = (double *)malloc(sizeof(double) * nd);
    static const double X4[4] = {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526};
    static const double W4[4] = {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538};
    for (uint32_t a = 0; a < nu; ++a)
        for (uint32_t b = 0; b < nphi; ++b) {
            const double x = nu == 4 ? X4[a] : (nu == 3 ? GL_X[a] : 0.0);
            const double w = nu == 4 ? W4[a] : (nu == 3 ? GL_W[a] : 2.0);
            orc_sun_sample(P, (float)(0.5 + 0.5 * x), (float)((b + 0.5) / nphi), ld[a * nphi + b]);
            lw[a * nphi + b] = 0.5 * w / nphi;
        }
    const float p2 = orc_sun_pdf(P, P->sun_dir);  /* the Pdf of any direction inside the cone */
    for (uint32_t r = 0; r < n_rays; ++r) {
        const double o[3] = {ro[3 * r], ro[3 * r + 1], ro[3 * r + 2]}, d[3] = {rd[3 * r], rd[3 * r + 1], rd[3 * r + 2]};
        /* collision nodes along the camera ray */
        float rof[3] = {ro[3 * r], ro[3 * r + 1], ro[3 * r + 2]}, rdf[3] = {rd[3 * r], rd[3 * r + 1], rd[3 * r + 2]};
        uint32_t ln[4096];
        float tr0[4096], tr1[4096];
        uint32_t nl = orc_leaf_sequence(S->nodes, rof, rdf, 4096, ln, tr0, tr1);
        cam_ctx cc = {o, d, nodes, 0, CAP, 0.0};
        for (uint32_t i = 0; i < nl; ++i) {
            const orc_node *q = &S->nodes[ln[i]];
            if (q->volx[ORC_FOG] == ORC_NONE || q->qval[ORC_FOG] == 0.0f) continue;
            if (!isfinite(tr0[i]) || !isfinite(tr1[i])) continue;
            double ta = tr0[i] > 0.0f ? (double)tr0[i] : 0.0, tb = (double)tr1[i];
            if (tb > ta) for_cell_segments(S, q, o, d, ta, tb, cam_seg, &cc);
        }
        double acc[3] = {0, 0, 0};
        for (uint32_t j = 0; j < cc.n; ++j) {
            const cnode *q = &nodes[j];
            if (q->rho == 0.0) continue;
            const double T0 = exp(-st * q->tau);
            const double x[3] = {o[0] + d[0] * q->t, o[1] + d[1] * q->t, o[2] + d[2] * q->t};
            double G[3] = {0, 0, 0};
            double gsh[64][3];
            double tsh[64];
            for (uint32_t k = 0; k < nd && k < 64; ++k) {
                const double ldd[3] = {ld[k][0], ld[k][1], ld[k][2]};
                tsh[k] = exp(-st * od_scaled(S, x, ldd, 0, 0.0));
                float p3[3];
                orc_phase_eval_rgb(P, ld[k][0] * rdf[0] + ld[k][1] * rdf[1] + ld[k][2] * rdf[2], p3);
                for (int c = 0; c < 3; ++c) {
                    gsh[k][c] = (double)(p3[c] / (p3[c] + p2));
                    G[c] += lw[k] * gsh[k][c] * tsh[k];
                }
            }
            const double base = q->w * st * q->rho * T0;
            for (int c = 0; c < 3; ++c) acc[c] += base * G[c];
            if (!grad) continue;
            const double k3 = (double)f * p_hit;
            double wg = 0.0;  /* sum_c wc sun_c G_c */
            for (int c = 0; c < 3; ++c) wg += wc[c] * (double)P->sun_color[c] * G[c];
            const uint32_t lv3 = S->lvoxc * S->lvoxc * S->lvoxc;
            /* d rho at the node */
            for (int k = 0; k < 8; ++k)
                grad[(size_t)q->brick * lv3 + q->i8[k]] += k3 * q->w * st * q->w8[k] * T0 * wg;
            /* d T0: -sigma_t T0 d tau(camera -> t) */
            cam_tau_grad(S, o, d, nodes, j, q->t, grad, -k3 * base * st * wg);
            /* d T_sh per cone direction */
            for (uint32_t k = 0; k < nd && k < 64; ++k) {
                double wk = 0.0;
                for (int c = 0; c < 3; ++c) wk += wc[c] * (double)P->sun_color[c] * gsh[k][c];
                const double ldd[3] = {ld[k][0], ld[k][1], ld[k][2]};
                od_scaled(S, x, ldd, grad, -k3 * base * lw[k] * wk * tsh[k] * st);
            }
        }
        for (int c = 0; c < 3; ++c) out[3 * r + c] = (double)f * p_hit * (double)P->sun_color[c] * acc[c];
    }
    free(nodes);
    free(ld);
    free(lw);
}

/* Fraction of n sun-cone samples (u1, u2 on a stratified n1 x n2 grid of
 * cell midpoints) that pass the cone's own strict test: p_hit above. */
double orc_sun_hit_fraction(const orc_params *P, uint32_t n1, uint32_t n2) {
    uint64_t hit = 0;
    for (uint32_t a = 0; a < n1; ++a)
        for (uint32_t b = 0; b < n2; ++b) {
            float d[3];
            orc_sun_sample(P, (float)((a + 0.5) / n1), (float)((b + 0.5) / n2), d);
            hit += orc_sun_pdf(P, d) > 0.0f;
        }
    return (double)hit / ((double)n1 * n2);
}
