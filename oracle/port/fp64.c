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
