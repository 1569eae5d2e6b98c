/* ORACLE TEST INFRASTRUCTURE — the reference estimator (SampleVolume,
 * src/kernel.cpp:128-445) restated as an iterative per-path loop.
 *
 * Recursion unrolled: SampleVolume(r) returns, per sample,
 *   escaped & r>0 : sun(rd) into the sun buffer, sky(rd) into the sky buffer
 *   collided & r<scattevs : (S1 w1 + S2 w2) sigma_s/sigma_t, where S1 is the
 *       continuation SampleVolume(r+1) along the phase sample and S2 the
 *       shadow SampleVolume(scattevs) along the sun sample (sky of S2 dropped)
 *   otherwise 0;  alpha = 1 iff the camera segment collided (r = 0).
 * Written as a throughput loop: shadow rays add T * w2 * f * sun(lrd) when
 * they escape, T *= w1 * f, f = sigma_s/sigma_t (src/kernel.cpp:387-441).
 *
 * Tracking (src/kernel.cpp:207-317, fog-only leaves): a leaf ahead of the
 * current position is entered at its entry distance (empty space skipped);
 * a leaf the ray is already inside continues from the current position; a
 * candidate with sc <= tr0 collides without a density lookup; otherwise it is
 * accepted when rho/smax >= q.
 */
#include "oracle.h"
#include "orc_math.h"
#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

size_t orc_trav_size(void);
void orc_trav_init(void *T, const orc_node *nodes, const float ro[3], const float rd[3]);
int orc_trav_next(void *T, const orc_node *nodes, uint32_t *node, float *tr0, float *tr1, uint64_t *visits);

static inline float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* Visitor of the collision decisions that involved a density lookup (the
 * adjoint's gradient scatter); NULL for rendering. */
typedef void (*orc_visit_fn)(void *ctx, const float *brick, const float ce[4], const float rc[3], float rho,
                             float smax, int real);

static int track_depth_v(const orc_scene *S, const orc_params *P, const float ro[3], const float rd[3], orc_rng *g,
                         float depth, float *td_out, orc_counters *cnt, orc_visit_fn visit, void *vctx);

static int track_depth(const orc_scene *S, const orc_params *P, const float ro[3], const float rd[3], orc_rng *g,
                       float depth, float *td_out, orc_counters *cnt) {
    return track_depth_v(S, P, ro, rd, g, depth, td_out, cnt, 0, 0);
}

static int track_depth_v(const orc_scene *S, const orc_params *P, const float ro[3], const float rd[3], orc_rng *g,
                         float depth, float *td_out, orc_counters *cnt, orc_visit_fn visit, void *vctx) {
    const float sigma_e = P->sigma_a + P->sigma_s;
    const uint32_t N = S->lvoxc, lv3 = N * N * N;
    _Alignas(16) unsigned char tbuf[2048];
    void *T = tbuf;
    orc_trav_init(T, S->nodes, ro, rd);
    if (cnt) cnt->vertices++;
    float td = 0.0f;
    uint32_t node;
    float tra, trb;
    for (;;) {
        if (!orc_trav_next(T, S->nodes, &node, &tra, &trb, cnt ? &cnt->node_visits : 0)) break;
        if (!(td < depth)) break;
        const orc_node *o = &S->nodes[node];
        const float lo = td;
        const float tr0 = tra - td, tr1 = trb - td;
        /* src/kernel.cpp:245-251: a leaf with a surface brick takes majorant 1 */
        const int sdf = o->volx[ORC_SDF] != ORC_NONE && S->sdf_bricks, fog = o->volx[ORC_FOG] != ORC_NONE;
        const float *sbrick = sdf ? S->sdf_bricks + (size_t)o->volx[ORC_SDF] * lv3 : 0;
        const float smax = sdf ? 1.0f : o->qval[ORC_FOG];
        float s0;
        if (sdf) {
            /* src/kernel.cpp:253-263: sm = (tra > td) & (d0 > 0) with d0 the
             * distance at the leaf entry (a full mask: VM is 0) */
            int skip = 0;
            if (tra > td) {
                float r0[3];
                for (int k = 0; k < 3; ++k) r0[k] = ro[k] + rd[k] * tra;
                skip = orc_sample_voxel_space(r0, sbrick, o->ce, N) > 0.0f;
                if (cnt) cnt->density_lookups++;
            }
            if (skip) {
                td = tra;
                s0 = tr0;
            } else {
                s0 = 0.0f;
            }
        } else if (tra > td) {
            /* src/kernel.cpp:241-265: sm = (tra > td) | VM with VM the integer 1 for
             * fog leaves, so the masked selects below are bitwise blends: past the
             * leaf entry, td keeps all but its lowest bit and s0 becomes the lowest
             * bit of tr0 (0 or the smallest denormal). */
            td = tra;
            s0 = tr0;
        } else {
            td = orc_u2f((orc_f2u(td) & ~1u) | (orc_f2u(tra) & 1u));
            s0 = orc_u2f(orc_f2u(tr0) & 1u);
        }
        const float *brick = fog ? S->bricks + (size_t)o->volx[ORC_FOG] * lv3 : 0;
        const float denom = sigma_e * smax;
        float sr = -orc_log(orc_rng_uniform(g)) / denom;
        for (;;) {
            const float sc = s0 + sr;
            td = lo + sc;
            if (!(sc < tr1)) {
                td = trb;
                break;
            }
            int rm = sc > tr0;
            float rho = -1.0f, dist = 1.0f;
            int fog_decides = rm;
            if (rm) {
                float rc[3];
                for (int k = 0; k < 3; ++k) rc[k] = ro[k] + rd[k] * td;
                if (sdf) {
                    /* src/kernel.cpp:287-300: inside the surface (dist <= 0) always
                     * collides; outside, the fog brick (if any) decides */
                    dist = orc_sample_voxel_space(rc, sbrick, o->ce, N);
                    if (cnt) cnt->density_lookups++;
                    fog_decides = dist > 0.0f && fog;
                    if (fog_decides) {
                        rho = orc_sample_voxel_space(rc, brick, o->ce, N);
                        if (cnt) cnt->density_lookups++;
                    }
                } else {
                    rho = orc_sample_voxel_space(rc, brick, o->ce, N);
                    if (cnt) cnt->density_lookups++;
                }
            }
            const float q = orc_rng_uniform(g);
            rm = rm && (rho / smax < q) && (dist > 0.0f);
            if (fog_decides && visit) {
                float rc[3];
                for (int k = 0; k < 3; ++k) rc[k] = ro[k] + rd[k] * td;
                visit(vctx, brick, o->ce, rc, rho, smax, !rm);
            }
            if (!rm) {
                /* src/kernel.cpp:214-217, 370-384: the lane's mask mm = td < depth
                 * is re-evaluated on the next leaf step; alpha is taken from rm
                 * first (1: collided), then rm |= !mm makes a collision at or
                 * beyond the depth no scattering event (2). */
                *td_out = td;
                return td < depth ? 0 : 2;
            }
            sr = sr - orc_log(orc_rng_uniform(g)) / denom;
        }
    }
    *td_out = td;
    return 1;
}

/* ---- occluders: SceneOcclusion::Intersect (src/SceneOcclusion.cpp:58-91) ----
 * Embree's query (tnear 0, tfar MAX_OCCLUSION_DIST = 1e6) answers whether the
 * ray hits any occluder triangle.  Restated as Moller-Trumbore (1997) without
 * culling, the division by the determinant folded into the comparisons. */
static int occ_triangle(const float *T, const float o[3], const float d[3]) {
    const float *a = T, *e1 = T + 4, *e2 = T + 8;
    const float px = d[1] * e2[2] - d[2] * e2[1], py = d[2] * e2[0] - d[0] * e2[2], pz = d[0] * e2[1] - d[1] * e2[0];
    const float det = e1[0] * px + e1[1] * py + e1[2] * pz;
    const float sx = o[0] - a[0], sy = o[1] - a[1], sz = o[2] - a[2];
    const float u = sx * px + sy * py + sz * pz;
    const float qx = sy * e1[2] - sz * e1[1], qy = sz * e1[0] - sx * e1[2], qz = sx * e1[1] - sy * e1[0];
    const float v = d[0] * qx + d[1] * qy + d[2] * qz;
    const float t = e2[0] * qx + e2[1] * qy + e2[2] * qz;
    const float uv = u + v;
    if (det > 0.0f) return u >= 0.0f && v >= 0.0f && uv <= det && t >= 0.0f && t <= det * 1e6f;
    if (det < 0.0f) return u <= 0.0f && v <= 0.0f && uv >= det && t <= 0.0f && t >= det * 1e6f;
    return 0;
}

int orc_occluded(const orc_scene *S, const float o[3], const float d[3]) {
    for (uint32_t i = 0; i < S->occ_n; ++i)
        if (occ_triangle(S->occ_tris + 12 * (size_t)i, o, d)) return 1;
    return 0;
}

int orc_occluded_fp64(const orc_scene *S, const double o[3], const double d[3], double *margin) {
    int hit = 0;
    double best = 1e300;
    for (uint32_t i = 0; i < S->occ_n; ++i) {
        const float *T = S->occ_tris + 12 * (size_t)i;
        double a[3], e1[3], e2[3];
        for (int k = 0; k < 3; ++k) {
            a[k] = T[k];
            e1[k] = T[4 + k]; /* the triangle (v0, v0 + e1, v0 + e2) the binary32 test sees, exactly */
            e2[k] = T[8 + k];
        }
        const double p[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
        const double det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2];
        if (det == 0.0) continue;
        const double s[3] = {o[0] - a[0], o[1] - a[1], o[2] - a[2]};
        const double u = (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) / det;
        const double q[3] = {s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
        const double v = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) / det;
        const double t = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) / det;
        if (t < -1e-9 || t > 1e6) continue;
        double m = u < v ? u : v;
        if (1.0 - u - v < m) m = 1.0 - u - v;
        const double am = m < 0 ? -m : m;
        if (am < best) best = am;
        if (m >= 0.0 && t >= 0.0) hit = 1;
    }
    if (margin) *margin = best;
    return hit;
}

/* The shadow pass's segment of one (pixel, sample): origin on the camera ray at
 * the pixel's depth and the sun-cone direction (orc_shadow_path's first steps);
 * returns whether the pixel has geometry before the far plane. */
int orc_shadow_ray(const orc_params *P, uint32_t px, uint32_t py, uint64_t seed, uint64_t sample, float ro1[3],
                   float lrd[3]) {
    float ro[3], rd[3];
    int inf;
    orc_camera_ray(P, px, py, ro, rd, &inf);
    const float zz = P->proji[8 + 2] + P->proji[12 + 2], zw = P->proji[8 + 3] + P->proji[12 + 3];
    const float clip_end = -zz / zw;
    const float depth = P->depth_map ? P->depth_map[(size_t)py * P->w + px] : FLT_MAX;
    orc_rng g;
    orc_rng_seed(&g, seed, (uint64_t)py * P->w + px, sample);
    const float u3 = orc_rng_uniform(&g), u4 = orc_rng_uniform(&g);
    orc_sun_sample(P, u3, u4, lrd);
    for (int k = 0; k < 3; ++k) ro1[k] = ro[k] + rd[k] * depth;
    return inf && depth < clip_end;
}

static inline int occ_blocks(const orc_scene *S, const orc_params *P, const float o[3], const float d[3]) {
    return P->embree && S->occ_n && orc_occluded(S, o, d);
}

int orc_track(const orc_scene *S, const orc_params *P, const float ro[3], const float rd[3], void *rng, float *td,
              orc_counters *cnt) {
    return track_depth(S, P, ro, rd, (orc_rng *)rng, FLT_MAX, td, cnt) != 0;
}

void orc_render_path(const orc_scene *S, const orc_params *P, uint32_t px, uint32_t py, uint64_t seed,
                     uint64_t sample, float out_sun[4], float out_sky[4], orc_counters *cnt) {
    for (int k = 0; k < 4; ++k) out_sun[k] = out_sky[k] = 0.0f;
    float ro[3], rd[3];
    int inf;
    orc_camera_ray(P, px, py, ro, rd, &inf);
    if (!inf) return;
    orc_rng g;
    orc_rng_seed(&g, seed, (uint64_t)py * P->w + px, sample);
    if (cnt) cnt->paths++;
    const float f = P->sigma_s / (P->sigma_a + P->sigma_s);
    const float depth0 = (P->depth_map && P->depthcomp) ? P->depth_map[(size_t)py * P->w + px] : P->depth;
    float T[3] = {1.0f, 1.0f, 1.0f};
    uint32_t r = 0;
    for (;;) {
        float td;
        int esc = track_depth(S, P, ro, rd, &g, r == 0 ? depth0 : FLT_MAX, &td, cnt);
        /* alpha: the camera segment collided (1) or escaped (0); a collision at
         * or beyond the depth counts as 1, except in the USE_EMBREE build whose
         * depth mask zeroes it (src/kernel.cpp:379) */
        if (r == 0) out_sun[3] = out_sky[3] = (esc == 0 || (esc == 2 && !P->embree)) ? 1.0f : 0.0f;
        if (esc == 2) break;
        if (esc) {
            if (r > 0 && !occ_blocks(S, P, ro, rd)) {
                float sun[3], sky[3];
                orc_sun_eval(P, rd, sun);
                orc_sky_light(P, rd, sky);
                for (int k = 0; k < 3; ++k) {
                    out_sun[k] = out_sun[k] + T[k] * sun[k];
                    out_sky[k] = out_sky[k] + T[k] * sky[k];
                }
            }
            break;
        }
        if (r >= P->scattevs) break;
        float srd[3], lrd[3], p1[3], p3[3], rc[3];
        const float u1 = orc_rng_uniform(&g), u2 = orc_rng_uniform(&g);
        orc_phase_sample(P, rd, u1, u2, srd);
        const float u3 = orc_rng_uniform(&g), u4 = orc_rng_uniform(&g);
        orc_sun_sample(P, u3, u4, lrd);
        orc_phase_eval_rgb(P, dot3(srd, rd), p1);
        const float p2 = orc_sun_pdf(P, lrd);
        orc_phase_eval_rgb(P, dot3(lrd, rd), p3);
        const float q1 = orc_sun_pdf(P, srd);
        if (cnt) cnt->mie_evals += 3;
        for (int k = 0; k < 3; ++k) rc[k] = ro[k] + rd[k] * td;
        float tds;
        if (track_depth(S, P, rc, lrd, &g, FLT_MAX, &tds, cnt) && !occ_blocks(S, P, rc, lrd)) {
            float sun[3];
            orc_sun_eval(P, lrd, sun);
            for (int k = 0; k < 3; ++k) out_sun[k] = out_sun[k] + (T[k] * ((p3[k] / (p3[k] + p2)) * f)) * sun[k];
        }
        for (int k = 0; k < 3; ++k) {
            T[k] = T[k] * ((p1[k] / (p1[k] + q1)) * f);
            ro[k] = rc[k];
            rd[k] = srd[k];
        }
        ++r;
    }
    /* the reference's sky term is 0/0 for rd.y == 0 (rd.x / rd.y times 0,
     * src/kernel.cpp:338-342); with finite_paths such a sample adds nothing */
    if (P->finite_paths) {
        int ok = 1;
        for (int k = 0; k < 3; ++k) ok = ok && isfinite(out_sun[k]) && isfinite(out_sky[k]);
        if (!ok)
            for (int k = 0; k < 3; ++k) out_sun[k] = out_sky[k] = 0.0f;
    }
}

/* RenderKernel::Shadow for one (pixel, sample), src/kernel.cpp:569-607.  The
 * camera ray is cut at the pixel's depth when that lies before the far clip
 * plane (clip_end = -z/w of (0,0,1,1) * projInv); from there one shadow segment
 * runs along a sun-cone sample with r = scattevs (SampleVolume: escape gives
 * sun(lrd), a collision 0).  A pixel without geometry in front of the far plane
 * traces nothing and gets sun(lrd), as its mask lane keeps "not scattering".
 * The result is divided by float4::load(&color), whose w is 0: alpha becomes
 * 1/0 = +inf per sample (scattevs > 0: the r > 0 branch sets alpha 1 on every
 * lane), rgb = sun(lrd) / colour. */
void orc_shadow_path(const orc_scene *S, const orc_params *P, uint32_t px, uint32_t py, uint64_t seed,
                     uint64_t sample, float out[4], orc_counters *cnt) {
    for (int k = 0; k < 4; ++k) out[k] = 0.0f;
    float ro[3], rd[3];
    int inf;
    orc_camera_ray(P, px, py, ro, rd, &inf);
    if (!inf) return;
    if (cnt) cnt->paths++;
    const float zz = P->proji[8 + 2] + P->proji[12 + 2], zw = P->proji[8 + 3] + P->proji[12 + 3];
    const float clip_end = -zz / zw;
    const float depth = P->depth_map ? P->depth_map[(size_t)py * P->w + px] : FLT_MAX;
    const int active = depth < clip_end;
    orc_rng g;
    orc_rng_seed(&g, seed, (uint64_t)py * P->w + px, sample);
    const float u3 = orc_rng_uniform(&g), u4 = orc_rng_uniform(&g);
    float lrd[3];
    orc_sun_sample(P, u3, u4, lrd);
    int esc = 1, occ = 0;
    if (active) {
        float ro1[3], td;
        for (int k = 0; k < 3; ++k) ro1[k] = ro[k] + rd[k] * depth;
        esc = track_depth(S, P, ro1, lrd, &g, FLT_MAX, &td, cnt);
        /* USE_EMBREE build: an escaped segment whose ray hits an occluder
         * gathers nothing, alpha included (src/kernel.cpp:375-383) */
        occ = esc == 1 && occ_blocks(S, P, ro1, lrd);
    }
    float lc[3] = {0.0f, 0.0f, 0.0f};
    if (P->scattevs > 0 && esc && !occ) orc_sun_eval(P, lrd, lc);
    const float color_w = 0.0f;
    const float a = ((P->scattevs > 0 || !esc) && !occ) ? 1.0f : 0.0f;
    for (int k = 0; k < 3; ++k) out[k] = lc[k] / P->sun_color[k];
    out[3] = a / color_w;
}

typedef struct {
    const orc_scene *S;
    const orc_params *P;
    uint32_t x0, y0, tw, th, spp, rows;
    uint64_t seed, base;
    float *sun, *sky;
    orc_counters cnt;
    int next_row_mod, nthreads, tid;
    int shadow;
} tile_job;

static void *tile_worker(void *arg) {
    tile_job *J = (tile_job *)arg;
    const uint32_t cols = 2 * (J->tw / 2);
    for (uint32_t j = (uint32_t)J->tid; j < J->rows; j += (uint32_t)J->nthreads) {
        for (uint32_t i = 0; i < cols; ++i) {
            float acc_sun[4] = {0, 0, 0, 0}, acc_sky[4] = {0, 0, 0, 0};
            int any = 0;
            for (uint32_t s = 0; s < J->spp; ++s) {
                float a[4], b[4];
                float ro[3], rd[3];
                int inf;
                orc_camera_ray(J->P, J->x0 + i, J->y0 + j, ro, rd, &inf);
                if (!inf) break;
                any = 1;
                if (J->shadow) {
                    orc_shadow_path(J->S, J->P, J->x0 + i, J->y0 + j, J->seed, J->base + s, a, &J->cnt);
                    for (int k = 0; k < 4; ++k) b[k] = 0.0f;
                } else {
                    orc_render_path(J->S, J->P, J->x0 + i, J->y0 + j, J->seed, J->base + s, a, b, &J->cnt);
                }
                for (int k = 0; k < 4; ++k) {
                    acc_sun[k] += a[k];
                    acc_sky[k] += b[k];
                }
            }
            if (any) {
                memcpy(&J->sun[4 * ((size_t)j * J->tw + i)], acc_sun, 16);
                if (J->sky) memcpy(&J->sky[4 * ((size_t)j * J->tw + i)], acc_sky, 16);
            }
        }
    }
    return 0;
}

static int tile_run(const orc_scene *S, const orc_params *P, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th,
                    uint32_t spp, uint64_t seed, uint64_t sample_base, float *out_sun, float *out_sky,
                    orc_counters *cnt, int nthreads, int shadow) {
    memset(out_sun, 0, sizeof(float) * 4 * (size_t)tw * th);
    if (out_sky) memset(out_sky, 0, sizeof(float) * 4 * (size_t)tw * th);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    tile_job jobs[256];
    pthread_t th_ids[256];
    for (int t = 0; t < nthreads; ++t) {
        tile_job *J = &jobs[t];
        memset(J, 0, sizeof(*J));
        J->S = S; J->P = P; J->x0 = x0; J->y0 = y0; J->tw = tw; J->th = th; J->spp = spp;
        J->rows = 2 * (th / 2); J->seed = seed; J->base = sample_base; J->sun = out_sun; J->sky = out_sky;
        J->nthreads = nthreads; J->tid = t; J->shadow = shadow;
    }
    for (int t = 1; t < nthreads; ++t) pthread_create(&th_ids[t], 0, tile_worker, &jobs[t]);
    tile_worker(&jobs[0]);
    for (int t = 1; t < nthreads; ++t) pthread_join(th_ids[t], 0);
    if (cnt) {
        for (int t = 0; t < nthreads; ++t) {
            cnt->vertices += jobs[t].cnt.vertices;
            cnt->node_visits += jobs[t].cnt.node_visits;
            cnt->density_lookups += jobs[t].cnt.density_lookups;
            cnt->mie_evals += jobs[t].cnt.mie_evals;
            cnt->paths += jobs[t].cnt.paths;
        }
    }
    return 0;
}

int orc_render_tile_mt(const orc_scene *S, const orc_params *P, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th,
                       uint32_t spp, uint64_t seed, uint64_t sample_base, float *out_sun, float *out_sky,
                       orc_counters *cnt, int nthreads) {
    return tile_run(S, P, x0, y0, tw, th, spp, seed, sample_base, out_sun, out_sky, cnt, nthreads, 0);
}

int orc_shadow_tile_mt(const orc_scene *S, const orc_params *P, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th,
                       uint32_t spp, uint64_t seed, uint64_t sample_base, float *out, orc_counters *cnt,
                       int nthreads) {
    return tile_run(S, P, x0, y0, tw, th, spp, seed, sample_base, out, 0, cnt, nthreads, 1);
}

int orc_render_tile(const orc_scene *S, const orc_params *P, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th,
                    uint32_t spp, uint64_t seed, uint64_t sample_base, float *out_sun, float *out_sky,
                    orc_counters *cnt) {
    return orc_render_tile_mt(S, P, x0, y0, tw, th, spp, seed, sample_base, out_sun, out_sky, cnt, 1);
}

/* Fraction of nrays x nsamp delta-tracked segments from ro along rd that
 * escape, using streams (seed, ray, sample).  Used by the transmittance gate. */
double orc_transmittance_mc(const orc_scene *S, const orc_params *P, const float ro[3], const float rd[3],
                            uint64_t seed, uint64_t nsamp) {
    uint64_t esc = 0;
    for (uint64_t s = 0; s < nsamp; ++s) {
        orc_rng g;
        orc_rng_seed(&g, seed, 0, s);
        float td;
        esc += (uint64_t)track_depth(S, P, ro, rd, &g, FLT_MAX, &td, 0);
    }
    return (double)esc / (double)nsamp;
}


/* ---- path-replay adjoint ---------------------------------------------------------
 * The same estimator gradient as the GPU's adjoint (score-function form over
 * the delta-tracking decisions, majorants fixed; C_after weights; albedo via
 * the count of f factors), with the same float operations, so per-path totals
 * and scattered terms equal the GPU's; the gradient sums are doubles here. */

/* corner offsets and trilinear weights of orc_sample_voxel_space */
static void voxel_weights(const float p[3], const float ce[4], uint32_t N, uint32_t idx[8], float w[8]) {
    const float nm1 = (float)N - 1.0f;
    const float top = (float)(N - 1);
    uint32_t ia[3], ib[3];
    float nl[3];
    for (int k = 0; k < 3; ++k) {
        float ni = ((-0.5f * ((ce[k] - ce[3]) - p[k])) * nm1) / ce[3];
        float nf = floorf(ni) > 0.0f ? floorf(ni) : 0.0f;
        float nc = ceilf(ni) < nm1 ? ceilf(ni) : nm1;
        nl[k] = ni - nf;
        nc = nc < top ? nc : top;
        nc = nc > 0.0f ? nc : 0.0f;
        nf = nf < top ? nf : top;
        nf = nf > 0.0f ? nf : 0.0f;
        ia[k] = (uint32_t)nf;
        ib[k] = (uint32_t)nc;
    }
    for (int c = 0; c < 8; ++c) {
        uint32_t x = (c & 1) ? ib[0] : ia[0], y = (c & 2) ? ib[1] : ia[1], z = (c & 4) ? ib[2] : ia[2];
        idx[c] = (z * N + y) * N + x;
        w[c] = ((c & 1) ? nl[0] : 1.0f - nl[0]) * ((c & 2) ? nl[1] : 1.0f - nl[1]) * ((c & 4) ? nl[2] : 1.0f - nl[2]);
    }
}

typedef struct {
    float w;
    double *grad;
    const float *bricks;
    uint32_t N;
} scatter_ctx;

static void scatter_visit(void *vctx, const float *brick, const float ce[4], const float rc[3], float rho, float smax,
                          int real) {
    scatter_ctx *c = (scatter_ctx *)vctx;
    if (c->w == 0.0f) return;
    float sc;
    if (real) {
        if (!(rho > 0.0f)) return;
        sc = c->w / rho;
    } else {
        const float d = smax - rho;
        if (!(d > 0.0f)) return;
        sc = (0.0f - c->w) / d;
    }
    uint32_t idx[8];
    float wt[8];
    voxel_weights(rc, ce, c->N, idx, wt);
    double *gb = c->grad + (brick - c->bricks);
    for (int k = 0; k < 8; ++k)
        if (wt[k] != 0.0f) gb[idx[k]] += (double)(sc * wt[k]);
}

static inline float dot3v(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* reweighted replay: each decision drawn from S->bricks is weighted by its
 * probability under pert over its probability under S->bricks */
typedef struct {
    float w;
    const float *pert, *bricks;
    uint32_t N;
} ratio_ctx;

static void ratio_visit(void *vctx, const float *brick, const float ce[4], const float rc[3], float rho, float smax,
                        int real) {
    ratio_ctx *c = (ratio_ctx *)vctx;
    const float rp = orc_sample_voxel_space(rc, c->pert + (brick - c->bricks), ce, c->N);
    if (real) {
        if (rho > 0.0f) c->w = c->w * (rp / rho);
    } else {
        const float d = smax - rho;
        if (d > 0.0f) c->w = c->w * ((smax - rp) / d);
    }
}

/* pass 0 fills tot[12] (sun, sky, m*sun, m*sky); pass 1 scatters with tot known;
 * pass 2 fills tot[0..5] with the reweighted replay's contribution (pert) */
static void adjoint_pass(const orc_scene *S, const orc_params *P, uint32_t px, uint32_t py, uint64_t seed,
                         uint64_t sample, const float dsun[3], const float dsky[3], float tot[12], double *grad,
                         int pass, const float *pert) {
    const int scatter = pass == 1, ratio = pass == 2;
    float ro[3], rd[3];
    int inf;
    orc_camera_ray(P, px, py, ro, rd, &inf);
    if (!inf) return;
    orc_rng g;
    orc_rng_seed(&g, seed, (uint64_t)py * P->w + px, sample);
    const float f = P->sigma_s / (P->sigma_a + P->sigma_s);
    const float depth0 = (P->depth_map && P->depthcomp) ? P->depth_map[(size_t)py * P->w + px] : P->depth;
    float T[3] = {1.0f, 1.0f, 1.0f};
    float acc_sun[3] = {0, 0, 0}, acc_sky[3] = {0, 0, 0}, a_sun[3] = {0, 0, 0}, a_sky[3] = {0, 0, 0};
    scatter_ctx sc = {0.0f, grad, S->bricks, S->lvoxc};
    for (uint32_t r = 0;; ++r) {
        float td;
        int res;
        if (scatter) {
            /* C_after weight: the path's total weight minus what it added before */
            const float wtot = dot3v(dsun, tot) + dot3v(dsky, tot + 3);
            sc.w = wtot - (dot3v(dsun, acc_sun) + dot3v(dsky, acc_sky));
            res = track_depth_v(S, P, ro, rd, &g, r == 0 ? depth0 : FLT_MAX, &td, 0, scatter_visit, &sc);
        } else if (ratio) {
            ratio_ctx rv = {1.0f, pert, S->bricks, S->lvoxc};
            res = track_depth_v(S, P, ro, rd, &g, r == 0 ? depth0 : FLT_MAX, &td, 0, ratio_visit, &rv);
            for (int k = 0; k < 3; ++k) T[k] = T[k] * rv.w;
        } else {
            res = track_depth_v(S, P, ro, rd, &g, r == 0 ? depth0 : FLT_MAX, &td, 0, 0, 0);
        }
        if (res == 2) break;
        if (res == 1) {
            if (r > 0 && !occ_blocks(S, P, ro, rd)) {
                float sun[3], sky[3];
                orc_sun_eval(P, rd, sun);
                orc_sky_light(P, rd, sky);
                const float m = (float)r;
                for (int k = 0; k < 3; ++k) {
                    const float cs = T[k] * sun[k], ck = T[k] * sky[k];
                    acc_sun[k] = acc_sun[k] + cs;
                    acc_sky[k] = acc_sky[k] + ck;
                    a_sun[k] = a_sun[k] + m * cs;
                    a_sky[k] = a_sky[k] + m * ck;
                }
            }
            break;
        }
        if (r >= P->scattevs) break;
        float srd[3], lrd[3], p1[3], p3[3], rc[3];
        const float u1 = orc_rng_uniform(&g), u2 = orc_rng_uniform(&g);
        orc_phase_sample(P, rd, u1, u2, srd);
        const float u3 = orc_rng_uniform(&g), u4 = orc_rng_uniform(&g);
        orc_sun_sample(P, u3, u4, lrd);
        orc_phase_eval_rgb(P, dot3(srd, rd), p1);
        const float p2 = orc_sun_pdf(P, lrd);
        orc_phase_eval_rgb(P, dot3(lrd, rd), p3);
        const float q1 = orc_sun_pdf(P, srd);
        for (int k = 0; k < 3; ++k) rc[k] = ro[k] + rd[k] * td;
        const orc_rng g0 = g;
        float tds;
        ratio_ctx rs = {1.0f, pert, S->bricks, S->lvoxc};
        if (track_depth_v(S, P, rc, lrd, &g, FLT_MAX, &tds, 0, ratio ? ratio_visit : 0, ratio ? &rs : 0) == 1 &&
            !occ_blocks(S, P, rc, lrd)) {
            float sun[3], cn[3];
            orc_sun_eval(P, lrd, sun);
            for (int k = 0; k < 3; ++k) cn[k] = (T[k] * ((p3[k] / (p3[k] + p2)) * f)) * sun[k];
            if (ratio)
                for (int k = 0; k < 3; ++k) cn[k] = cn[k] * rs.w;
            if (scatter) {
                scatter_ctx sv = {dot3v(dsun, cn), grad, S->bricks, S->lvoxc};
                if (sv.w != 0.0f) {
                    orc_rng g1 = g0;
                    float t2;
                    (void)track_depth_v(S, P, rc, lrd, &g1, FLT_MAX, &t2, 0, scatter_visit, &sv);
                }
            }
            const float m = (float)(r + 1);
            for (int k = 0; k < 3; ++k) {
                acc_sun[k] = acc_sun[k] + cn[k];
                a_sun[k] = a_sun[k] + m * cn[k];
            }
        }
        for (int k = 0; k < 3; ++k) {
            T[k] = T[k] * ((p1[k] / (p1[k] + q1)) * f);
            ro[k] = rc[k];
            rd[k] = srd[k];
        }
    }
    if (!scatter) { /* passes 0 and 2 */
        for (int k = 0; k < 3; ++k) {
            tot[k] = acc_sun[k];
            tot[3 + k] = acc_sky[k];
            tot[6 + k] = a_sun[k];
            tot[9 + k] = a_sky[k];
        }
    }
}

typedef struct {
    const orc_scene *S;
    const orc_params *P;
    uint32_t x0, y0, tw, spp, cols, rows;
    uint64_t seed, base;
    const float *dsun, *dsky;
    double *grad, galb;
    int nthreads, tid;
} adj_job;

static void *adj_worker(void *arg) {
    adj_job *J = (adj_job *)arg;
    const float f = J->P->sigma_s / (J->P->sigma_a + J->P->sigma_s);
    for (uint32_t j = (uint32_t)J->tid; j < J->rows; j += (uint32_t)J->nthreads)
        for (uint32_t i = 0; i < J->cols; ++i) {
            const float *ds = J->dsun + 4 * ((size_t)j * J->tw + i), *dk = J->dsky + 4 * ((size_t)j * J->tw + i);
            if (dot3v(ds, ds) + dot3v(dk, dk) > 0.0f)
                for (uint32_t s = 0; s < J->spp; ++s) {
                    float tot[12] = {0};
                    adjoint_pass(J->S, J->P, J->x0 + i, J->y0 + j, J->seed, J->base + s, ds, dk, tot, J->grad, 0, 0);
                    int ok = 1;
                    for (int k = 0; k < 6; ++k) ok = ok && isfinite(tot[k]);
                    if (!ok) continue; /* non-finite contribution: left out of the gradient */
                    adjoint_pass(J->S, J->P, J->x0 + i, J->y0 + j, J->seed, J->base + s, ds, dk, tot, J->grad, 1, 0);
                    J->galb += (double)((dot3v(ds, tot + 6) + dot3v(dk, tot + 9)) / f);
                }
        }
    return 0;
}

int orc_adjoint_tile_mt(const orc_scene *S, const orc_params *P, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th,
                        uint32_t spp, uint64_t seed, uint64_t sample_base, const float *dsun, const float *dsky,
                        double *grad, double *galb, int nthreads) {
    const size_t ng = (size_t)S->n_leaves * S->lvoxc * S->lvoxc * S->lvoxc;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 64) nthreads = 64;
    adj_job jobs[64];
    pthread_t ids[64];
    for (int t = 0; t < nthreads; ++t) {
        adj_job *J = &jobs[t];
        memset(J, 0, sizeof(*J));
        J->S = S; J->P = P; J->x0 = x0; J->y0 = y0; J->tw = tw; J->spp = spp;
        J->cols = 2 * (tw / 2); J->rows = 2 * (th / 2); J->seed = seed; J->base = sample_base;
        J->dsun = dsun; J->dsky = dsky; J->nthreads = nthreads; J->tid = t;
        J->grad = t == 0 ? grad : (double *)calloc(ng, sizeof(double));
        if (!J->grad) return -1;
    }
    for (int t = 1; t < nthreads; ++t) pthread_create(&ids[t], 0, adj_worker, &jobs[t]);
    adj_worker(&jobs[0]);
    for (int t = 1; t < nthreads; ++t) pthread_join(ids[t], 0);
    double ga = 0.0;
    for (int t = 0; t < nthreads; ++t) {
        ga += jobs[t].galb;
        if (t > 0) {
            for (size_t k = 0; k < ng; ++k) grad[k] += jobs[t].grad[k];
            free(jobs[t].grad);
        }
    }
    *galb += ga;
    return 0;
}

/* Linearised loss of the reweighted replay (the GPU's dr_reweighted_loss_async):
 * sum over the tile's paths of dsun . C_sun + dsky . C_sky, decisions from
 * S->bricks weighted by their probability ratios under pert; a path whose
 * contribution is not finite is left out. */
double orc_reweighted_loss(const orc_scene *S, const orc_params *P, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th,
                           uint32_t spp, uint64_t seed, uint64_t sample_base, const float *dsun, const float *dsky,
                           const float *pert) {
    double l = 0.0;
    const uint32_t cols = 2 * (tw / 2), rows = 2 * (th / 2);
    for (uint32_t j = 0; j < rows; ++j)
        for (uint32_t i = 0; i < cols; ++i) {
            const float *ds = dsun + 4 * ((size_t)j * tw + i), *dk = dsky + 4 * ((size_t)j * tw + i);
            if (!(dot3v(ds, ds) + dot3v(dk, dk) > 0.0f)) continue;
            for (uint32_t s = 0; s < spp; ++s) {
                float tot[12] = {0};
                adjoint_pass(S, P, x0 + i, y0 + j, seed, sample_base + s, ds, dk, tot, 0, 2, pert);
                int ok = 1;
                for (int k = 0; k < 6; ++k) ok = ok && isfinite(tot[k]);
                if (ok) l += (double)(dot3v(ds, tot) + dot3v(dk, tot + 3));
            }
        }
    return l;
}

/* Gradient of sum_r w_r T_r over the brick samples (streams (seed, r, s)). */
void orc_adjoint_transmittance(const orc_scene *S, const orc_params *P, const float *ro, const float *rd,
                               const float *wr, uint32_t n, uint64_t nsamp, uint64_t seed, double *grad, double *T) {
    for (uint32_t r = 0; r < n; ++r) {
        uint64_t esc = 0;
        scatter_ctx sv = {wr[r] / (float)nsamp, grad, S->bricks, S->lvoxc};
        for (uint64_t s = 0; s < nsamp; ++s) {
            orc_rng g;
            orc_rng_seed(&g, seed, r, s);
            const orc_rng g0 = g;
            float td;
            if (track_depth_v(S, P, ro + 3 * r, rd + 3 * r, &g, FLT_MAX, &td, 0, 0, 0) == 1) {
                ++esc;
                orc_rng g1 = g0;
                (void)track_depth_v(S, P, ro + 3 * r, rd + 3 * r, &g1, FLT_MAX, &td, 0, scatter_visit, &sv);
            }
        }
        if (T) T[r] = (double)esc / (double)nsamp;
    }
}
