/* ORACLE TEST INFRASTRUCTURE — restatement of the reference's parametric
 * octree traversal (Revelles et al., "An efficient parametric algorithm for
 * octree traversal", 2000) as implemented in src/KernelOctree.cpp:
 *
 *   OctreeFirstNode   src/KernelOctree.cpp:9-34
 *   OctreeNextNode    src/KernelOctree.cpp:62-71
 *   OctreeInitialize  src/KernelOctree.cpp:78-110
 *   OctreeStepTraverser::Initialize / OctreeProcessSubtree
 *                     src/KernelOctree.cpp:230-349
 *
 * Same binary32 operations in the same order, so leaf sequences and the
 * (tr0, tr1) interval of each leaf are bit-identical to the reference.  One
 * deliberate difference: a root that is itself a leaf is reported once and
 * the iteration ends, where the reference underflows its stack level.
 */
#include "oracle.h"
#include <math.h>
#include <stddef.h>

static inline float smax_(float a, float b) { return (a < b) ? b : a; } /* std::max */
static inline float smin_(float a, float b) { return (b < a) ? b : a; } /* std::min */

static uint32_t first_node(const float t0[3], const float tm[3]) {
    uint32_t a = 0;
    if (t0[0] > t0[1]) {
        if (t0[0] > t0[2]) {
            if (tm[1] < t0[0]) a |= 2;
            if (tm[2] < t0[0]) a |= 1;
            return a;
        }
    } else {
        if (t0[1] > t0[2]) {
            if (tm[0] < t0[1]) a |= 4;
            if (tm[2] < t0[1]) a |= 1;
            return a;
        }
    }
    if (tm[0] < t0[2]) a |= 4;
    if (tm[1] < t0[2]) a |= 2;
    return a;
}

static uint32_t next_node(const float tm[3], uint32_t x, uint32_t y, uint32_t z) {
    if (tm[0] < tm[1]) {
        if (tm[0] < tm[2]) return x;
    } else {
        if (tm[1] < tm[2]) return y;
    }
    return z;
}

static const uint32_t NLA[8] = {0, 4, 2, 6, 1, 5, 3, 7};

typedef struct {
    float t0[ORC_MAX_DEPTH][3], t1[ORC_MAX_DEPTH][3], tm[ORC_MAX_DEPTH][3];
    uint32_t n[ORC_MAX_DEPTH], tn[ORC_MAX_DEPTH];
    int p[ORC_MAX_DEPTH];
    uint32_t a;
    int l;
    int active;
} trav;

static void trav_init(trav *T, const orc_node *nodes, const float ro[3], const float rd[3]) {
    const float *ce = nodes[0].ce;
    float ros[3], rds[3];
    for (int k = 0; k < 3; ++k) {
        ros[k] = (ro[k] - ce[k]) + ce[3];
        rds[k] = rd[k];
    }
    uint32_t a = 0;
    static const uint32_t bit[3] = {4, 2, 1};
    for (int k = 0; k < 3; ++k)
        if (rds[k] < 0.0f) {
            ros[k] = 2.0f * ce[3] - ros[k];
            rds[k] = -rds[k];
            a |= bit[k];
        }
    float mx = 2.0f * ce[3];
    for (int k = 0; k < 3; ++k) {
        T->t0[0][k] = (0.0f - ros[k]) / rds[k];
        T->t1[0][k] = (mx - ros[k]) / rds[k];
    }
    T->a = a;
    T->active = 0;
    if (smax_(smax_(T->t0[0][0], T->t0[0][1]), T->t0[0][2]) < smin_(smin_(T->t1[0][0], T->t1[0][1]), T->t1[0][2])) {
        T->active = 1;
        T->l = 0;
        T->n[0] = 0;
        T->p[0] = 0;
    }
}

static void set3(float d[3], float x, float y, float z) { d[0] = x; d[1] = y; d[2] = z; }

/* Returns 1 with the next leaf, 0 when the ray has no more leaves. */
static int trav_next(trav *T, const orc_node *nodes, uint32_t *node, float *tr0, float *tr1, uint64_t *visits) {
    if (!T->active) return 0;
    const uint32_t a = T->a;
    for (;;) {
        int l = T->l;
        if (T->p[l]) {
            uint32_t tn = T->tn[l];
            if (tn >= 8) {
                if (l == 0) { T->active = 0; return 0; }
                T->l = l - 1;
                continue;
            }
            float *t0 = T->t0[l], *t1 = T->t1[l], *tm = T->tm[l];
            float *c0 = T->t0[l + 1], *c1 = T->t1[l + 1];
            uint32_t q0, q1, q2;
            switch (tn) {
            case 0: set3(c0, t0[0], t0[1], t0[2]); set3(c1, tm[0], tm[1], tm[2]); q0 = 4; q1 = 2; q2 = 1; break;
            case 1: set3(c0, t0[0], t0[1], tm[2]); set3(c1, tm[0], tm[1], t1[2]); q0 = 5; q1 = 3; q2 = 8; break;
            case 2: set3(c0, t0[0], tm[1], t0[2]); set3(c1, tm[0], t1[1], tm[2]); q0 = 6; q1 = 8; q2 = 3; break;
            case 3: set3(c0, t0[0], tm[1], tm[2]); set3(c1, tm[0], t1[1], t1[2]); q0 = 7; q1 = 8; q2 = 8; break;
            case 4: set3(c0, tm[0], t0[1], t0[2]); set3(c1, t1[0], tm[1], tm[2]); q0 = 8; q1 = 6; q2 = 5; break;
            case 5: set3(c0, tm[0], t0[1], tm[2]); set3(c1, t1[0], tm[1], t1[2]); q0 = 8; q1 = 7; q2 = 8; break;
            case 6: set3(c0, tm[0], tm[1], t0[2]); set3(c1, t1[0], t1[1], tm[2]); q0 = 8; q1 = 8; q2 = 7; break;
            default: set3(c0, tm[0], tm[1], tm[2]); set3(c1, t1[0], t1[1], t1[2]); q0 = q1 = q2 = 8; break;
            }
            T->tn[l] = (tn == 7) ? 8 : next_node(c1, q0, q1, q2);
            T->n[l + 1] = nodes[T->n[l]].chn[NLA[tn ^ a]];
            T->p[l + 1] = 0;
            T->l = l + 1;
        } else {
            float *t0 = T->t0[l], *t1 = T->t1[l];
            uint32_t n = T->n[l];
            if (t1[0] < 0.0f || t1[1] < 0.0f || t1[2] < 0.0f || (n == 0 && l > 0)) {
                if (l == 0) { T->active = 0; return 0; }
                T->l = l - 1;
                continue;
            }
            if (visits) ++*visits;
            const orc_node *o = &nodes[n];
            if (o->volx[ORC_SDF] != ORC_NONE || o->volx[ORC_FOG] != ORC_NONE) {
                *node = n;
                *tr0 = smax_(smax_(t0[0], t0[1]), t0[2]);
                *tr1 = smin_(smin_(t1[0], t1[1]), t1[2]);
                if (l == 0) T->active = 0; /* root leaf: report once */
                else T->l = l - 1;
                return 1;
            }
            float *tm = T->tm[l];
            if (l + 1 >= ORC_MAX_DEPTH) { T->active = 0; return 0; }
            for (int k = 0; k < 3; ++k) tm[k] = 0.5f * (t0[k] + t1[k]);
            T->tn[l] = first_node(t0, tm);
            T->p[l] = 1;
        }
    }
}

/* public wrappers over an opaque state, used by the estimator */
typedef trav orc_trav_state;
size_t orc_trav_size(void) { return sizeof(trav); }
void orc_trav_init(void *T, const orc_node *nodes, const float ro[3], const float rd[3]) {
    trav_init((trav *)T, nodes, ro, rd);
}
int orc_trav_next(void *T, const orc_node *nodes, uint32_t *node, float *tr0, float *tr1, uint64_t *visits) {
    return trav_next((trav *)T, nodes, node, tr0, tr1, visits);
}

uint32_t orc_leaf_sequence(const orc_node *nodes, const float ro[3], const float rd[3], uint32_t maxn,
                           uint32_t *out_nodes, float *out_tr0, float *out_tr1) {
    trav T;
    trav_init(&T, nodes, ro, rd);
    uint32_t n = 0;
    while (n < maxn && trav_next(&T, nodes, &out_nodes[n], &out_tr0[n], &out_tr1[n], 0)) ++n;
    return n;
}

uint32_t orc_point_lookup(const orc_node *nodes, const double p[3], int *depth) {
    uint32_t n = 0;
    int l = 0;
    for (;;) {
        const orc_node *o = &nodes[n];
        if (o->volx[ORC_SDF] != ORC_NONE || o->volx[ORC_FOG] != ORC_NONE) break;
        const double e = (double)o->ce[3];
        for (int k = 0; k < 3; ++k)
            if (p[k] < (double)o->ce[k] - e || p[k] > (double)o->ce[k] + e) {
                if (depth) *depth = l;
                return ORC_NONE;
            }
        uint32_t i = (p[0] > (double)o->ce[0] ? 1u : 0u) | (p[1] > (double)o->ce[1] ? 2u : 0u) |
                     (p[2] > (double)o->ce[2] ? 4u : 0u);
        uint32_t c = o->chn[i];
        if (c == 0) {
            if (depth) *depth = l + 1;
            return ORC_NONE;
        }
        n = c;
        ++l;
    }
    if (depth) *depth = l;
    return n;
}
