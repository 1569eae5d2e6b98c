/* ORACLE TEST INFRASTRUCTURE — restatement of the OpenVDB-free part of the
 * reference scene build (src/scene.cpp), used to feed the compiled reference
 * renderer and to pin the product's octree builder.
 *
 *   leaf boxes        src/scene.cpp:676-701  (active bbox of each 8^3 leaf)
 *   root box, depth   src/scene.cpp:703-716
 *   Octree::BuildPath src/scene.cpp:267-305  (1.1x child boxes, DFS numbering)
 *   BoundingBox::Intersects(BoundingBox) src/scene.cpp:230-243
 *   brick resampling  src/scene.cpp:870-908  (loop over [0, index), which skips
 *                     the last-created node; that leaf keeps majorant 0)
 *
 * OpenVDB arithmetic that the reference relies on (not present here, so this
 * boundary is unpinned): leaf iteration order of a Tree4<float,5,4,3>,
 * CoordBBox::getCenter/dim, UniformScaleMap index<->world maps and the
 * BoxSampler trilinear interpolation (z, then y, then x; weights in double).
 */
#include "oracle.h"
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>

#define LVC 8

typedef struct {
    int32_t ox, oy, oz;
    uint32_t idx;
} blk_key;

static uint64_t vdb_order_key(const blk_key *k) {
    /* Tree4<float,5,4,3>: root map (x,y,z lexicographic on 4096-aligned
     * origins), then 32^3 children x-major, then 16^3 leaves x-major. */
    uint64_t x = (uint32_t)k->ox, y = (uint32_t)k->oy, z = (uint32_t)k->oz;
    uint64_t key = 0;
    key = (x >> 12);
    key = (key << 8) | (y >> 12);
    key = (key << 8) | (z >> 12);
    key = (key << 5) | ((x >> 7) & 31);
    key = (key << 5) | ((y >> 7) & 31);
    key = (key << 5) | ((z >> 7) & 31);
    key = (key << 4) | ((x >> 3) & 15);
    key = (key << 4) | ((y >> 3) & 15);
    key = (key << 4) | ((z >> 3) & 15);
    return key;
}

static int cmp_blk(const void *a, const void *b) {
    uint64_t ka = vdb_order_key((const blk_key *)a), kb = vdb_order_key((const blk_key *)b);
    return ka < kb ? -1 : (ka > kb ? 1 : 0);
}

/* ---- sparse grid lookup (open addressing on block origin) ---------------- */
typedef struct {
    uint32_t cap;
    int32_t *keys; /* 3 per slot */
    uint32_t *vals;
} blk_map;

static uint32_t hash3(int32_t x, int32_t y, int32_t z) {
    uint32_t h = (uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)z * 83492791u;
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    return h;
}

static void map_init(blk_map *m, uint32_t n) {
    m->cap = 16;
    while (m->cap < 2 * n + 16) m->cap <<= 1;
    m->keys = (int32_t *)malloc(sizeof(int32_t) * 3 * m->cap);
    m->vals = (uint32_t *)malloc(sizeof(uint32_t) * m->cap);
    for (uint32_t i = 0; i < m->cap; ++i) m->vals[i] = ORC_NONE;
}

static void map_put(blk_map *m, int32_t x, int32_t y, int32_t z, uint32_t v) {
    uint32_t h = hash3(x, y, z) & (m->cap - 1);
    while (m->vals[h] != ORC_NONE) h = (h + 1) & (m->cap - 1);
    m->keys[3 * h] = x;
    m->keys[3 * h + 1] = y;
    m->keys[3 * h + 2] = z;
    m->vals[h] = v;
}

static uint32_t map_get(const blk_map *m, int32_t x, int32_t y, int32_t z) {
    uint32_t h = hash3(x, y, z) & (m->cap - 1);
    while (m->vals[h] != ORC_NONE) {
        if (m->keys[3 * h] == x && m->keys[3 * h + 1] == y && m->keys[3 * h + 2] == z) return m->vals[h];
        h = (h + 1) & (m->cap - 1);
    }
    return ORC_NONE;
}

static float grid_value(const blk_map *m, const float *values, int32_t x, int32_t y, int32_t z) {
    int32_t bx = x & ~7, by = y & ~7, bz = z & ~7;
    uint32_t b = map_get(m, bx, by, bz);
    if (b == ORC_NONE) return 0.0f; /* background */
    return values[(size_t)b * 512 + (size_t)((z - bz) * 64 + (y - by) * 8 + (x - bx))];
}

/* BoxSampler: data[i][j][k] at (x+i, y+j, z+k); interpolate z, then y, then x,
 * each as a + float((b - a) * w) with the weight in double. */
static float vdb_lerp(float a, float b, double w) { return a + (float)((double)(b - a) * w); }

static float box_sample_ws(const blk_map *m, const float *values, const float pw[3], float s) {
    double inv = 1.0 / (double)s;
    double ix = (double)pw[0] * inv, iy = (double)pw[1] * inv, iz = (double)pw[2] * inv;
    double fx = floor(ix), fy = floor(iy), fz = floor(iz);
    int32_t x = (int32_t)fx, y = (int32_t)fy, z = (int32_t)fz;
    double u = ix - fx, v = iy - fy, w = iz - fz;
    float d[2][2][2];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int k = 0; k < 2; ++k) d[i][j][k] = grid_value(m, values, x + i, y + j, z + k);
    float a0 = vdb_lerp(d[0][0][0], d[0][0][1], w);
    float b0 = vdb_lerp(d[0][1][0], d[0][1][1], w);
    float r1 = vdb_lerp(a0, b0, v);
    float a1 = vdb_lerp(d[1][0][0], d[1][0][1], w);
    float b1 = vdb_lerp(d[1][1][0], d[1][1][1], w);
    float r2 = vdb_lerp(a1, b1, v);
    return r1 + (float)(u * (double)(r2 - r1));
}

/* ---- BuildPath ----------------------------------------------------------- */
typedef struct {
    orc_node *nodes;
    uint32_t n, cap;
    uint32_t leafx;
} build_ctx;

static uint32_t new_node(build_ctx *B) {
    if (B->n == B->cap) {
        B->cap = B->cap ? 2 * B->cap : 1024;
        B->nodes = (orc_node *)realloc(B->nodes, sizeof(orc_node) * B->cap);
    }
    orc_node *o = &B->nodes[B->n];
    memset(o, 0, sizeof(*o));
    o->volx[0] = o->volx[1] = ORC_NONE;
    return B->n++;
}

/* BoundingBox::Intersects(BoundingBox), src/scene.cpp:230-243 */
static int box_intersects(const float ca[3], const float ea[3], const float cb[3], const float eb[3]) {
    for (int k = 0; k < 3; ++k) {
        float mina = ca[k] - ea[k], maxa = ca[k] + ea[k];
        float minb = cb[k] - eb[k], maxb = cb[k] + eb[k];
        if (mina > maxb || minb > maxa) return 0;
    }
    return 1;
}

/* src/scene.cpp:267-305; c and e are float4 with e splatted, c1/e1 the leaf box */
static void build_path(build_ctx *B, uint32_t x, const float c[4], const float e[4], const float c1[3],
                       const float e1[3], uint32_t level, uint32_t mlevel) {
    orc_node *o = &B->nodes[x];
    o->ce[0] = c[0];
    o->ce[1] = c[1];
    o->ce[2] = c[2];
    o->ce[3] = e[3];
    o->qval[0] = o->qval[1] = 0.0f;
    if (level >= mlevel - 1) {
        if (o->volx[ORC_FOG] == ORC_NONE) o->volx[ORC_FOG] = B->leafx++;
        return;
    }
    float ee[4] = {0.5f * e[0], 0.5f * e[1], 0.5f * e[2], 0.5f * e[3]};
    for (uint32_t i = 0; i < 8; ++i) {
        float sv[4] = {2.0f * (float)(i % 2) - 1.0f, 2.0f * (float)((i / 2) % 2) - 1.0f, 2.0f * (float)(i / 4) - 1.0f,
                       2.0f * 0.0f - 1.0f};
        float cc[4], be[3];
        for (int k = 0; k < 4; ++k) cc[k] = c[k] + sv[k] * ee[k];
        for (int k = 0; k < 3; ++k) be[k] = 1.1f * ee[k];
        if (box_intersects(cc, be, c1, e1)) {
            uint32_t ch = B->nodes[x].chn[i];
            if (ch == 0) {
                ch = new_node(B);
                B->nodes[x].chn[i] = ch;
            }
            build_path(B, ch, cc, ee, c1, e1, level + 1, mlevel);
        }
    }
}

int orc_build_octree(const int32_t *block_origin, const float *block_values, uint32_t n_blocks, float s,
                     uint32_t maxdepth, orc_node **out_nodes, uint32_t *n_nodes, float **out_bricks,
                     uint32_t *n_leaves, uint32_t *out_lvoxc, uint32_t *out_mlevel) {
    if (n_blocks == 0 || !(s > 0.0f)) return -1;
    blk_key *keys = (blk_key *)malloc(sizeof(blk_key) * n_blocks);
    blk_map map;
    map_init(&map, n_blocks);
    for (uint32_t b = 0; b < n_blocks; ++b) {
        keys[b].ox = block_origin[3 * b];
        keys[b].oy = block_origin[3 * b + 1];
        keys[b].oz = block_origin[3 * b + 2];
        keys[b].idx = b;
        if (keys[b].ox < 0 || keys[b].oy < 0 || keys[b].oz < 0 || (keys[b].ox & 7) || (keys[b].oy & 7) ||
            (keys[b].oz & 7)) {
            free(keys);
            return -2;
        }
        map_put(&map, keys[b].ox, keys[b].oy, keys[b].oz, b);
    }
    qsort(keys, n_blocks, sizeof(blk_key), cmp_blk);

    /* leaf boxes, src/scene.cpp:676-701 */
    float *bsc = (float *)malloc(sizeof(float) * 3 * n_blocks);
    float *bse = (float *)malloc(sizeof(float) * 3 * n_blocks);
    uint32_t nbox = 0;
    float mn[4] = {FLT_MAX, FLT_MAX, FLT_MAX, FLT_MAX}, mx[4] = {-FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t q = 0; q < n_blocks; ++q) {
        const float *v = block_values + (size_t)keys[q].idx * 512;
        int32_t lo[3] = {8, 8, 8}, hi[3] = {-1, -1, -1};
        for (int z = 0; z < 8; ++z)
            for (int y = 0; y < 8; ++y)
                for (int x = 0; x < 8; ++x)
                    if (v[z * 64 + y * 8 + x] != 0.0f) {
                        if (x < lo[0]) lo[0] = x;
                        if (y < lo[1]) lo[1] = y;
                        if (z < lo[2]) lo[2] = z;
                        if (x > hi[0]) hi[0] = x;
                        if (y > hi[1]) hi[1] = y;
                        if (z > hi[2]) hi[2] = z;
                    }
        if (hi[0] < 0) continue; /* no active voxels: OpenVDB would hold no leaf */
        int32_t org[3] = {keys[q].ox, keys[q].oy, keys[q].oz};
        for (int k = 0; k < 3; ++k) {
            int32_t cmin = org[k] + lo[k], cmax = org[k] + hi[k];
            double posi = 0.5 * (double)(cmin + cmax);
            bsc[3 * nbox + k] = (float)(posi * (double)s);
            float dimi = (float)(cmax - cmin + 1);
            bse[3 * nbox + k] = (0.5f * dimi) * s;
        }
        float c4[4] = {bsc[3 * nbox], bsc[3 * nbox + 1], bsc[3 * nbox + 2], 0.0f};
        float e4[4] = {bse[3 * nbox], bse[3 * nbox + 1], bse[3 * nbox + 2], 0.0f};
        for (int k = 0; k < 4; ++k) {
            float a = c4[k] - e4[k], b = c4[k] + e4[k];
            mn[k] = a < mn[k] ? a : mn[k];  /* _mm_min_ps(c-e, min) */
            mx[k] = b > mx[k] ? b : mx[k];  /* _mm_max_ps(c+e, max) */
        }
        ++nbox;
    }
    if (nbox == 0) {
        free(keys); free(bsc); free(bse); free(map.keys); free(map.vals);
        return -3;
    }
    /* root and depth, src/scene.cpp:703-716 */
    float c[4], e[4];
    for (int k = 0; k < 4; ++k) {
        c[k] = 0.5f * (mx[k] + mn[k]);
        e[k] = 0.5f * (mx[k] - mn[k]);
    }
    float m01 = e[0] > e[1] ? e[0] : e[1];
    float a = m01 > e[2] ? m01 : e[2];
    float a4[4] = {a, a, a, a};
    float d = 2.0f * a;
    float lvc = (float)LVC;
    float mlf = ceilf(logf(d / (lvc * s)) / 0.69315f);
    if (!(mlf >= 2.0f)) {
        /* depth < 2 puts a leaf at the root, which the reference's step
         * traverser cannot handle (src/KernelOctree.cpp:332-336); refuse. */
        free(keys); free(bsc); free(bse); free(map.keys); free(map.vals);
        return -4;
    }
    uint32_t mlevel = (uint32_t)mlf;
    if (mlevel > maxdepth) {
        lvc *= powf(2.0f, (float)(mlevel - maxdepth));
        mlevel = maxdepth;
    }
    uint32_t lvoxc = (uint32_t)lvc;

    build_ctx B = {0, 0, 0, 0};
    new_node(&B); /* root, index 0 */
    for (uint32_t j = 0; j < nbox; ++j) build_path(&B, 0, c, a4, &bsc[3 * j], &bse[3 * j], 0, mlevel);

    /* resampling, src/scene.cpp:870-908: nodes [0, index) with index = the
     * last assigned node index, so node B.n-1 is left untouched */
    uint32_t lv3 = lvoxc * lvoxc * lvoxc;
    float *bricks = (float *)calloc((size_t)B.leafx * lv3 + 1, sizeof(float));
    float nv = (float)lvoxc;
    uint32_t index = B.n - 1;
    for (uint32_t i = 0; i < index; ++i) {
        orc_node *o = &B.nodes[i];
        if (o->volx[ORC_SDF] == ORC_NONE && o->volx[ORC_FOG] == ORC_NONE) continue;
        o->qval[ORC_SDF] = FLT_MAX;
        o->qval[ORC_FOG] = 0.01f;
        for (uint32_t j = 0; j < lv3; ++j) {
            float jv[3] = {(float)(j % lvoxc), (float)((j / lvoxc) % lvoxc), (float)(j / (lvoxc * lvoxc))};
            float pw[3];
            for (int k = 0; k < 3; ++k) {
                float nn = ((nv - 2.0f * jv[k]) - 1.0f) / (nv - 1.0f);
                pw[k] = o->ce[k] - o->ce[3] * nn;
            }
            float val = box_sample_ws(&map, block_values, pw, s);
            val = (1.0f < val) ? 1.0f : val; /* openvdb::math::Min(v, 1) = std::min */
            val = (val < 0.0f) ? 0.0f : val; /* openvdb::math::Max(., 0) = std::max */
            bricks[(size_t)o->volx[ORC_FOG] * lv3 + j] = val;
            if (o->qval[ORC_FOG] < val) o->qval[ORC_FOG] = val;
        }
    }
    free(keys);
    free(bsc);
    free(bse);
    free(map.keys);
    free(map.vals);
    *out_nodes = B.nodes;
    *n_nodes = B.n;
    *out_bricks = bricks;
    *n_leaves = B.leafx;
    *out_lvoxc = lvoxc;
    *out_mlevel = mlevel;
    return 0;
}

void orc_free(void *p) { free(p); }
