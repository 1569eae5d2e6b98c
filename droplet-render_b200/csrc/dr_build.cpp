// Host-side scene construction of droplet_b200: the OpenVDB-free part of the
// reference scene build, producing the reference's node records and brick pool
// bit for bit (see the per-step citations), plus the Hosek-Wilkie state cook.
//
//   leaf boxes       src/scene.cpp:676-701 (active bounding box of each 8^3 leaf)
//   root and depth   src/scene.cpp:703-716
//   BuildPath        src/scene.cpp:267-305 (child boxes grown by 1.1, DFS numbering)
//   resampling       src/scene.cpp:870-908 (nodes [0, last index): the node
//                    created last is not resampled and keeps majorant 0)
//
// Input blocks stand in for OpenVDB leaves; the OpenVDB pieces the reference
// relies on are restated here: leaf order of a Tree4<float,5,4,3>,
// CoordBBox::getCenter/dim, the uniform-scale index<->world maps and
// BoxSampler trilinear interpolation (z, then y, then x, weights in double).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>
#include "../../include/droplet_b200.h"
#include "dr_internal.h"

namespace dr {

void set_error(int code, const std::string &msg);

namespace {

struct LeafBox {
    float c[3], e[3];
};

inline uint64_t block_key(int32_t x, int32_t y, int32_t z) {
    return ((uint64_t)(uint32_t)(x >> 3) << 42) | ((uint64_t)(uint32_t)(y >> 3) << 21) | (uint64_t)(uint32_t)(z >> 3);
}

// Position of an 8^3 leaf in the iteration order of an OpenVDB Tree4<float,5,4,3>
// (root table sorted by origin, then 32^3 and 16^3 child tables in x-major order).
inline uint64_t vdb_leaf_rank(int32_t ox, int32_t oy, int32_t oz) {
    const uint64_t x = (uint32_t)ox, y = (uint32_t)oy, z = (uint32_t)oz;
    uint64_t k = x >> 12;
    k = (k << 8) | (y >> 12);
    k = (k << 8) | (z >> 12);
    k = (k << 5) | ((x >> 7) & 31u);
    k = (k << 5) | ((y >> 7) & 31u);
    k = (k << 5) | ((z >> 7) & 31u);
    k = (k << 4) | ((x >> 3) & 15u);
    k = (k << 4) | ((y >> 3) & 15u);
    k = (k << 4) | ((z >> 3) & 15u);
    return k;
}

class SparseGrid {
public:
    SparseGrid(const int32_t *org, const float *vals, uint32_t n) : vals_(vals) {
        map_.reserve((size_t)n * 2);
        for (uint32_t b = 0; b < n; ++b) map_.emplace(block_key(org[3 * b], org[3 * b + 1], org[3 * b + 2]), b);
    }
    float at(int32_t x, int32_t y, int32_t z) const {
        if (x < 0 || y < 0 || z < 0) return 0.0f;
        auto it = map_.find(block_key(x, y, z));
        if (it == map_.end()) return 0.0f;
        return vals_[(size_t)it->second * 512 + (size_t)(((z & 7) << 6) | ((y & 7) << 3) | (x & 7))];
    }
    // GridSampler<FloatGrid, BoxSampler>::wsSample for a uniform scale map of voxel size s
    float ws_sample(const float pw[3], float s) const {
        const double inv = 1.0 / (double)s;
        double idx[3], fl[3];
        int32_t i0[3];
        for (int k = 0; k < 3; ++k) {
            idx[k] = (double)pw[k] * inv;
            fl[k] = std::floor(idx[k]);
            i0[k] = (int32_t)fl[k];
        }
        const double u = idx[0] - fl[0], v = idx[1] - fl[1], w = idx[2] - fl[2];
        auto L = [](float a, float b, double t) { return a + (float)((double)(b - a) * t); };
        const float x0y0 = L(at(i0[0], i0[1], i0[2]), at(i0[0], i0[1], i0[2] + 1), w);
        const float x0y1 = L(at(i0[0], i0[1] + 1, i0[2]), at(i0[0], i0[1] + 1, i0[2] + 1), w);
        const float x0 = L(x0y0, x0y1, v);
        const float x1y0 = L(at(i0[0] + 1, i0[1], i0[2]), at(i0[0] + 1, i0[1], i0[2] + 1), w);
        const float x1y1 = L(at(i0[0] + 1, i0[1] + 1, i0[2]), at(i0[0] + 1, i0[1] + 1, i0[2] + 1), w);
        const float x1 = L(x1y0, x1y1, v);
        return x0 + (float)(u * (double)(x1 - x0));
    }

private:
    const float *vals_;
    std::unordered_map<uint64_t, uint32_t> map_;
};

class OctreeBuilder {
public:
    explicit OctreeBuilder(uint32_t mlevel) : mlevel_(mlevel) { add_node(); }

    // Octree::BuildPath for one leaf box (c1, e1) from the root (c, e).
    void insert(const float c[4], const float e[4], const LeafBox &box) { path(0, c, e, box, 0); }

    std::vector<dr_node> nodes;
    uint32_t leaves = 0;

private:
    uint32_t add_node() {
        dr_node n;
        std::memset(&n, 0, sizeof(n));
        n.volx[0] = n.volx[1] = DR_NONE;
        nodes.push_back(n);
        return (uint32_t)nodes.size() - 1;
    }

    static bool overlaps(const float ca[4], const float ea[3], const LeafBox &b) {
        for (int k = 0; k < 3; ++k) {
            const float amin = ca[k] - ea[k], amax = ca[k] + ea[k];
            const float bmin = b.c[k] - b.e[k], bmax = b.c[k] + b.e[k];
            if (amin > bmax || bmin > amax) return false;
        }
        return true;
    }

    void path(uint32_t x, const float c[4], const float e[4], const LeafBox &box, uint32_t level) {
        dr_node &n = nodes[x];
        n.ce[0] = c[0];
        n.ce[1] = c[1];
        n.ce[2] = c[2];
        n.ce[3] = e[3];
        n.qval[0] = n.qval[1] = 0.0f;
        if (level >= mlevel_ - 1) {
            if (n.volx[1] == DR_NONE) n.volx[1] = leaves++;
            return;
        }
        float ee[4];
        for (int k = 0; k < 4; ++k) ee[k] = 0.5f * e[k];
        float grown[3];
        for (int k = 0; k < 3; ++k) grown[k] = 1.1f * ee[k];
        for (uint32_t i = 0; i < 8; ++i) {
            const float sign[4] = {(i & 1) ? 1.0f : -1.0f, (i & 2) ? 1.0f : -1.0f, (i & 4) ? 1.0f : -1.0f, -1.0f};
            float cc[4];
            for (int k = 0; k < 4; ++k) cc[k] = c[k] + sign[k] * ee[k];
            if (!overlaps(cc, grown, box)) continue;
            uint32_t ch = nodes[x].chn[i];
            if (ch == 0) {
                ch = add_node();  // may reallocate: index nodes[x] again below
                nodes[x].chn[i] = ch;
            }
            path(ch, cc, ee, box, level + 1);
        }
    }

    uint32_t mlevel_;
};

}  // namespace

int build_octree(const int32_t *org, const float *vals, uint32_t n_blocks, float s, uint32_t maxdepth,
                 int nthreads, dr_octree *out) {
    if (!org || !vals || !out || n_blocks == 0 || !(s > 0.0f) || maxdepth < 2) {
        set_error(DR_ERR_INVALID, "dr_build_octree: need blocks, a positive voxel size and maxdepth >= 2");
        return DR_ERR_INVALID;
    }
    for (uint32_t b = 0; b < n_blocks; ++b)
        for (int k = 0; k < 3; ++k)
            if (org[3 * b + k] < 0 || (org[3 * b + k] & 7) || org[3 * b + k] >= (1 << 24)) {
                set_error(DR_ERR_INVALID, "dr_build_octree: block origins must be non-negative multiples of 8 below 2^24");
                return DR_ERR_INVALID;
            }
    std::vector<uint32_t> order(n_blocks);
    for (uint32_t b = 0; b < n_blocks; ++b) order[b] = b;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return vdb_leaf_rank(org[3 * a], org[3 * a + 1], org[3 * a + 2]) <
               vdb_leaf_rank(org[3 * b], org[3 * b + 1], org[3 * b + 2]);
    });

    // leaf boxes and scene bounds
    std::vector<LeafBox> boxes;
    boxes.reserve(n_blocks);
    float lo4[4] = {FLT_MAX, FLT_MAX, FLT_MAX, FLT_MAX}, hi4[4] = {-FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t q : order) {
        const float *v = vals + (size_t)q * 512;
        int32_t mn[3] = {8, 8, 8}, mx[3] = {-1, -1, -1};
        for (int i = 0; i < 512; ++i) {
            if (v[i] == 0.0f) continue;
            const int32_t c[3] = {i & 7, (i >> 3) & 7, i >> 6};
            for (int k = 0; k < 3; ++k) {
                mn[k] = std::min(mn[k], c[k]);
                mx[k] = std::max(mx[k], c[k]);
            }
        }
        if (mx[0] < 0) continue;
        LeafBox b;
        for (int k = 0; k < 3; ++k) {
            const int32_t a = org[3 * q + k] + mn[k], z = org[3 * q + k] + mx[k];
            b.c[k] = (float)((0.5 * (double)(a + z)) * (double)s);
            b.e[k] = (0.5f * (float)(z - a + 1)) * s;
        }
        const float c4[4] = {b.c[0], b.c[1], b.c[2], 0.0f}, e4[4] = {b.e[0], b.e[1], b.e[2], 0.0f};
        for (int k = 0; k < 4; ++k) {
            const float l = c4[k] - e4[k], h = c4[k] + e4[k];
            lo4[k] = l < lo4[k] ? l : lo4[k];
            hi4[k] = h > hi4[k] ? h : hi4[k];
        }
        boxes.push_back(b);
    }
    if (boxes.empty()) {
        set_error(DR_ERR_INVALID, "dr_build_octree: no active voxels");
        return DR_ERR_INVALID;
    }
    float c[4], e[4];
    for (int k = 0; k < 4; ++k) {
        c[k] = 0.5f * (hi4[k] + lo4[k]);
        e[k] = 0.5f * (hi4[k] - lo4[k]);
    }
    const float exy = e[0] > e[1] ? e[0] : e[1];
    const float a = exy > e[2] ? exy : e[2];
    const float a4[4] = {a, a, a, a};
    float lvc = 8.0f;
    const float depth = std::ceil(std::log((2.0f * a) / (lvc * s)) / 0.69315f);
    if (!(depth >= 2.0f)) {
        set_error(DR_ERR_INVALID, "dr_build_octree: the volume spans less than two octree levels");
        return DR_ERR_INVALID;
    }
    uint32_t mlevel = (uint32_t)depth;
    if (mlevel > maxdepth) {
        lvc *= std::pow(2.0f, (float)(mlevel - maxdepth));
        mlevel = maxdepth;
    }
    if ((uint32_t)lvc != kLvox) {
        set_error(DR_ERR_INVALID, "dr_build_octree: maxdepth too small for this volume (bricks would exceed 8^3)");
        return DR_ERR_INVALID;
    }

    OctreeBuilder B(mlevel);
    for (const LeafBox &b : boxes) B.insert(c, a4, b);

    // brick resampling over nodes [0, last index)
    SparseGrid grid(org, vals, n_blocks);
    const uint32_t nn = (uint32_t)B.nodes.size();
    const uint32_t index = nn - 1;
    std::vector<float> bricks((size_t)B.leaves * kBrick + 1, 0.0f);
    auto work = [&](uint32_t t, uint32_t nt) {
        for (uint32_t i = t; i < index; i += nt) {
            dr_node &o = B.nodes[i];
            if (o.volx[0] == DR_NONE && o.volx[1] == DR_NONE) continue;
            o.qval[0] = FLT_MAX;
            o.qval[1] = 0.01f;
            float *dst = &bricks[(size_t)o.volx[1] * kBrick];
            const float nv = (float)kLvox;
            for (uint32_t j = 0; j < kBrick; ++j) {
                const float jj[3] = {(float)(j % kLvox), (float)((j / kLvox) % kLvox), (float)(j / (kLvox * kLvox))};
                float pw[3];
                for (int k = 0; k < 3; ++k) pw[k] = o.ce[k] - o.ce[3] * (((nv - 2.0f * jj[k]) - 1.0f) / (nv - 1.0f));
                float v = grid.ws_sample(pw, s);
                v = (1.0f < v) ? 1.0f : v;
                v = (v < 0.0f) ? 0.0f : v;
                dst[j] = v;
                if (o.qval[1] < v) o.qval[1] = v;
            }
        }
    };
    uint32_t nt = nthreads > 0 ? (uint32_t)nthreads : std::max(1u, std::thread::hardware_concurrency());
    nt = std::min<uint32_t>(nt, 256);
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < nt; ++t) pool.emplace_back(work, t, nt);
    work(0, nt);
    for (auto &th : pool) th.join();

    out->n_nodes = nn;
    out->nodes = (dr_node *)std::malloc(sizeof(dr_node) * nn);
    out->n_leaves = B.leaves;
    out->bricks = (float *)std::malloc(sizeof(float) * ((size_t)B.leaves * kBrick + 1));
    if (!out->nodes || !out->bricks) {
        std::free(out->nodes);
        std::free(out->bricks);
        set_error(DR_ERR_NOMEM, "dr_build_octree: host allocation failed");
        return DR_ERR_NOMEM;
    }
    std::memcpy(out->nodes, B.nodes.data(), sizeof(dr_node) * nn);
    std::memcpy(out->bricks, bricks.data(), sizeof(float) * ((size_t)B.leaves * kBrick + 1));
    out->lvoxc = kLvox;
    out->mlevel = mlevel;
    return DR_OK;
}

// Hosek-Wilkie cook (src/ArHosekSkyModel.cpp:147-289): a degree-5 Bernstein
// polynomial in (elevation / (pi/2))^(1/3), blended linearly over the two
// albedo tables and the two nearest integer turbidities.
static double cook_one(const double *ds, int stride_k, int stride_alb, int stride_t, int i, double turbidity,
                       double albedo, double elevation) {
    const int it = (int)turbidity;
    const double tr = turbidity - (double)it;
    const double x = std::pow(elevation / (3.141592653589793 / 2.0), 1.0 / 3.0);
    auto bez = [&](const double *m) {
        return std::pow(1.0 - x, 5.0) * m[0] + 5.0 * std::pow(1.0 - x, 4.0) * x * m[stride_k] +
               10.0 * std::pow(1.0 - x, 3.0) * std::pow(x, 2.0) * m[2 * stride_k] +
               10.0 * std::pow(1.0 - x, 2.0) * std::pow(x, 3.0) * m[3 * stride_k] +
               5.0 * (1.0 - x) * std::pow(x, 4.0) * m[4 * stride_k] + std::pow(x, 5.0) * m[5 * stride_k];
    };
    double r = (1.0 - albedo) * (1.0 - tr) * bez(ds + stride_t * (it - 1) + i);
    r += albedo * (1.0 - tr) * bez(ds + stride_alb + stride_t * (it - 1) + i);
    if (it == 10) return r;
    r += (1.0 - albedo) * tr * bez(ds + stride_t * it + i);
    r += albedo * tr * bez(ds + stride_alb + stride_t * it + i);
    return r;
}

int sky_cook(const double *const rgb[3], const double *const rad[3], double turbidity, double albedo,
             double elevation, double configs[3][9], double radiances[3]) {
    if (!rgb || !rad || !configs || !radiances || !(turbidity >= 1.0 && turbidity <= 10.0) ||
        !(albedo >= 0.0 && albedo <= 1.0) || !(elevation >= 0.0 && elevation <= 3.141592653589793 / 2.0)) {
        set_error(DR_ERR_INVALID, "dr_sky_cook: need turbidity in [1,10], albedo in [0,1], elevation in [0,pi/2]");
        return DR_ERR_INVALID;
    }
    for (int c = 0; c < 3; ++c) {
        if (!rgb[c] || !rad[c]) {
            set_error(DR_ERR_INVALID, "dr_sky_cook: missing dataset channel");
            return DR_ERR_INVALID;
        }
        for (int i = 0; i < 9; ++i) configs[c][i] = cook_one(rgb[c], 9, 9 * 6 * 10, 9 * 6, i, turbidity, albedo, elevation);
        radiances[c] = cook_one(rad[c], 1, 6 * 10, 6, 0, turbidity, albedo, elevation);
    }
    return DR_OK;
}

}  // namespace dr
