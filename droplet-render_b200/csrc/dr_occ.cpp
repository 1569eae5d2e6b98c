// Occluder BVH: the GPU replacement of SceneOcclusion's Embree scene
// (src/SceneOcclusion.cpp:19-56).  Host build only; the any-hit traversal is
// occluded() in dr_device.cuh.
//
// Binary BVH, binned surface-area heuristic (16 bins over the centroid extent
// of the longest axis; median split by index when all centroids coincide),
// at most 4 triangles per leaf and depth <= kOccMaxDepth.  Each node holds the
// boxes of both children (one 64-byte record), so a visit decides both
// children with one fetch.  Boxes are padded by 1e-4 of the geometry's scale:
// the traversal's slab test then never rejects a box whose triangle the exact
// ray/triangle test would accept (its rounding is far below the padding), so
// the any-hit answer equals a test of every triangle.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dr_host.h"

namespace dr {

namespace {

struct Prim {
    float lo[3], hi[3], c[3];
    uint32_t tri;
};

struct Box {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void grow(const float *a, const float *b) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], a[k]);
            hi[k] = std::max(hi[k], b[k]);
        }
    }
    double area() const {
        if (!(lo[0] <= hi[0])) return 0.0;
        const double x = (double)hi[0] - lo[0], y = (double)hi[1] - lo[1], z = (double)hi[2] - lo[2];
        return 2.0 * (x * y + y * z + z * x);
    }
};

constexpr uint32_t kLeafMax = 4;
constexpr int kBins = 16;

struct Builder {
    std::vector<Prim> prims;
    std::vector<float> nodes;  // 16 floats per node
    std::vector<uint32_t> order;
    float pad = 0.0f;

    Box bounds(uint32_t b, uint32_t e) const {
        Box x;
        for (uint32_t i = b; i < e; ++i) x.grow(prims[i].lo, prims[i].hi);
        return x;
    }

    // Splits [b, e) in two; returns the split point (b < m < e).
    uint32_t split(uint32_t b, uint32_t e) {
        Box cb;
        for (uint32_t i = b; i < e; ++i) cb.grow(prims[i].c, prims[i].c);
        int axis = 0;
        float ext = cb.hi[0] - cb.lo[0];
        for (int k = 1; k < 3; ++k)
            if (cb.hi[k] - cb.lo[k] > ext) {
                ext = cb.hi[k] - cb.lo[k];
                axis = k;
            }
        const uint32_t mid = b + (e - b) / 2;
        if (!(ext > 0.0f)) return mid;  // coincident centroids: halve by index
        auto bin_of = [&](const Prim &p) {
            int i = (int)((p.c[axis] - cb.lo[axis]) / ext * kBins);
            return std::min(std::max(i, 0), kBins - 1);
        };
        Box bb[kBins];
        uint32_t cnt[kBins] = {};
        for (uint32_t i = b; i < e; ++i) {
            const int k = bin_of(prims[i]);
            bb[k].grow(prims[i].lo, prims[i].hi);
            ++cnt[k];
        }
        double best = INFINITY;
        int bs = -1;
        for (int s = 1; s < kBins; ++s) {
            Box l, r;
            uint32_t nl = 0, nr = 0;
            for (int k = 0; k < s; ++k)
                if (cnt[k]) l.grow(bb[k].lo, bb[k].hi), nl += cnt[k];
            for (int k = s; k < kBins; ++k)
                if (cnt[k]) r.grow(bb[k].lo, bb[k].hi), nr += cnt[k];
            if (!nl || !nr) continue;
            const double cost = nl * l.area() + nr * r.area();
            if (cost < best) best = cost, bs = s;
        }
        if (bs < 0) return mid;
        Prim *p = prims.data();
        Prim *m = std::partition(p + b, p + e, [&](const Prim &q) { return bin_of(q) < bs; });
        const uint32_t mi = (uint32_t)(m - p);
        return (mi == b || mi == e) ? mid : mi;
    }

    void put_box(float *dst, const Box &x) const {
        for (int k = 0; k < 3; ++k) {
            dst[k] = x.lo[k] - pad;
            dst[3 + k] = x.hi[k] + pad;
        }
    }

    // Node for [b, e) (at least two children's worth, or the whole set).
    uint32_t build(uint32_t b, uint32_t e, int depth) {
        const uint32_t id = (uint32_t)(nodes.size() / 16);
        nodes.resize(nodes.size() + 16, 0.0f);
        uint32_t ref[2], count[2];
        Box box[2];
        if (e - b <= kLeafMax) {
            // one leaf on the left, no right child
            ref[0] = b;
            count[0] = e - b;
            box[0] = bounds(b, e);
            ref[1] = kNone;
            count[1] = 0;
        } else {
            const uint32_t m = split(b, e);
            const uint32_t rb[2] = {b, m}, re[2] = {m, e};
            for (int c = 0; c < 2; ++c) {
                box[c] = bounds(rb[c], re[c]);
                if (re[c] - rb[c] <= kLeafMax || depth + 1 >= kOccMaxDepth) {
                    ref[c] = rb[c];
                    count[c] = re[c] - rb[c];
                } else {
                    ref[c] = build(rb[c], re[c], depth + 1);
                    count[c] = 0;
                }
            }
        }
        float *n = &nodes[(size_t)id * 16];
        put_box(n, box[0]);
        if (ref[1] != kNone) put_box(n + 6, box[1]);
        uint32_t w[4] = {ref[0], ref[1], count[0], count[1]};
        std::memcpy(n + 12, w, 16);
        return id;
    }
};

}  // namespace

int build_occluder_bvh(const dr_surface *s, uint32_t n, uint32_t mode, OccBvh &out) {
    out.nodes.clear();
    out.tris.clear();
    out.source.clear();
    if (n && !s) return need(false, DR_ERR_INVALID, "occluders: null surface list");
    if (mode != DR_OCCLUDE_ALL_SURFACES && mode != DR_OCCLUDE_HOLDOUT_ONLY)
        return need(false, DR_ERR_INVALID, "occluders: unknown mode");
    // selected triangles, in input order
    std::vector<float> v;  // 9 floats per triangle
    float scale = 0.0f;
    for (uint32_t i = 0; i < n; ++i) {
        const dr_surface &o = s[i];
        if (mode == DR_OCCLUDE_HOLDOUT_ONLY && !(o.flags & DR_SURFACE_HOLDOUT)) continue;
        if (o.n_triangles && (!o.vertices || !o.indices))
            return need(false, DR_ERR_INVALID, "occluders: surface without vertices or indices");
        for (uint32_t t = 0; t < o.n_triangles; ++t)
            for (int c = 0; c < 3; ++c) {
                const uint32_t k = o.indices[3 * (size_t)t + c];
                if (k >= o.n_vertices) return need(false, DR_ERR_INVALID, "occluders: vertex index out of range");
                for (int a = 0; a < 3; ++a) {
                    const float x = o.vertices[3 * (size_t)k + a];
                    if (!std::isfinite(x)) return need(false, DR_ERR_INVALID, "occluders: vertex not finite");
                    scale = std::max(scale, std::fabs(x));
                    v.push_back(x);
                }
            }
    }
    const size_t nt = v.size() / 9;
    if (nt == 0) return DR_OK;
    if (nt >= (size_t)kNone / 2) return need(false, DR_ERR_INVALID, "occluders: too many triangles");
    Builder B;
    B.pad = 1e-4f * std::max(scale, 1e-3f);
    B.prims.resize(nt);
    for (size_t t = 0; t < nt; ++t) {
        Prim &p = B.prims[t];
        const float *a = &v[9 * t];
        for (int k = 0; k < 3; ++k) {
            p.lo[k] = std::min(a[k], std::min(a[3 + k], a[6 + k]));
            p.hi[k] = std::max(a[k], std::max(a[3 + k], a[6 + k]));
            p.c[k] = 0.5f * (p.lo[k] + p.hi[k]);
        }
        p.tri = (uint32_t)t;
    }
    B.build(0, (uint32_t)nt, 0);
    out.nodes = std::move(B.nodes);
    out.tris.resize(nt * 12);
    out.source.resize(nt);
    for (size_t i = 0; i < nt; ++i) {
        const uint32_t t = B.prims[i].tri;
        const float *a = &v[9 * (size_t)t];
        float *d = &out.tris[12 * i];
        for (int k = 0; k < 3; ++k) {
            d[k] = a[k];
            d[4 + k] = a[3 + k] - a[k];
            d[8 + k] = a[6 + k] - a[k];
        }
        d[3] = d[7] = d[11] = 0.0f;
        out.source[i] = t;
    }
    return DR_OK;
}

}  // namespace dr

int dr_build_occluder_bvh(const dr_surface *surfaces, uint32_t n_surfaces, uint32_t mode, float *nodes,
                          uint32_t *n_nodes, float *triangles, uint32_t *source, uint32_t *n_triangles) {
    if (!n_nodes || !n_triangles) return dr::need(false, DR_ERR_INVALID, "dr_build_occluder_bvh: null count");
    dr::OccBvh b;
    const int rc = dr::build_occluder_bvh(surfaces, n_surfaces, mode, b);
    if (rc != DR_OK) return rc;
    const uint32_t nn = (uint32_t)(b.nodes.size() / 16), nt = (uint32_t)b.source.size();
    if (nodes) {
        if (*n_nodes < nn) return dr::need(false, DR_ERR_INVALID, "dr_build_occluder_bvh: node buffer too small");
        std::memcpy(nodes, b.nodes.data(), b.nodes.size() * sizeof(float));
    }
    if (triangles || source) {
        if (*n_triangles < nt)
            return dr::need(false, DR_ERR_INVALID, "dr_build_occluder_bvh: triangle buffer too small");
        if (triangles) std::memcpy(triangles, b.tris.data(), b.tris.size() * sizeof(float));
        if (source) std::memcpy(source, b.source.data(), b.source.size() * sizeof(uint32_t));
    }
    *n_nodes = nn;
    *n_triangles = nt;
    return DR_OK;
}
