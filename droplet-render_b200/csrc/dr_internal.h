// Internal host/device layouts of the droplet_b200 library (not part of the C ABI).
#pragma once
#include <cstdint>
#include <cstddef>
#include <vector_types.h>

#ifdef __CUDACC__
#define DR_HD __host__ __device__
#else
#define DR_HD
#endif

namespace dr {

constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kLvox = 8;            // brick edge; the builder and upload enforce it
constexpr uint32_t kBrick = kLvox * kLvox * kLvox;
constexpr int kMaxDepth = 16;            // traversal stack, src/KernelOctree.h:35
constexpr uint32_t kMieMax = 4096;
constexpr uint32_t kStepBudget = 1u << 24;  // tracking steps per segment before a path gives up

// Device scene.  Node ids are the reference's (DFS creation order).
//   child[2*id], child[2*id+1]: the eight child entries of node id, remapped:
//       0 = no child, kLeafBit|c = leaf node c, c = internal node c
//   leaf[2*id]   = (center.xyz, half extent)
//   leaf[2*id+1] = (majorant, FOG brick index bits, SDF brick index bits, 0);
//                  an index kNone = no such brick; SDF leaves have majorant 1
struct DevScene {
    const uint4 *child;
    const float4 *leaf;
    const float *bricks;
    const float *sdf_bricks;   // SDF pool, or null when no leaf has a surface brick
    float root_ce[4];
    uint32_t n_nodes;
    uint32_t n_leaves;
    // Leaf grid for the cell-walk traversal (all leaves at one depth):
    // n = 2^levels leaf cells per axis; macro cells of 8^3 leaf cells;
    // macro[mz][my][mx] = block index or kNone (no leaf in the macro cell);
    // cells[block*512 + z*64 + y*8 + x] = leaf node id or kNone.
    const uint32_t *macro;
    const uint32_t *cells;
    uint32_t levels;     // leaf depth below the root (0 = no grid; stack traversal only)
    uint32_t n;          // leaf cells per axis
    uint32_t mdim;       // macro cells per axis
    // Entries the stack traversal can push on any ray: internal nodes below the
    // root on the deepest root-to-leaf path (0: unknown, e.g. leaves at mixed
    // depths or a DAG, or 2^25 nodes or more; then only the local-memory stack
    // is used).
    uint32_t stack_levels;
    // Occluder BVH (null: no occluders).  Node i = occ_nodes[4i .. 4i+3]: left
    // box (min xyz, max x), (max yz, right min xy), (right min z, right max
    // xyz), then (left ref, right ref, left count, right count) as uint32
    // bits: count > 0 = leaf of `count` triangles from ref, count 0 = internal
    // node ref, ref kNone = no child.  Triangle j = occ_tris[3j .. 3j+2]:
    // v0, e1 = v1 - v0, e2 = v2 - v0 (w unused).
    const float4 *occ_nodes;
    const float4 *occ_tris;
    uint32_t occ_n_nodes;
};

constexpr uint32_t kPhaseHG = 2;     // DR_PHASE_HG
constexpr uint32_t kEnvHosek = 0, kEnvNone = 1, kEnvMap = 2;  // DR_ENV_*

constexpr int kOccMaxDepth = 48;     // occluder BVH depth (the traversal stack holds one entry per level)
constexpr float kOccFar = 1e6f;      // MAX_OCCLUSION_DIST, src/SceneOcclusion.h:4

struct DevParams {
    float sigma_s, sigma_a, sigma_e, albedo;   // albedo = sigma_s / (sigma_a + sigma_s) in binary32
    uint32_t scattevs;
    float sun_dir[3], sun_color[3], sun_cos, sun_pdf;
    float sky_cfg[3][9], sky_rad[3];
    const float *mie_pdf;     // mie_n * 3
    const float *mie_cdf;     // mie_n * 3
    const float *mie_exact;   // exact sampler table (mie_n + 1 CDF values of pdf*sin) or null
    uint32_t mie_n;
    uint32_t phase_mode;
    float viewi[16], proji[16];
    uint32_t w, h;
    const float *depth;       // w*h or null
    uint32_t depthcomp;       // KERNEL_DEPTHCOMP: camera rays stop at depth
    uint32_t finite_paths;    // a path whose contribution is not finite adds nothing
    uint32_t embree;          // the reference's USE_EMBREE build: occluder and depth masks on gathered light
    float hg_g;               // kPhaseHG: anisotropy
    uint32_t env_mode;        // kEnvHosek, kEnvNone or kEnvMap
    const float *env_map;     // kEnvMap: env_w * env_h RGBA texels (device)
    uint32_t env_w, env_h;
    float clip_end;           // far clip distance: -z/w of (0,0,1,1) * projInv (src/kernel.cpp:574-575)
    uint32_t step_budget;     // tracking steps per segment before a path gives up (kStepBudget unless set)
};

// What a tracking loop needs of the parameters: the extinction and the step budget.
struct SegMedium {
    float sigma_e;
    uint32_t budget;
};
DR_HD inline SegMedium seg_medium(const DevParams &P) { return SegMedium{P.sigma_e, P.step_budget}; }

// Exact unsigned 32-bit division by an invariant d >= 1 (Granlund and
// Montgomery, "Division by invariant integers using multiplication", PLDI
// 1994, fig. 4.1): with l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0), t = mulhi(m, n), for
// every 32-bit n.  The path kernels use it where a path index becomes a pixel.
struct FastDiv {
    uint32_t m, s1, s2;
};

inline FastDiv make_fastdiv(uint32_t d) {
    if (d == 0) d = 1;  // unused divisor (an empty extent)
    uint32_t l = 0;
    while (l < 32 && (1ull << l) < d) ++l;
    FastDiv f;
    f.m = (uint32_t)(((((1ull << l) - d) << 32) / d) + 1);
    f.s1 = l < 1 ? l : 1u;
    f.s2 = l > 0 ? l - 1 : 0u;
    return f;
}

struct TileArgs {
    uint32_t x0, y0, tw, th;
    uint32_t cols, rows;      // rendered extent: even parts of tw, th
    uint32_t spp;
    uint32_t tile;            // persistent kernel: pixel order in tile x tile squares (0 = row-major)
    uint32_t tiles_x;         // squares per row when tile > 0
    uint64_t seed, sample_base;
    uint64_t n_paths;         // path indices: cols * rows * spp (row-major) or squares * tile^2 * spp
    FastDiv spp_div, cols_div, t2_div, tx_div, tile_div;  // division by spp, cols, tile^2, tiles_x, tile
    // Persistent kernel only (its launcher sets it): the sky term of a path
    // that escapes after scattering goes to the warp's queue of sky terms and is
    // evaluated 32 at a time (Hosek sky, no whole-path finiteness check).
    uint32_t defer_sky;
    // Persistent kernel, stack traversals: the camera rays' leaf sequences,
    // built once per launch by camera_list_kernel (every sample of a pixel
    // shares its camera ray).  Pixel q = iy * cols + ix: cam_head[2q] = (first
    // entry in cam_pool, leaves, node visits of the root test, node visits
    // after the last leaf), or x = ~0 when the pixel's list did not fit (its
    // samples traverse); cam_head[2q + 1] = (the ray's direction bits, 1 if the
    // pixel has a ray); cam_pool entries = (leaf, tra bits, trb bits, node
    // visits since the previous leaf).  Null: rays are generated per sample and
    // every segment traverses.
    const uint4 *cam_head;
    const uint4 *cam_pool;
};

struct DevCounters {
    unsigned long long paths, vertices, node_visits, density_lookups, mie_evals, gave_up;
};

// Launch-shape choices of the persistent renderer (chosen by the autotuner).
struct Tuning {
    uint32_t kernel;        // 0 = persistent path kernel, 1 = one thread per path
    uint32_t block;         // threads per block (multiple of 32)
    uint32_t blocks_per_sm; // 0 = as many as fit
    uint32_t event_batch;   // lanes of a warp that must be waiting before events run
    uint32_t traversal;     // 0 = octree stack traversal, 1 = leaf-grid cell walk
    uint32_t tile;          // pixel order of the persistent kernel: 0 = row-major, else square side
    uint32_t visits;        // stack traversal: node examinations per loop iteration (0 = to the next leaf)
    uint32_t steps;         // free-flight steps per loop iteration (0 = 1)
};

// One view of a batched launch: its parameters, tile and output, the scene it
// renders and the first global path index it owns.
struct BatchView {
    DevParams P;
    TileArgs A;
    float4 *sun, *sky;
    uint32_t scene;
    uint32_t pad;
    uint64_t begin;
};

// A batched launch: every view's paths form one index space [0, n_paths) in
// view order; begins[v] = views[v].begin (binary-searched per fetched path).
struct BatchArgs {
    const BatchView *views;
    const DevScene *scenes;
    const uint64_t *begins;
    uint32_t n_views;
    uint64_t n_paths;
    const unsigned long long *step;  // launches so far: view samples start at sample_base + step * spp
};

// Work queue of the persistent kernel: next path index to hand out.
struct WorkQueue {
    unsigned long long next;
};

}  // namespace dr
