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
//   leaf[2*id+1] = (majorant, brick index bits, 0, 0)
struct DevScene {
    const uint4 *child;
    const float4 *leaf;
    const float *bricks;
    float root_ce[4];
    uint32_t n_nodes;
    uint32_t n_leaves;
};

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
};

struct TileArgs {
    uint32_t x0, y0, tw, th;
    uint32_t cols, rows;      // rendered extent: even parts of tw, th
    uint32_t spp;
    uint64_t seed, sample_base;
    uint64_t n_paths;         // cols * rows * spp
};

struct DevCounters {
    unsigned long long paths, vertices, node_visits, density_lookups, mie_evals, gave_up;
};

}  // namespace dr
