// Host-side helpers of the C ABI: errors, scene and settings conversion.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "dr_host.h"

namespace dr {

static thread_local std::string g_error;

void set_error(int code, const std::string &msg) {
    (void)code;
    g_error = msg;
}

const char *last_error() { return g_error.c_str(); }

int cuda_fail(cudaError_t e, const char *what) {
    g_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return e == cudaErrorMemoryAllocation ? DR_ERR_NOMEM : DR_ERR_CUDA;
}

int need(bool ok, int code, const char *msg) {
    if (!ok) set_error(code, msg);
    return ok ? DR_OK : code;
}

// Exact-mode phase sampler table (DR_PHASE_MIE_EXACT).  Target density over
// phi = acos(-ct): f(phi) sin(phi), f the red pdf column interpolated linearly
// in phi as MiePhase::Evaluate does (src/KernelSampler.cpp:214-231; knots at
// k pi / n, the last bin extrapolating the last two entries, clamped at 0).
// Per bin k, in FP64: f0 = f(phi_k), beta = slope, mass
//   M_k = S[(f0 + beta d) sin d - beta (1 - cos d)] + C[f0 (1 - cos d) + beta (sin d - d cos d)]
// (the integral of f sin over the bin, d = pi/n, S, C = sin, cos phi_k).
// Layout (float): per bin (cdf_k, f0, beta, M_k), (S, C, d, 0); then (1, 0, 0, 0).
static void mie_exact_table(const float *pdf_rgb, uint32_t n, float *out) {
    const double d = 3.14159265358979323846 / (double)n;
    std::vector<double> mass(n);
    double total = 0.0;
    for (uint32_t k = 0; k < n; ++k) {
        double fa = k + 1 < n ? (double)pdf_rgb[3 * k] : (double)pdf_rgb[3 * (n - 1)];
        double fb = k + 1 < n ? (double)pdf_rgb[3 * (k + 1)]
                              : 2.0 * (double)pdf_rgb[3 * (n - 1)] - (double)pdf_rgb[3 * (n - 2)];
        fa = fa < 0.0 ? 0.0 : fa;
        fb = fb < 0.0 ? 0.0 : fb;
        const double beta = (fb - fa) / d, phi = d * (double)k;
        const double S = std::sin(phi), C = std::cos(phi);
        const double m = S * ((fa + beta * d) * std::sin(d) - beta * (1.0 - std::cos(d))) +
                         C * (fa * (1.0 - std::cos(d)) + beta * (std::sin(d) - d * std::cos(d)));
        mass[k] = m > 0.0 ? m : 0.0;
        float *o = out + 8 * (size_t)k;
        o[1] = (float)fa;
        o[2] = (float)beta;
        o[3] = (float)mass[k];
        o[4] = (float)S;
        o[5] = (float)C;
        o[6] = (float)d;
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
}

int prepare_scene(const dr_scene_desc *s, HostScene &out) {
    if (!s || !s->nodes || !s->bricks) return need(false, DR_ERR_INVALID, "dr_upload_scene: null argument");
    if (s->lvoxc != kLvox) return need(false, DR_ERR_INVALID, "dr_upload_scene: bricks must be 8^3");
    if (s->n_nodes < 2 || s->n_nodes >= kLeafBit)
        return need(false, DR_ERR_INVALID, "dr_upload_scene: need 2 <= n_nodes < 2^31");
    const dr_node *N = s->nodes;
    auto is_leaf = [&](uint32_t i) { return N[i].volx[0] != DR_NONE || N[i].volx[1] != DR_NONE; };
    if (is_leaf(0)) return need(false, DR_ERR_INVALID, "dr_upload_scene: the root must be an internal node");
    std::vector<uint32_t> &child = out.child;
    std::vector<float4> &leaf = out.leaf;
    child.assign((size_t)s->n_nodes * 8, 0u);
    leaf.assign((size_t)s->n_nodes * 2, make_float4(0.f, 0.f, 0.f, 0.f));
    for (uint32_t i = 0; i < s->n_nodes; ++i) {
        const dr_node &o = N[i];
        if (is_leaf(i)) {
            const bool sdf = o.volx[0] != DR_NONE, fog = o.volx[1] != DR_NONE;
            if (sdf && (!s->sdf_bricks || o.volx[0] >= s->n_sdf_leaves))
                return need(false, DR_ERR_INVALID, "dr_upload_scene: SDF brick index out of range (or no SDF pool)");
            if (fog && o.volx[1] >= s->n_leaves)
                return need(false, DR_ERR_INVALID, "dr_upload_scene: brick index out of range");
            if (!(o.ce[3] > 0.0f) || !std::isfinite(o.ce[3]) ||
                (!sdf && (!(o.qval[1] >= 0.0f) || !std::isfinite(o.qval[1]))))
                return need(false, DR_ERR_INVALID, "dr_upload_scene: leaf with bad extent or majorant");
            float fb, sb;
            std::memcpy(&fb, &o.volx[1], 4);  // index bits (kNone when absent)
            std::memcpy(&sb, &o.volx[0], 4);
            leaf[2 * (size_t)i] = make_float4(o.ce[0], o.ce[1], o.ce[2], o.ce[3]);
            // src/kernel.cpp:245-251: an SDF leaf's majorant is 1, a fog leaf's qval[FOG]
            leaf[2 * (size_t)i + 1] = make_float4(sdf ? 1.0f : o.qval[1], fb, sb, 0.0f);
        } else {
            leaf[2 * (size_t)i] = make_float4(o.ce[0], o.ce[1], o.ce[2], o.ce[3]);
            leaf[2 * (size_t)i + 1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        for (int k = 0; k < 8; ++k) {
            const uint32_t ch = o.chn[k];
            if (ch == 0) {
                child[8 * (size_t)i + k] = 0;
                continue;
            }
            if (ch >= s->n_nodes || ch == i)
                return need(false, DR_ERR_INVALID, "dr_upload_scene: child index out of range");
            child[8 * (size_t)i + k] = is_leaf(ch) ? (ch | kLeafBit) : ch;
        }
    }
    // Leaf grid for the cell-walk traversal: valid when the tree is a tree (each
    // node reached once from the root) and every leaf sits at the same depth.
    std::vector<uint32_t> &macro = out.macro, &cells = out.cells;
    macro.clear();
    cells.clear();
    uint32_t levels = 0, n = 0, mdim = 0;
    {
        struct Item { uint32_t node, depth, x, y, z; };
        std::vector<Item> stack{{0u, 0u, 0u, 0u, 0u}};
        std::vector<uint8_t> seen(s->n_nodes, 0);
        std::vector<Item> leaves;
        bool ok = true;
        int leaf_depth = -1;
        while (!stack.empty() && ok) {
            Item it = stack.back();
            stack.pop_back();
            if (seen[it.node] || it.depth > 11) { ok = false; break; }
            seen[it.node] = 1;
            if (is_leaf(it.node)) {
                if (leaf_depth < 0) leaf_depth = (int)it.depth;
                if ((int)it.depth != leaf_depth) ok = false;
                leaves.push_back(it);
                continue;
            }
            for (uint32_t k = 0; k < 8; ++k) {
                const uint32_t ch = N[it.node].chn[k];
                if (ch) stack.push_back({ch, it.depth + 1, 2 * it.x + (k & 1), 2 * it.y + ((k >> 1) & 1), 2 * it.z + (k >> 2)});
            }
        }
        if (ok && leaf_depth >= 1) {
            levels = (uint32_t)leaf_depth;
            n = 1u << levels;
            mdim = n >= 8 ? n / 8 : 1;
            macro.assign((size_t)mdim * mdim * mdim, kNone);
            for (const Item &lf : leaves) {
                const size_t m = ((size_t)(lf.z >> 3) * mdim + (lf.y >> 3)) * mdim + (lf.x >> 3);
                if (macro[m] == kNone) {
                    macro[m] = (uint32_t)(cells.size() / 512);
                    cells.resize(cells.size() + 512, kNone);
                }
                cells[(size_t)macro[m] * 512 + (lf.z & 7) * 64 + (lf.y & 7) * 8 + (lf.x & 7)] = lf.node;
            }
        } else {
            macro.assign(1, kNone);
        }
        if (cells.empty()) cells.assign(512, kNone);
    }
    out.levels = levels;
    // a tree with every leaf at depth d pushes at most d - 1 ancestors; the
    // shared-memory stack packs node ids into 25 bits
    out.stack_levels = (levels >= 2 && s->n_nodes < (1u << 25)) ? levels - 1 : 0u;
    out.n = n;
    out.mdim = mdim;
    out.n_nodes = s->n_nodes;
    out.n_leaves = s->n_leaves;
    for (int k = 0; k < 4; ++k) out.root_ce[k] = N[0].ce[k];
    out.leaf_flag.assign(s->n_nodes, 0);
    for (uint32_t i = 0; i < s->n_nodes; ++i) out.leaf_flag[i] = is_leaf(i) ? 1 : 0;
    out.bricks = s->bricks;
    out.sdf = s->sdf_bricks;
    out.n_sdf = s->sdf_bricks ? s->n_sdf_leaves : 0u;
    for (uint32_t i = 0; i < s->n_nodes; ++i)
        if (is_leaf(i)) out.leaf_flag[i] = (uint8_t)(1u | (N[i].volx[1] != DR_NONE ? 2u : 0u) | (N[i].volx[0] != DR_NONE ? 4u : 0u));
    return DR_OK;
}

int upload_scene(const HostScene &h, SceneBufs &b, bool use_grid, cudaStream_t st, DevScene &S) {
    const size_t nb = (size_t)h.n_leaves * kBrick;
    DR_CUDA(cudaStreamSynchronize(st), "dr_upload_scene: sync");
    DR_CUDA(b.macro.reserve(h.macro.size()), "dr_upload_scene: alloc grid");
    DR_CUDA(b.cells.reserve(h.cells.size()), "dr_upload_scene: alloc grid");
    DR_CUDA(cudaMemcpyAsync(b.macro.p, h.macro.data(), h.macro.size() * 4, cudaMemcpyHostToDevice, st),
            "dr_upload_scene: copy grid");
    DR_CUDA(cudaMemcpyAsync(b.cells.p, h.cells.data(), h.cells.size() * 4, cudaMemcpyHostToDevice, st),
            "dr_upload_scene: copy grid");
    DR_CUDA(b.child.reserve((size_t)h.n_nodes * 2), "dr_upload_scene: alloc nodes");
    DR_CUDA(b.leaf.reserve((size_t)h.n_nodes * 2), "dr_upload_scene: alloc leaves");
    DR_CUDA(b.bricks.reserve(nb + 1), "dr_upload_scene: alloc bricks");
    DR_CUDA(cudaMemcpyAsync(b.child.p, h.child.data(), h.child.size() * 4, cudaMemcpyHostToDevice, st),
            "dr_upload_scene: copy nodes");
    DR_CUDA(cudaMemcpyAsync(b.leaf.p, h.leaf.data(), h.leaf.size() * sizeof(float4), cudaMemcpyHostToDevice, st),
            "dr_upload_scene: copy leaves");
    if (nb)
        DR_CUDA(cudaMemcpyAsync(b.bricks.p, h.bricks, nb * 4, cudaMemcpyHostToDevice, st),
                "dr_upload_scene: copy bricks");
    const size_t ns = (size_t)h.n_sdf * kBrick;
    if (ns) {
        DR_CUDA(b.sdf.reserve(ns), "dr_upload_scene: alloc SDF bricks");
        DR_CUDA(cudaMemcpyAsync(b.sdf.p, h.sdf, ns * 4, cudaMemcpyHostToDevice, st), "dr_upload_scene: copy SDF bricks");
    }
    DR_CUDA(cudaStreamSynchronize(st), "dr_upload_scene: sync");
    S.child = b.child.p;
    S.leaf = b.leaf.p;
    S.bricks = b.bricks.p;
    S.sdf_bricks = ns ? b.sdf.p : nullptr;
    for (int k = 0; k < 4; ++k) S.root_ce[k] = h.root_ce[k];
    S.n_nodes = h.n_nodes;
    S.n_leaves = h.n_leaves;
    S.macro = b.macro.p;
    S.cells = b.cells.p;
    S.levels = use_grid ? h.levels : 0u;
    S.n = h.n;
    S.mdim = h.mdim;
    S.stack_levels = h.stack_levels;
    S.occ_nodes = nullptr;
    S.occ_tris = nullptr;
    S.occ_n_nodes = 0;
    return DR_OK;
}

int prepare_params(const dr_render_params *p, DevParams &d, std::vector<unsigned char> &pack) {
    if (!p) return need(false, DR_ERR_INVALID, "dr_set_params: null argument");
    if (p->phase_mode != DR_PHASE_MIE_REFERENCE && p->phase_mode != DR_PHASE_MIE_EXACT && p->phase_mode != DR_PHASE_HG)
        return need(false, DR_ERR_INVALID, "dr_set_params: unknown phase mode");
    if (p->phase_mode == DR_PHASE_HG && !(std::fabs(p->hg_g) < 1.0f))
        return need(false, DR_ERR_INVALID, "dr_set_params: HG anisotropy needs |g| < 1");
    // the HG phase needs no table: stage a 4-entry placeholder when none is given
    static const float kNoTable[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    dr_render_params q = *p;
    if (p->phase_mode == DR_PHASE_HG && (!p->mie_pdf || !p->mie_cdf || p->mie_n == 0)) {
        q.mie_pdf = kNoTable;
        q.mie_cdf = kNoTable;
        q.mie_n = 4;
    }
    p = &q;
    if (!p->mie_pdf || !p->mie_cdf || p->mie_n < 4 || p->mie_n > kMieMax || (p->mie_n % 4))
        return need(false, DR_ERR_INVALID, "dr_set_params: phase tables need 4 <= mie_n <= 4096, mie_n % 4 == 0");
    if (p->env_mode != DR_ENV_HOSEK && p->env_mode != DR_ENV_NONE && p->env_mode != DR_ENV_MAP)
        return need(false, DR_ERR_INVALID, "dr_set_params: unknown environment mode");
    // texel indices are formed in binary32 (as MapEnv::Evaluate does): exact below 2^24
    if (p->env_mode == DR_ENV_MAP && (!p->env_map || p->env_w < 2 || p->env_h < 2 ||
                                      (uint64_t)p->env_w * p->env_h > (1ull << 24)))
        return need(false, DR_ERR_INVALID, "dr_set_params: environment map needs 2 <= w, h and w*h <= 2^24 texels");
    if (p->phase_mode == DR_PHASE_MIE_EXACT && p->mie_n > 512)
        return need(false, DR_ERR_INVALID, "dr_set_params: the exact phase sampler takes mie_n <= 512");
    for (uint32_t i = 0; i < p->mie_n; ++i)
        if (!(p->mie_pdf[3 * i] >= 0.0f) || !std::isfinite(p->mie_pdf[3 * i]))
            return need(false, DR_ERR_INVALID, "dr_set_params: phase pdf must be finite and >= 0");
    if (p->w == 0 || p->h == 0) return need(false, DR_ERR_INVALID, "dr_set_params: empty image");
    if (p->scattevs > 100000u) return need(false, DR_ERR_INVALID, "dr_set_params: scattevs above 100000");
    if (!(p->sigma_s >= 0.0f) || !(p->sigma_a >= 0.0f) || !(p->sigma_s + p->sigma_a > 0.0f))
        return need(false, DR_ERR_INVALID, "dr_set_params: cross sections must be >= 0 with a positive sum");
    d = DevParams{};
    d.sigma_s = p->sigma_s;
    d.sigma_a = p->sigma_a;
    d.sigma_e = p->sigma_a + p->sigma_s;                 // msigmae = msigmaa + msigmas
    d.albedo = p->sigma_s / (p->sigma_a + p->sigma_s);
    d.scattevs = p->scattevs;
    for (int k = 0; k < 3; ++k) {
        d.sun_dir[k] = p->sun_dir[k];
        d.sun_color[k] = p->sun_color[k];
    }
    d.sun_cos = std::cos(p->sun_angle);                  // SunLight ctor: cosf(angle)
    const float ctm = d.sun_cos;
    d.sun_pdf = 1.0f / ((2.0f * 3.14159265358979f) * (1.0f - ctm * ctm));  // SunLight::Pdf
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 9; ++j) d.sky_cfg[i][j] = (float)p->sky_configs[i][j];
        d.sky_rad[i] = (float)p->sky_radiances[i];
    }
    d.mie_n = p->mie_n;
    d.phase_mode = p->phase_mode;
    std::memcpy(d.viewi, p->viewi, sizeof(d.viewi));
    std::memcpy(d.proji, p->proji, sizeof(d.proji));
    d.w = p->w;
    d.h = p->h;
    d.depthcomp = (p->flags & DR_KERNEL_DEPTHCOMP) ? 1u : 0u;
    d.finite_paths = (p->flags & DR_KERNEL_FINITE_PATHS) ? 1u : 0u;
    d.embree = (p->flags & DR_KERNEL_EMBREE) ? 1u : 0u;
    d.hg_g = p->hg_g;
    d.env_mode = p->env_mode;
    d.env_w = p->env_mode == DR_ENV_MAP ? p->env_w : 0u;
    d.env_h = p->env_mode == DR_ENV_MAP ? p->env_h : 0u;
    d.env_map = nullptr;  // the caller copies the texels to the device
    if (p->flags & ~(DR_KERNEL_DEPTHCOMP | DR_KERNEL_FINITE_PATHS | DR_KERNEL_EMBREE))
        return need(false, DR_ERR_INVALID, "dr_set_params: unknown flags");
    {
        // RenderKernel::Shadow: zfar = (0,0,1,1) * projInv, clip_end = -zfar.z / zfar.w
        const float zz = p->proji[8 + 2] + p->proji[12 + 2], zw = p->proji[8 + 3] + p->proji[12 + 3];
        d.clip_end = -zz / zw;
    }
    d.step_budget = kStepBudget;
    const size_t n_ex = p->phase_mode == DR_PHASE_MIE_EXACT ? 8 * (size_t)p->mie_n + 4 : 0;
    pack.assign((size_t)p->mie_n * 20 + 4 * n_ex, 0);
    for (uint32_t i = 0; i < p->mie_n; ++i) {
        float4 v = make_float4(p->mie_pdf[3 * i], p->mie_pdf[3 * i + 1], p->mie_pdf[3 * i + 2], 0.0f);
        std::memcpy(&pack[16 * (size_t)i], &v, 16);
        std::memcpy(&pack[16 * (size_t)p->mie_n + 4 * (size_t)i], &p->mie_cdf[3 * i], 4);
    }
    if (n_ex) {
        std::vector<float> ex(n_ex);
        mie_exact_table(p->mie_pdf, p->mie_n, ex.data());
        std::memcpy(&pack[20 * (size_t)p->mie_n], ex.data(), 4 * n_ex);
    }
    d.depth = nullptr;
    d.mie_pdf = nullptr;
    d.mie_cdf = nullptr;
    d.mie_exact = nullptr;
    return DR_OK;
}

size_t mie_pack_bytes(const DevParams &d) {
    return (size_t)d.mie_n * 20u + (d.phase_mode == DR_PHASE_MIE_EXACT ? (2u * (size_t)d.mie_n + 1u) * 16u : 0u);
}

int make_tile_args(uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed, uint64_t base,
                   uint32_t tile, TileArgs &A) {
    if (tw == 0 || th == 0) return need(false, DR_ERR_INVALID, "render: empty tile");
    if (tile > 64) return need(false, DR_ERR_INVALID, "render: tile side above 64");
    A.x0 = x0;
    A.y0 = y0;
    A.tw = tw;
    A.th = th;
    A.cols = 2 * (tw / 2);
    A.rows = 2 * (th / 2);
    A.spp = spp;
    A.tile = tile;
    A.tiles_x = tile ? (A.cols + tile - 1) / tile : 0u;
    A.seed = seed;
    A.sample_base = base;
    A.defer_sky = 0;
    A.cam_head = nullptr;
    A.cam_pool = nullptr;
    A.spp_div = make_fastdiv(spp);
    A.cols_div = make_fastdiv(A.cols);
    A.t2_div = make_fastdiv(tile * tile);
    A.tx_div = make_fastdiv(A.tiles_x);
    A.tile_div = make_fastdiv(tile);
    if (tile) {
        const uint64_t ty = (A.rows + tile - 1) / tile;
        A.n_paths = (uint64_t)A.tiles_x * ty * tile * tile * spp;
    } else {
        A.n_paths = (uint64_t)A.cols * A.rows * spp;
    }
    return DR_OK;
}

bool valid_tuning(const dr_tuning *t) {
    return t && t->kernel <= DR_KERNEL_PER_PATH && t->event_batch <= 32 && t->blocks_per_sm <= 64 &&
           t->traversal <= 2 && t->tile <= 64 && t->visits <= 255 && t->steps <= 255;
}

}  // namespace dr
