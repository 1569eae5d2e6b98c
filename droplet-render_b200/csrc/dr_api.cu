// C ABI of droplet_b200 (declared in include/droplet_b200.h).
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/droplet_b200.h"
#include "dr_internal.h"
#include "dr_kernels.h"

namespace dr {

static thread_local std::string g_error;

void set_error(int code, const std::string &msg) {
    (void)code;
    g_error = msg;
}

int build_octree(const int32_t *org, const float *vals, uint32_t n_blocks, float s, uint32_t maxdepth, int nthreads,
                 dr_octree *out);
int sky_cook(const double *const rgb[3], const double *const rad[3], double turbidity, double albedo,
             double elevation, double configs[3][9], double radiances[3]);

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

static int cuda_fail(cudaError_t e, const char *what) {
    g_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return e == cudaErrorMemoryAllocation ? DR_ERR_NOMEM : DR_ERR_CUDA;
}

#define DR_CUDA(call, what)                                  \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(e_, what);   \
    } while (0)

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaError_t reserve(size_t count) {
        if (count <= n && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, sizeof(T) * (count ? count : 1));
        if (e == cudaSuccess) n = count;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

}  // namespace dr

using namespace dr;

struct dr_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    bool has_scene = false, has_params = false;
    DevScene scene{};
    DevParams params{};
    DevBuf<uint4> child;
    DevBuf<float4> leaf;
    DevBuf<float> bricks;
    DevBuf<unsigned char> mie_pack;
    DevBuf<float> depth;
    DevBuf<DevCounters> counters;
    DevBuf<float4> tile_sun, tile_sky;
    DevBuf<unsigned char> scratch;
    DevBuf<WorkQueue> work;
    DevBuf<uint32_t> macro, cells;
    bool use_grid = true;
    Tuning tuning{0u, 128u, 0u, 8u, 0u};
    std::vector<uint8_t> leaf_flag;  // host copy: node i is a leaf (for validating probe inputs)
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int need(bool ok, int code, const char *msg) {
    if (!ok) set_error(code, msg);
    return ok ? DR_OK : code;
}

}  // namespace

extern "C" {

int dr_version(void) { return 100; }

const char *dr_last_error(void) { return g_error.c_str(); }

int dr_device_count(int *count) {
    if (!count) return need(false, DR_ERR_INVALID, "dr_device_count: null output");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *count = 0;
        if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) {
            set_error(DR_ERR_NODEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
            return DR_ERR_NODEVICE;
        }
        return cuda_fail(e, "cudaGetDeviceCount");
    }
    *count = n;
    return DR_OK;
}

int dr_create(int device, dr_ctx **out) {
    if (!out) return need(false, DR_ERR_INVALID, "dr_create: null output");
    *out = nullptr;
    int n = 0;
    int rc = dr_device_count(&n);
    if (rc != DR_OK) return rc;
    if (device < 0 || device >= n) {
        set_error(DR_ERR_NODEVICE, "dr_create: device index out of range");
        return DR_ERR_NODEVICE;
    }
    DeviceGuard g(device);
    dr_ctx *c = new dr_ctx();
    c->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = c->counters.reserve(1);
    if (e == cudaSuccess) e = cudaMemset(c->counters.p, 0, sizeof(DevCounters));
    if (e == cudaSuccess) e = c->work.reserve(1);
    if (e != cudaSuccess) {
        int r = cuda_fail(e, "dr_create");
        if (c->stream) cudaStreamDestroy(c->stream);
        c->counters.release();
        delete c;
        return r;
    }
    *out = c;
    return DR_OK;
}

int dr_destroy(dr_ctx *c) {
    if (!c) return DR_OK;
    {
        DeviceGuard g(c->device);
        std::lock_guard<std::mutex> lk(c->mu);
        if (c->stream) cudaStreamSynchronize(c->stream);
        c->child.release();
        c->leaf.release();
        c->bricks.release();
        c->mie_pack.release();
        c->depth.release();
        c->counters.release();
        c->tile_sun.release();
        c->tile_sky.release();
        c->scratch.release();
        c->work.release();
        c->macro.release();
        c->cells.release();
        if (c->stream) cudaStreamDestroy(c->stream);
    }
    delete c;
    return DR_OK;
}

int dr_build_octree(const int32_t *block_origin, const float *block_values, uint32_t n_blocks, float voxel_size,
                    uint32_t maxdepth, int nthreads, dr_octree *out) {
    if (out) std::memset(out, 0, sizeof(*out));
    return build_octree(block_origin, block_values, n_blocks, voxel_size, maxdepth, nthreads, out);
}

void dr_octree_free(dr_octree *oct) {
    if (!oct) return;
    std::free(oct->nodes);
    std::free(oct->bricks);
    std::memset(oct, 0, sizeof(*oct));
}

int dr_sky_cook(const double *const dataset_rgb[3], const double *const dataset_rad[3], double turbidity,
                double albedo, double elevation, double configs[3][9], double radiances[3]) {
    return sky_cook(dataset_rgb, dataset_rad, turbidity, albedo, elevation, configs, radiances);
}

int dr_upload_scene(dr_ctx *c, const dr_scene_desc *s) {
    if (!c || !s || !s->nodes || !s->bricks) return need(false, DR_ERR_INVALID, "dr_upload_scene: null argument");
    if (s->lvoxc != kLvox) return need(false, DR_ERR_INVALID, "dr_upload_scene: bricks must be 8^3");
    if (s->n_nodes < 2 || s->n_nodes >= kLeafBit)
        return need(false, DR_ERR_INVALID, "dr_upload_scene: need 2 <= n_nodes < 2^31");
    const dr_node *N = s->nodes;
    auto is_leaf = [&](uint32_t i) { return N[i].volx[0] != DR_NONE || N[i].volx[1] != DR_NONE; };
    if (is_leaf(0)) return need(false, DR_ERR_INVALID, "dr_upload_scene: the root must be an internal node");
    std::vector<uint32_t> child((size_t)s->n_nodes * 8);
    std::vector<float4> leaf((size_t)s->n_nodes * 2);
    for (uint32_t i = 0; i < s->n_nodes; ++i) {
        const dr_node &o = N[i];
        if (o.volx[0] != DR_NONE)
            return need(false, DR_ERR_INVALID, "dr_upload_scene: surface (SDF) leaves are not supported");
        if (is_leaf(i)) {
            if (o.volx[1] >= s->n_leaves)
                return need(false, DR_ERR_INVALID, "dr_upload_scene: brick index out of range");
            if (!(o.ce[3] > 0.0f) || !std::isfinite(o.ce[3]) || !(o.qval[1] >= 0.0f) || !std::isfinite(o.qval[1]))
                return need(false, DR_ERR_INVALID, "dr_upload_scene: leaf with bad extent or majorant");
            uint32_t bits;
            std::memcpy(&bits, &o.volx[1], 4);
            float fb;
            std::memcpy(&fb, &bits, 4);
            leaf[2 * (size_t)i] = make_float4(o.ce[0], o.ce[1], o.ce[2], o.ce[3]);
            leaf[2 * (size_t)i + 1] = make_float4(o.qval[1], fb, 0.0f, 0.0f);
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
    std::vector<uint32_t> macro, cells;
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
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    const size_t nb = (size_t)s->n_leaves * kBrick;
    DR_CUDA(cudaStreamSynchronize(c->stream), "dr_upload_scene: sync");
    DR_CUDA(c->macro.reserve(macro.size()), "dr_upload_scene: alloc grid");
    DR_CUDA(c->cells.reserve(cells.size()), "dr_upload_scene: alloc grid");
    DR_CUDA(cudaMemcpyAsync(c->macro.p, macro.data(), macro.size() * 4, cudaMemcpyHostToDevice, c->stream),
            "dr_upload_scene: copy grid");
    DR_CUDA(cudaMemcpyAsync(c->cells.p, cells.data(), cells.size() * 4, cudaMemcpyHostToDevice, c->stream),
            "dr_upload_scene: copy grid");
    DR_CUDA(c->child.reserve((size_t)s->n_nodes * 2), "dr_upload_scene: alloc nodes");
    DR_CUDA(c->leaf.reserve((size_t)s->n_nodes * 2), "dr_upload_scene: alloc leaves");
    DR_CUDA(c->bricks.reserve(nb + 1), "dr_upload_scene: alloc bricks");
    DR_CUDA(cudaMemcpyAsync(c->child.p, child.data(), child.size() * 4, cudaMemcpyHostToDevice, c->stream),
            "dr_upload_scene: copy nodes");
    DR_CUDA(cudaMemcpyAsync(c->leaf.p, leaf.data(), leaf.size() * sizeof(float4), cudaMemcpyHostToDevice, c->stream),
            "dr_upload_scene: copy leaves");
    if (nb)
        DR_CUDA(cudaMemcpyAsync(c->bricks.p, s->bricks, nb * 4, cudaMemcpyHostToDevice, c->stream),
                "dr_upload_scene: copy bricks");
    DR_CUDA(cudaStreamSynchronize(c->stream), "dr_upload_scene: sync");
    c->scene.child = c->child.p;
    c->scene.leaf = c->leaf.p;
    c->scene.bricks = c->bricks.p;
    for (int k = 0; k < 4; ++k) c->scene.root_ce[k] = N[0].ce[k];
    c->scene.n_nodes = s->n_nodes;
    c->scene.n_leaves = s->n_leaves;
    c->scene.macro = c->macro.p;
    c->scene.cells = c->cells.p;
    c->scene.levels = c->use_grid ? levels : 0u;
    c->scene.n = n;
    c->scene.mdim = mdim;
    c->leaf_flag.assign(s->n_nodes, 0);
    for (uint32_t i = 0; i < s->n_nodes; ++i) c->leaf_flag[i] = is_leaf(i) ? 1 : 0;
    c->has_scene = true;
    return DR_OK;
}

int dr_set_params(dr_ctx *c, const dr_render_params *p) {
    if (!c || !p) return need(false, DR_ERR_INVALID, "dr_set_params: null argument");
    if (!p->mie_pdf || !p->mie_cdf || p->mie_n < 4 || p->mie_n > kMieMax || (p->mie_n % 4))
        return need(false, DR_ERR_INVALID, "dr_set_params: phase tables need 4 <= mie_n <= 4096, mie_n % 4 == 0");
    if (p->phase_mode != DR_PHASE_MIE_REFERENCE && p->phase_mode != DR_PHASE_MIE_EXACT)
        return need(false, DR_ERR_INVALID, "dr_set_params: unknown phase mode");
    if (p->phase_mode == DR_PHASE_MIE_EXACT && p->mie_n > 512)
        return need(false, DR_ERR_INVALID, "dr_set_params: the exact phase sampler takes mie_n <= 512");
    for (uint32_t i = 0; i < p->mie_n; ++i)
        if (!(p->mie_pdf[3 * i] >= 0.0f) || !std::isfinite(p->mie_pdf[3 * i]))
            return need(false, DR_ERR_INVALID, "dr_set_params: phase pdf must be finite and >= 0");
    if (p->w == 0 || p->h == 0) return need(false, DR_ERR_INVALID, "dr_set_params: empty image");
    if (p->scattevs > 100000u) return need(false, DR_ERR_INVALID, "dr_set_params: scattevs above 100000");
    if (!(p->sigma_s >= 0.0f) || !(p->sigma_a >= 0.0f) || !(p->sigma_s + p->sigma_a > 0.0f))
        return need(false, DR_ERR_INVALID, "dr_set_params: cross sections must be >= 0 with a positive sum");
    DevParams d{};
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
    {
        // RenderKernel::Shadow: zfar = (0,0,1,1) * projInv, clip_end = -zfar.z / zfar.w
        const float zz = p->proji[8 + 2] + p->proji[12 + 2], zw = p->proji[8 + 3] + p->proji[12 + 3];
        d.clip_end = -zz / zw;
    }
    const size_t n_ex = p->phase_mode == DR_PHASE_MIE_EXACT ? 8 * (size_t)p->mie_n + 4 : 0;
    std::vector<unsigned char> pack((size_t)p->mie_n * 20 + 4 * n_ex);
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
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    DR_CUDA(cudaStreamSynchronize(c->stream), "dr_set_params: sync");
    DR_CUDA(c->mie_pack.reserve(pack.size()), "dr_set_params: alloc tables");
    DR_CUDA(cudaMemcpy(c->mie_pack.p, pack.data(), pack.size(), cudaMemcpyHostToDevice), "dr_set_params: copy tables");
    if (p->depth) {
        DR_CUDA(c->depth.reserve((size_t)p->w * p->h), "dr_set_params: alloc depth");
        DR_CUDA(cudaMemcpy(c->depth.p, p->depth, sizeof(float) * p->w * p->h, cudaMemcpyHostToDevice),
                "dr_set_params: copy depth");
        d.depth = c->depth.p;
    } else {
        d.depth = nullptr;
    }
    d.mie_pdf = nullptr;
    d.mie_cdf = nullptr;
    d.mie_exact = nullptr;
    c->params = d;
    c->has_params = true;
    return DR_OK;
}

static int tile_args(const dr_ctx *c, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed,
                     uint64_t base, TileArgs &A) {
    if (!c->has_scene || !c->has_params)
        return need(false, DR_ERR_STATE, "render: upload a scene and set parameters first");
    if (tw == 0 || th == 0) return need(false, DR_ERR_INVALID, "render: empty tile");
    A.x0 = x0;
    A.y0 = y0;
    A.tw = tw;
    A.th = th;
    A.cols = 2 * (tw / 2);
    A.rows = 2 * (th / 2);
    A.spp = spp;
    A.seed = seed;
    A.sample_base = base;
    A.n_paths = (uint64_t)A.cols * A.rows * spp;
    return DR_OK;
}

int dr_render_tile_async(dr_ctx *c, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed,
                         uint64_t sample_base, float *sun_dev, float *sky_dev, void *stream) {
    if (!c || !sun_dev || !sky_dev) return need(false, DR_ERR_INVALID, "dr_render_tile_async: null argument");
    TileArgs A;
    int rc = tile_args(c, x0, y0, tw, th, spp, seed, sample_base, A);
    if (rc != DR_OK) return rc;
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    const size_t bytes = (size_t)tw * th * sizeof(float4);
    DR_CUDA(cudaMemsetAsync(sun_dev, 0, bytes, st), "render: clear");
    DR_CUDA(cudaMemsetAsync(sky_dev, 0, bytes, st), "render: clear");
    if (c->tuning.kernel == DR_KERNEL_PER_PATH) {
        DR_CUDA(launch_render_tile(c->scene, c->params, A, c->mie_pack.p, (float4 *)sun_dev, (float4 *)sky_dev,
                                   c->counters.p, st),
                "render: launch");
    } else {
        DR_CUDA(launch_render_persistent(c->scene, c->params, A, c->mie_pack.p, (float4 *)sun_dev, (float4 *)sky_dev,
                                         c->counters.p, c->work.p, c->tuning, c->device, st),
                "render: launch");
    }
    return DR_OK;
}

int dr_shadow_tile_async(dr_ctx *c, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed,
                         uint64_t sample_base, float *out_dev, void *stream) {
    if (!c || !out_dev) return need(false, DR_ERR_INVALID, "dr_shadow_tile_async: null argument");
    TileArgs A;
    int rc = tile_args(c, x0, y0, tw, th, spp, seed, sample_base, A);
    if (rc != DR_OK) return rc;
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    DR_CUDA(cudaMemsetAsync(out_dev, 0, (size_t)tw * th * sizeof(float4), st), "shadow: clear");
    DR_CUDA(launch_shadow_tile(c->scene, c->params, A, (float4 *)out_dev, c->counters.p, st), "shadow: launch");
    return DR_OK;
}

int dr_shadow_tile(dr_ctx *c, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed,
                   uint64_t sample_base, float *out) {
    if (!c || !out) return need(false, DR_ERR_INVALID, "dr_shadow_tile: null argument");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    const size_t n = (size_t)tw * th;
    DR_CUDA(c->tile_sun.reserve(n), "shadow: alloc tile");
    int rc = dr_shadow_tile_async(c, x0, y0, tw, th, spp, seed, sample_base, (float *)c->tile_sun.p, nullptr);
    if (rc != DR_OK) return rc;
    DR_CUDA(cudaMemcpyAsync(out, c->tile_sun.p, n * sizeof(float4), cudaMemcpyDeviceToHost, c->stream),
            "shadow: copy out");
    DR_CUDA(cudaStreamSynchronize(c->stream), "shadow: sync");
    return DR_OK;
}

int dr_set_tuning(dr_ctx *c, const dr_tuning *t) {
    if (!c || !t) return need(false, DR_ERR_INVALID, "dr_set_tuning: null argument");
    if (t->kernel > DR_KERNEL_PER_PATH || t->event_batch > 32 || t->blocks_per_sm > 64 || t->traversal > 1)
        return need(false, DR_ERR_INVALID,
                    "dr_set_tuning: kernel 0/1, event_batch <= 32, blocks_per_sm <= 64, traversal 0/1");
    c->tuning.kernel = t->kernel;
    c->tuning.block = kPersistentBlock;
    c->tuning.blocks_per_sm = t->blocks_per_sm;
    c->tuning.event_batch = t->event_batch;
    c->tuning.traversal = t->traversal;
    return DR_OK;
}

int dr_get_tuning(dr_ctx *c, dr_tuning *t) {
    if (!c || !t) return need(false, DR_ERR_INVALID, "dr_get_tuning: null argument");
    t->kernel = c->tuning.kernel;
    t->blocks_per_sm = c->tuning.blocks_per_sm;
    t->event_batch = c->tuning.event_batch;
    t->traversal = c->tuning.traversal;
    return DR_OK;
}

int dr_render_tile(dr_ctx *c, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed,
                   uint64_t sample_base, float *sun_out, float *sky_out) {
    if (!c || !sun_out || !sky_out) return need(false, DR_ERR_INVALID, "dr_render_tile: null argument");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    const size_t n = (size_t)tw * th;
    DR_CUDA(c->tile_sun.reserve(n), "render: alloc tile");
    DR_CUDA(c->tile_sky.reserve(n), "render: alloc tile");
    int rc = dr_render_tile_async(c, x0, y0, tw, th, spp, seed, sample_base, (float *)c->tile_sun.p,
                                  (float *)c->tile_sky.p, nullptr);
    if (rc != DR_OK) return rc;
    DR_CUDA(cudaMemcpyAsync(sun_out, c->tile_sun.p, n * sizeof(float4), cudaMemcpyDeviceToHost, c->stream),
            "render: copy out");
    DR_CUDA(cudaMemcpyAsync(sky_out, c->tile_sky.p, n * sizeof(float4), cudaMemcpyDeviceToHost, c->stream),
            "render: copy out");
    DR_CUDA(cudaStreamSynchronize(c->stream), "render: sync");
    return DR_OK;
}

int dr_synchronize(dr_ctx *c) {
    if (!c) return need(false, DR_ERR_INVALID, "dr_synchronize: null context");
    DeviceGuard g(c->device);
    DR_CUDA(cudaStreamSynchronize(c->stream), "dr_synchronize");
    return DR_OK;
}

int dr_get_counters(dr_ctx *c, dr_counters *out) {
    if (!c || !out) return need(false, DR_ERR_INVALID, "dr_get_counters: null argument");
    DeviceGuard g(c->device);
    DevCounters h{};
    DR_CUDA(cudaStreamSynchronize(c->stream), "dr_get_counters: sync");
    DR_CUDA(cudaMemcpy(&h, c->counters.p, sizeof(h), cudaMemcpyDeviceToHost), "dr_get_counters: copy");
    out->paths = h.paths;
    out->vertices = h.vertices;
    out->node_visits = h.node_visits;
    out->density_lookups = h.density_lookups;
    out->mie_evals = h.mie_evals;
    out->gave_up = h.gave_up;
    return DR_OK;
}

int dr_reset_counters(dr_ctx *c) {
    if (!c) return need(false, DR_ERR_INVALID, "dr_reset_counters: null context");
    DeviceGuard g(c->device);
    DR_CUDA(cudaMemsetAsync(c->counters.p, 0, sizeof(DevCounters), c->stream), "dr_reset_counters");
    DR_CUDA(cudaStreamSynchronize(c->stream), "dr_reset_counters: sync");
    return DR_OK;
}

// ---- probes -------------------------------------------------------------------
// Each probe copies its inputs into one scratch allocation, runs one kernel on
// the context stream and copies the results back.
namespace {
struct Scratch {
    std::vector<std::pair<size_t, size_t>> parts;  // offset, size
    size_t total = 0;
    size_t add(size_t bytes) {
        size_t off = (total + 255) & ~size_t(255);
        total = off + bytes;
        return off;
    }
};
}  // namespace

int dr_probe_leaf_sequence(dr_ctx *c, const float *ro, const float *rd, uint32_t n, uint32_t maxn, uint32_t *nodes,
                           float *tr0, float *tr1, uint32_t *counts) {
    if (!c || !ro || !rd || !nodes || !tr0 || !tr1 || !counts || n == 0 || maxn == 0)
        return need(false, DR_ERR_INVALID, "dr_probe_leaf_sequence: bad argument");
    if (!c->has_scene) return need(false, DR_ERR_STATE, "dr_probe_leaf_sequence: no scene");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    Scratch S;
    size_t o_ro = S.add(12ull * n), o_rd = S.add(12ull * n), o_nd = S.add(4ull * n * maxn), o_t0 = S.add(4ull * n * maxn),
           o_t1 = S.add(4ull * n * maxn), o_ct = S.add(4ull * n);
    DR_CUDA(c->scratch.reserve(S.total), "probe: alloc");
    unsigned char *b = c->scratch.p;
    DR_CUDA(cudaMemcpy(b + o_ro, ro, 12ull * n, cudaMemcpyHostToDevice), "probe: copy");
    DR_CUDA(cudaMemcpy(b + o_rd, rd, 12ull * n, cudaMemcpyHostToDevice), "probe: copy");
    DR_CUDA(launch_probe_leaf(c->scene, (float *)(b + o_ro), (float *)(b + o_rd), n, maxn, (uint32_t *)(b + o_nd),
                              (float *)(b + o_t0), (float *)(b + o_t1), (uint32_t *)(b + o_ct), c->stream),
            "probe: launch");
    DR_CUDA(cudaStreamSynchronize(c->stream), "probe: sync");
    DR_CUDA(cudaMemcpy(nodes, b + o_nd, 4ull * n * maxn, cudaMemcpyDeviceToHost), "probe: copy out");
    DR_CUDA(cudaMemcpy(tr0, b + o_t0, 4ull * n * maxn, cudaMemcpyDeviceToHost), "probe: copy out");
    DR_CUDA(cudaMemcpy(tr1, b + o_t1, 4ull * n * maxn, cudaMemcpyDeviceToHost), "probe: copy out");
    DR_CUDA(cudaMemcpy(counts, b + o_ct, 4ull * n, cudaMemcpyDeviceToHost), "probe: copy out");
    return DR_OK;
}

int dr_probe_density(dr_ctx *c, const uint32_t *nodes, const float *points, uint32_t n, float *out) {
    if (!c || !nodes || !points || !out || n == 0) return need(false, DR_ERR_INVALID, "dr_probe_density: bad argument");
    if (!c->has_scene) return need(false, DR_ERR_STATE, "dr_probe_density: no scene");
    for (uint32_t i = 0; i < n; ++i)
        if (nodes[i] >= c->leaf_flag.size() || !c->leaf_flag[nodes[i]])
            return need(false, DR_ERR_INVALID, "dr_probe_density: node is not a leaf of the scene");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    Scratch S;
    size_t o_n = S.add(4ull * n), o_p = S.add(12ull * n), o_o = S.add(4ull * n);
    DR_CUDA(c->scratch.reserve(S.total), "probe: alloc");
    unsigned char *b = c->scratch.p;
    DR_CUDA(cudaMemcpy(b + o_n, nodes, 4ull * n, cudaMemcpyHostToDevice), "probe: copy");
    DR_CUDA(cudaMemcpy(b + o_p, points, 12ull * n, cudaMemcpyHostToDevice), "probe: copy");
    DR_CUDA(launch_probe_density(c->scene, (uint32_t *)(b + o_n), (float *)(b + o_p), n, (float *)(b + o_o), c->stream),
            "probe: launch");
    DR_CUDA(cudaStreamSynchronize(c->stream), "probe: sync");
    DR_CUDA(cudaMemcpy(out, b + o_o, 4ull * n, cudaMemcpyDeviceToHost), "probe: copy out");
    return DR_OK;
}

int dr_probe_paths(dr_ctx *c, const uint32_t *px, const uint32_t *py, const uint64_t *sample, uint32_t n,
                   uint64_t seed, float *out_sun, float *out_sky) {
    if (!c || !px || !py || !sample || !out_sun || !out_sky || n == 0)
        return need(false, DR_ERR_INVALID, "dr_probe_paths: bad argument");
    if (!c->has_scene || !c->has_params) return need(false, DR_ERR_STATE, "dr_probe_paths: no scene or parameters");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    Scratch S;
    size_t o_x = S.add(4ull * n), o_y = S.add(4ull * n), o_s = S.add(8ull * n), o_a = S.add(16ull * n),
           o_b = S.add(16ull * n);
    DR_CUDA(c->scratch.reserve(S.total), "probe: alloc");
    unsigned char *b = c->scratch.p;
    DR_CUDA(cudaMemcpy(b + o_x, px, 4ull * n, cudaMemcpyHostToDevice), "probe: copy");
    DR_CUDA(cudaMemcpy(b + o_y, py, 4ull * n, cudaMemcpyHostToDevice), "probe: copy");
    DR_CUDA(cudaMemcpy(b + o_s, sample, 8ull * n, cudaMemcpyHostToDevice), "probe: copy");
    DR_CUDA(launch_probe_paths(c->scene, c->params, c->mie_pack.p, (uint32_t *)(b + o_x), (uint32_t *)(b + o_y),
                               (uint64_t *)(b + o_s), n, seed, (float4 *)(b + o_a), (float4 *)(b + o_b), c->counters.p,
                               c->stream),
            "probe: launch");
    DR_CUDA(cudaStreamSynchronize(c->stream), "probe: sync");
    DR_CUDA(cudaMemcpy(out_sun, b + o_a, 16ull * n, cudaMemcpyDeviceToHost), "probe: copy out");
    DR_CUDA(cudaMemcpy(out_sky, b + o_b, 16ull * n, cudaMemcpyDeviceToHost), "probe: copy out");
    return DR_OK;
}

int dr_probe_sampler(dr_ctx *c, uint32_t what, const float *in, uint32_t n, float *out) {
    if (!c || !in || !out || n == 0 || what > DR_PROBE_MIE_EXACT_DIR)
        return need(false, DR_ERR_INVALID, "dr_probe_sampler: bad argument");
    if (!c->has_params) return need(false, DR_ERR_STATE, "dr_probe_sampler: no parameters");
    if (what == DR_PROBE_MIE_EXACT_DIR && c->params.phase_mode != DR_PHASE_MIE_EXACT)
        return need(false, DR_ERR_STATE, "dr_probe_sampler: the exact sampler needs DR_PHASE_MIE_EXACT");
    const size_t in_n = what == DR_PROBE_MIE_SAMPLE ? 5ull * n
                        : what == DR_PROBE_SUN_SAMPLE ? 2ull * n
                        : what == DR_PROBE_SKY ? 3ull * n
                        : (size_t)n;
    const size_t out_n = what == DR_PROBE_MIE_THETA ? (size_t)n : what == DR_PROBE_MIE_EXACT_DIR ? 2ull * n : 3ull * n;
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    Scratch S;
    size_t o_i = S.add(4 * in_n), o_o = S.add(4 * out_n);
    DR_CUDA(c->scratch.reserve(S.total), "probe: alloc");
    unsigned char *b = c->scratch.p;
    DR_CUDA(cudaMemcpy(b + o_i, in, 4 * in_n, cudaMemcpyHostToDevice), "probe: copy");
    DR_CUDA(launch_probe_sampler(c->params, c->mie_pack.p, what, (float *)(b + o_i), n, (float *)(b + o_o), c->stream),
            "probe: launch");
    DR_CUDA(cudaStreamSynchronize(c->stream), "probe: sync");
    DR_CUDA(cudaMemcpy(out, b + o_o, 4 * out_n, cudaMemcpyDeviceToHost), "probe: copy out");
    return DR_OK;
}

int dr_probe_transmittance(dr_ctx *c, const float *ro, const float *rd, uint32_t n, uint64_t nsamp, uint64_t seed,
                           double *out) {
    if (!c || !ro || !rd || !out || n == 0 || nsamp == 0)
        return need(false, DR_ERR_INVALID, "dr_probe_transmittance: bad argument");
    if (!c->has_scene || !c->has_params) return need(false, DR_ERR_STATE, "dr_probe_transmittance: no scene");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    Scratch S;
    size_t o_ro = S.add(12ull * n), o_rd = S.add(12ull * n), o_e = S.add(8ull * n);
    DR_CUDA(c->scratch.reserve(S.total), "probe: alloc");
    unsigned char *b = c->scratch.p;
    DR_CUDA(cudaMemcpy(b + o_ro, ro, 12ull * n, cudaMemcpyHostToDevice), "probe: copy");
    DR_CUDA(cudaMemcpy(b + o_rd, rd, 12ull * n, cudaMemcpyHostToDevice), "probe: copy");
    DR_CUDA(cudaMemset(b + o_e, 0, 8ull * n), "probe: clear");
    DR_CUDA(launch_probe_transmittance(c->scene, c->params, (float *)(b + o_ro), (float *)(b + o_rd), n, nsamp, seed,
                                       (unsigned long long *)(b + o_e), c->stream),
            "probe: launch");
    DR_CUDA(cudaStreamSynchronize(c->stream), "probe: sync");
    std::vector<unsigned long long> esc(n);
    DR_CUDA(cudaMemcpy(esc.data(), b + o_e, 8ull * n, cudaMemcpyDeviceToHost), "probe: copy out");
    for (uint32_t i = 0; i < n; ++i) out[i] = (double)esc[i] / (double)nsamp;
    return DR_OK;
}

int dr_transmittance_noalloc(dr_ctx *c, const float *ro_dev, const float *rd_dev, uint32_t n_rays, uint64_t nsamp,
                             uint64_t seed, double *out_dev, void *stream) {
    if (!c || !ro_dev || !rd_dev || !out_dev || n_rays == 0 || nsamp == 0)
        return need(false, DR_ERR_INVALID, "dr_transmittance_noalloc: bad argument");
    if (n_rays > noalloc_max_rays())
        return need(false, DR_ERR_INVALID,
                    "dr_transmittance_noalloc: n_rays exceeds DR_NOALLOC_MAX_RAYS (65536); split the batch");
    if (!c->has_scene || !c->has_params)
        return need(false, DR_ERR_STATE, "dr_transmittance_noalloc: upload a scene and set parameters first");
    DeviceGuard g(c->device);
    unsigned long long *scratch = nullptr;
    DR_CUDA(noalloc_scratch(c->device, &scratch), "dr_transmittance_noalloc: scratch address");
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    DR_CUDA(launch_transmittance_noalloc(c->scene, c->params, scratch, ro_dev, rd_dev, n_rays, nsamp, seed, out_dev,
                                         st),
            "dr_transmittance_noalloc: launch");
    return DR_OK;
}

}  // extern "C"
