// Batched rendering: many scenes and views in one launch of a CUDA graph
// (declared in include/droplet_b200.h, dr_batch_*).
//
// The reference renders one tile of one view per RenderKernel::Render call
// (src/kernel.cpp:536-567).  A batch uploads every scene once, lays the paths
// of all views out as one index space (view-major; inside a view, pixels in
// the tuned order with consecutive samples), and captures
//   memset(outputs, queues) -> camera leaf lists of every view
//     -> persistent kernel over all views -> step counter += 1
// as a graph.  With a split (dr_batch_set_split), each view of at least
// min_paths paths gets a plain persistent kernel of its own instead (its
// parameters in kernel arguments rather than per-lane records in global
// memory); those kernels and the batched kernel over the remaining views are
// independent branches between the lists and the step counter, on up to
// kBranches capture streams, so a kernel's tail overlaps the next one's start.  Launch k of a batch renders samples [k spp, (k+1) spp) of every
// view, the same streams dr_render_tile draws with sample_base = k spp.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/droplet_b200.h"
#include "dr_host.h"
#include "dr_kernels.h"

using namespace dr;

namespace {
constexpr uint32_t kBranches = 4;         // capture streams of a split graph (kernels side by side)
constexpr uint64_t kSplitAutoPerLane = 8;  // DR_BATCH_SPLIT_AUTO: paths per lane of a full grid
}  // namespace

struct dr_batch {
    dr_ctx *ctx = nullptr;
    cudaStream_t stream = nullptr;  // capture stream
    std::vector<std::unique_ptr<SceneBufs>> scene_bufs;
    std::vector<std::unique_ptr<DevBuf<float>>> depth_bufs;  // per-view depth textures and environment maps
    DevBuf<DevScene> scenes;
    DevBuf<BatchView> views;
    DevBuf<uint64_t> begins;
    DevBuf<float4> out;
    DevBuf<unsigned char> mie_pack;
    DevBuf<WorkQueue> work;  // [0]: the batched kernel; [1 + v]: view v's own kernel
    DevBuf<unsigned long long> step;
    // split graphs: the views left to the batched kernel, their first path indices
    DevBuf<BatchView> rest_views;
    DevBuf<uint64_t> rest_begins;
    std::vector<DevScene> host_scenes;
    uint64_t split = DR_BATCH_SPLIT_AUTO;  // dr_batch_set_split
    uint32_t own_kernels = 0;              // views with a kernel of their own in the current graph
    cudaStream_t branch[kBranches] = {};
    cudaEvent_t fork = nullptr, join[kBranches] = {};
    // camera leaf lists (one header per pixel of every view, one entry pool)
    DevBuf<uint4> cam_head, cam_pool;
    DevBuf<unsigned int> cam_used;
    DevBuf<uint32_t> pix_begins;
    uint32_t n_pix = 0;
    std::vector<BatchView> host_views;
    std::vector<size_t> out_off;  // float4 offset of view v's sun tile; its sky tile follows
    size_t out_n = 0;             // float4 count of all outputs
    DevParams p0{};
    Tuning tuning{0u, 128u, 0u, 8u, 0u, 0u, 0u, 0u};
    uint64_t n_paths = 0, launches = 0;
    bool any_sdf = false;  // a scene with surface (SDF) leaves
    uint32_t stack_levels = 0;  // deepest traversal stack of the scenes (0: some scene's depth is unknown)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

void drop_graph(dr_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// Lays the view's paths out for the current tile order and (re)captures the graph.
int build_graph(dr_batch *b) {
    drop_graph(b);
    bool ext = b->any_sdf;  // surface leaves, or a view with the HG phase or a non-Hosek environment
    for (const BatchView &v : b->host_views) ext = ext || v.P.phase_mode == kPhaseHG || v.P.env_mode != kEnvHosek;
    // camera leaf lists for the stack traversals (the cell walk counts grid
    // cells and keeps its own traversal); without the storage the views traverse
    const bool lists = b->tuning.traversal != 1u && b->cam_head.p && b->cam_pool.p && b->cam_used.p;
    uint64_t begin = 0;
    uint32_t pix = 0;
    std::vector<uint64_t> begins(b->host_views.size());
    std::vector<uint32_t> pix_begins(b->host_views.size());
    for (size_t v = 0; v < b->host_views.size(); ++v) {
        BatchView &V = b->host_views[v];
        TileArgs A;
        int rc = make_tile_args(V.A.x0, V.A.y0, V.A.tw, V.A.th, V.A.spp, V.A.seed, 0, b->tuning.tile, A);
        if (rc != DR_OK) return rc;
        // sky terms through the warps' queues (not with a whole-path finiteness check)
        A.defer_sky = (!ext && !V.P.finite_paths) ? 1u : 0u;
        pix_begins[v] = pix;
        if (lists) {
            A.cam_head = b->cam_head.p + 2 * (size_t)pix;
            A.cam_pool = b->cam_pool.p;
        }
        pix += A.cols * A.rows;
        V.A = A;
        V.begin = begin;
        begins[v] = begin;
        begin += A.n_paths;
    }
    b->n_paths = begin;
    DR_CUDA(cudaMemcpy(b->views.p, b->host_views.data(), sizeof(BatchView) * b->host_views.size(),
                       cudaMemcpyHostToDevice),
            "dr_batch: copy views");
    DR_CUDA(cudaMemcpy(b->begins.p, begins.data(), sizeof(uint64_t) * begins.size(), cudaMemcpyHostToDevice),
            "dr_batch: copy views");
    DR_CUDA(cudaMemcpy(b->pix_begins.p, pix_begins.data(), sizeof(uint32_t) * pix_begins.size(),
                       cudaMemcpyHostToDevice),
            "dr_batch: copy views");
    BatchLists bl;
    if (lists) {
        bl.lists.head = b->cam_head.p;
        bl.lists.pool = b->cam_pool.p;
        bl.lists.cap = (uint32_t)b->cam_pool.n;
        bl.lists.used = b->cam_used.p;
        bl.pix_begins = b->pix_begins.p;
        bl.n_pix = pix;
    }
    BatchArgs B;
    B.views = b->views.p;
    B.scenes = b->scenes.p;
    B.begins = b->begins.p;
    B.n_views = (uint32_t)b->host_views.size();
    B.n_paths = b->n_paths;
    B.step = b->step.p;
    // which views get a kernel of their own
    uint64_t min_own = b->split;
    if (min_own == DR_BATCH_SPLIT_AUTO) {
        int sms = 0;
        DR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->ctx->device), "dr_batch: SM count");
        const uint64_t bps = b->tuning.blocks_per_sm ? b->tuning.blocks_per_sm : 8u;
        min_own = kSplitAutoPerLane * (uint64_t)sms * bps * 128u;
    }
    std::vector<uint32_t> own;
    std::vector<BatchView> rest;
    std::vector<uint64_t> rest_begins;
    uint64_t rest_paths = 0;
    for (uint32_t v = 0; v < (uint32_t)b->host_views.size(); ++v) {
        const BatchView &V = b->host_views[v];
        if (min_own && V.A.n_paths >= min_own) {
            own.push_back(v);
        } else {
            rest.push_back(V);
            rest.back().begin = rest_paths;
            rest_begins.push_back(rest_paths);
            rest_paths += V.A.n_paths;
        }
    }
    BatchArgs R = B;  // the batched kernel's views
    if (!own.empty()) {
        if (!rest.empty()) {
            DR_CUDA(cudaMemcpy(b->rest_views.p, rest.data(), sizeof(BatchView) * rest.size(), cudaMemcpyHostToDevice),
                    "dr_batch: copy views");
            DR_CUDA(cudaMemcpy(b->rest_begins.p, rest_begins.data(), sizeof(uint64_t) * rest.size(),
                               cudaMemcpyHostToDevice),
                    "dr_batch: copy views");
        }
        R.views = b->rest_views.p;
        R.begins = b->rest_begins.p;
        R.n_views = (uint32_t)rest.size();
        R.n_paths = rest_paths;
        for (uint32_t k = 0; k < kBranches && k < own.size(); ++k) {
            if (!b->branch[k])
                DR_CUDA(cudaStreamCreateWithFlags(&b->branch[k], cudaStreamNonBlocking), "dr_batch: branch stream");
            if (!b->join[k])
                DR_CUDA(cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming), "dr_batch: branch event");
        }
        if (!b->fork) DR_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "dr_batch: branch event");
    }
    const uint32_t nbr = (uint32_t)std::min<size_t>(kBranches, own.size());
    DR_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "dr_batch: begin capture");
    cudaError_t e = cudaMemsetAsync(b->out.p, 0, sizeof(float4) * b->out_n, b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->work.p, 0, sizeof(WorkQueue) * b->work.n, b->stream);
    if (e == cudaSuccess) e = launch_batch_lists(B, bl, b->stream);
    if (e == cudaSuccess && nbr) e = cudaEventRecord(b->fork, b->stream);
    for (uint32_t k = 0; k < nbr && e == cudaSuccess; ++k) e = cudaStreamWaitEvent(b->branch[k], b->fork, 0);
    for (size_t k = 0; k < own.size() && e == cudaSuccess; ++k) {
        const BatchView &V = b->host_views[own[k]];
        e = launch_batch_view(b->host_scenes[V.scene], V.P, V.A, b->mie_pack.p, V.sun, V.sky, b->ctx->counters.p,
                              b->work.p + 1 + own[k], b->step.p, b->tuning, b->ctx->device, b->branch[k % nbr]);
    }
    if (e == cudaSuccess)
        e = launch_batch_kernel(R, b->p0, b->mie_pack.p, b->ctx->counters.p, b->work.p, b->tuning, ext,
                                b->stack_levels, b->ctx->device, b->stream);
    // every branch joins the capture stream (also after an error, so that the capture can end)
    for (uint32_t k = 0; k < nbr; ++k) {
        const cudaError_t j = cudaEventRecord(b->join[k], b->branch[k]);
        const cudaError_t w = j == cudaSuccess ? cudaStreamWaitEvent(b->stream, b->join[k], 0) : j;
        if (e == cudaSuccess) e = w;
    }
    if (e == cudaSuccess) e = launch_batch_step(b->step.p, b->stream);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_fail(e, "dr_batch: capture");
    }
    if (e2 != cudaSuccess) return cuda_fail(e2, "dr_batch: end capture");
    b->graph = g;
    b->own_kernels = (uint32_t)own.size();
    DR_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0), "dr_batch: instantiate graph");
    return DR_OK;
}

void release(dr_batch *b) {
    drop_graph(b);
    for (auto &s : b->scene_bufs) s->release();
    for (auto &d : b->depth_bufs) d->release();
    b->scenes.release();
    b->views.release();
    b->begins.release();
    b->out.release();
    b->mie_pack.release();
    b->work.release();
    b->step.release();
    b->cam_head.release();
    b->cam_pool.release();
    b->cam_used.release();
    b->pix_begins.release();
    b->rest_views.release();
    b->rest_begins.release();
    for (uint32_t k = 0; k < kBranches; ++k) {
        if (b->branch[k]) cudaStreamDestroy(b->branch[k]);
        if (b->join[k]) cudaEventDestroy(b->join[k]);
        b->branch[k] = nullptr;
        b->join[k] = nullptr;
    }
    if (b->fork) cudaEventDestroy(b->fork);
    b->fork = nullptr;
    if (b->stream) cudaStreamDestroy(b->stream);
    b->stream = nullptr;
}

}  // namespace

extern "C" {

int dr_batch_create(dr_ctx *c, const dr_scene_desc *scenes, uint32_t n_scenes, const dr_batch_view *views,
                    uint32_t n_views, dr_batch **out) {
    if (out) *out = nullptr;
    if (!c || !scenes || !views || !out || n_scenes == 0 || n_views == 0)
        return need(false, DR_ERR_INVALID, "dr_batch_create: null argument or empty batch");
    // Validate and convert everything on the host first.
    std::vector<HostScene> hs(n_scenes);
    for (uint32_t i = 0; i < n_scenes; ++i) {
        int rc = prepare_scene(&scenes[i], hs[i]);
        if (rc != DR_OK) return rc;
    }
    std::vector<BatchView> hv(n_views);
    std::vector<unsigned char> pack0;
    for (uint32_t v = 0; v < n_views; ++v) {
        const dr_batch_view &bv = views[v];
        if (bv.scene >= n_scenes) return need(false, DR_ERR_INVALID, "dr_batch_create: view scene index out of range");
        if (!bv.params) return need(false, DR_ERR_INVALID, "dr_batch_create: view without parameters");
        std::vector<unsigned char> pack;
        int rc = prepare_params(bv.params, hv[v].P, pack);
        if (rc != DR_OK) return rc;
        hv[v].P.step_budget = c->step_budget;
        if (v == 0) pack0 = pack;
        else if (pack != pack0)
            return need(false, DR_ERR_INVALID, "dr_batch_create: every view must use the same phase tables and mode");
        TileArgs A;
        rc = make_tile_args(bv.x0, bv.y0, bv.tw, bv.th, bv.spp, bv.seed, 0, 0, A);
        if (rc != DR_OK) return rc;
        hv[v].A = A;
        hv[v].scene = bv.scene;
    }
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    std::unique_ptr<dr_batch> b(new dr_batch());
    b->ctx = c;
    b->tuning = c->tuning;
    b->tuning.kernel = DR_KERNEL_PERSISTENT;
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "dr_batch_create: stream");
    int rc = DR_OK;
    auto fail = [&](int code) {
        release(b.get());
        return code;
    };
    std::vector<DevScene> ds(n_scenes);
    bool depth_known = true;
    for (uint32_t i = 0; i < n_scenes; ++i) {
        b->scene_bufs.emplace_back(new SceneBufs());
        rc = upload_scene(hs[i], *b->scene_bufs.back(), c->use_grid, b->stream, ds[i]);
        b->any_sdf = b->any_sdf || ds[i].sdf_bricks != nullptr;
        if (rc != DR_OK) return fail(rc);
        depth_known = depth_known && ds[i].stack_levels > 0;
        b->stack_levels = std::max(b->stack_levels, ds[i].stack_levels);
    }
    if (!depth_known) b->stack_levels = 0;
    size_t total = 0;
    b->out_off.resize(n_views);
    for (uint32_t v = 0; v < n_views; ++v) {
        b->out_off[v] = total;
        total += 2 * (size_t)hv[v].A.tw * hv[v].A.th;
    }
    b->out_n = total;
#define BATCH_CUDA(call, what)                        \
    do {                                              \
        cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) return fail(cuda_fail(e_, what)); \
    } while (0)
    BATCH_CUDA(b->out.reserve(total), "dr_batch_create: alloc outputs");
    for (uint32_t v = 0; v < n_views; ++v) {
        hv[v].sun = b->out.p + b->out_off[v];
        hv[v].sky = hv[v].sun + (size_t)hv[v].A.tw * hv[v].A.th;
        const dr_render_params *p = views[v].params;
        if (p->depth) {
            b->depth_bufs.emplace_back(new DevBuf<float>());
            DevBuf<float> &d = *b->depth_bufs.back();
            BATCH_CUDA(d.reserve((size_t)p->w * p->h), "dr_batch_create: alloc depth");
            BATCH_CUDA(cudaMemcpy(d.p, p->depth, sizeof(float) * p->w * p->h, cudaMemcpyHostToDevice),
                       "dr_batch_create: copy depth");
            hv[v].P.depth = d.p;
        }
        if (p->env_mode == DR_ENV_MAP) {
            const size_t n = (size_t)p->env_w * p->env_h * 4;
            b->depth_bufs.emplace_back(new DevBuf<float>());
            DevBuf<float> &d = *b->depth_bufs.back();
            BATCH_CUDA(d.reserve(n), "dr_batch_create: alloc environment map");
            BATCH_CUDA(cudaMemcpy(d.p, p->env_map, sizeof(float) * n, cudaMemcpyHostToDevice),
                       "dr_batch_create: copy environment map");
            hv[v].P.env_map = d.p;
        }
    }
    BATCH_CUDA(b->scenes.reserve(n_scenes), "dr_batch_create: alloc scenes");
    BATCH_CUDA(cudaMemcpy(b->scenes.p, ds.data(), sizeof(DevScene) * n_scenes, cudaMemcpyHostToDevice),
               "dr_batch_create: copy scenes");
    BATCH_CUDA(b->views.reserve(n_views), "dr_batch_create: alloc views");
    BATCH_CUDA(b->begins.reserve(n_views), "dr_batch_create: alloc views");
    BATCH_CUDA(b->pix_begins.reserve(n_views), "dr_batch_create: alloc views");
    {
        // camera leaf lists: two header words per pixel, a pool of up to 4 leaves per
        // pixel (at most 2^26 entries); without them the views traverse
        uint64_t n_pix = 0;
        for (uint32_t v = 0; v < n_views; ++v) n_pix += (uint64_t)hv[v].A.cols * hv[v].A.rows;
        const uint64_t n_pool = std::min<uint64_t>(4 * n_pix, 1ull << 26);
        if (n_pix == 0 || n_pix >= (1ull << 31) || b->cam_head.reserve(2 * n_pix) != cudaSuccess ||
            b->cam_pool.reserve(n_pool) != cudaSuccess || b->cam_used.reserve(1) != cudaSuccess) {
            b->cam_head.release();
            b->cam_pool.release();
            b->cam_used.release();
            cudaGetLastError();  // not an error of the batch
        }
    }
    BATCH_CUDA(b->mie_pack.reserve(pack0.size()), "dr_batch_create: alloc tables");
    BATCH_CUDA(cudaMemcpy(b->mie_pack.p, pack0.data(), pack0.size(), cudaMemcpyHostToDevice),
               "dr_batch_create: copy tables");
    BATCH_CUDA(b->work.reserve(1 + (size_t)n_views), "dr_batch_create: alloc queue");
    BATCH_CUDA(b->rest_views.reserve(n_views), "dr_batch_create: alloc views");
    BATCH_CUDA(b->rest_begins.reserve(n_views), "dr_batch_create: alloc views");
    BATCH_CUDA(b->step.reserve(1), "dr_batch_create: alloc step");
    BATCH_CUDA(cudaMemset(b->step.p, 0, sizeof(unsigned long long)), "dr_batch_create: clear step");
#undef BATCH_CUDA
    b->p0 = hv[0].P;
    b->host_views = std::move(hv);
    b->host_scenes = ds;
    rc = build_graph(b.get());
    if (rc != DR_OK) return fail(rc);
    *out = b.release();
    return DR_OK;
}

int dr_batch_destroy(dr_batch *b) {
    if (!b) return DR_OK;
    {
        DeviceGuard g(b->ctx->device);
        // launches may run on any caller stream: wait for the device before
        // the graph and its buffers go
        cudaDeviceSynchronize();
        release(b);
    }
    delete b;
    return DR_OK;
}

int dr_batch_set_tuning(dr_batch *b, const dr_tuning *t) {
    if (!b || !valid_tuning(t)) return need(false, DR_ERR_INVALID, "dr_batch_set_tuning: bad argument");
    if (t->kernel != DR_KERNEL_PERSISTENT)
        return need(false, DR_ERR_INVALID, "dr_batch_set_tuning: a batch runs the persistent kernel");
    DeviceGuard g(b->ctx->device);
    // a launch on any caller stream may still read the views: wait for the device
    DR_CUDA(cudaDeviceSynchronize(), "dr_batch_set_tuning: sync");
    b->tuning.kernel = DR_KERNEL_PERSISTENT;
    b->tuning.blocks_per_sm = t->blocks_per_sm;
    b->tuning.event_batch = t->event_batch;
    b->tuning.traversal = t->traversal;
    b->tuning.tile = t->tile;
    b->tuning.visits = t->visits;
    b->tuning.steps = t->steps;
    return build_graph(b);
}

int dr_batch_get_tuning(dr_batch *b, dr_tuning *t) {
    if (!b || !t) return need(false, DR_ERR_INVALID, "dr_batch_get_tuning: null argument");
    t->kernel = DR_KERNEL_PERSISTENT;
    t->blocks_per_sm = b->tuning.blocks_per_sm;
    t->event_batch = b->tuning.event_batch;
    t->traversal = b->tuning.traversal;
    t->tile = b->tuning.tile;
    t->visits = b->tuning.visits;
    t->steps = b->tuning.steps;
    return DR_OK;
}

int dr_batch_launch(dr_batch *b, void *stream) {
    if (!b || !b->exec) return need(false, DR_ERR_INVALID, "dr_batch_launch: no batch");
    DeviceGuard g(b->ctx->device);
    DR_CUDA(cudaGraphLaunch(b->exec, stream ? (cudaStream_t)stream : b->ctx->stream), "dr_batch_launch");
    ++b->launches;
    return DR_OK;
}

int dr_batch_output(dr_batch *b, uint32_t view, float **sun_dev, float **sky_dev) {
    if (!b || view >= b->host_views.size() || !sun_dev || !sky_dev)
        return need(false, DR_ERR_INVALID, "dr_batch_output: bad argument");
    *sun_dev = (float *)b->host_views[view].sun;
    *sky_dev = (float *)b->host_views[view].sky;
    return DR_OK;
}

int dr_batch_read(dr_batch *b, uint32_t view, float *sun_out, float *sky_out) {
    if (!b || view >= b->host_views.size() || !sun_out || !sky_out)
        return need(false, DR_ERR_INVALID, "dr_batch_read: bad argument");
    DeviceGuard g(b->ctx->device);
    const BatchView &V = b->host_views[view];
    const size_t n = (size_t)V.A.tw * V.A.th;
    DR_CUDA(cudaDeviceSynchronize(), "dr_batch_read: sync");
    DR_CUDA(cudaMemcpy(sun_out, V.sun, n * sizeof(float4), cudaMemcpyDeviceToHost), "dr_batch_read: copy");
    DR_CUDA(cudaMemcpy(sky_out, V.sky, n * sizeof(float4), cudaMemcpyDeviceToHost), "dr_batch_read: copy");
    return DR_OK;
}

int dr_batch_set_split(dr_batch *b, uint64_t min_paths) {
    if (!b) return need(false, DR_ERR_INVALID, "dr_batch_set_split: null batch");
    DeviceGuard g(b->ctx->device);
    DR_CUDA(cudaDeviceSynchronize(), "dr_batch_set_split: sync");
    b->split = min_paths;
    return build_graph(b);
}

int dr_batch_get_split(dr_batch *b, uint64_t *min_paths, uint32_t *own_kernels) {
    if (!b) return need(false, DR_ERR_INVALID, "dr_batch_get_split: null batch");
    if (min_paths) *min_paths = b->split;
    if (own_kernels) *own_kernels = b->own_kernels;
    return DR_OK;
}

int dr_batch_info(dr_batch *b, uint64_t *n_paths, uint64_t *launches) {
    if (!b) return need(false, DR_ERR_INVALID, "dr_batch_info: null batch");
    if (n_paths) *n_paths = b->n_paths;
    if (launches) *launches = b->launches;
    return DR_OK;
}

}  // extern "C"
