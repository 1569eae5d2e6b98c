// C ABI of droplet_b200 (declared in include/droplet_b200.h).
#include <algorithm>
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
#include "dr_host.h"
#include "dr_internal.h"
#include "dr_kernels.h"

namespace dr {

int build_octree(const int32_t *org, const float *vals, uint32_t n_blocks, float s, uint32_t maxdepth, int nthreads,
                 dr_octree *out);
int sky_cook(const double *const rgb[3], const double *const rad[3], double turbidity, double albedo,
             double elevation, double configs[3][9], double radiances[3]);

}  // namespace dr

using namespace dr;



extern "C" {

int dr_version(void) { return DR_VERSION; }

const char *dr_last_error(void) { return last_error(); }

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
        c->bufs.release();
        c->mie_pack.release();
        c->depth.release();
        c->counters.release();
        c->call_counters.release();
        c->tile_sun.release();
        c->tile_sky.release();
        c->scratch.release();
        c->work.release();
        c->leaf_nodes.release();
        c->grad_copies.release();
        c->albedo_slots.release();
        c->path_rec.release();
        c->occ_nodes.release();
        c->env.release();
        c->occ_tris.release();
        c->band_work.release();
        c->cam_head.release();
        c->cam_pool.release();
        c->band_cam_head.release();
        c->band_cam_pool.release();
        c->cam_used.release();
        for (int k = 0; k < 2; ++k)
            if (c->band_stream[k]) cudaStreamSynchronize(c->band_stream[k]), cudaStreamDestroy(c->band_stream[k]);
        if (c->copy_stream) cudaStreamSynchronize(c->copy_stream), cudaStreamDestroy(c->copy_stream);
        if (c->ev_clear) cudaEventDestroy(c->ev_clear);
        for (int k = 0; k < dr_ctx::kBands; ++k) {
            if (c->band_done[k]) cudaEventDestroy(c->band_done[k]);
            if (c->copy_done[k]) cudaEventDestroy(c->copy_done[k]);
        }
        if (c->pinned) cudaFreeHost(c->pinned);
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
    if (!c) return need(false, DR_ERR_INVALID, "dr_upload_scene: null argument");
    HostScene h;
    int rc = prepare_scene(s, h);
    if (rc != DR_OK) return rc;
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    rc = upload_scene(h, c->bufs, c->use_grid, c->stream, c->scene);
    if (rc != DR_OK) return rc;
    if (c->occ_n_nodes) {
        c->scene.occ_nodes = c->occ_nodes.p;
        c->scene.occ_tris = c->occ_tris.p;
        c->scene.occ_n_nodes = c->occ_n_nodes;
    }
    std::vector<uint32_t> ln;
    for (uint32_t i = 0; i < h.n_nodes; ++i)  // leaves whose majorant comes from their fog brick
        if ((h.leaf_flag[i] & 2u) && !(h.leaf_flag[i] & 4u)) ln.push_back(i);
    DR_CUDA(c->leaf_nodes.reserve(ln.size()), "dr_upload_scene: alloc leaf list");
    if (!ln.empty())
        DR_CUDA(cudaMemcpy(c->leaf_nodes.p, ln.data(), ln.size() * 4, cudaMemcpyHostToDevice),
                "dr_upload_scene: copy leaf list");
    c->n_leaf_nodes = (uint32_t)ln.size();
    c->leaf_flag = std::move(h.leaf_flag);
    c->has_scene = true;
    return DR_OK;
}

int dr_set_occluders(dr_ctx *c, const dr_surface *surfaces, uint32_t n_surfaces, uint32_t mode) {
    if (!c) return need(false, DR_ERR_INVALID, "dr_set_occluders: null argument");
    OccBvh b;
    int rc = build_occluder_bvh(surfaces, n_surfaces, mode, b);
    if (rc != DR_OK) return rc;
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    DR_CUDA(cudaStreamSynchronize(c->stream), "dr_set_occluders: sync");
    const uint32_t nn = (uint32_t)(b.nodes.size() / 16);
    if (nn) {
        DR_CUDA(c->occ_nodes.reserve((size_t)nn * 4), "dr_set_occluders: alloc nodes");
        DR_CUDA(c->occ_tris.reserve(b.tris.size() / 4), "dr_set_occluders: alloc triangles");
        DR_CUDA(cudaMemcpy(c->occ_nodes.p, b.nodes.data(), b.nodes.size() * sizeof(float), cudaMemcpyHostToDevice),
                "dr_set_occluders: copy nodes");
        DR_CUDA(cudaMemcpy(c->occ_tris.p, b.tris.data(), b.tris.size() * sizeof(float), cudaMemcpyHostToDevice),
                "dr_set_occluders: copy triangles");
    }
    c->occ_n_nodes = nn;
    c->scene.occ_nodes = nn ? c->occ_nodes.p : nullptr;
    c->scene.occ_tris = nn ? c->occ_tris.p : nullptr;
    c->scene.occ_n_nodes = nn;
    return DR_OK;
}

int dr_set_params(dr_ctx *c, const dr_render_params *p) {
    if (!c || !p) return need(false, DR_ERR_INVALID, "dr_set_params: null argument");
    DevParams d;
    std::vector<unsigned char> pack;
    int rc = prepare_params(p, d, pack);
    if (rc != DR_OK) return rc;
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
    }
    if (p->env_mode == DR_ENV_MAP) {
        const size_t n = (size_t)p->env_w * p->env_h * 4;
        DR_CUDA(c->env.reserve(n), "dr_set_params: alloc environment map");
        DR_CUDA(cudaMemcpy(c->env.p, p->env_map, sizeof(float) * n, cudaMemcpyHostToDevice),
                "dr_set_params: copy environment map");
        d.env_map = c->env.p;
    }
    d.step_budget = c->step_budget;
    c->params = d;
    c->has_params = true;
    // camera leaf list storage for tiles up to the whole frame, so that renders
    // allocate nothing (without it their camera segments traverse)
    const size_t frame = (size_t)p->w * p->h;
    if (c->cam_used.reserve(3) != cudaSuccess || c->cam_head.reserve(2 * frame) != cudaSuccess ||
        c->band_cam_head.reserve(2 * frame) != cudaSuccess || c->cam_pool.reserve(c->cam_cap) != cudaSuccess ||
        c->band_cam_pool.reserve(2 * (size_t)c->cam_cap) != cudaSuccess) {
        c->cam_head.release();
        c->band_cam_head.release();
        cudaGetLastError();  // not an error of the parameters
    }
    return DR_OK;
}

int dr_set_camera_lists(dr_ctx *c, uint32_t pool_entries) {
    if (!c) return need(false, DR_ERR_INVALID, "dr_set_camera_lists: null context");
    if (pool_entries != DR_NONE && pool_entries > (1u << 28))
        return need(false, DR_ERR_INVALID, "dr_set_camera_lists: at most 2^28 entries per pool");
    std::lock_guard<std::mutex> lk(c->mu);
    c->cam_cap = pool_entries == DR_NONE ? 0u : pool_entries ? pool_entries : dr_ctx::kCamPool;
    return DR_OK;
}

int dr_set_step_budget(dr_ctx *c, uint32_t steps) {
    if (!c) return need(false, DR_ERR_INVALID, "dr_set_step_budget: null context");
    std::lock_guard<std::mutex> lk(c->mu);
    c->step_budget = steps ? steps : kStepBudget;
    c->params.step_budget = c->step_budget;
    return DR_OK;
}

// A blocking call's give-ups: its own counters are added to the context's, and
// a call whose paths gave up reports DR_ERR_GAVE_UP (its outputs are written,
// but those paths are cut short).
static int finish_call_counters(dr_ctx *c, const char *what) {
    DR_CUDA(launch_add_counters(c->counters.p, c->call_counters.p, c->stream), what);
    DevCounters h{};
    DR_CUDA(cudaMemcpyAsync(&h, c->call_counters.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream), what);
    DR_CUDA(cudaStreamSynchronize(c->stream), what);
    if (h.gave_up == 0) return DR_OK;
    c->gave_up_reported += h.gave_up;
    char msg[160];
    std::snprintf(msg, sizeof(msg), "%s: %llu path segments or blocks gave up (iteration budget): the result is incomplete",
                  what, (unsigned long long)h.gave_up);
    set_error(DR_ERR_GAVE_UP, msg);
    return DR_ERR_GAVE_UP;
}

int dr_check_complete(dr_ctx *c, void *stream) {
    if (!c) return need(false, DR_ERR_INVALID, "dr_check_complete: null context");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    DR_CUDA(cudaStreamSynchronize(stream ? (cudaStream_t)stream : c->stream), "dr_check_complete: sync");
    DR_CUDA(cudaStreamSynchronize(c->stream), "dr_check_complete: sync");
    DevCounters h{};
    DR_CUDA(cudaMemcpy(&h, c->counters.p, sizeof(h), cudaMemcpyDeviceToHost), "dr_check_complete: copy");
    if (h.gave_up <= c->gave_up_reported) return DR_OK;
    const unsigned long long n = h.gave_up - c->gave_up_reported;
    c->gave_up_reported = h.gave_up;
    char msg[160];
    std::snprintf(msg, sizeof(msg),
                  "dr_check_complete: %llu path segments or blocks gave up (iteration budget) since the last check", n);
    set_error(DR_ERR_GAVE_UP, msg);
    return DR_ERR_GAVE_UP;
}

static int tile_args(const dr_ctx *c, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed,
                     uint64_t base, uint32_t tile, TileArgs &A) {
    if (!c->has_scene || !c->has_params)
        return need(false, DR_ERR_STATE, "render: upload a scene and set parameters first");
    return make_tile_args(x0, y0, tw, th, spp, seed, base, tile, A);
}

// Camera leaf list storage of a persistent launch: slot 0 for the asynchronous
// render, 1 + (band & 1) for the blocking render's band streams (head_off: the
// band's first pixel among the tile's headers).  A failed allocation leaves
// the launch without lists (its camera segments traverse).
static CamLists cam_lists(dr_ctx *c, uint32_t slot, size_t head_pixels, size_t head_off) {
    CamLists L;
    if (c->cam_cap == 0) return L;
    DevBuf<uint4> &head = slot ? c->band_cam_head : c->cam_head;
    DevBuf<uint4> &pool = slot ? c->band_cam_pool : c->cam_pool;
    const size_t pool_n = (slot ? 2u : 1u) * (size_t)c->cam_cap;
    if (c->cam_used.reserve(3) != cudaSuccess || head.reserve(2 * head_pixels) != cudaSuccess ||
        pool.reserve(pool_n) != cudaSuccess) {
        cudaGetLastError();  // not an error of the render
        return L;
    }
    L.head = head.p + 2 * head_off;
    L.pool = pool.p + (slot == 2 ? (size_t)c->cam_cap : 0u);
    L.cap = c->cam_cap;
    L.used = c->cam_used.p + slot;
    return L;
}

int dr_render_tile_async(dr_ctx *c, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed,
                         uint64_t sample_base, float *sun_dev, float *sky_dev, void *stream) {
    if (!c || !sun_dev || !sky_dev) return need(false, DR_ERR_INVALID, "dr_render_tile_async: null argument");
    TileArgs A;
    const uint32_t tile = c->tuning.kernel == DR_KERNEL_PER_PATH ? 0u : c->tuning.tile;
    int rc = tile_args(c, x0, y0, tw, th, spp, seed, sample_base, tile, A);
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
        const CamLists lists = cam_lists(c, 0, (size_t)A.cols * A.rows, 0);
        DR_CUDA(launch_render_persistent(c->scene, c->params, A, c->mie_pack.p, (float4 *)sun_dev, (float4 *)sky_dev,
                                         c->counters.p, c->work.p, c->tuning, c->device, st, lists),
                "render: launch");
    }
    return DR_OK;
}

int dr_shadow_tile_async(dr_ctx *c, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed,
                         uint64_t sample_base, float *out_dev, void *stream) {
    if (!c || !out_dev) return need(false, DR_ERR_INVALID, "dr_shadow_tile_async: null argument");
    TileArgs A;
    int rc = tile_args(c, x0, y0, tw, th, spp, seed, sample_base, 0u, A);
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
    DR_CUDA(c->call_counters.reserve(1), "shadow: alloc counters");
    TileArgs A;
    int rc = tile_args(c, x0, y0, tw, th, spp, seed, sample_base, 0u, A);
    if (rc != DR_OK) return rc;
    DR_CUDA(cudaMemsetAsync(c->call_counters.p, 0, sizeof(DevCounters), c->stream), "shadow: clear");
    DR_CUDA(cudaMemsetAsync(c->tile_sun.p, 0, n * sizeof(float4), c->stream), "shadow: clear");
    DR_CUDA(launch_shadow_tile(c->scene, c->params, A, c->tile_sun.p, c->call_counters.p, c->stream), "shadow: launch");
    DR_CUDA(cudaMemcpyAsync(out, c->tile_sun.p, n * sizeof(float4), cudaMemcpyDeviceToHost, c->stream),
            "shadow: copy out");
    return finish_call_counters(c, "dr_shadow_tile");
}

int dr_set_tuning(dr_ctx *c, const dr_tuning *t) {
    if (!c || !t) return need(false, DR_ERR_INVALID, "dr_set_tuning: null argument");
    if (!valid_tuning(t))
        return need(false, DR_ERR_INVALID,
                    "dr_set_tuning: kernel 0/1, event_batch <= 32, blocks_per_sm <= 64, traversal 0/1/2, tile <= 64, "
                    "visits <= 255, steps <= 255");
    c->tuning.kernel = t->kernel;
    c->tuning.block = kPersistentBlock;
    c->tuning.blocks_per_sm = t->blocks_per_sm;
    c->tuning.event_batch = t->event_batch;
    c->tuning.traversal = t->traversal;
    c->tuning.tile = t->tile;
    c->tuning.visits = t->visits;
    c->tuning.steps = t->steps;
    return DR_OK;
}

int dr_get_tuning(dr_ctx *c, dr_tuning *t) {
    if (!c || !t) return need(false, DR_ERR_INVALID, "dr_get_tuning: null argument");
    t->kernel = c->tuning.kernel;
    t->blocks_per_sm = c->tuning.blocks_per_sm;
    t->event_batch = c->tuning.event_batch;
    t->traversal = c->tuning.traversal;
    t->tile = c->tuning.tile;
    t->visits = c->tuning.visits;
    t->steps = c->tuning.steps;
    return DR_OK;
}

// Pipeline objects of dr_render_tile, created on first use.
static int ensure_pipeline(dr_ctx *c, size_t n) {
    if (!c->copy_stream) {
        DR_CUDA(cudaStreamCreateWithFlags(&c->band_stream[0], cudaStreamNonBlocking), "render: streams");
        DR_CUDA(cudaStreamCreateWithFlags(&c->band_stream[1], cudaStreamNonBlocking), "render: streams");
        DR_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "render: streams");
        DR_CUDA(cudaEventCreateWithFlags(&c->ev_clear, cudaEventDisableTiming), "render: events");
        for (int k = 0; k < dr_ctx::kBands; ++k) {
            DR_CUDA(cudaEventCreateWithFlags(&c->band_done[k], cudaEventDisableTiming), "render: events");
            DR_CUDA(cudaEventCreateWithFlags(&c->copy_done[k], cudaEventDisableTiming), "render: events");
        }
        DR_CUDA(c->band_work.reserve(dr_ctx::kBands), "render: queues");
    }
    if (c->pinned_n < n) {
        if (c->pinned) cudaFreeHost(c->pinned);
        c->pinned = nullptr;
        c->pinned_n = 0;
        DR_CUDA(cudaHostAlloc((void **)&c->pinned, 2 * n * sizeof(float4), cudaHostAllocDefault),
                "render: pinned staging");
        c->pinned_n = n;
    }
    return DR_OK;
}

// Blocking render into host buffers.  The tile's rows are cut into up to
// kBands even bands; band k renders on stream k % 2 (so a band starts while the
// previous one drains), is copied to pinned staging on the copy stream when it
// is done, and the host moves it to the caller's buffers while later bands
// still render.  Paths depend only on (pixel, sample): banding does not change
// the result.
int dr_render_tile(dr_ctx *c, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed,
                   uint64_t sample_base, float *sun_out, float *sky_out) {
    if (!c || !sun_out || !sky_out) return need(false, DR_ERR_INVALID, "dr_render_tile: null argument");
    if (!c->has_scene || !c->has_params)
        return need(false, DR_ERR_STATE, "render: upload a scene and set parameters first");
    if (tw == 0 || th == 0) return need(false, DR_ERR_INVALID, "render: empty tile");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    const size_t n = (size_t)tw * th;
    DR_CUDA(c->tile_sun.reserve(n), "render: alloc tile");
    DR_CUDA(c->tile_sky.reserve(n), "render: alloc tile");
    DR_CUDA(c->call_counters.reserve(1), "render: alloc counters");
    int rc = ensure_pipeline(c, n);
    if (rc != DR_OK) return rc;
    const uint32_t rows = 2 * (th / 2);
    const uint32_t nb = rows >= 512 ? 8u : rows >= 128 ? 4u : 1u;
    uint32_t hb = (rows + nb - 1) / nb;
    hb += hb & 1u;
    DR_CUDA(cudaMemsetAsync(c->tile_sun.p, 0, n * sizeof(float4), c->stream), "render: clear");
    DR_CUDA(cudaMemsetAsync(c->tile_sky.p, 0, n * sizeof(float4), c->stream), "render: clear");
    DR_CUDA(cudaMemsetAsync(c->call_counters.p, 0, sizeof(DevCounters), c->stream), "render: clear");
    DR_CUDA(cudaEventRecord(c->ev_clear, c->stream), "render: record");
    DR_CUDA(cudaStreamWaitEvent(c->band_stream[0], c->ev_clear, 0), "render: wait");
    DR_CUDA(cudaStreamWaitEvent(c->band_stream[1], c->ev_clear, 0), "render: wait");
    const uint32_t tile = c->tuning.kernel == DR_KERNEL_PER_PATH ? 0u : c->tuning.tile;
    std::vector<std::pair<size_t, size_t>> spans;  // (float4 offset, float4 count) per band
    cudaError_t err = cudaSuccess;
    for (uint32_t k = 0, r0 = 0; r0 < rows && err == cudaSuccess; ++k, r0 += hb) {
        const uint32_t rk = rows - r0 < hb ? rows - r0 : hb;
        TileArgs A;
        rc = make_tile_args(x0, y0 + r0, tw, rk, spp, seed, sample_base, tile, A);
        if (rc != DR_OK) break;
        const size_t off = (size_t)r0 * tw, cnt = (size_t)rk * tw;
        float4 *sd = c->tile_sun.p + off, *kd = c->tile_sky.p + off;
        cudaStream_t bs = c->band_stream[k & 1];
        if (c->tuning.kernel == DR_KERNEL_PER_PATH)
            err = launch_render_tile(c->scene, c->params, A, c->mie_pack.p, sd, kd, c->call_counters.p, bs);
        else
            err = launch_render_persistent(c->scene, c->params, A, c->mie_pack.p, sd, kd, c->call_counters.p,
                                           c->band_work.p + k, c->tuning, c->device, bs,
                                           cam_lists(c, 1u + (k & 1u), (size_t)rows * A.cols, (size_t)r0 * A.cols));
        if (err == cudaSuccess) err = cudaEventRecord(c->band_done[k], bs);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(c->copy_stream, c->band_done[k], 0);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(c->pinned + 4 * off, sd, cnt * sizeof(float4), cudaMemcpyDeviceToHost,
                                  c->copy_stream);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(c->pinned + 4 * (c->pinned_n + off), kd, cnt * sizeof(float4),
                                  cudaMemcpyDeviceToHost, c->copy_stream);
        if (err == cudaSuccess) err = cudaEventRecord(c->copy_done[k], c->copy_stream);
        spans.emplace_back(off, cnt);
    }
    for (size_t k = 0; k < spans.size(); ++k) {
        const cudaError_t e = cudaEventSynchronize(c->copy_done[k]);
        if (e != cudaSuccess && err == cudaSuccess) err = e;
        if (err != cudaSuccess) break;
        const CopyPool::Range r[2] = {
            {sun_out + 4 * spans[k].first, c->pinned + 4 * spans[k].first, spans[k].second * sizeof(float4)},
            {sky_out + 4 * spans[k].first, c->pinned + 4 * (c->pinned_n + spans[k].first),
             spans[k].second * sizeof(float4)}};
        c->copies.copy(r, 2);
    }
    // keep the context stream ordered after the bands and the copies
    if (err == cudaSuccess) err = cudaStreamSynchronize(c->copy_stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(c->band_stream[0]);
    if (err == cudaSuccess) err = cudaStreamSynchronize(c->band_stream[1]);
    if (err != cudaSuccess) {
        cudaDeviceSynchronize();
        return cuda_fail(err, "render");
    }
    if (rc != DR_OK) return rc;
    if (rows < th) {  // odd tile: the last row is not rendered (2x2 pixel blocks)
        std::memset(sun_out + 4 * (size_t)rows * tw, 0, (size_t)tw * sizeof(float4));
        std::memset(sky_out + 4 * (size_t)rows * tw, 0, (size_t)tw * sizeof(float4));
    }
    return finish_call_counters(c, "dr_render_tile");
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
    c->gave_up_reported = 0;
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

int dr_probe_occlusion(dr_ctx *c, const float *ro, const float *rd, uint32_t n, uint32_t *hit) {
    if (!c || !ro || !rd || !hit || n == 0) return need(false, DR_ERR_INVALID, "dr_probe_occlusion: bad argument");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    Scratch S;
    size_t o_o = S.add(12ull * n), o_d = S.add(12ull * n), o_h = S.add(4ull * n);
    DR_CUDA(c->scratch.reserve(S.total), "probe: alloc");
    unsigned char *b = c->scratch.p;
    DR_CUDA(cudaMemcpy(b + o_o, ro, 12ull * n, cudaMemcpyHostToDevice), "probe: copy");
    DR_CUDA(cudaMemcpy(b + o_d, rd, 12ull * n, cudaMemcpyHostToDevice), "probe: copy");
    DR_CUDA(launch_probe_occlusion(c->scene, (const float *)(b + o_o), (const float *)(b + o_d), n,
                                   (uint32_t *)(b + o_h), c->stream),
            "probe: launch");
    DR_CUDA(cudaStreamSynchronize(c->stream), "probe: sync");
    DR_CUDA(cudaMemcpy(hit, b + o_h, 4ull * n, cudaMemcpyDeviceToHost), "probe: copy out");
    return DR_OK;
}

int dr_probe_density(dr_ctx *c, const uint32_t *nodes, const float *points, uint32_t n, float *out) {
    if (!c || !nodes || !points || !out || n == 0) return need(false, DR_ERR_INVALID, "dr_probe_density: bad argument");
    if (!c->has_scene) return need(false, DR_ERR_STATE, "dr_probe_density: no scene");
    for (uint32_t i = 0; i < n; ++i)
        if (nodes[i] >= c->leaf_flag.size() || !(c->leaf_flag[nodes[i]] & 2u))
            return need(false, DR_ERR_INVALID, "dr_probe_density: node is not a leaf with a fog brick");
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
    if (!c || !in || !out || n == 0 || what > DR_PROBE_ENV_MAP)
        return need(false, DR_ERR_INVALID, "dr_probe_sampler: bad argument");
    if (!c->has_params) return need(false, DR_ERR_STATE, "dr_probe_sampler: no parameters");
    if (what == DR_PROBE_MIE_EXACT_DIR && c->params.phase_mode != DR_PHASE_MIE_EXACT)
        return need(false, DR_ERR_STATE, "dr_probe_sampler: the exact sampler needs DR_PHASE_MIE_EXACT");
    if (what == DR_PROBE_ENV_MAP && c->params.env_mode != DR_ENV_MAP)
        return need(false, DR_ERR_STATE, "dr_probe_sampler: the environment map probe needs DR_ENV_MAP");
    const size_t in_n = (what == DR_PROBE_MIE_SAMPLE || what == DR_PROBE_HG_SAMPLE) ? 5ull * n
                        : what == DR_PROBE_SUN_SAMPLE ? 2ull * n
                        : (what == DR_PROBE_SKY || what == DR_PROBE_SKY_LIGHT || what == DR_PROBE_ENV_MAP) ? 3ull * n
                        : (size_t)n;
    const size_t out_n = (what == DR_PROBE_MIE_THETA || what == DR_PROBE_HG_EVAL) ? (size_t)n
                         : what == DR_PROBE_MIE_EXACT_DIR ? 2ull * n : 3ull * n;
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


// ---- differentiable rendering --------------------------------------------------
int dr_set_bricks_dev(dr_ctx *c, const float *bricks_dev, uint32_t n_leaves, float majorant_scale, void *stream) {
    if (!c || !bricks_dev) return need(false, DR_ERR_INVALID, "dr_set_bricks_dev: null argument");
    if (!c->has_scene) return need(false, DR_ERR_STATE, "dr_set_bricks_dev: no scene");
    if (n_leaves != c->scene.n_leaves)
        return need(false, DR_ERR_INVALID, "dr_set_bricks_dev: brick count differs from the scene's");
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    DR_CUDA(cudaMemcpyAsync(c->bufs.bricks.p, bricks_dev, (size_t)n_leaves * kBrick * sizeof(float),
                            cudaMemcpyDeviceToDevice, st),
            "dr_set_bricks_dev: copy");
    if (!(majorant_scale == 0.0f || majorant_scale >= 1.0f) || !std::isfinite(majorant_scale))
        return need(false, DR_ERR_INVALID, "dr_set_bricks_dev: majorant_scale must be 0 or >= 1");
    if (majorant_scale > 0.0f)
        DR_CUDA(launch_leaf_majorants(c->bufs.leaf.p, c->leaf_nodes.p, c->n_leaf_nodes, c->bufs.bricks.p,
                                      majorant_scale, st),
                "dr_set_bricks_dev: majorants");
    return DR_OK;
}

int dr_get_majorants(dr_ctx *c, float *out) {
    if (!c || !out) return need(false, DR_ERR_INVALID, "dr_get_majorants: null argument");
    if (!c->has_scene) return need(false, DR_ERR_STATE, "dr_get_majorants: no scene");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    std::vector<float4> leaf((size_t)c->scene.n_nodes * 2);
    DR_CUDA(cudaStreamSynchronize(c->stream), "dr_get_majorants: sync");
    DR_CUDA(cudaMemcpy(leaf.data(), c->bufs.leaf.p, leaf.size() * sizeof(float4), cudaMemcpyDeviceToHost),
            "dr_get_majorants: copy");
    for (uint32_t i = 0; i < c->scene.n_nodes; ++i) out[i] = c->leaf_flag[i] ? leaf[2 * (size_t)i + 1].x : 0.0f;
    return DR_OK;
}

int dr_adjoint_tile_async(dr_ctx *c, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed,
                          uint64_t sample_base, const float *dsun_dev, const float *dsky_dev, float *grad_bricks_dev,
                          double *grad_albedo_dev, void *stream) {
    if (!c || !dsun_dev || !dsky_dev || !grad_bricks_dev || !grad_albedo_dev)
        return need(false, DR_ERR_INVALID, "dr_adjoint_tile_async: null argument");
    TileArgs A;
    int rc = tile_args(c, x0, y0, tw, th, spp, seed, sample_base, 0u, A);
    if (rc != DR_OK) return rc;
    if (!(c->params.albedo > 0.0f))
        return need(false, DR_ERR_INVALID, "dr_adjoint_tile_async: the albedo gradient needs sigma_s > 0");
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    // spread copies of the gradient: up to 16, within 256 MB
    const size_t gbytes = (size_t)c->scene.n_leaves * kBrick * sizeof(float);
    uint32_t copies = (uint32_t)std::min<size_t>(16, (256u << 20) / (gbytes ? gbytes : 1));
    if (copies > 1 && c->grad_copies.reserve((size_t)copies * c->scene.n_leaves * kBrick) != cudaSuccess) copies = 1;
    if (!c->albedo_slots.p) {
        DR_CUDA(c->albedo_slots.reserve(adjoint_slots()), "adjoint: alloc slots");
        DR_CUDA(cudaMemset(c->albedo_slots.p, 0, sizeof(double) * adjoint_slots()), "adjoint: clear slots");
    }
    // one 16-byte record per path of a chunk (at most 2^23 paths, 128 MB)
    const uint64_t chunk = std::min<uint64_t>(A.n_paths, 1ull << 23);
    DR_CUDA(c->path_rec.reserve(chunk), "adjoint: alloc path records");
    DR_CUDA(launch_adjoint_tile(c->scene, c->params, A, c->mie_pack.p, (const float4 *)dsun_dev,
                                (const float4 *)dsky_dev, grad_bricks_dev, copies > 1 ? c->grad_copies.p : nullptr,
                                copies, c->path_rec.p, chunk, grad_albedo_dev, c->albedo_slots.p, c->counters.p, st),
            "adjoint: launch");
    return DR_OK;
}

int dr_reweighted_loss_async(dr_ctx *c, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp,
                             uint64_t seed, uint64_t sample_base, const float *dsun_dev, const float *dsky_dev,
                             const float *pert_bricks_dev, double *loss_dev, void *stream) {
    if (!c || !dsun_dev || !dsky_dev || !pert_bricks_dev || !loss_dev)
        return need(false, DR_ERR_INVALID, "dr_reweighted_loss_async: null argument");
    TileArgs A;
    int rc = tile_args(c, x0, y0, tw, th, spp, seed, sample_base, 0u, A);
    if (rc != DR_OK) return rc;
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    if (!c->albedo_slots.p) {
        DR_CUDA(c->albedo_slots.reserve(adjoint_slots()), "reweighted loss: alloc slots");
        DR_CUDA(cudaMemset(c->albedo_slots.p, 0, sizeof(double) * adjoint_slots()), "reweighted loss: clear slots");
    }
    DR_CUDA(launch_reweighted_loss(c->scene, c->params, A, c->mie_pack.p, (const float4 *)dsun_dev,
                                   (const float4 *)dsky_dev, pert_bricks_dev, loss_dev, c->albedo_slots.p,
                                   c->counters.p, st),
            "reweighted loss: launch");
    return DR_OK;
}

int dr_adjoint_transmittance(dr_ctx *c, const float *ro, const float *rd, const float *weights, uint32_t n,
                             uint64_t nsamp, uint64_t seed, float *grad_bricks, double *transmittance) {
    if (!c || !ro || !rd || !weights || !grad_bricks || n == 0 || nsamp == 0)
        return need(false, DR_ERR_INVALID, "dr_adjoint_transmittance: bad argument");
    if (!c->has_scene || !c->has_params) return need(false, DR_ERR_STATE, "dr_adjoint_transmittance: no scene");
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    const size_t ng = (size_t)c->scene.n_leaves * kBrick;
    Scratch S;
    size_t o_ro = S.add(12 * (size_t)n), o_rd = S.add(12 * (size_t)n), o_w = S.add(4 * (size_t)n),
           o_e = S.add(8 * (size_t)n), o_g = S.add(4 * ng);
    DR_CUDA(c->scratch.reserve(S.total), "adjoint: alloc");
    unsigned char *b = c->scratch.p;
    DR_CUDA(cudaMemcpy(b + o_ro, ro, 12 * (size_t)n, cudaMemcpyHostToDevice), "adjoint: copy");
    DR_CUDA(cudaMemcpy(b + o_rd, rd, 12 * (size_t)n, cudaMemcpyHostToDevice), "adjoint: copy");
    DR_CUDA(cudaMemcpy(b + o_w, weights, 4 * (size_t)n, cudaMemcpyHostToDevice), "adjoint: copy");
    DR_CUDA(cudaMemset(b + o_e, 0, 8 * (size_t)n), "adjoint: clear");
    DR_CUDA(cudaMemset(b + o_g, 0, 4 * ng), "adjoint: clear");
    DR_CUDA(launch_adjoint_transmittance(c->scene, c->params, (const float *)(b + o_ro), (const float *)(b + o_rd),
                                         (const float *)(b + o_w), n, nsamp, seed, (float *)(b + o_g),
                                         (unsigned long long *)(b + o_e), c->stream),
            "adjoint: launch");
    DR_CUDA(cudaStreamSynchronize(c->stream), "adjoint: sync");
    DR_CUDA(cudaMemcpy(grad_bricks, b + o_g, 4 * ng, cudaMemcpyDeviceToHost), "adjoint: copy out");
    if (transmittance) {
        std::vector<unsigned long long> esc(n);
        DR_CUDA(cudaMemcpy(esc.data(), b + o_e, 8 * (size_t)n, cudaMemcpyDeviceToHost), "adjoint: copy out");
        for (uint32_t i = 0; i < n; ++i) transmittance[i] = (double)esc[i] / (double)nsamp;
    }
    return DR_OK;
}

}  // extern "C"
