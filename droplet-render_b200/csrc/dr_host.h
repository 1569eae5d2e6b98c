// Host-side helpers shared by the C-ABI entry points (dr_api.cu, dr_batch.cu):
// error reporting, device buffers, and the validation + conversion of scenes
// and render settings into their device layouts.
#pragma once
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/droplet_b200.h"
#include "dr_internal.h"

namespace dr {

void set_error(int code, const std::string &msg);
const char *last_error();
int cuda_fail(cudaError_t e, const char *what);
// Returns DR_OK when ok, else records msg and returns code.
int need(bool ok, int code, const char *msg);

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

// A validated scene in its device layout, still on the host.
struct HostScene {
    std::vector<uint32_t> child;   // 8 per node (see DevScene)
    std::vector<float4> leaf;      // 2 per node
    std::vector<uint32_t> macro, cells;
    std::vector<uint8_t> leaf_flag;
    uint32_t levels = 0, n = 0, mdim = 0;
    uint32_t stack_levels = 0;  // traversal stack entries a ray can need (0: unknown, local stack only)
    uint32_t n_nodes = 0, n_leaves = 0;
    float root_ce[4] = {0, 0, 0, 0};
    const float *bricks = nullptr;  // the caller's brick pool (n_leaves * 512 floats)
    const float *sdf = nullptr;     // the caller's SDF pool (n_sdf * 512 floats) or null
    uint32_t n_sdf = 0;
};

// Device buffers of one uploaded scene.
struct SceneBufs {
    DevBuf<uint4> child;
    DevBuf<float4> leaf;
    DevBuf<float> bricks;
    DevBuf<float> sdf;
    DevBuf<uint32_t> macro, cells;
    void release() {
        child.release();
        leaf.release();
        bricks.release();
        sdf.release();
        macro.release();
        cells.release();
    }
};

// Checks a scene descriptor (src/scene.h:21-31 records) and builds the device
// layout: remapped child entries, leaf records, and the leaf grid of the cell walk.
int prepare_scene(const dr_scene_desc *s, HostScene &out);
// Copies a prepared scene into bufs (synchronously on st) and fills S.
int upload_scene(const HostScene &h, SceneBufs &bufs, bool use_grid, cudaStream_t st, DevScene &S);
// Checks render settings and converts them (the depth pointer is left null);
// pack receives the phase tables as staged in shared memory.
int prepare_params(const dr_render_params *p, DevParams &d, std::vector<unsigned char> &pack);
// Shared-memory pack size of the phase tables for d.
size_t mie_pack_bytes(const DevParams &d);
// Tile arguments of a render call (tile > 0: square pixel order of the persistent kernel).
int make_tile_args(uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed, uint64_t base,
                   uint32_t tile, TileArgs &A);
bool valid_tuning(const dr_tuning *t);

// Occluder BVH as built on the host (layout of DevScene::occ_nodes/occ_tris,
// 16 and 12 floats per node and triangle); source[j] = the selected triangle
// (in surface order) stored at position j.
struct OccBvh {
    std::vector<float> nodes;
    std::vector<float> tris;
    std::vector<uint32_t> source;
};
int build_occluder_bvh(const dr_surface *s, uint32_t n, uint32_t mode, OccBvh &out);

}  // namespace dr

// The context behind the C ABI's opaque dr_ctx handle.
namespace dr {
// Host threads that share the copies from pinned staging into the caller's
// buffers (dr_render_tile).  The costly bands of a frame (the cloud's rows)
// tend to finish last and close together, so one thread copying each 8 MB band
// after it lands (about 1 ms each) put several milliseconds after the last
// kernel; split over the pool's threads and the calling thread, each copy
// takes a fraction of that.  Threads start on the first large copy and stop
// when the pool is destroyed.
class CopyPool {
  public:
    struct Range {
        void *dst;
        const void *src;
        size_t bytes;
    };
    CopyPool() = default;
    CopyPool(const CopyPool &) = delete;
    CopyPool &operator=(const CopyPool &) = delete;
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lk(m_);
            quit_ = true;
        }
        work_.notify_all();
        for (std::thread &t : threads_) t.join();
    }
    // Copies every range; returns when all bytes are in place.
    void copy(const Range *r, size_t n) {
        size_t total = 0;
        for (size_t i = 0; i < n; ++i) total += r[i].bytes;
        start();
        if (threads_.empty() || total < kMinSplit) {
            for (size_t i = 0; i < n; ++i) std::memcpy(r[i].dst, r[i].src, r[i].bytes);
            return;
        }
        const size_t parts = threads_.size() + 1;
        const size_t chunk = ((total / parts) + 4095) & ~(size_t)4095;
        {
            std::lock_guard<std::mutex> lk(m_);
            jobs_.clear();
            next_ = 0;
            for (size_t i = 0; i < n; ++i)
                for (size_t o = 0; o < r[i].bytes; o += chunk)
                    jobs_.push_back({static_cast<char *>(r[i].dst) + o, static_cast<const char *>(r[i].src) + o,
                                     r[i].bytes - o < chunk ? r[i].bytes - o : chunk});
            pending_ = jobs_.size();
        }
        work_.notify_all();
        for (;;) {  // the calling thread copies too
            Job j;
            {
                std::lock_guard<std::mutex> lk(m_);
                if (next_ >= jobs_.size()) break;
                j = jobs_[next_++];
            }
            run(j);
        }
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [&] { return pending_ == 0; });
    }

  private:
    static constexpr size_t kMinSplit = 4u << 20;
    struct Job {
        char *dst;
        const char *src;
        size_t n;
    };
    void run(const Job &j) {
        std::memcpy(j.dst, j.src, j.n);
        std::lock_guard<std::mutex> lk(m_);
        if (--pending_ == 0) done_.notify_all();
    }
    void start() {
        if (started_) return;
        started_ = true;
        const unsigned hw = std::thread::hardware_concurrency();
        const unsigned n = hw > 1 ? (hw < 8 ? hw : 8) - 1 : 0;
        try {
            for (unsigned i = 0; i < n; ++i) threads_.emplace_back([this] { loop(); });
        } catch (...) {  // fewer threads (or none): the calling thread copies the rest
        }
    }
    void loop() {
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(m_);
                work_.wait(lk, [&] { return quit_ || next_ < jobs_.size(); });
                if (quit_) return;
                j = jobs_[next_++];
            }
            run(j);
        }
    }
    std::mutex m_;
    std::condition_variable work_, done_;
    std::vector<std::thread> threads_;
    std::vector<Job> jobs_;
    size_t next_ = 0, pending_ = 0;
    bool quit_ = false, started_ = false;
};
}  // namespace dr

struct dr_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    bool has_scene = false, has_params = false;
    dr::DevScene scene{};
    dr::DevParams params{};
    dr::SceneBufs bufs;
    dr::DevBuf<unsigned char> mie_pack;
    dr::DevBuf<float> depth;
    dr::DevBuf<float> env;            // environment map texels (DR_ENV_MAP)
    dr::DevBuf<dr::DevCounters> counters;
    dr::DevBuf<dr::DevCounters> call_counters;  // a blocking call's own counts (added to `counters` at its end)
    uint32_t step_budget = dr::kStepBudget;     // dr_set_step_budget
    unsigned long long gave_up_reported = 0;    // counters.gave_up when dr_check_complete last looked
    dr::DevBuf<float4> tile_sun, tile_sky;
    dr::DevBuf<unsigned char> scratch;
    dr::DevBuf<dr::WorkQueue> work;
    dr::DevBuf<uint32_t> leaf_nodes;  // ids of the leaf nodes (majorant updates)
    dr::DevBuf<float> grad_copies;    // adjoint: spread copies of the brick-pool gradient
    dr::DevBuf<double> albedo_slots;  // adjoint: partial sums of the albedo gradient (kept zeroed)
    dr::DevBuf<uint4> path_rec;       // adjoint: one record per path of a chunk (totals pass -> scatter pass)
    dr::DevBuf<float4> occ_nodes, occ_tris;  // occluder BVH (kept across scene uploads)
    uint32_t occ_n_nodes = 0;
    uint32_t n_leaf_nodes = 0;
    bool use_grid = true;
    dr::Tuning tuning{0u, 128u, 0u, 8u, 0u, 0u, 0u, 0u};
    std::vector<uint8_t> leaf_flag;  // host copy: node i is a leaf (for validating probe inputs)
    // host-buffer render pipeline (dr_render_tile): row bands rendered on two
    // streams, each copied to pinned staging as soon as it is done
    static constexpr int kBands = 8;
    cudaStream_t band_stream[2] = {nullptr, nullptr};
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_clear = nullptr;
    cudaEvent_t band_done[kBands] = {};
    cudaEvent_t copy_done[kBands] = {};
    dr::DevBuf<dr::WorkQueue> band_work;
    // camera leaf lists of the persistent kernel (TileArgs::cam_head): headers
    // per pixel of a launch and a pool of kCamPool entries with a fill counter,
    // for the asynchronous render (slot 0) and each band stream of the blocking
    // render (slots 1, 2); allocated on first use
    static constexpr uint32_t kCamPool = 1u << 23;
    uint32_t cam_cap = kCamPool;  // entries per pool (dr_set_camera_lists; 0: no lists)
    dr::DevBuf<uint4> cam_head, cam_pool, band_cam_head, band_cam_pool;
    dr::DevBuf<unsigned int> cam_used;
    float *pinned = nullptr;  // 2 * pinned_n float4: sun then sky
    size_t pinned_n = 0;
    dr::CopyPool copies;      // host threads for the staging -> caller copies
};
