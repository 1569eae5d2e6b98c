// Kernel launchers (host side, C++ linkage, internal to the library).
#pragma once
#include <cuda_runtime.h>
#include "dr_internal.h"

namespace dr {

constexpr int kRenderBlock = 128;
constexpr int kPersistentBlock = 128;

cudaError_t launch_render_tile(const DevScene &S, const DevParams &P, const TileArgs &A, const void *mie_pack,
                               float4 *sun_out, float4 *sky_out, DevCounters *C, cudaStream_t st);
cudaError_t launch_shadow_tile(const DevScene &S, const DevParams &P, const TileArgs &A, float4 *out, DevCounters *C,
                               cudaStream_t st);
// Camera leaf list storage for one persistent launch: head[2 * cols * rows],
// pool[cap] and its fill counter (head null: no lists).
struct CamLists {
    uint4 *head = nullptr;
    uint4 *pool = nullptr;
    uint32_t cap = 0;
    unsigned int *used = nullptr;
};
// Persistent path kernel; Q->next must be 0 (the launcher clears it on st).
// With a stack traversal and lists given, the camera rays' leaf lists are built
// on st first (camera_list_kernel).
cudaError_t launch_render_persistent(const DevScene &S, const DevParams &P, const TileArgs &A, const void *mie_pack,
                                     float4 *sun_out, float4 *sky_out, DevCounters *C, WorkQueue *Q,
                                     const Tuning &tune, int device, cudaStream_t st, const CamLists &lists = {});
// Batched persistent launch over all views of B (P0: the first view's parameters,
// which fix the shared phase tables), then one increment of *step; Q->next is
// cleared on st first.  The three launches are what a batch's graph captures.
// stack_levels: the deepest traversal stack any of the batch's scenes needs (0: unknown)
// lists: the views' camera leaf lists (the views' TileArgs::cam_head point at
// lists.head + pix_begins[v]; head null when the views traverse), built first.
struct BatchLists {
    CamLists lists;
    const uint32_t *pix_begins = nullptr;  // first pixel of each view among the batch's pixels
    uint32_t n_pix = 0;
};
cudaError_t launch_render_batch(const BatchArgs &B, const DevParams &P0, const void *mie_pack, DevCounters *C,
                                WorkQueue *Q, unsigned long long *step, const Tuning &tune, bool ext,
                                uint32_t stack_levels, int device, cudaStream_t st, const BatchLists &lists = {});
// The parts of launch_render_batch, for graphs that split a batch:
// the camera leaf lists of every view of B (nothing when lists.head is null);
cudaError_t launch_batch_lists(const BatchArgs &B, const BatchLists &lists, cudaStream_t st);
// one batched persistent kernel over the views of B (Q->next must be 0);
cudaError_t launch_batch_kernel(const BatchArgs &B, const DevParams &P0, const void *mie_pack, DevCounters *C,
                                WorkQueue *Q, const Tuning &tune, bool ext, uint32_t stack_levels, int device,
                                cudaStream_t st);
// one view of a batch as a plain persistent kernel of its own: the view's
// parameters and tile are kernel arguments (A.cam_head: its lists, already
// built; A.sample_base + *step * spp is its first sample; Q->next must be 0);
cudaError_t launch_batch_view(const DevScene &S, const DevParams &P, const TileArgs &A, const void *mie_pack,
                              float4 *sun_out, float4 *sky_out, DevCounters *C, WorkQueue *Q,
                              const unsigned long long *step, const Tuning &tune, int device, cudaStream_t st);
// *step += 1 (the last node of a batch's graph).
cudaError_t launch_batch_step(unsigned long long *step, cudaStream_t st);
// Resident blocks per SM of the persistent kernel for the given dynamic shared memory.
int persistent_max_blocks_per_sm(uint32_t variant, uint32_t traversal, size_t smem_bytes);
cudaError_t launch_probe_leaf(const DevScene &S, const float *ro, const float *rd, uint32_t n, uint32_t maxn,
                              uint32_t *nodes, float *tr0, float *tr1, uint32_t *counts, cudaStream_t st);
cudaError_t launch_probe_occlusion(const DevScene &S, const float *ro, const float *rd, uint32_t n, uint32_t *hit,
                                   cudaStream_t st);
cudaError_t launch_probe_density(const DevScene &S, const uint32_t *nodes, const float *pts, uint32_t n, float *out,
                                 cudaStream_t st);
cudaError_t launch_probe_paths(const DevScene &S, const DevParams &P, const void *mie_pack, const uint32_t *px,
                               const uint32_t *py, const uint64_t *sample, uint32_t n, uint64_t seed,
                               float4 *out_sun, float4 *out_sky, DevCounters *C, cudaStream_t st);
cudaError_t launch_probe_sampler(const DevParams &P, const void *mie_pack, uint32_t what, const float *in, uint32_t n,
                                 float *out, cudaStream_t st);
cudaError_t launch_probe_transmittance(const DevScene &S, const DevParams &P, const float *ro, const float *rd,
                                       uint32_t n_rays, uint64_t nsamp, uint64_t seed, unsigned long long *escapes,
                                       cudaStream_t st);

// Path-replay adjoint of a tile (delta images in tile layout) and of a set of
// transmittance rays; gradients accumulate into grad (brick-pool layout).
// copies > 1: gradients are first spread over `copies` zeroed copies in
// copies_buf (copies * n_leaves * 512 floats), then summed into grad.
// The albedo gradient is gathered in adjoint_slots() zeroed doubles (slots),
// then added to *grad_albedo (and the slots zeroed again).  The paths run in
// chunks of `chunk`: a totals launch writes a 16-byte record per path to
// records (chunk records: the path's weight and which shadow segments escape),
// then a scatter launch replays the chunk's paths.
cudaError_t launch_adjoint_tile(const DevScene &S, const DevParams &P, const TileArgs &A, const void *mie_pack,
                                const float4 *dsun, const float4 *dsky, float *grad, float *copies_buf,
                                uint32_t copies, void *records, uint64_t chunk, double *grad_albedo, double *slots,
                                DevCounters *C, cudaStream_t st);
uint32_t adjoint_slots();
// Reweighted replay of a tile (decisions from S's bricks, weights from pert):
// adds the linearised loss to *loss through the zeroed slots.
cudaError_t launch_reweighted_loss(const DevScene &S, const DevParams &P, const TileArgs &A, const void *mie_pack,
                                   const float4 *dsun, const float4 *dsky, const float *pert, double *loss,
                                   double *slots, DevCounters *C, cudaStream_t st);
cudaError_t launch_adjoint_transmittance(const DevScene &S, const DevParams &P, const float *ro, const float *rd,
                                         const float *wr, uint32_t n_rays, uint64_t nsamp, uint64_t seed, float *grad,
                                         unsigned long long *escapes, cudaStream_t st);
// Leaf majorants of the listed leaf nodes recomputed from the brick pool.
cudaError_t launch_leaf_majorants(float4 *leaf, const uint32_t *leaf_nodes, uint32_t n_leafnodes, const float *bricks,
                                  float scale, cudaStream_t st);

// dst += src, field by field (one thread; a blocking call's counters).
cudaError_t launch_add_counters(DevCounters *dst, const DevCounters *src, cudaStream_t st);

// Allocation-free transmittance: scratch in a file-scope device array.
uint32_t noalloc_max_rays();
cudaError_t noalloc_scratch(int device, unsigned long long **out);
cudaError_t launch_transmittance_noalloc(const DevScene &S, const DevParams &P, unsigned long long *scratch,
                                         const float *ro, const float *rd, uint32_t n_rays, uint64_t nsamp,
                                         uint64_t seed, double *out, cudaStream_t st);

}  // namespace dr
