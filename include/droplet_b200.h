/* droplet_b200 — B200 (sm_100a) implementation of droplet-render's volumetric
 * path-tracing hot path, exposed as a plain C ABI (no CUDA or torch types).
 *
 * Each entry point names the reference interface it replaces.  The reference
 * renderer is RenderKernel (src/kernel.h:11-59) driven from the CPython module
 * libdroplet (src/main.cpp:64-771); its scene is the octree + 8^3 brick pool of
 * class Scene (src/scene.h:146-159).
 *
 * Conventions
 *  - Every function returns DR_OK (0) or a negative DR_ERR_* code; the text
 *    of the last error on the calling thread is returned by dr_last_error().
 *  - Host pointers unless a name ends in _dev; a stream argument is a
 *    cudaStream_t passed as void* (NULL = the context's own stream).
 *  - Images are float4 per pixel (r, g, b, alpha), row-major within a tile.
 */
#ifndef DROPLET_B200_H
#define DROPLET_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DR_OK 0
#define DR_ERR_INVALID (-1)   /* bad argument or descriptor */
#define DR_ERR_CUDA (-2)      /* CUDA runtime failure (message has the CUDA error) */
#define DR_ERR_STATE (-3)     /* call out of order (no scene, no parameters, busy) */
#define DR_ERR_NOMEM (-4)     /* host or device allocation failed */
#define DR_ERR_GAVE_UP (-5)   /* some paths hit an iteration budget and were cut short: the outputs
                                  are written but incomplete (dr_render_tile, dr_shadow_tile,
                                  dr_check_complete) */
#define DR_ERR_NODEVICE (-6)  /* no CUDA device */

#define DR_NONE 0xffffffffu

/* Octree node record, identical to the reference's OctreeStructure
 * (src/scene.h:21-31): 64 bytes. */
typedef struct {
    float ce[4];        /* center x, y, z; half extent */
    uint32_t chn[8];    /* child node index, 0 = none; child i sits at offset (i&1, i>>1&1, i>>2) */
    uint32_t volx[2];   /* brick index in the [SDF, FOG] pools or DR_NONE */
    float qval[2];      /* per-leaf query value; FOG: max density (majorant), floor 0.01 */
} dr_node;

/* A built scene: what Scene::Initialize leaves in Scene::ob / Scene::pvol
 * (src/scene.cpp:840-917). */
typedef struct {
    dr_node *nodes;
    uint32_t n_nodes;
    float *bricks;      /* FOG brick pool: n_leaves * lvoxc^3 floats, x fastest */
    uint32_t n_leaves;
    uint32_t lvoxc;     /* samples per brick edge (8) */
    uint32_t mlevel;    /* octree depth; leaves sit at level mlevel-1 */
} dr_octree;

/* Scene description handed to dr_upload_scene (the fields of dr_octree, plus
 * the surface pool Scene::pvol[VOLUME_BUFFER_SDF]).  A leaf carries a FOG brick
 * (volx[1]), an SDF brick (volx[0]: signed distance samples, same layout), or
 * both; SDF leaves take majorant 1 (src/kernel.cpp:245-251). */
typedef struct {
    const dr_node *nodes;
    uint32_t n_nodes;
    const float *bricks;        /* FOG pool: n_leaves bricks */
    uint32_t n_leaves;
    uint32_t lvoxc;
    const float *sdf_bricks;    /* SDF pool: n_sdf_leaves bricks, or NULL when no leaf has one */
    uint32_t n_sdf_leaves;
} dr_scene_desc;

#define DR_PHASE_MIE_REFERENCE 0u  /* the reference's tabulated sampler (src/KernelSampler.cpp:257-285) */
#define DR_PHASE_MIE_EXACT 1u      /* exact inverse CDF of the tabulated phase x sin(theta); mie_n <= 512 */
#define DR_PHASE_HG 2u             /* HGPhase (src/KernelSampler.cpp:164-204), anisotropy hg_g; Mie tables optional */

#define DR_ENV_HOSEK 0u  /* sky light from the Hosek-Wilkie state (the reference built with USE_ARHOSEK_SKYMODEL) */
#define DR_ENV_NONE 1u   /* NullEnv: no sky light (its default build without an environment texture) */
#define DR_ENV_MAP 2u    /* MapEnv (src/KernelSampler.cpp:377-417): pow(bilinear equirectangular texel, 2.2) */

/* Everything RenderKernel::Initialize receives (src/kernel.cpp:497-534) plus
 * the sun light (src/main.cpp:374-404) and the sky state the reference
 * hard-codes (src/kernel.cpp:521-526). */
typedef struct {
    float sigma_s, sigma_a;        /* macroscopic cross sections (msigmas, msigmaa) */
    uint32_t scattevs;             /* max scattering events */
    float sun_dir[3];              /* unit vector towards the sun */
    float sun_color[3];            /* colour * intensity */
    float sun_angle;               /* cone half angle, radians */
    double sky_configs[3][9];      /* cooked Hosek-Wilkie RGB state (ArHosekSkyModelState.configs) */
    double sky_radiances[3];       /* ArHosekSkyModelState.radiances */
    const float *mie_pdf;          /* mie_n RGB entries, index 0 = backscatter */
    const float *mie_cdf;          /* mie_n RGB entries */
    uint32_t mie_n;                /* 256 for the reference table; 2..4096 */
    uint32_t phase_mode;           /* DR_PHASE_* */
    float viewi[16];               /* inverse view matrix, rows r[0..3] */
    float proji[16];               /* inverse projection matrix, rows r[0..3] */
    uint32_t w, h;                 /* full image size */
    const float *depth;            /* optional w*h depth texture (distance along the camera ray), or NULL */
    uint32_t flags;                /* DR_KERNEL_* below */
    float hg_g;                    /* DR_PHASE_HG: HGPhase::g1 (blcloudsampling.phasea), |g| < 1 */
    uint32_t env_mode;             /* DR_ENV_*: where escaping light comes from (src/kernel.cpp:329-364) */
    const float *env_map;          /* DR_ENV_MAP: env_w * env_h RGBA floats, row-major (MapEnv::Initialize) */
    uint32_t env_w, env_h;         /* DR_ENV_MAP: texels, each >= 2, env_w * env_h <= 2^24 */
} dr_render_params;
#define DR_KERNEL_DEPTHCOMP 0x1u     /* camera rays stop at depth (src/kernel.h:4) */
#define DR_KERNEL_FINITE_PATHS 0x2u  /* a path sample whose sun or sky sum is not finite adds nothing (the
                                        reference's sky term is 0/0 for rd.y == 0, src/kernel.cpp:338-342) */
#define DR_KERNEL_EMBREE 0x4u        /* the reference built with USE_EMBREE (its occlusion option): light that a
                                        segment gathers on escape is zeroed when the segment's ray hits an
                                        occluder (src/kernel.cpp:149-153, 375-383), and a camera ray cut at its
                                        depth gets alpha 0 instead of 1 (the same block's depth mask) */

/* In-kernel counters accumulated over all launches since the last reset. */
typedef struct {
    uint64_t paths;            /* camera path samples started */
    uint64_t vertices;         /* traced segments: camera + continuation + shadow */
    uint64_t node_visits;      /* octree node records examined */
    uint64_t density_lookups;  /* trilinear brick lookups */
    uint64_t mie_evals;        /* phase table evaluations and samples */
    uint64_t gave_up;          /* path segments cut by the step budget, plus blocks whose table
                                  staging timed out (and so rendered nothing) */
} dr_counters;

typedef struct dr_ctx dr_ctx;

/* ---- library ------------------------------------------------------------- */
/* Version of the interface in this header.  dr_version() returns the version
 * the library was built with; a caller built against another header must not
 * pass it structs (200: dr_scene_desc gained the SDF pool, dr_render_params the
 * phase and environment fields). */
#define DR_VERSION 200
int dr_version(void);
const char *dr_last_error(void);
int dr_device_count(int *count);

/* ---- context: replaces the module globals gpkernel/gpscene (src/main.cpp:16-18) */
int dr_create(int device, dr_ctx **out);
int dr_destroy(dr_ctx *ctx);                 /* DRE_EndRender, src/main.cpp:688-716 */

/* ---- scene --------------------------------------------------------------- */
/* Host octree build from sparse 8^3 blocks (OpenVDB-leaf shaped input):
 * Scene::Initialize + S_Create leaf/octree/brick stages (src/scene.cpp:676-762,
 * 840-908, BuildPath 267-305).  Voxel (i,j,k) sits at world (i,j,k)*voxel_size
 * and is active when non-zero.  block_origin: 3 int32 per block, multiples of 8,
 * non-negative; block_values: 512 floats per block (x fastest).  Free the
 * result with dr_octree_free. */
int dr_build_octree(const int32_t *block_origin, const float *block_values, uint32_t n_blocks, float voxel_size,
                    uint32_t maxdepth, int nthreads, dr_octree *out);
void dr_octree_free(dr_octree *oct);

/* Copies nodes and bricks to the device (the reference reads Scene::ob/pvol
 * in place, src/kernel.cpp:225-305). */
int dr_upload_scene(dr_ctx *ctx, const dr_scene_desc *scene);

/* ---- occlusion geometry: SceneOcclusion (src/SceneOcclusion.cpp:19-91) -------
 * Triangle meshes (SceneData::Surface: world-space vertices vl, triangle index
 * list tl, object flags) replace the Embree scene.  With DR_KERNEL_EMBREE set in
 * the parameters, a segment whose ray (origin, direction; t in [0, 1e6]) hits
 * any occluder triangle gathers no sun or sky light when it escapes.  Replaces
 * rtcIntersect4 with a BVH built here and an any-hit traversal on the GPU. */
typedef struct {
    const float *vertices;     /* 3 * n_vertices floats */
    uint32_t n_vertices;
    const uint32_t *indices;   /* 3 * n_triangles vertex indices */
    uint32_t n_triangles;
    uint32_t flags;            /* DR_SURFACE_HOLDOUT (SCENEOBJ_HOLDOUT, src/scene.h:54) */
} dr_surface;
#define DR_SURFACE_HOLDOUT 0x2u
#define DR_OCCLUDE_ALL_SURFACES 0u  /* the reference: `!flags & SCENEOBJ_HOLDOUT` (src/SceneOcclusion.cpp:27) is
                                       always 0, so every surface occludes */
#define DR_OCCLUDE_HOLDOUT_ONLY 1u  /* the evident intent: only surfaces flagged DR_SURFACE_HOLDOUT occlude */
/* Builds the occluder BVH on the host and uploads it; n_surfaces == 0 (or no
 * triangle selected) removes the occluders.  Kept across dr_upload_scene. */
int dr_set_occluders(dr_ctx *ctx, const dr_surface *surfaces, uint32_t n_surfaces, uint32_t mode);
/* The BVH dr_set_occluders would build, for inspection (host buffers, NULL to
 * query sizes): nodes = 16 floats each (left box min xyz, max xyz, right box
 * min xyz, max xyz, then left ref, right ref, left count, right count as
 * uint32 bits; count 0 = internal node ref, else first triangle ref),
 * triangles = 12 floats each (v0 xyz, 0, e1 = v1 - v0 xyz, 0, e2 = v2 - v0
 * xyz, 0) in leaf order, source = the selected triangle each came from. */
int dr_build_occluder_bvh(const dr_surface *surfaces, uint32_t n_surfaces, uint32_t mode, float *nodes,
                          uint32_t *n_nodes, float *triangles, uint32_t *source, uint32_t *n_triangles);

/* ---- render settings: RenderKernel::Initialize (src/kernel.cpp:497-534) ---- */
int dr_set_params(dr_ctx *ctx, const dr_render_params *params);

/* Hosek-Wilkie state cook (src/ArHosekSkyModel.cpp:147-339) from the RGB
 * dataset supplied by the caller: dataset_rgb[c] holds 2*10*6*9 doubles and
 * dataset_rad[c] 2*10*6 doubles per channel c. */
int dr_sky_cook(const double *const dataset_rgb[3], const double *const dataset_rad[3], double turbidity,
                double albedo, double elevation, double configs[3][9], double radiances[3]);

/* ---- render: RenderKernel::Render (src/kernel.cpp:536-567) ---------------- */
/* Renders tile (x0, y0, tw, th) with spp samples per pixel and writes the SUMS
 * over those samples into sun_out (phb[0]) and sky_out (phb[1]), tw*th float4
 * each.  As in the reference only the even part of an odd tile is rendered
 * (2x2 pixel blocks); pixels outside the image or not rendered are 0.
 * Path (pixel p = py*w + px, sample s) draws from stream (seed, p, sample_base + s).
 * Blocking; host buffers.  Returns DR_ERR_GAVE_UP, with the tiles written,
 * when some of the call's paths were cut short by an iteration budget (the
 * reference has no budget: it renders every path to its end).  Large tiles
 * are copied into the caller's buffers by up to 7 host threads of the context,
 * started on the first such copy and joined by dr_destroy. */
int dr_render_tile(dr_ctx *ctx, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed,
                   uint64_t sample_base, float *sun_out, float *sky_out);
/* Same on device buffers, enqueued on stream (NULL = context stream); returns
 * without waiting. */
int dr_render_tile_async(dr_ctx *ctx, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp,
                         uint64_t seed, uint64_t sample_base, float *sun_out_dev, float *sky_out_dev, void *stream);
/* ---- shadow pass: RenderKernel::Shadow (src/kernel.cpp:569-607) ----------
 * For each pixel of the tile whose depth-texture value lies before the far clip
 * plane, spp shadow segments run from that point towards sun-cone samples; out
 * (phb[0], tw*th float4) receives per pixel the SUM over samples of
 * sun(lrd)/colour for segments that escape (pixels without such geometry count
 * every sample as lit).  Alpha is +inf, as in the reference (its division by
 * float4::load(&colour) has w = 0).  Sample s of pixel p draws from stream
 * (seed, p, sample_base + s).  Blocking; host buffer; DR_ERR_GAVE_UP as for
 * dr_render_tile. */
int dr_shadow_tile(dr_ctx *ctx, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp, uint64_t seed,
                   uint64_t sample_base, float *out);
int dr_shadow_tile_async(dr_ctx *ctx, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp,
                         uint64_t seed, uint64_t sample_base, float *out_dev, void *stream);

/* Waits for all work on the context stream. */
int dr_synchronize(dr_ctx *ctx);

/* Give-up report for the calls that return before their work ends
 * (dr_render_tile_async, dr_shadow_tile_async, dr_batch_launch,
 * dr_adjoint_tile_async, ...).  Waits for `stream` (NULL = the context stream)
 * and the context stream, then returns DR_ERR_GAVE_UP if the context's
 * gave_up counter rose since the previous check (or dr_reset_counters), i.e.
 * some path segment hit the tracking-step budget or some block timed out
 * staging its tables; the outputs are then incomplete.  Give-ups that a
 * blocking call already reported are not reported again.  No reference
 * counterpart: the reference has no budgets. */
int dr_check_complete(dr_ctx *ctx, void *stream);

/* Tracking steps (null collisions) a path segment may take before it gives up
 * (0 = the default, 2^24).  Applies to the context's parameters and to batches
 * created afterwards.  No reference counterpart (the reference loops until
 * the segment ends); a small budget makes give-ups reproducible in tests. */
int dr_set_step_budget(dr_ctx *ctx, uint32_t steps);

/* Camera leaf lists of the persistent kernel: before a launch, each pixel's
 * camera ray is traversed once and its samples read the leaf sequence instead
 * of traversing (every sample of a pixel shares its camera ray).  Results and
 * counters are the same with or without them.  pool_entries: entries of 16
 * bytes per list pool (0 = the default 2^23; DR_NONE = no lists); the pixels
 * whose lists do not fit traverse.  Applies to later renders of the context.
 * No reference counterpart (the reference traverses per sample). */
int dr_set_camera_lists(dr_ctx *ctx, uint32_t pool_entries);

/* ---- launch shape (no reference counterpart: the reference schedules 2x2
 * pixel blocks with TBB, src/kernel.cpp:453) ------------------------------- */
#define DR_KERNEL_PERSISTENT 0u  /* resident warps take paths from a queue (default) */
#define DR_KERNEL_PER_PATH 1u    /* one thread per path sample */
typedef struct {
    uint32_t kernel;         /* DR_KERNEL_* */
    uint32_t blocks_per_sm;  /* persistent kernel: resident blocks per SM, 0 = as many as fit */
    uint32_t event_batch;    /* persistent kernel: waiting lanes before a warp shades (1..32, 0 = 8) */
    uint32_t traversal;      /* persistent kernel: DR_TRAVERSAL_* */
    uint32_t tile;           /* persistent kernel: pixel order in tile x tile squares, 0 = row-major (<= 64) */
    uint32_t visits;         /* persistent kernel, stack traversal: node examinations per iteration, 0 = to the
                                next leaf (<= 255) */
    uint32_t steps;          /* persistent kernel: free-flight steps per iteration, 0 = 1 (<= 255) */
} dr_tuning;
#define DR_TRAVERSAL_STACK 0u  /* octree descent with a node stack (the reference's order) */
#define DR_TRAVERSAL_WALK 1u   /* cell walk over the leaf grid, same leaf order and intervals */
#define DR_TRAVERSAL_STACK_SHARED 2u  /* the octree descent with its stack in shared memory (frames and batches
                                         without optional features whose octrees keep every leaf at one depth
                                         <= 8 and have fewer than 2^25 nodes; otherwise DR_TRAVERSAL_STACK) */
int dr_set_tuning(dr_ctx *ctx, const dr_tuning *tuning);
int dr_get_tuning(dr_ctx *ctx, dr_tuning *tuning);

/* ---- batched rendering (no reference counterpart: the reference renders one
 * tile of one view per RenderKernel::Render call, src/kernel.cpp:536-567) ----
 * A batch holds several scenes and views and renders every view's spp new
 * samples in ONE launch of a CUDA graph: a persistent kernel over the views
 * (large views may get kernels of their own, dr_batch_set_split).  Launch k of a
 * batch renders, for each view, the samples dr_render_tile would render with
 * sample_base = k * spp; outputs hold the sums of the last launch. */
typedef struct dr_batch dr_batch;
typedef struct {
    uint32_t scene;                  /* index into the scenes given to dr_batch_create */
    const dr_render_params *params;  /* settings of this view; phase tables and mode equal across views */
    uint32_t x0, y0, tw, th;         /* region of the view's image */
    uint32_t spp;                    /* samples per pixel per launch */
    uint64_t seed;                   /* path streams (seed, pixel, sample) as in dr_render_tile */
} dr_batch_view;
/* Uploads every scene, copies every view's settings (and depth texture) and
 * captures the launch graph with the context's tuning (kernel forced to
 * DR_KERNEL_PERSISTENT).  Counters accumulate into the context's. */
int dr_batch_create(dr_ctx *ctx, const dr_scene_desc *scenes, uint32_t n_scenes, const dr_batch_view *views,
                    uint32_t n_views, dr_batch **out);
int dr_batch_destroy(dr_batch *batch);
/* Re-lays the views out and recaptures the graph for another launch shape
 * (waits for the device first: launches may run on any stream). */
int dr_batch_set_tuning(dr_batch *batch, const dr_tuning *tuning);
int dr_batch_get_tuning(dr_batch *batch, dr_tuning *tuning);
/* Enqueues one graph launch on stream (NULL = the context stream). */
int dr_batch_launch(dr_batch *batch, void *stream);
/* Device pointers of a view's output tiles (tw*th float4 each; sums of the last launch). */
int dr_batch_output(dr_batch *batch, uint32_t view, float **sun_dev, float **sky_dev);
/* Waits for the device and copies a view's output tiles to the host. */
int dr_batch_read(dr_batch *batch, uint32_t view, float *sun_out, float *sky_out);
/* Path indices per launch (tile padding included) and launches so far. */
int dr_batch_info(dr_batch *batch, uint64_t *n_paths, uint64_t *launches);
/* Views of at least min_paths path samples per launch (cols*rows*spp) get a
 * persistent kernel of their own in the batch's graph, with their parameters
 * as kernel arguments; those kernels and the one batched kernel over the other
 * views are independent graph branches (up to 4 run side by side), so one
 * kernel's tail overlaps the next one's start.  Results are unchanged (same
 * paths and streams).  min_paths 0: every view in the one batched kernel;
 * DR_BATCH_SPLIT_AUTO (the default): 8 paths per lane of a full grid
 * (SMs x blocks per SM x 128).  Waits for the device, then recaptures the graph. */
#define DR_BATCH_SPLIT_AUTO UINT64_MAX
int dr_batch_set_split(dr_batch *batch, uint64_t min_paths);
/* The split setting and how many views have a kernel of their own in the
 * current graph (either pointer may be NULL). */
int dr_batch_get_split(dr_batch *batch, uint64_t *min_paths, uint32_t *own_kernels);

/* ---- differentiable rendering (path-replay adjoint) -------------------------
 * No reference counterpart: the reference renders only (src/kernel.cpp).
 * The parameters are the brick samples (n_leaves * 512 floats, the scene's
 * FOG pool) and the single-scatter albedo sigma_s / (sigma_s + sigma_a). */
/* Replaces the scene's brick pool with a device array (device-to-device copy).
 * majorant_scale >= 1 recomputes every leaf majorant as majorant_scale x the
 * brick maximum, floor 0.01 (1: the reference's rule, src/scene.cpp:889-904;
 * leaves whose majorant is 0 keep 0); 0 keeps the current majorants, which
 * must then bound the new samples. */
int dr_set_bricks_dev(dr_ctx *ctx, const float *bricks_dev, uint32_t n_leaves, float majorant_scale, void *stream);
/* Majorant of every node (0 for internal nodes), host buffer of n_nodes floats. */
int dr_get_majorants(dr_ctx *ctx, float *out);
/* Path-replay adjoint of dr_render_tile(_async) with the same arguments:
 * given dsun_dev / dsky_dev = dL/d(tile sums) (tw*th float4 each, rgb used),
 * ADDS dL/d(brick sample) into grad_bricks_dev (n_leaves * 512 floats) and
 * dL/d(albedo) into *grad_albedo_dev.  Each path is replayed from its own
 * random stream (no stored tape): unbiased for the expected image, with the
 * leaf majorants held fixed.  A path whose contribution is not finite is
 * left out.  Enqueued on stream (NULL = context stream). */
int dr_adjoint_tile_async(dr_ctx *ctx, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp,
                          uint64_t seed, uint64_t sample_base, const float *dsun_dev, const float *dsky_dev,
                          float *grad_bricks_dev, double *grad_albedo_dev, void *stream);
/* Gradient check of dr_adjoint_tile_async: replays the same paths with every
 * delta-tracking decision drawn from the context's bricks and weighted by its
 * probability under pert_bricks_dev (n_leaves * 512 floats, same majorants)
 * over its probability under the context's bricks, and ADDS the linearised
 * loss  sum over paths of dsun . C_sun + dsky . C_sky  (dsun / dsky as in the
 * adjoint) into *loss_dev.  Unbiased for the loss of the perturbed field and
 * smooth in the perturbation: central differences of it with common random
 * numbers estimate the gradient the adjoint returns.  With pert_bricks_dev =
 * the context's bricks it is the plain estimator's loss.  Enqueued on stream
 * (NULL = context stream). */
int dr_reweighted_loss_async(dr_ctx *ctx, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th, uint32_t spp,
                             uint64_t seed, uint64_t sample_base, const float *dsun_dev, const float *dsky_dev,
                             const float *pert_bricks_dev, double *loss_dev, void *stream);
/* Transmittance of n rays (ro, rd: 3n floats) by delta tracking over nsamp
 * samples (streams (seed, ray, sample)) and the gradient of
 * sum_r weights[r] * T_r with respect to the brick samples (host buffers:
 * grad_bricks n_leaves * 512 floats, transmittance n doubles or NULL). */
int dr_adjoint_transmittance(dr_ctx *ctx, const float *ro, const float *rd, const float *weights, uint32_t n,
                             uint64_t nsamp, uint64_t seed, float *grad_bricks, double *transmittance);

/* ---- counters ------------------------------------------------------------ */
int dr_get_counters(dr_ctx *ctx, dr_counters *out);
int dr_reset_counters(dr_ctx *ctx);

/* ---- parity probes (test support; they run the same device code) --------- */
/* Leaf sequence of one ray: node ids and (tr0, tr1); returns the count in *n.
 * src/KernelOctree.cpp:230-349. */
int dr_probe_leaf_sequence(dr_ctx *ctx, const float *ro, const float *rd, uint32_t n_rays, uint32_t maxn,
                           uint32_t *nodes, float *tr0, float *tr1, uint32_t *counts);
/* SampleVoxelSpace at n points inside leaf nodes[i] (src/kernel.cpp:96-126). */
int dr_probe_density(dr_ctx *ctx, const uint32_t *nodes, const float *points, uint32_t n, float *out);
/* Occluder any-hit of n rays (ro, rd: 3n floats): hit[i] = 1 when the ray hits
 * an occluder triangle at t in [0, 1e6]. */
int dr_probe_occlusion(dr_ctx *ctx, const float *ro, const float *rd, uint32_t n, uint32_t *hit);
/* Per-path sample (sun rgba, sky rgba) for n (px, py, sample) triples. */
int dr_probe_paths(dr_ctx *ctx, const uint32_t *px, const uint32_t *py, const uint64_t *sample, uint32_t n,
                   uint64_t seed, float *out_sun, float *out_sky);
/* Phase / sun / sky evaluations for n directions (see DR_PROBE_*). */
#define DR_PROBE_MIE_EVAL_RGB 0u   /* in: ct[n]            out: 3n */
#define DR_PROBE_MIE_SAMPLE 1u     /* in: iv[3n],u1[n],u2[n] out: 3n */
#define DR_PROBE_SUN_SAMPLE 2u     /* in: u1[n],u2[n]      out: 3n */
#define DR_PROBE_SKY 3u            /* in: rd[3n]           out: 3n */
#define DR_PROBE_MIE_THETA 4u      /* in: u1[n]            out: n (theta / pi) */
#define DR_PROBE_MIE_EXACT_DIR 5u  /* in: u1[n]            out: 2n (ct, st) of the exact sampler */
#define DR_PROBE_HG_EVAL 6u        /* in: ct[n]            out: n  (HGPhase::Evaluate) */
#define DR_PROBE_HG_SAMPLE 7u      /* in: iv[3n],u1[n],u2[n] out: 3n */
#define DR_PROBE_SKY_LIGHT 8u      /* in: rd[3n]           out: 3n (light of an escaping ray, per env_mode) */
#define DR_PROBE_ENV_MAP 9u        /* in: rd[3n]           out: 3n (MapEnv::Evaluate, before the 2.2 power) */
int dr_probe_sampler(dr_ctx *ctx, uint32_t what, const float *in, uint32_t n, float *out);
/* Fraction of nsamp delta-tracked segments along each ray that escape. */
int dr_probe_transmittance(dr_ctx *ctx, const float *ro, const float *rd, uint32_t n_rays, uint64_t nsamp,
                           uint64_t seed, double *out);

/* ---- transmittance for callers that cannot allocate ------------------------
 * This entry point has no counterpart in the reference.  It serves callers that
 * cannot let this library allocate device memory.  One example is an
 * application that owns the GPU's memory budget, such as a host renderer
 * sharing the device.  Another is a caller whose other streams cannot afford
 * the device-wide synchronisation that cudaMalloc and cudaFree can cause.
 *
 * The call allocates nothing.  The caller passes device buffers for the rays
 * (ro_dev and rd_dev, 3 floats per ray) and for the result (out_dev, one double
 * per ray).  The result is the fraction of nsamp delta-tracked segments that
 * escape, drawn from the same streams as dr_probe_transmittance.
 *
 * The per-ray counters live in a fixed device array of DR_NOALLOC_MAX_RAYS
 * entries (512 KB).  Every GPU that loads the library holds it until the
 * process exits.  Larger batches are rejected with DR_ERR_INVALID.
 *
 * The first call on a device looks up the array's address and caches it, so
 * make that first call before any stream capture.  The cached address belongs
 * to the device's primary context: do not reset the device (cudaDeviceReset,
 * or a primary-context reset by the application) while the library is loaded.
 * All calls share the array, so calls that overlap on the GPU race.
 *
 * The work is enqueued on `stream` (NULL = the context stream) and the call
 * returns without waiting. */
#define DR_NOALLOC_MAX_RAYS 65536u
int dr_transmittance_noalloc(dr_ctx *ctx, const float *ro_dev, const float *rd_dev, uint32_t n_rays, uint64_t nsamp,
                             uint64_t seed, double *out_dev, void *stream);

#ifdef __cplusplus
}
#endif
#endif
