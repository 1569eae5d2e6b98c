/* ORACLE TEST INFRASTRUCTURE — CPU restatement of droplet-render's volumetric
 * path-tracing hot path.  Only tests, the smoke check and the CPU-baseline leg
 * of the benchmark may load it; the product never links it.
 *
 * Every function cites the reference file:line it restates.  Octree traversal,
 * leaf indexing and brick lookups repeat the reference's binary32 operations in
 * the same order; the estimator is the reference's (src/kernel.cpp:128-445)
 * written as a loop, drawing from a per-path PCG32 stream instead of the
 * reference's thread-order-seeded packet Tausworthe generator.
 */
#ifndef DR_ORACLE_H
#define DR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NONE 0xffffffffu
#define ORC_SDF 0
#define ORC_FOG 1
#define ORC_MAX_DEPTH 16

/* src/scene.h:21-31 OctreeStructure, 64 bytes. */
typedef struct {
    float ce[4];        /* center.xyz, half extent */
    uint32_t chn[8];    /* child node index, 0 = none; child i offset (i&1, i>>1&1, i>>2) */
    uint32_t volx[2];   /* brick index per buffer or ORC_NONE */
    float qval[2];      /* per-leaf majorant (FOG: max density, floor 0.01) */
} orc_node;

typedef struct {
    const orc_node *nodes;
    uint32_t n_nodes;
    const float *bricks;   /* FOG bricks, lvoxc^3 floats each, z-major then y then x */
    uint32_t n_leaves;
    uint32_t lvoxc;
    /* occluder triangles (SceneOcclusion's Embree scene, src/SceneOcclusion.cpp:19-56),
     * 12 floats each: v0 xyz, 0, e1 = v1 - v0 xyz, 0, e2 = v2 - v0 xyz, 0; tested one by one */
    const float *occ_tris;
    uint32_t occ_n;
    /* surface bricks (Scene::pvol[VOLUME_BUFFER_SDF]) of leaves with volx[ORC_SDF] set, or NULL */
    const float *sdf_bricks;
} orc_scene;

typedef struct {
    /* medium */
    float sigma_s, sigma_a;
    uint32_t scattevs;
    /* sun: src/KernelSampler.cpp:305-345 */
    float sun_dir[3], sun_color[3], sun_cos_angle;
    /* Hosek sky, as the reference kernel consumes it (binary32 copies of the
     * cooked double state, src/kernel.cpp:343-358) */
    float sky_cfg[3][9], sky_rad[3];
    /* Mie tables: 256 RGB entries each, index 0 = backscatter */
    const float *mie_pdf, *mie_cdf;
    uint32_t mie_n;
    /* camera: rows r[0..3] of the inverse view / projection matrices */
    float viewi[16], proji[16];
    uint32_t w, h;
    float depth;           /* compositing depth of every camera ray (FLT_MAX when unused) */
    /* per-pixel depth texture, w*h row-major, or NULL (src/kernel.cpp:548-554, 579-585) */
    const float *depth_map;
    uint32_t depthcomp;    /* KERNEL_DEPTHCOMP: camera rays stop at depth_map */
    uint32_t phase_mode;   /* 0 = the reference's sampler, 1 = exact inverse CDF */
    const float *mie_exact;/* exact-mode table (orc_mie_exact_table), 8 n + 4 floats */
    uint32_t finite_paths; /* a path whose sun or sky sum is not finite adds nothing */
    uint32_t embree;       /* the reference built with USE_EMBREE (src/kernel.cpp:149-153, 375-383) */
    float hg_g;            /* phase_mode 2: HGPhase::g1 */
    uint32_t env_mode;     /* 0 Hosek sky, 1 NullEnv, 2 MapEnv */
    const float *env_map;  /* env_mode 2: env_w * env_h RGBA floats, row-major */
    uint32_t env_w, env_h;
} orc_params;

typedef struct {
    uint64_t vertices;       /* traced segments: camera, continuation and shadow */
    uint64_t node_visits;    /* octree node records examined by the traverser */
    uint64_t density_lookups;/* trilinear brick lookups */
    uint64_t mie_evals;      /* phase table evaluations + phase samples */
    uint64_t paths;
} orc_counters;

/* ---- scene build: src/scene.cpp:267-305, 676-762, 840-908 ---------------- */
/* Sparse input in the shape of OpenVDB leaves: n_blocks blocks of 8^3 values
 * (x fastest within a block's z-major order), block origins in voxel units
 * (multiples of 8).  Voxel (i,j,k) sits at world (i,j,k)*s; a voxel is active
 * iff its value is non-zero.  Returns 0 on success. */
int orc_build_octree(const int32_t *block_origin, const float *block_values, uint32_t n_blocks, float s,
                     uint32_t maxdepth, orc_node **out_nodes, uint32_t *n_nodes, float **out_bricks,
                     uint32_t *n_leaves, uint32_t *out_lvoxc, uint32_t *out_mlevel);
void orc_free(void *p);

/* ---- traversal: src/KernelOctree.cpp ------------------------------------- */
uint32_t orc_leaf_sequence(const orc_node *nodes, const float ro[3], const float rd[3], uint32_t maxn,
                           uint32_t *out_nodes, float *out_tr0, float *out_tr1);
/* FP64 point location: the leaf whose box contains p, descending by
 * child bit (p > center) per axis, src/scene.cpp:285 numbering.  Returns the
 * node index or ORC_NONE; *depth receives the level reached. */
uint32_t orc_point_lookup(const orc_node *nodes, const double p[3], int *depth);

/* ---- samplers ------------------------------------------------------------ */
float orc_sample_voxel_space(const float p[3], const float *brick, const float ce[4], uint32_t lvoxc);
void orc_mie_eval_rgb(const orc_params *P, float ct, float out[3]);
float orc_mie_eval(const orc_params *P, float ct);
float orc_mie_sample_theta_scan(const orc_params *P, float u1);   /* reference linear scan */
float orc_mie_sample_theta_bisect(const orc_params *P, float u1); /* same bin by bisection */
void orc_mie_sample(const orc_params *P, const float iv[3], float u1, float u2, float out[3]);
/* exact-mode sampler: table from the red pdf column, direction of a sample */
void orc_mie_exact_table(const float *pdf_rgb, uint32_t n, float *out);
void orc_mie_exact_dir(const float *tab, uint32_t n, float u1, float *ct, float *st);
void orc_mie_exact_dirs(const float *tab, uint32_t n, const float *u1, uint32_t count, float *ct, float *st);
void orc_mie_sample_exact(const orc_params *P, const float iv[3], float u1, float u2, float out[3]);
/* HGPhase (src/KernelSampler.cpp:164-204) */
float orc_hg_eval(float g, float ct);
void orc_hg_sample(float g, const float iv[3], float u1, float u2, float out[3]);
/* the reference's polynomial atan2 (src/smmath.inl:430-445) */
float orc_atan2_ref(float y, float x);
/* MapEnv::Evaluate (src/KernelSampler.cpp:384-417), before the 2.2 power */
void orc_env_map_eval(const orc_params *P, const float rd[3], float out[3]);
/* light of an escaping ray: the Hosek sky, or pow(environment, 2.2) (src/kernel.cpp:329-364) */
void orc_sky_light(const orc_params *P, const float rd[3], float out[3]);
/* phase function of the path: Mie (either sampler) or HG */
void orc_phase_eval_rgb(const orc_params *P, float ct, float out[3]);
void orc_phase_sample(const orc_params *P, const float iv[3], float u1, float u2, float out[3]);
void orc_sun_eval(const orc_params *P, const float rd[3], float out[3]);
float orc_sun_pdf(const orc_params *P, const float v[3]);
void orc_sun_sample(const orc_params *P, float u1, float u2, float out[3]);
void orc_sky_eval(const orc_params *P, const float rd[3], float out[3]);
void orc_camera_ray(const orc_params *P, uint32_t px, uint32_t py, float ro[3], float rd[3], int *in_frame);

/* ---- FP64 checks --------------------------------------------------------- */
/* Optical depth integral of the brick density along ro + t rd, t in [0, tmax],
 * leaf by leaf, exact Gauss-Legendre on every brick-cell segment. */
double orc_optical_depth(const orc_scene *S, const double ro[3], const double rd[3], double tmax);
/* FP64 quadrature of the single-scatter (scattevs = 1) sun image and its
 * brick gradient: the adjoint's independent check (fp64.c). */
void orc_single_scatter_sun(const orc_scene *S, const orc_params *P, const float *ro, const float *rd, uint32_t n_rays,
                            double p_hit, uint32_t nu, uint32_t nphi, const double wc[3], double *out, double *grad);
double orc_sun_hit_fraction(const orc_params *P, uint32_t n1, uint32_t n2);
void orc_math_eval(int kind, const float *x, uint32_t n, float *out);

/* ---- estimator ----------------------------------------------------------- */
/* Free-flight tracking of one segment (src/kernel.cpp:197-317, fog leaves).
 * Returns 1 when the ray leaves the volume without a real collision. */
int orc_track(const orc_scene *S, const orc_params *P, const float ro[3], const float rd[3], void *rng,
              float *td, orc_counters *cnt);
/* One tile of RenderKernel::Render (src/kernel.cpp:447-487, 536-567): sums of
 * spp path samples per pixel into out_sun/out_sky (float4, row-major tile).
 * Path (pixel p = py*w + px, sample s) draws from PCG32 stream
 * (seed, p, sample_base + s). */
int orc_render_tile(const orc_scene *S, const orc_params *P, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th,
                    uint32_t spp, uint64_t seed, uint64_t sample_base, float *out_sun, float *out_sky,
                    orc_counters *cnt);
/* A single path sample, for per-path comparisons. */
/* One tile of RenderKernel::Shadow (src/kernel.cpp:569-607): per pixel, the
 * sum over spp sun-direction samples of the shadow-segment result divided by
 * the sun colour, from the point at the pixel's depth along the camera ray.
 * Sample s of pixel p draws from PCG32 stream (seed, p, sample_base + s). */
int orc_shadow_tile_mt(const orc_scene *S, const orc_params *P, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th,
                       uint32_t spp, uint64_t seed, uint64_t sample_base, float *out, orc_counters *cnt,
                       int nthreads);
void orc_shadow_path(const orc_scene *S, const orc_params *P, uint32_t px, uint32_t py, uint64_t seed,
                     uint64_t sample, float out[4], orc_counters *cnt);
/* Path-replay adjoint of orc_render_tile (the GPU adjoint's algorithm):
 * adds dL/d(brick sample) to grad (doubles) and dL/d(albedo) to *galb for
 * dsun/dsky = dL/d(tile sums) (tw*th float4). */
int orc_adjoint_tile_mt(const orc_scene *S, const orc_params *P, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th,
                        uint32_t spp, uint64_t seed, uint64_t sample_base, const float *dsun, const float *dsky,
                        double *grad, double *galb, int nthreads);
/* Occlusion query of SceneOcclusion::Intersect (t in [0, 1e6], any triangle):
 * binary32 Moller-Trumbore, the GPU's arithmetic, over every triangle. */
int orc_occluded(const orc_scene *S, const float o[3], const float d[3]);
/* Origin and direction of the shadow pass's segment for one (pixel, sample);
 * returns 1 when the pixel traces one (geometry before the far plane). */
int orc_shadow_ray(const orc_params *P, uint32_t px, uint32_t py, uint64_t seed, uint64_t sample, float ro1[3],
                   float lrd[3]);
/* The same test in FP64 with the division by the determinant; *margin receives
 * the smallest of u, v, 1 - u - v of the nearest hit candidate (how far the
 * answer is from an edge), for pinning the binary32 test. */
int orc_occluded_fp64(const orc_scene *S, const double o[3], const double d[3], double *margin);
/* Linearised loss of the reweighted replay (decisions from S->bricks, ratios under pert). */
double orc_reweighted_loss(const orc_scene *S, const orc_params *P, uint32_t x0, uint32_t y0, uint32_t tw, uint32_t th,
                           uint32_t spp, uint64_t seed, uint64_t sample_base, const float *dsun, const float *dsky,
                           const float *pert);
/* Gradient of sum_r w_r T_r (delta-tracking transmittance over nsamp samples). */
void orc_adjoint_transmittance(const orc_scene *S, const orc_params *P, const float *ro, const float *rd,
                               const float *wr, uint32_t n, uint64_t nsamp, uint64_t seed, double *grad, double *T);
void orc_render_path(const orc_scene *S, const orc_params *P, uint32_t px, uint32_t py, uint64_t seed,
                     uint64_t sample, float out_sun[4], float out_sky[4], orc_counters *cnt);

#ifdef __cplusplus
}
#endif
#endif
