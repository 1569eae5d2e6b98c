/* ORACLE TEST INFRASTRUCTURE — not product code.
 *
 * Drives the reference renderer (src/kernel.cpp RenderKernel, compiled
 * unmodified) on a scene whose octree and 8^3 bricks are supplied by the
 * caller, because the reference's own scene build (src/scene.cpp) needs
 * OpenVDB, which is absent.  Only what the hot path links against is defined
 * here: DebugPrintf (src/main.cpp:28-41), the OctreeStructure/Scene/Octree
 * constructors (src/scene.cpp:249-262, 817-823) and BaseLight::lights setup
 * as done by DRE_BeginRender (src/main.cpp:374-404).
 *
 * Node records are the reference's OctreeStructure layout (src/scene.h:21-31):
 * float ce[4]; uint chn[8]; uint volx[2]; float qval[2]  (64 bytes).
 */
#include "main.h"
#include "scene.h"
#include "SceneOcclusion.h"
#include "kernel.h"
#include "KernelOctree.h"
#include "KernelSampler.h"
#include "ArHosekSkyModel.h"

#include <cstring>
#include <vector>
#include <cstdio>
#include <cstdarg>
#include <cmath>

extern "C" int dr_tbbshim_threads = 1;

void DebugPrintf(const char *pfmt, ...) {
    if (!getenv("DR_ORACLE_VERBOSE")) return;
    va_list args;
    va_start(args, pfmt);
    vprintf(pfmt, args);
    va_end(args);
}

OctreeStructure::OctreeStructure() {
    for (uint i = 0; i < VOLUME_BUFFER_COUNT; ++i) volx[i] = ~0u;
    memset(chn, 0, sizeof(chn));
    qval[0] = qval[1] = 0.0f;
}
OctreeStructure::~OctreeStructure() {}
Octree::Octree(uint _x) : x(_x) { memset(pch, 0, sizeof(pch)); }
Octree::Octree() : x(0) { memset(pch, 0, sizeof(pch)); }
Octree::~Octree() {}
Scene::Scene() {}
Scene::~Scene() {}

static_assert(sizeof(OctreeStructure) == 64, "reference node layout must be 64 bytes");

extern "C" void ref_set_threads(int n) { dr_tbbshim_threads = n; }

extern "C" void *ref_scene_create(const void *nodes, unsigned n_nodes, const float *fog_bricks,
                                  unsigned n_fog_leaves, unsigned lvoxc) {
    Scene *s = new Scene();
    s->ob.resize(n_nodes);
    std::memcpy(&s->ob[0], nodes, (size_t)n_nodes * 64);
    s->lvoxc = lvoxc;
    s->lvoxc3 = lvoxc * lvoxc * lvoxc;
    s->index = n_nodes;
    s->leafx[VOLUME_BUFFER_SDF] = 0;
    s->leafx[VOLUME_BUFFER_FOG] = n_fog_leaves;
    s->pvol[VOLUME_BUFFER_SDF] = new float[1];
    s->pvol[VOLUME_BUFFER_FOG] = new float[(size_t)n_fog_leaves * s->lvoxc3 + 1];
    std::memcpy(s->pvol[VOLUME_BUFFER_FOG], fog_bricks, (size_t)n_fog_leaves * s->lvoxc3 * sizeof(float));
    return s;
}

/* As ref_scene_create, with the surface pool Scene::pvol[VOLUME_BUFFER_SDF]
 * (n_sdf_leaves bricks) for nodes whose volx[VOLUME_BUFFER_SDF] is set. */
extern "C" void *ref_scene_create_sdf(const void *nodes, unsigned n_nodes, const float *fog_bricks,
                                      unsigned n_fog_leaves, const float *sdf_bricks, unsigned n_sdf_leaves,
                                      unsigned lvoxc) {
    Scene *s = (Scene *)ref_scene_create(nodes, n_nodes, fog_bricks, n_fog_leaves, lvoxc);
    delete[] s->pvol[VOLUME_BUFFER_SDF];
    s->leafx[VOLUME_BUFFER_SDF] = n_sdf_leaves;
    s->pvol[VOLUME_BUFFER_SDF] = new float[(size_t)n_sdf_leaves * s->lvoxc3 + 1];
    std::memcpy(s->pvol[VOLUME_BUFFER_SDF], sdf_bricks, (size_t)n_sdf_leaves * s->lvoxc3 * sizeof(float));
    return s;
}

extern "C" void ref_scene_destroy(void *p) {
    Scene *s = (Scene *)p;
    delete[] s->pvol[0];
    delete[] s->pvol[1];
    delete s;
}

/* Leaf sequence of one ray through the reference traversers
 * (src/KernelOctree.cpp:128-220 full, 230-349 step).  Returns the count. */
extern "C" unsigned ref_leaf_sequence(void *p, int full, const float ro[3], const float rd[3], unsigned maxn,
                                      unsigned *nodes, float *tr0, float *tr1) {
    Scene *s = (Scene *)p;
    sfloat4 RO, RD;
    for (int k = 0; k < 3; ++k) {
        RO.v[k] = sfloat1(ro[k], 0.0f, 0.0f, 0.0f);
        RD.v[k] = sfloat1(rd[k], 1.0f, 1.0f, 1.0f);
    }
    RO.v[3] = sfloat1::zero();
    RD.v[3] = sfloat1::zero();
    sint1 gm(-1, 0, 0, 0);
    KernelOctree::OctreeFullTraverser ft;
    KernelOctree::OctreeStepTraverser st;
    KernelOctree::BaseOctreeTraverser *t = full ? (KernelOctree::BaseOctreeTraverser *)&ft : &st;
    t->Initialize(RO, RD, gm, &s->ob);
    unsigned n = 0;
    for (unsigned i = 0; n < maxn; ++i) {
        duintN nn;
        sfloat1 a, b;
        dintN m = t->GetLeaf(i, &nn, a, b);
        if (m.v[0] == 0) break;
        nodes[n] = nn.v[0];
        tr0[n] = a.get<0>();
        tr1[n] = b.get<0>();
        ++n;
    }
    return n;
}

/* Cooked Hosek-Wilkie RGB state (src/ArHosekSkyModel.cpp:306-339). */
extern "C" void ref_sky_state(double turbidity, double albedo, double elevation, double *configs27,
                              double *radiances3) {
    ArHosekSkyModelState *st = arhosek_rgb_skymodelstate_alloc_init(turbidity, albedo, elevation);
    for (int c = 0; c < 3; ++c) {
        for (int j = 0; j < 9; ++j) configs27[9 * c + j] = st->configs[c][j];
        radiances3[c] = st->radiances[c];
    }
    arhosekskymodelstate_free(st);
}

/* Solar elevation exactly as RenderKernel::Initialize derives it (src/kernel.cpp:522-524). */
extern "C" float ref_solar_elevation(const float sun_dir[3]) {
    float th = acosf(sun_dir[2]);
    return XM_PIDIV2 - th;
}

/* One RenderKernel::Render call (src/kernel.cpp:536-567) over a tile, with the
 * Hosek state re-cooked for (turbidity, albedo) in place of the hard-coded
 * (7, 0.15) of src/kernel.cpp:525.  Outputs are the two tile buffers phb[0]
 * (sun) and phb[1] (sky) as float4 per pixel, row-major in the tile; pixels the
 * reference leaves unwritten (outside the frame, odd last row/column) are 0. */
struct PhaseEnv {
    int phase;               /* 0 MiePhase, 2 HGPhase */
    float g;                 /* HGPhase::g1 */
    unsigned env_w, env_h;   /* MapEnv texels (0: NullEnv) */
    const float *env_rgba;
};

static int ref_run(void *p, const float viewi[16], const float proji[16], const float sun_dir[3],
                   const float sun_color[3], float sun_angle, double turbidity, double albedo, unsigned scattevs,
                   float sigma_s, float sigma_a, unsigned w, unsigned h, unsigned x0, unsigned y0, unsigned tw,
                   unsigned th, unsigned spp, const float *depth, unsigned flags, int shadow, float *out_sun,
                   float *out_sky, const PhaseEnv &pe = PhaseEnv{0, 0.0f, 0, 0, 0}) {
    Scene *s = (Scene *)p;
    KernelSampler::BaseLight::DeleteAll();
    dfloat3 D(sun_dir[0], sun_dir[1], sun_dir[2]);
    dfloat3 C(sun_color[0], sun_color[1], sun_color[2]);
    new KernelSampler::SunLight(&D, &C, sun_angle);

    dmatrix44 vi, pi;
    for (int r = 0; r < 4; ++r) {
        vi.r[r] = dfloat4(viewi[4 * r + 0], viewi[4 * r + 1], viewi[4 * r + 2], viewi[4 * r + 3]);
        pi.r[r] = dfloat4(proji[4 * r + 0], proji[4 * r + 1], proji[4 * r + 2], proji[4 * r + 3]);
    }
    std::vector<float> dcopy;
    if (depth) dcopy.assign(depth, depth + (size_t)w * h);
    /* phase function and environment as DRE_BeginRender selects them (src/main.cpp:522-587) */
    KernelSampler::PhaseFunction *ppf = &KernelSampler::MiePhase::gmie;
    if (pe.phase == 2) {
        KernelSampler::HGPhase::ghg.g1 = pe.g;
        ppf = &KernelSampler::HGPhase::ghg;
    }
    KernelSampler::BaseEnv *penv = &KernelSampler::NullEnv::nenv;
    if (pe.env_w) {
        dfloat4 *t = KernelSampler::MapEnv::genv.Initialize(pe.env_w, pe.env_h);
        std::memcpy((void *)t, pe.env_rgba, (size_t)pe.env_w * pe.env_h * 16);
        penv = &KernelSampler::MapEnv::genv;
    }
    RenderKernel k;
    if (!k.Initialize(s, 0, &vi, &pi, ppf, penv, depth ? dcopy.data() : 0, scattevs, sigma_s, sigma_a, tw, th, w, h,
                      flags))
        return -1;
#ifdef USE_ARHOSEK_SKYMODEL
    arhosekskymodelstate_free(k.pskyms);
    float se = ref_solar_elevation(sun_dir);
    k.pskyms = arhosek_rgb_skymodelstate_alloc_init(turbidity, albedo, se);
#endif
    std::memset(k.phb[0], 0, (size_t)tw * th * 16);
    std::memset(k.phb[1], 0, (size_t)tw * th * 16);
    if (shadow)
        k.Shadow(x0, y0, tw, th, spp);
    else
        k.Render(x0, y0, tw, th, spp);
    std::memcpy(out_sun, k.phb[0], (size_t)tw * th * 16);
    if (out_sky) std::memcpy(out_sky, k.phb[1], (size_t)tw * th * 16);
    k.Destroy();
    if (pe.env_w) KernelSampler::MapEnv::genv.Destroy();  // as DRE_EndRender does (src/main.cpp:691-693)
    KernelSampler::BaseLight::DeleteAll();
    return 0;
}

/* RenderKernel::Render over one tile (src/kernel.cpp:536-567); depth (w*h or
 * NULL) and flags (KERNEL_DEPTHCOMP) as RenderKernel::Initialize takes them. */
extern "C" int ref_render(void *p, const float viewi[16], const float proji[16], const float sun_dir[3],
                          const float sun_color[3], float sun_angle, double turbidity, double albedo,
                          unsigned scattevs, float sigma_s, float sigma_a, unsigned w, unsigned h, unsigned x0,
                          unsigned y0, unsigned tw, unsigned th, unsigned spp, float *out_sun, float *out_sky,
                          const float *depth, unsigned flags) {
    return ref_run(p, viewi, proji, sun_dir, sun_color, sun_angle, turbidity, albedo, scattevs, sigma_s, sigma_a, w,
                   h, x0, y0, tw, th, spp, depth, flags, 0, out_sun, out_sky);
}

/* ref_render with the phase function (0 Mie, 2 HG with anisotropy g) and the
 * environment (env_w == 0: NullEnv, else a MapEnv of env_w x env_h RGBA
 * texels) chosen as DRE_BeginRender does; the environment is read only by the
 * build without USE_ARHOSEK_SKYMODEL. */
extern "C" int ref_render_ex(void *p, const float viewi[16], const float proji[16], const float sun_dir[3],
                             const float sun_color[3], float sun_angle, double turbidity, double albedo,
                             unsigned scattevs, float sigma_s, float sigma_a, unsigned w, unsigned h, unsigned x0,
                             unsigned y0, unsigned tw, unsigned th, unsigned spp, float *out_sun, float *out_sky,
                             const float *depth, unsigned flags, int phase, float g, unsigned env_w, unsigned env_h,
                             const float *env_rgba) {
    const PhaseEnv pe{phase, g, env_w, env_h, env_rgba};
    return ref_run(p, viewi, proji, sun_dir, sun_color, sun_angle, turbidity, albedo, scattevs, sigma_s, sigma_a, w,
                   h, x0, y0, tw, th, spp, depth, flags, 0, out_sun, out_sky, pe);
}

/* Whether this library is the reference built with USE_ARHOSEK_SKYMODEL. */
extern "C" int ref_has_hosek(void) {
#ifdef USE_ARHOSEK_SKYMODEL
    return 1;
#else
    return 0;
#endif
}

/* RenderKernel::Shadow over one tile (src/kernel.cpp:569-607): phb[0] only. */
extern "C" int ref_shadow(void *p, const float viewi[16], const float proji[16], const float sun_dir[3],
                          const float sun_color[3], float sun_angle, unsigned scattevs, float sigma_s, float sigma_a,
                          unsigned w, unsigned h, unsigned x0, unsigned y0, unsigned tw, unsigned th, unsigned spp,
                          const float *depth, float *out) {
    return ref_run(p, viewi, proji, sun_dir, sun_color, sun_angle, 3.0, 0.3, scattevs, sigma_s, sigma_a, w, h, x0,
                   y0, tw, th, spp, depth, 0, 1, out, 0);
}
