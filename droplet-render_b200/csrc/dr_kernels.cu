// Kernels of the droplet_b200 hot path and their launchers.
#include <cstdio>
#include <mutex>
#include <cuda_runtime.h>
#include "dr_device.cuh"
#include "dr_kernels.h"

namespace dr {

// ---- shared-memory staging of the phase tables ------------------------------
// Layout in global and shared memory: pdf as float4 (r, g, b, 0) x n, then the
// red CDF x n (n % 4 == 0, so the block is a multiple of 16 bytes).  One thread
// issues a bulk copy (cp.async.bulk, completion counted on an mbarrier); the
// wait is bounded and reports a give-up instead of spinning forever.
// Exact mode appends its sampler table: (2n + 1) float4 after the CDF.
__device__ __forceinline__ uint32_t mie_bytes(const DevParams &P) {
    return P.mie_n * 20u + (P.phase_mode == 1u ? (2u * P.mie_n + 1u) * 16u : 0u);
}

__device__ __forceinline__ MieSmem mie_view(const DevParams &P, unsigned char *smem) {
    return MieSmem{reinterpret_cast<float4 *>(smem), reinterpret_cast<float *>(smem + 16u * P.mie_n), P.mie_n,
                   P.phase_mode == 1u ? reinterpret_cast<const float4 *>(smem + 20u * P.mie_n) : nullptr};
}

__device__ __forceinline__ bool stage_mie(const void *src, uint32_t bytes, unsigned char *smem, uint64_t *mbar) {
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(mbar);
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(smem);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
            "l"(src), "r"(bytes), "r"(bar)
            : "memory");
    }
    uint32_t done = 0;
    for (uint32_t it = 0; it < (1u << 22) && !done; ++it) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar)
            : "memory");
    }
    return done != 0;
}

__device__ __forceinline__ void warp_sum_counts(Count &c, DevCounters *C, uint32_t paths) {
    const uint32_t full = 0xffffffffu;
    uint32_t v = __reduce_add_sync(full, c.vertices);
    uint32_t nv = __reduce_add_sync(full, c.node_visits);
    uint32_t dl = __reduce_add_sync(full, c.density_lookups);
    uint32_t me = __reduce_add_sync(full, c.mie_evals);
    uint32_t gu = __reduce_add_sync(full, c.gave_up);
    uint32_t pa = __reduce_add_sync(full, paths);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&C->vertices, (unsigned long long)v);
        atomicAdd(&C->node_visits, (unsigned long long)nv);
        atomicAdd(&C->density_lookups, (unsigned long long)dl);
        atomicAdd(&C->mie_evals, (unsigned long long)me);
        if (gu) atomicAdd(&C->gave_up, (unsigned long long)gu);
        atomicAdd(&C->paths, (unsigned long long)pa);
    }
}

__device__ __forceinline__ float4 shfl_xor4(float4 v, int m) {
    v.x = __shfl_xor_sync(0xffffffffu, v.x, m);
    v.y = __shfl_xor_sync(0xffffffffu, v.y, m);
    v.z = __shfl_xor_sync(0xffffffffu, v.z, m);
    v.w = __shfl_xor_sync(0xffffffffu, v.w, m);
    return v;
}

__device__ __forceinline__ float4 add4(float4 a, float4 b) {
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

// One thread per (pixel, sample) path; thread g renders pixel g / spp, sample
// g % spp, so a warp holds 32 consecutive samples of a pixel when spp % 32 == 0
// and reduces them with a fixed shuffle tree before one float4 atomic.
template <uint32_t FEAT>
__global__ void __launch_bounds__(kRenderBlock) render_tile_kernel(DevScene S, DevParams P, TileArgs A,
                                                                   const void *mie_pack, float4 *sun_out,
                                                                   float4 *sky_out, DevCounters *C) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t mbar;
    const bool staged = stage_mie(mie_pack, mie_bytes(P), smem, &mbar);
    const MieSmem M = mie_view(P, smem);
    Count cnt;
    cnt.zero();
    uint32_t nstack[kMaxDepth];
    const uint64_t g = (uint64_t)blockIdx.x * kRenderBlock + threadIdx.x;
    const bool valid = staged && g < A.n_paths;
    float4 sa = make_float4(0.f, 0.f, 0.f, 0.f), sk = sa;
    uint32_t pix = 0xffffffffu, paths = 0;
    if (valid) {
        const uint64_t pl = g / A.spp;
        const uint32_t s = (uint32_t)(g - pl * A.spp);
        pix = (uint32_t)pl;
        const uint32_t i = pix % A.cols, j = pix / A.cols;
        float ro[3], rd[3];
        if (camera_ray(P, A.x0 + i, A.y0 + j, ro, rd)) {
            paths = 1;
            path_sample<FEAT>(S, P, M, A.x0 + i, A.y0 + j, A.seed, A.sample_base + s, sa, sk, nstack, cnt);
        }
    }
    if (!staged) cnt.gave_up += (g < A.n_paths) ? 1u : 0u;
    const uint32_t grp = __match_any_sync(0xffffffffu, pix);
    if (grp == 0xffffffffu) {
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) {
            sa = add4(sa, shfl_xor4(sa, m));
            sk = add4(sk, shfl_xor4(sk, m));
        }
        if ((threadIdx.x & 31) == 0 && valid) {
            const uint32_t i = pix % A.cols, j = pix / A.cols;
            const size_t o = (size_t)j * A.tw + i;
            atomicAdd(&sun_out[o], sa);
            atomicAdd(&sky_out[o], sk);
        }
    } else if (valid) {
        const uint32_t i = pix % A.cols, j = pix / A.cols;
        const size_t o = (size_t)j * A.tw + i;
        atomicAdd(&sun_out[o], sa);
        atomicAdd(&sky_out[o], sk);
    }
    warp_sum_counts(cnt, C, paths);
}

// Shadow pass (RenderKernel::Shadow, src/kernel.cpp:569-607): one thread per
// (pixel, sample), same pixel/sample layout and warp reduction as the render
// kernel; the result goes to one tile (the reference writes phb[0] only).
__global__ void __launch_bounds__(kRenderBlock) shadow_tile_kernel(DevScene S, DevParams P, TileArgs A, float4 *out,
                                                                   DevCounters *C) {
    Count cnt;
    cnt.zero();
    uint32_t nstack[kMaxDepth];
    const uint64_t g = (uint64_t)blockIdx.x * kRenderBlock + threadIdx.x;
    const bool valid = g < A.n_paths;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    uint32_t pix = 0xffffffffu, paths = 0;
    if (valid) {
        const uint64_t pl = g / A.spp;
        const uint32_t s = (uint32_t)(g - pl * A.spp);
        pix = (uint32_t)pl;
        const uint32_t i = pix % A.cols, j = pix / A.cols;
        float ro[3], rd[3];
        if (camera_ray(P, A.x0 + i, A.y0 + j, ro, rd)) {
            paths = 1;
            acc = shadow_sample(S, P, A.x0 + i, A.y0 + j, A.seed, A.sample_base + s, ro, rd, nstack, cnt);
        } else {
            pix = 0xfffffffeu;  // outside the frame: nothing is written, as in the reference
        }
    }
    const uint32_t grp = __match_any_sync(0xffffffffu, pix);
    if (grp == 0xffffffffu) {
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) acc = add4(acc, shfl_xor4(acc, m));
        if ((threadIdx.x & 31) == 0 && pix < 0xfffffffeu) {
            const uint32_t i = pix % A.cols, j = pix / A.cols;
            atomicAdd(&out[(size_t)j * A.tw + i], acc);
        }
    } else if (pix < 0xfffffffeu) {
        const uint32_t i = pix % A.cols, j = pix / A.cols;
        atomicAdd(&out[(size_t)j * A.tw + i], acc);
    }
    warp_sum_counts(cnt, C, paths);
}

// ---- persistent path kernel ------------------------------------------------------
// Each lane of a resident warp holds one path sample as a small state machine
// and takes the next path from a global counter as soon as its path ends, so
// lanes never idle behind a warp-mate's long path.  One loop iteration does
// one unit of work per lane:
//   kTrav  advance the octree traversal to the next leaf (then fall into kStep)
//   kStep  one free-flight step of delta tracking inside the current leaf
//   kEvent a segment ended (escape or collision): shade, start the next segment
// Events are the long, divergent part (phase/sun sampling, sky radiance); a
// warp runs them only when at least `event_batch` of its lanes wait on one, or
// when nothing else is left, so the common tracking step stays converged.
// Per path, the operations and random draws are those of path_sample()/track():
// a path's result is bit-identical to the one-thread-per-path kernel.
enum : uint32_t { kFetch = 0, kTrav = 1, kStep = 2, kEvent = 3, kDone = 4 };
// Segment result of a path that escaped after scattering and left its sky term
// to the warp's sky queue (the loop enqueues it after the event pass).
constexpr uint32_t kTrackDeferSky = 3;
// Per warp in dynamic shared memory: 32 sky terms, 7 words each (rd.xyz,
// T.xyz, output offset; the batch adds the view), stored word-major so a
// lane's slot is one column.
template <bool BATCH> __host__ __device__ constexpr uint32_t sky_queue_words() { return (BATCH ? 8u : 7u) * 32u; }
enum : uint32_t { kSegMain = 0, kSegShadow = 1 };

template <bool WALK> struct SegTrav;
template <> struct SegTrav<true> { Walk w; };
template <> struct SegTrav<false> { Trav t; };

// PathLane::wmode of a camera segment that reads its pixel's leaf list
constexpr uint32_t kWalkListed = 4;

template <bool WALK>
struct PathLane {
    // path
    uint32_t px, py;
    Rng g;
    float ro[3], rd[3];
    float T[3];
    float4 sun, sky;
    uint32_t r, seg;
    float srd[3], tn[3], sw[3];  // pending continuation while the shadow segment runs
    // segment
    SegTrav<WALK> st;
    uint32_t wmode;  // 0 no leaf on the ray, 1 cell walk, 2 stack traversal in local memory, 3 stack traversal,
                     // 4 (kWalkListed) the pixel's camera leaf list
    float td, depth;
    uint32_t budget;
    uint32_t esc;  // segment result: kTrackCollided, kTrackEscaped or kTrackCut
    // leaf
    float lo, tr0, tr1, trb, s0, sr, smax, denom;
    float4 ce;
    const float *brick;
    const float *sdf;  // surface brick of an SDF leaf (kFeatSdf instantiations), else null
};

// Stack traversal for the rare segments the cell walk does not take (a zero
// direction component).  Its state lives in local memory; arguments and results
// travel by value so that no lane state has its address taken.
struct SlowLeaf {
    uint32_t ok, leaf, visits;
    float tra, trb;
};

__device__ __noinline__ uint32_t slow_init(Trav *T, DevScene S, float ox, float oy, float oz, float dx, float dy,
                                           float dz) {
    const float o[3] = {ox, oy, oz}, d[3] = {dx, dy, dz};
    Count c;
    c.zero();
    trav_init(*T, S, o, d, c);
    return c.node_visits;
}

__device__ __noinline__ SlowLeaf slow_next(Trav *T, DevScene S, uint32_t *nstack) {
    SlowLeaf r;
    Count c;
    c.zero();
    r.leaf = 0;
    r.tra = r.trb = 0.0f;
    r.ok = trav_next(*T, S, nstack, r.leaf, r.tra, r.trb, c) ? 1u : 0u;
    r.visits = c.node_visits;
    return r;
}

template <bool WALK>
__device__ __forceinline__ void begin_segment(PathLane<WALK> &L, const DevScene &S, uint32_t budget, Count &cnt,
                                              uint32_t &state, Trav *slow) {
    if constexpr (WALK) {
        L.wmode = walk_init(L.st.w, S, L.ro, L.rd, cnt);
        if (L.wmode == 2u)
            cnt.node_visits += slow_init(slow, S, L.ro[0], L.ro[1], L.ro[2], L.rd[0], L.rd[1], L.rd[2]);
    } else {
        trav_init(L.st.t, S, L.ro, L.rd, cnt);
        L.wmode = L.st.t.active ? 3u : 0u;
    }
    ++cnt.vertices;
    L.td = 0.0f;
    L.budget = budget;
    state = kTrav;
}

template <bool WALK>
__device__ __forceinline__ void finish_path(PathLane<WALK> &L, const DevParams &P, const TileArgs &A, float4 *sun_out,
                                            float4 *sky_out) {
    drop_nonfinite(P, L.sun, L.sky);
    const bool any = (L.sun.x != 0.0f) | (L.sun.y != 0.0f) | (L.sun.z != 0.0f) | (L.sun.w != 0.0f) |
                     (L.sky.x != 0.0f) | (L.sky.y != 0.0f) | (L.sky.z != 0.0f) | (L.sky.w != 0.0f);
    if (any) {
        const size_t o = (size_t)(L.py - A.y0) * A.tw + (L.px - A.x0);
        atomicAdd(&sun_out[o], L.sun);
        atomicAdd(&sky_out[o], L.sky);
    }
}

// One traversal step.  Returns 0 after moving to another cell (call again), 1
// when a leaf was entered and its free flight prepared, 2 when the segment has
// no further leaf (or the depth mask stops it): the segment escaped.
// SHS: the traversal stack lives in shared memory (column shcol, shlevels
// entries) instead of the lane's local arrays nstack / tstack.
template <bool WALK, uint32_t FEAT, bool SHS>
__device__ __forceinline__ uint32_t trav_step(PathLane<WALK> &L, const DevScene &S, const DevParams &P,
                                              const uint4 *cam_pool, uint32_t *nstack, Trav *slow, Count &cnt,
                                              uint32_t visits, float (*tstack)[6], float *shcol, int shlevels) {
    uint32_t leaf = 0;
    float tra = 0.0f, trb = 0.0f;
    uint32_t r;
    if constexpr (!WALK) {
        // at most `visits` examinations per loop iteration (0: up to the next leaf)
        const uint32_t budget = visits ? visits : 0xffffffffu;
        if (L.wmode == kWalkListed) {
            // camera segment: the next leaf of the pixel's list (node = next
            // entry, l = entries left, tn = node visits after the last leaf)
            if (L.st.t.l > 0) {
                const uint4 e = __ldg(&cam_pool[L.st.t.node]);
                ++L.st.t.node;
                --L.st.t.l;
                leaf = e.x;
                tra = __uint_as_float(e.y);
                trb = __uint_as_float(e.z);
                cnt.node_visits += e.w;
                r = kTravLeaf;
            } else {
                cnt.node_visits += L.st.t.tn;
                L.st.t.tn = 0;
                r = kTravDone;
            }
        } else if constexpr (SHS)
            r = L.wmode == 3u ? trav_next_s(L.st.t, S, SharedStack<kPersistentBlock>{shcol, shlevels}, leaf, tra,
                                            trb, cnt, budget)
                              : kTravDone;
        else
            r = L.wmode == 3u ? trav_next_k(L.st.t, S, nstack, leaf, tra, trb, cnt, budget, tstack) : kTravDone;
    } else if (L.wmode == 1u) {
        r = walk_step(L.st.w, S, leaf, tra, trb, cnt);
    } else if (L.wmode == 2u) {
        const SlowLeaf sl = slow_next(slow, S, nstack);
        cnt.node_visits += sl.visits;
        r = sl.ok ? 1u : 2u;
        leaf = sl.leaf;
        tra = sl.tra;
        trb = sl.trb;
    } else {
        r = 2u;
    }
    if (r != 1u) return r;
    if (!(L.td < L.depth)) return 2u;
    L.ce = __ldg(&S.leaf[2 * leaf]);
    const float4 meta = __ldg(&S.leaf[2 * leaf + 1]);
    L.smax = meta.x;
    L.brick = S.bricks + (size_t)__float_as_uint(meta.y) * kBrick;
    L.lo = L.td;
    L.tr0 = tra - L.td;
    L.tr1 = trb - L.td;
    L.trb = trb;
    bool sdf_leaf = false;
    if constexpr ((FEAT & kFeatSdf) != 0) {
        const uint32_t sdfx = __float_as_uint(meta.z);
        sdf_leaf = sdfx != kNone;
        L.sdf = sdf_leaf ? S.sdf_bricks + (size_t)sdfx * kBrick : nullptr;
        if (__float_as_uint(meta.y) == kNone) L.brick = nullptr;  // a surface leaf without fog
    }
    if (sdf_leaf) {
        // src/kernel.cpp:253-263: entered only when before it and outside the surface there
        bool skip = false;
        if (tra > L.td) {
            const float r0[3] = {L.ro[0] + L.rd[0] * tra, L.ro[1] + L.rd[1] * tra, L.ro[2] + L.rd[2] * tra};
            skip = sample_voxel_space(r0, L.sdf, L.ce) > 0.0f;
            ++cnt.density_lookups;
        }
        if (skip) {
            L.td = tra;
            L.s0 = L.tr0;
        } else {
            L.s0 = 0.0f;
        }
    } else if (tra > L.td) {
        L.td = tra;
        L.s0 = L.tr0;
    } else {
        L.td = __uint_as_float((__float_as_uint(L.td) & ~1u) | (__float_as_uint(tra) & 1u));
        L.s0 = __uint_as_float(__float_as_uint(L.tr0) & 1u);
    }
    L.denom = P.sigma_e * L.smax;
    // the first free-flight distance is drawn by the first track_step:
    // 0 - l/d equals -l/d here (l < 0), and the draw order is unchanged
    L.sr = 0.0f;
    return 1u;
}

// One delta-tracking step: draws the next free-flight distance, then tests
// it.  Returns 0 = continue in this leaf, 1 = leaf left, 2 = segment ended
// (collision, or the step budget ran out).  Drawing at the start of a step
// rather than at the end of the previous one (or at leaf entry) consumes the
// same stream in the same order, and lets lanes that just entered a leaf draw
// together with lanes already tracking.
template <bool WALK, uint32_t FEAT>
__device__ __forceinline__ uint32_t track_step(PathLane<WALK> &L, Count &cnt) {
    L.sr = L.sr - dlog(L.g.uniform()) / L.denom;
    const float sc = L.s0 + L.sr;
    L.td = L.lo + sc;
    if (!(sc < L.tr1)) {
        L.td = L.trb;
        return 1;
    }
    bool rm = sc > L.tr0;
    float rho = -1.0f, dist = 1.0f;
    if (rm) {
        const float rc[3] = {L.ro[0] + L.rd[0] * L.td, L.ro[1] + L.rd[1] * L.td, L.ro[2] + L.rd[2] * L.td};
        if ((FEAT & kFeatSdf) && L.sdf) {
            // src/kernel.cpp:287-300: inside the surface always collides
            dist = sample_voxel_space(rc, L.sdf, L.ce);
            ++cnt.density_lookups;
            if (dist > 0.0f && L.brick) {
                rho = sample_voxel_space(rc, L.brick, L.ce);
                ++cnt.density_lookups;
            }
        } else {
            rho = sample_voxel_space(rc, L.brick, L.ce);
            ++cnt.density_lookups;
        }
    }
    const float q = L.g.uniform();
    rm = rm && (rho / L.smax < q) && (dist > 0.0f);
    if (!rm) {
        L.esc = L.td < L.depth ? kTrackCollided : kTrackCut;
        return 2;
    }
    if (--L.budget == 0) {
        ++cnt.gave_up;
        L.esc = kTrackEscaped;
        return 2;
    }
    return 0;
}

// The end of a main segment: light gathered on escape, the path finished at a
// cut or the event limit (state becomes kFetch), or a scattering event that
// sets up the shadow segment and the pending continuation.
template <bool WALK, uint32_t FEAT>
__device__ __forceinline__ void scatter_event(PathLane<WALK> &L, const DevScene &S, const DevParams &P,
                                              const MieSmem &M, const TileArgs &A, float4 *sun_out, float4 *sky_out,
                                              Count &cnt, uint32_t &state) {
    const float f = P.albedo;
    if (L.r == 0) L.sun.w = L.sky.w = first_alpha(P, L.esc);
    if (L.esc == kTrackEscaped) {
        if (L.r > 0 && !((FEAT & kFeatOcc) && occluded(S, L.ro, L.rd))) {
            if (sun_hit(P, L.rd)) {
                L.sun.x = L.sun.x + L.T[0] * P.sun_color[0];
                L.sun.y = L.sun.y + L.T[1] * P.sun_color[1];
                L.sun.z = L.sun.z + L.T[2] * P.sun_color[2];
            } else {
                L.sun.x = L.sun.x + L.T[0] * 0.0f;
                L.sun.y = L.sun.y + L.T[1] * 0.0f;
                L.sun.z = L.sun.z + L.T[2] * 0.0f;
            }
            if (FEAT == 0 && A.defer_sky) {
                // the sky term, T * sky(rd) (the path's sky sum is 0 until this
                // escape), goes to the warp's sky queue after the event pass
                L.esc = kTrackDeferSky;
            } else {
                const float3 sky = escape_sky<FEAT>(P, L.rd);
                L.sky.x = L.sky.x + L.T[0] * sky.x;
                L.sky.y = L.sky.y + L.T[1] * sky.y;
                L.sky.z = L.sky.z + L.T[2] * sky.z;
            }
        }
    }
    // one store for escaped, cut and last-event paths alike
    if (L.esc == kTrackEscaped || L.esc == kTrackDeferSky || L.esc == kTrackCut || L.r >= P.scattevs) {
        finish_path(L, P, A, sun_out, sky_out);
        state = kFetch;
        return;
    }
    float lrd[3];
    const float u1 = L.g.uniform(), u2 = L.g.uniform();
    if constexpr ((FEAT & kFeatExt) != 0) phase_sample(P, M, L.rd, u1, u2, L.srd);
    else mie_sample(M, L.rd, u1, u2, L.srd);
    const float u3 = L.g.uniform(), u4 = L.g.uniform();
    sun_sample(P, u3, u4, lrd);
    const float3 p1 = (FEAT & kFeatExt) ? phase_eval_rgb(P, M, dot3(L.srd, L.rd)) : mie_eval_rgb(M, dot3(L.srd, L.rd));
    const float p2 = sun_hit(P, lrd) ? P.sun_pdf : 0.0f;
    const float3 p3 = (FEAT & kFeatExt) ? phase_eval_rgb(P, M, dot3(lrd, L.rd)) : mie_eval_rgb(M, dot3(lrd, L.rd));
    const float q1 = sun_hit(P, L.srd) ? P.sun_pdf : 0.0f;
    cnt.mie_evals += 3;
    L.sw[0] = L.T[0] * ((p3.x / (p3.x + p2)) * f);
    L.sw[1] = L.T[1] * ((p3.y / (p3.y + p2)) * f);
    L.sw[2] = L.T[2] * ((p3.z / (p3.z + p2)) * f);
    L.tn[0] = L.T[0] * ((p1.x / (p1.x + q1)) * f);
    L.tn[1] = L.T[1] * ((p1.y / (p1.y + q1)) * f);
    L.tn[2] = L.T[2] * ((p1.z / (p1.z + q1)) * f);
    for (int k = 0; k < 3; ++k) {
        L.ro[k] = L.ro[k] + L.rd[k] * L.td;
        L.rd[k] = lrd[k];
    }
    L.seg = kSegShadow;
}

// Segment end: the body of path_sample() between two track() calls.
template <bool WALK, uint32_t FEAT>
__device__ __forceinline__ void path_event(PathLane<WALK> &L, const DevScene &S, const DevParams &P, const MieSmem &M,
                                        const TileArgs &A, float4 *sun_out, float4 *sky_out, Count &cnt,
                                        uint32_t &state, Trav *slow) {
    if (L.seg == kSegShadow) {
        if (L.esc == kTrackEscaped && !((FEAT & kFeatOcc) && occluded(S, L.ro, L.rd))) {
            const bool hit = sun_hit(P, L.rd);
            const float s0 = hit ? P.sun_color[0] : 0.0f, s1 = hit ? P.sun_color[1] : 0.0f,
                        s2 = hit ? P.sun_color[2] : 0.0f;
            L.sun.x = L.sun.x + L.sw[0] * s0;
            L.sun.y = L.sun.y + L.sw[1] * s1;
            L.sun.z = L.sun.z + L.sw[2] * s2;
        }
        for (int k = 0; k < 3; ++k) {
            L.T[k] = L.tn[k];
            L.rd[k] = L.srd[k];
        }
        L.r += 1;
        L.seg = kSegMain;
    } else {
        scatter_event<WALK, FEAT>(L, S, P, M, A, sun_out, sky_out, cnt, state);
        if (state == kFetch) return;
    }
    // one segment start for both kinds of event, so that lanes of a batch that
    // ended a shadow segment and lanes that scattered run it together
    L.depth = 3.402823466e+38f;
    begin_segment(L, S, P.step_budget, cnt, state, slow);
}

// Starts path number p; returns false when p lies outside the frame (no work).
// Path index p -> (pixel, sample): samples of a pixel are consecutive; pixels
// run row-major, or square by square (tile x tile, row-major inside) when
// A.tile > 0, where indices of pixels past the tile's edge carry no work.
template <bool WALK>
__device__ __forceinline__ bool start_path(PathLane<WALK> &L, uint64_t p, const DevScene &S, const DevParams &P,
                                           const TileArgs &A, uint64_t shift, Count &cnt, uint32_t &paths,
                                           uint32_t &state, Trav *slow) {
    uint32_t pix, s;
    if (p <= 0xffffffffull) {  // multiply-high divisions (FastDiv) instead of 64-bit division
        const uint32_t p32 = (uint32_t)p;
        pix = fastdiv(p32, A.spp_div);
        s = p32 - pix * A.spp;
    } else {
        const uint64_t pl = p / A.spp;
        s = (uint32_t)(p - pl * A.spp);
        pix = (uint32_t)pl;
    }
    uint32_t ix, iy;
    if (A.tile) {
        const uint32_t sq = fastdiv(pix, A.t2_div), r = pix - sq * (A.tile * A.tile);
        const uint32_t sy = fastdiv(sq, A.tx_div), ry = fastdiv(r, A.tile_div);
        ix = (sq - sy * A.tiles_x) * A.tile + (r - ry * A.tile);
        iy = sy * A.tile + ry;
        if (ix >= A.cols || iy >= A.rows) return false;
    } else {
        iy = fastdiv(pix, A.cols_div);
        ix = pix - iy * A.cols;
    }
    L.px = A.x0 + ix;
    L.py = A.y0 + iy;
    // the pixel's header (leaf list and camera ray, every sample of the pixel
    // shares them), or none: the ray is generated and the segment traverses
    uint4 h = make_uint4(kNone, 0u, 0u, 0u);
    if constexpr (!WALK) {
        if (A.cam_head) {
            const size_t hx = 2 * ((size_t)iy * A.cols + ix);
            h = __ldg(&A.cam_head[hx]);
            const uint4 ray = __ldg(&A.cam_head[hx + 1]);
            if (!ray.w) return false;
            for (int k = 0; k < 3; ++k) L.ro[k] = P.viewi[12 + k];  // camera_ray's origin
            L.rd[0] = __uint_as_float(ray.x);
            L.rd[1] = __uint_as_float(ray.y);
            L.rd[2] = __uint_as_float(ray.z);
        } else if (!camera_ray(P, L.px, L.py, L.ro, L.rd)) {
            return false;
        }
    } else {
        if (!camera_ray(P, L.px, L.py, L.ro, L.rd)) return false;
    }
    ++paths;
    L.T[0] = L.T[1] = L.T[2] = 1.0f;
    L.sun = make_float4(0.f, 0.f, 0.f, 0.f);
    L.sky = L.sun;
    L.r = 0;
    L.seg = kSegMain;
    L.depth = (P.depth && P.depthcomp) ? __ldg(&P.depth[(size_t)L.py * P.w + L.px]) : 3.402823466e+38f;
    bool listed = false;
    if constexpr (!WALK) {
        if (h.x != kNone) {
            // the pixel's camera leaf list: what trav_init and the traversal
            // would find, node visits included (h.z = 1: the root test passed)
            ++cnt.vertices;
            cnt.node_visits += h.z;
            L.wmode = h.z ? kWalkListed : 0u;
            L.st.t.node = h.x;
            L.st.t.l = (int)h.y;
            L.st.t.tn = h.w;
            L.td = 0.0f;
            L.budget = P.step_budget;
            state = kTrav;
            listed = true;
        }
    }
    if (!listed) begin_segment(L, S, P.step_budget, cnt, state, slow);
    // A camera ray that misses the root box draws no random number: its
    // sample is exactly zero.  Seed the stream only for rays that enter.
    if (L.wmode != 0u) L.g = rng_seed(A.seed, (uint64_t)L.py * P.w + L.px, A.sample_base + shift + s);
    return true;
}

// One loop iteration of a lane that holds a path (see render_persistent_kernel).
template <bool WALK, uint32_t FEAT, bool SHS>
__device__ __forceinline__ void lane_work(PathLane<WALK> &L, bool events, const DevScene &S, const DevParams &P,
                                          const MieSmem &M, const TileArgs &A, float4 *sun_out, float4 *sky_out,
                                          Count &cnt, uint32_t &state, uint32_t *nstack, Trav *slow, uint32_t visits,
                                          uint32_t steps, float (*tstack)[6], float *shcol, int shlevels) {
    if (events) {
        if (state == kEvent) path_event<WALK, FEAT>(L, S, P, M, A, sun_out, sky_out, cnt, state, slow);
        return;
    }
    if (state == kTrav) {
        const uint32_t r =
            trav_step<WALK, FEAT, SHS>(L, S, P, A.cam_pool, nstack, slow, cnt, visits, tstack, shcol, shlevels);
        if (r == 1u) {
            state = kStep;
        } else if (r == 2u) {
            L.esc = kTrackEscaped;
            state = kEvent;
        }
    }
    // up to `steps` free-flight steps while the lane stays in its leaf
    for (uint32_t k = 0; k < steps && state == kStep; ++k) {
        const uint32_t rs = track_step<WALK, FEAT>(L, cnt);
        if (rs == 1) state = kTrav;
        else if (rs == 2) state = kEvent;
    }
}

// The sky terms of a persistent launch are evaluated by full warps: after an
// event pass, the lanes whose path escaped with its sky term deferred append
// (rd, T, pixel[, view]) to the warp's queue (q: sky_queue_words floats, nq
// entries, warp-uniform); whenever it holds 32, every lane evaluates one,
// T * sky(rd), and adds it to the pixel.  That is the value the path would
// have added in place (its sky sum is 0 before the escape); the pixel's total
// differs only in the order of the float additions, as between any two runs.
template <bool BATCH>
__device__ __forceinline__ void sky_queue_eval(const DevParams &P, float4 *sky_out, const BatchArgs &B, const float *q,
                                               uint32_t lane) {
    const float rd[3] = {q[lane], q[32 + lane], q[64 + lane]};
    const uint32_t off = __float_as_uint(q[192 + lane]);
    float3 sky;
    float4 *out;
    if constexpr (BATCH) {
        const BatchView &V = B.views[__float_as_uint(q[224 + lane])];
        sky = escape_sky<0>(V.P, rd);
        out = V.sky;
    } else {
        sky = escape_sky<0>(P, rd);
        out = sky_out;
    }
    atomicAdd(&out[off], make_float4(q[96 + lane] * sky.x, q[128 + lane] * sky.y, q[160 + lane] * sky.z, 0.0f));
}

template <bool BATCH, bool WALK>
__device__ __forceinline__ void sky_queue_put(float *q, uint32_t slot, const PathLane<WALK> &L, const TileArgs &A,
                                              uint32_t view) {
    q[slot] = L.rd[0];
    q[32 + slot] = L.rd[1];
    q[64 + slot] = L.rd[2];
    q[96 + slot] = L.T[0];
    q[128 + slot] = L.T[1];
    q[160 + slot] = L.T[2];
    q[192 + slot] = __uint_as_float((L.py - A.y0) * A.tw + (L.px - A.x0));
    if constexpr (BATCH) q[224 + slot] = __uint_as_float(view);
}

// Called by the whole warp after an event pass; A and view are the lane's.
template <bool BATCH, bool WALK>
__device__ __forceinline__ void sky_queue_push(PathLane<WALK> &L, const TileArgs &A, uint32_t view,
                                               const DevParams &P, float4 *sky_out, const BatchArgs &B, float *q,
                                               uint32_t &nq, uint32_t lane, uint32_t lt_mask) {
    const bool mine = L.esc == kTrackDeferSky;
    const uint32_t dm = __ballot_sync(0xffffffffu, mine);
    if (!dm) return;
    const uint32_t pos = nq + __popc(dm & lt_mask);
    const uint32_t total = nq + __popc(dm);
    if (mine) {
        L.esc = kTrackEscaped;
        if (pos < 32u) sky_queue_put<BATCH>(q, pos, L, A, view);
    }
    if (total < 32u) {
        nq = total;
        return;
    }
    __syncwarp();
    sky_queue_eval<BATCH>(P, sky_out, B, q, lane);
    __syncwarp();
    if (mine && pos >= 32u) sky_queue_put<BATCH>(q, pos - 32u, L, A, view);
    nq = total - 32u;
}

// The rest of the queue (whole warp, after its last path).
template <bool BATCH>
__device__ __forceinline__ void sky_queue_flush(const DevParams &P, float4 *sky_out, const BatchArgs &B,
                                                const float *q, uint32_t nq, uint32_t lane) {
    __syncwarp();
    if (lane < nq) sky_queue_eval<BATCH>(P, sky_out, B, q, lane);
}

// View owning global path index p: the last v with begins[v] <= p.
__device__ __forceinline__ uint32_t find_view(const BatchArgs &B, uint64_t p) {
    uint32_t lo = 0, hi = B.n_views - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&B.begins[mid]) <= p) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// BATCH: the paths of many views (each with its own scene, parameters, tile
// and output) share one work queue; a lane looks its view up when it fetches
// a path and reads that view's records from global memory (L1-resident).
// SHS (stack traversal only): the traversal stack of each lane lives in
// dynamic shared memory after the phase tables, `knobs` bits 24-31 entries
// deep (kShWords words per entry and lane), instead of local memory.
template <int MINB, bool WALK, bool BATCH, uint32_t FEAT, bool SHS = false>
__global__ void __launch_bounds__(kPersistentBlock, MINB) render_persistent_kernel(DevScene S, DevParams P, TileArgs A,
                                                                            const void *mie_pack, float4 *sun_out,
                                                                            float4 *sky_out, DevCounters *C,
                                                                            WorkQueue *Q, uint32_t knobs,
                                                                            BatchArgs B) {
    // knobs: bits 0-7 the event batch, bits 8-15 the traversal visits per
    // iteration (0: to the next leaf), bits 16-23 the tracking steps per iteration
    const uint32_t event_batch = knobs & 0xffu, visits = (knobs >> 8) & 0xffu;
    const uint32_t steps = ((knobs >> 16) & 0xffu) ? ((knobs >> 16) & 0xffu) : 1u;
    const int shlevels = (int)(knobs >> 24);
    static_assert(!(SHS && WALK), "the shared-memory stack serves the stack traversal");
    float ts[kMaxDepth][6];  // ancestors' intervals of the stack traversal (local memory)
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t mbar;
    uint32_t mb;
    MieSmem M;
    uint64_t n_total, shift = 0;
    if constexpr (BATCH) {
        mb = mie_bytes(B.views[0].P);
        M = mie_view(B.views[0].P, smem);
        n_total = B.n_paths;
        shift = *B.step;
    } else {
        mb = mie_bytes(P);
        M = mie_view(P, smem);
        n_total = A.n_paths;
        // a large view of a batch, as a kernel of its own in the batch's graph:
        // launch k draws samples [k spp, (k+1) spp) like the batched kernel
        if (B.step) shift = *B.step * A.spp;
    }
    const bool staged = stage_mie(mie_pack, mb, smem, &mbar);
    float *const shcol = reinterpret_cast<float *>(smem + ((mb + 15u) & ~15u)) + threadIdx.x;
    Count cnt;
    cnt.zero();
    uint32_t paths = 0;
    uint32_t nstack[kMaxDepth];
    Trav slow[1];
    PathLane<WALK> L;
    L.esc = kTrackEscaped;  // read by every lane after an event pass (sky queue), before its first segment ends
    uint32_t view = 0;
    uint32_t state = staged ? kFetch : kDone;
    if (!staged && threadIdx.x == 0) atomicAdd(&C->gave_up, 1ull);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const unsigned FULL = 0xffffffffu;
    // this warp's sky queue, after the phase tables and the shared traversal stack
    float *const skyq = reinterpret_cast<float *>(smem + ((mb + 15u) & ~15u) +
                                                  (size_t)shlevels * kShWords * 4u * kPersistentBlock) +
                        (threadIdx.x >> 5) * sky_queue_words<BATCH>();
    uint32_t nsky = 0;
    for (;;) {
        const uint32_t want = __ballot_sync(FULL, state == kFetch);
        if (want) {
            const uint32_t leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(&Q->next, (unsigned long long)__popc(want));
            base = __shfl_sync(FULL, base, leader);
            if (state == kFetch) {
                const uint64_t p = base + __popc(want & lt_mask);
                if (p >= n_total) {
                    state = kDone;
                } else {
                    bool ok;
                    if constexpr (BATCH) {
                        view = find_view(B, p);
                        const BatchView &V = B.views[view];
                        ok = start_path(L, p - V.begin, B.scenes[V.scene], V.P, V.A, shift * V.A.spp, cnt, paths,
                                        state, slow);
                    } else {
                        ok = start_path(L, p, S, P, A, shift, cnt, paths, state, slow);
                    }
                    if (!ok) state = kFetch;
                }
            }
        }
        if (__all_sync(FULL, state == kDone)) break;
        const uint32_t ev = __ballot_sync(FULL, state == kEvent);
        const uint32_t busy = __ballot_sync(FULL, state == kTrav || state == kStep);
        const bool events = ev && ((uint32_t)__popc(ev) >= event_batch || busy == 0);
        if constexpr (BATCH) {
            const BatchView &V = B.views[view];
            lane_work<WALK, FEAT, SHS>(L, events, B.scenes[V.scene], V.P, M, V.A, V.sun, V.sky, cnt, state, nstack,
                                      slow, visits, steps, ts, shcol, shlevels);
            // FEAT == 0: the launcher reserved the queue (views that defer set V.A.defer_sky)
            if constexpr (FEAT == 0) {
                if (events) sky_queue_push<true>(L, V.A, view, P, sky_out, B, skyq, nsky, lane, lt_mask);
            }
        } else {
            lane_work<WALK, FEAT, SHS>(L, events, S, P, M, A, sun_out, sky_out, cnt, state, nstack, slow, visits,
                                      steps, ts, shcol, shlevels);
            if constexpr (FEAT == 0) {
                if (events && A.defer_sky)
                    sky_queue_push<false>(L, A, 0u, P, sky_out, B, skyq, nsky, lane, lt_mask);
            }
        }
    }
    if constexpr (FEAT == 0) {
        if (BATCH || A.defer_sky) sky_queue_flush<BATCH>(P, sky_out, B, skyq, nsky, lane);
    }
    warp_sum_counts(cnt, C, paths);
}

// Advances the launch counter of a batch (the last node of its graph).
__global__ void batch_step_kernel(unsigned long long *step) { *step += 1ull; }

// Adds a blocking call's own counters into the context's.
__global__ void add_counters_kernel(DevCounters *dst, const DevCounters *src) {
    dst->paths += src->paths;
    dst->vertices += src->vertices;
    dst->node_visits += src->node_visits;
    dst->density_lookups += src->density_lookups;
    dst->mie_evals += src->mie_evals;
    dst->gave_up += src->gave_up;
}

// Leaf list of one camera ray (pixel ix, iy of the tile A): the stack
// traversal of the pixel's camera ray run to its end, as every sample of the
// pixel would run it, recorded for the persistent kernel (TileArgs::cam_head /
// cam_pool).  The leaves are counted first, then a contiguous range of the
// pool is taken and filled by a second traversal; a pixel whose range does not
// fit gets x = ~0 and its samples traverse.  `ray`: the ray's direction bits
// and whether the pixel has a ray (camera_ray's result).
__device__ __forceinline__ uint4 camera_list(const DevScene &S, const DevParams &P, const TileArgs &A, uint32_t ix,
                                             uint32_t iy, uint4 *pool, uint32_t cap, unsigned int *used, uint4 &ray) {
    float ro[3], rd[3];
    uint4 h = make_uint4(0u, 0u, 0u, 0u);
    const bool ok = camera_ray(P, A.x0 + ix, A.y0 + iy, ro, rd);
    ray = make_uint4(__float_as_uint(rd[0]), __float_as_uint(rd[1]), __float_as_uint(rd[2]), ok ? 1u : 0u);
    if (!ok) return h;
    uint32_t nstack[kMaxDepth];
    float tstack[kMaxDepth][6];
    Trav T;
    Count c;
    c.zero();
    trav_init(T, S, ro, rd, c);
    h.z = c.node_visits;
    uint32_t leaf, n = 0;
    float tra, trb;
    while (trav_next_k(T, S, nstack, leaf, tra, trb, c, 0xffffffffu, tstack) == kTravLeaf) ++n;
    const unsigned int off = n ? atomicAdd(used, n) : 0u;
    if (n && (off > cap || n > cap - off)) {
        h.x = kNone;
        return h;
    }
    h.x = off;
    h.y = n;
    trav_init(T, S, ro, rd, c);
    c.zero();
    for (uint32_t k = 0; k < n; ++k) {
        trav_next_k(T, S, nstack, leaf, tra, trb, c, 0xffffffffu, tstack);
        pool[off + k] = make_uint4(leaf, __float_as_uint(tra), __float_as_uint(trb), c.node_visits);
        c.zero();
    }
    trav_next_k(T, S, nstack, leaf, tra, trb, c, 0xffffffffu, tstack);  // kTravDone
    h.w = c.node_visits;
    return h;
}

// The camera leaf lists of a single-tile launch (one thread per pixel).
__global__ void __launch_bounds__(128) camera_list_kernel(DevScene S, DevParams P, TileArgs A, uint4 *head,
                                                          uint4 *pool, uint32_t cap, unsigned int *used) {
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= A.cols * A.rows) return;
    const uint32_t iy = pix / A.cols, ix = pix - iy * A.cols;
    uint4 ray;
    head[2 * (size_t)pix] = camera_list(S, P, A, ix, iy, pool, cap, used, ray);
    head[2 * (size_t)pix + 1] = ray;
}

// The camera leaf lists of every view of a batch: pixel p of the batch belongs
// to the last view v with pix_begins[v] <= p; its header is head[2p, 2p + 1]
// (the view's TileArgs::cam_head points at head + 2 pix_begins[v]).
__global__ void __launch_bounds__(128) batch_camera_list_kernel(BatchArgs B, const uint32_t *pix_begins,
                                                                uint32_t n_pix, uint4 *head, uint4 *pool,
                                                                uint32_t cap, unsigned int *used) {
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= n_pix) return;
    uint32_t lo = 0, hi = B.n_views - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&pix_begins[mid]) <= pix) lo = mid;
        else hi = mid - 1;
    }
    const BatchView &V = B.views[lo];
    const uint32_t q = pix - __ldg(&pix_begins[lo]);
    const uint32_t iy = q / V.A.cols, ix = q - iy * V.A.cols;
    uint4 ray;
    head[2 * (size_t)pix] = camera_list(B.scenes[V.scene], V.P, V.A, ix, iy, pool, cap, used, ray);
    head[2 * (size_t)pix + 1] = ray;
}

// ---- parity probes ------------------------------------------------------------
__global__ void probe_leaf_kernel(DevScene S, const float *ro, const float *rd, uint32_t n, uint32_t maxn,
                                  uint32_t *nodes, float *tr0, float *tr1, uint32_t *counts) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const float o[3] = {ro[3 * r], ro[3 * r + 1], ro[3 * r + 2]}, d[3] = {rd[3 * r], rd[3 * r + 1], rd[3 * r + 2]};
    Count cnt;
    cnt.zero();
    uint32_t nstack[kMaxDepth];
    uint32_t k = 0, leaf = 0;
    float a = 0.0f, b = 0.0f;
    Walk W;
    const uint32_t mode = walk_init(W, S, o, d, cnt);
    if (mode == 1u) {
        for (uint32_t guard = 0; k < maxn && guard < (1u << 22); ++guard) {
            const uint32_t st = walk_step(W, S, leaf, a, b, cnt);
            if (st == 2u) break;
            if (st == 1u) {
                nodes[(size_t)r * maxn + k] = leaf;
                tr0[(size_t)r * maxn + k] = a;
                tr1[(size_t)r * maxn + k] = b;
                ++k;
            }
        }
    } else if (mode == 2u) {
        Trav T;
        trav_init(T, S, o, d, cnt);
        while (k < maxn && trav_next(T, S, nstack, leaf, a, b, cnt)) {
            nodes[(size_t)r * maxn + k] = leaf;
            tr0[(size_t)r * maxn + k] = a;
            tr1[(size_t)r * maxn + k] = b;
            ++k;
        }
    }
    counts[r] = k;
}

__global__ void probe_occlusion_kernel(DevScene S, const float *ro, const float *rd, uint32_t n, uint32_t *hit) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float o[3] = {ro[3 * (size_t)i], ro[3 * (size_t)i + 1], ro[3 * (size_t)i + 2]};
    const float d[3] = {rd[3 * (size_t)i], rd[3 * (size_t)i + 1], rd[3 * (size_t)i + 2]};
    hit[i] = occluded(S, o, d) ? 1u : 0u;
}

__global__ void probe_density_kernel(DevScene S, const uint32_t *nodes, const float *pts, uint32_t n, float *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t leaf = nodes[i];
    const float4 ce = S.leaf[2 * leaf];
    const float4 meta = S.leaf[2 * leaf + 1];
    const float p[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
    out[i] = sample_voxel_space(p, S.bricks + (size_t)__float_as_uint(meta.y) * kBrick, ce);
}

__global__ void probe_paths_kernel(DevScene S, DevParams P, const void *mie_pack, const uint32_t *px,
                                   const uint32_t *py, const uint64_t *sample, uint32_t n, uint64_t seed,
                                   float4 *out_sun, float4 *out_sky, DevCounters *C) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t mbar;
    const bool staged = stage_mie(mie_pack, mie_bytes(P), smem, &mbar);
    const MieSmem M = mie_view(P, smem);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    Count cnt;
    cnt.zero();
    uint32_t nstack[kMaxDepth];
    uint32_t paths = 0;
    if (staged && i < n) {
        float4 a, b;
        path_sample(S, P, M, px[i], py[i], seed, sample[i], a, b, nstack, cnt);
        out_sun[i] = a;
        out_sky[i] = b;
        paths = 1;
    }
    warp_sum_counts(cnt, C, paths);
}

__global__ void probe_sampler_kernel(DevParams P, const void *mie_pack, uint32_t what, const float *in, uint32_t n,
                                     float *out) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t mbar;
    const bool staged = stage_mie(mie_pack, mie_bytes(P), smem, &mbar);
    const MieSmem M = mie_view(P, smem);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (!staged || i >= n) return;
    if (what == 0u) {
        const float3 r = mie_eval_rgb(M, in[i]);
        out[3 * i] = r.x;
        out[3 * i + 1] = r.y;
        out[3 * i + 2] = r.z;
    } else if (what == 1u) {
        const float iv[3] = {in[3 * i], in[3 * i + 1], in[3 * i + 2]};
        float d[3];
        mie_sample(M, iv, in[3 * n + i], in[4 * n + i], d);
        out[3 * i] = d[0];
        out[3 * i + 1] = d[1];
        out[3 * i + 2] = d[2];
    } else if (what == 2u) {
        float d[3];
        sun_sample(P, in[i], in[n + i], d);
        out[3 * i] = d[0];
        out[3 * i + 1] = d[1];
        out[3 * i + 2] = d[2];
    } else if (what == 3u) {
        const float rd[3] = {in[3 * i], in[3 * i + 1], in[3 * i + 2]};
        const float3 s = sky_eval(P, rd);
        out[3 * i] = s.x;
        out[3 * i + 1] = s.y;
        out[3 * i + 2] = s.z;
    } else if (what == 4u) {
        out[i] = mie_theta_ref(M, in[i]);
    } else if (what == 5u && M.ex) {
        float ct, st;
        mie_exact_dir(M.ex, M.n, in[i], ct, st);
        out[2 * i] = ct;
        out[2 * i + 1] = st;
    } else if (what == 6u) {
        out[i] = hg_eval(P.hg_g, in[i]);
    } else if (what == 7u) {
        const float iv[3] = {in[3 * i], in[3 * i + 1], in[3 * i + 2]};
        float d[3];
        hg_sample(P.hg_g, iv, in[3 * n + i], in[4 * n + i], d);
        out[3 * i] = d[0];
        out[3 * i + 1] = d[1];
        out[3 * i + 2] = d[2];
    } else if (what == 8u || (what == 9u && P.env_mode == kEnvMap)) {
        const float rd[3] = {in[3 * i], in[3 * i + 1], in[3 * i + 2]};
        const float3 s = what == 8u ? sky_light(P, rd) : env_map_eval(P, rd);
        out[3 * i] = s.x;
        out[3 * i + 1] = s.y;
        out[3 * i + 2] = s.z;
    }
}

// One thread per (ray, chunk of 64 samples); escapes summed per ray.
__global__ void probe_transmittance_kernel(DevScene S, DevParams P, const float *ro, const float *rd, uint32_t n_rays,
                                           uint64_t nsamp, uint64_t seed, unsigned long long *escapes) {
    const uint64_t chunks = (nsamp + 63) / 64;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= chunks * n_rays) return;
    const uint32_t r = (uint32_t)(t / chunks);
    const uint64_t c = t - (uint64_t)r * chunks;
    const float o[3] = {ro[3 * r], ro[3 * r + 1], ro[3 * r + 2]}, d[3] = {rd[3 * r], rd[3 * r + 1], rd[3 * r + 2]};
    Count cnt;
    cnt.zero();
    uint32_t nstack[kMaxDepth];
    uint32_t esc = 0;
    const uint64_t s1 = (c + 1) * 64 < nsamp ? (c + 1) * 64 : nsamp;
    for (uint64_t s = c * 64; s < s1; ++s) {
        Rng g = rng_seed(seed, r, s);
        float td;
        esc += track(S, P, o, d, g, 3.402823466e+38f, td, nstack, cnt) == kTrackEscaped ? 1u : 0u;
    }
    atomicAdd(&escapes[r], (unsigned long long)esc);
}

// ---- path-replay adjoint -------------------------------------------------------------
// Gradient of a loss L(image) with respect to the brick samples and the
// single-scatter albedo, given delta = dL/d(image sums) per pixel.  Delta
// tracking decides each tentative collision with P(real) = rho/smax; with the
// majorant held fixed the estimator's expectation depends on rho only through
// these decisions, so (score-function form)
//   dE[C]/dv = E[ sum_decisions C_after * dlog P(decision)/dv ],
//   dlog P/dv = (drho/dv) / rho   (real),   -(drho/dv) / (smax - rho)   (null),
// with drho/dv the trilinear weight of sample v.  C_after is the part of the
// path's contribution that the decision can change: for a decision on the
// camera or continuation segment r, everything the path adds from segment r
// on (its total minus what it added before); on a shadow segment, that
// segment's next-event contribution.  The albedo f enters each contribution as
// f^m (m = scattering events before it): dC/df = sum m * c / f.
// Each path is replayed from its random stream twice, as in path replay
// backpropagation: pass 1 recomputes its total contribution and keeps one
// float per path (its weight dsun . C_sun + dsky . C_sky), pass 2 replays the
// same decisions and scatters gradients.  The passes are separate launches, so
// the lanes of a warp run the same tracking code; no per-path tape is stored.
// A shadow segment is tracked once to learn whether it escapes and, if it
// did, again from the saved stream state to scatter.

struct ScatterVisit {
    float w;  // dL/dC_after of the current segment
    float *grad;
    const float *bricks;
    __device__ __forceinline__ void operator()(const float *brick, const float4 &ce, const float *rc, float rho,
                                               float smax, bool real) const {
        if (w == 0.0f) return;
        float sc;
        if (real) {
            if (!(rho > 0.0f)) return;
            sc = w / rho;
        } else {
            const float d = smax - rho;
            if (!(d > 0.0f)) return;
            sc = (0.0f - w) / d;
        }
        uint32_t idx[8];
        float wt[8];
        voxel_weights(rc, ce, idx, wt);
        float *gb = grad + (brick - bricks);
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (wt[c] != 0.0f) atomicAdd(gb + idx[c], sc * wt[c]);
    }
};

// One copy of the tracking loop per visitor for the whole adjoint (each call
// site inlining it would multiply the code the warps fetch).
template <bool SDF>
__device__ __noinline__ uint32_t track_plain(const DevScene S, SegMedium med, const float *ro, const float *rd, Rng &g,
                                             float depth, float &td, uint32_t *nstack, Count &cnt) {
    const NoVisit nv;
    return track_v<NoVisit, SDF>(S, med, ro, rd, g, depth, td, nstack, cnt, nv);
}

template <bool SDF>
__device__ __noinline__ uint32_t track_scatter(const DevScene S, SegMedium med, const float *ro, const float *rd,
                                               Rng &g, float depth, float &td, uint32_t *nstack, Count &cnt,
                                               const ScatterVisit &sv) {
    return track_v<ScatterVisit, SDF>(S, med, ro, rd, g, depth, td, nstack, cnt, sv);
}

constexpr uint32_t kEscBits = 64;  // shadow segments whose outcome pass 1 records

// Reweighted replay (the finite-difference check of the adjoint): decisions are
// drawn from the context's bricks, and each is weighted by its probability under
// a perturbed brick pool over its probability under the drawn one (rho'/rho
// for real, (smax - rho')/(smax - rho) for null).  The weighted estimator is
// unbiased for the perturbed image and smooth in the perturbation, so its
// central differences with common random numbers are not swamped by decisions
// that flip.
struct RatioVisit {
    float *w;  // running product of the segment's ratios
    const float *pert;
    const float *bricks;
    __device__ __forceinline__ void operator()(const float *brick, const float4 &ce, const float *rc, float rho,
                                               float smax, bool real) const {
        const float rp = sample_voxel_space(rc, pert + (brick - bricks), ce);
        if (real) {
            if (rho > 0.0f) *w = *w * (rp / rho);
        } else {
            const float d = smax - rho;
            if (d > 0.0f) *w = *w * ((smax - rp) / d);
        }
    }
};

template <bool SDF>
__device__ __noinline__ uint32_t track_ratio(const DevScene S, SegMedium med, const float *ro, const float *rd, Rng &g,
                                             float depth, float &td, uint32_t *nstack, Count &cnt,
                                             const RatioVisit &rv) {
    return track_v<RatioVisit, SDF>(S, med, ro, rd, g, depth, td, nstack, cnt, rv);
}

struct PathTotals {
    float w;            // dsun . (sun contribution) + dsky . (sky contribution) of the whole path
    uint64_t esc;       // bit r: the shadow segment after scattering event r is lit (r < kEscBits)
    float3 asun, asky;  // sum over contributions of (scattering events before it) * contribution
    bool ok;            // every component of the path's contribution is finite
};

// What pass 1 keeps per path for pass 2 (16 bytes): the weight (NaN: path left
// out) and the bits of its lit shadow segments (escaped, no occluder hit).
struct __align__(16) PathRecord {
    float w;
    uint32_t esc_lo, esc_hi, pad;
};

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float dot3f(const float3 a, const float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// MODE kPassTotals fills tot; kPassScatter scatters with tot known;
// kPassRatio fills tot.w for the reweighted replay (pert = perturbed bricks).
enum : int { kPassTotals = 0, kPassScatter = 1, kPassRatio = 2 };
template <int MODE, uint32_t FEAT>
__device__ __forceinline__ void adjoint_pass(const DevScene &S, const DevParams &P, const MieSmem &M, uint32_t px,
                                             uint32_t py, uint64_t seed, uint64_t sample, float3 dsun, float3 dsky,
                                             PathTotals &tot, float *grad, uint32_t *nstack,
                                             const float *pert = nullptr) {
    constexpr bool SCATTER = MODE == kPassScatter;
    constexpr bool RATIO = MODE == kPassRatio;
    float ro[3], rd[3];
    if (!camera_ray(P, px, py, ro, rd)) return;
    Count cnt;
    cnt.zero();
    Rng g = rng_seed(seed, (uint64_t)py * P.w + px, sample);
    const float f = P.albedo;
    float T0 = 1.0f, T1 = 1.0f, T2 = 1.0f;
    const float depth0 = (P.depth && P.depthcomp) ? __ldg(&P.depth[(size_t)py * P.w + px]) : 3.402823466e+38f;
    float3 acc_sun = f3(0.f, 0.f, 0.f), acc_sky = acc_sun, a_sun = acc_sun, a_sky = acc_sun;
    ScatterVisit vis{0.0f, grad, S.bricks};
    for (uint32_t r = 0;; ++r) {
        float td;
        uint32_t res;
        if constexpr (SCATTER) {
            vis.w = tot.w - (dot3f(dsun, acc_sun) + dot3f(dsky, acc_sky));
            res = track_scatter<(FEAT & kFeatSdf) != 0>(S, seg_medium(P), ro, rd, g, r == 0 ? depth0 : 3.402823466e+38f, td, nstack, cnt, vis);
        } else if constexpr (RATIO) {
            // the segment's ratios scale everything the path adds from here on
            float ws = 1.0f;
            const RatioVisit rv{&ws, pert, S.bricks};
            res = track_ratio<(FEAT & kFeatSdf) != 0>(S, seg_medium(P), ro, rd, g, r == 0 ? depth0 : 3.402823466e+38f, td, nstack, cnt, rv);
            T0 = T0 * ws;
            T1 = T1 * ws;
            T2 = T2 * ws;
        } else {
            res = track_plain<(FEAT & kFeatSdf) != 0>(S, seg_medium(P), ro, rd, g, r == 0 ? depth0 : 3.402823466e+38f, td, nstack, cnt);
        }
        if (res == kTrackCut) break;
        if (res == kTrackEscaped) {
            if (r > 0 && !((FEAT & kFeatOcc) && P.embree && occluded(S, ro, rd))) {
                const bool hit = sun_hit(P, rd);
                const float3 cs = f3(T0 * (hit ? P.sun_color[0] : 0.0f), T1 * (hit ? P.sun_color[1] : 0.0f),
                                     T2 * (hit ? P.sun_color[2] : 0.0f));
                const float3 sk = escape_sky<FEAT>(P, rd);
                const float3 ck = f3(T0 * sk.x, T1 * sk.y, T2 * sk.z);
                const float m = (float)r;
                acc_sun = f3(acc_sun.x + cs.x, acc_sun.y + cs.y, acc_sun.z + cs.z);
                acc_sky = f3(acc_sky.x + ck.x, acc_sky.y + ck.y, acc_sky.z + ck.z);
                a_sun = f3(a_sun.x + m * cs.x, a_sun.y + m * cs.y, a_sun.z + m * cs.z);
                a_sky = f3(a_sky.x + m * ck.x, a_sky.y + m * ck.y, a_sky.z + m * ck.z);
            }
            break;
        }
        if (r >= P.scattevs) break;
        float srd[3], lrd[3], rc[3];
        const float u1 = g.uniform(), u2 = g.uniform();
        path_phase_sample<FEAT>(P, M, rd, u1, u2, srd);
        const float u3 = g.uniform(), u4 = g.uniform();
        sun_sample(P, u3, u4, lrd);
        const float3 p1 = path_phase_eval<FEAT>(P, M, dot3(srd, rd));
        const float p2 = sun_hit(P, lrd) ? P.sun_pdf : 0.0f;
        const float3 p3 = path_phase_eval<FEAT>(P, M, dot3(lrd, rd));
        const float q1 = sun_hit(P, srd) ? P.sun_pdf : 0.0f;
#pragma unroll
        for (int k = 0; k < 3; ++k) rc[k] = ro[k] + rd[k] * td;
        const bool hit = sun_hit(P, lrd);
        float3 cn = f3((T0 * ((p3.x / (p3.x + p2)) * f)) * (hit ? P.sun_color[0] : 0.0f),
                             (T1 * ((p3.y / (p3.y + p2)) * f)) * (hit ? P.sun_color[1] : 0.0f),
                             (T2 * ((p3.z / (p3.z + p2)) * f)) * (hit ? P.sun_color[2] : 0.0f));
        float tds;
        bool lit;  // the shadow segment escaped and no occluder blocks its ray
        if constexpr (SCATTER) {
            // segments 0..63: pass 1 recorded whether the shadow is lit, so it
            // is tracked once with its weight (zero unless it is lit)
            const bool known = r < kEscBits;
            const Rng g0 = g;
            ScatterVisit sv{(known && ((tot.esc >> r) & 1ull)) ? dot3f(dsun, cn) : 0.0f, grad, S.bricks};
            const uint32_t sres = track_scatter<(FEAT & kFeatSdf) != 0>(S, seg_medium(P), rc, lrd, g, 3.402823466e+38f, tds, nstack, cnt, sv);
            if (known) {
                lit = (tot.esc >> r) & 1ull;
            } else {
                lit = sres == kTrackEscaped && !((FEAT & kFeatOcc) && P.embree && occluded(S, rc, lrd));
                sv.w = dot3f(dsun, cn);
                if (lit && sv.w != 0.0f) {
                    Rng g1 = g0;  // the same draws again: ends in the state g already holds
                    float t2;
                    (void)track_scatter<(FEAT & kFeatSdf) != 0>(S, seg_medium(P), rc, lrd, g1, 3.402823466e+38f, t2, nstack, cnt, sv);
                }
            }
        } else if constexpr (RATIO) {
            float ws = 1.0f;
            const RatioVisit rv{&ws, pert, S.bricks};
            const uint32_t sres = track_ratio<(FEAT & kFeatSdf) != 0>(S, seg_medium(P), rc, lrd, g, 3.402823466e+38f, tds, nstack, cnt, rv);
            lit = sres == kTrackEscaped && !((FEAT & kFeatOcc) && P.embree && occluded(S, rc, lrd));
            cn = f3(cn.x * ws, cn.y * ws, cn.z * ws);
        } else {
            const uint32_t sres = track_plain<(FEAT & kFeatSdf) != 0>(S, seg_medium(P), rc, lrd, g, 3.402823466e+38f, tds, nstack, cnt);
            lit = sres == kTrackEscaped && !((FEAT & kFeatOcc) && P.embree && occluded(S, rc, lrd));
            if (lit && r < kEscBits) tot.esc |= 1ull << r;
        }
        if (lit) {
            const float m = (float)(r + 1);
            acc_sun = f3(acc_sun.x + cn.x, acc_sun.y + cn.y, acc_sun.z + cn.z);
            a_sun = f3(a_sun.x + m * cn.x, a_sun.y + m * cn.y, a_sun.z + m * cn.z);
        }
        T0 = T0 * ((p1.x / (p1.x + q1)) * f);
        T1 = T1 * ((p1.y / (p1.y + q1)) * f);
        T2 = T2 * ((p1.z / (p1.z + q1)) * f);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            ro[k] = rc[k];
            rd[k] = srd[k];
        }
    }
    if constexpr (!SCATTER) {
        tot.w = dot3f(dsun, acc_sun) + dot3f(dsky, acc_sky);
        tot.asun = a_sun;
        tot.asky = a_sky;
        tot.ok = isfinite(acc_sun.x) && isfinite(acc_sun.y) && isfinite(acc_sun.z) && isfinite(acc_sky.x) &&
                 isfinite(acc_sky.y) && isfinite(acc_sky.z);
    }
}

// Warp-wide sum of one float added to one of kSlots double accumulators
// (slot = global warp index % kSlots; no block barrier, so a block's warps
// retire independently); the slots are summed into the output afterwards.
constexpr uint32_t kSlots = 1024;
__device__ __forceinline__ void warp_add(float v, double *slots) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    if ((threadIdx.x & 31) == 0 && v != 0.0f) {
        const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        atomicAdd(&slots[w % kSlots], (double)v);
    }
}

__global__ void sum_slots_kernel(double *out, double *slots) {
    __shared__ double part[32];
    double v = 0.0;
    for (uint32_t k = threadIdx.x; k < kSlots; k += blockDim.x) {
        v += slots[k];
        slots[k] = 0.0;
    }
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (uint32_t k = 0; k < blockDim.x / 32; ++k) s += part[k];
        *out += s;
    }
}

// Path gi of a tile (one thread per (pixel, sample), the render kernel's
// layout): its pixel column i and row j in the tile and its sample s.
__device__ __forceinline__ void tile_path(const TileArgs &A, uint64_t gi, uint32_t &i, uint32_t &j, uint32_t &s) {
    const uint64_t pl = gi / A.spp;
    s = (uint32_t)(gi - pl * A.spp);
    const uint32_t pix = (uint32_t)pl;
    i = pix % A.cols;
    j = pix / A.cols;
}

// Pass 1 over paths [p0, p0 + n) of a tile (delta images in tile layout,
// tw x th float4, rgb used): rec[gi - p0] = the path's weight dsun . C_sun +
// dsky . C_sky (NaN for a path left out: zero delta at its pixel, or a
// contribution that is not finite, the sky term's 0/0 for rd.y == 0) and its
// lit-shadow bits; the albedo term goes to the slots.
template <uint32_t FEAT>
__global__ void __launch_bounds__(kRenderBlock) adjoint_totals_kernel(DevScene S, DevParams P, TileArgs A,
                                                                      uint64_t p0, uint64_t n, const void *mie_pack,
                                                                      const float4 *dsun, const float4 *dsky,
                                                                      PathRecord *rec, double *albedo_slots,
                                                                      DevCounters *C) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t mbar;
    const bool staged = stage_mie(mie_pack, mie_bytes(P), smem, &mbar);
    const MieSmem M = mie_view(P, smem);
    uint32_t nstack[kMaxDepth];
    const uint64_t k = (uint64_t)blockIdx.x * kRenderBlock + threadIdx.x;
    float galb = 0.0f;
    if (staged && k < n) {
        uint32_t i, j, s;
        tile_path(A, p0 + k, i, j, s);
        const size_t o = (size_t)j * A.tw + i;
        const float4 ds = __ldg(&dsun[o]), dk = __ldg(&dsky[o]);
        const float3 dsun3 = f3(ds.x, ds.y, ds.z), dsky3 = f3(dk.x, dk.y, dk.z);
        PathRecord pr{__int_as_float(0x7fffffff), 0u, 0u, 0u};
        if (dot3f(dsun3, dsun3) + dot3f(dsky3, dsky3) > 0.0f) {
            PathTotals tot{};
            adjoint_pass<kPassTotals, FEAT>(S, P, M, A.x0 + i, A.y0 + j, A.seed, A.sample_base + s, dsun3, dsky3, tot, nullptr,
                                nstack);
            if (tot.ok) {
                pr.w = tot.w;
                pr.esc_lo = (uint32_t)tot.esc;
                pr.esc_hi = (uint32_t)(tot.esc >> 32);
                galb = (dot3f(dsun3, tot.asun) + dot3f(dsky3, tot.asky)) / P.albedo;
            }
        }
        rec[k] = pr;
    }
    if (!staged && threadIdx.x == 0) atomicAdd(&C->gave_up, 1ull);
    warp_add(galb, albedo_slots);
}

// Pass 2 over the same paths: replays each path kept by pass 1 and scatters
// its gradient.  Gradients go to copy blockIdx.x % copies of the brick-pool
// gradient (grad + copy * stride): the surface samples every path meets
// first are hit by all warps at once, and spreading them over copies divides
// the conflicts on each address; the copies are summed afterwards.
template <uint32_t FEAT>
__global__ void __launch_bounds__(kRenderBlock) adjoint_scatter_kernel(DevScene S, DevParams P, TileArgs A,
                                                                       uint64_t p0, uint64_t n, const void *mie_pack,
                                                                       const float4 *dsun, const float4 *dsky,
                                                                       const PathRecord *rec, float *grad,
                                                                       uint32_t copies, size_t stride,
                                                                       DevCounters *C) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t mbar;
    const bool staged = stage_mie(mie_pack, mie_bytes(P), smem, &mbar);
    const MieSmem M = mie_view(P, smem);
    uint32_t nstack[kMaxDepth];
    const uint64_t k = (uint64_t)blockIdx.x * kRenderBlock + threadIdx.x;
    grad += (size_t)(blockIdx.x % copies) * stride;
    if (staged && k < n) {
        const PathRecord pr = rec[k];
        if (!isnan(pr.w)) {
            uint32_t i, j, s;
            tile_path(A, p0 + k, i, j, s);
            const size_t o = (size_t)j * A.tw + i;
            const float4 ds = __ldg(&dsun[o]), dk = __ldg(&dsky[o]);
            PathTotals tot{};
            tot.w = pr.w;
            tot.esc = ((uint64_t)pr.esc_hi << 32) | pr.esc_lo;
            adjoint_pass<kPassScatter, FEAT>(S, P, M, A.x0 + i, A.y0 + j, A.seed, A.sample_base + s, f3(ds.x, ds.y, ds.z),
                               f3(dk.x, dk.y, dk.z), tot, grad, nstack);
        }
    }
    if (!staged && threadIdx.x == 0) atomicAdd(&C->gave_up, 1ull);
}

// Warp-wide double sum added to one of kSlots accumulators (as warp_add).
__device__ __forceinline__ void warp_add_d(double v, double *slots) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    if ((threadIdx.x & 31) == 0 && v != 0.0) {
        const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        atomicAdd(&slots[w % kSlots], v);
    }
}

// Reweighted replay of a tile's paths: the linearised loss sum over paths of
// dsun . C_sun + dsky . C_sky, each path weighted by its decisions' ratios
// under pert (paths whose contribution is not finite are left out, as in the
// adjoint).
template <uint32_t FEAT>
__global__ void __launch_bounds__(kRenderBlock) reweighted_loss_kernel(DevScene S, DevParams P, TileArgs A,
                                                                       const void *mie_pack, const float4 *dsun,
                                                                       const float4 *dsky, const float *pert,
                                                                       double *slots, DevCounters *C) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t mbar;
    const bool staged = stage_mie(mie_pack, mie_bytes(P), smem, &mbar);
    const MieSmem M = mie_view(P, smem);
    uint32_t nstack[kMaxDepth];
    const uint64_t k = (uint64_t)blockIdx.x * kRenderBlock + threadIdx.x;
    double l = 0.0;
    if (staged && k < A.n_paths) {
        uint32_t i, j, s;
        tile_path(A, k, i, j, s);
        const size_t o = (size_t)j * A.tw + i;
        const float4 ds = __ldg(&dsun[o]), dk = __ldg(&dsky[o]);
        const float3 dsun3 = f3(ds.x, ds.y, ds.z), dsky3 = f3(dk.x, dk.y, dk.z);
        if (dot3f(dsun3, dsun3) + dot3f(dsky3, dsky3) > 0.0f) {
            PathTotals tot{};
            adjoint_pass<kPassRatio, FEAT>(S, P, M, A.x0 + i, A.y0 + j, A.seed, A.sample_base + s, dsun3, dsky3, tot,
                                     nullptr, nstack, pert);
            if (tot.ok) l = (double)tot.w;
        }
    }
    if (!staged && threadIdx.x == 0) atomicAdd(&C->gave_up, 1ull);
    warp_add_d(l, slots);
}

// out[k] += sum over copies c of src[c * stride + k].
__global__ void sum_copies_kernel(float *out, const float *src, uint32_t copies, size_t stride) {
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < stride; k += (size_t)gridDim.x * blockDim.x) {
        float v = 0.0f;
        for (uint32_t c = 0; c < copies; ++c) v += src[(size_t)c * stride + k];
        out[k] += v;
    }
}

// Gradient of sum_r w_r T_r (T_r: delta-tracking transmittance of ray r over
// nsamp samples, streams (seed, r, s) as probe_transmittance_kernel) with
// respect to the brick samples: an escaped sample replays its null decisions
// with weight w_r / nsamp; a collided one contributes nothing.
__global__ void adjoint_transmittance_kernel(DevScene S, DevParams P, const float *ro, const float *rd,
                                             const float *wr, uint32_t n_rays, uint64_t nsamp, uint64_t seed,
                                             float *grad, unsigned long long *escapes) {
    const uint64_t chunks = (nsamp + 63) / 64;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= chunks * n_rays) return;
    const uint32_t r = (uint32_t)(t / chunks);
    const uint64_t c = t - (uint64_t)r * chunks;
    const float o[3] = {ro[3 * r], ro[3 * r + 1], ro[3 * r + 2]}, d[3] = {rd[3 * r], rd[3 * r + 1], rd[3 * r + 2]};
    Count cnt;
    cnt.zero();
    uint32_t nstack[kMaxDepth];
    uint32_t esc = 0;
    ScatterVisit sv{wr[r] / (float)nsamp, grad, S.bricks};
    const uint64_t s1 = (c + 1) * 64 < nsamp ? (c + 1) * 64 : nsamp;
    for (uint64_t s = c * 64; s < s1; ++s) {
        Rng g = rng_seed(seed, r, s);
        const Rng g0 = g;
        float td;
        if (track_plain<true>(S, seg_medium(P), o, d, g, 3.402823466e+38f, td, nstack, cnt) == kTrackEscaped) {
            ++esc;
            Rng g1 = g0;
            (void)track_scatter<true>(S, seg_medium(P), o, d, g1, 3.402823466e+38f, td, nstack, cnt, sv);
        }
    }
    atomicAdd(&escapes[r], (unsigned long long)esc);
}

// Majorants after a brick update: max over the leaf's samples, floor 0.01
// (src/scene.cpp:889-904), times scale (>= 1: headroom that lets samples grow
// while the majorant stays fixed); a leaf whose majorant was 0 (never
// resampled) keeps 0.
__global__ void leaf_majorant_kernel(float4 *leaf, const uint32_t *leaf_nodes, uint32_t n_leafnodes,
                                     const float *bricks, float scale) {
    const uint32_t i = blockIdx.x;
    if (i >= n_leafnodes) return;
    const uint32_t node = leaf_nodes[i];
    float4 meta = leaf[2 * (size_t)node + 1];
    const float *b = bricks + (size_t)__float_as_uint(meta.y) * kBrick;
    float m = 0.0f;
    for (uint32_t k = threadIdx.x; k < kBrick; k += blockDim.x) m = fmaxf(m, b[k]);
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, s));
    __shared__ float wm[32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t k = 1; k < (blockDim.x + 31) / 32; ++k) m = fmaxf(m, wm[k]);
        wm[0] = fmaxf(m, wm[0]);
        if (meta.x != 0.0f) meta.x = fmaxf(wm[0], 0.01f) * scale;
        leaf[2 * (size_t)node + 1] = meta;
    }
}

// ---- transmittance without allocation ----------------------------------------------
// Scratch of the allocation-free entry point: one escape counter per ray in a
// file-scope device array (512 KB on every GPU that loads the library, for the
// life of the process).  Every call shares it, so calls that overlap on the
// GPU race; each call clears the counters it uses before counting.
constexpr uint32_t kNoAllocMaxRays = 65536;
static __device__ __align__(256) unsigned long long g_noalloc_escapes[kNoAllocMaxRays];

__global__ void noalloc_clear_kernel(unsigned long long *escapes, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) escapes[i] = 0ull;
}

__global__ void noalloc_finish_kernel(const unsigned long long *escapes, uint32_t n, uint64_t nsamp, double *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (double)escapes[i] / (double)nsamp;
}

uint32_t noalloc_max_rays() { return kNoAllocMaxRays; }

// Device address of the scratch array, looked up once per device (with that
// device current) and cached.
static std::mutex g_noalloc_mu;
static unsigned long long *g_noalloc_ptr[64] = {nullptr};

cudaError_t noalloc_scratch(int device, unsigned long long **out) {
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_escapes);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[device] = static_cast<unsigned long long *>(p);
    }
    *out = g_noalloc_ptr[device];
    return cudaSuccess;
}

cudaError_t launch_transmittance_noalloc(const DevScene &S, const DevParams &P, unsigned long long *scratch,
                                         const float *ro, const float *rd, uint32_t n_rays, uint64_t nsamp,
                                         uint64_t seed, double *out, cudaStream_t st) {
    noalloc_clear_kernel<<<(n_rays + 255) / 256, 256, 0, st>>>(scratch, n_rays);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = launch_probe_transmittance(S, P, ro, rd, n_rays, nsamp, seed, scratch, st);
    if (e != cudaSuccess) return e;
    noalloc_finish_kernel<<<(n_rays + 255) / 256, 256, 0, st>>>(scratch, n_rays, nsamp, out);
    return cudaGetLastError();
}

// ---- launchers ------------------------------------------------------------------
static size_t mie_smem(const DevParams &P) {
    return (size_t)P.mie_n * 20u + (P.phase_mode == 1u ? (2u * (size_t)P.mie_n + 1u) * 16u : 0u);
}

// Dynamic shared memory above the default 48 KB (phase tables of more than
// about 2,400 entries) needs the kernel's opt-in, up to the 227 KB a block can have.
template <class F> static cudaError_t allow_smem(F fn, size_t smem) {
    if (smem <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(reinterpret_cast<const void *>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem);
}

// Feature bits a frame needs.
static uint32_t frame_features(const DevScene &S, const DevParams &P) {
    return ((S.occ_nodes && P.embree) ? kFeatOcc : 0u) |
           ((P.phase_mode == kPhaseHG || P.env_mode != kEnvHosek) ? kFeatExt : 0u) | (S.sdf_bricks ? kFeatSdf : 0u);
}

cudaError_t launch_render_tile(const DevScene &S, const DevParams &P, const TileArgs &A, const void *mie_pack,
                               float4 *sun_out, float4 *sky_out, DevCounters *C, cudaStream_t st) {
    if (A.n_paths == 0) return cudaSuccess;
    const uint64_t blocks = (A.n_paths + kRenderBlock - 1) / kRenderBlock;
    if (blocks > 0x7fffffffull) return cudaErrorInvalidValue;
    const auto fn = frame_features(S, P) ? render_tile_kernel<kFeatAll> : render_tile_kernel<0>;
    const cudaError_t e = allow_smem(fn, mie_smem(P));
    if (e != cudaSuccess) return e;
    fn<<<(unsigned)blocks, kRenderBlock, mie_smem(P), st>>>(S, P, A, mie_pack, sun_out, sky_out, C);
    return cudaGetLastError();
}

cudaError_t launch_shadow_tile(const DevScene &S, const DevParams &P, const TileArgs &A, float4 *out, DevCounters *C,
                               cudaStream_t st) {
    if (A.n_paths == 0) return cudaSuccess;
    const uint64_t blocks = (A.n_paths + kRenderBlock - 1) / kRenderBlock;
    if (blocks > 0x7fffffffull) return cudaErrorInvalidValue;
    shadow_tile_kernel<<<(unsigned)blocks, kRenderBlock, 0, st>>>(S, P, A, out, C);
    return cudaGetLastError();
}

// Variants of the persistent kernel compiled for 4, 5, 6 and 8 resident
// blocks per SM (fewer registers, some spilled to L1-resident local memory),
// each with the stack traversal or the cell walk, single frame or batch.  The
// feature variants (occluders, HG phase / environment maps) exist for 5 and 8
// blocks per SM; a tuned 4 or 6 maps to the nearest of those.
using PersistentFn = void (*)(DevScene, DevParams, TileArgs, const void *, float4 *, float4 *, DevCounters *,
                              WorkQueue *, uint32_t, BatchArgs);
template <bool BATCH, uint32_t FEAT>
static PersistentFn persistent_variant_of(uint32_t minb, uint32_t traversal) {
    if constexpr (FEAT != 0) {
        if (traversal == 1u) return minb >= 7 ? render_persistent_kernel<8, true, BATCH, FEAT>
                                              : render_persistent_kernel<5, true, BATCH, FEAT>;
        return minb >= 7 ? render_persistent_kernel<8, false, BATCH, FEAT> : render_persistent_kernel<5, false, BATCH, FEAT>;
    } else {
        if (traversal == 2u) {
            if (minb >= 8) return render_persistent_kernel<8, false, BATCH, 0, true>;
            if (minb >= 6) return render_persistent_kernel<6, false, BATCH, 0, true>;
            if (minb >= 5) return render_persistent_kernel<5, false, BATCH, 0, true>;
            return render_persistent_kernel<4, false, BATCH, 0, true>;
        }
        if (traversal == 1u) {
            if (minb >= 8) return render_persistent_kernel<8, true, BATCH, 0>;
            if (minb >= 6) return render_persistent_kernel<6, true, BATCH, 0>;
            if (minb >= 5) return render_persistent_kernel<5, true, BATCH, 0>;
            return render_persistent_kernel<4, true, BATCH, 0>;
        }
        if (minb >= 8) return render_persistent_kernel<8, false, BATCH, 0>;
        if (minb >= 6) return render_persistent_kernel<6, false, BATCH, 0>;
        if (minb >= 5) return render_persistent_kernel<5, false, BATCH, 0>;
        return render_persistent_kernel<4, false, BATCH, 0>;
    }
}

// Frames that use any feature (occluders, HG phase / environment maps, surface
// leaves) take the instantiation with all of them.  Batches carry no occluders
// (their scenes come from dr_scene_desc records), so the flag stays off there.
static PersistentFn persistent_variant(uint32_t minb, uint32_t traversal, bool batch, uint32_t feat = 0) {
    if (batch) return feat ? persistent_variant_of<true, kFeatAll>(minb, traversal)
                           : persistent_variant_of<true, 0>(minb, traversal);
    return feat ? persistent_variant_of<false, kFeatAll>(minb, traversal)
                : persistent_variant_of<false, 0>(minb, traversal);
}

int persistent_max_blocks_per_sm(uint32_t variant, uint32_t traversal, size_t smem_bytes) {
    int nb = 0;
    const PersistentFn fn = persistent_variant(variant, traversal, false);
    if (allow_smem(fn, smem_bytes) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kPersistentBlock, smem_bytes) != cudaSuccess)
        return 1;
    return nb > 0 ? nb : 1;
}

// Grid of the persistent kernel: SMs x resident blocks (the tuned count, capped
// by what fits).
static cudaError_t persistent_grid(const Tuning &tune, int device, size_t smem, bool batch, uint32_t feat,
                                   PersistentFn &fn, int &blocks, uint32_t &event_batch) {
    int sms = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    const uint32_t variant = tune.blocks_per_sm ? tune.blocks_per_sm : 4u;
    fn = persistent_variant(variant, tune.traversal, batch, feat);
    e = allow_smem(fn, smem);
    if (e != cudaSuccess) return e;
    int maxb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxb, fn, kPersistentBlock, smem) != cudaSuccess || maxb < 1)
        maxb = 1;
    const int bps = tune.blocks_per_sm && (int)tune.blocks_per_sm < maxb ? (int)tune.blocks_per_sm : maxb;
    blocks = sms * bps;
    event_batch = tune.event_batch ? (tune.event_batch > 32 ? 32u : tune.event_batch) : 8u;
    event_batch |= (tune.visits > 255 ? 255u : tune.visits) << 8;
    event_batch |= (tune.steps > 255 ? 255u : tune.steps) << 16;
    return cudaSuccess;
}

// Largest octree depth whose traversal stack goes to shared memory: 7 entries
// x 16 B x 128 lanes = 14 KB per block besides the phase tables.
constexpr uint32_t kShStackMax = 7;

// DR_TRAVERSAL_STACK_SHARED: only for the plain instantiation and octrees of
// known, modest depth (and within the default 48 KB of dynamic shared memory);
// otherwise the local-memory stack.  Returns the stack entries (0: local).
static uint32_t shared_stack_plan(Tuning &tune, uint32_t feat, uint32_t stack_levels, size_t &smem) {
    if (tune.traversal != 2u) return 0;
    const size_t with = ((smem + 15) & ~(size_t)15) + (size_t)stack_levels * kShWords * 4 * kPersistentBlock;
    if (feat == 0 && stack_levels >= 1 && stack_levels <= kShStackMax && with <= 48 * 1024) {
        smem = with;
        return stack_levels;
    }
    tune.traversal = 0;
    return 0;
}

cudaError_t launch_render_persistent(const DevScene &S, const DevParams &P, const TileArgs &A, const void *mie_pack,
                                     float4 *sun_out, float4 *sky_out, DevCounters *C, WorkQueue *Q,
                                     const Tuning &tune_in, int device, cudaStream_t st, const CamLists &lists) {
    if (A.n_paths == 0) return cudaSuccess;
    size_t smem = mie_smem(P);
    const uint32_t feat = frame_features(S, P);
    Tuning tune = tune_in;
    const uint32_t shlevels = shared_stack_plan(tune, feat, S.stack_levels, smem);
    // sky terms evaluated by full warps (Hosek sky only; a whole-path
    // finiteness check needs the path's sky sum in place)
    TileArgs Ad = A;
    Ad.defer_sky = (feat == 0 && !P.finite_paths) ? 1u : 0u;
    if (Ad.defer_sky) smem = ((smem + 15) & ~(size_t)15) + (size_t)sky_queue_words<false>() * 4u * (kPersistentBlock / 32);
    PersistentFn fn;
    int blocks;
    uint32_t batch;
    cudaError_t e = persistent_grid(tune, device, smem, false, feat, fn, blocks, batch);
    if (e != cudaSuccess) return e;
    batch |= shlevels << 24;
    e = cudaMemsetAsync(Q, 0, sizeof(WorkQueue), st);
    if (e != cudaSuccess) return e;
    if (lists.head && tune.traversal != 1u) {  // the cell walk counts grid cells: it keeps its own traversal
        e = cudaMemsetAsync(lists.used, 0, sizeof(unsigned int), st);
        if (e != cudaSuccess) return e;
        const uint32_t npix = A.cols * A.rows;
        camera_list_kernel<<<(npix + 127) / 128, 128, 0, st>>>(S, P, A, lists.head, lists.pool, lists.cap,
                                                               lists.used);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        Ad.cam_head = lists.head;
        Ad.cam_pool = lists.pool;
    }
    fn<<<blocks, kPersistentBlock, smem, st>>>(S, P, Ad, mie_pack, sun_out, sky_out, C, Q, batch, BatchArgs{});
    return cudaGetLastError();
}

cudaError_t launch_batch_lists(const BatchArgs &B, const BatchLists &lists, cudaStream_t st) {
    if (!B.n_paths || !lists.lists.head || !lists.n_pix) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(lists.lists.used, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    batch_camera_list_kernel<<<(lists.n_pix + 127) / 128, 128, 0, st>>>(
        B, lists.pix_begins, lists.n_pix, lists.lists.head, lists.lists.pool, lists.lists.cap, lists.lists.used);
    return cudaGetLastError();
}

cudaError_t launch_batch_kernel(const BatchArgs &B, const DevParams &P0, const void *mie_pack, DevCounters *C,
                                WorkQueue *Q, const Tuning &tune_in, bool ext, uint32_t stack_levels, int device,
                                cudaStream_t st) {
    if (!B.n_paths) return cudaSuccess;
    size_t smem = mie_smem(P0);
    Tuning tune = tune_in;
    const uint32_t shlevels = shared_stack_plan(tune, ext ? kFeatAll : 0u, stack_levels, smem);
    if (!ext) smem = ((smem + 15) & ~(size_t)15) + (size_t)sky_queue_words<true>() * 4u * (kPersistentBlock / 32);
    PersistentFn fn;
    int blocks;
    uint32_t knobs;
    cudaError_t e = persistent_grid(tune, device, smem, true, ext ? kFeatAll : 0u, fn, blocks, knobs);
    if (e != cudaSuccess) return e;
    knobs |= shlevels << 24;
    fn<<<blocks, kPersistentBlock, smem, st>>>(DevScene{}, DevParams{}, TileArgs{}, mie_pack, nullptr, nullptr, C, Q,
                                               knobs, B);
    return cudaGetLastError();
}

cudaError_t launch_batch_view(const DevScene &S, const DevParams &P, const TileArgs &A, const void *mie_pack,
                              float4 *sun_out, float4 *sky_out, DevCounters *C, WorkQueue *Q,
                              const unsigned long long *step, const Tuning &tune_in, int device, cudaStream_t st) {
    if (A.n_paths == 0) return cudaSuccess;
    size_t smem = mie_smem(P);
    const uint32_t feat = frame_features(S, P);
    Tuning tune = tune_in;
    const uint32_t shlevels = shared_stack_plan(tune, feat, S.stack_levels, smem);
    TileArgs Ad = A;
    Ad.defer_sky = (feat == 0 && !P.finite_paths) ? 1u : 0u;
    if (Ad.defer_sky) smem = ((smem + 15) & ~(size_t)15) + (size_t)sky_queue_words<false>() * 4u * (kPersistentBlock / 32);
    PersistentFn fn;
    int blocks;
    uint32_t knobs;
    cudaError_t e = persistent_grid(tune, device, smem, false, feat, fn, blocks, knobs);
    if (e != cudaSuccess) return e;
    knobs |= shlevels << 24;
    BatchArgs B{};
    B.step = step;
    fn<<<blocks, kPersistentBlock, smem, st>>>(S, P, Ad, mie_pack, sun_out, sky_out, C, Q, knobs, B);
    return cudaGetLastError();
}

cudaError_t launch_batch_step(unsigned long long *step, cudaStream_t st) {
    batch_step_kernel<<<1, 1, 0, st>>>(step);
    return cudaGetLastError();
}

cudaError_t launch_render_batch(const BatchArgs &B, const DevParams &P0, const void *mie_pack, DevCounters *C,
                                WorkQueue *Q, unsigned long long *step, const Tuning &tune, bool ext,
                                uint32_t stack_levels, int device, cudaStream_t st, const BatchLists &lists) {
    cudaError_t e = cudaMemsetAsync(Q, 0, sizeof(WorkQueue), st);
    if (e != cudaSuccess) return e;
    e = launch_batch_lists(B, lists, st);  // the views' TileArgs point into these lists
    if (e != cudaSuccess) return e;
    e = launch_batch_kernel(B, P0, mie_pack, C, Q, tune, ext, stack_levels, device, st);
    if (e != cudaSuccess) return e;
    return launch_batch_step(step, st);
}

cudaError_t launch_add_counters(DevCounters *dst, const DevCounters *src, cudaStream_t st) {
    add_counters_kernel<<<1, 1, 0, st>>>(dst, src);
    return cudaGetLastError();
}

cudaError_t launch_probe_leaf(const DevScene &S, const float *ro, const float *rd, uint32_t n, uint32_t maxn,
                              uint32_t *nodes, float *tr0, float *tr1, uint32_t *counts, cudaStream_t st) {
    probe_leaf_kernel<<<(n + 127) / 128, 128, 0, st>>>(S, ro, rd, n, maxn, nodes, tr0, tr1, counts);
    return cudaGetLastError();
}

cudaError_t launch_probe_occlusion(const DevScene &S, const float *ro, const float *rd, uint32_t n, uint32_t *hit,
                                   cudaStream_t st) {
    probe_occlusion_kernel<<<(n + 127) / 128, 128, 0, st>>>(S, ro, rd, n, hit);
    return cudaGetLastError();
}

cudaError_t launch_probe_density(const DevScene &S, const uint32_t *nodes, const float *pts, uint32_t n, float *out,
                                 cudaStream_t st) {
    probe_density_kernel<<<(n + 127) / 128, 128, 0, st>>>(S, nodes, pts, n, out);
    return cudaGetLastError();
}

cudaError_t launch_probe_paths(const DevScene &S, const DevParams &P, const void *mie_pack, const uint32_t *px,
                               const uint32_t *py, const uint64_t *sample, uint32_t n, uint64_t seed,
                               float4 *out_sun, float4 *out_sky, DevCounters *C, cudaStream_t st) {
    const cudaError_t e = allow_smem(probe_paths_kernel, mie_smem(P));
    if (e != cudaSuccess) return e;
    probe_paths_kernel<<<(n + 127) / 128, 128, mie_smem(P), st>>>(S, P, mie_pack, px, py, sample, n, seed, out_sun,
                                                                  out_sky, C);
    return cudaGetLastError();
}

cudaError_t launch_probe_sampler(const DevParams &P, const void *mie_pack, uint32_t what, const float *in, uint32_t n,
                                 float *out, cudaStream_t st) {
    const cudaError_t e = allow_smem(probe_sampler_kernel, mie_smem(P));
    if (e != cudaSuccess) return e;
    probe_sampler_kernel<<<(n + 127) / 128, 128, mie_smem(P), st>>>(P, mie_pack, what, in, n, out);
    return cudaGetLastError();
}

cudaError_t launch_probe_transmittance(const DevScene &S, const DevParams &P, const float *ro, const float *rd,
                                       uint32_t n_rays, uint64_t nsamp, uint64_t seed, unsigned long long *escapes,
                                       cudaStream_t st) {
    const uint64_t threads = ((nsamp + 63) / 64) * n_rays;
    const uint64_t blocks = (threads + 127) / 128;
    if (blocks == 0) return cudaSuccess;
    if (blocks > 0x7fffffffull) return cudaErrorInvalidValue;
    probe_transmittance_kernel<<<(unsigned)blocks, 128, 0, st>>>(S, P, ro, rd, n_rays, nsamp, seed, escapes);
    return cudaGetLastError();
}


uint32_t adjoint_slots() { return kSlots; }

cudaError_t launch_adjoint_tile(const DevScene &S, const DevParams &P, const TileArgs &A, const void *mie_pack,
                                const float4 *dsun, const float4 *dsky, float *grad, float *copies_buf,
                                uint32_t copies, void *records, uint64_t chunk, double *grad_albedo, double *slots,
                                DevCounters *C, cudaStream_t st) {
    if (A.n_paths == 0) return cudaSuccess;
    if (chunk == 0 || (chunk + kRenderBlock - 1) / kRenderBlock > 0x7fffffffull) return cudaErrorInvalidValue;
    const size_t stride = (size_t)S.n_leaves * kBrick;
    const bool spread = copies > 1 && copies_buf;
    cudaError_t e;
    if (spread) {
        e = cudaMemsetAsync(copies_buf, 0, sizeof(float) * stride * copies, st);
        if (e != cudaSuccess) return e;
    }
    const size_t smem = mie_smem(P);
    const uint32_t feat = frame_features(S, P);
    e = allow_smem(feat ? adjoint_totals_kernel<kFeatAll> : adjoint_totals_kernel<0>, smem);
    if (e != cudaSuccess) return e;
    e = allow_smem(feat ? adjoint_scatter_kernel<kFeatAll> : adjoint_scatter_kernel<0>, smem);
    if (e != cudaSuccess) return e;
    PathRecord *rec = (PathRecord *)records;
    for (uint64_t p0 = 0; p0 < A.n_paths; p0 += chunk) {
        const uint64_t n = A.n_paths - p0 < chunk ? A.n_paths - p0 : chunk;
        const unsigned blocks = (unsigned)((n + kRenderBlock - 1) / kRenderBlock);
        if (feat)
            adjoint_totals_kernel<kFeatAll><<<blocks, kRenderBlock, smem, st>>>(S, P, A, p0, n, mie_pack, dsun, dsky,
                                                                             rec, slots, C);
        else
            adjoint_totals_kernel<0><<<blocks, kRenderBlock, smem, st>>>(S, P, A, p0, n, mie_pack, dsun, dsky, rec,
                                                                      slots, C);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (feat)
            adjoint_scatter_kernel<kFeatAll><<<blocks, kRenderBlock, smem, st>>>(
                S, P, A, p0, n, mie_pack, dsun, dsky, rec, spread ? copies_buf : grad, spread ? copies : 1u, stride, C);
        else
            adjoint_scatter_kernel<0><<<blocks, kRenderBlock, smem, st>>>(
                S, P, A, p0, n, mie_pack, dsun, dsky, rec, spread ? copies_buf : grad, spread ? copies : 1u, stride, C);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (spread) {
        sum_copies_kernel<<<592, 256, 0, st>>>(grad, copies_buf, copies, stride);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    sum_slots_kernel<<<1, 256, 0, st>>>(grad_albedo, slots);
    return cudaGetLastError();
}

cudaError_t launch_reweighted_loss(const DevScene &S, const DevParams &P, const TileArgs &A, const void *mie_pack,
                                   const float4 *dsun, const float4 *dsky, const float *pert, double *loss,
                                   double *slots, DevCounters *C, cudaStream_t st) {
    if (A.n_paths > 0) {
        const uint64_t blocks = (A.n_paths + kRenderBlock - 1) / kRenderBlock;
        if (blocks > 0x7fffffffull) return cudaErrorInvalidValue;
        const auto fn = frame_features(S, P) ? reweighted_loss_kernel<kFeatAll> : reweighted_loss_kernel<0>;
        cudaError_t e = allow_smem(fn, mie_smem(P));
        if (e != cudaSuccess) return e;
        fn<<<(unsigned)blocks, kRenderBlock, mie_smem(P), st>>>(S, P, A, mie_pack, dsun, dsky, pert, slots, C);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    sum_slots_kernel<<<1, 256, 0, st>>>(loss, slots);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_transmittance(const DevScene &S, const DevParams &P, const float *ro, const float *rd,
                                         const float *wr, uint32_t n_rays, uint64_t nsamp, uint64_t seed, float *grad,
                                         unsigned long long *escapes, cudaStream_t st) {
    const uint64_t threads = ((nsamp + 63) / 64) * n_rays;
    const uint64_t blocks = (threads + 127) / 128;
    if (blocks == 0) return cudaSuccess;
    if (blocks > 0x7fffffffull) return cudaErrorInvalidValue;
    adjoint_transmittance_kernel<<<(unsigned)blocks, 128, 0, st>>>(S, P, ro, rd, wr, n_rays, nsamp, seed, grad,
                                                                   escapes);
    return cudaGetLastError();
}

cudaError_t launch_leaf_majorants(float4 *leaf, const uint32_t *leaf_nodes, uint32_t n_leafnodes, const float *bricks,
                                  float scale, cudaStream_t st) {
    if (n_leafnodes == 0) return cudaSuccess;
    leaf_majorant_kernel<<<n_leafnodes, 128, 0, st>>>(leaf, leaf_nodes, n_leafnodes, bricks, scale);
    return cudaGetLastError();
}

}  // namespace dr
