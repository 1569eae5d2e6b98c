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
__device__ __forceinline__ bool stage_mie(const void *src, uint32_t n, unsigned char *smem, uint64_t *mbar) {
    const uint32_t bytes = n * 20u;
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
__global__ void __launch_bounds__(kRenderBlock) render_tile_kernel(DevScene S, DevParams P, TileArgs A,
                                                                   const void *mie_pack, float4 *sun_out,
                                                                   float4 *sky_out, DevCounters *C) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint64_t mbar;
    const bool staged = stage_mie(mie_pack, P.mie_n, smem, &mbar);
    MieSmem M{reinterpret_cast<float4 *>(smem), reinterpret_cast<float *>(smem + 16u * P.mie_n), P.mie_n};
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
            path_sample(S, P, M, A.x0 + i, A.y0 + j, A.seed, A.sample_base + s, sa, sk, nstack, cnt);
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

// ---- parity probes ------------------------------------------------------------
__global__ void probe_leaf_kernel(DevScene S, const float *ro, const float *rd, uint32_t n, uint32_t maxn,
                                  uint32_t *nodes, float *tr0, float *tr1, uint32_t *counts) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const float o[3] = {ro[3 * r], ro[3 * r + 1], ro[3 * r + 2]}, d[3] = {rd[3 * r], rd[3 * r + 1], rd[3 * r + 2]};
    Trav T;
    Count cnt;
    cnt.zero();
    uint32_t nstack[kMaxDepth];
    trav_init(T, S, o, d, cnt);
    uint32_t k = 0, leaf;
    float a, b;
    while (k < maxn && trav_next(T, S, nstack, leaf, a, b, cnt)) {
        nodes[(size_t)r * maxn + k] = leaf;
        tr0[(size_t)r * maxn + k] = a;
        tr1[(size_t)r * maxn + k] = b;
        ++k;
    }
    counts[r] = k;
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
    const bool staged = stage_mie(mie_pack, P.mie_n, smem, &mbar);
    MieSmem M{reinterpret_cast<float4 *>(smem), reinterpret_cast<float *>(smem + 16u * P.mie_n), P.mie_n};
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
    const bool staged = stage_mie(mie_pack, P.mie_n, smem, &mbar);
    MieSmem M{reinterpret_cast<float4 *>(smem), reinterpret_cast<float *>(smem + 16u * P.mie_n), P.mie_n};
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
        esc += track(S, P, o, d, g, 3.402823466e+38f, td, nstack, cnt) ? 1u : 0u;
    }
    atomicAdd(&escapes[r], (unsigned long long)esc);
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
static size_t mie_smem(const DevParams &P) { return (size_t)P.mie_n * 20u; }

cudaError_t launch_render_tile(const DevScene &S, const DevParams &P, const TileArgs &A, const void *mie_pack,
                               float4 *sun_out, float4 *sky_out, DevCounters *C, cudaStream_t st) {
    if (A.n_paths == 0) return cudaSuccess;
    const uint64_t blocks = (A.n_paths + kRenderBlock - 1) / kRenderBlock;
    if (blocks > 0x7fffffffull) return cudaErrorInvalidValue;
    render_tile_kernel<<<(unsigned)blocks, kRenderBlock, mie_smem(P), st>>>(S, P, A, mie_pack, sun_out, sky_out, C);
    return cudaGetLastError();
}

cudaError_t launch_probe_leaf(const DevScene &S, const float *ro, const float *rd, uint32_t n, uint32_t maxn,
                              uint32_t *nodes, float *tr0, float *tr1, uint32_t *counts, cudaStream_t st) {
    probe_leaf_kernel<<<(n + 127) / 128, 128, 0, st>>>(S, ro, rd, n, maxn, nodes, tr0, tr1, counts);
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
    probe_paths_kernel<<<(n + 127) / 128, 128, mie_smem(P), st>>>(S, P, mie_pack, px, py, sample, n, seed, out_sun,
                                                                  out_sky, C);
    return cudaGetLastError();
}

cudaError_t launch_probe_sampler(const DevParams &P, const void *mie_pack, uint32_t what, const float *in, uint32_t n,
                                 float *out, cudaStream_t st) {
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

}  // namespace dr
