// Device code of the droplet_b200 hot path.  Compiled with -fmad=false: every
// multiply and add below rounds separately, exactly as the reference's SSE4
// build does (src/smmath.inl madd/msub are mul+add there); fused operations are
// written explicitly as fmaf().  With IEEE division and square root (nvcc's
// defaults) this reproduces the reference's binary32 arithmetic for the
// octree traversal, leaf intervals and brick lookups bit for bit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "dr_internal.h"

namespace dr {

// ---- comparisons with the reference's semantics --------------------------
__device__ __forceinline__ float sse_max(float a, float b) { return a > b ? a : b; }  // _mm_max_ps(a, b)
__device__ __forceinline__ float sse_min(float a, float b) { return a < b ? a : b; }  // _mm_min_ps(a, b)
__device__ __forceinline__ float std_max(float a, float b) { return (a < b) ? b : a; } // std::max
__device__ __forceinline__ float std_min(float a, float b) { return (b < a) ? b : a; } // std::min
__device__ __forceinline__ float lerp_ref(float a, float b, float t) { return t * (b - a) + a; }  // t.madd(b-a, a)

// n / d for the FastDiv record of d (exact for every 32-bit n, see make_fastdiv)
__device__ __forceinline__ uint32_t fastdiv(uint32_t n, const FastDiv &f) {
    const uint32_t t = __umulhi(n, f.m);
    return (t + ((n - t) >> f.s1)) >> f.s2;
}
// sfloat1::saturate = _mm_max_ps(_mm_min_ps(x, 1), 0): NaN gives 1.  The NaN case
// is explicit so that no rewrite into a hardware saturate (NaN -> 0) applies.
__device__ __forceinline__ float sat_ref(float x) { return x != x ? 1.0f : sse_max(sse_min(x, 1.0f), 0.0f); }

// ---- bit-reproducible transcendentals --------------------------------------
// Same operation sequences as the CPU restatement, built from IEEE binary32
// operations and explicit fused multiply-adds:
//   log : e ln2 + 2 atanh(s), s = (m-1)/(m+1), atanh by Maclaurin series to s^9
//         (|s| <= 0.1716: the next term is below 2e-9 relative)
//   exp : Cody-Waite reduction by ln2, Taylor series to r^7 (|r| <= ln2/2: the
//         next term is below 8e-9 relative)
//   sincos: Cody-Waite reduction by pi/2 (three parts), Taylor series of sin to
//         r^9 and cos to r^10 on |r| <= pi/4 (next terms below 3e-9)
//   x^1.5 : x sqrt(x)
constexpr float kLn2Hi = 0.693115234375f;
constexpr float kLn2Lo = 3.19461833e-05f;
constexpr float kPio2_1 = 1.5703125f;
constexpr float kPio2_2 = 4.83751297e-04f;
constexpr float kPio2_3 = 7.54979013e-08f;
constexpr float kPi = 3.14159265358979f;   // SM_PI, src/smmath.inl:16

__device__ __forceinline__ float dlog(float x) {
    if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : __int_as_float(0x7fc00000);
    if (x == INFINITY) return x;
    int e = 0;
    uint32_t u = __float_as_uint(x);
    if (u < 0x00800000u) { x = x * 16777216.0f; u = __float_as_uint(x); e = -24; }
    e += (int)(u >> 23) - 127;
    float m = __uint_as_float((u & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
    float s = (m - 1.0f) / (m + 1.0f);
    float s2 = s * s;
    float p = 0.111111111f;
    p = fmaf(p, s2, 0.142857143f);
    p = fmaf(p, s2, 0.2f);
    p = fmaf(p, s2, 0.333333333f);
    float t = s * s2;
    float atanh2 = fmaf(t * p, 2.0f, s * 2.0f);
    float fe = (float)e;
    return fmaf(fe, kLn2Hi, fmaf(fe, kLn2Lo, atanh2));
}

__device__ __forceinline__ float dexp(float x) {
    if (x != x) return x;
    if (x > 88.7f) return INFINITY;
    if (x < -103.0f) return 0.0f;
    float k = floorf(fmaf(x, 1.44269504f, 0.5f));
    float r = fmaf(-k, kLn2Hi, x);
    r = fmaf(-k, kLn2Lo, r);
    float p = 1.98412698e-04f;
    p = fmaf(p, r, 1.38888889e-03f);
    p = fmaf(p, r, 8.33333333e-03f);
    p = fmaf(p, r, 4.16666667e-02f);
    p = fmaf(p, r, 1.66666667e-01f);
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    int ki = (int)k;
    int k1 = ki / 2, k2 = ki - k1;
    float s1 = __uint_as_float((uint32_t)(k1 + 127) << 23);
    float s2 = __uint_as_float((uint32_t)(k2 + 127) << 23);
    return (p * s1) * s2;
}

__device__ __forceinline__ float dpow(float x, float y) {
    if (x == 0.0f) return y > 0.0f ? 0.0f : (y == 0.0f ? 1.0f : INFINITY);
    if (x < 0.0f || x != x) return __int_as_float(0x7fc00000);
    return dexp(y * dlog(x));
}

// x^1.5 for x >= 0 (the sky's and HG's exponent); negative x or NaN gives NaN.
__device__ __forceinline__ float dpow15(float x) {
    if (x < 0.0f || x != x) return __int_as_float(0x7fc00000);
    return x * sqrtf(x);
}

__device__ __forceinline__ void dsincos(float x, float *ps, float *pc) {
    float k = rintf(x * 0.636619772f);
    float r = fmaf(-k, kPio2_1, x);
    r = fmaf(-k, kPio2_2, r);
    r = fmaf(-k, kPio2_3, r);
    float r2 = r * r;
    float sp = 2.75573192e-06f;
    sp = fmaf(sp, r2, -1.98412698e-04f);
    sp = fmaf(sp, r2, 8.33333333e-03f);
    sp = fmaf(sp, r2, -1.66666667e-01f);
    float sn = fmaf(sp * r2, r, r);
    float cp = -2.75573192e-07f;
    cp = fmaf(cp, r2, 2.48015873e-05f);
    cp = fmaf(cp, r2, -1.38888889e-03f);
    cp = fmaf(cp, r2, 4.16666667e-02f);
    cp = fmaf(cp, r2, -0.5f);
    float cs = fmaf(cp, r2, 1.0f);
    int q = ((int)k) & 3;
    float s, c;
    if (q == 0) { s = sn; c = cs; }
    else if (q == 1) { s = cs; c = -sn; }
    else if (q == 2) { s = -sn; c = -cs; }
    else { s = -cs; c = sn; }
    *ps = s;
    *pc = c;
}

// The reference's polynomial arccos, src/smmath.inl:414-420.
__device__ __forceinline__ float acos_ref(float s) {
    float z = 0.0f - s;
    float x = z > s ? z : s;
    float r = -0.0187293f * x + 0.0742610f;
    r = r * x - 0.2121144f;
    r = r * x + 1.5707288f;
    r = r * sqrtf(1.0f - x);
    bool n = s < 0.0f;
    r = r - (n ? 2.0f * r : 0.0f);
    return (n ? kPi : 0.0f) + r;
}

// ---- PCG32 (O'Neill 2014, XSH-RR) with SplitMix64-hashed streams ----------
struct Rng {
    uint64_t state, inc;
    __device__ __forceinline__ uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ull + inc;
        uint32_t xs = (uint32_t)(((old >> 18) ^ old) >> 27);
        uint32_t rot = (uint32_t)(old >> 59);
        return __funnelshift_r(xs, xs, rot);
    }
    // (2k+1) 2^-24 on the open interval (0,1)
    __device__ __forceinline__ float uniform() {
        return (float)(((next() >> 9) << 1) | 1u) * 5.96046448e-08f;
    }
};

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ Rng rng_seed(uint64_t seed, uint64_t pixel, uint64_t sample) {
    uint64_t a = mix64(seed ^ mix64(pixel * 0x9e3779b97f4a7c15ull + sample));
    uint64_t b = mix64(a + 0x632be59bd9b4e019ull);
    Rng g;
    g.state = 0u;
    g.inc = (b << 1) | 1u;
    (void)g.next();
    g.state += a;
    (void)g.next();
    return g;
}

// ---- per-thread counters ----------------------------------------------------
struct Count {
    uint32_t vertices, node_visits, density_lookups, mie_evals, gave_up;
    __device__ __forceinline__ void zero() { vertices = node_visits = density_lookups = mie_evals = gave_up = 0; }
};

// ---- octree traversal ----------------------------------------------------
// The reference's step traverser (src/KernelOctree.cpp:230-349) keeps t0, t1,
// tm for all 16 levels.  Here only the current internal node's (t0, t1) stay
// in registers; ancestor node ids and the ancestors' (t0, t1) live in a stack
// (per-thread arrays in local memory, or a per-lane column of shared memory),
// written on each descent and read back on a pop.  Without the intervals (the
// probes) a pop
// rebuilds the interval from the root by replaying the child slots (3 bits per
// level), which repeats the reference's tm = 0.5f*(t0+t1) selections: the same
// floats either way.
// Child numbers here are in the node record's slot order (x bit 0, y bit 1, z
// bit 2, src/scene.cpp:285); Revelles' paper and src/KernelOctree.cpp number
// them with x in bit 2 and z in bit 0 and remap through nla = {0,4,2,6,1,5,3,7}.
// The decisions are the same; in slot order the remap is one XOR with the
// mirror mask.
__device__ __forceinline__ uint32_t first_node(const float t0[3], const float tm[3]) {
    // the entry axis: x when t0.x exceeds both others, y when t0.x <= t0.y and
    // t0.y > t0.z, else z (the reference's branches, NaN compares false); the
    // first child has the bit of every other axis whose midplane lies before
    // the entry.  Written with selects: the entry axis's own bit is never set
    // (tm >= t0 on that axis, or NaN), and it is cleared all the same.
    const bool xy = t0[0] > t0[1];
    const bool ax = xy && (t0[0] > t0[2]);
    const bool ay = !xy && (t0[1] > t0[2]);
    const float te = ax ? t0[0] : (ay ? t0[1] : t0[2]);
    const uint32_t own = ax ? 1u : (ay ? 2u : 4u);
    const uint32_t a = (tm[0] < te ? 1u : 0u) | (tm[1] < te ? 2u : 0u) | (tm[2] < te ? 4u : 0u);
    return a & ~own;
}

__device__ __forceinline__ uint32_t child_entry(const DevScene &S, uint32_t node, uint32_t slot) {
    const uint32_t *c = reinterpret_cast<const uint32_t *>(S.child) + 8u * node + slot;
    return __ldg(c);
}

struct Trav {
    float t0r[3], t1r[3];
    float t0[3], t1[3];
    uint64_t slots, tns;
    uint32_t a, node, tn;
    int l;
    bool active;
    bool fresh;  // the origin lies in the root box: the first call descends straight to it
};

__device__ __forceinline__ void trav_init(Trav &T, const DevScene &S, const float ro[3], const float rd[3],
                                          Count &cnt) {
    float ros[3], rds[3];
    for (int k = 0; k < 3; ++k) {
        ros[k] = (ro[k] - S.root_ce[k]) + S.root_ce[3];
        rds[k] = rd[k];
    }
    uint32_t a = 0;
    // mirror mask in slot order (x bit 0, z bit 2), see first_node
    if (rds[0] < 0.0f) { ros[0] = 2.0f * S.root_ce[3] - ros[0]; rds[0] = -rds[0]; a |= 1; }
    if (rds[1] < 0.0f) { ros[1] = 2.0f * S.root_ce[3] - ros[1]; rds[1] = -rds[1]; a |= 2; }
    if (rds[2] < 0.0f) { ros[2] = 2.0f * S.root_ce[3] - ros[2]; rds[2] = -rds[2]; a |= 4; }
    const float mx = 2.0f * S.root_ce[3];
    for (int k = 0; k < 3; ++k) {
        T.t0r[k] = (0.0f - ros[k]) / rds[k];
        T.t1r[k] = (mx - ros[k]) / rds[k];
    }
    T.a = a;
    T.active = std_max(std_max(T.t0r[0], T.t0r[1]), T.t0r[2]) < std_min(std_min(T.t1r[0], T.t1r[1]), T.t1r[2]);
    if (T.active && (T.t1r[0] < 0.0f || T.t1r[1] < 0.0f || T.t1r[2] < 0.0f)) T.active = false;
    if (T.active) {
        ++cnt.node_visits;  // the root is examined; it is never a leaf (depth >= 2)
        T.l = 0;
        T.node = 0;
        T.slots = 0;
        T.tns = 0;
        float tm[3];
        for (int k = 0; k < 3; ++k) {
            T.t0[k] = T.t0r[k];
            T.t1[k] = T.t1r[k];
            tm[k] = 0.5f * (T.t0[k] + T.t1[k]);
        }
        T.tn = first_node(T.t0, tm);
    }
    // A segment that starts inside the root box (max t0 <= 0; finite planes,
    // i.e. no zero direction component) can start its traversal at the node
    // holding its origin: see trav_next_s.
    T.fresh = T.active && std_max(std_max(T.t0r[0], T.t0r[1]), T.t0r[2]) <= 0.0f && isfinite(T.t0r[0]) &&
              isfinite(T.t0r[1]) && isfinite(T.t0r[2]) && isfinite(T.t1r[0]) && isfinite(T.t1r[1]) &&
              isfinite(T.t1r[2]);
}

// Up to `budget` loop iterations towards the next leaf, each one child
// examination preceded by the pops of exhausted nodes (at most one per level,
// so that lanes that pop examine in the same iteration as lanes that do not):
// returns kTravLeaf with (leaf, tra, trb), kTravDone when the ray has no further
// leaf, or kTravMore when the budget ran out first (call again: the state is
// complete after every iteration).
// The stack (see LocalStack / SharedStack) saves the ancestors' node ids and,
// when it has room for them, their intervals at each descent, read back on a
// pop; without intervals a pop rebuilds the interval from the root by replaying
// the 3-bit child slots (the same floats).
enum : uint32_t { kTravMore = 0, kTravLeaf = 1, kTravDone = 2 };

// Where the traversal keeps its ancestors.  push(T, l, cb) saves level l at a
// descent into the child with slot bits cb (T still holds the parent: its node,
// next child T.tn and interval); pop(T, l) restores level l's node and next
// child and, when the stack keeps intervals, its interval (returns true).
// LocalStack: node ids and intervals in the lane's own arrays (local memory),
// the next child at each level in 4-bit fields of T.tns; without `iv` a pop
// replays the interval from the root (returns false).
// SharedStack: level l of this lane at col[(kShWords l + k) * STRIDE], one
// column per lane of the block, so the lanes of a warp touch 32 consecutive
// words whatever their levels (no bank conflicts).  k = 0..2: per axis, the
// parent's bound the child does not share (t0 where the child lies in the upper
// half, else t1); k = 3: the node id (below 2^25), the child's slot bits at 25-27
// and the next child at 28-31.  A pop happens when the child's subtree is done,
// with the child's interval still in T: the child shares the parent's t1 on
// the axes where its bit is set and the parent's t0 elsewhere, so the saved
// bound completes the parent's interval with the same floats.  `levels` entries
// fit, and a descent that would need more gives up like the reference's depth
// limit (the host sizes the stack from the octree's depth, so that never happens).
constexpr int kShWords = 4;

struct LocalStack {
    uint32_t *nodes;
    float (*iv)[6];
    __device__ __forceinline__ void push(Trav &T, int l, uint32_t) const {
        nodes[l] = T.node;
        T.tns = (T.tns & ~(15ull << (4 * l))) | ((uint64_t)T.tn << (4 * l));
        if (iv) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                iv[l][k] = T.t0[k];
                iv[l][3 + k] = T.t1[k];
            }
        }
    }
    __device__ __forceinline__ bool pop(Trav &T, int l) const {
        T.node = nodes[l];
        T.tn = (uint32_t)(T.tns >> (4 * l)) & 15u;
        if (!iv) return false;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            T.t0[k] = iv[l][k];
            T.t1[k] = iv[l][3 + k];
        }
        return true;
    }
    __device__ __forceinline__ bool has_iv() const { return iv != nullptr; }
    __device__ __forceinline__ bool full(int l) const { return l + 1 >= kMaxDepth - 1; }
};

template <int STRIDE>
struct SharedStack {
    float *col;
    int levels;
    __device__ __forceinline__ void push(Trav &T, int l, uint32_t cb) const {
        col[(kShWords * l + 0) * STRIDE] = (cb & 1u) ? T.t0[0] : T.t1[0];
        col[(kShWords * l + 1) * STRIDE] = (cb & 2u) ? T.t0[1] : T.t1[1];
        col[(kShWords * l + 2) * STRIDE] = (cb & 4u) ? T.t0[2] : T.t1[2];
        col[(kShWords * l + 3) * STRIDE] = __uint_as_float(T.node | (cb << 25) | (T.tn << 28));
    }
    __device__ __forceinline__ bool pop(Trav &T, int l) const {
        const uint32_t w = __float_as_uint(col[(kShWords * l + 3) * STRIDE]);
        T.node = w & 0x01ffffffu;
        T.tn = w >> 28;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float o = col[(kShWords * l + k) * STRIDE];
            if ((w >> (25 + k)) & 1u) T.t0[k] = o;
            else T.t1[k] = o;
        }
        return true;
    }
    __device__ __forceinline__ bool has_iv() const { return true; }
    // levels <= 13 (the host allows at most 7), so the reference's depth limit is implied
    __device__ __forceinline__ bool full(int l) const { return l >= levels; }
};

template <class ST>
__device__ __forceinline__ uint32_t trav_next_s(Trav &T, const DevScene &S, const ST &stk, uint32_t &leaf,
                                                float &tra, float &trb, Count &cnt, uint32_t budget) {
    if (!T.active) return kTravDone;
    if (T.fresh) {
        // Straight descent to the child holding t = 0 at each level.  In the
        // examination order below (children in ray order from first_node),
        // every child before that one exits behind the origin (some c1 < 0)
        // and is skipped uncounted, so the state reached here -- stack
        // entries, next children, intervals, node visits -- is the state the
        // loop reaches when it arrives at that child.  The descent stops at a
        // leaf, an empty child or a full stack and leaves that child for the
        // loop to examine.  A leaf or an empty child reached this way is
        // examined here (both are not behind the origin).
        T.fresh = false;
        for (;;) {
            float tm[3], c0[3], c1[3];
            for (int k = 0; k < 3; ++k) tm[k] = 0.5f * (T.t0[k] + T.t1[k]);
            const uint32_t tn = (tm[0] < 0.0f ? 1u : 0u) | (tm[1] < 0.0f ? 2u : 0u) | (tm[2] < 0.0f ? 4u : 0u);
            const bool bx = tn & 1, by = tn & 2, bz = tn & 4;
            c0[0] = bx ? tm[0] : T.t0[0]; c1[0] = bx ? T.t1[0] : tm[0];
            c0[1] = by ? tm[1] : T.t0[1]; c1[1] = by ? T.t1[1] : tm[1];
            c0[2] = bz ? tm[2] : T.t0[2]; c1[2] = bz ? T.t1[2] : tm[2];
            const uint32_t child = child_entry(S, T.node, tn ^ T.a);
            const int l = T.l;
            if (stk.full(l) && child != 0u && !(child & kLeafBit)) {
                T.tn = tn;
                break;
            }
            // this child is what the loop below would examine next, and it is
            // not behind the origin (every c1 >= 0): its examination is done
            // here -- the next child, then an empty child is passed, a leaf
            // returned and an internal node entered, as in the loop
            const uint32_t eb = (c1[0] < c1[1]) ? ((c1[0] < c1[2]) ? 1u : 4u) : ((c1[1] < c1[2]) ? 2u : 4u);
            T.tn = (tn & eb) ? 8u : (tn | eb);
            if (child == 0u) break;
            ++cnt.node_visits;
            if (child & kLeafBit) {
                leaf = child & ~kLeafBit;
                tra = std_max(std_max(c0[0], c0[1]), c0[2]);
                trb = std_min(std_min(c1[0], c1[1]), c1[2]);
                return kTravLeaf;
            }
            stk.push(T, l, tn);
            if (!stk.has_iv()) T.slots = (T.slots & ~(7ull << (3 * l))) | ((uint64_t)tn << (3 * l));
            T.l = l + 1;
            T.node = child;
            for (int k = 0; k < 3; ++k) {
                T.t0[k] = c0[k];
                T.t1[k] = c1[k];
            }
        }
    }
    for (uint32_t it = 0;; ++it) {
        if (it == budget) return kTravMore;
        while (T.tn >= 8) {  // T.l falls by one per pop: at most kMaxDepth pops
            if (T.l == 0) {
                T.active = false;
                return kTravDone;
            }
            const int l = T.l - 1;
            T.l = l;
            if (stk.pop(T, l)) continue;
            float t0[3] = {T.t0r[0], T.t0r[1], T.t0r[2]}, t1[3] = {T.t1r[0], T.t1r[1], T.t1r[2]};
            for (int k = 0; k < l; ++k) {
                const uint32_t s = (uint32_t)(T.slots >> (3 * k)) & 7u;
                const float mx = 0.5f * (t0[0] + t1[0]), my = 0.5f * (t0[1] + t1[1]), mz = 0.5f * (t0[2] + t1[2]);
                if (s & 1) t0[0] = mx; else t1[0] = mx;
                if (s & 2) t0[1] = my; else t1[1] = my;
                if (s & 4) t0[2] = mz; else t1[2] = mz;
            }
            for (int k = 0; k < 3; ++k) {
                T.t0[k] = t0[k];
                T.t1[k] = t1[k];
            }
            continue;
        }
        const uint32_t tn = T.tn;
        float tm[3], c0[3], c1[3];
        for (int k = 0; k < 3; ++k) tm[k] = 0.5f * (T.t0[k] + T.t1[k]);
        const bool bx = tn & 1, by = tn & 2, bz = tn & 4;
        c0[0] = bx ? tm[0] : T.t0[0]; c1[0] = bx ? T.t1[0] : tm[0];
        c0[1] = by ? tm[1] : T.t0[1]; c1[1] = by ? T.t1[1] : tm[1];
        c0[2] = bz ? tm[2] : T.t0[2]; c1[2] = bz ? T.t1[2] : tm[2];
        // OctreeNextNode's choice (src/KernelOctree.cpp:62-71: x if t1.x is below
        // both others, else y if t1.y < t1.z, else z) as the exit axis's bit:
        // past the node's far side on that axis (bit set) the node is done (8)
        const uint32_t eb = (c1[0] < c1[1]) ? ((c1[0] < c1[2]) ? 1u : 4u) : ((c1[1] < c1[2]) ? 2u : 4u);
        T.tn = (tn & eb) ? 8u : (tn | eb);
        const uint32_t slot = tn ^ T.a;  // slot order throughout: no bit reversal (see first_node)
        const uint32_t child = child_entry(S, T.node, slot);
        if (c1[0] < 0.0f || c1[1] < 0.0f || c1[2] < 0.0f || child == 0u) continue;
        ++cnt.node_visits;
        if (child & kLeafBit) {
            leaf = child & ~kLeafBit;
            tra = std_max(std_max(c0[0], c0[1]), c0[2]);
            trb = std_min(std_min(c1[0], c1[1]), c1[2]);
            return kTravLeaf;
        }
        const int l = T.l;
        if (stk.full(l)) {  // an internal node at level 15 has no stack room (reference limit)
            T.active = false;
            ++cnt.gave_up;
            return kTravDone;
        }
        stk.push(T, l, tn);
        if (!stk.has_iv()) T.slots = (T.slots & ~(7ull << (3 * l))) | ((uint64_t)tn << (3 * l));  // replay path only
        T.l = l + 1;
        T.node = child;
        for (int k = 0; k < 3; ++k) {
            T.t0[k] = c0[k];
            T.t1[k] = c1[k];
            tm[k] = 0.5f * (c0[k] + c1[k]);
        }
        T.tn = first_node(T.t0, tm);
    }
}

__device__ __forceinline__ uint32_t trav_next_k(Trav &T, const DevScene &S, uint32_t *nstack, uint32_t &leaf,
                                                float &tra, float &trb, Count &cnt, uint32_t budget,
                                                float (*tstack)[6] = nullptr) {
    return trav_next_s(T, S, LocalStack{nstack, tstack}, leaf, tra, trb, cnt, budget);
}

__device__ __forceinline__ bool trav_next(Trav &T, const DevScene &S, uint32_t *nstack, uint32_t &leaf,
                                          float &tra, float &trb, Count &cnt) {
    return trav_next_k(T, S, nstack, leaf, tra, trb, cnt, 0xffffffffu) == kTravLeaf;
}

// ---- cell walk: the same leaf sequence without a stack -----------------------
// When every leaf sits at one depth L, the Revelles traversal above visits leaf
// cells of a 2^L grid.  Every t value it compares is a plane value: the root's
// (t0, t1) per axis, or a midpoint 0.5f*(lo + hi) of two coarser planes, so
// plane(k, i) for plane index i in [0, 2^L] is recomputed exactly by descending
// the binary subdivision (grid_plane).  In the mirrored frame:
//  * the first leaf is the cell containing te = max(t0) (first_node picks, at
//    every level, the upper half of axis k iff tm_k < te);
//  * leaving a cell, OctreeNextNode moves across the exit plane with the smallest t,
//    ties going to z, then y, then x; this choice is the same at every tree
//    level, since an ancestor's exit planes are never nearer than the cell's;
//  * entering the sibling subtree (2^t cells per axis, t = trailing zeros of the
//    new index), first_node's descent gives, in every other axis k, the cell
//    holding te = the crossed plane's t; that is the current cell unless its
//    entry plane equals te (a tie), which is the only case that re-descends;
//  * a cell is reported when it holds a leaf and no exit plane is negative (the
//    reference prunes nodes with any t1 < 0).
// Rays with a zero direction component give NaN planes, for which the tree's
// tie handling differs level by level: they use the stack traversal.  Empty
// 8^3 macro cells are crossed in one step with their macro-level exit planes.
struct Walk {
    float t0r[3], t1r[3];
    float N[3], X[3];      // entry / exit planes of the current cell
    uint32_t c[3];         // current leaf cell, mirrored frame
    uint32_t a;            // mirror bits, x = 4, y = 2, z = 1
    bool macro_mode;       // current macro cell is empty: step at macro granularity
    bool check;            // current cell not yet examined
};

// Plane value of plane index i in [0, n] between the root planes (lo, hi).
__device__ __forceinline__ float grid_plane(float lo, float hi, uint32_t i, uint32_t n) {
    if (i == 0) return lo;
    if (i >= n) return hi;
    uint32_t base = 0, span = n;
    for (int it = 0; it < 16; ++it) {
        span >>= 1;
        const float mid = 0.5f * (lo + hi);
        const uint32_t m = base + span;
        if (i == m) return mid;
        if (i < m) {
            hi = mid;
        } else {
            lo = mid;
            base = m;
        }
    }
    return lo;
}

__device__ __forceinline__ float sel3(int k, float a, float b, float c) { return k == 0 ? a : (k == 1 ? b : c); }

// first_node's descent inside [base, base + 2^t) of one axis for entry te:
// the cell index and its entry / exit planes.
__device__ __forceinline__ void grid_descend(float r0, float r1, uint32_t base, uint32_t t, float te, uint32_t n,
                                             uint32_t &c, float &N, float &X) {
    float lo = grid_plane(r0, r1, base, n), hi = grid_plane(r0, r1, base + (1u << t), n);
    uint32_t cc = base, span = 1u << t;
    for (uint32_t l = 0; l < t; ++l) {
        span >>= 1;
        const float mid = 0.5f * (lo + hi);
        if (mid < te) {
            lo = mid;
            cc += span;
        } else {
            hi = mid;
        }
    }
    c = cc;
    N = lo;
    X = hi;
}

__device__ __forceinline__ uint32_t grid_macro(const Walk &W, const DevScene &S) {
    const uint32_t x = ((W.a & 4u) ? S.n - 1 - W.c[0] : W.c[0]) >> 3;
    const uint32_t y = ((W.a & 2u) ? S.n - 1 - W.c[1] : W.c[1]) >> 3;
    const uint32_t z = ((W.a & 1u) ? S.n - 1 - W.c[2] : W.c[2]) >> 3;
    return __ldg(&S.macro[((size_t)z * S.mdim + y) * S.mdim + x]);
}

__device__ __forceinline__ void grid_macro_planes(Walk &W, const DevScene &S) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const uint32_t b = ((W.c[k] >> 3) + 1) << 3;
        W.X[k] = grid_plane(W.t0r[k], W.t1r[k], b < S.n ? b : S.n, S.n);
    }
}

// Returns 0: no leaf on this ray, 1: walk ready, 2: use the stack traversal.
__device__ __forceinline__ uint32_t walk_init(Walk &W, const DevScene &S, const float ro[3], const float rd[3],
                                              Count &cnt) {
    float ros[3], rds[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        ros[k] = (ro[k] - S.root_ce[k]) + S.root_ce[3];
        rds[k] = rd[k];
    }
    uint32_t a = 0;
    if (rds[0] < 0.0f) { ros[0] = 2.0f * S.root_ce[3] - ros[0]; rds[0] = -rds[0]; a |= 4; }
    if (rds[1] < 0.0f) { ros[1] = 2.0f * S.root_ce[3] - ros[1]; rds[1] = -rds[1]; a |= 2; }
    if (rds[2] < 0.0f) { ros[2] = 2.0f * S.root_ce[3] - ros[2]; rds[2] = -rds[2]; a |= 1; }
    const float mx = 2.0f * S.root_ce[3];
    bool finite = true;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        W.t0r[k] = (0.0f - ros[k]) / rds[k];
        W.t1r[k] = (mx - ros[k]) / rds[k];
        finite = finite && (rds[k] != 0.0f) && isfinite(W.t0r[k]) && isfinite(W.t1r[k]);
    }
    if (!finite || S.levels == 0) return 2u;
    W.a = a;
    if (!(std_max(std_max(W.t0r[0], W.t0r[1]), W.t0r[2]) < std_min(std_min(W.t1r[0], W.t1r[1]), W.t1r[2])))
        return 0u;
    if (W.t1r[0] < 0.0f || W.t1r[1] < 0.0f || W.t1r[2] < 0.0f) return 0u;
    ++cnt.node_visits;  // the root
    const float te = std_max(std_max(W.t0r[0], W.t0r[1]), W.t0r[2]);
#pragma unroll
    for (int k = 0; k < 3; ++k) grid_descend(W.t0r[k], W.t1r[k], 0u, S.levels, te, S.n, W.c[k], W.N[k], W.X[k]);
    W.macro_mode = grid_macro(W, S) == kNone;
    if (W.macro_mode) grid_macro_planes(W, S);
    W.check = true;
    return 1u;
}

// One step of the walk.  Returns 1 with a reported leaf, 0 after moving to the
// next cell (call again), 2 when the ray leaves the root box.
__device__ __forceinline__ uint32_t walk_step(Walk &W, const DevScene &S, uint32_t &leaf, float &tra, float &trb,
                                              Count &cnt) {
    if (W.check) {
        W.check = false;
        if (!W.macro_mode) {
            const uint32_t blk = grid_macro(W, S);
            const uint32_t x = ((W.a & 4u) ? S.n - 1 - W.c[0] : W.c[0]) & 7u;
            const uint32_t y = ((W.a & 2u) ? S.n - 1 - W.c[1] : W.c[1]) & 7u;
            const uint32_t z = ((W.a & 1u) ? S.n - 1 - W.c[2] : W.c[2]) & 7u;
            const uint32_t id = __ldg(&S.cells[(size_t)blk * 512u + z * 64u + y * 8u + x]);
            ++cnt.node_visits;
            if (id != kNone && !(W.X[0] < 0.0f) && !(W.X[1] < 0.0f) && !(W.X[2] < 0.0f)) {
                leaf = id;
                tra = std_max(std_max(W.N[0], W.N[1]), W.N[2]);
                trb = std_min(std_min(W.X[0], W.X[1]), W.X[2]);
                return 1u;
            }
        }
    }
    const int ax = (W.X[0] < W.X[1]) ? ((W.X[0] < W.X[2]) ? 0 : 2) : ((W.X[1] < W.X[2]) ? 1 : 2);
    const uint32_t cax = ax == 0 ? W.c[0] : (ax == 1 ? W.c[1] : W.c[2]);
    const uint32_t b = W.macro_mode ? ((cax >> 3) + 1) << 3 : cax + 1;
    if (b >= S.n) return 2u;
    const float Xa = sel3(ax, W.X[0], W.X[1], W.X[2]);
    const uint32_t t = (uint32_t)(__ffs((int)b) - 1);
    const bool was_macro = W.macro_mode;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (k == ax) {
            W.c[k] = b;
            W.N[k] = Xa;
        } else if (was_macro || (t != 0u && !(W.N[k] < Xa))) {
            grid_descend(W.t0r[k], W.t1r[k], W.c[k] & ~((1u << t) - 1u), t, Xa, S.n, W.c[k], W.N[k], W.X[k]);
        }
    }
    W.macro_mode = grid_macro(W, S) == kNone;
    if (W.macro_mode) {
        grid_macro_planes(W, S);
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (k == ax) W.X[k] = grid_plane(W.t0r[k], W.t1r[k], b + 1u, S.n);
    }
    W.check = true;
    return 0u;
}

// ---- brick lookup: SampleVoxelSpace, src/kernel.cpp:96-126 ----------------
__device__ __forceinline__ float sample_voxel_space(const float p[3], const float *__restrict__ v, const float4 ce) {
    const float nm1 = (float)kLvox - 1.0f;
    const float top = (float)(kLvox - 1);
    const float cc[3] = {ce.x, ce.y, ce.z};
    uint32_t ia[3], ib[3];
    float nl[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float ni = ((-0.5f * ((cc[k] - ce.w) - p[k])) * nm1) / ce.w;
        float nf = sse_max(floorf(ni), 0.0f);
        float nc = sse_min(ceilf(ni), nm1);
        nl[k] = ni - nf;
        nc = sse_max(sse_min(nc, top), 0.0f);
        nf = sse_max(sse_min(nf, top), 0.0f);
        ia[k] = (uint32_t)nf;
        ib[k] = (uint32_t)nc;
    }
    const uint32_t za = ia[2] * 64u, zb = ib[2] * 64u, ya = ia[1] * 8u, yb = ib[1] * 8u;
    const float u0 = lerp_ref(__ldg(v + za + ya + ia[0]), __ldg(v + za + ya + ib[0]), nl[0]);
    const float u1 = lerp_ref(__ldg(v + za + yb + ia[0]), __ldg(v + za + yb + ib[0]), nl[0]);
    const float u2 = lerp_ref(__ldg(v + zb + ya + ia[0]), __ldg(v + zb + ya + ib[0]), nl[0]);
    const float u3 = lerp_ref(__ldg(v + zb + yb + ia[0]), __ldg(v + zb + yb + ib[0]), nl[0]);
    const float v0 = lerp_ref(u0, u1, nl[1]);
    const float v1 = lerp_ref(u2, u3, nl[1]);
    return lerp_ref(v0, v1, nl[2]);
}

// Corner offsets (within the brick) and trilinear weights of the lookup above:
// rho = sum_k w[k] * v[idx[k]] (lerp_ref(a, b, t) = (1 - t) a + t b), the
// derivative of rho with respect to each brick sample.
__device__ __forceinline__ void voxel_weights(const float p[3], const float4 ce, uint32_t idx[8], float w[8]) {
    const float nm1 = (float)kLvox - 1.0f;
    const float top = (float)(kLvox - 1);
    const float cc[3] = {ce.x, ce.y, ce.z};
    uint32_t ia[3], ib[3];
    float nl[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float ni = ((-0.5f * ((cc[k] - ce.w) - p[k])) * nm1) / ce.w;
        float nf = sse_max(floorf(ni), 0.0f);
        float nc = sse_min(ceilf(ni), nm1);
        nl[k] = ni - nf;
        nc = sse_max(sse_min(nc, top), 0.0f);
        nf = sse_max(sse_min(nf, top), 0.0f);
        ia[k] = (uint32_t)nf;
        ib[k] = (uint32_t)nc;
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const uint32_t x = (c & 1) ? ib[0] : ia[0], y = (c & 2) ? ib[1] : ia[1], z = (c & 4) ? ib[2] : ia[2];
        idx[c] = z * 64u + y * 8u + x;
        w[c] = ((c & 1) ? nl[0] : 1.0f - nl[0]) * ((c & 2) ? nl[1] : 1.0f - nl[1]) * ((c & 4) ? nl[2] : 1.0f - nl[2]);
    }
}

// ---- phase function: MiePhase, src/KernelSampler.cpp:214-285 --------------
// Tables staged in shared memory: pdf as float4 (r, g, b, -), red CDF.
struct MieSmem {
    float4 *pdf;
    float *cdf;
    uint32_t n;
    const float4 *ex;  // exact-mode sampler table (2n + 1 float4) or null
};

__device__ __forceinline__ float3 mie_eval_rgb(const MieSmem &M, float ct) {
    float ct1 = sse_max(sse_min(ct, 1.0f), -1.0f);
    float a = acos_ref(0.0f - ct1) / kPi;
    float b = (float)M.n * a;
    float c = floorf(b);
    c = sse_min(c, (float)(M.n - 2));
    c = sse_max(c, 0.0f);
    const float t = b - c;
    const uint32_t X = (uint32_t)c;
    const float4 pa = M.pdf[X], pb = M.pdf[X + 1];
    return make_float3(lerp_ref(pa.x, pb.x, t), lerp_ref(pa.y, pb.y, t), lerp_ref(pa.z, pb.z, t));
}

__device__ __forceinline__ float mie_scan_cdf(const MieSmem &M, float ub, uint32_t i, float &t_out) {
    float b = sse_max(ub, (float)i);
    float c = sse_min(floorf(b), (float)(M.n - 1));
    float t = b - c;
    t_out = t;
    return lerp_ref(M.cdf[i], M.cdf[i + 1], t);
}

// The reference scans i = 0..n-2 and keeps the last step whose interpolated
// CDF is below u1; the predicate is non-decreasing in i, so bisection finds
// the same step in log2(n) probes.
__device__ __forceinline__ float mie_theta_ref(const MieSmem &M, float u1) {
    const float ub = (float)M.n * u1;
    uint32_t lo = 0, hi = M.n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        float t;
        if (mie_scan_cdf(M, ub, mid, t) < u1) lo = mid + 1;
        else hi = mid;
    }
    if (lo == 0) return 0.0f;
    float t;
    (void)mie_scan_cdf(M, ub, lo - 1, t);
    return (float)(lo - 1) / (float)M.n + t / (float)M.n;
}

// SamplingBasis, src/KernelSampler.cpp:145-154, and the direction composition
__device__ __forceinline__ void compose_dir(const float iv[3], float st, float ct, float ph, float out[3]) {
    const float len = sqrtf(iv[0] * iv[0] + 0.0f * 0.0f + iv[2] * iv[2]);
    const float b1[3] = {(0.0f - iv[2]) / len, 0.0f / len, iv[0] / len};
    const float b2[3] = {iv[1] * b1[2] - iv[2] * b1[1], iv[2] * b1[0] - iv[0] * b1[2], iv[0] * b1[1] - iv[1] * b1[0]};
    float sph, cph;
    dsincos(ph, &sph, &cph);
#pragma unroll
    for (int k = 0; k < 3; ++k) out[k] = ((b1[k] * st) * cph + (b2[k] * st) * sph) + iv[k] * ct;
}

// ---- exact-mode sampler (DR_PHASE_MIE_EXACT) ------------------------------------
// Inverts the CDF of f(phi) sin(phi), phi = acos(-ct), f the red table column
// interpolated linearly in phi as MiePhase::Evaluate does (knots k pi / n, the
// last bin extrapolated).  Bin k: f = f0 + beta x on x = phi - phi_k in [0, pi/n],
// mass H_k(x) = S[(f0 + beta x) sin x - beta (1 - cos x)] + C[f0 (1 - cos x) +
// beta (sin x - x cos x)] with S, C = sin, cos(phi_k) (the integral of f sin).
// Table per bin: (cdf_k, f0, beta, M_k), (S, C, pi/n, 0); then (1, 0, 0, 0).
// The bin comes from bisection on cdf_k, x from 8 safeguarded Newton steps.

// sin x, 1 - cos x and sin x - x cos x from their Taylor series (x <= pi/4)
__device__ __forceinline__ void local_trig(float x, float &sx, float &omc, float &sxc) {
    const float x2 = x * x;
    sx = x * (1.0f - (x2 / 6.0f) * (1.0f - (x2 / 20.0f) * (1.0f - (x2 / 42.0f) * (1.0f - x2 / 72.0f))));
    omc = (x2 / 2.0f) * (1.0f - (x2 / 12.0f) * (1.0f - (x2 / 30.0f) * (1.0f - (x2 / 56.0f) * (1.0f - x2 / 90.0f))));
    sxc = ((x2 * x) / 3.0f) * (1.0f - (x2 / 10.0f) * (1.0f - (x2 / 28.0f) * (1.0f - x2 / 54.0f)));
}

__device__ __forceinline__ void mie_exact_dir(const float4 *ex, uint32_t n, float u1, float &ct, float &st) {
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (ex[2 * mid].x <= u1) lo = mid;
        else hi = mid - 1;
    }
    const float4 a = ex[2 * lo], b = ex[2 * lo + 1];
    const float c0 = a.x, c1 = ex[2 * (lo + 1)].x;
    const float f0 = a.y, beta = a.z, mk = a.w, S = b.x, C = b.y, dx = b.z;
    const float d = c1 - c0;
    const float up = d > 0.0f ? (u1 - c0) / d : 0.5f;
    const float m = up * mk;
    float xl = 0.0f, xh = dx, x = up * dx;
#pragma unroll 1
    for (int it = 0; it < 8; ++it) {
        float sx, omc, sxc;
        local_trig(x, sx, omc, sxc);
        const float fx = f0 + beta * x;
        const float h = (S * (fx * sx - beta * omc) + C * (f0 * omc + beta * sxc)) - m;
        const float hp = fx * (S * (1.0f - omc) + C * sx);
        if (h > 0.0f) xh = x;
        else xl = x;
        float xn = hp > 0.0f ? x - h / hp : 0.5f * (xl + xh);
        if (!(xn > xl && xn < xh)) xn = 0.5f * (xl + xh);
        x = xn;
    }
    float sx, omc, sxc;
    local_trig(x, sx, omc, sxc);
    const float cx = 1.0f - omc;
    ct = 0.0f - (C * cx - S * sx);
    st = sse_max(S * cx + C * sx, 0.0f);
}

__device__ __forceinline__ void mie_sample(const MieSmem &M, const float iv[3], float u1, float u2, float out[3]) {
    if (M.ex) {
        float ct, st;
        mie_exact_dir(M.ex, M.n, u1, ct, st);
        compose_dir(iv, st, ct, (2.0f * kPi) * u2, out);
        return;
    }
    const float th = mie_theta_ref(M, u1) * kPi;
    const float ph = (2.0f * kPi) * u2;
    float s_, c_;
    dsincos(th, &s_, &c_);
    const float ct = -c_;
    const float st = sqrtf(sse_max(1.0f - ct * ct, 0.0f));
    compose_dir(iv, st, ct, ph, out);
}

// ---- phase function: HGPhase, src/KernelSampler.cpp:164-204 (DR_PHASE_HG) ----
// g = HGPhase::g1 (blcloudsampling.phasea); the same value for r, g and b.
__device__ __forceinline__ float hg_eval(float g, float ct) {
    const float den = 12.566371f * dpow15((1.0f + g * g) - (2.0f * g) * ct);  // float(4 SM_PI) * pow(., 1.5)
    return (1.0f - g * g) / den;
}

__device__ __forceinline__ void hg_sample(float g, const float iv[3], float u1, float u2, float out[3]) {
    const float sq = (1.0f - g * g) / ((1.0f - g) + (2.0f * g) * u1);
    const float ct = ((1.0f + g * g) - sq * sq) / (2.0f * g);
    const float st = sqrtf(sse_max(1.0f - ct * ct, 0.0f));
    compose_dir(iv, st, ct, (2.0f * kPi) * u2, out);
}

// The path's phase function: PhaseFunction::EvaluateRGB / Sample of the
// selected model (src/main.cpp:522-536).
__device__ __forceinline__ float3 phase_eval_rgb(const DevParams &P, const MieSmem &M, float ct) {
    if (P.phase_mode == kPhaseHG) {
        const float v = hg_eval(P.hg_g, ct);
        return make_float3(v, v, v);
    }
    return mie_eval_rgb(M, ct);
}

__device__ __forceinline__ void phase_sample(const DevParams &P, const MieSmem &M, const float iv[3], float u1, float u2,
                                             float out[3]) {
    if (P.phase_mode == kPhaseHG) hg_sample(P.hg_g, iv, u1, u2, out);
    else mie_sample(M, iv, u1, u2, out);
}

// ---- sun: SunLight, src/KernelSampler.cpp:318-345 --------------------------
__device__ __forceinline__ float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

__device__ __forceinline__ bool sun_hit(const DevParams &P, const float v[3]) {
    return dot3(v, P.sun_dir) > P.sun_cos;
}

__device__ __forceinline__ void sun_sample(const DevParams &P, float u1, float u2, float out[3]) {
    const float ctm = P.sun_cos;
    const float ct = (1.0f - u1) + u1 * ctm;
    const float st = sqrtf(1.0f - ct * ct);
    const float ph = (2.0f * kPi) * u2;
    compose_dir(P.sun_dir, st, ct, ph, out);
}

// ---- Hosek-Wilkie sky radiance as the reference evaluates it (src/kernel.cpp:329-360)
__device__ __forceinline__ float3 sky_eval(const DevParams &P, const float rd[3]) {
    const float *sd = P.sun_dir;
    const float rdz = rd[2];
    const float sth = sqrtf(1.0f - rd[2] * rd[2]);
    const float cth = rdz;
    const float slth = sqrtf(1.0f - sd[2] * sd[2]);
    const float clth = sd[2];
    const float slph = sd[1];
    const float clph = sd[0];
    const float rdd = rd[0] / rd[1];
    const float acr = 1.0f / sqrtf(rdd * rdd + 1.0f);
    const float czp = acr * (rdd * slph + clph);
    const float cph = (sth * slth) * czp + cth * clth;
    const float gmma = acos_ref(cph);
    const float gacs = sat_ref(cph);
    const float thcs = sse_max(rdz, 0.0f);
    const float raym = gacs * gacs;
    const float zenh = sqrtf(thcs);
    const float izen = 1.0f / (thcs + 0.01f);  // c1 / (thcs + 0.01) as c1 * izen: one division for three channels
    float out[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float *c = P.sky_cfg[i];
        const float expm = dexp(c[4] * gmma);
        const float miem = (1.0f + raym) / dpow15((1.0f + c[8] * c[8]) - (2.0f * c[8]) * gacs);
        float ca = (1.0f + c[0] * dexp(c[1] * izen)) *
                   ((((c[2] + c[3] * expm) + c[5] * raym) + c[6] * miem) + c[7] * zenh);
        ca = ca * P.sky_rad[i];
        out[i] = 1e-3f * dpow(ca, 2.2f);
    }
    return make_float3(out[0], out[1], out[2]);
}

// atan2 of smmath.inl (src/smmath.inl:430-445): polynomial in min/max ratio,
// then the octant corrections.
__device__ __forceinline__ float atan2_ref(float y, float x) {
    const float X = sse_max(0.0f - x, x), Y = sse_max(0.0f - y, y);
    float a = sse_min(X, Y) / sse_max(X, Y);
    const float b = a * a;
    float p = -0.013480470f * b + 0.057477314f;
    p = p * b - 0.121239071f;
    p = p * b + 0.195635925f;
    p = p * b - 0.332994597f;
    p = p * b + 0.999995630f;
    a = a * p;
    if (Y > X) a = 1.57079637f - a;  // float(0.5 SM_PI)
    if (x < 0.0f) a = kPi - a;
    if (y < 0.0f) a = 0.0f - a;
    return a;
}

// MapEnv::Evaluate (src/KernelSampler.cpp:384-417): bilinear lookup of an
// equirectangular RGBA map (theta rows from acos(-rd.z), phi columns from
// atan2(rd.y, -rd.x)); texel indices are formed in binary32 as there.
__device__ __forceinline__ float3 env_map_eval(const DevParams &P, const float rd[3]) {
    const float fw = (float)P.env_w, fh = (float)P.env_h;
    const float tha = acos_ref(0.0f - rd[2]) / kPi;
    const float thb = fh * sat_ref(tha);
    float thc = floorf(thb);
    thc = sse_min(thc, (float)(P.env_h - 2));
    thc = sse_max(thc, 0.0f);
    const float tht = thb - thc;
    const float pha = 0.5f + atan2_ref(rd[1], 0.0f - rd[0]) / 6.2831855f;  // float(2 SM_PI)
    const float phb = fw * sat_ref(pha);
    float phc = floorf(phb);
    phc = sse_min(phc, (float)(P.env_w - 2));
    phc = sse_max(phc, 0.0f);
    const float pht = phb - phc;
    const float4 *T = reinterpret_cast<const float4 *>(P.env_map);
    const float4 ca = __ldg(&T[(uint32_t)(fw * thc + phc)]), cb = __ldg(&T[(uint32_t)(fw * (thc + 1.0f) + phc)]);
    const float4 da = __ldg(&T[(uint32_t)(fw * thc + phc + 1.0f)]),
                 db = __ldg(&T[(uint32_t)(fw * (thc + 1.0f) + phc + 1.0f)]);
    return make_float3(lerp_ref(lerp_ref(ca.x, cb.x, tht), lerp_ref(da.x, db.x, tht), pht),
                       lerp_ref(lerp_ref(ca.y, cb.y, tht), lerp_ref(da.y, db.y, tht), pht),
                       lerp_ref(lerp_ref(ca.z, cb.z, tht), lerp_ref(da.z, db.z, tht), pht));
}

// Light gathered from the sky on escape: the Hosek model (the reference built
// with USE_ARHOSEK_SKYMODEL), or pow(environment, 2.2) of its default build
// with NullEnv (zero) or MapEnv (src/kernel.cpp:361-364).
__device__ __forceinline__ float3 sky_light(const DevParams &P, const float rd[3]) {
    if (P.env_mode == kEnvHosek) return sky_eval(P, rd);
    if (P.env_mode == kEnvNone) return make_float3(dpow(0.0f, 2.2f), dpow(0.0f, 2.2f), dpow(0.0f, 2.2f));
    const float3 e = env_map_eval(P, rd);
    return make_float3(dpow(e.x, 2.2f), dpow(e.y, 2.2f), dpow(e.z, 2.2f));
}

// Feature bits of a kernel instantiation.  Frames that use neither run the
// instantiation without their code (its register use and size stay those of
// the Mie/Hosek path).
enum : uint32_t {
    kFeatOcc = 1,  // occluders present and the USE_EMBREE build's masks apply
    kFeatExt = 2,  // HG phase or an environment other than the Hosek sky
    kFeatSdf = 4,  // surface (SDF) leaves in the scene
    kFeatAll = 7,
};

// Escape light of a segment: the Hosek sky, or (kFeatExt) whichever
// environment the parameters select.
template <uint32_t FEAT>
__device__ __forceinline__ float3 escape_sky(const DevParams &P, const float rd[3]) {
    if constexpr ((FEAT & kFeatExt) != 0) return sky_light(P, rd);
    else return sky_eval(P, rd);
}

template <uint32_t FEAT>
__device__ __forceinline__ float3 path_phase_eval(const DevParams &P, const MieSmem &M, float ct) {
    if constexpr ((FEAT & kFeatExt) != 0) return phase_eval_rgb(P, M, ct);
    else return mie_eval_rgb(M, ct);
}

template <uint32_t FEAT>
__device__ __forceinline__ void path_phase_sample(const DevParams &P, const MieSmem &M, const float iv[3], float u1,
                                                  float u2, float out[3]) {
    if constexpr ((FEAT & kFeatExt) != 0) phase_sample(P, M, iv, u1, u2, out);
    else mie_sample(M, iv, u1, u2, out);
}

// ---- camera ray, K_ParallelRender (src/kernel.cpp:461-474) -----------------
__device__ __forceinline__ bool camera_ray(const DevParams &P, uint32_t px, uint32_t py, float ro[3], float rd[3]) {
    const float hx = 0.0f - (((2.0f * ((float)px + 0.5f)) / (float)P.w) - 1.0f);
    const float hy = 0.0f - (((2.0f * ((float)py + 0.5f)) / (float)P.h) - 1.0f);
    const float *V = P.viewi, *Q = P.proji;
    float rv[3], d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) rv[k] = ((hx * Q[k] + hy * Q[4 + k]) + 0.0f * Q[8 + k]) + 1.0f * Q[12 + k];
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = ((rv[0] * V[k] + rv[1] * V[4 + k]) + rv[2] * V[8 + k]) + 0.0f * V[12 + k];
    const float len = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        rd[k] = d[k] / len;
        ro[k] = V[12 + k];
    }
    return (hx > -1.0f && hx < 1.0f) && (hy > -1.0f && hy < 1.0f);
}

// ---- free-flight tracking of one segment (src/kernel.cpp:197-317) ----------
// Returns kTrackEscaped when the segment leaves the volume (or passes `depth` at
// a leaf boundary) without a real collision, kTrackCollided for a real
// collision before `depth`, and kTrackCut for a collision at or beyond `depth`:
// the reference re-evaluates its mask mm = td < depth on the next leaf step and
// sets rm |= !mm after taking alpha from rm (src/kernel.cpp:214-217, 370-384),
// so such a collision counts for coverage but does not scatter.  td receives
// the distance of the collision (or of the last leaf exit).
enum : uint32_t { kTrackCollided = 0, kTrackEscaped = 1, kTrackCut = 2 };

// ---- occluders: SceneOcclusion::Intersect (src/SceneOcclusion.cpp:58-91) ----
// Embree's query with tnear 0 and tfar MAX_OCCLUSION_DIST reports whether the
// ray hits any occluder triangle; only that answer is used
// (src/kernel.cpp:149-153, 375-383).  The triangle test is Moller-Trumbore
// (1997) without culling, with the division by the determinant folded into
// the comparisons: hit when u, v >= 0, u + v <= det and 0 <= t <= det * tfar
// (signs reversed for det < 0; det == 0 is a miss).
__device__ __forceinline__ bool occ_triangle(const float4 *__restrict__ T, uint32_t i, const float o[3],
                                             const float d[3]) {
    const float4 a = __ldg(&T[3 * (size_t)i]), e1 = __ldg(&T[3 * (size_t)i + 1]), e2 = __ldg(&T[3 * (size_t)i + 2]);
    const float px = d[1] * e2.z - d[2] * e2.y, py = d[2] * e2.x - d[0] * e2.z, pz = d[0] * e2.y - d[1] * e2.x;
    const float det = e1.x * px + e1.y * py + e1.z * pz;
    const float sx = o[0] - a.x, sy = o[1] - a.y, sz = o[2] - a.z;
    const float u = sx * px + sy * py + sz * pz;
    const float qx = sy * e1.z - sz * e1.y, qy = sz * e1.x - sx * e1.z, qz = sx * e1.y - sy * e1.x;
    const float v = d[0] * qx + d[1] * qy + d[2] * qz;
    const float t = e2.x * qx + e2.y * qy + e2.z * qz;
    const float uv = u + v;
    if (det > 0.0f) return u >= 0.0f && v >= 0.0f && uv <= det && t >= 0.0f && t <= det * kOccFar;
    if (det < 0.0f) return u <= 0.0f && v <= 0.0f && uv >= det && t <= 0.0f && t >= det * kOccFar;
    return false;
}

// Slab test of a (padded) box against t in [0, tfar]; the far end is widened
// by 1 + 2 gamma(3) (robust traversal, Ize 2013).  A zero direction component
// gives infinite slab bounds, which fminf/fmaxf order correctly.
__device__ __forceinline__ bool occ_box(float x0, float y0, float z0, float x1, float y1, float z1, const float o[3],
                                        const float inv[3]) {
    const float ax = (x0 - o[0]) * inv[0], bx = (x1 - o[0]) * inv[0];
    const float ay = (y0 - o[1]) * inv[1], by = (y1 - o[1]) * inv[1];
    const float az = (z0 - o[2]) * inv[2], bz = (z1 - o[2]) * inv[2];
    const float t0 = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fmaxf(fminf(az, bz), 0.0f));
    const float t1 = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fminf(fmaxf(az, bz), kOccFar));
    return t0 <= t1 * 1.00000048f;
}

// Any-hit traversal of the occluder BVH.  Every node is visited at most once,
// so the loop ends within occ_n_nodes iterations; the stack holds at most one
// entry per level of the (depth-capped) tree.  Not inlined: its stack then sits
// in its own frame.  Inlined into the shadow-pass kernel, the kernel's local
// frame came out smaller (384 B) than its node and interval stacks need at once
// (448 B), and that kernel read out of bounds; every caller's frame now holds
// all three stacks.
__device__ __noinline__ bool occluded_bvh(const float4 *__restrict__ nodes, const float4 *__restrict__ tris,
                                          uint32_t n_nodes, float ox, float oy, float oz, float dx, float dy,
                                          float dz) {
    const float o[3] = {ox, oy, oz}, d[3] = {dx, dy, dz};
    const float inv[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
    uint32_t stack[kOccMaxDepth + 2];
    int sp = 0;
    uint32_t node = 0;
    for (uint32_t it = 0; it < n_nodes; ++it) {
        const float4 n0 = __ldg(&nodes[4 * (size_t)node]), n1 = __ldg(&nodes[4 * (size_t)node + 1]);
        const float4 n2 = __ldg(&nodes[4 * (size_t)node + 2]);
        const uint4 n3 = __ldg(reinterpret_cast<const uint4 *>(nodes) + 4 * (size_t)node + 3);
        bool hl = n3.x != kNone && occ_box(n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, o, inv);
        bool hr = n3.y != kNone && occ_box(n1.z, n1.w, n2.x, n2.y, n2.z, n2.w, o, inv);
        if (hl && n3.z) {
            for (uint32_t k = 0; k < n3.z; ++k)
                if (occ_triangle(tris, n3.x + k, o, d)) return true;
            hl = false;
        }
        if (hr && n3.w) {
            for (uint32_t k = 0; k < n3.w; ++k)
                if (occ_triangle(tris, n3.y + k, o, d)) return true;
            hr = false;
        }
        if (hl && hr) {
            if (sp < kOccMaxDepth + 2) stack[sp++] = n3.y;
            node = n3.x;
        } else if (hl) {
            node = n3.x;
        } else if (hr) {
            node = n3.y;
        } else {
            if (sp == 0) return false;
            node = stack[--sp];
        }
    }
    return false;
}

// Whether the ray (o, d) hits an occluder (false without occluders).
__device__ __forceinline__ bool occluded(const DevScene &S, const float o[3], const float d[3]) {
    return S.occ_nodes && occluded_bvh(S.occ_nodes, S.occ_tris, S.occ_n_nodes, o[0], o[1], o[2], d[0], d[1], d[2]);
}

// A tracking visitor sees every collision decision that involved a density
// lookup: the leaf's brick and box, the position, rho, the majorant and
// whether the collision was real (rho / smax >= q).  The forward renderer's
// visitor does nothing; the adjoint's accumulates gradients.
struct NoVisit {
    __device__ __forceinline__ void operator()(const float *, const float4 &, const float *, float, float, bool) const {}
};

// SDF: the scene may hold surface leaves (src/kernel.cpp:241-305); without it
// every leaf is a fog leaf and the surface tests are not compiled in.
template <class Visit, bool SDF = true>
__device__ __forceinline__ uint32_t track_v(const DevScene &S, SegMedium med, const float ro[3], const float rd[3],
                                            Rng &g, float depth, float &td_out, uint32_t *nstack, Count &cnt,
                                            const Visit &visit);

template <bool SDF = true>
__device__ __forceinline__ uint32_t track(const DevScene &S, const DevParams &P, const float ro[3], const float rd[3],
                                          Rng &g, float depth, float &td_out, uint32_t *nstack, Count &cnt) {
    const NoVisit nv;
    return track_v<NoVisit, SDF>(S, seg_medium(P), ro, rd, g, depth, td_out, nstack, cnt, nv);
}

template <class Visit, bool SDF>
__device__ __forceinline__ uint32_t track_v(const DevScene &S, SegMedium med, const float ro[3], const float rd[3],
                                            Rng &g, float depth, float &td_out, uint32_t *nstack, Count &cnt,
                                            const Visit &visit) {
    const float sigma_e = med.sigma_e;
    Trav T;
    trav_init(T, S, ro, rd, cnt);
    ++cnt.vertices;
    float td = 0.0f;
    uint32_t leaf;
    float tra, trb;
    uint32_t budget = med.budget;
    float tstack[kMaxDepth][6];
    while (trav_next_k(T, S, nstack, leaf, tra, trb, cnt, 0xffffffffu, tstack) == kTravLeaf) {
        if (!(td < depth)) break;
        const float4 ce = __ldg(&S.leaf[2 * leaf]);
        const float4 meta = __ldg(&S.leaf[2 * leaf + 1]);
        const float smax = meta.x;
        const uint32_t fogx = __float_as_uint(meta.y);
        const float *brick = S.bricks + (size_t)fogx * kBrick;
        const float *sbrick = nullptr;  // surface brick of an SDF leaf
        if constexpr (SDF) {
            const uint32_t sdfx = __float_as_uint(meta.z);
            if (sdfx != kNone) sbrick = S.sdf_bricks + (size_t)sdfx * kBrick;
        }
        const float lo = td;
        const float tr0 = tra - td, tr1 = trb - td;
        float s0;
        if (SDF && sbrick) {
            // src/kernel.cpp:253-263: an SDF leaf is entered (td = tra, s0 = tr0)
            // only when the ray is before it and the distance there is positive;
            // otherwise tracking starts from td with s0 = 0
            bool skip = false;
            if (tra > td) {
                const float r0[3] = {ro[0] + rd[0] * tra, ro[1] + rd[1] * tra, ro[2] + rd[2] * tra};
                skip = sample_voxel_space(r0, sbrick, ce) > 0.0f;
                ++cnt.density_lookups;
            }
            if (skip) {
                td = tra;
                s0 = tr0;
            } else {
                s0 = 0.0f;
            }
        } else if (tra > td) {
            // src/kernel.cpp:241-265: sm = (tra > td) | VM with VM the integer 1 for
            // fog leaves, so the masked selects are bitwise blends: past the leaf
            // entry, td keeps all but its lowest bit and s0 becomes the lowest bit
            // of tr0 (0 or the smallest denormal).
            td = tra;
            s0 = tr0;
        } else {
            td = __uint_as_float((__float_as_uint(td) & ~1u) | (__float_as_uint(tra) & 1u));
            s0 = __uint_as_float(__float_as_uint(tr0) & 1u);
        }
        const float denom = sigma_e * smax;
        float sr = -dlog(g.uniform()) / denom;
        for (;;) {
            const float sc = s0 + sr;
            td = lo + sc;
            if (!(sc < tr1)) {
                td = trb;
                break;
            }
            bool rm = sc > tr0;
            float rho = -1.0f, dist = 1.0f;
            bool fog_decides = rm;  // the decision depends on the fog density (what the visitor differentiates)
            if (rm) {
                const float rc[3] = {ro[0] + rd[0] * td, ro[1] + rd[1] * td, ro[2] + rd[2] * td};
                if (SDF && sbrick) {
                    // src/kernel.cpp:287-300: inside the surface (dist <= 0) always
                    // collides; outside, the fog brick (if any) decides
                    dist = sample_voxel_space(rc, sbrick, ce);
                    ++cnt.density_lookups;
                    fog_decides = dist > 0.0f && fogx != kNone;
                    if (fog_decides) {
                        rho = sample_voxel_space(rc, brick, ce);
                        ++cnt.density_lookups;
                    }
                } else {
                    rho = sample_voxel_space(rc, brick, ce);
                    ++cnt.density_lookups;
                }
            }
            const float q = g.uniform();
            rm = rm && (rho / smax < q) && (dist > 0.0f);
            if (fog_decides) {
                const float rc[3] = {ro[0] + rd[0] * td, ro[1] + rd[1] * td, ro[2] + rd[2] * td};
                visit(brick, ce, rc, rho, smax, !rm);
            }
            if (!rm) {
                td_out = td;
                return td < depth ? kTrackCollided : kTrackCut;
            }
            if (--budget == 0) {
                ++cnt.gave_up;
                td_out = td;
                return kTrackEscaped;
            }
            sr = sr - dlog(g.uniform()) / denom;
        }
    }
    td_out = td;
    return kTrackEscaped;
}

// DR_KERNEL_FINITE_PATHS: a path sample whose sun or sky sum is not finite is
// dropped (the reference's sky term is 0/0 for a direction with rd.y == 0:
// rd.x / rd.y is infinite and is multiplied by 0, src/kernel.cpp:338-342).
__device__ __forceinline__ void drop_nonfinite(const DevParams &P, float4 &sun, float4 &sky) {
    if (!P.finite_paths) return;
    const bool ok = isfinite(sun.x) && isfinite(sun.y) && isfinite(sun.z) && isfinite(sky.x) && isfinite(sky.y) &&
                    isfinite(sky.z);
    if (!ok) {
        sun = make_float4(0.0f, 0.0f, 0.0f, sun.w);
        sky = make_float4(0.0f, 0.0f, 0.0f, sky.w);
    }
}

// ---- one camera path sample: SampleVolume recursion as a loop --------------
// (src/kernel.cpp:128-445; see the CPU restatement for the derivation)
// Alpha of a path sample = what its camera segment did: 0 when it escaped, 1
// when it collided; a collision at or beyond the depth (cut) counts as 1, but
// the USE_EMBREE build's depth mask (src/kernel.cpp:379) zeroes it.
__device__ __forceinline__ float first_alpha(const DevParams &P, uint32_t res) {
    return (res == kTrackCollided || (res == kTrackCut && !P.embree)) ? 1.0f : 0.0f;
}

template <uint32_t FEAT = kFeatAll>
__device__ __forceinline__ void path_sample(const DevScene &S, const DevParams &P, const MieSmem &M, uint32_t px,
                                            uint32_t py, uint64_t seed, uint64_t sample, float4 &sun_acc,
                                            float4 &sky_acc, uint32_t *nstack, Count &cnt) {
    float ro[3], rd[3];
    sun_acc = make_float4(0.f, 0.f, 0.f, 0.f);
    sky_acc = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!camera_ray(P, px, py, ro, rd)) return;
    Rng g = rng_seed(seed, (uint64_t)py * P.w + px, sample);
    const float f = P.albedo;
    float T0 = 1.0f, T1 = 1.0f, T2 = 1.0f;
    const float depth0 = (P.depth && P.depthcomp) ? __ldg(&P.depth[(size_t)py * P.w + px]) : 3.402823466e+38f;
    for (uint32_t r = 0;; ++r) {
        float td;
        const uint32_t res = track<(FEAT & kFeatSdf) != 0>(S, P, ro, rd, g, r == 0 ? depth0 : 3.402823466e+38f, td, nstack, cnt);
        if (r == 0) sun_acc.w = sky_acc.w = first_alpha(P, res);
        if (res == kTrackCut) break;
        if (res == kTrackEscaped) {
            if (r > 0 && !((FEAT & kFeatOcc) && P.embree && occluded(S, ro, rd))) {
                if (sun_hit(P, rd)) {
                    sun_acc.x = sun_acc.x + T0 * P.sun_color[0];
                    sun_acc.y = sun_acc.y + T1 * P.sun_color[1];
                    sun_acc.z = sun_acc.z + T2 * P.sun_color[2];
                } else {
                    sun_acc.x = sun_acc.x + T0 * 0.0f;
                    sun_acc.y = sun_acc.y + T1 * 0.0f;
                    sun_acc.z = sun_acc.z + T2 * 0.0f;
                }
                const float3 sky = escape_sky<FEAT>(P, rd);
                sky_acc.x = sky_acc.x + T0 * sky.x;
                sky_acc.y = sky_acc.y + T1 * sky.y;
                sky_acc.z = sky_acc.z + T2 * sky.z;
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
        cnt.mie_evals += 3;
#pragma unroll
        for (int k = 0; k < 3; ++k) rc[k] = ro[k] + rd[k] * td;
        float tds;
        if (track<(FEAT & kFeatSdf) != 0>(S, P, rc, lrd, g, 3.402823466e+38f, tds, nstack, cnt) == kTrackEscaped &&
            !((FEAT & kFeatOcc) && P.embree && occluded(S, rc, lrd))) {
            const bool hit = sun_hit(P, lrd);
            const float s0 = hit ? P.sun_color[0] : 0.0f, s1 = hit ? P.sun_color[1] : 0.0f,
                        s2 = hit ? P.sun_color[2] : 0.0f;
            sun_acc.x = sun_acc.x + (T0 * ((p3.x / (p3.x + p2)) * f)) * s0;
            sun_acc.y = sun_acc.y + (T1 * ((p3.y / (p3.y + p2)) * f)) * s1;
            sun_acc.z = sun_acc.z + (T2 * ((p3.z / (p3.z + p2)) * f)) * s2;
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
    drop_nonfinite(P, sun_acc, sky_acc);
}

// ---- one shadow-pass sample: RenderKernel::Shadow (src/kernel.cpp:569-607) ----
// The camera ray is cut at the pixel's depth when that lies before the far clip
// plane; from there one shadow segment (SampleVolume with r = scattevs) runs
// along a sun-cone sample.  A pixel without geometry before the far plane traces
// nothing and keeps "not scattering".  The result is divided by
// float4::load(&colour), whose w is 0: rgb = sun(lrd) / colour, alpha = 1/0 per
// sample (0/0 only when scattevs == 0 and the segment escaped).
__device__ __forceinline__ float4 shadow_sample(const DevScene &S, const DevParams &P, uint32_t px, uint32_t py,
                                                uint64_t seed, uint64_t sample, const float ro[3], const float rd[3],
                                                uint32_t *nstack, Count &cnt) {
    const float depth = P.depth ? __ldg(&P.depth[(size_t)py * P.w + px]) : 3.402823466e+38f;
    const bool active = depth < P.clip_end;
    Rng g = rng_seed(seed, (uint64_t)py * P.w + px, sample);
    const float u3 = g.uniform(), u4 = g.uniform();
    float lrd[3];
    sun_sample(P, u3, u4, lrd);
    uint32_t res = kTrackEscaped;
    bool occ = false;
    if (active) {
        const float ro1[3] = {ro[0] + rd[0] * depth, ro[1] + rd[1] * depth, ro[2] + rd[2] * depth};
        float td;
        res = track(S, P, ro1, lrd, g, 3.402823466e+38f, td, nstack, cnt);
        // USE_EMBREE build: an escaped segment whose ray hits an occluder
        // gathers nothing, alpha included (src/kernel.cpp:375-383)
        occ = res == kTrackEscaped && P.embree && occluded(S, ro1, lrd);
    }
    const bool esc = res == kTrackEscaped;
    const bool lit = P.scattevs > 0u && esc && !occ && sun_hit(P, lrd);
    float4 o;
    o.x = __fdiv_rn(lit ? P.sun_color[0] : 0.0f, P.sun_color[0]);
    o.y = __fdiv_rn(lit ? P.sun_color[1] : 0.0f, P.sun_color[1]);
    o.z = __fdiv_rn(lit ? P.sun_color[2] : 0.0f, P.sun_color[2]);
    o.w = __fdiv_rn(((P.scattevs > 0u || !esc) && !occ) ? 1.0f : 0.0f, 0.0f);
    return o;
}

}  // namespace dr
