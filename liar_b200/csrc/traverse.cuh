// traverse.cuh -- sm_100a closest-hit / any-hit traversal of the 4-wide tree (qbvh.h).
//
// Replaces the per-ray Lass traversal behind TriangleMesh::doIntersect / doIsIntersecting
// (src/liar/scenery/triangle_mesh.cpp:291-330) and ObjectTree::doIntersect / doIsIntersecting
// (src/liar/scenery/object_trees.h:110-143).
//
// Organisation (one lane per ray, persistent warps with per-lane refill):
//   * a grid of (SM count x resident blocks) blocks; each warp takes batches of BATCH ray indices
//     (32..256, sized so that the n rays cover every resident warp)
//     from one atomic work counter and hands them to its lanes one by one: whenever at least
//     REFILL lanes have finished their ray, those lanes load the next rays of the batch, so short
//     rays (most random rays miss the mesh after a node or two) do not leave lanes idle while a
//     long ray of the same warp is still traversing (dynamic fetch, Aila & Laine 2009);
//   * one loop turn = a node phase and a leaf phase: every lane still descending visits one node
//     (a lane whose node hit nothing pops its next entry at once), and lanes that have reached a
//     leaf wait until LEAF_AT of them have (or none descends any more), then test their leaves
//     together and pop; refills are checked every turn. Compared with running each lane down to
//     its next leaf per turn, lanes idle far less (random rays of very different lengths): on the
//     1.31M-triangle icosphere with 16.7M random rays, 5.76 against 4.20 Grays/s closest hit and
//     6.36 against 4.76 any hit, hits identical;
//   * a node is one 128-byte line read with seven 16-byte loads that carry an L2 evict-last
//     policy; rays and hits stream with evict-first, so the 512 MiB ray stream does not push the
//     tree out of L2;
//   * hit children are ordered by entry distance (5-comparator network on distance-bit keys);
//     the farther ones are pushed with their entry distance onto a per-lane stack whose top S
//     entries live in shared memory (column per lane: conflict-free) and whose deeper entries
//     spill to local memory; popped entries farther than the current closest hit are dropped;
//   * triangles are tested with the exact Moller-Trumbore of tri_exact.h, so t is bit-identical
//     to the CPU restatement, and equal t resolves to the lower original triangle index.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/liar_gpu.h"
#include "qbvh.h"
#include "tri_exact.h"

namespace liar_gpu {

// device-side status bits (ORed into the status word of a launch)
enum : uint32_t { STATUS_STACK_OVERFLOW = 1u, STATUS_BAD_NODE = 2u };

// total stack entries per lane (shared top + local spill); the host refuses deeper trees
constexpr int kTraceStackTotal = 64;

struct TraceCounters {
    unsigned long long nodes;
    unsigned long long tris;
};

// ---- loads and stores with L2 eviction policies (PTX createpolicy / cache_hint)
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ float4 ld_hint(const void* ptr, uint64_t pol) {
    float4 v;
    asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(ptr), "l"(pol));
    return v;
}
__device__ __forceinline__ int4 ld_hint_i(const void* ptr, uint64_t pol) {
    int4 v;
    asm("ld.global.nc.L2::cache_hint.v4.s32 {%0, %1, %2, %3}, [%4], %5;"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(ptr), "l"(pol));
    return v;
}
__device__ __forceinline__ void st_hint(void* ptr, int a, int b, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.v2.s32 [%0], {%1, %2}, %3;" ::"l"(ptr), "r"(a), "r"(b), "l"(pol) : "memory");
}

__device__ __forceinline__ float safe_rcp(float d) {
    // keeps 1/d finite so that inverted (empty) boxes can never produce NaN slab distances
    const float ad = fabsf(d);
    return 1.0f / (ad > 1e-20f ? d : copysignf(1e-20f, d));
}

__device__ __forceinline__ float max4f(float a, float b, float c, float d) { return fmaxf(fmaxf(a, b), fmaxf(c, d)); }
__device__ __forceinline__ float min4f(float a, float b, float c, float d) { return fminf(fminf(a, b), fminf(c, d)); }
__device__ __forceinline__ int sel4i(const int4& v, uint32_t s) { return s == 0 ? v.x : s == 1 ? v.y : s == 2 ? v.z : v.w; }
__device__ __forceinline__ float sel4f(float a, float b, float c, float d, uint32_t s) {
    return s == 0 ? a : s == 1 ? b : s == 2 ? c : d;
}
__device__ __forceinline__ void cswap(uint32_t& a, uint32_t& b) {
    const uint32_t lo = min(a, b), hi = max(a, b);
    a = lo;
    b = hi;
}

constexpr int kNodeNone = -1;  // "no node": 0xffffffff is never a real leaf (leaf counts are <= 8)

// Per-lane traversal state.
struct RayState {
    float ox, oy, oz, tmin, dx, dy, dz, tmax;
    float idx, idy, idz, oix, oiy, oiz;
    float tbest;
    int best;
    int node;
    int sp;
};

template <int S, int BLOCK>
struct LaneStack {
    static constexpr int L = kTraceStackTotal - S > 0 ? kTraceStackTotal - S : 1;
    int* s_node;
    float* s_t;
    int l_node[L];
    float l_t[L];

    __device__ __forceinline__ void push(int sp, int node, float t) {
        if (sp < S) {
            s_node[sp * BLOCK + threadIdx.x] = node;
            s_t[sp * BLOCK + threadIdx.x] = t;
        } else {
            l_node[sp - S] = node;
            l_t[sp - S] = t;
        }
    }
    __device__ __forceinline__ void get(int sp, int& node, float& t) const {
        if (sp < S) {
            node = s_node[sp * BLOCK + threadIdx.x];
            t = s_t[sp * BLOCK + threadIdx.x];
        } else {
            node = l_node[sp - S];
            t = l_t[sp - S];
        }
    }
};

// One inner node: st.node >= 0 on entry. Its hit children are ordered by entry distance, the
// farther ones pushed; on exit st.node is the nearest hit child (inner node or leaf), or kNodeNone
// when no child is hit.
// PF: 1 = prefetch the next node's line into L1 once it is known, 2 = also the first triangle line
// of a leaf reached (the loads of the next turn then find it there)
template <bool ANY, int S, int BLOCK, bool COUNT, int PF = 0>
__device__ __forceinline__ void visit_node(const QNode* __restrict__ nodes, RayState& st, LaneStack<S, BLOCK>& stack,
                                           uint64_t pol_tree, uint32_t& status, uint32_t& n_nodes,
                                           const QTri* __restrict__ tris = nullptr) {
    const bool nx = st.dx < 0.0f, ny = st.dy < 0.0f, nz = st.dz < 0.0f;
    if (COUNT) ++n_nodes;
    const QNode* q = nodes + st.node;
    // the planes a ray meets first along each axis (lo for a positive direction, hi for a negative
    // one; hi_* follows lo_* by 16 bytes) selected by address rather than by value, so the four
    // children's near and far rows arrive in place of the six rows and their 24 selects
    const char* qb = reinterpret_cast<const char*>(q);
    const uint32_t onx = nx ? 16u : 0u, ony = ny ? 48u : 32u, onz = nz ? 80u : 64u;
    const float4 nxp = ld_hint(qb + onx, pol_tree), fxp = ld_hint(qb + (onx ^ 16u), pol_tree);
    const float4 nyp = ld_hint(qb + ony, pol_tree), fyp = ld_hint(qb + (ony ^ 16u), pol_tree);
    const float4 nzp = ld_hint(qb + onz, pol_tree), fzp = ld_hint(qb + (onz ^ 16u), pol_tree);
    const int4 ch = ld_hint_i(&q->child, pol_tree);
    float tn[4], tf[4];
    tn[0] = max4f(fmaf(nxp.x, st.idx, -st.oix), fmaf(nyp.x, st.idy, -st.oiy), fmaf(nzp.x, st.idz, -st.oiz), st.tmin);
    tn[1] = max4f(fmaf(nxp.y, st.idx, -st.oix), fmaf(nyp.y, st.idy, -st.oiy), fmaf(nzp.y, st.idz, -st.oiz), st.tmin);
    tn[2] = max4f(fmaf(nxp.z, st.idx, -st.oix), fmaf(nyp.z, st.idy, -st.oiy), fmaf(nzp.z, st.idz, -st.oiz), st.tmin);
    tn[3] = max4f(fmaf(nxp.w, st.idx, -st.oix), fmaf(nyp.w, st.idy, -st.oiy), fmaf(nzp.w, st.idz, -st.oiz), st.tmin);
    tf[0] = min4f(fmaf(fxp.x, st.idx, -st.oix), fmaf(fyp.x, st.idy, -st.oiy), fmaf(fzp.x, st.idz, -st.oiz), st.tbest);
    tf[1] = min4f(fmaf(fxp.y, st.idx, -st.oix), fmaf(fyp.y, st.idy, -st.oiy), fmaf(fzp.y, st.idz, -st.oiz), st.tbest);
    tf[2] = min4f(fmaf(fxp.z, st.idx, -st.oix), fmaf(fyp.z, st.idy, -st.oiy), fmaf(fzp.z, st.idz, -st.oiz), st.tbest);
    tf[3] = min4f(fmaf(fxp.w, st.idx, -st.oix), fmaf(fyp.w, st.idy, -st.oiy), fmaf(fzp.w, st.idz, -st.oiz), st.tbest);
    // sortable keys: entry distance bits (tn >= tmin >= 0 for valid rays) with the slot in
    // the two low bits; misses become 0xffffffff
    uint32_t key[4];
#pragma unroll
    for (int c = 0; c < 4; ++c)
        key[c] = tn[c] <= tf[c] ? ((__float_as_uint(fmaxf(tn[c], 0.0f)) & ~3u) | (uint32_t)c) : 0xffffffffu;
    if (!ANY) {
        cswap(key[0], key[1]);
        cswap(key[2], key[3]);
        cswap(key[0], key[2]);
        cswap(key[1], key[3]);
        cswap(key[1], key[2]);
    }
    const int first = key[0] != 0xffffffffu ? 0 : key[1] != 0xffffffffu ? 1 : key[2] != 0xffffffffu ? 2
                                                                    : key[3] != 0xffffffffu ? 3 : -1;
    if (first < 0) {
        st.node = kNodeNone;  // nothing hit below this node
        return;
    }
    // push the other hit children, farthest first
#pragma unroll
    for (int c = 3; c >= 0; --c) {
        if (c == first || key[c] == 0xffffffffu) continue;
        const uint32_t slot = key[c] & 3u;
        if (st.sp >= kTraceStackTotal) {
            status |= STATUS_STACK_OVERFLOW;
            continue;
        }
        stack.push(st.sp, sel4i(ch, slot), sel4f(tn[0], tn[1], tn[2], tn[3], slot));
        ++st.sp;
    }
    const uint32_t kf = first == 0 ? key[0] : first == 1 ? key[1] : first == 2 ? key[2] : key[3];
    st.node = sel4i(ch, kf & 3u);
    if (PF >= 1 && st.node >= 0) {
        asm volatile("prefetch.global.L1 [%0];" ::"l"(nodes + st.node));
    } else if (PF >= 2 && st.node != kNodeNone) {
        asm volatile("prefetch.global.L1 [%0];" ::"l"(tris + ((uint32_t)st.node & 0x07ffffffu)));
    }
}

// Tests the leaf st.node (packed 0x80000000 | count << 27 | first). True when an any-hit ray is
// finished by it.
template <bool ANY, bool COUNT>
__device__ __forceinline__ bool test_leaf(const QTri* __restrict__ tris, RayState& st, uint64_t pol_tree,
                                          uint32_t& n_tris) {
    const uint32_t packed = (uint32_t)st.node;
    const uint32_t count = (packed >> 27) & 15u;
    const uint32_t first = packed & 0x07ffffffu;
    for (uint32_t k = 0; k < count; ++k) {
        if (COUNT) ++n_tris;
        const QTri* tp = tris + first + k;
        const float4 a = ld_hint(&tp->v0, pol_tree), e1 = ld_hint(&tp->e1, pol_tree), e2 = ld_hint(&tp->e2, pol_tree);
        float t, u, v;
        bool hit;
        if (e1.w != 0.0f) {
            // a sphere: its nearer root beyond tmin, else the farther one
            float t1;
            hit = sphere_intersect_exact(st.ox, st.oy, st.oz, st.dx, st.dy, st.dz, a.x, a.y, a.z, e1.x, t, t1);
            if (hit && !(t > st.tmin)) t = t1;
        } else {
            hit = tri_intersect_exact(st.ox, st.oy, st.oz, st.dx, st.dy, st.dz, a.x, a.y, a.z, e1.x, e1.y, e1.z, e2.x,
                                      e2.y, e2.z, t, u, v);
        }
        if (hit) {
            const int prim = __float_as_int(a.w);
            if (ANY) {
                if (t > st.tmin && t < st.tmax) {
                    st.best = prim;
                    st.tbest = t;
                    return true;
                }
            } else if (t > st.tmin && (t < st.tbest || (t == st.tbest && prim < st.best))) {
                st.tbest = t;
                st.best = prim;
            }
        }
    }
    return false;
}

// Pops the next entry that can still hold a closer hit into st.node; true when there is none (the
// ray is finished).
template <bool ANY, int S, int BLOCK>
__device__ __forceinline__ bool pop_next(RayState& st, const LaneStack<S, BLOCK>& stack) {
    while (st.sp > 0) {
        --st.sp;
        int nd;
        float te;
        stack.get(st.sp, nd, te);
        if (ANY || te <= st.tbest) {
            st.node = nd;
            return false;
        }
    }
    return true;
}

// rays per warp fetch: the n rays spread evenly over the launch's warps, rounded up to a multiple
// of 32 and kept within [32, 256] (fewer fetches for large waves, full occupancy for small ones)
__host__ __device__ __forceinline__ uint32_t trace_batch(uint32_t n, uint32_t warps) {
    const uint32_t per = warps ? (n + warps - 1) / warps : n;
    const uint32_t b = (per + 31u) & ~31u;
    return b < 32u ? 32u : (b > 256u ? 256u : b);
}

// REFILL: idle lanes that trigger a refill; LEAF_AT: lanes waiting at a leaf that start the leaf
// phase (see below); MINB: resident blocks the register allocation must allow
template <bool ANY, int S, int BLOCK, bool COUNT, int REFILL = 8, int LEAF_AT = 8, int MINB = 1, int PF = 0>
__global__ void __launch_bounds__(BLOCK, MINB) trace_kernel(const QNode* __restrict__ nodes, const QTri* __restrict__ tris,
                                                      const liar_ray* __restrict__ rays, liar_hit* __restrict__ hits,
                                                      uint32_t n_rays, uint32_t* __restrict__ work_counter,
                                                      uint32_t* __restrict__ status_word,
                                                      TraceCounters* __restrict__ counters, uint32_t BATCH,
                                                      const uint32_t* __restrict__ n_dev) {
    // BATCH: ray indices a warp takes from the global counter at once (trace_batch: n spread over
    // all resident warps, 32..256, so that a small wave still keeps every warp busy).
    // n_dev: the ray count in device memory, at most n_rays (a queue whose size the host does not
    // wait for); the launch was sized for n_rays
    if (n_dev) {
        n_rays = min(*n_dev, n_rays);
        BATCH = trace_batch(n_rays, gridDim.x * (BLOCK / 32));
    }
    extern __shared__ int trace_smem[];  // S * BLOCK node entries, then S * BLOCK distances
    LaneStack<S, BLOCK> stack;
    stack.s_node = trace_smem;
    stack.s_t = reinterpret_cast<float*>(trace_smem + S * BLOCK);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint64_t pol_tree = policy_evict_last();
    const uint64_t pol_stream = policy_evict_first();
    uint32_t status = 0, n_nodes = 0, n_tris = 0;

    uint32_t w_next = 0, w_end = 0;  // the warp's current batch [w_next, w_end), uniform
    bool exhausted = false;          // uniform: the global counter has passed n_rays
    int rid = -1;                    // this lane's ray, -1 when idle
    RayState st;

    while (true) {
        const uint32_t idle = __ballot_sync(0xffffffffu, rid < 0);
        if (exhausted) {
            if (idle == 0xffffffffu) break;
        } else if ((uint32_t)__popc(idle) >= (uint32_t)REFILL) {
            if (w_next >= w_end) {
                uint32_t b = 0;
                if (lane == 0) b = atomicAdd(work_counter, BATCH);
                b = __shfl_sync(0xffffffffu, b, 0);
                if (b >= n_rays) {
                    exhausted = true;
                } else {
                    w_next = b;
                    w_end = min(b + BATCH, n_rays);
                }
            }
            if (!exhausted) {
                const uint32_t avail = w_end - w_next;
                const uint32_t rank = __popc(idle & lt_mask);
                if (rid < 0 && rank < avail) {
                    rid = (int)(w_next + rank);
                    const float4* rp = reinterpret_cast<const float4*>(rays + rid);
                    const float4 r0 = ld_hint(rp, pol_stream), r1 = ld_hint(rp + 1, pol_stream);
                    st.ox = r0.x;
                    st.oy = r0.y;
                    st.oz = r0.z;
                    st.tmin = r0.w;
                    st.dx = r1.x;
                    st.dy = r1.y;
                    st.dz = r1.z;
                    st.tmax = r1.w;
                    st.idx = safe_rcp(st.dx);
                    st.idy = safe_rcp(st.dy);
                    st.idz = safe_rcp(st.dz);
                    st.oix = st.ox * st.idx;
                    st.oiy = st.oy * st.idy;
                    st.oiz = st.oz * st.idz;
                    // closest hit keeps candidates strictly below range_far(tmax); any hit below tmax
                    st.tbest = ANY ? st.tmax : range_far(st.tmax);
                    st.best = -1;
                    st.sp = 0;
                    const bool finite = isfinite(r0.x) && isfinite(r0.y) && isfinite(r0.z) && isfinite(r1.x) &&
                                        isfinite(r1.y) && isfinite(r1.z) && !isnan(r0.w) && !isnan(r1.w);
                    st.node = finite ? 0 : kNodeNone;
                }
                w_next += min(avail, (uint32_t)__popc(idle));
            }
        }
        // node phase: every descending lane visits one node; a lane whose node hit nothing pops at
        // once (a ray turned away near the root finishes here and is replaced next turn)
        bool done = false;
        if (rid >= 0) {
            if (st.node >= 0) {
                visit_node<ANY, S, BLOCK, COUNT, PF>(nodes, st, stack, pol_tree, status, n_nodes, tris);
                if (st.node == kNodeNone) done = pop_next<ANY, S, BLOCK>(st, stack);
            } else if (st.node == kNodeNone) {
                done = true;  // a ray with non-finite components, retired untraced
            }
        }
        // leaf phase: lanes that reached a leaf wait until LEAF_AT of them have (or no lane is
        // descending any more), then test their leaves together and pop
        const bool at_leaf = rid >= 0 && !done && st.node < 0;
        const uint32_t leafw = __ballot_sync(0xffffffffu, at_leaf);
        if (leafw) {
            const uint32_t desc = __ballot_sync(0xffffffffu, rid >= 0 && !done && st.node >= 0);
            if ((uint32_t)__popc(leafw) >= (uint32_t)LEAF_AT || desc == 0u) {
                if (at_leaf)
                    done = test_leaf<ANY, COUNT>(tris, st, pol_tree, n_tris) || pop_next<ANY, S, BLOCK>(st, stack);
            }
        }
        if (done) {
            int prim = st.best;
            float t = st.tbest;
            if (!ANY && prim >= 0 && !(t > range_near(st.tmin))) prim = -1;  // BoundedRay::inRange near side
            if (prim < 0) t = INFINITY;
            st_hint(hits + rid, prim, __float_as_int(t), pol_stream);
            rid = -1;
        }
    }
    if (status) atomicOr(status_word, status);
    if (COUNT) {
        unsigned long long a = n_nodes, b = n_tris;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (lane == 0) {
            atomicAdd(&counters->nodes, a);
            atomicAdd(&counters->tris, b);
        }
    }
}

// ---- many trees in one launch (batched rendering): each ray names its scene, whose tree comes
// from a table; the ray count is read from device memory, so the launch can sit in a CUDA graph
// whose queue sizes are only known on the device
struct TreeRoot {
    const QNode* nodes;
    const QTri* tris;
};

template <int S, int BLOCK>
__global__ void __launch_bounds__(BLOCK) trace_multi_kernel(const TreeRoot* __restrict__ roots,
                                                            const liar_ray* __restrict__ rays,
                                                            const uint32_t* __restrict__ ray_scene,
                                                            liar_hit* __restrict__ hits, const uint32_t* __restrict__ n_dev,
                                                            uint32_t* __restrict__ work_counter,
                                                            uint32_t* __restrict__ status_word) {
    constexpr int REFILL = 8, LEAF_AT = 8;  // as trace_kernel
    extern __shared__ int trace_smem[];
    LaneStack<S, BLOCK> stack;
    stack.s_node = trace_smem;
    stack.s_t = reinterpret_cast<float*>(trace_smem + S * BLOCK);
    const uint32_t n_rays = *n_dev;
    const uint32_t BATCH = trace_batch(n_rays, gridDim.x * (BLOCK / 32));
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint64_t pol_tree = policy_evict_last();
    const uint64_t pol_stream = policy_evict_first();
    uint32_t status = 0, n_nodes = 0, n_tris = 0;
    uint32_t w_next = 0, w_end = 0;
    bool exhausted = false;
    int rid = -1;
    RayState st;
    const QNode* nodes = nullptr;
    const QTri* tris = nullptr;
    while (true) {
        const uint32_t idle = __ballot_sync(0xffffffffu, rid < 0);
        if (exhausted) {
            if (idle == 0xffffffffu) break;
        } else if ((uint32_t)__popc(idle) >= (uint32_t)REFILL) {
            if (w_next >= w_end) {
                uint32_t b = 0;
                if (lane == 0) b = atomicAdd(work_counter, BATCH);
                b = __shfl_sync(0xffffffffu, b, 0);
                if (b >= n_rays) {
                    exhausted = true;
                } else {
                    w_next = b;
                    w_end = min(b + BATCH, n_rays);
                }
            }
            if (!exhausted) {
                const uint32_t avail = w_end - w_next;
                const uint32_t rank = __popc(idle & lt_mask);
                if (rid < 0 && rank < avail) {
                    rid = (int)(w_next + rank);
                    const TreeRoot root = roots[ray_scene[rid]];
                    nodes = root.nodes;
                    tris = root.tris;
                    const float4* rp = reinterpret_cast<const float4*>(rays + rid);
                    const float4 r0 = ld_hint(rp, pol_stream), r1 = ld_hint(rp + 1, pol_stream);
                    st.ox = r0.x;
                    st.oy = r0.y;
                    st.oz = r0.z;
                    st.tmin = r0.w;
                    st.dx = r1.x;
                    st.dy = r1.y;
                    st.dz = r1.z;
                    st.tmax = r1.w;
                    st.idx = safe_rcp(st.dx);
                    st.idy = safe_rcp(st.dy);
                    st.idz = safe_rcp(st.dz);
                    st.oix = st.ox * st.idx;
                    st.oiy = st.oy * st.idy;
                    st.oiz = st.oz * st.idz;
                    st.tbest = range_far(st.tmax);
                    st.best = -1;
                    st.sp = 0;
                    const bool finite = isfinite(r0.x) && isfinite(r0.y) && isfinite(r0.z) && isfinite(r1.x) &&
                                        isfinite(r1.y) && isfinite(r1.z) && !isnan(r0.w) && !isnan(r1.w);
                    st.node = finite ? 0 : kNodeNone;
                }
                w_next += min(avail, (uint32_t)__popc(idle));
            }
        }
        // the node and leaf phases of trace_kernel
        bool done = false;
        if (rid >= 0) {
            if (st.node >= 0) {
                visit_node<false, S, BLOCK, false>(nodes, st, stack, pol_tree, status, n_nodes);
                if (st.node == kNodeNone) done = pop_next<false, S, BLOCK>(st, stack);
            } else if (st.node == kNodeNone) {
                done = true;
            }
        }
        const bool at_leaf = rid >= 0 && !done && st.node < 0;
        const uint32_t leafw = __ballot_sync(0xffffffffu, at_leaf);
        if (leafw) {
            const uint32_t desc = __ballot_sync(0xffffffffu, rid >= 0 && !done && st.node >= 0);
            if ((uint32_t)__popc(leafw) >= (uint32_t)LEAF_AT || desc == 0u) {
                if (at_leaf) done = test_leaf<false, false>(tris, st, pol_tree, n_tris) || pop_next<false, S, BLOCK>(st, stack);
            }
        }
        if (done) {
            int prim = st.best;
            float t = st.tbest;
            if (prim >= 0 && !(t > range_near(st.tmin))) prim = -1;
            if (prim < 0) t = INFINITY;
            st_hint(hits + rid, prim, __float_as_int(t), pol_stream);
            rid = -1;
        }
    }
    if (status) atomicOr(status_word, status);
}

}  // namespace liar_gpu
