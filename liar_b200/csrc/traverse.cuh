// traverse.cuh -- sm_100a closest-hit / any-hit traversal of the 4-wide tree (qbvh.h).
//
// Replaces the per-ray Lass traversal behind TriangleMesh::doIntersect / doIsIntersecting
// (src/liar/scenery/triangle_mesh.cpp:291-330) and ObjectTree::doIntersect / doIsIntersecting
// (src/liar/scenery/object_trees.h:110-143).
//
// Organisation (one thread per ray):
//   * persistent warps: a grid of (SM count x resident blocks) blocks whose warps pull batches of
//     32 rays from an atomic counter until the ray array is exhausted;
//   * a node is one 128-byte line read with seven 16-byte read-only loads; the four child boxes
//     are slab-tested with the near/far planes chosen by the ray's direction signs;
//   * hit children are ordered by entry distance; the farther ones are pushed with their entry
//     distance onto a per-thread stack that lives in shared memory (column per thread, so the
//     32 lanes of a warp hit 32 different banks), and popped entries farther than the current
//     closest hit are dropped without touching the node;
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

struct TraceCounters {
    unsigned long long nodes;
    unsigned long long tris;
};

__device__ __forceinline__ float4 ldg4(const F4* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ int4 ldg4i(const I4* p) { return __ldg(reinterpret_cast<const int4*>(p)); }

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

// One ray against the tree. Returns hit prim (-1 on miss) and t. Template:
//   ANY   : any-hit (early exit, tmin < t < tmax) instead of closest-hit
//   S     : stack entries per thread
//   COUNT : collect node-visit / triangle-test counters
template <bool ANY, int S, int BLOCK, bool COUNT>
__device__ __forceinline__ void trace_one(const QNode* __restrict__ nodes, const QTri* __restrict__ tris, float ox, float oy,
                                          float oz, float tmin, float dx, float dy, float dz, float tmax,
                                          int* __restrict__ st_node, float* __restrict__ st_t, int& out_prim,
                                          float& out_t, uint32_t& status, uint32_t& n_nodes, uint32_t& n_tris) {
    const float idx = safe_rcp(dx), idy = safe_rcp(dy), idz = safe_rcp(dz);
    const float ooxx = ox * idx, ooyy = oy * idy, oozz = oz * idz;
    const bool nx = dx < 0.0f, ny = dy < 0.0f, nz = dz < 0.0f;

    // closest hit keeps candidates strictly below range_far(tmax); any hit strictly below tmax
    float tbest = ANY ? tmax : range_far(tmax);
    int best = -1;
    int sp = 0;
    int node = 0;  // root
    const int tid = threadIdx.x;

    while (true) {
        if (node >= 0) {
            // ---- inner node: test four child boxes
            if (COUNT) ++n_nodes;
            const QNode* q = nodes + node;
            const float4 lx = ldg4(&q->lo_x), hx = ldg4(&q->hi_x);
            const float4 ly = ldg4(&q->lo_y), hy = ldg4(&q->hi_y);
            const float4 lz = ldg4(&q->lo_z), hz = ldg4(&q->hi_z);
            const int4 ch = ldg4i(&q->child);
            const float4 nxp = nx ? hx : lx, fxp = nx ? lx : hx;
            const float4 nyp = ny ? hy : ly, fyp = ny ? ly : hy;
            const float4 nzp = nz ? hz : lz, fzp = nz ? lz : hz;
            float tn[4], tf[4];
            tn[0] = max4f(fmaf(nxp.x, idx, -ooxx), fmaf(nyp.x, idy, -ooyy), fmaf(nzp.x, idz, -oozz), tmin);
            tn[1] = max4f(fmaf(nxp.y, idx, -ooxx), fmaf(nyp.y, idy, -ooyy), fmaf(nzp.y, idz, -oozz), tmin);
            tn[2] = max4f(fmaf(nxp.z, idx, -ooxx), fmaf(nyp.z, idy, -ooyy), fmaf(nzp.z, idz, -oozz), tmin);
            tn[3] = max4f(fmaf(nxp.w, idx, -ooxx), fmaf(nyp.w, idy, -ooyy), fmaf(nzp.w, idz, -oozz), tmin);
            tf[0] = min4f(fmaf(fxp.x, idx, -ooxx), fmaf(fyp.x, idy, -ooyy), fmaf(fzp.x, idz, -oozz), tbest);
            tf[1] = min4f(fmaf(fxp.y, idx, -ooxx), fmaf(fyp.y, idy, -ooyy), fmaf(fzp.y, idz, -oozz), tbest);
            tf[2] = min4f(fmaf(fxp.z, idx, -ooxx), fmaf(fyp.z, idy, -ooyy), fmaf(fzp.z, idz, -oozz), tbest);
            tf[3] = min4f(fmaf(fxp.w, idx, -ooxx), fmaf(fyp.w, idy, -ooyy), fmaf(fzp.w, idz, -oozz), tbest);
            // sortable keys: entry distance bits (tn >= tmin >= 0 for valid rays) with the slot
            // in the two low bits; misses become 0xffffffff
            uint32_t key[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const bool h = tn[c] <= tf[c];
                key[c] = h ? ((__float_as_uint(fmaxf(tn[c], 0.0f)) & ~3u) | (uint32_t)c) : 0xffffffffu;
            }
            if (!ANY) {
                cswap(key[0], key[1]);
                cswap(key[2], key[3]);
                cswap(key[0], key[2]);
                cswap(key[1], key[3]);
                cswap(key[1], key[2]);
            }
            if (key[0] == 0xffffffffu && key[1] == 0xffffffffu && key[2] == 0xffffffffu && key[3] == 0xffffffffu) {
                node = -1;  // nothing hit: pop below
            } else {
                // the nearest valid key is the smallest; for ANY the order does not matter,
                // so take the first valid one
                int first = 0;
                if (ANY) first = key[0] != 0xffffffffu ? 0 : key[1] != 0xffffffffu ? 1 : key[2] != 0xffffffffu ? 2 : 3;
                // push the others, farthest first
#pragma unroll
                for (int c = 3; c >= 0; --c) {
                    if (c == first || key[c] == 0xffffffffu) continue;
                    const uint32_t slot = key[c] & 3u;
                    if (sp >= S) {
                        status |= STATUS_STACK_OVERFLOW;
                        continue;
                    }
                    st_node[sp * BLOCK + tid] = sel4i(ch, slot);
                    st_t[sp * BLOCK + tid] = sel4f(tn[0], tn[1], tn[2], tn[3], slot);
                    ++sp;
                }
                const uint32_t kf = first == 0 ? key[0] : first == 1 ? key[1] : first == 2 ? key[2] : key[3];
                node = sel4i(ch, kf & 3u);  // a leaf is handled at the next loop turn
                continue;
            }
        } else if (node != -1) {
            // ---- leaf: packed 0x80000000 | count << 27 | first
            const uint32_t packed = (uint32_t)node;
            const uint32_t count = (packed >> 27) & 15u;
            const uint32_t first = packed & 0x07ffffffu;
            for (uint32_t k = 0; k < count; ++k) {
                if (COUNT) ++n_tris;
                const QTri* tp = tris + first + k;
                const float4 a = ldg4(&tp->v0), e1 = ldg4(&tp->e1), e2 = ldg4(&tp->e2);
                float t, u, v;
                if (tri_intersect_exact(ox, oy, oz, dx, dy, dz, a.x, a.y, a.z, e1.x, e1.y, e1.z, e2.x, e2.y, e2.z, t, u,
                                        v)) {
                    const int prim = __float_as_int(a.w);
                    if (ANY) {
                        if (t > tmin && t < tmax) {
                            out_prim = prim;
                            out_t = t;
                            return;
                        }
                    } else if (t > tmin && (t < tbest || (t == tbest && prim < best))) {
                        tbest = t;
                        best = prim;
                    }
                }
            }
        }
        // ---- pop the next entry that can still contain a closer hit
        bool found = false;
        while (sp > 0) {
            --sp;
            const float te = st_t[sp * BLOCK + tid];
            if (ANY || te <= tbest) {
                node = st_node[sp * BLOCK + tid];
                found = true;
                break;
            }
        }
        if (!found) break;
    }
    if (!ANY && best >= 0 && !(tbest > range_near(tmin))) best = -1;  // BoundedRay::inRange near side
    out_prim = best;
    out_t = best >= 0 ? tbest : INFINITY;
    if (ANY) {
        out_prim = -1;
        out_t = INFINITY;
    }
}

template <bool ANY, int S, int BLOCK, bool COUNT>
__global__ void __launch_bounds__(BLOCK) trace_kernel(const QNode* __restrict__ nodes, const QTri* __restrict__ tris,
                                                      const liar_ray* __restrict__ rays, liar_hit* __restrict__ hits,
                                                      uint32_t n_rays, uint32_t* __restrict__ work_counter,
                                                      uint32_t* __restrict__ status_word,
                                                      TraceCounters* __restrict__ counters) {
    extern __shared__ int trace_smem[];  // S * BLOCK node entries, then S * BLOCK distances
    int* st_node = trace_smem;
    float* st_t = reinterpret_cast<float*>(trace_smem + S * BLOCK);
    const int lane = threadIdx.x & 31;
    uint32_t status = 0, n_nodes = 0, n_tris = 0;
    while (true) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(work_counter, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n_rays) break;
        const uint32_t i = base + (uint32_t)lane;
        if (i < n_rays) {
            const float4* rp = reinterpret_cast<const float4*>(rays + i);
            const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
            int prim = -1;
            float t = INFINITY;
            const bool finite = isfinite(r0.x) && isfinite(r0.y) && isfinite(r0.z) && isfinite(r1.x) &&
                                isfinite(r1.y) && isfinite(r1.z) && !isnan(r0.w) && !isnan(r1.w);
            if (finite)
                trace_one<ANY, S, BLOCK, COUNT>(nodes, tris, r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, st_node,
                                                st_t, prim, t, status, n_nodes, n_tris);
            reinterpret_cast<int2*>(hits)[i] = make_int2(prim, __float_as_int(t));
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

}  // namespace liar_gpu
