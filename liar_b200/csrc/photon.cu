// photon.cu -- photon-map build and k-nearest gather on sm_100a.
//
// Replaces the Lass KdTree<Photon> that PhotonMapper::buildPhotonMap resets
// (src/liar/tracers/photon_mapper.cpp:798-835, photon_mapper.h:153) and its rangeSearch(point,
// maxRadius, maxCount) calls (photon_mapper.cpp:1097, 1257, 1312, 1352): the up to k photons
// nearest to a point, all closer than r_max, the farthest first in the reference's heap.
//
// Build (spatial hashing, Teschner et al. 2003): a bounding-box reduction fixes the grid origin;
// the cell width follows the photons' density (map_build_impl: about 60 photons per cell on
// surfaces, 4 in volumes, between r_max and r_max / 8), cell = floor((p - origin) / cell_size),
// bucket = hash(cell) mod 2^m; a counting sort (histogram, exclusive scan, scatter) orders the photons by
// bucket into float4 (x, y, z, original index) records, each with its packed cell key beside it.
// Gather: one warp per query visits the cells around the query in rings of growing Chebyshev
// distance R and stops after ring R as soon as the current k-th distance is at most R cell
// widths (every photon of a later ring is farther than that), or R cell widths reach r_max --
// the grid form of the kd-tree search that shrinks its radius as it finds neighbours. Candidates
// are filtered by their cell key, so buckets shared by colliding cells never yield a photon twice.
// The k = 64 nearest are a sorted list of 64-bit keys (d^2 bits << 32 | photon index), two per
// lane; a batch of 32 candidates is sorted by a shuffle bitonic network and merged in with
// half-cleaners, batches with no key below the current k-th are skipped.
// Distances use explicitly rounded IEEE operations in a fixed order, so every (query, photon) key
// and therefore the neighbour set, ties included (equal d^2: lower index first), equals the CPU
// restatement's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/liar_gpu.h"
#include "ctx.h"

using namespace liar_gpu;

struct liar_gpu_photon_map {
    int device = -1;
    size_t n = 0;
    float r_max = 0.0f, cell = 0.0f;
    float origin[3] = {0, 0, 0};
    float extent = 0.0f;
    uint32_t bucket_bits = 0;
    float4* sorted = nullptr;          // bucket order: x, y, z, original index bits
    uint64_t* cell_key = nullptr;      // packed cell of each sorted photon
    uint32_t* bucket_start = nullptr;  // 2^bits + 1
    void* scratch = nullptr;           // build scratch (bucket keys, counts, bounds), kept for rebuilds
    size_t scratch_bytes = 0;
    size_t cap_n = 0, cap_buckets = 0; // capacities of sorted / cell_key and of bucket_start
};

namespace {

constexpr int kGatherK = 64;
constexpr float kRefine = 4.0f;              // cells per r_max
constexpr int kCellBits = 21;                // per axis in the packed cell key
constexpr int kCellLimit = (1 << kCellBits) - 2;
constexpr uint32_t kStatusBadBucket = 1u << 4;  // device status bit of the photon kernels

__host__ __device__ __forceinline__ uint32_t bucket_of(int ix, int iy, int iz, uint32_t mask) {
    const uint32_t h = ((uint32_t)ix * 73856093u) ^ ((uint32_t)iy * 19349663u) ^ ((uint32_t)iz * 83492791u);
    return h & mask;
}
__host__ __device__ __forceinline__ uint64_t pack_cell(int ix, int iy, int iz) {
    return ((uint64_t)(uint32_t)ix << (2 * kCellBits)) | ((uint64_t)(uint32_t)iy << kCellBits) | (uint64_t)(uint32_t)iz;
}
__device__ __forceinline__ int cell_coord(float p, float o, float inv) { return (int)floorf((p - o) * inv); }

// squared distance with fixed IEEE roundings (the CPU restatement performs the same operations)
__device__ __forceinline__ float dist2_exact(float px, float py, float pz, float qx, float qy, float qz) {
    const float dx = __fsub_rn(px, qx), dy = __fsub_rn(py, qy), dz = __fsub_rn(pz, qz);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

struct BuildParams {
    float ox, oy, oz, inv;
    uint32_t mask;
};

// ---- bounding box (min x, y, z then max x, y, z as order-preserving integer keys)
__device__ __forceinline__ uint32_t fkey(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __forceinline__ float fkey_inv(uint32_t k) {
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
__global__ void k_bounds(const float* __restrict__ pos, uint32_t n, uint32_t* __restrict__ bounds) {
    uint32_t lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const uint32_t k = fkey(pos[3 * i + a]);
            lo[a] = min(lo[a], k);
            hi[a] = max(hi[a], k);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    if ((threadIdx.x & 31u) == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            atomicMin(bounds + a, lo[a]);
            atomicMax(bounds + 3 + a, hi[a]);
        }
    }
}

__global__ void k_bucket_count(const float* __restrict__ pos, uint32_t n, BuildParams P, uint32_t* __restrict__ keys,
                               uint32_t* __restrict__ counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    const uint32_t b = bucket_of(cell_coord(x, P.ox, P.inv), cell_coord(y, P.oy, P.inv), cell_coord(z, P.oz, P.inv), P.mask);
    keys[i] = b;
    atomicAdd(counts + b, 1u);
}

// sum over buckets of count^2 (the photon-weighted bucket occupancy times n)
__global__ void k_sumsq(const uint32_t* __restrict__ counts, uint32_t nb, unsigned long long* __restrict__ out) {
    unsigned long long s = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
        const unsigned long long c = counts[i];
        s += c * c;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31u) == 0 && s) atomicAdd(out, s);
}

// exclusive scan of `counts` (n_buckets + 1 entries written to `start`), one block per 1024 x 4 entries
constexpr int kScanBlock = 1024;
constexpr int kScanItems = 4;

__global__ void k_scan_local(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ out,
                             uint32_t* __restrict__ block_sums) {
    __shared__ uint32_t warp_sums[32];
    const uint32_t base = blockIdx.x * kScanBlock * kScanItems + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0u;
        s += v[k];
    }
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (kScanBlock / 32) ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (uint32_t)o) w += t;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t run = incl - s + (warp > 0 ? warp_sums[warp - 1] : 0u);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == kScanBlock - 1) block_sums[blockIdx.x] = run;
}

__global__ void k_scan_add(uint32_t* __restrict__ out, uint32_t n, const uint32_t* __restrict__ block_offsets) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += block_offsets[i / (kScanBlock * kScanItems)];
}

// ---- spatial order of gather queries: a counting sort by the Morton code of a 64^3 grid over the
// map, so that the warps running at the same time gather from overlapping cells
constexpr int kOrderBits = 6;
constexpr uint32_t kOrderCells = 1u << (3 * kOrderBits);

__device__ __forceinline__ uint32_t spread3(uint32_t v) {  // bit k of v to bit 3k
    uint32_t r = 0;
#pragma unroll
    for (int k = 0; k < kOrderBits; ++k) r |= ((v >> k) & 1u) << (3 * k);
    return r;
}

__device__ __forceinline__ uint32_t order_key(float x, float y, float z, float ox, float oy, float oz, float inv) {
    const float c[3] = {(x - ox) * inv, (y - oy) * inv, (z - oz) * inv};
    uint32_t k = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float f = fminf(fmaxf(c[a], 0.0f), (float)((1 << kOrderBits) - 1));  // NaN -> 0
        k |= spread3((uint32_t)f) << a;
    }
    return k;
}

__global__ void k_order_count(const float* __restrict__ q, uint32_t n, float ox, float oy, float oz, float inv,
                              uint32_t* __restrict__ keys, uint32_t* __restrict__ counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = order_key(q[3 * i], q[3 * i + 1], q[3 * i + 2], ox, oy, oz, inv);
    keys[i] = k;
    atomicAdd(counts + k, 1u);
}

__global__ void k_order_scatter(const float* __restrict__ q, uint32_t n, const uint32_t* __restrict__ keys,
                                uint32_t* __restrict__ cursor, float4* __restrict__ ordered, uint32_t* __restrict__ status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t slot = atomicAdd(cursor + keys[i], 1u);
    if (slot >= n) {  // cannot happen with consistent counts: record, write nothing
        atomicOr(status, kStatusBadBucket);
        return;
    }
    ordered[slot] = make_float4(q[3 * i], q[3 * i + 1], q[3 * i + 2], __uint_as_float(i));
}

__global__ void k_scatter(const float* __restrict__ pos, uint32_t n, BuildParams P, const uint32_t* __restrict__ keys,
                          uint32_t* __restrict__ cursor, float4* __restrict__ sorted, uint64_t* __restrict__ cell_key,
                          uint32_t* __restrict__ status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t slot = atomicAdd(cursor + keys[i], 1u);
    if (slot >= n) {  // a bucket range past the photon array: record it, write nothing
        atomicOr(status, kStatusBadBucket);
        return;
    }
    const float x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    sorted[slot] = make_float4(x, y, z, __uint_as_float(i));
    cell_key[slot] = pack_cell(cell_coord(x, P.ox, P.inv), cell_coord(y, P.oy, P.inv), cell_coord(z, P.oz, P.inv));
}

// bit 31 of a bucket's start marks a bucket that holds photons of more than one cell (hash
// collisions): the photons of a bucket are contiguous, so two neighbours in the same bucket with
// different cell keys mark it; the gather checks the cell keys of such buckets photon by photon
// and those of the other buckets once
constexpr uint32_t kBucketMixed = 0x80000000u;
__device__ __forceinline__ uint32_t bucket_of_key(uint64_t k, uint32_t mask) {
    const uint32_t m = (1u << kCellBits) - 1u;
    return bucket_of((int)(uint32_t)(k >> (2 * kCellBits)), (int)((uint32_t)(k >> kCellBits) & m), (int)((uint32_t)k & m), mask);
}
__global__ void k_mark_mixed(const uint64_t* __restrict__ cell_key, uint32_t n, uint32_t mask, uint32_t* __restrict__ start) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 || i >= n) return;
    const uint64_t a = cell_key[i - 1], b = cell_key[i];
    if (a == b) return;
    const uint32_t ba = bucket_of_key(a, mask), bb = bucket_of_key(b, mask);
    if (ba == bb) atomicOr(start + bb, kBucketMixed);
}

// ---- warp sorting helpers on 64-bit keys
__device__ __forceinline__ uint64_t shfl_xor64(uint64_t v, int m) {
    return __shfl_xor_sync(0xffffffffu, (unsigned long long)v, m);
}
// compare-exchange of lanes l and l^j; ascending where `up` holds for the pair's lower lane
__device__ __forceinline__ uint64_t cmpx(uint64_t v, int j, bool up) {
    const uint64_t o = shfl_xor64(v, j);
    const bool lower = ((threadIdx.x & 31u) & (uint32_t)j) == 0u;
    const bool take_min = lower == up;
    return take_min ? (v < o ? v : o) : (v > o ? v : o);
}
// the same on 32-bit keys
__device__ __forceinline__ uint32_t warp_sort32u(uint32_t v) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const uint32_t o = __shfl_xor_sync(0xffffffffu, v, j);
            const bool lower = (lane & (uint32_t)j) == 0u;
            const bool take_min = lower == ((lane & (uint32_t)k) == 0u);
            v = take_min ? min(v, o) : max(v, o);
        }
    }
    return v;
}

// full ascending bitonic sort of one key per lane
__device__ __forceinline__ uint64_t warp_sort32(uint64_t v) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) v = cmpx(v, j, (lane & (uint32_t)k) == 0u);
    }
    return v;
}
// sorts a bitonic sequence of one key per lane ascending
__device__ __forceinline__ uint64_t warp_bitonic_merge32(uint64_t v) {
#pragma unroll
    for (int j = 16; j > 0; j >>= 1) v = cmpx(v, j, true);
    return v;
}
__device__ __forceinline__ uint64_t reverse_lanes(uint64_t v) {
    return __shfl_sync(0xffffffffu, (unsigned long long)v, 31 - (threadIdx.x & 31u));
}

// i / d for 0 <= i < 2^22, 0 < d, through a float reciprocal with one correction step
__device__ __forceinline__ int div_small(int i, int d, float inv_d) {
    int q = (int)(((float)i + 0.5f) * inv_d);
    if (q * d > i) --q;
    else if ((q + 1) * d <= i) ++q;
    return q;
}

// cell i of the shell at Chebyshev distance R >= 1 around a cell ((2R+1)^3 - (2R-1)^3 cells): the
// two z faces, then the square rings of the levels between them
__device__ __forceinline__ void shell_cell(int i, int R, int& dx, int& dy, int& dz) {
    const int side = 2 * R + 1, face = side * side;
    if (i < 2 * face) {
        const int j = i < face ? i : i - face;
        dz = i < face ? -R : R;
        const int y = div_small(j, side, 1.0f / (float)side);
        dy = y - R;
        dx = j - y * side - R;
    } else {
        const int per = 8 * R, i2 = i - 2 * face;
        const int level = div_small(i2, per, 1.0f / (float)per);
        dz = level - R + 1;
        const int p = i2 - level * per;
        const int k = div_small(p, 2 * R, 1.0f / (float)(2 * R)), t = p - k * 2 * R;
        dx = k == 0 ? -R + t : k == 1 ? R : k == 2 ? R - t : -R;
        dy = k == 0 ? -R : k == 1 ? -R + t : k == 2 ? R : R - t;
    }
}

// inserts key x into the ascending 64-list (lo: slots 0..31, hi: 32..63, one of each per lane),
// dropping the largest; every lane takes part (the branches are warp-uniform)
constexpr int kInsertMax = 8;  // batches with more keys below the k-th take the bitonic merge
__device__ __forceinline__ void insert_key(uint64_t x, uint64_t& lo, uint64_t& hi) {
    const uint32_t lane = threadIdx.x & 31u;
    const int p = __popc(__ballot_sync(0xffffffffu, lo < x));  // lo is ascending: the entries below x lead
    const uint64_t lo_up = __shfl_up_sync(0xffffffffu, (unsigned long long)lo, 1);
    const uint64_t lo_last = __shfl_sync(0xffffffffu, (unsigned long long)lo, 31);
    const uint64_t hi_up = __shfl_up_sync(0xffffffffu, (unsigned long long)hi, 1);
    if (p < 32) {
        // x at slot p; lo[31] becomes hi[0]; hi moves up one slot
        lo = (int)lane < p ? lo : ((int)lane == p ? x : lo_up);
        hi = lane == 0 ? lo_last : hi_up;
    } else {
        const int q = __popc(__ballot_sync(0xffffffffu, hi < x));
        if (q < 32) hi = (int)lane < q ? hi : ((int)lane == q ? x : hi_up);
    }
}

struct GatherParams {
    BuildParams B;
    float r2max;
    float cell;
    float slack;      // cell-assignment round-off allowance in the ring stopping rule
    int max_ring;
    uint32_t n_photons;
};

__global__ void __launch_bounds__(256) k_gather(const float4* __restrict__ sorted, const uint64_t* __restrict__ cell_key,
                                                const uint32_t* __restrict__ start, GatherParams G,
                                                const float* __restrict__ queries, uint32_t nq, int k_out,
                                                int32_t* __restrict__ out_idx, float* __restrict__ out_d2,
                                                int32_t* __restrict__ out_count, uint32_t* __restrict__ status,
                                                const float4* __restrict__ ordered) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
    constexpr uint64_t INF = ~0ull;
    const BuildParams& P = G.B;
    for (uint32_t w = warp_global; w < nq; w += n_warps) {
        // ordered: the queries in spatial order, each with its own index in w (results go there)
        uint32_t q = w;
        float qx, qy, qz;
        if (ordered) {
            const float4 o = ordered[w];
            qx = o.x;
            qy = o.y;
            qz = o.z;
            q = __float_as_uint(o.w);
            if (q >= nq) {  // a slot the reorder pass did not fill: record it, write nothing
                if (lane == 0) atomicOr(status, kStatusBadBucket);
                continue;
            }
        } else {
            qx = queries[3 * q];
            qy = queries[3 * q + 1];
            qz = queries[3 * q + 2];
        }
        const int cx = cell_coord(qx, P.ox, P.inv), cy = cell_coord(qy, P.oy, P.inv), cz = cell_coord(qz, P.oz, P.inv);
        // the k nearest so far, ascending: slot `lane` in lo, slot `32 + lane` in hi
        uint64_t lo = INF, hi = INF;
        uint64_t kth = INF;  // key of the current k-th (64th) nearest
        for (int R = 0; R <= G.max_ring; ++R) {
            // the cells at Chebyshev distance R, 32 at a time (lane: one cell)
            const int shell = R == 0 ? 1 : (2 * R + 1) * (2 * R + 1) * (2 * R + 1) - (2 * R - 1) * (2 * R - 1) * (2 * R - 1);
            for (int c0 = 0; c0 < shell; c0 += 32) {
                const int c = c0 + (int)lane;
                int dx = 0, dy = 0, dz = 0;
                bool mine = c < shell;
                if (mine && R > 0) shell_cell(c, R, dx, dy, dz);
                int ix = cx + dx, iy = cy + dy, iz = cz + dz;
                mine = mine && ix >= 0 && iy >= 0 && iz >= 0 && ix <= kCellLimit && iy <= kCellLimit && iz <= kCellLimit;
                float cell_d2 = 0.0f;  // after the sort: lane j's cell's distance bound (ascending in j)
                if (R > 0) {
                    // the query's distance to the cell's box, less the cell-assignment round-off: a
                    // cell farther than the current k-th (or r_max) cannot contribute and is skipped;
                    // the others are taken nearest first, so that the k-th falls early and later
                    // candidates fail the batch test instead of entering the list
                    float md2 = 0.0f;
                    if (mine) {
                        const float bx = P.ox + (float)ix * G.cell, by = P.oy + (float)iy * G.cell, bz = P.oz + (float)iz * G.cell;
                        const float ex = fmaxf(fmaxf(bx - qx, qx - (bx + G.cell)), 0.0f);
                        const float ey = fmaxf(fmaxf(by - qy, qy - (by + G.cell)), 0.0f);
                        const float ez = fmaxf(fmaxf(bz - qz, qz - (bz + G.cell)), 0.0f);
                        const float md = fmaxf(sqrtf(ex * ex + ey * ey + ez * ez) - G.slack, 0.0f);
                        md2 = md * md;
                        const float bound = kth != INF ? fminf(__uint_as_float((uint32_t)(kth >> 32)), G.r2max) : G.r2max;
                        mine = md2 <= bound;
                    }
                    const uint32_t live = __ballot_sync(0xffffffffu, mine);
                    if (live == 0u) continue;  // nothing in this chunk can come within the k-th
                    if (live & (live - 1u)) {
                        // 32-bit sort keys: the bound with its 5 low bits cleared (a lower bound
                        // still, so that the order stays ascending in the bound the batches test)
                        // and the lane in those bits
                        const uint32_t ck = warp_sort32u(mine ? ((__float_as_uint(md2) & ~31u) | lane) : 0xffffffffu);
                        const int src = (int)(ck & 31u);
                        mine = ck != 0xffffffffu;
                        cell_d2 = __uint_as_float(ck & ~31u);
                        ix = __shfl_sync(0xffffffffu, ix, src);
                        iy = __shfl_sync(0xffffffffu, iy, src);
                        iz = __shfl_sync(0xffffffffu, iz, src);
                    } else {
                        // one cell: lane 0 takes it
                        const int src = __ffs(live) - 1;
                        cell_d2 = __uint_as_float(__float_as_uint(__shfl_sync(0xffffffffu, md2, src)) & ~31u);
                        ix = __shfl_sync(0xffffffffu, ix, src);
                        iy = __shfl_sync(0xffffffffu, iy, src);
                        iz = __shfl_sync(0xffffffffu, iz, src);
                        mine = lane == 0;
                    }
                }
                uint32_t s0 = 0, s1 = 0;
                uint64_t my_key = pack_cell(ix, iy, iz);
                if (mine) {
                    const uint32_t b = bucket_of(ix, iy, iz, P.mask);
                    const uint32_t r0 = __ldg(start + b);
                    s0 = r0 & ~kBucketMixed;
                    s1 = __ldg(start + b + 1) & ~kBucketMixed;
                    if (s0 > s1 || s1 > G.n_photons) {  // corrupt bucket range: record it, skip the cell
                        atomicOr(status, kStatusBadBucket);
                        s0 = s1 = 0;
                    }
                    if (s1 > s0 && !(r0 & kBucketMixed)) {
                        // a single-cell bucket: its first key tells whether it is this cell's
                        if (__ldg(reinterpret_cast<const unsigned long long*>(cell_key) + s0) != my_key) s1 = s0;
                        else my_key |= 1ull << 63;  // every photon of the range belongs to the cell
                    }
                }
                // the chunk's photons as one list: lane j's cell owns items [excl_j, excl_j + cnt_j)
                // of it, so that a batch of 32 candidates spans as many cells as it takes (cells
                // hold a photon or two on average; one batch per cell would leave most lanes idle)
                // (64-bit counts: 32 colliding cells of one huge bucket must not wrap)
                const uint64_t cnt = s1 - s0;
                uint64_t incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint64_t t = __shfl_up_sync(0xffffffffu, (unsigned long long)incl, o);
                    if ((int)lane >= o) incl += t;
                }
                const uint64_t total = __shfl_sync(0xffffffffu, (unsigned long long)incl, 31);
                const uint64_t excl = incl - cnt;
                for (uint64_t base = 0; base < total; base += 32) {
                    const uint64_t item = base + lane;
                    // the owning cell: the last lane whose list starts at or before the item
                    // (every lane runs the same shuffles)
                    uint32_t owner = 0;
#pragma unroll
                    for (uint32_t step = 16; step > 0; step >>= 1) {
                        const uint64_t e = __shfl_sync(0xffffffffu, (unsigned long long)excl, (int)(owner + step));
                        if (e <= item) owner += step;
                    }
                    // the cells are in ascending distance order: once the batch's first cell lies
                    // beyond the current k-th, so do all that follow
                    if (R > 0 && kth != INF) {
                        const float first_d2 = __shfl_sync(0xffffffffu, cell_d2, (int)__shfl_sync(0xffffffffu, owner, 0));
                        if (first_d2 > __uint_as_float((uint32_t)(kth >> 32))) break;
                    }
                    const uint32_t o_s0 = __shfl_sync(0xffffffffu, s0, (int)owner);
                    const uint64_t o_excl = __shfl_sync(0xffffffffu, (unsigned long long)excl, (int)owner);
                    const uint64_t target = __shfl_sync(0xffffffffu, (unsigned long long)my_key, (int)owner);
                    uint64_t key = INF;
                    if (item < total) {
                        const uint32_t i = o_s0 + (uint32_t)(item - o_excl);
                        const float4 p = __ldg(sorted + i);
                        const bool in_cell = (target >> 63) != 0ull ||
                                             __ldg(reinterpret_cast<const unsigned long long*>(cell_key) + i) == target;
                        if (in_cell) {
                            const float d2 = dist2_exact(p.x, p.y, p.z, qx, qy, qz);
                            if (d2 < G.r2max) key = ((uint64_t)__float_as_uint(d2) << 32) | (uint64_t)__float_as_uint(p.w);
                        }
                    }
                    const uint32_t better = __ballot_sync(0xffffffffu, key < kth);
                    if (better == 0u) continue;
                    if (__popc(better) <= kInsertMax) {
                        // a few keys below the k-th: insert them one at a time
                        uint32_t m = better;
                        while (m) {
                            const int src = __ffs(m) - 1;
                            m &= m - 1;
                            insert_key(__shfl_sync(0xffffffffu, (unsigned long long)key, src), lo, hi);
                        }
                        kth = __shfl_sync(0xffffffffu, (unsigned long long)hi, 31);
                        continue;
                    }
                    const uint64_t bsort = warp_sort32(key);
                    // smallest 32 of hi and the batch: half-cleaner against the reversed batch
                    // (every shuffle is executed by all 32 lanes, outside lane-dependent branches)
                    const uint64_t brev = reverse_lanes(bsort);
                    uint64_t m = hi < brev ? hi : brev;
                    m = warp_bitonic_merge32(m);
                    // lo (sorted) and m (sorted): split into the lower and upper 32
                    const uint64_t mr = reverse_lanes(m);
                    const uint64_t nlo = lo < mr ? lo : mr;
                    const uint64_t nhi = lo < mr ? mr : lo;
                    lo = warp_bitonic_merge32(nlo);
                    hi = warp_bitonic_merge32(nhi);
                    kth = __shfl_sync(0xffffffffu, (unsigned long long)hi, 31);
                }
            }
            // every photon outside rings 0..R is farther than R cells (minus round-off)
            const float reach = fmaxf((float)R * G.cell - G.slack, 0.0f);
            const uint64_t kk = __shfl_sync(0xffffffffu, (unsigned long long)(k_out > 32 ? hi : lo), (k_out - 1) & 31);
            if (kk != INF && __uint_as_float((uint32_t)(kk >> 32)) <= reach * reach) break;
            if (reach * reach >= G.r2max) break;
        }
        // write the first k_out entries (k_out <= 64) in ascending order
        const uint32_t cnt_lo = __popc(__ballot_sync(0xffffffffu, lo != INF));
        const uint32_t cnt_hi = __popc(__ballot_sync(0xffffffffu, hi != INF));
        const int count = min((int)(cnt_lo + cnt_hi), k_out);
        int32_t* oi = out_idx + (size_t)q * k_out;
        float* od = out_d2 + (size_t)q * k_out;
        if ((int)lane < k_out) {
            oi[lane] = lo != INF ? (int32_t)(uint32_t)lo : -1;
            od[lane] = lo != INF ? __uint_as_float((uint32_t)(lo >> 32)) : INFINITY;
        }
        if ((int)(32 + lane) < k_out) {
            oi[32 + lane] = hi != INF ? (int32_t)(uint32_t)hi : -1;
            od[32 + lane] = hi != INF ? __uint_as_float((uint32_t)(hi >> 32)) : INFINITY;
        }
        if (lane == 0 && out_count) out_count[q] = count;
    }
}

// PhotonMapper::estimateIrradianceImpl (photon_mapper.cpp:1254-1279): sum of the powers of the
// neighbours arriving from the normal's side, over pi r^2 with r the farthest neighbour's distance
__global__ void k_estimate(const float* __restrict__ power, const float* __restrict__ omega_in,
                           const float* __restrict__ normals, uint32_t nq, int k, const int32_t* __restrict__ idx,
                           const float* __restrict__ d2, const int32_t* __restrict__ count, float power_scale,
                           uint32_t n_photons, float* __restrict__ out, uint32_t* __restrict__ status) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const int c = count[q];
    float x = 0.0f, y = 0.0f, z = 0.0f;
    if (c > 0) {
        const float nx = normals[3 * q], ny = normals[3 * q + 1], nz = normals[3 * q + 2];
        for (int j = 0; j < c && j < k; ++j) {
            const int32_t i = idx[(size_t)q * k + j];
            if (i < 0 || (uint32_t)i >= n_photons) {
                atomicOr(status, kStatusBadBucket);
                continue;
            }
            if (omega_in[3 * i] * nx + omega_in[3 * i + 1] * ny + omega_in[3 * i + 2] * nz > 0.0f) {
                x += power[3 * i];
                y += power[3 * i + 1];
                z += power[3 * i + 2];
            }
        }
        const float r2 = d2[(size_t)q * k + (c < k ? c : k) - 1];
        const float s = r2 > 0.0f ? power_scale / (3.14159265358979323846f * r2) : 0.0f;
        x *= s;
        y *= s;
        z *= s;
    }
    out[3 * q] = x;
    out[3 * q + 1] = y;
    out[3 * q + 2] = z;
}

int map_build_impl(liar_gpu_ctx* ctx, liar_gpu_photon_map* m, const float* d_pos, size_t n, cudaStream_t st) {
    // buckets: the next power of two >= 2n, at most 2^23 (the two-level scan covers 2^24 entries)
    uint32_t bits = 10;
    while (bits < 23 && (1ull << bits) < 2ull * n) ++bits;
    m->bucket_bits = bits;
    const size_t nb = (size_t)1 << bits;
    const size_t scan_blocks = (nb + 1 + kScanBlock * kScanItems - 1) / (kScanBlock * kScanItems);
    const size_t need = n * 4 + 2 * (((nb + 1) * 4 + 255) / 256) * 256 + (scan_blocks + 1) * 8 + 4096;
    if (m->scratch_bytes < need) {
        if (m->scratch) cudaFree(m->scratch);
        m->scratch = nullptr;
        m->scratch_bytes = 0;
        cudaError_t e = cudaMalloc(&m->scratch, need);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return ctx_cuda(ctx, e, "photon map build scratch");
        }
        m->scratch_bytes = need;
    }
    cudaError_t e = cudaSuccess;
    if (m->cap_n < std::max<size_t>(n, 1)) {
        // photons beyond the buffers' capacity (a first build, or a rebuild with more photons)
        if (m->sorted) cudaFree(m->sorted);
        if (m->cell_key) cudaFree(m->cell_key);
        m->sorted = nullptr;
        m->cell_key = nullptr;
        m->cap_n = 0;
        e = cudaMalloc((void**)&m->sorted, std::max<size_t>(n, 1) * sizeof(float4));
        if (e == cudaSuccess) e = cudaMalloc((void**)&m->cell_key, std::max<size_t>(n, 1) * sizeof(uint64_t));
        if (e == cudaSuccess) m->cap_n = std::max<size_t>(n, 1);
    }
    if (e == cudaSuccess && m->cap_buckets < nb + 1) {
        if (m->bucket_start) cudaFree(m->bucket_start);
        m->bucket_start = nullptr;
        m->cap_buckets = 0;
        e = cudaMalloc((void**)&m->bucket_start, (nb + 1) * sizeof(uint32_t));
        if (e == cudaSuccess) m->cap_buckets = nb + 1;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_cuda(ctx, e, "photon map");
    }
    char* p = static_cast<char*>(m->scratch);
    uint32_t* keys = reinterpret_cast<uint32_t*>(p);
    p += ((n * 4 + 255) / 256) * 256;
    uint32_t* counts = reinterpret_cast<uint32_t*>(p);
    p += (((nb + 1) * 4 + 255) / 256) * 256;
    uint32_t* cursor = reinterpret_cast<uint32_t*>(p);
    p += (((nb + 1) * 4 + 255) / 256) * 256;
    uint32_t* bounds = reinterpret_cast<uint32_t*>(p);
    p += 256;
    uint32_t* block_sums = reinterpret_cast<uint32_t*>(p);
    uint32_t* block_offs = block_sums + scan_blocks + 1;
    // grid origin and extent from the photons' bounding box
    m->origin[0] = m->origin[1] = m->origin[2] = 0.0f;
    m->extent = 0.0f;
    m->cell = m->r_max / kRefine;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    // one cell of margin below the lowest photon keeps every cell index positive
    auto set_grid = [&](float cell) -> bool {
        m->cell = cell;
        m->extent = 0.0f;
        for (int a = 0; a < 3; ++a) {
            m->origin[a] = lo[a] - cell;
            m->extent = std::max(m->extent, hi[a] - m->origin[a]);
        }
        return m->extent / cell <= (float)(kCellLimit - 4);
    };
    if (n) {
        const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
        e = cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon bounds");
        const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 4);
        k_bounds<<<blocks, 256, 0, st>>>(d_pos, (uint32_t)n, bounds);
        uint32_t hb[6];
        e = cudaMemcpyAsync(hb, bounds, sizeof(hb), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon bounds");
        for (int a = 0; a < 3; ++a) {
            lo[a] = fkey_inv(hb[a]);
            hi[a] = fkey_inv(hb[3 + a]);
            if (!std::isfinite(lo[a]) || !std::isfinite(hi[a]))
                return ctx_fail(ctx, LIAR_ERR_INVALID, "photon position is not finite");
        }
        // the cell width from the photons' density: the photon-weighted number of other photons
        // sharing a photon's cell, lambda(c) (a bucket's count squared summed over the buckets, over
        // n, less the photon itself and the expected share of colliding cells n / nb), at r_max / 2
        // and r_max / 4 gives the local dimension D = log2(lambda1 / lambda2) (2 for photons on
        // surfaces, 3 in volumes) and the width at which lambda = T(D), 60 on surfaces and 4 in
        // volumes (geometric in between), measured optima of the ring walk's cost: the bucket
        // lookups of the cells visited (queries with fewer than k photons within r_max visit all
        // of them) against the candidates tested; cells r_max / 1 .. r_max / 8
        if (n >= 1024) {
            double lam[2] = {0.0, 0.0};
            unsigned long long* d_sum = reinterpret_cast<unsigned long long*>(bounds + 8);
            for (int t = 0; t < 2 && e == cudaSuccess; ++t) {
                if (!set_grid(m->r_max / (t == 0 ? 2.0f : 4.0f))) break;
                const BuildParams T{m->origin[0], m->origin[1], m->origin[2], 1.0f / m->cell, (uint32_t)(nb - 1)};
                e = cudaMemsetAsync(counts, 0, nb * 4, st);
                if (e == cudaSuccess) e = cudaMemsetAsync(d_sum, 0, 8, st);
                if (e != cudaSuccess) break;
                k_bucket_count<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_pos, (uint32_t)n, T, keys, counts);
                k_sumsq<<<(unsigned)ctx->num_sms * 4, 256, 0, st>>>(counts, (uint32_t)nb, d_sum);
                unsigned long long hs = 0;
                e = cudaMemcpyAsync(&hs, d_sum, 8, cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                lam[t] = (double)hs / (double)n - 1.0 - (double)n / (double)nb;
            }
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon density");
            float refine = kRefine;
            if (lam[0] > 0.0 && lam[1] > 0.0) {
                const double D = std::min(3.0, std::max(1.5, std::log2(lam[0] / lam[1])));
                const double target = 60.0 * std::pow(4.0 / 60.0, D - 2.0);
                refine = (float)std::min(8.0, std::max(1.0, 2.0 * std::pow(lam[0] / target, 1.0 / D)));
            }
            while (!set_grid(m->r_max / refine) && refine > 1.0f) refine = std::max(1.0f, refine * 0.5f);
        }
        if (!set_grid(m->cell))
            return ctx_fail(ctx, LIAR_ERR_UNSUPPORTED, "photons span more than %d grid cells per axis; raise r_max",
                            kCellLimit - 4);
    }
    BuildParams P{m->origin[0], m->origin[1], m->origin[2], 1.0f / m->cell, (uint32_t)(nb - 1)};
    e = cudaMemsetAsync(counts, 0, (nb + 1) * 4, st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon map counts");
    if (n) k_bucket_count<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_pos, (uint32_t)n, P, keys, counts);
    // exclusive scan of counts[0 .. nb] -> bucket_start (start[nb] = n)
    k_scan_local<<<(unsigned)scan_blocks, kScanBlock, 0, st>>>(counts, (uint32_t)(nb + 1), m->bucket_start, block_sums);
    if (scan_blocks > 1) {
        const size_t blocks2 = (scan_blocks + kScanBlock * kScanItems - 1) / (kScanBlock * kScanItems);
        if (blocks2 > 1) return ctx_fail(ctx, LIAR_ERR_UNSUPPORTED, "photon map too large to scan");
        k_scan_local<<<1, kScanBlock, 0, st>>>(block_sums, (uint32_t)scan_blocks, block_offs, block_sums + scan_blocks);
        k_scan_add<<<(unsigned)((nb + 1 + 255) / 256), 256, 0, st>>>(m->bucket_start, (uint32_t)(nb + 1), block_offs);
    }
    e = cudaMemcpyAsync(cursor, m->bucket_start, (nb + 1) * 4, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon map cursor");
    if (n) {
        k_scatter<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_pos, (uint32_t)n, P, keys, cursor, m->sorted,
                                                              m->cell_key, ctx->d_scratch + kStatusWord);
        k_mark_mixed<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(m->cell_key, (uint32_t)n, (uint32_t)(nb - 1), m->bucket_start);
    }
    m->n = n;
    return ctx_cuda(ctx, cudaGetLastError(), "photon map build");
}

}  // namespace

extern "C" int liar_gpu_photon_map_build_device(liar_gpu_ctx* ctx, const float* d_positions, size_t n, float r_max,
                                                liar_gpu_photon_map** out, void* stream) {
    if (!ctx || !out) return LIAR_ERR_INVALID;
    *out = nullptr;
    if (n && !d_positions) return ctx_fail(ctx, LIAR_ERR_INVALID, "null photon positions");
    if (!(r_max > 0.0f) || !std::isfinite(r_max)) return ctx_fail(ctx, LIAR_ERR_INVALID, "r_max must be positive");
    if (n >= (1ull << 31)) return ctx_fail(ctx, LIAR_ERR_INVALID, "too many photons (limit 2^31)");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    liar_gpu_photon_map* m = new (std::nothrow) liar_gpu_photon_map();
    if (!m) return ctx_fail(ctx, LIAR_ERR_OOM, "host allocation");
    m->device = ctx->device;
    m->r_max = r_max;
    m->cell = r_max / kRefine;
    rc = map_build_impl(ctx, m, d_positions, n, stream ? (cudaStream_t)stream : ctx->stream);
    if (rc) {
        liar_gpu_photon_map_destroy(m);
        return rc;
    }
    *out = m;
    return LIAR_OK;
}

extern "C" int liar_gpu_photon_map_rebuild_device(liar_gpu_ctx* ctx, liar_gpu_photon_map* m, const float* d_positions,
                                                  size_t n, float r_max, void* stream) {
    if (!ctx || !m) return LIAR_ERR_INVALID;
    if (n && !d_positions) return ctx_fail(ctx, LIAR_ERR_INVALID, "null photon positions");
    if (!(r_max > 0.0f) || !std::isfinite(r_max)) return ctx_fail(ctx, LIAR_ERR_INVALID, "r_max must be positive");
    if (n >= (1ull << 31)) return ctx_fail(ctx, LIAR_ERR_INVALID, "too many photons (limit 2^31)");
    if (m->device != ctx->device) return ctx_fail(ctx, LIAR_ERR_INVALID, "photon map belongs to another device");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    m->r_max = r_max;
    m->cell = r_max / kRefine;
    return map_build_impl(ctx, m, d_positions, n, stream ? (cudaStream_t)stream : ctx->stream);
}

extern "C" int liar_gpu_photon_map_build(liar_gpu_ctx* ctx, const float* positions, size_t n, float r_max,
                                         liar_gpu_photon_map** out) {
    if (!ctx || !out) return LIAR_ERR_INVALID;
    *out = nullptr;
    if (n && !positions) return ctx_fail(ctx, LIAR_ERR_INVALID, "null photon positions");
    for (size_t i = 0; i < 3 * n; ++i)
        if (!std::isfinite(positions[i])) return ctx_fail(ctx, LIAR_ERR_INVALID, "photon position is not finite");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    float* d = nullptr;
    cudaError_t e = cudaMalloc((void**)&d, std::max<size_t>(n, 1) * 12);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_cuda(ctx, e, "photon upload");
    }
    e = cudaMemcpyAsync(d, positions, n * 12, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) rc = liar_gpu_photon_map_build_device(ctx, d, n, r_max, out, ctx->stream);
    else rc = ctx_cuda(ctx, e, "photon upload");
    if (!rc) rc = ctx_cuda(ctx, cudaStreamSynchronize(ctx->stream), "photon map build");
    cudaFree(d);
    if (rc && *out) {
        liar_gpu_photon_map_destroy(*out);
        *out = nullptr;
    }
    if (!rc) rc = ctx_check_status(ctx);
    return rc;
}

extern "C" void liar_gpu_photon_map_destroy(liar_gpu_photon_map* m) {
    if (!m) return;
    int cur = -1;
    cudaGetDevice(&cur);
    if (m->device >= 0) cudaSetDevice(m->device);
    if (m->sorted) cudaFree(m->sorted);
    if (m->cell_key) cudaFree(m->cell_key);
    if (m->bucket_start) cudaFree(m->bucket_start);
    if (m->scratch) cudaFree(m->scratch);
    if (cur >= 0) cudaSetDevice(cur);
    delete m;
}

namespace {

constexpr size_t kOrderMinQueries = 1u << 15;  // below this the sort costs more than it saves

struct GatherOrder {
    void* mem = nullptr;
    size_t cap = 0;
    // end of the last gather that read the buffer: a gather on another stream waits for it, since
    // the buffer's entries decide where k_gather writes its results
    cudaEvent_t last_use = nullptr;
    bool used = false;
};

// the queries as float4 (x, y, z, own index) in the Morton order of a 64^3 grid over the map
int order_queries(liar_gpu_ctx* ctx, const liar_gpu_photon_map* m, const float* d_q, uint32_t n, cudaStream_t st,
                  const float4** out, GatherOrder** order) {
    GatherOrder* g = nullptr;
    for (auto& ext : ctx->extensions)
        if (ext.first == "gather_order") g = static_cast<GatherOrder*>(ext.second);
    if (!g) {
        g = new GatherOrder();
        ctx->extensions.emplace_back("gather_order", g);
        ctx->on_destroy.push_back([g]() {
            if (g->mem) cudaFree(g->mem);
            if (g->last_use) cudaEventDestroy(g->last_use);
            delete g;
        });
    }
    if (!g->last_use) {
        cudaError_t e = cudaEventCreateWithFlags(&g->last_use, cudaEventDisableTiming);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "gather order event");
    }
    if (g->used) {
        cudaError_t e = cudaStreamWaitEvent(st, g->last_use, 0);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "gather order wait");
    }
    const size_t nb = kOrderCells;
    const size_t scan_blocks = (nb + 1 + kScanBlock * kScanItems - 1) / (kScanBlock * kScanItems);
    const size_t a_ord = ((size_t)n * 16 + 255) / 256 * 256, a_keys = ((size_t)n * 4 + 255) / 256 * 256;
    const size_t a_cnt = ((nb + 1) * 4 + 255) / 256 * 256;
    int rc = ctx_grow(ctx, &g->mem, &g->cap, a_ord + a_keys + 3 * a_cnt + (scan_blocks + 1) * 8 + 256, "gather order");
    if (rc) return rc;
    char* p = static_cast<char*>(g->mem);
    float4* ordered = reinterpret_cast<float4*>(p);
    uint32_t* keys = reinterpret_cast<uint32_t*>(p + a_ord);
    uint32_t* counts = reinterpret_cast<uint32_t*>(p + a_ord + a_keys);
    uint32_t* start = reinterpret_cast<uint32_t*>(p + a_ord + a_keys + a_cnt);
    uint32_t* cursor = reinterpret_cast<uint32_t*>(p + a_ord + a_keys + 2 * a_cnt);
    uint32_t* block_sums = reinterpret_cast<uint32_t*>(p + a_ord + a_keys + 3 * a_cnt);
    uint32_t* block_offs = block_sums + scan_blocks + 1;
    cudaError_t e = cudaMemsetAsync(counts, 0, (nb + 1) * 4, st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "gather order");
    const float inv = (float)(1 << kOrderBits) / std::max(m->extent, 1e-30f);
    const unsigned blocks = (n + 255) / 256;
    k_order_count<<<blocks, 256, 0, st>>>(d_q, n, m->origin[0], m->origin[1], m->origin[2], inv, keys, counts);
    k_scan_local<<<(unsigned)scan_blocks, kScanBlock, 0, st>>>(counts, (uint32_t)(nb + 1), start, block_sums);
    if (scan_blocks > 1) {
        k_scan_local<<<1, kScanBlock, 0, st>>>(block_sums, (uint32_t)scan_blocks, block_offs, block_sums + scan_blocks);
        k_scan_add<<<(unsigned)((nb + 1 + 255) / 256), 256, 0, st>>>(start, (uint32_t)(nb + 1), block_offs);
    }
    e = cudaMemcpyAsync(cursor, start, (nb + 1) * 4, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "gather order");
    k_order_scatter<<<blocks, 256, 0, st>>>(d_q, n, keys, cursor, ordered, ctx->d_scratch + kStatusWord);
    e = cudaGetLastError();
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "gather order");
    *out = ordered;
    *order = g;
    return LIAR_OK;
}

}  // namespace

extern "C" int liar_gpu_photon_gather_device(liar_gpu_ctx* ctx, const liar_gpu_photon_map* m, const float* d_queries,
                                             size_t n_queries, int k, int32_t* d_idx, float* d_d2, int32_t* d_count,
                                             void* stream) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (!m || (n_queries && (!d_queries || !d_idx || !d_d2))) return ctx_fail(ctx, LIAR_ERR_INVALID, "null map or buffer");
    if (k < 1 || k > kGatherK) return ctx_fail(ctx, LIAR_ERR_INVALID, "k must be 1..%d", kGatherK);
    if (m->device != ctx->device) return ctx_fail(ctx, LIAR_ERR_INVALID, "photon map lives on another device");
    if (n_queries >= (1ull << 31)) return ctx_fail(ctx, LIAR_ERR_INVALID, "too many queries");
    if (n_queries == 0) return LIAR_OK;
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    GatherParams G;
    G.B = BuildParams{m->origin[0], m->origin[1], m->origin[2], 1.0f / m->cell,
                      (uint32_t)(((size_t)1 << m->bucket_bits) - 1)};
    G.r2max = m->r_max * m->r_max;
    G.cell = m->cell;
    G.slack = std::max(1e-3f * m->cell, 8.0f * 1.1920929e-07f * std::max(m->extent, 1.0f));
    G.max_ring = (int)std::ceil(m->r_max / m->cell) + 1;
    G.n_photons = (uint32_t)m->n;
    const float4* ordered = nullptr;
    GatherOrder* order = nullptr;
    if (n_queries >= kOrderMinQueries && m->n > 0) {
        rc = order_queries(ctx, m, d_queries, (uint32_t)n_queries, st, &ordered, &order);
        if (rc) return rc;
    }
    const unsigned blocks = (unsigned)std::min<size_t>((n_queries + 7) / 8, (size_t)ctx->num_sms * 8);
    k_gather<<<blocks, 256, 0, st>>>(m->sorted, m->cell_key, m->bucket_start, G, d_queries, (uint32_t)n_queries, k, d_idx,
                                     d_d2, d_count, ctx->d_scratch + kStatusWord, ordered);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && order) {
        e = cudaEventRecord(order->last_use, st);
        order->used = e == cudaSuccess;
    }
    return ctx_cuda(ctx, e, "photon gather launch");
}

extern "C" int liar_gpu_photon_gather(liar_gpu_ctx* ctx, const liar_gpu_photon_map* m, const float* queries,
                                      size_t n_queries, int k, int32_t* idx, float* d2, int32_t* count) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (!m || (n_queries && (!queries || !idx || !d2))) return ctx_fail(ctx, LIAR_ERR_INVALID, "null map or buffer");
    if (k < 1 || k > kGatherK) return ctx_fail(ctx, LIAR_ERR_INVALID, "k must be 1..%d", kGatherK);
    if (n_queries == 0) return LIAR_OK;
    for (size_t i = 0; i < 3 * n_queries; ++i)
        if (!std::isfinite(queries[i])) return ctx_fail(ctx, LIAR_ERR_INVALID, "query position is not finite");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    const size_t qb = n_queries * 12, ob = n_queries * (size_t)k * 4, cb = n_queries * 4;
    char* d = nullptr;
    cudaError_t e = cudaMalloc((void**)&d, qb + 2 * ob + cb + 64);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_cuda(ctx, e, "gather buffers");
    }
    float* dq = reinterpret_cast<float*>(d);
    int32_t* di = reinterpret_cast<int32_t*>(d + qb);
    float* dd = reinterpret_cast<float*>(d + qb + ob);
    int32_t* dc = reinterpret_cast<int32_t*>(d + qb + 2 * ob);
    e = cudaMemcpyAsync(dq, queries, qb, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) rc = liar_gpu_photon_gather_device(ctx, m, dq, n_queries, k, di, dd, dc, ctx->stream);
    else rc = ctx_cuda(ctx, e, "query upload");
    if (!rc) {
        e = cudaMemcpyAsync(idx, di, ob, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d2, dd, ob, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess && count) e = cudaMemcpyAsync(count, dc, cb, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = ctx_cuda(ctx, e, "gather results");
    }
    cudaFree(d);
    if (!rc) rc = ctx_check_status(ctx);
    return rc;
}

extern "C" int liar_gpu_photon_estimate_device(liar_gpu_ctx* ctx, const float* d_power, const float* d_omega_in,
                                               size_t n_photons, const float* d_normals, size_t n_queries, int k,
                                               const int32_t* d_idx, const float* d_d2, const int32_t* d_count,
                                               float power_scale, float* d_out, void* stream) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (n_queries && (!d_power || !d_omega_in || !d_normals || !d_idx || !d_d2 || !d_count || !d_out))
        return ctx_fail(ctx, LIAR_ERR_INVALID, "null buffer");
    if (k < 1 || k > kGatherK) return ctx_fail(ctx, LIAR_ERR_INVALID, "k must be 1..%d", kGatherK);
    if (n_queries >= (1ull << 31) || n_photons >= (1ull << 31)) return ctx_fail(ctx, LIAR_ERR_INVALID, "too many items");
    if (n_queries == 0) return LIAR_OK;
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    k_estimate<<<(unsigned)((n_queries + 255) / 256), 256, 0, st>>>(d_power, d_omega_in, d_normals, (uint32_t)n_queries, k,
                                                                   d_idx, d_d2, d_count, power_scale,
                                                                   (uint32_t)n_photons, d_out,
                                                                   ctx->d_scratch + kStatusWord);
    return ctx_cuda(ctx, cudaGetLastError(), "photon estimate launch");
}
